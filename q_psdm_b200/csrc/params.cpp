// params.cpp -- host-side parameter derivation of the engine.
//
// These are the integer sizes and constants the reference computes on the
// host before any device work; they decide sample and bin indices, so the
// float/double mix of each reference expression is kept exactly.
#include <math.h>
#include <string.h>

#include <algorithm>

#include "qpsdm_engine.h"

namespace {

// Valid prime-factor FFT lengths: one optional factor from each coprime
// group {2,4,8,16}, {3,9}, {5}, {7}, {11}, {13} (the 240 lengths of
// src/fft.cc:275-353, generated rather than tabulated).
struct PfaLengths {
  int v[240];
  PfaLengths() {
    const int g2[5] = {1, 2, 4, 8, 16}, g3[3] = {1, 3, 9};
    int k = 0;
    for (int a : g2)
      for (int b : g3)
        for (int m = 0; m < 16; ++m)
          v[k++] = a * b * ((m & 1) ? 5 : 1) * ((m & 2) ? 7 : 1) *
                   ((m & 4) ? 11 : 1) * ((m & 8) ? 13 : 1);
    std::sort(v, v + 240);
  }
};
const PfaLengths &pfa() {
  static PfaLengths t;
  return t;
}

// npfa: first valid length >= nmin, capped at 720720 (src/fft.cc:439-447).
int npfa(int nmin) {
  const int *v = pfa().v;
  const int *it = std::lower_bound(v, v + 240, nmin);
  return it == v + 240 ? v[239] : *it;
}

}  // namespace

extern "C" int qpsdm_npfar(int nmin) { return 2 * npfa((nmin + 1) / 2); }

// src/q-psdm.cu:1167-1193.
extern "C" int qpsdm_build_iaztab(float eps, int *tab, int cap) {
  if (!tab || eps <= 0.0f) return -1;
  const int naz = (int)(2.0 / eps + 1.5);
  if (naz > cap) return -1;
  const double rad = 0.0174532925199;
  // sector edge in (1 - cos) units of a direction angle a (degrees), after
  // the reference's compression a -> (1 - cos a) * pi / 2.
  auto squash = [&](float deg) -> float {
    return (float)((1.0 - (double)cosf((float)(deg * rad))) * M_PI * 0.5);
  };
  float e = squash(10.0f);
  e = (float)(1.0 - (double)cosf((float)(e * 0.5)));
  int upper = (int)(e / eps);
  for (int i = 0; i < upper; ++i) tab[i] = 0;
  for (int iaz = 1; iaz < 18; ++iaz) {
    float c = (float)(iaz * 10.0);
    float a = squash((float)(c - 10.0));
    float b = squash(c);
    float d = squash((float)(c + 10.0));
    float lo = (float)(1.0 - (double)cosf((float)(b - (b - a) * 0.5)));
    float hi = (float)(1.0 - (double)cosf((float)(b + (d - b) * 0.5)));
    const int i1 = (int)(lo / eps);
    upper = (int)(hi / eps);
    for (int i = i1; i < upper; ++i) tab[i] = iaz;
  }
  for (int i = upper; i < naz; ++i) tab[i] = 0;
  return naz;
}

// src/q-psdm.cu:1201-1287 (+ the f3/f4 Nyquist clamps of main, :711-723).
extern "C" int qpsdm_static_params_init(qpsdm_static_params *p) {
  if (!p || p->ntl <= 0 || p->dt <= 0.0f || p->nzi <= 0 || p->nxi <= 0)
    return QPSDM_EINVAL;
  if (p->f3 > 0.5 / p->dt - 10.0) p->f3 = (float)(0.5 / p->dt - 10.0);
  if (p->f4 > 0.5 / p->dt - 5.0) p->f4 = (float)(0.5 / p->dt - 5.0);
  if (p->f4 - p->f3 <= 5.0) p->f3 = (float)(p->f4 - 5.0);
  p->eps = 0.001f;
  p->nfft = qpsdm_npfar(p->ntl);
  p->nffti = qpsdm_npfar(p->ntl * 2);
  p->df = (float)(1.0 / (p->nfft * p->dt));
  p->dw = (float)(2.0 * M_PI * p->df);
  const float odt1 = p->nffti * p->df;
  p->dt1 = (float)(1.0 / odt1);
  const float G = p->threshold;
  p->lnG = logf(G);
  p->coef1 = (float)(G * (1.0 - p->lnG - 2.5 * p->lnG * p->lnG));
  p->coef2 = (float)(G * (1.0 + 5.0 * p->lnG));
  p->coef3 = (float)(-2.5 * G);
  p->coef4 = (float)(1.1 * G);
  p->contract = (float)(p->contract * 0.01745329251994);
  p->taperzone = (float)(p->taperzone * 0.01745329251994);
  if (p->max_batch <= 0) p->max_batch = 4096;
  return QPSDM_OK;
}

// src/q-psdm.cu:1593-1645 with t00 = 0 and t11 = (ntl-1)*dt as shipped.
extern "C" int qpsdm_offset_params_init(const qpsdm_static_params *p,
                                        int ixstart, int ixend,
                                        qpsdm_offset_params *o) {
  if (!p || !o || ixstart < 0 || ixend <= ixstart || ixend > p->nxi)
    return QPSDM_EINVAL;
  const float dt = p->dt;
  const int pre = (int)(0.48 / dt), suf = (int)(0.36 / dt);
  const float t00 = 0.0f, t11 = (p->ntl - 1) * dt;
  int nsb = (int)((t11 - t00 - pre * dt - suf * dt) / 2.0 / dt);
  o->itb1 = (int)(t00 / dt);
  o->tdstart1 = o->itb1 * dt;
  o->tdmid = t00 + pre * dt + nsb * dt;
  nsb = qpsdm_npfar(nsb + pre + suf);
  o->nsb = nsb;
  o->itb2 = (int)(t11 / dt - nsb + 1);
  o->tdstart2 = o->itb2 * dt;
  o->df = (float)(1.0 / nsb / dt);
  o->dw = (float)(2.0 * M_PI * o->df);
  o->nf1 = (int)(p->f1 / o->df);
  const int nf4 = (int)(p->f4 / o->df);
  o->nww = nf4 - o->nf1 + 1;
  o->ncoef1 = (int)(10.0 / o->df);
  o->ixstart = ixstart;
  o->ixend = ixend;
  return QPSDM_OK;
}
