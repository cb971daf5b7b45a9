/*
 * qpsdm_oracle.c -- CPU restatement of the q-psdm imaging path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA engine in
 * q_psdm_b200/: it is loaded by tests/, by __graft_entry__.smoke() and by the
 * cpu_baseline leg of bench.py, never by the product path.
 *
 * It restates, in plain C with IEEE float/double semantics and no FMA
 * contraction (built with -ffp-contract=off), the reference computations:
 *
 *   orc_npfa / orc_npfar      src/fft.cc:439-447, :491-494 (valid PFA lengths)
 *   orc_build_iaztab          src/q-psdm.cu:1167-1193 (azimuth sector table)
 *   orc_derive_static         src/q-psdm.cu:1201-1287 (nfft, nffti, dt1, lnG,
 *                             coef1..4, contract/taperzone in radians)
 *   orc_window_split          src/q-psdm.cu:1593-1645 (two FFT windows)
 *   orc_gate_trace            src/q-psdm.cu:2107-2171 (bbox, cdp, azimuth,
 *                             aperture, itibeg/ixi1/ixi2)
 *   orc_gain, orc_fetch_and_taper, orc_preprocess_trace
 *                             src/q-psdm.cu:2174-2209, src/psdmpkg.cc:208-231
 *   orc_image_compat          src/q-psdm.cu:2246-2379 (image_depth_gpu with
 *                             the reference's ts = tg = 1 stub)
 *
 * Parity pins: orc_npfar, orc_fetch_and_taper and the r2c spectra are checked
 * against the reference's own compiled fft.cc / psdmpkg.cc (oracle/_ref) and
 * the committed golden vectors in tests/golden/.  The physics-mode oracle
 * (FP64) lives in oracle/physics_oracle.c.
 */
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ------------------------------------------------------------------------ */
/* Valid prime-factor FFT lengths.                                           */
/* The reference keeps a 240-entry table (src/fft.cc:275-353) of lengths made */
/* of mutually prime factors from {2,3,4,5,7,8,9,11,13,16}; npfa returns the */
/* first entry >= nmin (src/fft.cc:439-447) and npfar returns               */
/* 2*npfa((nmin+1)/2) (src/fft.cc:491-494).  The same set is generated here: */
/* one optional factor from each coprime group {2,4,8,16},{3,9},{5},{7},     */
/* {11},{13} -> 5*3*2*2*2*2 = 240 lengths, sorted.                          */
/* ------------------------------------------------------------------------ */
static int g_pfa_tab[240];
static int g_pfa_n = 0;

static int cmp_int(const void *a, const void *b) {
  int x = *(const int *)a, y = *(const int *)b;
  return (x > y) - (x < y);
}

static void pfa_table_init(void) {
  if (g_pfa_n) return;
  static const int g2[5] = {1, 2, 4, 8, 16};
  static const int g3[3] = {1, 3, 9};
  int k = 0;
  for (int a = 0; a < 5; ++a)
    for (int b = 0; b < 3; ++b)
      for (int c5 = 0; c5 < 2; ++c5)
        for (int c7 = 0; c7 < 2; ++c7)
          for (int c11 = 0; c11 < 2; ++c11)
            for (int c13 = 0; c13 < 2; ++c13)
              g_pfa_tab[k++] = g2[a] * g3[b] * (c5 ? 5 : 1) * (c7 ? 7 : 1) *
                               (c11 ? 11 : 1) * (c13 ? 13 : 1);
  qsort(g_pfa_tab, 240, sizeof(int), cmp_int);
  g_pfa_n = 240;
}

int orc_pfa_table(int *out, int cap) {
  pfa_table_init();
  int n = cap < g_pfa_n ? cap : g_pfa_n;
  memcpy(out, g_pfa_tab, sizeof(int) * (size_t)n);
  return g_pfa_n;
}

int orc_npfa(int nmin) {
  pfa_table_init();
  int i = 0;
  while (i < g_pfa_n - 1 && g_pfa_tab[i] < nmin) ++i;
  return g_pfa_tab[i];
}

int orc_npfar(int nmin) { return 2 * orc_npfa((nmin + 1) / 2); }

/* ------------------------------------------------------------------------ */
/* Azimuth table: 18 sectors of 10 degrees indexed by (1 - cos) / eps.       */
/* src/q-psdm.cu:1167-1193.  The float/double mix of the reference is kept   */
/* on purpose: sector edges decide integer indices.                         */
/* ------------------------------------------------------------------------ */
int orc_build_iaztab(float eps, int *tab, int cap) {
  int naz = (int)(2.0 / eps + 1.5);
  if (naz > cap) return -1;
  const double deg = 0.0174532925199;
  float e, lo, mid, hi;
  int i, i1, i2;

  e = (float)((1.0 - (double)cosf((float)(10.0 * deg))) * M_PI * 0.5);
  e = (float)(1.0 - (double)cosf((float)(e * 0.5)));
  i2 = (int)(e / eps);
  for (i = 0; i < i2; ++i) tab[i] = 0;
  for (int iaz = 1; iaz < 18; ++iaz) {
    mid = (float)(iaz * 10.0);
    lo = (float)(mid - 10.0);
    hi = (float)(mid + 10.0);
    lo = (float)((1.0 - (double)cosf((float)(lo * deg))) * M_PI * 0.5);
    mid = (float)((1.0 - (double)cosf((float)(mid * deg))) * M_PI * 0.5);
    hi = (float)((1.0 - (double)cosf((float)(hi * deg))) * M_PI * 0.5);
    lo = (float)(1.0 - (double)cosf((float)(mid - (mid - lo) * 0.5)));
    mid = (float)(1.0 - (double)cosf((float)(mid + (hi - mid) * 0.5)));
    i1 = (int)(lo / eps);
    i2 = (int)(mid / eps);
    for (i = i1; i < i2; ++i) tab[i] = iaz;
  }
  for (i = i2; i < naz; ++i) tab[i] = 0;
  return naz;
}

/* ------------------------------------------------------------------------ */
/* Line-independent constants, src/q-psdm.cu:1201-1287.                     */
/* out_i: [nfft, nffti]                                                      */
/* out_f: [df, dw, dt1, lnG, coef1, coef2, coef3, coef4, contract_rad,       */
/*         taperzone_rad]                                                    */
/* ------------------------------------------------------------------------ */
void orc_derive_static(int ntl, float dt, float threshold, float contract_deg,
                       float taperzone_deg, int *out_i, float *out_f) {
  int nfft = orc_npfar(ntl);
  int nffti = orc_npfar(ntl * 2);
  float df = (float)(1.0 / (nfft * dt));
  float dw = (float)(2.0 * M_PI * df);
  float odt1 = nffti * df;
  float dt1 = (float)(1.0 / odt1);
  float lnG = logf(threshold);
  float c1 = (float)(threshold * (1.0 - lnG - 2.5 * lnG * lnG));
  float c2 = (float)(threshold * (1.0 + 5.0 * lnG));
  float c3 = (float)(-2.5 * threshold);
  float c4 = (float)(1.1 * threshold);
  out_i[0] = nfft;
  out_i[1] = nffti;
  out_f[0] = df;
  out_f[1] = dw;
  out_f[2] = dt1;
  out_f[3] = lnG;
  out_f[4] = c1;
  out_f[5] = c2;
  out_f[6] = c3;
  out_f[7] = c4;
  out_f[8] = (float)(contract_deg * 0.01745329251994);
  out_f[9] = (float)(taperzone_deg * 0.01745329251994);
}

/* ------------------------------------------------------------------------ */
/* Two-window split of a trace for the spectra, src/q-psdm.cu:1593-1645.    */
/* out_i: [itb1, itb2, nsb, nf1, nf4, nww, ncoef1]                           */
/* out_f: [tdstart1, tdstart2, tdmid, df, dw]                                */
/* ------------------------------------------------------------------------ */
void orc_window_split(int ntl, float dt, float f1, float f4, int *out_i,
                      float *out_f) {
  int pre = (int)(0.48 / dt);
  int suf = (int)(0.36 / dt);
  float t00 = 0.0f;
  float t11 = (ntl - 1) * dt;
  int nsb = (int)((t11 - t00 - pre * dt - suf * dt) / 2.0 / dt);
  int itb1 = (int)(t00 / dt);
  float tdstart1 = itb1 * dt;
  float tdmid = t00 + pre * dt + nsb * dt;
  nsb = orc_npfar(nsb + pre + suf);
  int itb2 = (int)(t11 / dt - nsb + 1);
  float tdstart2 = itb2 * dt;
  float df = (float)(1.0 / nsb / dt);
  float dw = (float)(2.0 * M_PI * df);
  int nf1 = (int)(f1 / df);
  int nf4 = (int)(f4 / df);
  out_i[0] = itb1;
  out_i[1] = itb2;
  out_i[2] = nsb;
  out_i[3] = nf1;
  out_i[4] = nf4;
  out_i[5] = nf4 - nf1 + 1;
  out_i[6] = (int)(10.0 / df);
  out_f[0] = tdstart1;
  out_f[1] = tdstart2;
  out_f[2] = tdmid;
  out_f[3] = df;
  out_f[4] = dw;
}

/* ------------------------------------------------------------------------ */
/* Per-trace geometry gate, src/q-psdm.cu:2107-2171.                         */
/* ------------------------------------------------------------------------ */
typedef struct {
  double scaled;
  float fxv1, fyv1, exv1, eyv1;
  double fxi, cyi;
  float dxi, dyi, eps;
  int nzi, ixstart, ixend;
  const int *iaztab; /* naztab entries */
  const int *aznx1, *aznx2, *azny1, *azny2; /* 18 entries, this offset group */
} orc_gate_params;

/* out_i: [status, cdpx, cdpy, iaz, ixi1, ixi2, ntibeg, izimin]
 *   status 0 = outside the velocity bbox, 1 = outside the y aperture,
 *          2 = no image column in the block, 3 = accepted
 * out_f: [sx, sy, gx, gy] relative to (fxi, cyi), as the kernel receives them.
 */
int orc_gate_trace_cap(const orc_gate_params *p, int isx, int isy, int igx,
                       int igy, int capx, int capy, int *out_i, float *out_f);

int orc_gate_trace(const orc_gate_params *p, int isx, int isy, int igx,
                   int igy, int *out_i, float *out_f) {
  return orc_gate_trace_cap(p, isx, isy, igx, igy, INT_MAX, INT_MAX, out_i, out_f);
}

/* The same with the trace's own aperture (half-widths capx cdps, capy
 * lines) capping the azimuth tables: the engine's per-trace aperture of
 * gathers recorded with different apertures. */
int orc_gate_trace_cap(const orc_gate_params *p, int isx, int isy, int igx,
                       int igy, int capx, int capy, int *out_i, float *out_f) {
  double sx = isx * p->scaled, sy = isy * p->scaled;
  double gx = igx * p->scaled, gy = igy * p->scaled;
  memset(out_i, 0, sizeof(int) * 8);
  memset(out_f, 0, sizeof(float) * 4);
  if (sx < p->fxv1 || sx > p->exv1) return out_i[0] = 0;
  if (gx < p->fxv1 || gx > p->exv1) return out_i[0] = 0;
  if (sy < p->fyv1 || sy > p->eyv1) return out_i[0] = 0;
  if (gy < p->fyv1 || gy > p->eyv1) return out_i[0] = 0;

  double ddx = gx - sx, ddy = gy - sy;
  double offset = sqrtf((float)(ddx * ddx + ddy * ddy));
  int cdpx = (int)(((sx + gx) * 0.5 - p->fxi) / p->dxi + 0.5);
  int cdpy = (int)(((sy + gy) * 0.5 - p->cyi) / p->dyi + 0.5);
  int iaz = 0;
  if (offset > 1.0) {
    float cosx = (float)fabs((double)(float)(ddx / offset));
    if (ddx * ddy < 0.0) cosx = -cosx;
    float c1 = (float)(1.0 - cosx);
    iaz = p->iaztab[(int)(c1 / p->eps)];
  }
  out_i[1] = cdpx;
  out_i[2] = cdpy;
  out_i[3] = iaz;
  int nx1 = p->aznx1[iaz], nx2 = p->aznx2[iaz];
  int ny1 = p->azny1[iaz], ny2 = p->azny2[iaz];
  if (nx1 > capx) nx1 = capx;
  if (nx2 > capx) nx2 = capx;
  if (ny1 > capy) ny1 = capy;
  if (ny2 > capy) ny2 = capy;
  if (cdpy > ny1 || cdpy < -ny2) return out_i[0] = 1;

  /* columns cdpx-nx1 .. cdpx+nx2-1 clipped to [ixstart, ixend); the start
   * depth of every column is 0 and columns exist only when nzi > 10. */
  int first = cdpx - nx1, last = cdpx + nx2 - 1;
  if (first < p->ixstart) first = p->ixstart;
  if (last > p->ixend - 1) last = p->ixend - 1;
  int ntibeg = (p->nzi > 10 && last >= first) ? last - first + 1 : 0;
  if (ntibeg == 0) return out_i[0] = 2;
  out_i[4] = first;
  out_i[5] = last;
  out_i[6] = ntibeg;
  out_i[7] = 0;
  out_f[0] = (float)(sx - p->fxi);
  out_f[1] = (float)(sy - p->cyi);
  out_f[2] = (float)(gx - p->fxi);
  out_f[3] = (float)(gy - p->cyi);
  return out_i[0] = 3;
}

/* ------------------------------------------------------------------------ */
/* Trace preprocessing, src/q-psdm.cu:2174-2209 and psdmpkg.cc:208-231.     */
/* ------------------------------------------------------------------------ */
void orc_gain(float *d, int ntl, float dt) {
  for (int it = 0; it < ntl; ++it) {
    float t = it * dt;
    if ((double)t < 0.1)
      d[it] = (float)(d[it] * (0.1 * 0.1));
    else
      d[it] *= t * t;
  }
}

void orc_fetch_and_taper(const float *data, int ns, int it1, int it2,
                         float *out) {
  for (int it = it1; it <= it2; ++it)
    out[it - it1] = (it < 0 || it >= ns) ? 0.0f : data[it];
  int n = it2 - it1 + 1;
  for (int it = 0; it < 200 && it < n; ++it) {
    float c = (float)(0.5 - 0.5 * cosf((float)(M_PI * it / 200.0)));
    out[it] *= c;
    out[n - 1 - it] *= c;
  }
}

/* Unnormalised forward real DFT, sign e^{-i w t}, bins 0..n/2, in double.
 * Direct summation with exact integer phase reduction: O(n^2) but exact to
 * double rounding, which is what an oracle wants. */
void orc_rdft(const float *x, int n, double *re, double *im) {
  for (int k = 0; k <= n / 2; ++k) {
    double sr = 0.0, si = 0.0;
    long long m = 0;
    for (int t = 0; t < n; ++t) {
      double a = -2.0 * M_PI * (double)m / (double)n;
      sr += x[t] * cos(a);
      si += x[t] * sin(a);
      m += k;
      if (m >= n) m -= n;
    }
    re[k] = sr;
    im[k] = si;
  }
}

/* Full per-trace preprocessing of psdm_kernel: t^2 gain, full-trace taper,
 * two tapered windows of nsb samples, r2c, -i*w filter over nww bins from
 * nf1.  Writes re[2*nww], im[2*nww] (window 1 then window 2). */
void orc_preprocess_trace(const float *trace, int ntl, float dt, int itb1,
                          int itb2, int nsb, int nf1, int nww, float dw,
                          float *re, float *im) {
  float *g = (float *)malloc(sizeof(float) * (size_t)ntl);
  float *full = (float *)malloc(sizeof(float) * (size_t)ntl);
  float *win = (float *)malloc(sizeof(float) * (size_t)nsb);
  double *xr = (double *)malloc(sizeof(double) * (size_t)(nsb / 2 + 1));
  double *xi = (double *)malloc(sizeof(double) * (size_t)(nsb / 2 + 1));
  memcpy(g, trace, sizeof(float) * (size_t)ntl);
  orc_gain(g, ntl, dt);
  orc_fetch_and_taper(g, ntl, 0, ntl - 1, full);
  for (int w = 0; w < 2; ++w) {
    int itb = w == 0 ? itb1 : itb2;
    orc_fetch_and_taper(full, ntl, itb, itb + nsb - 1, win);
    orc_rdft(win, nsb, xr, xi);
    float omega = nf1 * dw;
    for (int iw = 0; iw < nww; ++iw, omega += dw) {
      re[w * nww + iw] = (float)(xi[iw + nf1] * omega);
      im[w * nww + iw] = (float)(-xr[iw + nf1] * omega);
    }
  }
  free(g);
  free(full);
  free(win);
  free(xr);
  free(xi);
}

/* ------------------------------------------------------------------------ */
/* Stub imaging kernel, src/q-psdm.cu:2246-2379, reference-compat semantics. */
/* ------------------------------------------------------------------------ */
typedef struct {
  int nzi, nxb, ixstart, nt; /* nt = nffti */
  float dt1, dxi, dzi, taperzone;
  int tcdp1, tcdp2; /* table cdp range relative to fci */
} orc_image_params;

/* One point of one trace; returns the contribution (0 when masked). */
static inline float compat_point(const orc_image_params *p, const float *g,
                                 int ixi, int izi, float tanx1, float tanx2,
                                 float tany1, float tany2, int *masked) {
  float sx = g[0], sy = g[1], gx = g[2], gy = g[3];
  float z = izi * p->dzi;
  float z2 = z * z;
  float x = ixi * p->dxi;
  float dsx = sx - x, dgx = gx - x;
  float ds = sqrtf(dsx * dsx + sy * sy + z2);
  float dg = sqrtf(dgx * dgx + gy * gy + z2);
  float ux = dsx / ds + dgx / dg;
  float uy = sy / ds + gy / dg;
  float uz = z / ds + z / dg;
  float tanx = ux / uz, tany = uy / uz;
  float tz = p->taperzone;
  float tanx1c = tanx1 - tz * (1.0f + tanx1 * tanx1);
  float tanx2c = tanx2 + tz * (1.0f + tanx2 * tanx2);
  float tany1c = tany1 - tz * (1.0f + tany1 * tany1);
  float tany2c = tany2 + tz * (1.0f + tany2 * tany2);
  *masked = 1;
  /* Same test as the reference's `tanx <= tanx1c || ...` reject for every
   * number; a NaN tangent (0/0 at z = 0 when source, receiver and node are
   * collinear) is rejected as well, which is what the reference binary does
   * (its --use_fast_math divisions leave a tiny nonzero numerator there, so
   * the tangent is +-inf and fails the test). */
  if (!(tanx > tanx1c && tanx < tanx2c && tany > tany1c && tany < tany2c))
    return 0.0f;
  float w = 1.0f;
  if (tanx < tanx1) w *= (tanx - tanx1c) / (tanx1 - tanx1c);
  if (tanx > tanx2) w *= (tanx2c - tanx) / (tanx2c - tanx2);
  if (tany < tany1) w *= (tany - tany1c) / (tany1 - tany1c);
  if (tany > tany2) w *= (tany2c - tany) / (tany2c - tany2);
  float ts = 1.0f, tg = 1.0f;
  float t = ts + tg;
  int it1 = (int)(t / p->dt1);
  int it2 = it1 + 1;
  if (!(it1 > 0 && it2 < p->nt)) return 0.0f;
  *masked = 0;
  float v = 100.0f;
  if ((double)t > 0.1)
    v /= t * t;
  else
    v *= 100.0f;
  float r = ds / dg * ds / dg * ds / dg * tg / ts;
  r = (float)(w * ((double)r + 1.0 / (double)r));
  return v * r;
}

/* Accumulate ntr gated traces into img[nxb][nzi] in trace order.
 * geom: per trace [sx, sy, gx, gy] (floats, relative), ints: per trace
 * [ixi1, ixi2, izimin] (only accepted traces are passed).
 * Parallel over image columns; each column sums traces in order, so the
 * result does not depend on the thread count.
 * nmask (optional): per-trace count of evaluated-but-masked points. */
void orc_image_compat(const orc_image_params *p, int ntr, const float *geom,
                      const int *ints, const float *dipx1, const float *dipx2,
                      const float *dipy1, const float *dipy2, float *img,
                      long long *npt_out) {
  long long npt = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : npt)
  for (int ixb = 0; ixb < p->nxb; ++ixb) {
    int ixi = ixb + p->ixstart;
    for (int itr = 0; itr < ntr; ++itr) {
      const int *q = ints + 3 * itr;
      if (ixi < q[0] || ixi > q[1]) continue;
      if (ixi < p->tcdp1 || ixi > p->tcdp2) continue;
      const float *g = geom + 4 * itr;
      for (int izi = q[2]; izi < p->nzi; ++izi) {
        size_t k = (size_t)ixi * p->nzi + izi;
        int masked;
        float v = compat_point(p, g, ixi, izi, dipx1[k], dipx2[k], dipy1[k],
                               dipy2[k], &masked);
        npt += 1;
        if (!masked) img[(size_t)ixb * p->nzi + izi] += v;
      }
    }
  }
  if (npt_out) *npt_out = npt;
}

/* Final scale of get_image: img /= nsb (src/q-psdm.cu:1761-1765). */
void orc_scale_image(float *img, long long n, int nsb) {
  for (long long i = 0; i < n; ++i) img[i] /= nsb;
}

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
