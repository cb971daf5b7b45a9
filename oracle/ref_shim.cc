// ref_shim.cc -- C-linkage entry points over the reference's own CPU code.
//
// TEST INFRASTRUCTURE ONLY.  Linked with fft.o / psdmpkg.o / segy.o compiled
// from the reference sources in place (oracle/Makefile).  Used to pin the
// oracle (golden-vector generation, tests) and as the "reference" CPU
// baseline of bench.py.  Nothing here is shipped.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "psdmpkg.h"  // fetch_and_taper, getscale (reference header, in place)

// Defined in the reference's fft.cc (src/fft.cc:439, :491, :1838) without a
// header declaration; C++ linkage.
int npfa(int nmin);
int npfar(int nmin);
void pfarc(int isign, int n, float *rz, float *cz);

extern "C" {

int ref_npfa(int nmin) { return npfa(nmin); }
int ref_npfar(int nmin) { return npfar(nmin); }

// r2c as the reference drives it (src/fft.cc:3749-3757): isign = -1,
// unnormalised; cz holds n/2+1 interleaved (re, im) pairs.
void ref_pfarc(int isign, int n, float *rz, float *cz) { pfarc(isign, n, rz, cz); }

int ref_fetch_and_taper(const float *data, int ns, int it1, int it2,
                        float *out) {
  return fetch_and_taper(data, ns, it1, it2, out);
}

float ref_getscale(short scalco) { return getscale(scalco); }

// The preprocessing sequence of psdm_kernel (src/q-psdm.cu:2174-2209) driven
// through the reference's compiled fetch_and_taper and pfarc: t^2 gain,
// full-trace taper, two tapered windows of nsb samples, r2c, -i*w over nww
// bins from nf1.  ntr traces of ntl samples; re/im: [ntr][2*nww].
// Threads split the traces (each trace is independent).
void ref_preprocess_traces(const float *traces, int ntr, int ntl, float dt,
                           int itb1, int itb2, int nsb, int nf1, int nww,
                           float dw, float *re, float *im, int nthreads) {
#pragma omp parallel num_threads(nthreads)
  {
    float *d = (float *)malloc(sizeof(float) * ntl);
    float *data = (float *)malloc(sizeof(float) * ntl);
    float *win = (float *)malloc(sizeof(float) * (nsb + 2));
    float *spec = (float *)malloc(sizeof(float) * (nsb + 2));
#pragma omp for schedule(static)
    for (int itr = 0; itr < ntr; ++itr) {
      memcpy(d, traces + (size_t)itr * ntl, sizeof(float) * ntl);
      for (int it = 0; it < ntl; ++it) {
        if (it * dt < 0.1)
          d[it] *= 0.1 * 0.1;
        else
          d[it] *= (it * dt) * (it * dt);
      }
      fetch_and_taper(d, ntl, 0, ntl - 1, data);
      for (int w = 0; w < 2; ++w) {
        int itb = w == 0 ? itb1 : itb2;
        fetch_and_taper(data, ntl, itb, itb + nsb - 1, win);
        pfarc(-1, nsb, win, spec);
        float omega = nf1 * dw;
        float *r = re + (size_t)itr * 2 * nww + w * nww;
        float *m = im + (size_t)itr * 2 * nww + w * nww;
        for (int iw = 0; iw < nww; ++iw, omega += dw) {
          r[iw] = +spec[2 * (iw + nf1) + 1] * omega;
          m[iw] = -spec[2 * (iw + nf1) + 0] * omega;
        }
      }
    }
    free(d);
    free(data);
    free(win);
    free(spec);
  }
}

}  // extern "C"
