// ref_gpu_shim.cu -- drives the reference's own per-trace engine on a GPU.
//
// TEST INFRASTRUCTURE ONLY.  Linked with q-psdm.o, compiled from the
// reference's src/q-psdm.cu in place with the reference's own flags
// (-O2 --use_fast_math, src/Makefile:14) for sm_100a.  It calls the
// reference's psdm_kernel (src/q-psdm.cu:2063-2244), which gates each trace,
// runs the host preprocessing, copies spectra and launches image_depth_gpu
// (src/q-psdm.cu:2246-2380).  Inputs the reference leaves uninitialised
// (aznx1/aznx2/azny1/azny2, src/q-psdm.cu:1542-1545) are supplied here.
//
// Used only to make golden vectors and to pin the C restatement; the engine in
// q_psdm_b200/ never links it.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fft.h"
#include "segy.h"

extern FILE *fplog;  // defined in q-psdm.cu; set by main() in the reference

typedef struct {
  int64_t idx;
  uint16_t nys;
  uint16_t nxs;
  uint16_t dys;
  uint16_t dxs;
} ttt_desc_t;  // src/q-psdm.cu:103-109

// Signature of src/q-psdm.cu:252-283 with QMIG3D defined.
void psdm_kernel(segy tr, float dyi, float dxi, int nxi, int nzi, int ntl,
                 double scaled, int fci, float dzi, int ndipx, int ndipy,
                 float ddipx, float ddipy, float dt, float fc, float eps,
                 int *iaztab, float fxv1, float fyv1, float exv1, float eyv1,
                 int nfft, int nffti, float *ww, float dt1, int ndipx2,
                 int ndipy2, float taperzone, float lnG, float coef1,
                 float coef2, float coef3, float coef4, float dzii,
                 int ****aper, int **aznx1, int **aznx2, int **azny1,
                 int **azny2, double fxi, double cyi, float dw, int ioffs,
                 int itb1, int itb2, int nsb, float tdstart1, float tdstart2,
                 int nf1, float tdmid, int nww, int nxg, int nzg, int nxi1,
                 int nzi1, int ttt_cdp1, int ttt_cdp2, int qqq_cdp1,
                 int qqq_cdp2, int ncoef1, int ixstart, int ixend, int nxb,
                 float *re, float *im, float *red, float *imd, int igpu,
                 int *itibeg, int *itibegd, int *nf3d, float *Qd, float *datav,
                 fftwf_complex *wdatav, fftwf_plan planv, ttt_desc_t *qqq_descd,
                 float *qqqd, float *data, float *datad, float *dipx1d,
                 float *dipx2d, float *dipy1d, float *dipy2d,
                 ttt_desc_t *ttt_descd, float *tttd, float *imgd);

extern "C" {

// Plain-old-data argument block filled by the Python test harness.
typedef struct {
  float dyi, dxi;
  int nxi, nzi, ntl;
  double scaled;
  int fci;
  float dzi, dt, fc, eps;
  float fxv1, fyv1, exv1, eyv1;
  int nfft, nffti;
  float dt1, taperzone, lnG, coef1, coef2, coef3, coef4, dzii;
  double fxi, cyi;
  float dw;
  int itb1, itb2, nsb;
  float tdstart1, tdstart2;
  int nf1;
  float tdmid;
  int nww, ncoef1, ixstart, ixend, nxb;
  int ttt_cdp1, ttt_cdp2; /* absolute cdp numbers */
} ref_gpu_args;

// Runs ntr traces through psdm_kernel.  hdr: [ntr][4] = sx, sy, gx, gy (SU
// integer coordinates); traces: [ntr][ntl]; iaztab: naztab ints; az: 4 x 18
// ints (aznx1, aznx2, azny1, azny2 for this offset group); dips: 4 x nxi*nzi.
// Outputs: img [nxb][nzi] (before the /nsb of the writer), accepted[ntr],
// re/im [ntr][2*nww] (spectra copied after each accepted trace).
// Returns 0 on success, a CUDA error code otherwise.
int ref_gpu_run(const ref_gpu_args *a, int ntr, const int *hdr,
                const float *traces, int *iaztab, const int *az,
                const float *dips, float *img, int *accepted, float *re_out,
                float *im_out) {
  fplog = stderr;
  cudaError_t err;
  const size_t nxz = (size_t)a->nxi * a->nzi;
  int *aznx1 = (int *)az, *aznx2 = (int *)az + 18, *azny1 = (int *)az + 36,
      *azny2 = (int *)az + 54;
  int *aznx1p[1] = {aznx1}, *aznx2p[1] = {aznx2}, *azny1p[1] = {azny1},
      *azny2p[1] = {azny2};

  float *re = (float *)calloc(a->ntl * 4, sizeof(float));
  float *im = (float *)calloc(a->ntl * 4, sizeof(float));
  int *itibeg = (int *)calloc(a->nxi, sizeof(int));
  float *data = (float *)calloc(a->nffti + a->ntl, sizeof(float));
  float *datav = fftwf_alloc_real(a->ntl * 4);
  fftwf_complex *wdatav = fftwf_alloc_complex(a->ntl * 4);
  fftwf_plan planv = fftwf_plan_dft_r2c_1d(a->nsb, datav, wdatav, FFTW_MEASURE);

  float *red, *imd, *Qd, *datad, *dip_d, *imgd, *tttd, *qqqd;
  int *itibegd, *nf3d;
  ttt_desc_t *tdesc, *qdesc;
  cudaMalloc(&red, sizeof(float) * a->ntl * 4);
  cudaMalloc(&imd, sizeof(float) * a->ntl * 4);
  cudaMalloc(&itibegd, sizeof(int) * a->nxi);
  cudaMemset(itibegd, 0, sizeof(int) * a->nxi);
  cudaMalloc(&nf3d, sizeof(int) * nxz);
  cudaMalloc(&Qd, sizeof(float) * nxz);
  cudaMalloc(&datad, sizeof(float) * a->nffti);
  cudaMalloc(&dip_d, sizeof(float) * nxz * 4);
  cudaMalloc(&imgd, sizeof(float) * a->nxb * a->nzi);
  cudaMalloc(&tttd, 64);
  cudaMalloc(&qqqd, 64);
  cudaMalloc(&tdesc, sizeof(ttt_desc_t));
  cudaMalloc(&qdesc, sizeof(ttt_desc_t));
  cudaMemcpy(dip_d, dips, sizeof(float) * nxz * 4, cudaMemcpyHostToDevice);
  cudaMemset(imgd, 0, sizeof(float) * a->nxb * a->nzi);
  if ((err = cudaGetLastError()) != cudaSuccess) return (int)err;

  segy *tr = new segy;
  for (int itr = 0; itr < ntr; ++itr) {
    memset(tr, 0, sizeof(segy));
    tr->sx = hdr[4 * itr + 0];
    tr->sy = hdr[4 * itr + 1];
    tr->gx = hdr[4 * itr + 2];
    tr->gy = hdr[4 * itr + 3];
    tr->ns = a->ntl;
    memcpy(tr->data, traces + (size_t)itr * a->ntl, sizeof(float) * a->ntl);
    re[0] = NAN;
    psdm_kernel(*tr, a->dyi, a->dxi, a->nxi, a->nzi, a->ntl, a->scaled, a->fci,
                a->dzi, 0, 0, 1.0f, 1.0f, a->dt, a->fc, a->eps, iaztab, a->fxv1,
                a->fyv1, a->exv1, a->eyv1, a->nfft, a->nffti, NULL, a->dt1, 1,
                1, a->taperzone, a->lnG, a->coef1, a->coef2, a->coef3,
                a->coef4, a->dzii, NULL, aznx1p, aznx2p, azny1p, azny2p,
                a->fxi, a->cyi, a->dw, 0, a->itb1, a->itb2, a->nsb,
                a->tdstart1, a->tdstart2, a->nf1, a->tdmid, a->nww, 1, 1, 1, 1,
                a->ttt_cdp1, a->ttt_cdp2, a->ttt_cdp1, a->ttt_cdp2, a->ncoef1,
                a->ixstart, a->ixend, a->nxb, re, im, red, imd, 0, itibeg,
                itibegd, nf3d, Qd, datav, wdatav, planv, qdesc, qqqd, data,
                datad, dip_d, dip_d + nxz, dip_d + 2 * nxz, dip_d + 3 * nxz,
                tdesc, tttd, imgd);
    accepted[itr] = isnan(re[0]) ? 0 : 1;
    if (accepted[itr] && re_out) {
      memcpy(re_out + (size_t)itr * 2 * a->nww, re, sizeof(float) * 2 * a->nww);
      memcpy(im_out + (size_t)itr * 2 * a->nww, im, sizeof(float) * 2 * a->nww);
    }
  }
  delete tr;
  cudaDeviceSynchronize();
  err = cudaMemcpy(img, imgd, sizeof(float) * a->nxb * a->nzi,
                   cudaMemcpyDeviceToHost);

  cudaFree(red);
  cudaFree(imd);
  cudaFree(itibegd);
  cudaFree(nf3d);
  cudaFree(Qd);
  cudaFree(datad);
  cudaFree(dip_d);
  cudaFree(imgd);
  cudaFree(tttd);
  cudaFree(qqqd);
  cudaFree(tdesc);
  cudaFree(qdesc);
  free(re);
  free(im);
  free(itibeg);
  free(data);
  fftwf_free(datav);
  fftwf_free(wdatav);
  return (int)err;
}

}  // extern "C"
