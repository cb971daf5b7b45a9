// internal.h -- declarations shared by the engine's translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "qpsdm_engine.h"

namespace qpsdm {

// Counts every engine launch per kernel class; when `on`, also brackets each
// launch with a pair of CUDA events on its stream (qpsdm_profile_*).
struct KernelProfiler {
  bool on = false;
  int64_t launches[4] = {0, 0, 0, 0};
  struct Rec {
    cudaEvent_t a, b;
    int cls;
  };
  std::vector<Rec> recs;
  std::vector<cudaEvent_t> pool;
  cudaEvent_t take() {
    if (!pool.empty()) {
      cudaEvent_t e = pool.back();
      pool.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
  }
  int cur = -1;
  void begin(int cls, cudaStream_t s) {
    launches[cls] += 1;
    if (!on) return;
    Rec r{take(), take(), cls};
    cudaEventRecord(r.a, s);
    recs.push_back(r);
    cur = (int)recs.size() - 1;
  }
  void end(cudaStream_t s) {
    if (!on || cur < 0) return;
    cudaEventRecord(recs[cur].b, s);
    cur = -1;
  }
  void reset() {
    for (auto &r : recs) {
      pool.push_back(r.a);
      pool.push_back(r.b);
    }
    recs.clear();
    for (auto &l : launches) l = 0;
  }
  double total_ms(int cls) {
    double t = 0.0;
    for (auto &r : recs)
      if (r.cls == cls) {
        cudaEventSynchronize(r.b);
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) t += ms;
      }
    return t;
  }
  ~KernelProfiler() {
    reset();
    for (auto e : pool) cudaEventDestroy(e);
  }
};

struct FftPlan;
int fft_plan(int n, FftPlan *out, std::string *err);
int fft_set_smem_attr(const void *kernel, size_t bytes);

// Gate of a trace batch (src/q-psdm.cu:2107-2171), one thread per trace.
struct GateArgs {
  double scaled, fxi, cyi;
  float fxv1, fyv1, exv1, eyv1;
  float dxi, dyi, eps;
  int nzi, ixstart, ixend, naztab;
  const int *iaztab;              // device
  int az[4][QPSDM_NAZ];           // aznx1, aznx2, azny1, azny2
  // device, 2 per trace (half-width in cdps, in lines) capping the azimuth
  // tables: the aperture a gather was recorded with; null = tables only
  const int *cap;
};

int launch_gate(const uint8_t *d_rec, int rec_bytes, int ntr, int big_endian,
                const GateArgs &g, int *d_ints, float *d_geom,
                unsigned *d_err, unsigned long long *d_nacc, cudaStream_t s);

// Two-window spectra of accepted traces (src/q-psdm.cu:2174-2219).
struct SpectraArgs {
  int ntl, nsb, itb1, itb2, nf1, nww;
  float dt;
  const float *taper200;  // device, 200 reference taper factors
  const float *omega;     // device, nww frequencies (float accumulation)
};
int launch_spectra(const uint8_t *d_rec, int rec_bytes, int ntr, int big_endian,
                   const int *d_ints, const SpectraArgs &a, float *d_re,
                   float *d_im, cudaStream_t s);

// Stub imaging (src/q-psdm.cu:2246-2379) over a trace batch.
struct CompatImageArgs {
  int nzi, nxb, ixstart, nt;
  float dt1, dxi, dzi, taperzone;
  int tcdp1, tcdp2;  // table cdp range relative to fci
  size_t nxz;        // nxi * nzi (dip field stride)
};
int launch_image_compat(float *d_img, const CompatImageArgs &a,
                        const float *d_dips, const int *d_ints,
                        const float *d_geom, int ntr,
                        unsigned long long *d_npt, cudaStream_t s);

}  // namespace qpsdm
