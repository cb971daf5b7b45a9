// compat.cu -- the reference-compatible imaging path on sm_100a.
//
//   k_gate      psdm_kernel's per-trace geometry gate (src/q-psdm.cu:2107-2171)
//   k_spectra   psdm_kernel's preprocessing: t^2 gain, tapers, two r2c
//               windows, -i*w (src/q-psdm.cu:2174-2219, psdmpkg.cc:208-231)
//   k_image_compat  image_depth_gpu with the reference's ts = tg = 1 stub
//               (src/q-psdm.cu:2246-2379), batched over traces
//
// Rounding: every operation that feeds an index, a mask or the image uses an
// explicit IEEE intrinsic (__fadd_rn, __fdiv_rn, __fsqrt_rn, __dadd_rn, ...)
// so that nothing is contracted into an FMA or approximated; a plain C
// restatement built with -ffp-contract=off computes the same bits.
#include "common.cuh"
#include "fft.cuh"
#include "internal.h"

namespace qpsdm {

// ---------------------------------------------------------------------------
// Gate: one thread per trace.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool gate_trace(const uint8_t *__restrict__ rec, int rec_bytes,
                                           int itr, int be, const GateArgs &g,
                                           int *__restrict__ ints, float *__restrict__ geom,
                                           unsigned *err) {
  const uint8_t *r = rec + (size_t)itr * rec_bytes;
  int *o = ints + (size_t)itr * kGateInts;
  float *f = geom + (size_t)itr * kGateF;
#pragma unroll
  for (int i = 0; i < kGateInts; ++i) o[i] = 0;
#pragma unroll
  for (int i = 0; i < kGateF; ++i) f[i] = 0.0f;

  const double sx = __dmul_rn((double)su_i32(r, kOffSx, be), g.scaled);
  const double sy = __dmul_rn((double)su_i32(r, kOffSy, be), g.scaled);
  const double gx = __dmul_rn((double)su_i32(r, kOffGx, be), g.scaled);
  const double gy = __dmul_rn((double)su_i32(r, kOffGy, be), g.scaled);
  if (sx < g.fxv1 || sx > g.exv1 || gx < g.fxv1 || gx > g.exv1 ||
      sy < g.fyv1 || sy > g.eyv1 || gy < g.fyv1 || gy > g.eyv1) {
    o[0] = kRejBbox;
    return false;
  }
  const double ddx = __dsub_rn(gx, sx), ddy = __dsub_rn(gy, sy);
  const double offset = (double)__fsqrt_rn(
      __double2float_rn(__dadd_rn(__dmul_rn(ddx, ddx), __dmul_rn(ddy, ddy))));
  const int cdpx = __double2int_rz(__dadd_rn(
      __ddiv_rn(__dsub_rn(__dmul_rn(__dadd_rn(sx, gx), 0.5), g.fxi), (double)g.dxi), 0.5));
  const int cdpy = __double2int_rz(__dadd_rn(
      __ddiv_rn(__dsub_rn(__dmul_rn(__dadd_rn(sy, gy), 0.5), g.cyi), (double)g.dyi), 0.5));
  int iaz = 0;
  if (offset > 1.0) {
    float cosx = fabsf(__double2float_rn(__ddiv_rn(ddx, offset)));
    if (__dmul_rn(ddx, ddy) < 0.0) cosx = -cosx;
    const float c1 = __double2float_rn(__dsub_rn(1.0, (double)cosx));
    int i = __float2int_rz(__fdiv_rn(c1, g.eps));
    if (i < 0 || i >= g.naztab) {  // cannot happen for |cos| <= 1; never read out of bounds
      atomicOr(err, kErrIaz);
      i = i < 0 ? 0 : g.naztab - 1;
    }
    iaz = g.iaztab[i];
  }
  o[1] = cdpx;
  o[2] = cdpy;
  o[3] = iaz;
  int nx1 = g.az[0][iaz], nx2 = g.az[1][iaz];
  int ny1 = g.az[2][iaz], ny2 = g.az[3][iaz];
  if (g.cap) {  // the trace's own aperture caps the offset group's
    const int cx = g.cap[2 * (size_t)itr], cy = g.cap[2 * (size_t)itr + 1];
    nx1 = min(nx1, cx);
    nx2 = min(nx2, cx);
    ny1 = min(ny1, cy);
    ny2 = min(ny2, cy);
  }
  if (cdpy > ny1 || cdpy < -ny2) {
    o[0] = kRejY;
    return false;
  }
  // Columns cdpx-nx1 .. cdpx+nx2-1 clipped to the block; every column starts
  // at depth 0 and columns exist only when nzi > 10 (src/q-psdm.cu:2155-2171).
  int first = cdpx - nx1, last = cdpx + nx2 - 1;
  if (first < g.ixstart) first = g.ixstart;
  if (last > g.ixend - 1) last = g.ixend - 1;
  const int ntibeg = (g.nzi > 10 && last >= first) ? last - first + 1 : 0;
  if (ntibeg == 0) {
    o[0] = kRejCols;
    return false;
  }
  o[0] = kAccepted;
  o[4] = first;
  o[5] = last;
  o[6] = ntibeg;
  o[7] = 0;
  f[0] = __double2float_rn(__dsub_rn(sx, g.fxi));
  f[1] = __double2float_rn(__dsub_rn(sy, g.cyi));
  f[2] = __double2float_rn(__dsub_rn(gx, g.fxi));
  f[3] = __double2float_rn(__dsub_rn(gy, g.cyi));
  return true;
}

__global__ void k_gate(const uint8_t *__restrict__ rec, int rec_bytes, int ntr,
                       int be, GateArgs g, int *__restrict__ ints,
                       float *__restrict__ geom, unsigned *err,
                       unsigned long long *__restrict__ nacc) {
  const int itr = blockIdx.x * blockDim.x + threadIdx.x;
  // accepted traces of the block, one atomic per warp (graph replays count too)
  const bool accepted = itr < ntr && gate_trace(rec, rec_bytes, itr, be, g, ints, geom, err);
  const unsigned ballot = __ballot_sync(0xffffffffu, accepted);
  if (nacc && (threadIdx.x & 31) == 0 && ballot)
    atomicAdd(nacc, (unsigned long long)__popc(ballot));
}

int launch_gate(const uint8_t *d_rec, int rec_bytes, int ntr, int be,
                const GateArgs &g, int *d_ints, float *d_geom, unsigned *d_err,
                unsigned long long *d_nacc, cudaStream_t s) {
  if (ntr <= 0) return QPSDM_OK;
  k_gate<<<(ntr + 127) / 128, 128, 0, s>>>(d_rec, rec_bytes, ntr, be, g, d_ints,
                                           d_geom, d_err, d_nacc);
  return cudaGetLastError() == cudaSuccess ? QPSDM_OK : QPSDM_ECUDA;
}

// ---------------------------------------------------------------------------
// Spectra: one CTA per (accepted trace, window).
// ---------------------------------------------------------------------------

// Gained sample j of the trace, then the full-trace end taper applied in the
// reference's order (src/psdmpkg.cc:221-228: head factor at iteration j, tail
// factor at iteration n-1-j; the earlier iteration multiplies first).
__device__ __forceinline__ float tapered_sample(float v, int j, int n,
                                                const float *tap) {
  const int head = j, tail = n - 1 - j;
  const bool h = head < 200, t = tail < 200;
  if (h && t) {
    if (head <= tail) {
      v = __fmul_rn(v, tap[head]);
      v = __fmul_rn(v, tap[tail]);
    } else {
      v = __fmul_rn(v, tap[tail]);
      v = __fmul_rn(v, tap[head]);
    }
  } else if (h) {
    v = __fmul_rn(v, tap[head]);
  } else if (t) {
    v = __fmul_rn(v, tap[tail]);
  }
  return v;
}

__device__ __forceinline__ float gained(float v, int it, float dt) {
  const float t = __fmul_rn((float)it, dt);
  if ((double)t < 0.1) return __double2float_rn(__dmul_rn((double)v, 0.1 * 0.1));
  return __fmul_rn(v, __fmul_rn(t, t));
}

__global__ void __launch_bounds__(256) k_spectra(const uint8_t *__restrict__ rec,
                                                 int rec_bytes, int be,
                                                 const int *__restrict__ ints,
                                                 SpectraArgs a, FftPlan p,
                                                 float *__restrict__ re,
                                                 float *__restrict__ im) {
  const int itr = blockIdx.x, win = blockIdx.y;
  if (ints[(size_t)itr * kGateInts] != kAccepted) return;
  extern __shared__ float2 sm[];
  float2 *b0 = sm, *b1 = sm + p.m, *twm = sm + 2 * p.m, *twn = sm + 3 * p.m;
  for (int i = threadIdx.x; i < p.m; i += blockDim.x) twm[i] = p.tw_m[i];
  for (int i = threadIdx.x; i <= p.m; i += blockDim.x) twn[i] = p.tw_n[i];
  const uint8_t *r = rec + (size_t)itr * rec_bytes;
  const int itb = win == 0 ? a.itb1 : a.itb2;
  float *bf = reinterpret_cast<float *>(b0);
  for (int i = threadIdx.x; i < a.nsb; i += blockDim.x) {
    const int j = itb + i;
    float v = 0.0f;
    if (j >= 0 && j < a.ntl)
      v = tapered_sample(gained(su_sample(r, j, be), j, a.dt), j, a.ntl, a.taper200);
    bf[i] = tapered_sample(v, i, a.nsb, a.taper200);
  }
  __syncthreads();
  const int cur = fft_complex_smem(b0, b1, p, twm, false);
  const float2 *Z = cur ? b1 : b0;
  float *ro = re + (size_t)itr * 2 * a.nww + win * a.nww;
  float *io = im + (size_t)itr * 2 * a.nww + win * a.nww;
  for (int iw = threadIdx.x; iw < a.nww; iw += blockDim.x) {
    const float2 X = rfft_bin(Z, twn, p.m, iw + a.nf1);
    const float w = a.omega[iw];
    ro[iw] = __fmul_rn(X.y, w);
    io[iw] = -__fmul_rn(X.x, w);
  }
}

int launch_spectra(const uint8_t *d_rec, int rec_bytes, int ntr, int be,
                   const int *d_ints, const SpectraArgs &a, float *d_re,
                   float *d_im, cudaStream_t s) {
  if (ntr <= 0) return QPSDM_OK;
  FftPlan p;
  std::string err;
  int rc = fft_plan(a.nsb, &p, &err);
  if (rc) return rc;
  const size_t sm = fft_smem_bytes(p.m);
  if ((rc = fft_set_smem_attr((const void *)k_spectra, sm))) return rc;
  k_spectra<<<dim3(ntr, 2), 256, sm, s>>>(d_rec, rec_bytes, be, d_ints, a, p, d_re, d_im);
  return cudaGetLastError() == cudaSuccess ? QPSDM_OK : QPSDM_ECUDA;
}

// ---------------------------------------------------------------------------
// Stub imaging: one thread per image point, traces in submission order.
// ---------------------------------------------------------------------------
constexpr int kCompatBz = 32, kCompatBx = 8, kCompatChunk = 256;

__global__ void __launch_bounds__(kCompatBz *kCompatBx)
    k_image_compat(float *__restrict__ img, CompatImageArgs a,
                   const float *__restrict__ dips, const int *__restrict__ ints,
                   const float *__restrict__ geom, int ntr,
                   unsigned long long *npt) {
  __shared__ float4 s_geom[kCompatChunk];
  __shared__ int4 s_rng[kCompatChunk];  // ixi1, ixi2, izimin, accepted
  __shared__ unsigned long long s_cnt;
  const int tid = threadIdx.y * kCompatBz + threadIdx.x;
  const int izi = blockIdx.x * kCompatBz + threadIdx.x;
  const int ixb = blockIdx.y * kCompatBx + threadIdx.y;
  const bool live = izi < a.nzi && ixb < a.nxb;
  const int ixi = ixb + a.ixstart;
  if (tid == 0) s_cnt = 0;

  float tanx1 = 0.f, tanx2 = 0.f, tany1 = 0.f, tany2 = 0.f;
  float acc = 0.0f;
  const bool in_table = ixi >= a.tcdp1 && ixi <= a.tcdp2;
  if (live) {
    const size_t k = (size_t)ixi * a.nzi + izi;
    tanx1 = dips[k];
    tanx2 = dips[a.nxz + k];
    tany1 = dips[2 * a.nxz + k];
    tany2 = dips[3 * a.nxz + k];
    acc = img[(size_t)ixb * a.nzi + izi];
  }
  // Per-point constants of image_depth_gpu (src/q-psdm.cu:2303-2330).
  const float tz = a.taperzone;
  const float tanx1c = __fsub_rn(tanx1, __fmul_rn(tz, __fadd_rn(1.0f, __fmul_rn(tanx1, tanx1))));
  const float tanx2c = __fadd_rn(tanx2, __fmul_rn(tz, __fadd_rn(1.0f, __fmul_rn(tanx2, tanx2))));
  const float tany1c = __fsub_rn(tany1, __fmul_rn(tz, __fadd_rn(1.0f, __fmul_rn(tany1, tany1))));
  const float tany2c = __fadd_rn(tany2, __fmul_rn(tz, __fadd_rn(1.0f, __fmul_rn(tany2, tany2))));
  const float z = __fmul_rn((float)izi, a.dzi);
  const float z2 = __fmul_rn(z, z);
  const float x = __fmul_rn((float)ixi, a.dxi);
  // ts = tg = 1 in the reference: t, the sample indices and v are constants.
  const float ts = 1.0f, tg = 1.0f;
  const float t = __fadd_rn(ts, tg);
  const int it1 = __float2int_rz(__fdiv_rn(t, a.dt1));
  const bool t_ok = it1 > 0 && it1 + 1 < a.nt;
  const float v0 = ((double)t > 0.1) ? __fdiv_rn(100.0f, __fmul_rn(t, t))
                                     : __fmul_rn(100.0f, 100.0f);
  unsigned cnt = 0;

  for (int c0 = 0; c0 < ntr; c0 += kCompatChunk) {
    const int nc = min(kCompatChunk, ntr - c0);
    __syncthreads();
    for (int i = tid; i < nc; i += blockDim.x * blockDim.y) {
      const int *q = ints + (size_t)(c0 + i) * kGateInts;
      const float *gq = geom + (size_t)(c0 + i) * kGateF;
      s_rng[i] = make_int4(q[4], q[5], q[7], q[0] == kAccepted);
      s_geom[i] = make_float4(gq[0], gq[1], gq[2], gq[3]);
    }
    __syncthreads();
    if (!live || !in_table) continue;
    for (int i = 0; i < nc; ++i) {
      const int4 rg = s_rng[i];
      if (!rg.w || ixi < rg.x || ixi > rg.y || izi < rg.z) continue;
      ++cnt;
      const float4 gm = s_geom[i];
      const float dsx = __fsub_rn(gm.x, x), dgx = __fsub_rn(gm.z, x);
      const float ds = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(dsx, dsx), __fmul_rn(gm.y, gm.y)), z2));
      const float dg = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(dgx, dgx), __fmul_rn(gm.w, gm.w)), z2));
      const float ux = __fadd_rn(__fdiv_rn(dsx, ds), __fdiv_rn(dgx, dg));
      const float uy = __fadd_rn(__fdiv_rn(gm.y, ds), __fdiv_rn(gm.w, dg));
      const float uz = __fadd_rn(__fdiv_rn(z, ds), __fdiv_rn(z, dg));
      const float tanx = __fdiv_rn(ux, uz), tany = __fdiv_rn(uy, uz);
      // The reference rejects `tanx <= tanx1c || tanx2c <= tanx || ...`; the
      // negated form agrees for every number and also rejects a NaN tangent
      // (0/0 at z = 0 for collinear source, receiver and node), as the
      // reference binary does: its approximate divisions give +-inf there.
      if (!(tanx > tanx1c && tanx < tanx2c && tany > tany1c && tany < tany2c)) continue;
      float w = 1.0f;
      if (tanx < tanx1) w = __fmul_rn(w, __fdiv_rn(__fsub_rn(tanx, tanx1c), __fsub_rn(tanx1, tanx1c)));
      if (tanx > tanx2) w = __fmul_rn(w, __fdiv_rn(__fsub_rn(tanx2c, tanx), __fsub_rn(tanx2c, tanx2)));
      if (tany < tany1) w = __fmul_rn(w, __fdiv_rn(__fsub_rn(tany, tany1c), __fsub_rn(tany1, tany1c)));
      if (tany > tany2) w = __fmul_rn(w, __fdiv_rn(__fsub_rn(tany2c, tany), __fsub_rn(tany2c, tany2)));
      if (!t_ok) continue;
      // tr = ds/dg*ds/dg*ds/dg*tg/ts, evaluated left to right.
      float r = __fdiv_rn(ds, dg);
      r = __fdiv_rn(__fmul_rn(r, ds), dg);
      r = __fdiv_rn(__fmul_rn(r, ds), dg);
      r = __fdiv_rn(__fmul_rn(r, tg), ts);
      const double rd = (double)r;
      r = __double2float_rn(__dmul_rn((double)w, __dadd_rn(rd, __ddiv_rn(1.0, rd))));
      acc = __fadd_rn(acc, __fmul_rn(v0, r));
    }
  }
  if (live) img[(size_t)ixb * a.nzi + izi] = acc;
  if (npt) {
    // warp-aggregate the point-trace count
    for (int off = 16; off > 0; off >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, off);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(&s_cnt, (unsigned long long)cnt);
    __syncthreads();
    if (tid == 0 && s_cnt) atomicAdd(npt, s_cnt);
  }
}

int launch_image_compat(float *d_img, const CompatImageArgs &a,
                        const float *d_dips, const int *d_ints,
                        const float *d_geom, int ntr, unsigned long long *d_npt,
                        cudaStream_t s) {
  if (ntr <= 0) return QPSDM_OK;
  dim3 block(kCompatBz, kCompatBx);
  dim3 grid((a.nzi + kCompatBz - 1) / kCompatBz, (a.nxb + kCompatBx - 1) / kCompatBx);
  k_image_compat<<<grid, block, 0, s>>>(d_img, a, d_dips, d_ints, d_geom, ntr, d_npt);
  return cudaGetLastError() == cudaSuccess ? QPSDM_OK : QPSDM_ECUDA;
}

}  // namespace qpsdm
