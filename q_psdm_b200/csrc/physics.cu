// physics.cu -- Q-compensated imaging (physics mode) on sm_100a.
//
// The reference's kernel stages per-trace spectra, Q, nf3, the gain-limit
// constants and the ttt/qqq tables (src/q-psdm.cu:2246-2300) but stubs the
// imaging itself (ts = tg = 1, :2350-2351).  This mode computes what those
// inputs describe:
//
//   panels   per accepted trace: t^2 gain + end tapers (as psdm_kernel,
//            :2176-2183), r2c of length nfft, the -i*w band ramp ww of
//            qpsdm() (:1207-1250), the inverse-Q filter
//            A(pi f t*) exp(-2 i f t* ln(f/fc)) with the gain-limit law of
//            lnG/coef1..4 (:1277-1283) for nbins t* values, then c2r of length
//            nffti (the resampled grid dt1, :1201-1206).  The filter table is
//            evaluated once per engine on the host in double precision.
//   image    per image point and trace: traveltime and t* from the tables
//            (bilinear in surface position, linear in depth), t = ts + tg,
//            t* = t*s + t*g, linear interpolation in time and between the two
//            nearest t* panels, the reference's amplitude and dip weights
//            (:2303-2378), accumulated in FP32 (optionally Kahan).
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <math.h>

#include <cmath>
#include <vector>

#include "common.cuh"
#include "fft.cuh"
#include "internal.h"
#include "physics.h"

namespace qpsdm {

struct PhysicsState {
  int nfft = 0, nffti = 0, nbins = 0, max_batch = 0, dtype = 0;
  float dtstar = 0.0f;
  float2 *d_filter = nullptr;  // [nbins][nfft/2+1]
  float2 *d_spec = nullptr;    // [max_batch][nfft/2+1]
  void *d_panels = nullptr;    // [max_batch][nbins][nffti]
  float *d_comp = nullptr;     // Kahan compensation, [img_cap]
  size_t comp_cap = 0;
  // line tables
  qpsdm_ttt_desc *d_desc_t = nullptr, *d_desc_q = nullptr;
  float *d_ttt = nullptr, *d_qqq = nullptr;
  size_t desc_cap = 0, ttt_cap = 0, qqq_cap = 0;
  bool have_tables = false;
};

static size_t dtype_bytes(int t) { return t == QPSDM_PANEL_FP32 ? 4 : 2; }

// (-i ww_k) * A(pi f t*) * exp(-2 i f t* ln(f/fc)) / nfft for every bin.
static void filter_table(const qpsdm_static_params &p, int nbins, float dtstar,
                         std::vector<float2> &out) {
  const int nk = p.nfft / 2 + 1;
  const double df = 1.0 / ((double)p.nfft * (double)p.dt);
  const double dw = 2.0 * M_PI * df;
  const int n3 = (int)(p.f3 / df + 0.5), n4 = (int)(p.f4 / df + 0.5);
  const double G = p.threshold, lnG = std::log(G);
  const double c1 = G * (1.0 - lnG - 2.5 * lnG * lnG), c2 = G * (1.0 + 5.0 * lnG);
  const double c3 = -2.5 * G, c4 = 1.1 * G;
  out.assign((size_t)nbins * nk, make_float2(0.f, 0.f));
  for (int b = 0; b < nbins; ++b) {
    const double ts = b * (double)dtstar;
    for (int k = 1; k < nk; ++k) {
      double ww;
      if (k < n3)
        ww = k * dw;
      else if (k < n4)
        ww = n3 * dw * std::pow(std::cos((double)(k - n3) / (n4 - n3) * M_PI * 0.5), 2);
      else
        ww = 0.0;
      const double f = k * df;
      const double x = M_PI * f * ts;
      double a;
      if (x <= lnG)
        a = std::exp(x);
      else if (x <= lnG + 0.2)
        a = c1 + c2 * x + c3 * x * x;
      else
        a = c4;
      const double ph = -2.0 * f * ts * std::log(f / p.fc);
      // (-i ww) * a * (cos ph + i sin ph) / nfft
      const double re = ww * a * std::sin(ph) / p.nfft;
      const double im = -ww * a * std::cos(ph) / p.nfft;
      out[(size_t)b * nk + k] = make_float2((float)re, (float)im);
    }
  }
}

int physics_create(PhysicsState **out, const qpsdm_static_params &p, std::string *err) {
  *out = nullptr;
  if (p.nbins < 2 || p.nbins > 256 || p.dtstar <= 0.0f) {
    if (err) *err = "physics mode needs 2 <= nbins <= 256 and dtstar > 0";
    return QPSDM_EINVAL;
  }
  if (p.panel_dtype < 0 || p.panel_dtype > 2) {
    if (err) *err = "bad panel dtype";
    return QPSDM_EINVAL;
  }
  auto *s = new PhysicsState;
  s->nfft = p.nfft;
  s->nffti = p.nffti;
  s->nbins = p.nbins;
  s->dtstar = p.dtstar;
  s->max_batch = p.max_batch;
  s->dtype = p.panel_dtype;
  std::vector<float2> f;
  filter_table(p, p.nbins, p.dtstar, f);
  const size_t nk = (size_t)p.nfft / 2 + 1;
  auto bad = [&](const char *w) {
    if (err) *err = std::string("physics_create: ") + w;
    physics_destroy(s);
    return QPSDM_ENOMEM;
  };
  if (cudaMalloc(&s->d_filter, sizeof(float2) * f.size()) != cudaSuccess) return bad("filter");
  cudaMemcpy(s->d_filter, f.data(), sizeof(float2) * f.size(), cudaMemcpyHostToDevice);
  if (cudaMalloc(&s->d_spec, sizeof(float2) * nk * p.max_batch) != cudaSuccess) return bad("spectra");
  const size_t pb = dtype_bytes(p.panel_dtype) * (size_t)p.nbins * p.nffti * p.max_batch;
  if (cudaMalloc(&s->d_panels, pb) != cudaSuccess) return bad("panels");
  *out = s;
  return QPSDM_OK;
}

void physics_destroy(PhysicsState *s) {
  if (!s) return;
  cudaFree(s->d_filter);
  cudaFree(s->d_spec);
  cudaFree(s->d_panels);
  cudaFree(s->d_comp);
  cudaFree(s->d_desc_t);
  cudaFree(s->d_desc_q);
  cudaFree(s->d_ttt);
  cudaFree(s->d_qqq);
  delete s;
}

template <typename T>
static bool grow_dev(T **p, size_t *cap, size_t need) {
  if (*p && *cap >= need) return true;
  cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  if (cudaMalloc((void **)p, sizeof(T) * (need ? need : 1)) != cudaSuccess) return false;
  *cap = need;
  return true;
}

int physics_set_line(PhysicsState *s, const qpsdm_static_params &p,
                     const qpsdm_line_params &l, cudaStream_t st, std::string *err) {
  if (!l.ttt_desc || !l.qqq_desc || !l.ttt || !l.qqq || l.nxg <= 0 || l.nzg <= 0 ||
      l.nxi1 <= 0 || l.nzi1 <= 0) {
    if (err) *err = "physics mode needs ttt and qqq tables";
    return QPSDM_EINVAL;
  }
  if (l.ttt_cdp1 > l.ttt_cdp2) {
    if (err) *err = "travel time table cdp range error";  // src/q-psdm.cu:1455-1461
    return QPSDM_EINVAL;
  }
  const size_t ncell = (size_t)l.nxg * l.nzg;
  // every descriptor's block must lie inside its data array
  for (int w = 0; w < 2; ++w) {
    const qpsdm_ttt_desc *d = w ? l.qqq_desc : l.ttt_desc;
    const int64_t len = w ? l.qqq_len : l.ttt_len;
    for (size_t c = 0; c < ncell; ++c) {
      const int64_t blk = (int64_t)d[c].nys * d[c].nxs * l.nxi1 * l.nzi1;
      if (d[c].idx < 0 || d[c].nys == 0 || d[c].nxs == 0 || d[c].dys == 0 ||
          d[c].dxs == 0 || d[c].idx + blk > len) {
        if (err) *err = "table descriptor outside its data (or empty surface grid)";
        return QPSDM_EINVAL;
      }
    }
  }
  size_t dc = s->desc_cap, dq = s->desc_cap;
  if (!grow_dev(&s->d_desc_t, &dc, ncell) || !grow_dev(&s->d_desc_q, &dq, ncell) ||
      !grow_dev(&s->d_ttt, &s->ttt_cap, (size_t)l.ttt_len) ||
      !grow_dev(&s->d_qqq, &s->qqq_cap, (size_t)l.qqq_len)) {
    if (err) *err = "table allocation failed";
    return QPSDM_ENOMEM;
  }
  s->desc_cap = dc < dq ? dc : dq;
  cudaMemcpyAsync(s->d_desc_t, l.ttt_desc, sizeof(qpsdm_ttt_desc) * ncell,
                  cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s->d_desc_q, l.qqq_desc, sizeof(qpsdm_ttt_desc) * ncell,
                  cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s->d_ttt, l.ttt, sizeof(float) * l.ttt_len, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s->d_qqq, l.qqq, sizeof(float) * l.qqq_len, cudaMemcpyHostToDevice, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) {
    if (err) *err = "table upload failed";
    return QPSDM_ECUDA;
  }
  s->have_tables = true;
  (void)p;
  return QPSDM_OK;
}

int physics_begin_offset(PhysicsState *s, const qpsdm_static_params &p,
                         const qpsdm_offset_params &o, cudaStream_t st, std::string *err) {
  if (p.kahan) {
    const size_t n = (size_t)(o.ixend - o.ixstart) * p.nzi;
    if (!grow_dev(&s->d_comp, &s->comp_cap, n)) {
      if (err) *err = "compensation buffer allocation failed";
      return QPSDM_ENOMEM;
    }
    cudaMemsetAsync(s->d_comp, 0, sizeof(float) * n, st);
  }
  return QPSDM_OK;
}

// ---------------------------------------------------------------------------
// panels
// ---------------------------------------------------------------------------
__device__ __forceinline__ float phys_tapered(float v, int j, int n, const float *tap) {
  const int head = j, tail = n - 1 - j;
  if (head < 200 && tail < 200) {
    if (head <= tail) return __fmul_rn(__fmul_rn(v, tap[head]), tap[tail]);
    return __fmul_rn(__fmul_rn(v, tap[tail]), tap[head]);
  }
  if (head < 200) return __fmul_rn(v, tap[head]);
  if (tail < 200) return __fmul_rn(v, tap[tail]);
  return v;
}

__global__ void __launch_bounds__(256) k_phys_fwd(const uint8_t *__restrict__ rec, int rec_bytes,
                                                  int be, const int *__restrict__ ints, int ntl,
                                                  float dt, const float *__restrict__ tap,
                                                  FftPlan p, float2 *__restrict__ spec) {
  const int itr = blockIdx.x;
  if (ints[(size_t)itr * kGateInts] != kAccepted) return;
  extern __shared__ float2 sm[];
  float2 *b0 = sm, *b1 = sm + p.m, *twm = sm + 2 * p.m, *twn = sm + 3 * p.m;
  for (int i = threadIdx.x; i < p.m; i += blockDim.x) twm[i] = p.tw_m[i];
  for (int i = threadIdx.x; i <= p.m; i += blockDim.x) twn[i] = p.tw_n[i];
  const uint8_t *r = rec + (size_t)itr * rec_bytes;
  float *bf = reinterpret_cast<float *>(b0);
  for (int j = threadIdx.x; j < p.n; j += blockDim.x) {
    float v = 0.0f;
    if (j < ntl) {
      v = su_sample(r, j, be);
      const float t = __fmul_rn((float)j, dt);
      v = ((double)t < 0.1) ? __double2float_rn(__dmul_rn((double)v, 0.1 * 0.1))
                            : __fmul_rn(v, __fmul_rn(t, t));
      v = phys_tapered(v, j, ntl, tap);
    }
    bf[j] = v;
  }
  __syncthreads();
  const int cur = fft_complex_smem(b0, b1, p, twm, false);
  const float2 *Z = cur ? b1 : b0;
  float2 *o = spec + (size_t)itr * (p.m + 1);
  for (int k = threadIdx.x; k <= p.m; k += blockDim.x) o[k] = rfft_bin(Z, twn, p.m, k);
}

template <typename T>
__device__ __forceinline__ void store_sample(T *dst, float v);
template <>
__device__ __forceinline__ void store_sample<float>(float *d, float v) { *d = v; }
template <>
__device__ __forceinline__ void store_sample<__nv_bfloat16>(__nv_bfloat16 *d, float v) {
  *d = __float2bfloat16_rn(v);
}
template <>
__device__ __forceinline__ void store_sample<__half>(__half *d, float v) { *d = __float2half_rn(v); }

// One CTA per (trace, t* bin): filtered, zero-padded spectrum -> c2r nffti.
template <typename T>
__global__ void __launch_bounds__(256) k_phys_panels(const int *__restrict__ ints,
                                                     const float2 *__restrict__ spec, int nk,
                                                     const float2 *__restrict__ filt, FftPlan p,
                                                     int nbins, T *__restrict__ panels) {
  const int itr = blockIdx.x, b = blockIdx.y;
  if (ints[(size_t)itr * kGateInts] != kAccepted) return;
  extern __shared__ float2 sm[];
  float2 *b0 = sm, *b1 = sm + p.m, *twm = sm + 2 * p.m, *twn = sm + 3 * p.m;
  for (int i = threadIdx.x; i < p.m; i += blockDim.x) twm[i] = p.tw_m[i];
  for (int i = threadIdx.x; i <= p.m; i += blockDim.x) twn[i] = p.tw_n[i];
  __syncthreads();
  const float2 *X = spec + (size_t)itr * nk;
  const float2 *F = filt + (size_t)b * nk;
  for (int k = threadIdx.x; k < p.m; k += blockDim.x) {
    // Y[k] and Y[m-k] of the zero-padded filtered spectrum
    const int k2 = p.m - k;
    const float2 a = k < nk ? cmul(X[k], F[k]) : make_float2(0.f, 0.f);
    const float2 c = k2 < nk ? cmul(X[k2], F[k2]) : make_float2(0.f, 0.f);
    const float2 bb = cconj(c);
    const float2 e = make_float2(0.5f * (a.x + bb.x), 0.5f * (a.y + bb.y));
    const float2 d = make_float2(0.5f * (a.x - bb.x), 0.5f * (a.y - bb.y));
    const float2 o = cmul(d, cconj(twn[k]));
    b0[k] = make_float2(e.x - o.y, e.y + o.x);
  }
  __syncthreads();
  const int cur = fft_complex_smem(b0, b1, p, twm, true);
  const float2 *z = cur ? b1 : b0;
  T *out = panels + ((size_t)itr * nbins + b) * p.n;
  for (int j = threadIdx.x; j < p.m; j += blockDim.x) {
    store_sample<T>(out + 2 * j, 2.0f * z[j].x);
    store_sample<T>(out + 2 * j + 1, 2.0f * z[j].y);
  }
}

// ---------------------------------------------------------------------------
// plain imaging
// ---------------------------------------------------------------------------
struct PhysImageArgs {
  int nzi, nxb, ixstart, nt, nbins;
  float dt1, dxi, dzi, taperzone, dtstar, dzii;
  int tcdp1, tcdp2;  // relative to fci
  int nxg, nzg, nxi1, nzi1;
  size_t nxz;
};

template <typename T>
__device__ __forceinline__ float ld_sample(const T *p);
template <>
__device__ __forceinline__ float ld_sample<float>(const float *p) { return __ldg(p); }
template <>
__device__ __forceinline__ float ld_sample<__nv_bfloat16>(const __nv_bfloat16 *p) {
  return __bfloat162float(*p);
}
template <>
__device__ __forceinline__ float ld_sample<__half>(const __half *p) { return __half2float(*p); }

// Table value at one depth node of a cell for surface point (px, py).
// Returns false outside the cell's surface grid.
__device__ __forceinline__ bool table_node(const qpsdm_ttt_desc &d, const float *__restrict__ tab,
                                           float px, float py, float xc, int ixl, int izl,
                                           int nxi1, int nzi1, float &v) {
  const int nxs = d.nxs, nys = d.nys;
  const float fx = (px - xc) / (float)d.dxs + 0.5f * (nxs - 1);
  const float fy = py / (float)d.dys + 0.5f * (nys - 1);
  if (!(fx >= 0.0f && fx <= (float)(nxs - 1) && fy >= 0.0f && fy <= (float)(nys - 1)))
    return false;
  int ix = min((int)fx, max(nxs - 2, 0));
  int iy = min((int)fy, max(nys - 2, 0));
  const float wx = nxs > 1 ? fx - ix : 0.0f, wy = nys > 1 ? fy - iy : 0.0f;
  const int64_t sx = nxs > 1 ? (int64_t)nxi1 * nzi1 : 0;
  const int64_t sy = nys > 1 ? (int64_t)nxs * nxi1 * nzi1 : 0;
  const int64_t base = d.idx + ((int64_t)(iy * nxs + ix) * nxi1 + ixl) * nzi1 + izl;
  const float v00 = __ldg(tab + base), v01 = __ldg(tab + base + sx);
  const float v10 = __ldg(tab + base + sy), v11 = __ldg(tab + base + sy + sx);
  const float a = v00 + wx * (v01 - v00), b = v10 + wx * (v11 - v10);
  v = a + wy * (b - a);
  return true;
}

struct PointCells {
  bool ok;
  int ixl, izlA, izlB;
  float c2, xc;
  qpsdm_ttt_desc tA, tB, qA, qB;
};

__device__ __forceinline__ bool lookup_tq(const PointCells &pc, const float *__restrict__ ttt,
                                          const float *__restrict__ qqq, int nxi1, int nzi1,
                                          float px, float py, float &t, float &q) {
  float ta, tb, qa, qb;
  if (!table_node(pc.tA, ttt, px, py, pc.xc, pc.ixl, pc.izlA, nxi1, nzi1, ta)) return false;
  if (!table_node(pc.tB, ttt, px, py, pc.xc, pc.ixl, pc.izlB, nxi1, nzi1, tb)) return false;
  if (!table_node(pc.qA, qqq, px, py, pc.xc, pc.ixl, pc.izlA, nxi1, nzi1, qa)) return false;
  if (!table_node(pc.qB, qqq, px, py, pc.xc, pc.ixl, pc.izlB, nxi1, nzi1, qb)) return false;
  t = ta + pc.c2 * (tb - ta);
  q = qa + pc.c2 * (qb - qa);
  return true;
}

constexpr int kPhysBz = 32, kPhysBx = 8, kPhysChunk = 256;

template <typename T>
__global__ void __launch_bounds__(kPhysBz *kPhysBx)
    k_image_plain(float *__restrict__ img, float *__restrict__ comp, PhysImageArgs a,
                  const float *__restrict__ dips, const int *__restrict__ ints,
                  const float *__restrict__ geom, int ntr,
                  const qpsdm_ttt_desc *__restrict__ dt, const float *__restrict__ ttt,
                  const qpsdm_ttt_desc *__restrict__ dq, const float *__restrict__ qqq,
                  const T *__restrict__ panels, unsigned long long *npt) {
  __shared__ float4 s_geom[kPhysChunk];
  __shared__ int4 s_rng[kPhysChunk];
  __shared__ unsigned long long s_cnt;
  const int tid = threadIdx.y * kPhysBz + threadIdx.x;
  const int izi = blockIdx.x * kPhysBz + threadIdx.x;
  const int ixb = blockIdx.y * kPhysBx + threadIdx.y;
  const bool live = izi < a.nzi && ixb < a.nxb;
  const int ixi = ixb + a.ixstart;
  if (tid == 0) s_cnt = 0;

  // per-point constants: cells, depth weights, dip limits
  PointCells pc;
  pc.ok = false;
  float tanx1 = 0.f, tanx2 = 0.f, tany1 = 0.f, tany2 = 0.f, acc = 0.f, cmp = 0.f;
  const float z = izi * a.dzi;
  if (live) {
    const size_t k = (size_t)ixi * a.nzi + izi;
    tanx1 = dips[k];
    tanx2 = dips[a.nxz + k];
    tany1 = dips[2 * a.nxz + k];
    tany2 = dips[3 * a.nxz + k];
    acc = img[(size_t)ixb * a.nzi + izi];
    if (comp) cmp = comp[(size_t)ixb * a.nzi + izi];
    const int lx = ixi - a.tcdp1;
    if (ixi >= a.tcdp1 && ixi <= a.tcdp2) {
      const int ixg = lx / a.nxi1;
      pc.ixl = lx - ixg * a.nxi1;
      const float fz = z / a.dzii;
      const int izn = (int)fz;
      pc.c2 = fz - (float)izn;
      int izgA = izn / a.nzi1, izgB = (izn + 1) / a.nzi1;
      pc.izlA = izn - izgA * a.nzi1;
      pc.izlB = izn + 1 - izgB * a.nzi1;
      if (izgB >= a.nzg) {  // deepest node: no lower neighbour
        izgB = izgA;
        pc.izlB = pc.izlA;
        pc.c2 = 0.0f;
      }
      if (ixg < a.nxg && izgA < a.nzg) {
        pc.ok = true;
        pc.tA = dt[ixg * a.nzg + izgA];
        pc.tB = dt[ixg * a.nzg + izgB];
        pc.qA = dq[ixg * a.nzg + izgA];
        pc.qB = dq[ixg * a.nzg + izgB];
        pc.xc = (a.tcdp1 + ixg * a.nxi1 + 0.5f * (a.nxi1 - 1)) * a.dxi;
      }
    }
  }
  const float tz = a.taperzone;
  const float tanx1c = tanx1 - tz * (1.0f + tanx1 * tanx1);
  const float tanx2c = tanx2 + tz * (1.0f + tanx2 * tanx2);
  const float tany1c = tany1 - tz * (1.0f + tany1 * tany1);
  const float tany2c = tany2 + tz * (1.0f + tany2 * tany2);
  const float z2 = z * z;
  const float x = ixi * a.dxi;
  const float inv_dt1 = 1.0f / a.dt1, inv_dts = 1.0f / a.dtstar;
  const size_t pstride = (size_t)a.nbins * a.nt;
  // source terms are reused while consecutive traces share a source
  float last_sx = NAN, last_sy = NAN, ts = 0.f, qs = 0.f;
  bool s_ok = false;
  unsigned cnt = 0;

  for (int c0 = 0; c0 < ntr; c0 += kPhysChunk) {
    const int nc = min(kPhysChunk, ntr - c0);
    __syncthreads();
    for (int i = tid; i < nc; i += blockDim.x * blockDim.y) {
      const int *q = ints + (size_t)(c0 + i) * kGateInts;
      const float *gq = geom + (size_t)(c0 + i) * kGateF;
      s_rng[i] = make_int4(q[4], q[5], q[7], q[0] == kAccepted);
      s_geom[i] = make_float4(gq[0], gq[1], gq[2], gq[3]);
    }
    __syncthreads();
    if (!live || !pc.ok) continue;
    for (int i = 0; i < nc; ++i) {
      const int4 rg = s_rng[i];
      if (!rg.w || ixi < rg.x || ixi > rg.y || izi < rg.z) continue;
      ++cnt;
      const float4 gm = s_geom[i];
      if (gm.x != last_sx || gm.y != last_sy) {
        last_sx = gm.x;
        last_sy = gm.y;
        s_ok = lookup_tq(pc, ttt, qqq, a.nxi1, a.nzi1, gm.x, gm.y, ts, qs);
      }
      if (!s_ok) continue;
      float tg, qg;
      if (!lookup_tq(pc, ttt, qqq, a.nxi1, a.nzi1, gm.z, gm.w, tg, qg)) continue;
      // ray directions and dip taper (src/q-psdm.cu:2303-2340)
      const float dsx = gm.x - x, dgx = gm.z - x;
      const float ds = sqrtf(dsx * dsx + gm.y * gm.y + z2);
      const float dg = sqrtf(dgx * dgx + gm.w * gm.w + z2);
      const float rs = 1.0f / ds, rg2 = 1.0f / dg;
      const float ux = dsx * rs + dgx * rg2, uy = gm.y * rs + gm.w * rg2, uz = z * (rs + rg2);
      const float tanx = ux / uz, tany = uy / uz;
      if (!(tanx > tanx1c && tanx < tanx2c && tany > tany1c && tany < tany2c)) continue;
      float w = 1.0f;
      if (tanx < tanx1) w *= (tanx - tanx1c) / (tanx1 - tanx1c);
      if (tanx > tanx2) w *= (tanx2c - tanx) / (tanx2c - tanx2);
      if (tany < tany1) w *= (tany - tany1c) / (tany1 - tany1c);
      if (tany > tany2) w *= (tany2c - tany) / (tany2c - tany2);
      // time and t* picks
      const float t = ts + tg;
      const float ft = t * inv_dt1;
      const int it1 = (int)ft;
      if (!(it1 > 0 && it1 + 1 < a.nt)) continue;
      const float wt = ft - (float)it1;
      float fb = fminf(fmaxf((qs + qg) * inv_dts, 0.0f), (float)(a.nbins - 1));
      const int b0 = min((int)fb, a.nbins - 2);
      const float wb = fb - (float)b0;
      const T *pp = panels + (size_t)(c0 + i) * pstride + (size_t)b0 * a.nt + it1;
      const float p00 = ld_sample<T>(pp), p01 = ld_sample<T>(pp + 1);
      const float p10 = ld_sample<T>(pp + a.nt), p11 = ld_sample<T>(pp + a.nt + 1);
      const float s0 = p00 + wt * (p01 - p00), s1 = p10 + wt * (p11 - p10);
      const float smp = s0 + wb * (s1 - s0);
      // amplitude weight (src/q-psdm.cu:2366-2374)
      const float v = t > 0.1f ? 100.0f / (t * t) : 10000.0f;
      const float r = (ds * rg2) * (ds * rg2) * (ds * rg2) * (tg / ts);
      const float val = w * (r + 1.0f / r) * v * smp;
      if (comp) {  // Kahan-compensated sum
        const float y = val - cmp;
        const float tt = acc + y;
        cmp = (tt - acc) - y;
        acc = tt;
      } else {
        acc += val;
      }
    }
  }
  if (live) {
    img[(size_t)ixb * a.nzi + izi] = acc;
    if (comp) comp[(size_t)ixb * a.nzi + izi] = cmp;
  }
  if (npt) {
    for (int off = 16; off > 0; off >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, off);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(&s_cnt, (unsigned long long)cnt);
    __syncthreads();
    if (tid == 0 && s_cnt) atomicAdd(npt, s_cnt);
  }
}

int physics_process(PhysicsState *s, const qpsdm_static_params &p,
                    const qpsdm_line_params &l, const qpsdm_offset_params &o,
                    const PhysicsBatch &b, cudaStream_t st, std::string *err) {
  if (!s->have_tables) {
    if (err) *err = "physics mode: set_line without tables";
    return QPSDM_ESTATE;
  }
  const int ntr = b.ntr;
  // 1. forward spectra
  FftPlan pf, pi;
  int rc = fft_plan(p.nfft, &pf, err);
  if (rc) return rc;
  rc = fft_plan(p.nffti, &pi, err);
  if (rc) return rc;
  size_t sm = fft_smem_bytes(pf.m);
  if ((rc = fft_set_smem_attr((const void *)k_phys_fwd, sm))) return rc;
  b.prof->begin(QPSDM_K_PRE, st);
  k_phys_fwd<<<ntr, 256, sm, st>>>(b.d_rec, b.rec_bytes, b.big_endian, b.d_ints, p.ntl, p.dt,
                                   b.d_taper200, pf, s->d_spec);
  // 2. t*-binned panels
  const int nk = p.nfft / 2 + 1;
  sm = fft_smem_bytes(pi.m);
  dim3 gp(ntr, s->nbins);
  switch (s->dtype) {
    case QPSDM_PANEL_FP32:
      if ((rc = fft_set_smem_attr((const void *)k_phys_panels<float>, sm))) return rc;
      k_phys_panels<float><<<gp, 256, sm, st>>>(b.d_ints, s->d_spec, nk, s->d_filter, pi,
                                                s->nbins, (float *)s->d_panels);
      break;
    case QPSDM_PANEL_BF16:
      if ((rc = fft_set_smem_attr((const void *)k_phys_panels<__nv_bfloat16>, sm))) return rc;
      k_phys_panels<__nv_bfloat16><<<gp, 256, sm, st>>>(b.d_ints, s->d_spec, nk, s->d_filter,
                                                        pi, s->nbins,
                                                        (__nv_bfloat16 *)s->d_panels);
      break;
    default:
      if ((rc = fft_set_smem_attr((const void *)k_phys_panels<__half>, sm))) return rc;
      k_phys_panels<__half><<<gp, 256, sm, st>>>(b.d_ints, s->d_spec, nk, s->d_filter, pi,
                                                 s->nbins, (__half *)s->d_panels);
  }
  b.prof->end(st);
  // 3. image
  PhysImageArgs a{};
  a.nzi = p.nzi;
  a.nxb = o.ixend - o.ixstart;
  a.ixstart = o.ixstart;
  a.nt = p.nffti;
  a.nbins = s->nbins;
  a.dt1 = p.dt1;
  a.dxi = p.dxi;
  a.dzi = p.dzi;
  a.taperzone = p.taperzone;
  a.dtstar = s->dtstar;
  a.dzii = p.dzii;
  a.tcdp1 = l.ttt_cdp1 - p.fci;
  a.tcdp2 = l.ttt_cdp2 - p.fci;
  a.nxg = l.nxg;
  a.nzg = l.nzg;
  a.nxi1 = l.nxi1;
  a.nzi1 = l.nzi1;
  a.nxz = b.nxz;
  float *comp = p.kahan ? s->d_comp : nullptr;
  dim3 block(kPhysBz, kPhysBx);
  dim3 grid((a.nzi + kPhysBz - 1) / kPhysBz, (a.nxb + kPhysBx - 1) / kPhysBx);
  b.prof->begin(QPSDM_K_IMAGE, st);
  switch (s->dtype) {
    case QPSDM_PANEL_FP32:
      k_image_plain<float><<<grid, block, 0, st>>>(b.d_img, comp, a, b.d_dips, b.d_ints,
                                                   b.d_geom, ntr, s->d_desc_t, s->d_ttt,
                                                   s->d_desc_q, s->d_qqq,
                                                   (const float *)s->d_panels, b.d_npt);
      break;
    case QPSDM_PANEL_BF16:
      k_image_plain<__nv_bfloat16><<<grid, block, 0, st>>>(
          b.d_img, comp, a, b.d_dips, b.d_ints, b.d_geom, ntr, s->d_desc_t, s->d_ttt,
          s->d_desc_q, s->d_qqq, (const __nv_bfloat16 *)s->d_panels, b.d_npt);
      break;
    default:
      k_image_plain<__half><<<grid, block, 0, st>>>(
          b.d_img, comp, a, b.d_dips, b.d_ints, b.d_geom, ntr, s->d_desc_t, s->d_ttt,
          s->d_desc_q, s->d_qqq, (const __half *)s->d_panels, b.d_npt);
  }
  b.prof->end(st);
  if (cudaGetLastError() != cudaSuccess) {
    if (err) *err = "physics launch failed";
    return QPSDM_ECUDA;
  }
  return QPSDM_OK;
}

int physics_finalize_image(PhysicsState *s, float *d_img, size_t n, cudaStream_t st,
                           std::string *err) {
  (void)s;
  (void)d_img;
  (void)n;
  (void)st;
  (void)err;
  return QPSDM_OK;
}

}  // namespace qpsdm
