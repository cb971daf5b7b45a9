// surrogate.cu -- the learned traveltime / t* surrogate around the tables.
//
// The reference reads precomputed tables only (L<line>.ttt / .qqq,
// src/q-psdm.cu:2382-2627; its kernel stages them and, as a stub, never reads
// them, :2343-2357).  This file connects the network (mlp.cu) to them:
//
//   qpsdm_eikonal_samples   training samples drawn straight from the solved
//                           eikonal grids of a batch of sources (features in
//                           model coordinates, targets the corrections to the
//                           linear-gradient background), so a training set of
//                           sources x volume points is never materialised;
//   qpsdm_surrogate_gate    the network's traveltime error (ms) at every
//                           surface node of a line's tables, max-accumulated;
//   qpsdm_surrogate_tables  tables of a line on any surface grid from the
//                           network, keeping bilinear interpolation of the
//                           given tables wherever a patch's corner nodes
//                           missed by more than the gate.
//
// Table layout: the reference's (descriptor per cell, block
// [iys][ixs][ixl][izl], depth fastest) with the surface grid of a cell centred
// on the cell's middle cdp and on the line (q_psdm_b200/tables.py).
#include <cstring>
#include <vector>

#include "common.cuh"
#include "qpsdm_engine.h"

namespace qpsdm {

__device__ __forceinline__ uint64_t mix64(uint64_t z) {  // splitmix64 finaliser
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

// Exact traveltime (s) of v = v0 + kz z from a surface point, in double.
__device__ __forceinline__ double bg_time(double r, double z, double v0, double kz) {
  if (kz < 1e-9) return sqrt(r * r + z * z) / v0;
  const double v = v0 + kz * z;
  const double arg = 1.0 + kz * kz * (r * r + z * z) / (2.0 * v0 * v);
  return acosh(fmax(arg, 1.0)) / kz;
}

// ---------------------------------------------------------------------------
// training samples from solved grids
// ---------------------------------------------------------------------------
__global__ void k_eik_samples(const float *__restrict__ T, const float *__restrict__ S,
                              const float *__restrict__ Tb, const float *__restrict__ Sb,
                              qpsdm_eik_grid g, const float4 *__restrict__ src, int ns,
                              qpsdm_sur_background bg, uint64_t seed, int nsamples,
                              float *__restrict__ x, float *__restrict__ t) {
  const size_t n = (size_t)g.nx * g.ny * g.nz;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nsamples; k += gridDim.x * blockDim.x) {
    int s = 0;
    size_t j = 0;
    bool ok = false;
    float Tm = 0.f, Sm = 0.f, Tbs = 0.f, Sbs = 0.f;
    for (int a = 0; a < 8 && !ok; ++a) {  // redraw the (rare) unreached nodes
      const uint64_t h = mix64(seed ^ mix64((uint64_t)k * 8 + a));
      s = (int)((h >> 40) % (uint64_t)ns);
      j = (size_t)((h & 0xffffffffffull) % n);
      const size_t i = (size_t)s * n + j;
      Tm = T[i];
      Sm = S[i];
      Tbs = Tb ? Tb[i] : 0.f;
      Sbs = Sb ? Sb[i] : 0.f;
      ok = Tm < 1e29f && (!Tb || (Tbs < 1e29f && Sbs > 0.f));
    }
    const float4 sp = src[s];
    const int ix = (int)(j % g.nx), iy = (int)((j / g.nx) % g.ny);
    const int iz = (int)(j / ((size_t)g.nx * g.ny));
    float px = sp.x, py = sp.y, qx = sp.z + ix * g.h, qy = sp.w + iy * g.h, qz = iz * g.h;
    float y0 = 0.f, y1 = 0.f;
    if (ok) {
      const double r = hypot((double)qx - px, (double)qy - py);
      const double tb = bg_time(r, qz, bg.v0, bg.kz);
      // background-corrected values, as the tables are built
      // (q_psdm_b200/tables.py): T = T_bg + T - T_bgsolve, t* = t* t*_bg / t*_bgsolve
      const double tc = Tb ? tb + ((double)Tm - (double)Tbs) : (double)Tm;
      const double sc = Tb ? (double)Sm * (tb / bg.q_bg) / (double)Sbs : (double)Sm;
      y0 = (float)((tc - tb) * 1e3);
      y1 = (float)((sc - tb / bg.q_ref) * 1e3);
    } else {  // no reached node found: the source point itself (zero correction)
      qx = px, qy = py, qz = 0.f;
    }
    float *o = x + (size_t)k * 5;
    o[0] = px, o[1] = py, o[2] = qx, o[3] = qy, o[4] = qz;
    t[2 * (size_t)k] = y0;
    t[2 * (size_t)k + 1] = y1;
  }
}

// ---------------------------------------------------------------------------
// table elements <-> features
// ---------------------------------------------------------------------------
struct TabView {
  const qpsdm_ttt_desc *desc;   // [ncell]
  const int64_t *cell_base;     // [ncell + 1] prefix sums of block sizes
  const int *node_base;         // [ncell + 1] prefix sums of surface nodes
  int ncell;
};

struct ElemPos {
  int c, iys, ixs, ixl, izl;
  int64_t r;  // offset inside the cell's block
};

__device__ __forceinline__ ElemPos elem_pos(const TabView &v, int64_t e, int nxi1, int nzi1) {
  int lo = 0, hi = v.ncell;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (v.cell_base[mid] <= e) lo = mid; else hi = mid;
  }
  ElemPos p;
  p.c = lo;
  p.r = e - v.cell_base[lo];
  const int per_node = nxi1 * nzi1;
  const int node = (int)(p.r / per_node);
  const int rem = (int)(p.r - (int64_t)node * per_node);
  const int nxs = v.desc[lo].nxs;
  p.iys = node / nxs;
  p.ixs = node - p.iys * nxs;
  p.ixl = rem / nzi1;
  p.izl = rem - p.ixl * nzi1;
  return p;
}

// Model coordinates of the element: surface point (px, py), image point (x, y, z).
__device__ __forceinline__ void elem_feat(const TabView &v, const ElemPos &p,
                                          const qpsdm_sur_line &ln, float f[5]) {
  const qpsdm_ttt_desc d = v.desc[p.c];
  const int ixg = p.c / ln.nzg, izg = p.c - ixg * ln.nzg;
  const float xc = (ln.tcdp1 + ixg * ln.nxi1 + 0.5f * (ln.nxi1 - 1)) * ln.dxi;
  f[0] = xc + (p.ixs - 0.5f * (d.nxs - 1)) * d.dxs;
  f[1] = ln.line_y + (p.iys - 0.5f * (d.nys - 1)) * d.dys;
  f[2] = (ln.tcdp1 + ixg * ln.nxi1 + p.ixl) * ln.dxi;
  f[3] = ln.line_y;
  f[4] = (izg * ln.nzi1 + p.izl) * ln.dzii;
}

__global__ void k_tab_features(TabView v, qpsdm_sur_line ln, int64_t e0, int n,
                               float *__restrict__ x) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const ElemPos p = elem_pos(v, e0 + k, ln.nxi1, ln.nzi1);
    float f[5];
    elem_feat(v, p, ln, f);
    float *o = x + (size_t)k * 5;
#pragma unroll
    for (int j = 0; j < 5; ++j) o[j] = f[j];
  }
}

// Network traveltime (s) and t* (s) of an element from its corrections (ms).
__device__ __forceinline__ void net_values(const float f[5], const float *y,
                                           const qpsdm_sur_line &ln, double &T, double &S) {
  const double r = hypot((double)f[0] - f[2], (double)f[1] - f[3]);
  const double tb = bg_time(r, f[4], ln.v0, ln.kz);
  T = tb + 1e-3 * (double)y[0];
  S = tb / ln.q_ref + 1e-3 * (double)y[1];
}

__global__ void k_gate_err(TabView v, qpsdm_sur_line ln, int64_t e0, int n,
                           const float *__restrict__ y, const float *__restrict__ ttt,
                           float *__restrict__ node_err) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const ElemPos p = elem_pos(v, e0 + k, ln.nxi1, ln.nzi1);
    float f[5];
    elem_feat(v, p, ln, f);
    double T, S;
    net_values(f, y + 2 * (size_t)k, ln, T, S);
    const float err = (float)(fabs(T - (double)ttt[v.desc[p.c].idx + p.r]) * 1e3);
    // non-negative floats order like their bit patterns (NaN: the largest)
    const unsigned u = isnan(err) ? 0x7f800000u : __float_as_uint(err);
    atomicMax(reinterpret_cast<unsigned *>(node_err) + v.node_base[p.c] + p.iys * v.desc[p.c].nxs +
                  p.ixs,
              u);
  }
}

// Fine tables: the network, or bilinear interpolation of the coarse tables in
// the coarse patches whose corner nodes the network missed by > gate_ms.
__global__ void k_sur_tables(TabView fv, TabView cv, qpsdm_sur_line ln, int64_t e0, int n,
                             const float *__restrict__ y, const float *__restrict__ cttt,
                             const float *__restrict__ cqqq, const float *__restrict__ node_err,
                             float gate_ms, float *__restrict__ fttt, float *__restrict__ fqqq,
                             unsigned long long *gated) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const ElemPos p = elem_pos(fv, e0 + k, ln.nxi1, ln.nzi1);
    float f[5];
    elem_feat(fv, p, ln, f);
    // the fine node's place in the same cell's coarse surface grid
    const qpsdm_ttt_desc dc = cv.desc[p.c];
    const int ixg = p.c / ln.nzg;
    const float xc = (ln.tcdp1 + ixg * ln.nxi1 + 0.5f * (ln.nxi1 - 1)) * ln.dxi;
    const float fx = fminf(fmaxf((f[0] - xc) / dc.dxs + 0.5f * (dc.nxs - 1), 0.0f),
                           (float)(dc.nxs - 1));
    const float fy = fminf(fmaxf((f[1] - ln.line_y) / dc.dys + 0.5f * (dc.nys - 1), 0.0f),
                           (float)(dc.nys - 1));
    const int ix = min((int)fx, max(dc.nxs - 2, 0)), iy = min((int)fy, max(dc.nys - 2, 0));
    const int sx = dc.nxs > 1 ? 1 : 0, sy = dc.nys > 1 ? dc.nxs : 0;
    const float *ne = node_err + cv.node_base[p.c] + iy * dc.nxs + ix;
    const float worst = fmaxf(fmaxf(ne[0], ne[sx]), fmaxf(ne[sy], ne[sy + sx]));
    const int64_t fo = fv.desc[p.c].idx + p.r;
    if (!(worst <= gate_ms)) {  // NaN errors keep the tables too
      const float wx = dc.nxs > 1 ? fx - ix : 0.f, wy = dc.nys > 1 ? fy - iy : 0.f;
      const int64_t plane = (int64_t)ln.nxi1 * ln.nzi1;
      const int64_t b = dc.idx + (int64_t)(iy * dc.nxs + ix) * plane + p.ixl * ln.nzi1 + p.izl;
      const int64_t ox = sx * plane, oy = (int64_t)sy * plane;
      const float *tab[2] = {cttt, cqqq};
      float out[2];
#pragma unroll
      for (int w = 0; w < 2; ++w) {
        const float *q = tab[w] + b;
        const float a0 = q[0] + wx * (q[ox] - q[0]);
        const float a1 = q[oy] + wx * (q[oy + ox] - q[oy]);
        out[w] = a0 + wy * (a1 - a0);
      }
      fttt[fo] = out[0];
      fqqq[fo] = out[1];
      if (p.ixl == 0 && p.izl == 0) atomicAdd(gated, 1ull);
    } else {
      double T, S;
      net_values(f, y + 2 * (size_t)k, ln, T, S);
      fttt[fo] = (float)T;
      fqqq[fo] = (float)S;
    }
  }
}

// Background correction of eikonal tables in place (the first-order scheme's
// systematic error cancels): T = T_bg + T - T_bgsolve, t* = t* t*_bg / t*_bgsolve
// with T_bg exact and t*_bg = T_bg / q_bg.
__global__ void k_tab_correct(TabView v, qpsdm_sur_line ln, float q_bg, float *__restrict__ ttt,
                              float *__restrict__ qqq, const float *__restrict__ tb,
                              const float *__restrict__ qb, int64_t total) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const ElemPos p = elem_pos(v, e, ln.nxi1, ln.nzi1);
    float f[5];
    elem_feat(v, p, ln, f);
    const double r = hypot((double)f[0] - f[2], (double)f[1] - f[3]);
    const double ta = bg_time(r, f[4], ln.v0, ln.kz);
    const int64_t o = v.desc[p.c].idx + p.r;
    ttt[o] = (float)(ta + ((double)ttt[o] - (double)tb[o]));
    const double sb = qb[o];
    if (sb > 0.0) qqq[o] = (float)((double)qqq[o] * (ta / q_bg) / sb);
  }
}

// Tables of a line between two lines that have table files, as get_ttt_all
// interpolates them (src/q-psdm.cu:2584-2596): out = a c1 + b c2 in float,
// no fused multiply-add, c2 = (line - lo) / (hi - lo), c1 = 1 - c2.
__global__ void k_tab_lerp(const float *__restrict__ a, const float *__restrict__ b, int64_t n,
                           float c1, float c2, float *__restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = __fadd_rn(__fmul_rn(a[i], c1), __fmul_rn(b[i], c2));
}

// Host: a table's descriptors and prefix sums on the device (one allocation).
struct DevTab {
  void *mem = nullptr;
  TabView v{};
  int64_t total = 0;
  int nodes = 0;
  ~DevTab() { cudaFree(mem); }
  int upload(const qpsdm_ttt_desc *desc, int ncell, int nxi1, int nzi1, int64_t len,
             cudaStream_t st) {
    std::vector<int64_t> cb(ncell + 1, 0);
    std::vector<int> nb(ncell + 1, 0);
    for (int c = 0; c < ncell; ++c) {
      const qpsdm_ttt_desc &d = desc[c];
      if (d.nys == 0 || d.nxs == 0 || d.dxs == 0 || d.dys == 0) return QPSDM_EINVAL;
      const int64_t blk = (int64_t)d.nys * d.nxs * nxi1 * nzi1;
      if (d.idx < 0 || d.idx + blk > len) return QPSDM_EINVAL;
      cb[c + 1] = cb[c] + blk;
      nb[c + 1] = nb[c] + d.nys * d.nxs;
    }
    const size_t bd = sizeof(qpsdm_ttt_desc) * ncell, bc = sizeof(int64_t) * (ncell + 1);
    const size_t bn = sizeof(int) * (ncell + 1);
    if (cudaMalloc(&mem, bd + bc + bn) != cudaSuccess) return QPSDM_ENOMEM;
    char *m = (char *)mem;
    cudaMemcpyAsync(m, desc, bd, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(m + bd, cb.data(), bc, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(m + bd + bc, nb.data(), bn, cudaMemcpyHostToDevice, st);
    v.desc = (const qpsdm_ttt_desc *)m;
    v.cell_base = (const int64_t *)(m + bd);
    v.node_base = (const int *)(m + bd + bc);
    v.ncell = ncell;
    total = cb[ncell];
    nodes = nb[ncell];
    // the host vectors die with this call: wait for the copies
    return cudaStreamSynchronize(st) == cudaSuccess ? QPSDM_OK : QPSDM_ECUDA;
  }
};

constexpr int kSurChunk = 1 << 22;  // queries per network launch

struct Scratch {
  float *x = nullptr, *y = nullptr;
  ~Scratch() {
    cudaFree(x);
    cudaFree(y);
  }
  bool alloc() {
    return cudaMalloc(&x, sizeof(float) * 5 * (size_t)kSurChunk) == cudaSuccess &&
           cudaMalloc(&y, sizeof(float) * 2 * (size_t)kSurChunk) == cudaSuccess;
  }
};

static bool line_ok(const qpsdm_sur_line *ln) {
  return ln && ln->nxg > 0 && ln->nzg > 0 && ln->nxi1 > 0 && ln->nzi1 > 0 && ln->dxi > 0.f &&
         ln->dzii > 0.f && ln->v0 > 0.f && ln->q_ref > 0.f;
}

}  // namespace qpsdm

using namespace qpsdm;

extern "C" int qpsdm_eikonal_samples(const float *d_T, const float *d_tstar, const float *d_T_bg,
                                     const float *d_tstar_bg, const qpsdm_eik_grid *grid,
                                     const float *d_src, int ns, const qpsdm_sur_background *bg,
                                     uint64_t seed, int nsamples, float *d_x, float *d_t,
                                     void *stream) {
  if (!d_T || !d_tstar || !grid || !d_src || ns <= 0 || !bg || nsamples < 0 || !d_x || !d_t ||
      (!d_T_bg) != (!d_tstar_bg) || grid->nx < 1 || grid->ny < 1 || grid->nz < 1 ||
      bg->v0 <= 0.f || bg->q_ref <= 0.f || (d_T_bg && bg->q_bg <= 0.f))
    return QPSDM_EINVAL;
  if (nsamples == 0) return QPSDM_OK;
  k_eik_samples<<<148 * 4, 256, 0, (cudaStream_t)stream>>>(
      d_T, d_tstar, d_T_bg, d_tstar_bg, *grid, (const float4 *)d_src, ns, *bg, seed, nsamples,
      d_x, d_t);
  return cudaGetLastError() == cudaSuccess ? QPSDM_OK : QPSDM_ECUDA;
}

extern "C" int qpsdm_tables_lerp(const float *d_lo, const float *d_hi, int64_t n, int line,
                                 int line_lo, int line_hi, float *d_out, void *stream) {
  if (!d_lo || !d_hi || !d_out || n < 0 || line < line_lo || line > line_hi ||
      (line_hi == line_lo && line != line_lo))
    return QPSDM_EINVAL;
  if (n == 0) return QPSDM_OK;
  const float c2 = line_hi == line_lo ? 0.0f
                                      : (float)(1.0 * (line - line_lo) / (line_hi - line_lo));
  const float c1 = (float)(1.0 - c2);
  k_tab_lerp<<<148 * 8, 256, 0, (cudaStream_t)stream>>>(d_lo, d_hi, n, c1, c2, d_out);
  return cudaGetLastError() == cudaSuccess ? QPSDM_OK : QPSDM_ECUDA;
}

extern "C" int qpsdm_eikonal_correct(const qpsdm_sur_line *ln, const qpsdm_ttt_desc *desc,
                                     float *d_ttt, float *d_qqq, const float *d_ttt_bg,
                                     const float *d_qqq_bg, int64_t len, float q_bg,
                                     void *stream) {
  if (!line_ok(ln) || !desc || !d_ttt || !d_qqq || !d_ttt_bg || !d_qqq_bg || q_bg <= 0.f)
    return QPSDM_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  DevTab t;
  int rc = t.upload(desc, ln->nxg * ln->nzg, ln->nxi1, ln->nzi1, len, st);
  if (rc) return rc;
  k_tab_correct<<<148 * 8, 256, 0, st>>>(t.v, *ln, q_bg, d_ttt, d_qqq, d_ttt_bg, d_qqq_bg,
                                         t.total);
  if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
    return QPSDM_ECUDA;
  return QPSDM_OK;
}

extern "C" int qpsdm_surrogate_gate(qpsdm_mlp *net, const qpsdm_sur_line *ln,
                                    const qpsdm_ttt_desc *desc, const float *d_ttt, int64_t len,
                                    float *d_node_err, void *stream) {
  if (!net || !line_ok(ln) || !desc || !d_ttt || !d_node_err) return QPSDM_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  DevTab t;
  int rc = t.upload(desc, ln->nxg * ln->nzg, ln->nxi1, ln->nzi1, len, st);
  if (rc) return rc;
  Scratch sc;
  if (!sc.alloc()) return QPSDM_ENOMEM;
  for (int64_t e0 = 0; e0 < t.total; e0 += kSurChunk) {
    const int n = (int)std::min<int64_t>(kSurChunk, t.total - e0);
    k_tab_features<<<148 * 4, 256, 0, st>>>(t.v, *ln, e0, n, sc.x);
    if ((rc = qpsdm_mlp_forward(net, sc.x, n, sc.y, stream))) return rc;
    k_gate_err<<<148 * 4, 256, 0, st>>>(t.v, *ln, e0, n, sc.y, d_ttt, d_node_err);
  }
  if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
    return QPSDM_ECUDA;
  return qpsdm_mlp_status(net);
}

extern "C" int qpsdm_surrogate_tables(qpsdm_mlp *net, const qpsdm_sur_line *ln,
                                      const qpsdm_ttt_desc *coarse_desc, const float *d_cttt,
                                      const float *d_cqqq, int64_t coarse_len,
                                      const float *d_node_err, float gate_ms,
                                      const qpsdm_ttt_desc *fine_desc, float *d_fttt,
                                      float *d_fqqq, int64_t fine_len, int64_t *gated_nodes,
                                      void *stream) {
  if (!net || !line_ok(ln) || !coarse_desc || !d_cttt || !d_cqqq || !d_node_err || !fine_desc ||
      !d_fttt || !d_fqqq)
    return QPSDM_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  const int ncell = ln->nxg * ln->nzg;
  DevTab c, f;
  int rc = c.upload(coarse_desc, ncell, ln->nxi1, ln->nzi1, coarse_len, st);
  if (rc) return rc;
  if ((rc = f.upload(fine_desc, ncell, ln->nxi1, ln->nzi1, fine_len, st))) return rc;
  Scratch sc;
  if (!sc.alloc()) return QPSDM_ENOMEM;
  unsigned long long *d_gated = nullptr;
  if (cudaMalloc(&d_gated, sizeof(unsigned long long)) != cudaSuccess) return QPSDM_ENOMEM;
  cudaMemsetAsync(d_gated, 0, sizeof(unsigned long long), st);
  for (int64_t e0 = 0; e0 < f.total && !rc; e0 += kSurChunk) {
    const int n = (int)std::min<int64_t>(kSurChunk, f.total - e0);
    k_tab_features<<<148 * 4, 256, 0, st>>>(f.v, *ln, e0, n, sc.x);
    if ((rc = qpsdm_mlp_forward(net, sc.x, n, sc.y, stream))) break;
    k_sur_tables<<<148 * 4, 256, 0, st>>>(f.v, c.v, *ln, e0, n, sc.y, d_cttt, d_cqqq, d_node_err,
                                         gate_ms, d_fttt, d_fqqq, d_gated);
  }
  unsigned long long h = 0;
  if (!rc && (cudaGetLastError() != cudaSuccess ||
              cudaMemcpyAsync(&h, d_gated, sizeof(h), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
              cudaStreamSynchronize(st) != cudaSuccess))
    rc = QPSDM_ECUDA;
  cudaFree(d_gated);
  if (rc) return rc;
  if (gated_nodes) *gated_nodes = (int64_t)h;
  return qpsdm_mlp_status(net);
}
