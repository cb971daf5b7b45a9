// eikonal.cu -- traveltime and t* tables from a gridded velocity / Q model.
//
// The reference reads precomputed tables (L<line>.ttt / .qqq,
// src/q-psdm.cu:2382-2627); this is the generator that writes them.  Each
// source (a surface node of a table's local grids) gets its own local 3D grid
// (origin ox, oy at the surface, spacing h, common size per batch).  The
// eikonal equation |grad T| = 1/v is solved by first-order Godunov upwind
// updates (the update of Zhao's fast sweeping method, run as in-place
// parallel relaxation: each update only lowers T and stays an upper bound, so
// the iteration reaches the same fixed point as ordered sweeps), started from
// the linear-gradient analytic traveltime inside a radius around the source,
// which is held fixed.  t* then follows from grad T . grad t* = 1/(v^2 Q)
// with the same upwind neighbours:
//   t*_i = (f_i + sum_d w_d t*_d) / sum_d w_d,  w_d = (T_i - T_d)/h^2,
// accumulated in double precision (t* is a cumulative integral along the
// ray; the float result is written once, at the end).
#include <math.h>

#include "common.cuh"
#include "qpsdm_engine.h"

namespace qpsdm {

constexpr float kInf = 1e30f;

// Trilinear sample of a global model grid [nz][ny][nx] (clamped at edges).
__device__ __forceinline__ float model_at(const float *__restrict__ g, const qpsdm_eik_model &m,
                                          float x, float y, float z) {
  const float fx = fminf(fmaxf((x - m.ox) / m.h, 0.0f), (float)(m.nx - 1));
  const float fy = fminf(fmaxf((y - m.oy) / m.h, 0.0f), (float)(m.ny - 1));
  const float fz = fminf(fmaxf(z / m.h, 0.0f), (float)(m.nz - 1));
  const int ix = min((int)fx, max(m.nx - 2, 0)), iy = min((int)fy, max(m.ny - 2, 0));
  const int iz = min((int)fz, max(m.nz - 2, 0));
  const float wx = m.nx > 1 ? fx - ix : 0.f, wy = m.ny > 1 ? fy - iy : 0.f;
  const float wz = m.nz > 1 ? fz - iz : 0.f;
  const size_t sx = m.nx > 1 ? 1 : 0, sy = m.ny > 1 ? (size_t)m.nx : 0;
  const size_t sz = m.nz > 1 ? (size_t)m.nx * m.ny : 0;
  const float *p = g + ((size_t)iz * m.ny + iy) * m.nx + ix;
  const float c00 = p[0] + wx * (p[sx] - p[0]);
  const float c01 = p[sy] + wx * (p[sy + sx] - p[sy]);
  const float c10 = p[sz] + wx * (p[sz + sx] - p[sz]);
  const float c11 = p[sz + sy] + wx * (p[sz + sy + sx] - p[sz + sy]);
  const float c0 = c00 + wy * (c01 - c00), c1 = c10 + wy * (c11 - c10);
  return c0 + wz * (c1 - c0);
}

// Linear-gradient traveltime from a surface point (v = v0 + k z).
__device__ __forceinline__ float lin_grad_time(float r, float z, float v0, float k) {
  if (k < 1e-6f) return sqrtf(r * r + z * z) / v0;
  const float v = v0 + k * z;
  const float arg = 1.0f + k * k * (r * r + z * z) / (2.0f * v0 * v);
  return acoshf(fmaxf(arg, 1.0f)) / k;
}

struct EikNode {
  int s, ix, iy, iz;
  float x, y, z;  // model coordinates
};
__device__ __forceinline__ EikNode eik_node(size_t i, size_t n, const qpsdm_eik_grid &g,
                                            const float4 *__restrict__ src) {
  EikNode e;
  e.s = (int)(i / n);
  const size_t j = i - (size_t)e.s * n;
  e.ix = (int)(j % g.nx);
  e.iy = (int)((j / g.nx) % g.ny);
  e.iz = (int)(j / ((size_t)g.nx * g.ny));
  const float4 sp = src[e.s];  // source x, y; local grid origin ox, oy
  e.x = sp.z + e.ix * g.h;
  e.y = sp.w + e.iy * g.h;
  e.z = e.iz * g.h;
  return e;
}
__device__ __forceinline__ bool in_start(const EikNode &e, const float4 *__restrict__ src,
                                         float r0) {
  const float4 sp = src[e.s];
  const float dx = e.x - sp.x, dy = e.y - sp.y;
  return dx * dx + dy * dy + e.z * e.z <= r0 * r0;
}

// Per node: h/v, 1/(v^2 Q) and the analytic start values near the source.
__global__ void k_eik_setup(const float *__restrict__ vel, const float *__restrict__ invq,
                            qpsdm_eik_model m, const float4 *__restrict__ src, int nsrc,
                            qpsdm_eik_grid g, float r0, float *__restrict__ F,
                            float *__restrict__ QF, float *__restrict__ T,
                            double *__restrict__ TS) {
  const size_t n = (size_t)g.nx * g.ny * g.nz;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n * nsrc;
       i += (size_t)gridDim.x * blockDim.x) {
    const EikNode e = eik_node(i, n, g, src);
    const float v = fmaxf(model_at(vel, m, e.x, e.y, e.z), 1.0f);
    const float q = model_at(invq, m, e.x, e.y, e.z);
    F[i] = g.h / v;
    QF[i] = q / (v * v);
    if (in_start(e, src, r0)) {
      const float4 sp = src[e.s];
      const float r = sqrtf((e.x - sp.x) * (e.x - sp.x) + (e.y - sp.y) * (e.y - sp.y));
      const float t = lin_grad_time(r, e.z, m.v0, m.kz);
      T[i] = t;
      TS[i] = (double)t * model_at(invq, m, sp.x, sp.y, 0.0f);  // near-surface Q on the path
    } else {
      T[i] = kInf;
      TS[i] = 0.0;
    }
  }
}

// One in-place Godunov relaxation of every node of every source.
__global__ void k_eik_relax(const float *__restrict__ F, float *__restrict__ T,
                            const float4 *__restrict__ src, int nsrc, qpsdm_eik_grid g, float r0,
                            unsigned *changed) {
  const size_t n = (size_t)g.nx * g.ny * g.nz;
  const size_t sxy = (size_t)g.nx * g.ny;
  unsigned ch = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n * nsrc;
       i += (size_t)gridDim.x * blockDim.x) {
    const EikNode e = eik_node(i, n, g, src);
    if (in_start(e, src, r0)) continue;
    float a = kInf, b = kInf, c = kInf;
    if (e.ix > 0) a = T[i - 1];
    if (e.ix < g.nx - 1) a = fminf(a, T[i + 1]);
    if (e.iy > 0) b = T[i - g.nx];
    if (e.iy < g.ny - 1) b = fminf(b, T[i + g.nx]);
    if (e.iz > 0) c = T[i - sxy];
    if (e.iz < g.nz - 1) c = fminf(c, T[i + sxy]);
    const float t0 = fminf(a, fminf(b, c)), t2 = fmaxf(a, fmaxf(b, c));
    const float t1 = fminf(fmaxf(a, b), fmaxf(fminf(a, b), c));  // middle value
    if (t0 >= kInf) continue;
    const float f = F[i];
    float t = t0 + f;
    if (t > t1 && t1 < kInf) {
      const float s2 = t0 + t1, d2 = 2.0f * f * f - (t0 - t1) * (t0 - t1);
      t = 0.5f * (s2 + sqrtf(fmaxf(d2, 0.0f)));
      if (t > t2 && t2 < kInf) {
        const float s3 = t0 + t1 + t2;
        const float d3 = s3 * s3 - 3.0f * (t0 * t0 + t1 * t1 + t2 * t2 - f * f);
        t = (s3 + sqrtf(fmaxf(d3, 0.0f))) / 3.0f;
      }
    }
    if (t < T[i] * (1.0f - 1e-7f)) {
      T[i] = t;
      ch = 1;
    }
  }
  if (ch) atomicOr(changed, 1u);
}

// One in-place relaxation of t* along the upwind directions of T (FP64).
__global__ void k_tstar_relax(const float *__restrict__ T, const float *__restrict__ QF,
                              double *__restrict__ TS, const float4 *__restrict__ src, int nsrc,
                              qpsdm_eik_grid g, float r0) {
  const size_t n = (size_t)g.nx * g.ny * g.nz;
  const size_t sxy = (size_t)g.nx * g.ny;
  const double ih2 = 1.0 / ((double)g.h * g.h);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n * nsrc;
       i += (size_t)gridDim.x * blockDim.x) {
    const EikNode e = eik_node(i, n, g, src);
    const float ti = T[i];
    if (ti >= kInf || in_start(e, src, r0)) continue;
    double num = QF[i], den = 0.0;
    const size_t st[3] = {1, (size_t)g.nx, sxy};
    const int id[3] = {e.ix, e.iy, e.iz}, nd[3] = {g.nx, g.ny, g.nz};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      float best = ti;
      size_t nb = 0;
      bool has = false;
      if (id[d] > 0 && T[i - st[d]] < best) {
        best = T[i - st[d]];
        nb = i - st[d];
        has = true;
      }
      if (id[d] < nd[d] - 1 && T[i + st[d]] < best) {
        best = T[i + st[d]];
        nb = i + st[d];
        has = true;
      }
      if (has) {
        const double w = ((double)ti - (double)best) * ih2;
        num += w * TS[nb];
        den += w;
      }
    }
    if (den > 0.0) TS[i] = num / den;
  }
}

__global__ void k_tstar_store(const double *__restrict__ TS, float *__restrict__ out, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = (float)TS[i];
}

// Table entries (reference layout) whose source is solved in this batch.
// Entry e of the table (cells in descriptor order, cell_base prefix sums of
// block sizes) = cell c, surface node, ixl, izl; node_src gives the global
// source number of every (cell, node) (node_base prefix sums per cell).
__global__ void k_eik_fill(const float *__restrict__ T, const float *__restrict__ TS,
                           qpsdm_eik_grid g, const float4 *__restrict__ src, int s0, int ns,
                           const qpsdm_ttt_desc *__restrict__ desc,
                           const int64_t *__restrict__ cell_base, const int *__restrict__ node_base,
                           const int *__restrict__ node_src, int ncell, qpsdm_eik_fill_geom fg,
                           float *__restrict__ ttt, float *__restrict__ qqq) {
  const int64_t total = cell_base[ncell];
  const size_t n = (size_t)g.nx * g.ny * g.nz;
  const int per_node = fg.nxi1 * fg.nzi1;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    int lo = 0, hi = ncell;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (cell_base[mid] <= e) lo = mid; else hi = mid;
    }
    const int c = lo;
    const int64_t r = e - cell_base[c];
    const int node = (int)(r / per_node);
    const int rem = (int)(r - (int64_t)node * per_node);
    const int ixl = rem / fg.nzi1, izl = rem - ixl * fg.nzi1;
    const int sl = node_src[node_base[c] + node] - s0;
    if (sl < 0 || sl >= ns) continue;
    const float4 sp = src[sl];
    const int ixg = c / fg.nzg, izg = c - ixg * fg.nzg;
    const float x = fg.x_cdp1 + (ixg * fg.nxi1 + ixl) * fg.dxi;
    const float z = (izg * fg.nzi1 + izl) * fg.dzii;
    const float fx = fminf(fmaxf((x - sp.z) / g.h, 0.0f), (float)(g.nx - 1) - 1e-3f);
    const float fy = fminf(fmaxf((fg.line_y - sp.w) / g.h, 0.0f), (float)(g.ny - 1) - 1e-3f);
    const float fz = fminf(fmaxf(z / g.h, 0.0f), (float)(g.nz - 1) - 1e-3f);
    const int jx = (int)fx, jy = (int)fy, jz = (int)fz;
    const float wx = fx - jx, wy = fy - jy, wz = fz - jz;
    const size_t base = (size_t)sl * n + ((size_t)jz * g.ny + jy) * g.nx + jx;
    const size_t sx = 1, sy = g.ny > 1 ? (size_t)g.nx : 0, sz = (size_t)g.nx * g.ny;
    float out[2];
    const float *arr[2] = {T, TS};
#pragma unroll
    for (int w = 0; w < 2; ++w) {
      const float *p = arr[w] + base;
      const float c00 = p[0] + wx * (p[sx] - p[0]);
      const float c01 = p[sy] + wx * (p[sy + sx] - p[sy]);
      const float c10 = p[sz] + wx * (p[sz + sx] - p[sz]);
      const float c11 = p[sz + sy] + wx * (p[sz + sy + sx] - p[sz + sy]);
      const float c0 = c00 + wy * (c01 - c00), c1 = c10 + wy * (c11 - c10);
      out[w] = c0 + wz * (c1 - c0);
    }
    ttt[desc[c].idx + r] = out[0];
    qqq[desc[c].idx + r] = out[1];
  }
}

}  // namespace qpsdm

using namespace qpsdm;

extern "C" int qpsdm_eikonal_solve(const float *d_vel, const float *d_invq,
                                   const qpsdm_eik_model *model, const float *d_src, int nsrc,
                                   const qpsdm_eik_grid *grid, float init_radius, int max_iter,
                                   float *d_work, float *d_T, float *d_tstar, void *stream) {
  if (!d_vel || !d_invq || !model || !d_src || !grid || !d_work || !d_T || !d_tstar ||
      nsrc <= 0 || grid->nx < 2 || grid->ny < 1 || grid->nz < 2 || grid->h <= 0.f ||
      model->nx < 1 || model->ny < 1 || model->nz < 1 || model->h <= 0.f || max_iter <= 0)
    return QPSDM_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  const qpsdm_eik_grid g = *grid;
  const size_t n = (size_t)g.nx * g.ny * g.nz * nsrc;
  // work: F, QF (n floats each), t* in FP64 (n doubles, 8-byte aligned), a flag
  float *F = d_work, *QF = d_work + n;
  double *TS = reinterpret_cast<double *>(d_work + 2 * n + ((2 * n) & 1));
  unsigned *changed = reinterpret_cast<unsigned *>(TS + n);
  if (reinterpret_cast<uintptr_t>(d_work) % 8) return QPSDM_EINVAL;
  const float4 *src = (const float4 *)d_src;
  const int blk = 256, grd = 148 * 8;
  k_eik_setup<<<grd, blk, 0, st>>>(d_vel, d_invq, *model, src, nsrc, g, init_radius, F, QF,
                                   d_T, TS);
  // relax in rounds of 16 sweeps until a round changes nothing (or max_iter)
  int rounds = 0;
  for (int it = 0; it < max_iter; it += 16, ++rounds) {
    cudaMemsetAsync(changed, 0, sizeof(unsigned), st);
    for (int k = 0; k < 16; ++k)
      k_eik_relax<<<grd, blk, 0, st>>>(F, d_T, src, nsrc, g, init_radius, changed);
    unsigned h = 0;
    if (cudaMemcpyAsync(&h, changed, sizeof(unsigned), cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return QPSDM_ECUDA;
    if (!h) break;
  }
  // t* needs about as many sweeps as T took to settle
  const int tsweeps = (rounds + 1) * 16;
  for (int it = 0; it < tsweeps; ++it)
    k_tstar_relax<<<grd, blk, 0, st>>>(d_T, QF, TS, src, nsrc, g, init_radius);
  k_tstar_store<<<grd, blk, 0, st>>>(TS, d_tstar, n);
  return cudaGetLastError() == cudaSuccess ? QPSDM_OK : QPSDM_ECUDA;
}

extern "C" int qpsdm_eikonal_fill(const float *d_T, const float *d_tstar,
                                  const qpsdm_eik_grid *grid, const float *d_src, int s0, int ns,
                                  const qpsdm_ttt_desc *d_desc, const int64_t *d_cell_base,
                                  const int *d_node_base, const int *d_node_src, int ncell,
                                  const qpsdm_eik_fill_geom *fg, float *d_ttt, float *d_qqq,
                                  void *stream) {
  if (!d_T || !d_tstar || !grid || !d_src || !d_desc || !d_cell_base || !d_node_base ||
      !d_node_src || !fg || !d_ttt || !d_qqq || ncell <= 0 || ns <= 0)
    return QPSDM_EINVAL;
  k_eik_fill<<<148 * 8, 256, 0, (cudaStream_t)stream>>>(
      d_T, d_tstar, *grid, (const float4 *)d_src, s0, ns, d_desc, d_cell_base, d_node_base,
      d_node_src, ncell, *fg, d_ttt, d_qqq);
  return cudaGetLastError() == cudaSuccess ? QPSDM_OK : QPSDM_ECUDA;
}
