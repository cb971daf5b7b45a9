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

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <type_traits>
#include <cmath>
#include <cub/cub.cuh>
#include <vector>

#include "common.cuh"
#include "fft.cuh"
#include "internal.h"
#include "physics.h"

namespace qpsdm {

// One set of the batched form's grouping buffers (receiver keys, members,
// source positions, tile queue, deferred-tile list).  Consecutive image lines
// of a brick alternate between two sets, so that a line's grouping and image
// kernels can run on a second stream beside the previous line's: the tail of
// one line's persistent launch overlaps the start of the next.
struct GroupSet {
  unsigned long long *d_key[2] = {};
  int *d_val[2] = {};
  unsigned long long *d_ukey = nullptr;
  int *d_count = nullptr, *d_off = nullptr, *d_nruns = nullptr;
  int *d_srcflag = nullptr, *d_sid = nullptr;
  float2 *d_srcpos = nullptr;
  int4 *d_mem = nullptr;
  float2 *d_grppos = nullptr;
  int *d_memgrp = nullptr;
  int *d_tile_ctr = nullptr;
  int *d_defer = nullptr;
  size_t defer_cap = 0;
  int *d_ndefer = nullptr;
  int *d_nmem = nullptr;
  void *d_cub = nullptr;
};

struct PhysicsState {
  int nfft = 0, nffti = 0, nbins = 0, max_batch = 0, dtype = 0;
  float dtstar = 0.0f;
  float2 *d_filter = nullptr;  // [nbins][nfft/2+1]
  float2 *d_spec = nullptr;    // [max_batch][nfft/2+1]
  float *d_fmax = nullptr;     // [nfft/2+1] max over bins of |filter|
  float *d_pscale = nullptr;   // [max_batch] FP16 panels: per-trace sample multiplier
  void *d_panels = nullptr;    // [max_batch][nbins][nffti]
  float *d_comp = nullptr;     // Kahan compensation, [img_cap]
  size_t comp_cap = 0;
  // line tables
  struct LineTab {
    qpsdm_ttt_desc *dt = nullptr, *dq = nullptr;
    float *ttt = nullptr, *qqq = nullptr;
    size_t dt_cap = 0, dq_cap = 0, ttt_cap = 0, qqq_cap = 0;
    // batched form, t and t* tables with identical descriptors: (t, t*) pairs
    float2 *tq = nullptr;
    size_t tq_cap = 0;
    bool paired = false;
  };
  std::vector<LineTab> tabs;  // one per line of the brick
  float *d_tab_tmp = nullptr;  // batched form: table upload before the re-layout
  size_t tab_tmp_cap = 0;
  int ntabs = 0;
  int *d_any = nullptr;       // [max_batch] accepted by any line of the brick
  // batched form: grouping scratch (sized for max_batch at create)
  int form = QPSDM_FORM_PLAIN;
  unsigned long long *d_key[2] = {};  // receiver keys, unsorted / sorted
  int *d_val[2] = {};                 // trace indices, unsorted / sorted
  unsigned long long *d_ukey = nullptr;
  int *d_count = nullptr, *d_off = nullptr, *d_nruns = nullptr;
  int *d_srcflag = nullptr, *d_sid = nullptr;  // source run flags / ids (1-based)
  float2 *d_srcpos = nullptr;                  // [max_batch] source positions
  int4 *d_mem = nullptr;                       // [max_batch] member info
  float2 *d_grppos = nullptr;                  // [max_batch] receiver positions
  int *d_memgrp = nullptr;                     // [max_batch] group of each sorted member
  int *d_tile_ctr = nullptr;
  int *d_defer = nullptr;    // tiles the fast form leaves to k_image_batched
  size_t defer_cap = 0;
  int *d_ndefer = nullptr;
  int *d_nmem = nullptr;                       // accepted members of the current line's batch
  void *d_cub = nullptr;
  size_t cub_bytes = 0;
  int num_sms = 0;
  int tile_z = 0, tile_x = 0, forced_variant = 0;
  int variant = -1;          // batched kernel variant (autotuned)
  float *d_tune = nullptr;   // scratch image of the autotuner
  size_t tune_cap = 0;
  float tune_ms[32] = {};    // autotuner timings per variant (ms)
  // the two grouping sets (the d_key .. d_cub fields above are the selected
  // one) and the second stream of the line loop
  GroupSet sets[2];
  int cur_set = 0;
  cudaStream_t aux = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
};

// Points the grouping fields at set i (the launches enqueued afterwards use it).
static void select_set(PhysicsState *s, int i) {
  const GroupSet &g = s->sets[i];
  for (int k = 0; k < 2; ++k) {
    s->d_key[k] = g.d_key[k];
    s->d_val[k] = g.d_val[k];
  }
  s->d_ukey = g.d_ukey;
  s->d_count = g.d_count;
  s->d_off = g.d_off;
  s->d_nruns = g.d_nruns;
  s->d_srcflag = g.d_srcflag;
  s->d_sid = g.d_sid;
  s->d_srcpos = g.d_srcpos;
  s->d_mem = g.d_mem;
  s->d_grppos = g.d_grppos;
  s->d_memgrp = g.d_memgrp;
  s->d_tile_ctr = g.d_tile_ctr;
  s->d_defer = g.d_defer;
  s->defer_cap = g.defer_cap;
  s->d_ndefer = g.d_ndefer;
  s->d_nmem = g.d_nmem;
  s->d_cub = g.d_cub;
  s->cur_set = i;
}

static size_t dtype_bytes(int t) { return t == QPSDM_PANEL_FP32 ? 4 : 2; }
static int batched_alloc(PhysicsState *s, const qpsdm_static_params &p);

// (-i ww_k) * A(pi f t*) * exp(-2 i f t* ln(f/fc)) / nfft for every bin.
static void filter_table(const qpsdm_static_params &p, int nbins, float dtstar,
                         std::vector<float2> &out, std::vector<float> &fmax) {
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
  fmax.assign(nk, 0.0f);
  for (int b = 0; b < nbins; ++b)
    for (int k = 0; k < nk; ++k) {
      const float2 v = out[(size_t)b * nk + k];
      fmax[k] = std::max(fmax[k], std::hypot(v.x, v.y) * 1.0001f);
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
  if (p.form == QPSDM_FORM_BATCHED && p.max_batch >= (1 << 24)) {
    if (err) *err = "batched form: max_batch must be below 2^24 traces";
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
  std::vector<float> fmax;
  filter_table(p, p.nbins, p.dtstar, f, fmax);
  const size_t nk = (size_t)p.nfft / 2 + 1;
  auto bad = [&](const char *w) {
    if (err) *err = std::string("physics_create: ") + w;
    physics_destroy(s);
    return QPSDM_ENOMEM;
  };
  if (cudaMalloc(&s->d_filter, sizeof(float2) * f.size()) != cudaSuccess) return bad("filter");
  cudaMemcpy(s->d_filter, f.data(), sizeof(float2) * f.size(), cudaMemcpyHostToDevice);
  if (cudaMalloc(&s->d_spec, sizeof(float2) * nk * p.max_batch) != cudaSuccess) return bad("spectra");
  if (cudaMalloc(&s->d_fmax, sizeof(float) * nk) != cudaSuccess) return bad("filter bound");
  cudaMemcpy(s->d_fmax, fmax.data(), sizeof(float) * nk, cudaMemcpyHostToDevice);
  if (cudaMalloc(&s->d_pscale, sizeof(float) * p.max_batch) != cudaSuccess) return bad("scales");
  const size_t pb = dtype_bytes(p.panel_dtype) * (size_t)p.nbins * p.nffti * p.max_batch;
  if (cudaMalloc(&s->d_panels, pb) != cudaSuccess) return bad("panels");
  if (cudaMalloc(&s->d_any, sizeof(int) * p.max_batch) != cudaSuccess) return bad("flags");
  s->form = p.form;
  if (p.form == QPSDM_FORM_BATCHED) {
    if (batched_alloc(s, p)) return bad("batched scratch");
  } else if (p.form != QPSDM_FORM_PLAIN) {
    if (err) *err = "unknown physics form";
    physics_destroy(s);
    return QPSDM_EINVAL;
  }
  *out = s;
  return QPSDM_OK;
}

void physics_destroy(PhysicsState *s) {
  if (!s) return;
  if (s->aux) cudaStreamSynchronize(s->aux);
  for (GroupSet &g : s->sets) {
    for (int i = 0; i < 2; ++i) {
      cudaFree(g.d_key[i]);
      cudaFree(g.d_val[i]);
    }
    cudaFree(g.d_ukey);
    cudaFree(g.d_count);
    cudaFree(g.d_off);
    cudaFree(g.d_nruns);
    cudaFree(g.d_srcflag);
    cudaFree(g.d_sid);
    cudaFree(g.d_srcpos);
    cudaFree(g.d_mem);
    cudaFree(g.d_grppos);
    cudaFree(g.d_memgrp);
    cudaFree(g.d_tile_ctr);
    cudaFree(g.d_defer);
    cudaFree(g.d_ndefer);
    cudaFree(g.d_nmem);
    cudaFree(g.d_cub);
  }
  if (s->ev_fork) cudaEventDestroy(s->ev_fork);
  if (s->ev_join) cudaEventDestroy(s->ev_join);
  if (s->aux) cudaStreamDestroy(s->aux);
  cudaFree(s->d_filter);
  cudaFree(s->d_spec);
  cudaFree(s->d_fmax);
  cudaFree(s->d_pscale);
  cudaFree(s->d_panels);
  cudaFree(s->d_comp);
  for (auto &t : s->tabs) {
    cudaFree(t.dt);
    cudaFree(t.dq);
    cudaFree(t.ttt);
    cudaFree(t.qqq);
    cudaFree(t.tq);
  }
  cudaFree(s->d_any);
  cudaFree(s->d_tune);
  cudaFree(s->d_tab_tmp);
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

static int check_tables(const qpsdm_line_params &l, std::string *err) {
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
  return QPSDM_OK;
}

// Batched form: every surface node's [nxi1][nzi1] plane of a table cell
// (the reference layout, depth fastest) re-laid out as [nzi1][nxi1] (cdp
// fastest), so that image points of neighbouring cdps, which a warp of the
// batched kernel holds, read neighbouring table words.  Out of place:
// descriptors may share a block.
// (t, t*) pairs of two tables with identical descriptors.
__global__ void k_tab_pair(const float *__restrict__ t, const float *__restrict__ q,
                           float2 *__restrict__ tq, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    tq[i] = make_float2(t[i], q[i]);
}

__global__ void k_tab_xfast(const float *__restrict__ in, float *__restrict__ out,
                            const qpsdm_ttt_desc *__restrict__ desc, int nxi1, int nzi1) {
  const qpsdm_ttt_desc d = desc[blockIdx.y];
  const int nplanes = (int)d.nys * d.nxs, plane = nxi1 * nzi1;
  for (int pl = blockIdx.x; pl < nplanes; pl += gridDim.x) {
    const int64_t base = d.idx + (int64_t)pl * plane;
    for (int e = threadIdx.x; e < plane; e += blockDim.x) {
      const int ixl = e / nzi1, izl = e - ixl * nzi1;
      out[base + izl * nxi1 + ixl] = in[base + e];
    }
  }
}

// Table data may be host or device memory (cudaMemcpyDefault: unified
// addressing tells them apart); descriptors are host memory.
int physics_set_lines(PhysicsState *s, const qpsdm_static_params &p,
                      const qpsdm_line_params *lines, int nlines, cudaStream_t st,
                      std::string *err) {
  (void)p;
  for (int il = 0; il < nlines; ++il) {
    int rc = check_tables(lines[il], err);
    if (rc) return rc;
  }
  if ((int)s->tabs.size() < nlines) s->tabs.resize(nlines);
  for (int il = 0; il < nlines; ++il) {
    const qpsdm_line_params &l = lines[il];
    PhysicsState::LineTab &t = s->tabs[il];
    const size_t ncell = (size_t)l.nxg * l.nzg;
    if (!grow_dev(&t.dt, &t.dt_cap, ncell) || !grow_dev(&t.dq, &t.dq_cap, ncell) ||
        !grow_dev(&t.ttt, &t.ttt_cap, (size_t)l.ttt_len) ||
        !grow_dev(&t.qqq, &t.qqq_cap, (size_t)l.qqq_len)) {
      if (err) *err = "table allocation failed";
      return QPSDM_ENOMEM;
    }
    cudaMemcpyAsync(t.dt, l.ttt_desc, sizeof(qpsdm_ttt_desc) * ncell, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(t.dq, l.qqq_desc, sizeof(qpsdm_ttt_desc) * ncell, cudaMemcpyHostToDevice, st);
    if (s->form == QPSDM_FORM_BATCHED) {
      if (!grow_dev(&s->d_tab_tmp, &s->tab_tmp_cap,
                    (size_t)std::max(l.ttt_len, l.qqq_len))) {
        if (err) *err = "table re-layout scratch allocation failed";
        return QPSDM_ENOMEM;
      }
      const dim3 g(256, (unsigned)ncell);
      cudaMemcpyAsync(s->d_tab_tmp, l.ttt, sizeof(float) * l.ttt_len, cudaMemcpyDefault, st);
      k_tab_xfast<<<g, 256, 0, st>>>(s->d_tab_tmp, t.ttt, t.dt, l.nxi1, l.nzi1);
      cudaMemcpyAsync(s->d_tab_tmp, l.qqq, sizeof(float) * l.qqq_len, cudaMemcpyDefault, st);
      k_tab_xfast<<<g, 256, 0, st>>>(s->d_tab_tmp, t.qqq, t.dq, l.nxi1, l.nzi1);
      // identical descriptors (the reference writes both tables alike): the
      // image kernel reads t and t* of a node with one 8-byte load
      t.paired = l.ttt_len == l.qqq_len &&
                 std::memcmp(l.ttt_desc, l.qqq_desc, sizeof(qpsdm_ttt_desc) * ncell) == 0;
      if (t.paired) {
        if (!grow_dev(&t.tq, &t.tq_cap, (size_t)l.ttt_len)) {
          if (err) *err = "paired table allocation failed";
          return QPSDM_ENOMEM;
        }
        k_tab_pair<<<148 * 8, 256, 0, st>>>(t.ttt, t.qqq, t.tq, l.ttt_len);
      }
    } else {
      cudaMemcpyAsync(t.ttt, l.ttt, sizeof(float) * l.ttt_len, cudaMemcpyDefault, st);
      cudaMemcpyAsync(t.qqq, l.qqq, sizeof(float) * l.qqq_len, cudaMemcpyDefault, st);
    }
  }
  if (cudaStreamSynchronize(st) != cudaSuccess) {
    if (err) *err = "table upload failed";
    return QPSDM_ECUDA;
  }
  s->ntabs = nlines;
  return QPSDM_OK;
}

int physics_begin_offset(PhysicsState *s, const qpsdm_static_params &p,
                         const qpsdm_offset_params &o, int nlines, cudaStream_t st,
                         std::string *err) {
  if (s->form == QPSDM_FORM_BATCHED && s->variant < 0 &&
      !grow_dev(&s->d_tune, &s->tune_cap, (size_t)(o.ixend - o.ixstart) * p.nzi)) {
    if (err) *err = "autotuner scratch allocation failed";
    return QPSDM_ENOMEM;
  }
  if (s->form == QPSDM_FORM_BATCHED) {
    const size_t nxb = (size_t)(o.ixend - o.ixstart);
    for (GroupSet &g : s->sets)
      if (!grow_dev(&g.d_defer, &g.defer_cap, nxb * p.nzi / 32 + nxb + p.nzi + 1)) {
        if (err) *err = "deferred-tile list allocation failed";
        return QPSDM_ENOMEM;
      }
    select_set(s, s->cur_set);
  }
  if (p.kahan) {
    const size_t n = (size_t)(o.ixend - o.ixstart) * p.nzi * nlines;
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

// Forward spectra of the accepted traces; a persistent CTA loads the
// twiddles into shared memory once and then takes every gridDim.x-th trace.
// For FP16 panels also the trace's sample multiplier: every panel sample of
// the trace is bounded by B = 2 sum_k |X_k| max_b |F_b,k| (triangle
// inequality over the c2r sum), and the panels store x / 2^e with e chosen so
// that B / 2^e lies in [2^13, 2^14): no overflow of FP16 (max 65504) and no
// loss to its subnormal range; the image kernels multiply the samples by 2^e
// again (exact).
__global__ void __launch_bounds__(256) k_phys_fwd(const uint8_t *__restrict__ rec, int rec_bytes,
                                                  int be, const int *__restrict__ status,
                                                  int sstride, int ntr, int ntl,
                                                  float dt, const float *__restrict__ tap,
                                                  FftPlan p, float2 *__restrict__ spec,
                                                  const float *__restrict__ fmax,
                                                  float *__restrict__ pscale) {
  extern __shared__ float2 sm[];
  float2 *b0 = sm, *b1 = sm + p.m, *twm = sm + 2 * p.m, *twn = sm + 3 * p.m;
  __shared__ float s_part[8];
  for (int i = threadIdx.x; i < p.m; i += blockDim.x) twm[i] = p.tw_m[i];
  for (int i = threadIdx.x; i <= p.m; i += blockDim.x) twn[i] = p.tw_n[i];
  for (int itr = blockIdx.x; itr < ntr; itr += gridDim.x) {
    if (status[(size_t)itr * sstride] != kAccepted) continue;  // uniform in the CTA
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
    float bound = 0.0f;
    for (int k = threadIdx.x; k <= p.m; k += blockDim.x) {
      const float2 v = rfft_bin(Z, twn, p.m, k);
      o[k] = v;
      if (pscale) bound = fmaf(sqrtf(v.x * v.x + v.y * v.y), fmax[k], bound);
    }
    if (pscale) {
      for (int off = 16; off > 0; off >>= 1) bound += __shfl_xor_sync(0xffffffffu, bound, off);
      if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = bound;
    }
    __syncthreads();  // Z and s_part complete; b0 / b1 free for the next trace
    if (pscale && threadIdx.x == 0) {
      float b = 0.0f;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) b += s_part[w];
      b *= 2.0f;
      int e = 0;
      if (b > 0.0f && isfinite(b)) {
        frexpf(b, &e);  // b = m 2^e, m in [0.5, 1)
        e = min(max(e - 14, -126), 127);
      }
      pscale[itr] = ldexpf(1.0f, e);
    }
  }
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

// Four output samples (two complex points) of a panel row.
template <typename T>
__device__ __forceinline__ void store_quad(T *dst, float mul, float2 z0, float2 z1);
template <>
__device__ __forceinline__ void store_quad<float>(float *d, float mul, float2 z0, float2 z1) {
  *reinterpret_cast<float4 *>(d) = make_float4(mul * z0.x, mul * z0.y, mul * z1.x, mul * z1.y);
}
template <>
__device__ __forceinline__ void store_quad<__half>(__half *d, float mul, float2 z0, float2 z1) {
  const __half2 a = __halves2half2(__float2half_rn(mul * z0.x), __float2half_rn(mul * z0.y));
  const __half2 c = __halves2half2(__float2half_rn(mul * z1.x), __float2half_rn(mul * z1.y));
  uint2 u;
  u.x = *reinterpret_cast<const unsigned *>(&a);
  u.y = *reinterpret_cast<const unsigned *>(&c);
  *reinterpret_cast<uint2 *>(d) = u;
}
template <>
__device__ __forceinline__ void store_quad<__nv_bfloat16>(__nv_bfloat16 *d, float mul, float2 z0,
                                                         float2 z1) {
  const __nv_bfloat162 a =
      __halves2bfloat162(__float2bfloat16_rn(mul * z0.x), __float2bfloat16_rn(mul * z0.y));
  const __nv_bfloat162 c =
      __halves2bfloat162(__float2bfloat16_rn(mul * z1.x), __float2bfloat16_rn(mul * z1.y));
  uint2 u;
  u.x = *reinterpret_cast<const unsigned *>(&a);
  u.y = *reinterpret_cast<const unsigned *>(&c);
  *reinterpret_cast<uint2 *>(d) = u;
}

// Z[k] of the c2r split from a = Y[k], c = Y[m-k] (irfft_pre with the two
// spectrum values already at hand).
__device__ __forceinline__ float2 irfft_split(float2 a, float2 c, float2 tw) {
  const float2 bb = cconj(c);
  const float2 e = make_float2(0.5f * (a.x + bb.x), 0.5f * (a.y + bb.y));
  const float2 d = make_float2(0.5f * (a.x - bb.x), 0.5f * (a.y - bb.y));
  const float2 o = cmul(d, cconj(tw));
  return make_float2(e.x - o.y, e.y + o.x);
}

// t*-binned panels: for every accepted trace and bin b, the filtered,
// zero-padded spectrum X F_b -> c2r of length nffti.  A persistent CTA loads
// the twiddles into shared memory once, then takes every gridDim.x-th trace,
// keeps its spectrum in shared memory and runs all bins of it back to back.
// Shared memory: two FFT buffers, the m + (m+1) twiddles, the nk-point
// spectrum.  Each bin's input goes to the buffer the previous bin's result
// is not in, so one barrier per bin covers the previous bin's stores.
// Rows are stored two complex points (16 / 8 bytes) at a time when m is even.
template <typename T>
__global__ void __launch_bounds__(256, 3) k_phys_panels(const int *__restrict__ status, int sstride,
                                                     int ntr, const float2 *__restrict__ spec,
                                                     int nk, const float2 *__restrict__ filt,
                                                     FftPlan p, int nbins, T *__restrict__ panels,
                                                     const float *__restrict__ pscale) {
  extern __shared__ float2 sm[];
  float2 *twm = sm + 2 * p.m, *twn = sm + 3 * p.m, *Xs = sm + 4 * p.m + 1;
  for (int i = threadIdx.x; i < p.m; i += blockDim.x) twm[i] = p.tw_m[i];
  for (int i = threadIdx.x; i <= p.m; i += blockDim.x) twn[i] = p.tw_n[i];
  int in = 0;  // buffer the next bin's input goes to
  for (int itr = blockIdx.x; itr < ntr; itr += gridDim.x) {
    if (status[(size_t)itr * sstride] != kAccepted) continue;  // uniform in the CTA
    const float2 *X = spec + (size_t)itr * nk;
    for (int k = threadIdx.x; k < nk; k += blockDim.x) Xs[k] = X[k];
    __syncthreads();
    // 2 / 2^e for FP16 (exact), 2 otherwise
    const float mul = std::is_same<T, __half>::value ? 2.0f / pscale[itr] : 2.0f;
    for (int b = 0; b < nbins; ++b) {
      const float2 *F = filt + (size_t)b * nk;
      float2 *b0 = sm + in * p.m, *b1 = sm + (in ^ 1) * p.m;
      for (int k = threadIdx.x; 2 * k <= p.m; k += blockDim.x) {
        // Y[k] and Y[m-k] of the zero-padded filtered spectrum give both
        // Z[k] and Z[m-k] of the c2r split
        const int k2 = p.m - k;
        const float2 a = k < nk ? cmul(Xs[k], __ldg(F + k)) : make_float2(0.f, 0.f);
        const float2 c = k2 < nk ? cmul(Xs[k2], __ldg(F + k2)) : make_float2(0.f, 0.f);
        b0[k] = irfft_split(a, c, twn[k]);
        if (k > 0 && k < k2) b0[k2] = irfft_split(c, a, twn[k2]);
      }
      __syncthreads();
      const int cur = fft_complex_smem(b0, b1, p, twm, true);
      const float2 *z = cur ? b1 : b0;
      T *out = panels + ((size_t)itr * nbins + b) * p.n;
      if ((p.m & 1) == 0) {  // rows of 4m bytes (FP16) / 8m bytes: 8- / 16-byte aligned
        for (int j = threadIdx.x; 2 * j < p.m; j += blockDim.x)
          store_quad<T>(out + 4 * j, mul, z[2 * j], z[2 * j + 1]);
      } else {
        for (int j = threadIdx.x; j < p.m; j += blockDim.x) {
          store_sample<T>(out + 2 * j, mul * z[j].x);
          store_sample<T>(out + 2 * j + 1, mul * z[j].y);
        }
      }
      in = cur ? in : in ^ 1;
    }
    // the last bin's stores read the buffer other than `in`; the next trace
    // writes Xs (read by this trace's bins, all past a barrier), then `in`
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
  int xfast;  // tables stored [izl][ixl] inside each surface node's plane (batched form)
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

// The surface-grid test of every table lookup: fractional node coordinates
// of (px, py) in a grid of nxs x nys nodes at spacing 1/rdx, 1/rdy centred
// on (xc, 0), and whether they lie inside it.  Explicit IEEE operations (the
// oracle repeats them bit for bit), because a pair is evaluated -- and
// counted as a point-trace -- exactly when both its lookups pass this test.
__device__ __forceinline__ bool grid_pos(float px, float py, float xc, float rdx, float rdy,
                                         float hx, float hy, int nxs, int nys, float &fx,
                                         float &fy) {
  fx = __fmaf_rn(__fsub_rn(px, xc), rdx, hx);
  fy = __fmaf_rn(py, rdy, hy);
  return fx >= 0.0f && fx <= (float)(nxs - 1) && fy >= 0.0f && fy <= (float)(nys - 1);
}

// Packed FP32 pairs (sm_100's f32x2 instructions): two values in one 64-bit
// register pair, one instruction for both.  Each operation is the IEEE
// single-precision operation of each half (round to nearest), the same
// result as two scalar ones.
__device__ __forceinline__ unsigned long long f2_pack(float a, float b) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ float2 f2_unpack(unsigned long long r) {
  float2 v;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(v.x), "=f"(v.y) : "l"(r));
  return v;
}
__device__ __forceinline__ unsigned long long f2_add(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ unsigned long long f2_sub(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ unsigned long long f2_mul(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ unsigned long long f2_fma(unsigned long long a, unsigned long long b,
                                                     unsigned long long c) {
  unsigned long long r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}

// a + w (b - a) as one fused multiply-add (the form every table and sample
// interpolation of the image kernels takes; the FP32 oracle repeats it).
__device__ __forceinline__ float lerp(float a, float b, float w) {
  return __fmaf_rn(w, __fsub_rn(b, a), a);
}

// Bilinear value of a 2 x 2 node block starting at tab + base.
__device__ __forceinline__ float bilin(const float *__restrict__ tab, int64_t base, int64_t sx,
                                       int64_t sy, float wx, float wy) {
  const float v00 = __ldg(tab + base), v01 = __ldg(tab + base + sx);
  const float v10 = __ldg(tab + base + sy), v11 = __ldg(tab + base + sy + sx);
  return lerp(lerp(v00, v01, wx), lerp(v10, v11, wx), wy);
}

// Table value at one depth node of a cell for surface point (px, py).
// Returns false outside the cell's surface grid.
__device__ __forceinline__ bool table_node(const qpsdm_ttt_desc &d, const float *__restrict__ tab,
                                           float px, float py, float xc, int poff,
                                           int nxi1, int nzi1, float &v) {
  const int nxs = d.nxs, nys = d.nys;
  float fx, fy;
  if (!grid_pos(px, py, xc, __fdiv_rn(1.0f, (float)d.dxs), __fdiv_rn(1.0f, (float)d.dys),
                0.5f * (nxs - 1), 0.5f * (nys - 1), nxs, nys, fx, fy))
    return false;
  int ix = min((int)fx, max(nxs - 2, 0));
  int iy = min((int)fy, max(nys - 2, 0));
  const float wx = nxs > 1 ? __fsub_rn(fx, (float)ix) : 0.0f;
  const float wy = nys > 1 ? __fsub_rn(fy, (float)iy) : 0.0f;
  const int64_t sx = nxs > 1 ? (int64_t)nxi1 * nzi1 : 0;
  const int64_t sy = nys > 1 ? (int64_t)nxs * nxi1 * nzi1 : 0;
  const int64_t base = d.idx + (int64_t)(iy * nxs + ix) * nxi1 * nzi1 + poff;
  v = bilin(tab, base, sx, sy, wx, wy);
  return true;
}

struct PointCells {
  bool ok;
  bool same;  // all four descriptors share one surface grid
  int offA, offB;       // offsets of the point's two depth nodes inside a surface plane
  int cA, cB;          // cells of the two depth nodes
  int nxs, nys;        // shared surface grid (fast path)
  float c2, xc;
  float rdx, rdy, hx, hy;  // 1/dxs, 1/dys, (nxs-1)/2, (nys-1)/2 of the shared grid
  int64_t tA, tB, qA, qB;  // data offsets (idx) of the four blocks
};

__device__ __forceinline__ bool same_grid(const qpsdm_ttt_desc &a, const qpsdm_ttt_desc &b) {
  return a.nxs == b.nxs && a.nys == b.nys && a.dxs == b.dxs && a.dys == b.dys;
}

// Cell, depth node and descriptors of image point (ixi, z), src/q-psdm.cu:2343-2349.
__device__ __forceinline__ void setup_cells(PointCells &pc, int ixi, float z,
                                            const PhysImageArgs &a,
                                            const qpsdm_ttt_desc *__restrict__ dt,
                                            const qpsdm_ttt_desc *__restrict__ dq) {
  pc.ok = false;
  pc.same = false;
  if (ixi < a.tcdp1 || ixi > a.tcdp2) return;
  const int lx = ixi - a.tcdp1;
  const int ixg = lx / a.nxi1;
  const int ixl = lx - ixg * a.nxi1;
  const float fz = __fdiv_rn(z, a.dzii);
  const int izn = (int)fz;
  pc.c2 = __fsub_rn(fz, (float)izn);
  int izgA = izn / a.nzi1, izgB = (izn + 1) / a.nzi1;
  int izlA = izn - izgA * a.nzi1;
  int izlB = izn + 1 - izgB * a.nzi1;
  if (izgB >= a.nzg) {  // deepest node: no lower neighbour
    izgB = izgA;
    izlB = izlA;
    pc.c2 = 0.0f;
  }
  if (ixg >= a.nxg || izgA >= a.nzg) return;
  pc.ok = true;
  // [ixl][izl] planes (the reference layout) or [izl][ixl] (batched form)
  pc.offA = a.xfast ? izlA * a.nxi1 + ixl : ixl * a.nzi1 + izlA;
  pc.offB = a.xfast ? izlB * a.nxi1 + ixl : ixl * a.nzi1 + izlB;
  pc.cA = ixg * a.nzg + izgA;
  pc.cB = ixg * a.nzg + izgB;
  const qpsdm_ttt_desc tA = dt[pc.cA], tB = dt[pc.cB], qA = dq[pc.cA], qB = dq[pc.cB];
  pc.tA = tA.idx;
  pc.tB = tB.idx;
  pc.qA = qA.idx;
  pc.qB = qB.idx;
  pc.xc = __fmul_rn(__fadd_rn((float)(a.tcdp1 + ixg * a.nxi1), 0.5f * (a.nxi1 - 1)), a.dxi);
  pc.same = same_grid(tA, tB) && same_grid(tA, qA) && same_grid(tA, qB);
  pc.nxs = tA.nxs;
  pc.nys = tA.nys;
  pc.rdx = __fdiv_rn(1.0f, (float)tA.dxs);
  pc.rdy = __fdiv_rn(1.0f, (float)tA.dys);
  pc.hx = 0.5f * (tA.nxs - 1);
  pc.hy = 0.5f * (tA.nys - 1);
}


__device__ __forceinline__ bool lookup_tq(const PointCells &pc,
                                          const qpsdm_ttt_desc *__restrict__ dt,
                                          const float *__restrict__ ttt,
                                          const qpsdm_ttt_desc *__restrict__ dq,
                                          const float *__restrict__ qqq, int nxi1, int nzi1,
                                          float px, float py, float &t, float &q) {
  if (pc.same) {  // one set of surface weights for t and t*, both depth nodes
    const int nxs = pc.nxs, nys = pc.nys;
    float fx, fy;
    if (!grid_pos(px, py, pc.xc, pc.rdx, pc.rdy, pc.hx, pc.hy, nxs, nys, fx, fy)) return false;
    const int ix = min((int)fx, max(nxs - 2, 0));
    const int iy = min((int)fy, max(nys - 2, 0));
    const float wx = nxs > 1 ? __fsub_rn(fx, (float)ix) : 0.0f;
    const float wy = nys > 1 ? __fsub_rn(fy, (float)iy) : 0.0f;
    const int64_t plane = (int64_t)nxi1 * nzi1;
    const int64_t sx = nxs > 1 ? plane : 0, sy = nys > 1 ? (int64_t)nxs * plane : 0;
    const int64_t off = (int64_t)(iy * nxs + ix) * plane;
    const float ta = bilin(ttt, pc.tA + off + pc.offA, sx, sy, wx, wy);
    const float tb = bilin(ttt, pc.tB + off + pc.offB, sx, sy, wx, wy);
    const float qa = bilin(qqq, pc.qA + off + pc.offA, sx, sy, wx, wy);
    const float qb = bilin(qqq, pc.qB + off + pc.offB, sx, sy, wx, wy);
    t = lerp(ta, tb, pc.c2);
    q = lerp(qa, qb, pc.c2);
    return true;
  }
  // cells with different surface grids: one lookup per descriptor
  float ta, tb, qa, qb;
  if (!table_node(dt[pc.cA], ttt, px, py, pc.xc, pc.offA, nxi1, nzi1, ta)) return false;
  if (!table_node(dt[pc.cB], ttt, px, py, pc.xc, pc.offB, nxi1, nzi1, tb)) return false;
  if (!table_node(dq[pc.cA], qqq, px, py, pc.xc, pc.offA, nxi1, nzi1, qa)) return false;
  if (!table_node(dq[pc.cB], qqq, px, py, pc.xc, pc.offB, nxi1, nzi1, qb)) return false;
  t = lerp(ta, tb, pc.c2);
  q = lerp(qa, qb, pc.c2);
  return true;
}

// lookup_tq for a line whose t and t* tables have identical descriptors,
// read as (t, t*) pairs (tq): same values, same arithmetic, half the loads.
__device__ __forceinline__ float2 bilin2(const float2 *__restrict__ tab, int64_t base, int64_t sx,
                                         int64_t sy, float wx, float wy) {
  const float2 v00 = __ldg(tab + base), v01 = __ldg(tab + base + sx);
  const float2 v10 = __ldg(tab + base + sy), v11 = __ldg(tab + base + sy + sx);
  return make_float2(lerp(lerp(v00.x, v01.x, wx), lerp(v10.x, v11.x, wx), wy),
                     lerp(lerp(v00.y, v01.y, wx), lerp(v10.y, v11.y, wx), wy));
}
__device__ __forceinline__ bool lookup_tq(const PointCells &pc,
                                          const qpsdm_ttt_desc *__restrict__ dt,
                                          const float *__restrict__ ttt,
                                          const qpsdm_ttt_desc *__restrict__ dq,
                                          const float *__restrict__ qqq,
                                          const float2 *__restrict__ tq, int nxi1, int nzi1,
                                          float px, float py, float &t, float &q) {
  if (!tq || !pc.same) return lookup_tq(pc, dt, ttt, dq, qqq, nxi1, nzi1, px, py, t, q);
  const int nxs = pc.nxs, nys = pc.nys;
  float fx, fy;
  if (!grid_pos(px, py, pc.xc, pc.rdx, pc.rdy, pc.hx, pc.hy, nxs, nys, fx, fy)) return false;
  const int ix = min((int)fx, max(nxs - 2, 0));
  const int iy = min((int)fy, max(nys - 2, 0));
  const float wx = nxs > 1 ? __fsub_rn(fx, (float)ix) : 0.0f;
  const float wy = nys > 1 ? __fsub_rn(fy, (float)iy) : 0.0f;
  const int64_t plane = (int64_t)nxi1 * nzi1;
  const int64_t sx = nxs > 1 ? plane : 0, sy = nys > 1 ? (int64_t)nxs * plane : 0;
  const int64_t off = (int64_t)(iy * nxs + ix) * plane;
  const float2 a = bilin2(tq, pc.tA + off + pc.offA, sx, sy, wx, wy);
  const float2 b = bilin2(tq, pc.tB + off + pc.offB, sx, sy, wx, wy);
  t = lerp(a.x, b.x, pc.c2);
  q = lerp(a.y, b.y, pc.c2);
  return true;
}

constexpr int kPhysBz = 32, kPhysBx = 8, kPhysChunk = 256;

// Per-launch counters cnt[0..2] += the block's per-thread counts: point-traces
// (pairs in the aperture with table values at both ends), of which decided
// for a whole tile (members dropped before any point saw them), and imaged
// (past the dip test and the time window).  One atomic per counter and block.
__device__ __forceinline__ void add_counts(unsigned long long *cnt, unsigned long long *s,
                                           unsigned c0, unsigned c1, unsigned c2) {
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  const int nthr = blockDim.x * blockDim.y;
  if (tid < 3) s[tid] = 0;
  __syncthreads();
  for (int off = 16; off > 0; off >>= 1) {
    c0 += __shfl_down_sync(0xffffffffu, c0, off);
    c1 += __shfl_down_sync(0xffffffffu, c1, off);
    c2 += __shfl_down_sync(0xffffffffu, c2, off);
  }
  if ((tid & 31) == 0) {
    if (c0) atomicAdd(&s[0], (unsigned long long)c0);
    if (c1) atomicAdd(&s[1], (unsigned long long)c1);
    if (c2) atomicAdd(&s[2], (unsigned long long)c2);
  }
  __syncthreads();
  if (tid < 3 && s[tid]) atomicAdd(cnt + tid, s[tid]);
  (void)nthr;
}

template <typename T>
__global__ void __launch_bounds__(kPhysBz *kPhysBx)
    k_image_plain(float *__restrict__ img, float *__restrict__ comp, PhysImageArgs a,
                  const float *__restrict__ dips, const int *__restrict__ ints,
                  const float *__restrict__ geom, int ntr,
                  const qpsdm_ttt_desc *__restrict__ dt, const float *__restrict__ ttt,
                  const qpsdm_ttt_desc *__restrict__ dq, const float *__restrict__ qqq,
                  const T *__restrict__ panels, const float *__restrict__ pscale,
                  unsigned long long *npt) {
  __shared__ float4 s_geom[kPhysChunk];
  __shared__ int4 s_rng[kPhysChunk];
  __shared__ unsigned long long s_cnt[3];
  const int tid = threadIdx.y * kPhysBz + threadIdx.x;
  const int izi = blockIdx.x * kPhysBz + threadIdx.x;
  const int ixb = blockIdx.y * kPhysBx + threadIdx.y;
  const bool live = izi < a.nzi && ixb < a.nxb;
  const int ixi = ixb + a.ixstart;

  // per-point constants: cells, depth weights, dip limits
  PointCells pc;
  pc.ok = false;
  float tanx1 = 0.f, tanx2 = 0.f, tany1 = 0.f, tany2 = 0.f, acc = 0.f, cmp = 0.f;
  // Every operation below that feeds an index, a mask or the image is an
  // explicit IEEE operation (fused multiply-adds written out), so that the
  // FP32 C restatement in the oracle computes the same bits from the same
  // panels.
  const float z = __fmul_rn((float)izi, a.dzi);
  if (live) {
    const size_t k = (size_t)ixi * a.nzi + izi;
    tanx1 = dips[k];
    tanx2 = dips[a.nxz + k];
    tany1 = dips[2 * a.nxz + k];
    tany2 = dips[3 * a.nxz + k];
    acc = img[(size_t)ixb * a.nzi + izi];
    if (comp) cmp = comp[(size_t)ixb * a.nzi + izi];
    setup_cells(pc, ixi, z, a, dt, dq);
  }
  const float tz = a.taperzone;
  // tan -/+ tz (1 + tan^2): the limits widened by the taper zone
  const float tanx1c = __fsub_rn(tanx1, __fmul_rn(tz, __fmaf_rn(tanx1, tanx1, 1.0f)));
  const float tanx2c = __fadd_rn(tanx2, __fmul_rn(tz, __fmaf_rn(tanx2, tanx2, 1.0f)));
  const float tany1c = __fsub_rn(tany1, __fmul_rn(tz, __fmaf_rn(tany1, tany1, 1.0f)));
  const float tany2c = __fadd_rn(tany2, __fmul_rn(tz, __fmaf_rn(tany2, tany2, 1.0f)));
  const float z2 = __fmul_rn(z, z);
  const float x = __fmul_rn((float)ixi, a.dxi);
  const float inv_dt1 = __fdiv_rn(1.0f, a.dt1), inv_dts = __fdiv_rn(1.0f, a.dtstar);
  const size_t pstride = (size_t)a.nbins * a.nt;
  // source terms are reused while consecutive traces share a source
  float last_sx = NAN, last_sy = NAN, ts = 0.f, qs = 0.f;
  bool s_ok = false;
  unsigned cnt = 0, cimg = 0;

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
      const float4 gm = s_geom[i];
      if (gm.x != last_sx || gm.y != last_sy) {
        last_sx = gm.x;
        last_sy = gm.y;
        s_ok = lookup_tq(pc, dt, ttt, dq, qqq, a.nxi1, a.nzi1, gm.x, gm.y, ts, qs);
      }
      if (!s_ok) continue;
      float tg, qg;
      if (!lookup_tq(pc, dt, ttt, dq, qqq, a.nxi1, a.nzi1, gm.z, gm.w, tg, qg)) continue;
      ++cnt;  // a point-trace: in the aperture, table values at both ends
      // ray directions and dip taper (src/q-psdm.cu:2303-2340)
      const float dsx = __fsub_rn(gm.x, x), dgx = __fsub_rn(gm.z, x);
      const float ds = __fsqrt_rn(__fmaf_rn(dsx, dsx, __fmaf_rn(gm.y, gm.y, z2)));
      const float dg = __fsqrt_rn(__fmaf_rn(dgx, dgx, __fmaf_rn(gm.w, gm.w, z2)));
      const float rs = __fdiv_rn(1.0f, ds), rg2 = __fdiv_rn(1.0f, dg);
      const float ux = __fmaf_rn(dsx, rs, __fmul_rn(dgx, rg2));
      const float uy = __fmaf_rn(gm.y, rs, __fmul_rn(gm.w, rg2));
      const float uz = __fmul_rn(z, __fadd_rn(rs, rg2));
      const float tanx = __fdiv_rn(ux, uz), tany = __fdiv_rn(uy, uz);
      if (!(tanx > tanx1c && tanx < tanx2c && tany > tany1c && tany < tany2c)) continue;
      float w = 1.0f;
      if (tanx < tanx1)
        w = __fmul_rn(w, __fdiv_rn(__fsub_rn(tanx, tanx1c), __fsub_rn(tanx1, tanx1c)));
      if (tanx > tanx2)
        w = __fmul_rn(w, __fdiv_rn(__fsub_rn(tanx2c, tanx), __fsub_rn(tanx2c, tanx2)));
      if (tany < tany1)
        w = __fmul_rn(w, __fdiv_rn(__fsub_rn(tany, tany1c), __fsub_rn(tany1, tany1c)));
      if (tany > tany2)
        w = __fmul_rn(w, __fdiv_rn(__fsub_rn(tany2c, tany), __fsub_rn(tany2c, tany2)));
      // time and t* picks (src/q-psdm.cu:2354-2357)
      const float t = __fadd_rn(ts, tg);
      const float ft = __fmul_rn(t, inv_dt1);
      const int it1 = (int)ft;
      if (!(it1 > 0 && it1 + 1 < a.nt)) continue;
      ++cimg;
      const float wt = __fsub_rn(ft, (float)it1);
      const float fb = fminf(fmaxf(__fmul_rn(__fadd_rn(qs, qg), inv_dts), 0.0f),
                             (float)(a.nbins - 1));
      const int b0 = min((int)fb, a.nbins - 2);
      const float wb = __fsub_rn(fb, (float)b0);
      const T *pp = panels + (size_t)(c0 + i) * pstride + (size_t)b0 * a.nt + it1;
      const float p00 = ld_sample<T>(pp), p01 = ld_sample<T>(pp + 1);
      const float p10 = ld_sample<T>(pp + a.nt), p11 = ld_sample<T>(pp + a.nt + 1);
      float smp = lerp(lerp(p00, p01, wt), lerp(p10, p11, wt), wb);
      if (std::is_same<T, __half>::value) smp = __fmul_rn(smp, __ldg(pscale + c0 + i));
      // amplitude weight (src/q-psdm.cu:2366-2374): w v (r + 1/r),
      // r = (ds/dg)^3 tg/ts, v = 100 / t^2 (10^4 below 0.1 s)
      const float v = t > 0.1f ? __fdiv_rn(100.0f, __fmul_rn(t, t)) : 10000.0f;
      const float dr = __fmul_rn(ds, rg2);
      const float r = __fmul_rn(__fmul_rn(__fmul_rn(dr, dr), dr), __fdiv_rn(tg, ts));
      const float val =
          __fmul_rn(__fmul_rn(__fmul_rn(w, __fadd_rn(r, __fdiv_rn(1.0f, r))), v), smp);
      if (comp) {  // Kahan-compensated sum
        const float y = __fsub_rn(val, cmp);
        const float tt = __fadd_rn(acc, y);
        cmp = __fsub_rn(__fsub_rn(tt, acc), y);
        acc = tt;
      } else {
        acc = __fadd_rn(acc, val);
      }
    }
  }
  if (live) {
    img[(size_t)ixb * a.nzi + izi] = acc;
    if (comp) comp[(size_t)ixb * a.nzi + izi] = cmp;
  }
  if (npt) add_counts(npt, s_cnt, cnt, 0u, cimg);
}

// ---------------------------------------------------------------------------
// batched form
// ---------------------------------------------------------------------------
constexpr unsigned long long kNoKey = ~0ull;

// Receiver keys (accepted traces; position bits of the gate's relative
// coordinates), trace indices, and source-run flags from the raw headers.
__global__ void k_batch_keys(const uint8_t *__restrict__ rec, int rec_bytes, int be, int ntr,
                             const int *__restrict__ ints, const float *__restrict__ geom,
                             unsigned long long *__restrict__ key, int *__restrict__ val,
                             int *__restrict__ srcflag, int *__restrict__ naccepted) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  // accepted members of the batch (they sort first: rejected keys are the largest)
  const bool acc = i < ntr && ints[(size_t)i * kGateInts] == kAccepted;
  const unsigned ballot = __ballot_sync(0xffffffffu, acc);
  if ((threadIdx.x & 31) == 0 && ballot) atomicAdd(naccepted, __popc(ballot));
  if (i >= ntr) return;
  const uint8_t *r = rec + (size_t)i * rec_bytes;
  int flag = 1;
  if (i > 0) {
    const uint8_t *q = r - rec_bytes;
    flag = su_i32(r, kOffSx, be) != su_i32(q, kOffSx, be) ||
           su_i32(r, kOffSy, be) != su_i32(q, kOffSy, be);
  }
  srcflag[i] = flag;
  const bool ok = acc;
  const float gx = geom[(size_t)i * kGateF + 2], gy = geom[(size_t)i * kGateF + 3];
  key[i] = ok ? ((unsigned long long)__float_as_uint(gy) << 32) | __float_as_uint(gx) : kNoKey;
  val[i] = i;
}

// Receiver position of every receiver group (run of equal keys).
__global__ void k_batch_groups(const unsigned long long *__restrict__ ukey,
                               const int *__restrict__ nruns, float2 *__restrict__ grppos,
                               int ntr) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ntr || g >= *nruns) return;
  const unsigned long long k = ukey[g];  // rejected traces (kNoKey) are never imaged
  grppos[g] = make_float2(__uint_as_float((unsigned)(k & 0xffffffffu)),
                          __uint_as_float((unsigned)(k >> 32)));
}

// The group of every sorted position: the last run whose first position is
// at or before it (off: exclusive prefix sums of the run lengths).
__global__ void k_batch_memgrp(const int *__restrict__ off, const int *__restrict__ nruns,
                               int *__restrict__ memgrp, int ntr) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= ntr) return;
  int lo = 0, hi = *nruns;  // off[lo] <= p < off[hi] (off[nruns] taken as ntr)
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (off[mid] <= p) lo = mid; else hi = mid;
  }
  memgrp[p] = lo;
}

// Member info per sorted position (trace, source, column range) and the
// position of every source run (the gate's double-precision arithmetic).
__global__ void k_batch_members(const uint8_t *__restrict__ rec, int rec_bytes, int be, int ntr,
                                const int *__restrict__ sval, const int *__restrict__ ints,
                                const int *__restrict__ sid, const int *__restrict__ srcflag,
                                double scaled, double fxi, double cyi,
                                const float *__restrict__ pscale, int4 *__restrict__ mem,
                                float2 *__restrict__ srcpos) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= ntr) return;
  const int j = sval[p];
  const int *q = ints + (size_t)j * kGateInts;
  // member record: trace, source slot (bits 0-23) with the exponent of the
  // trace's FP16 sample multiplier + 128 (bits 24-31), cdp range
  int e = 0;
  if (pscale && q[0] == kAccepted) e = min(max(ilogbf(pscale[j]), -126), 127);
  mem[p] = q[0] == kAccepted ? make_int4(j, (sid[j] - 1) | ((e + 128) << 24), q[4], q[5])
                             : make_int4(j, -1, 1, 0);
  if (srcflag[p]) {  // p as a trace index: first trace of a source run
    const uint8_t *r = rec + (size_t)p * rec_bytes;
    const double sx = __dmul_rn((double)su_i32(r, kOffSx, be), scaled);
    const double sy = __dmul_rn((double)su_i32(r, kOffSy, be), scaled);
    srcpos[sid[p] - 1] = make_float2(__double2float_rn(__dsub_rn(sx, fxi)),
                                     __double2float_rn(__dsub_rn(sy, cyi)));
  }
}

// Source terms kept per (source, point) in shared memory, as four float2
// planes [plane][source][point]: (T, t* / dtstar), (CS = ds^3 / ts, AZ),
// (PX1, PX2), (PY1, PY2), with A the unit vector from the point to the source
// and
//   PX1 = AX - tanx1c AZ, PX2 = tanx2c AZ - AX   (PY likewise with tany)
// so that the dip test of a (source, receiver) pair needs no division: for
// uz = AZ + AZg > 0, tanx1c < ux / uz < tanx2c is PX1 > tanx1c AZg - AXg and
// PX2 > AXg - tanx2c AZg (the receiver's thresholds, once per receiver).
// The differences PX1 - (tanx1c AZg - AXg) etc. are the pair's dip-test
// functions, which also give the dip taper.
enum { kMapTQ = 0, kMapCZ, kMapPX, kMapPY, kMapN };

// Tile-level dip test.  A member (source S, receiver G) contributes to an
// image point P only if the bisector u = A_S + A_G of the unit vectors from
// P passes the four division-free dip tests
//   fx1 = ux - tanx1c uz > 0,  fx2 = tanx2c uz - ux > 0   (y likewise),
// so it can be dropped for a whole image tile when an upper bound of one of
// them over the tile is negative.  The bounds come from interval arithmetic
// over the tile's box (x in [x0, x1], y = 0 on the line, z in [z0, z1]) and
// the tile's ranges of the four dip limits; the margin 1e-4 max(1, |tan|)
// (|tan| the largest dip-limit tangent of the tile: the test functions'
// rounding grows with tan uz) covers the FP32 rounding of the per-point test,
// so no member that passes at some point of the tile is dropped (the kernel's
// sums are unchanged).
struct TileBox {
  float x0, x1, z0, z1;
  float t1lo, t1hi, t2lo, t2hi, u1lo, u1hi, u2lo, u2hi;  // tanx1c, tanx2c, tany1c, tany2c
  float margin;  // -1e-4 max(1, largest |tan| of the tile)
};
struct UnitBounds {
  float axl, axh, ayl, ayh, azl, azh;
  bool ok;
};
__device__ __forceinline__ UnitBounds unit_bounds(float px, float py, const TileBox &b) {
  UnitBounds u;
  const float dxl = px - b.x1, dxh = px - b.x0;
  const float adxmin = (dxl <= 0.0f && dxh >= 0.0f) ? 0.0f : fminf(fabsf(dxl), fabsf(dxh));
  const float adxmax = fmaxf(fabsf(dxl), fabsf(dxh));
  const float rmin2 = adxmin * adxmin + py * py + b.z0 * b.z0;
  const float rmax2 = adxmax * adxmax + py * py + b.z1 * b.z1;
  u.ok = rmin2 > 1e-6f;  // a point of the box (nearly) at the surface position: no bound
  // 1/rmin, 1/rmax (approximate reciprocal square roots: ~1e-7 relative,
  // far inside the test's margin)
  const float irmin = rsqrtf(fmaxf(rmin2, 1e-6f)), irmax = rsqrtf(fmaxf(rmax2, 1e-6f));
  u.axl = dxl >= 0.0f ? dxl * irmax : dxl * irmin;
  u.axh = dxh >= 0.0f ? dxh * irmin : dxh * irmax;
  u.ayl = py >= 0.0f ? py * irmax : py * irmin;
  u.ayh = py >= 0.0f ? py * irmin : py * irmax;
  u.azl = b.z0 * irmax;
  u.azh = b.z1 * irmin;
  return u;
}
// max of t * v over t in [tlo, thi], v in [vlo, vhi] (a corner of the box)
__device__ __forceinline__ float corner_max(float tlo, float thi, float vlo, float vhi) {
  return fmaxf(fmaxf(tlo * vlo, tlo * vhi), fmaxf(thi * vlo, thi * vhi));
}
__device__ __forceinline__ bool tile_keep(float2 sp, float2 gp, const TileBox &b) {
  const UnitBounds s = unit_bounds(sp.x, sp.y, b), g = unit_bounds(gp.x, gp.y, b);
  if (!s.ok || !g.ok) return true;
  const float uxl = s.axl + g.axl, uxh = s.axh + g.axh;
  const float uyl = s.ayl + g.ayl, uyh = s.ayh + g.ayh;
  const float uzl = s.azl + g.azl, uzh = s.azh + g.azh;
  const float fx1 = uxh + corner_max(-b.t1hi, -b.t1lo, uzl, uzh);
  const float fx2 = corner_max(b.t2lo, b.t2hi, uzl, uzh) - uxl;
  const float fy1 = uyh + corner_max(-b.u1hi, -b.u1lo, uzl, uzh);
  const float fy2 = corner_max(b.u2lo, b.u2hi, uzl, uzh) - uyl;
  const float m = b.margin;
  return !(fx1 < m || fx2 < m || fy1 < m || fy2 < m);  // NaN keeps the member
}

// The surface grid shared by every active point of a tile whose points all
// read the same table cells (one test decides a source's coverage for the
// whole tile).
struct TileGrid {
  float xc, rdx, rdy, hx, hy;
  int nxs, nys;
};
__device__ __forceinline__ bool tile_covers(const TileGrid &g, float2 p) {
  float fx, fy;
  return grid_pos(p.x, p.y, g.xc, g.rdx, g.rdy, g.hx, g.hy, g.nxs, g.nys, fx, fy);
}

template <int NW>
__device__ __forceinline__ float block_min(float v, float (*red)[NW], int k) {
  for (int off = 16; off > 0; off >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, off));
  if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = v;
  return v;
}

// Batched imaging.  A persistent CTA takes image tiles of TZ depths x TX
// cdps (one thread per point) from a counter.  Per tile and per chunk of sc
// sources: the source terms of every point in shared memory; then the
// members (traces in receiver order) in chunks of 32 x NT: the CTA keeps the
// members that pass the tile-level dip test (a bit mask), and every point
// runs over the kept members in order -- receiver terms once per receiver
// group, the members in blocks of U (the per-point aperture and dip tests,
// then the time/t* pick, weight and panel gathers).  Members dropped for the
// tile fail every point's dip test, so the image is that of running every
// member.  A point-trace is a pair in the trace's aperture whose source and
// receiver both have table values at the point: in a tile whose active
// points all read the same table cells (the usual case) one surface-grid
// test per member decides that for the whole tile, members outside the grid
// are dropped too, and a member dropped by the dip bound counts its
// in-aperture points; in any other tile every member goes to the points,
// which count for themselves.
template <int TZ, int TX, int MB, int U, typename T>
__global__ void __launch_bounds__(TZ *TX, MB)
    k_image_batched(float *__restrict__ img, float *__restrict__ comp, PhysImageArgs a,
                    const float *__restrict__ dips, const int *__restrict__ memgrp,
                    const float2 *__restrict__ grppos, const int4 *__restrict__ mem,
                    const int *__restrict__ nmem_ptr,
                    const float2 *__restrict__ srcpos, const int *__restrict__ nsrc_ptr,
                    const qpsdm_ttt_desc *__restrict__ dt, const float *__restrict__ ttt,
                    const qpsdm_ttt_desc *__restrict__ dq, const float *__restrict__ qqq,
                    const float2 *__restrict__ tqp, const T *__restrict__ panels,
                    int *__restrict__ tile_ctr, int ntz, int ntx, int sc,
                    unsigned long long *npt, const int *__restrict__ tile_list,
                    const int *__restrict__ ntile_list) {
  constexpr int NT = TZ * TX, NW = NT / 32, MC = 32 * NT;
  static_assert(NT % 32 == 0, "whole warps");
  const int nmem = *nmem_ptr;  // the accepted members (sorted first)
  extern __shared__ float2 smap[];  // [kMapN][sc][NT]
  __shared__ unsigned s_mask[NT];   // kept members of the chunk, one bit each
  __shared__ int s_col[TX + 1];     // active points of the tile's columns (prefix sums)
  __shared__ float s_red[13][NW];
  __shared__ TileGrid s_tg;         // the tile's shared surface grid (uniform tiles)
  __shared__ int s_tgw;             // the thread that writes it
  __shared__ int s_tile;
  __shared__ unsigned long long s_cnt[3];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int lz = tid % TZ, lx = tid / TZ;
  const int nsrc = *nsrc_ptr;
  const float inv_dt1 = 1.0f / a.dt1, inv_dts = 1.0f / a.dtstar;
  const size_t pstride = (size_t)a.nbins * a.nt;
  unsigned cnt = 0, cdrop = 0, cimg = 0;
  for (;;) {
    __syncthreads();
    if (tid == 0) {
      // the next tile: from the counter, or the next of a list of tiles
      const int q = atomicAdd(tile_ctr, 1);
      s_tile = tile_list ? (q < *ntile_list ? tile_list[q] : ntz * ntx) : q;
      s_tgw = -1;
    }
    if (tid <= TX) s_col[tid] = 0;
    __syncthreads();
    const int tile = s_tile;
    if (tile >= ntz * ntx) break;
    const int iz0 = (tile % ntz) * TZ, ixb0 = (tile / ntz) * TX;
    const int izi = iz0 + lz;
    const int ixb = ixb0 + lx;
    const bool live = izi < a.nzi && ixb < a.nxb;
    const int ixi = ixb + a.ixstart;
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
      setup_cells(pc, ixi, z, a, dt, dq);
    }
    const bool act = live && pc.ok;
    const float tz = a.taperzone;
    const float tanx1c = tanx1 - tz * (1.0f + tanx1 * tanx1);
    const float tanx2c = tanx2 + tz * (1.0f + tanx2 * tanx2);
    const float tany1c = tany1 - tz * (1.0f + tany1 * tany1);
    const float tany2c = tany2 + tz * (1.0f + tany2 * tany2);
    // inverse taper-zone widths: the taper factor at a passing pair is
    // min(1, f / (w uz)) for the test function f of each limit, w = |tan - tanc|
    const float iwx1 = 1.0f / (tanx1 - tanx1c), iwx2 = 1.0f / (tanx2c - tanx2);
    const float iwy1 = 1.0f / (tany1 - tany1c), iwy2 = 1.0f / (tany2c - tany2);
    const float z2 = z * z;
    const float x = ixi * a.dxi;
    // the tile's box and dip-limit ranges over its active points
    {
      const float big = 3.0e38f;
      block_min<NW>(act ? tanx1c : big, s_red, 0);
      block_min<NW>(act ? -tanx1c : big, s_red, 1);
      block_min<NW>(act ? tanx2c : big, s_red, 2);
      block_min<NW>(act ? -tanx2c : big, s_red, 3);
      block_min<NW>(act ? tany1c : big, s_red, 4);
      block_min<NW>(act ? -tany1c : big, s_red, 5);
      block_min<NW>(act ? tany2c : big, s_red, 6);
      block_min<NW>(act ? -tany2c : big, s_red, 7);
      // the table cells of the tile's points (exact in float: cells < 2^24)
      block_min<NW>(act ? (float)pc.cA : big, s_red, 8);
      block_min<NW>(act ? -(float)pc.cA : big, s_red, 9);
      block_min<NW>(act ? (float)pc.cB : big, s_red, 10);
      block_min<NW>(act ? -(float)pc.cB : big, s_red, 11);
      block_min<NW>(act ? (pc.same ? 0.0f : -1.0f) : big, s_red, 12);
      if (act) atomicAdd(&s_col[lx + 1], 1);
    }
    __syncthreads();
    if (tid == 0)
      for (int c = 1; c <= TX; ++c) s_col[c] += s_col[c - 1];
    TileBox box;
    bool uni;  // every active point reads the same cells on one surface grid
    {
      float r[13];
#pragma unroll
      for (int k = 0; k < 13; ++k) {
        r[k] = s_red[k][0];
#pragma unroll
        for (int w = 1; w < NW; ++w) r[k] = fminf(r[k], s_red[k][w]);
      }
      box.t1lo = r[0], box.t1hi = -r[1], box.t2lo = r[2], box.t2hi = -r[3];
      box.u1lo = r[4], box.u1hi = -r[5], box.u2lo = r[6], box.u2hi = -r[7];
      float tmax = 1.0f;
#pragma unroll
      for (int k = 0; k < 8; ++k) tmax = fmaxf(tmax, fabsf(r[k]));
      box.margin = -1e-4f * tmax;
      const int ncol = min(TX, a.nxb - ixb0), nrow = min(TZ, a.nzi - iz0);
      box.x0 = (ixb0 + a.ixstart) * a.dxi;
      box.x1 = (ixb0 + a.ixstart + ncol - 1) * a.dxi;
      box.z0 = iz0 * a.dzi;
      box.z1 = (iz0 + nrow - 1) * a.dzi;
      uni = r[8] == -r[9] && r[10] == -r[11] && r[12] == 0.0f;
      if (uni && act && atomicCAS(&s_tgw, -1, tid) == -1)
        s_tg = TileGrid{pc.xc, pc.rdx, pc.rdy, pc.hx, pc.hy, pc.nxs, pc.nys};
    }
    __syncthreads();  // s_col and s_tg complete
    if (s_col[TX] == 0) continue;  // no active point in the tile
    const int ixi_lo = ixb0 + a.ixstart, ixi_hi = ixi_lo + min(TX, a.nxb - ixb0) - 1;

    for (int s0 = 0; s0 < nsrc; s0 += sc) {
      const int ns = min(sc, nsrc - s0);
      // source terms of this chunk for this thread's point
      for (int s = 0; s < ns && act; ++s) {
        const float2 sp = srcpos[s0 + s];
        float ts, qs;
        float2 *m = smap + (size_t)s * NT + tid;
        if (!lookup_tq(pc, dt, ttt, dq, qqq, tqp, a.nxi1, a.nzi1, sp.x, sp.y, ts, qs)) {
          // no table value: NaN fails every member's dip test
          m[kMapTQ * sc * NT] = make_float2(NAN, 0.0f);
          m[kMapCZ * sc * NT] = make_float2(0.0f, NAN);
          m[kMapPX * sc * NT] = make_float2(NAN, NAN);
          m[kMapPY * sc * NT] = make_float2(NAN, NAN);
          continue;
        }
        const float dsx = sp.x - x;
        const float ds = sqrtf(dsx * dsx + sp.y * sp.y + z2);
        const float rds = __fdividef(1.0f, ds);
        const float ax = dsx * rds, ay = sp.y * rds, az = z * rds;
        m[kMapTQ * sc * NT] = make_float2(ts, qs * inv_dts);  // t* in bins
        // source factor of (ds/dg)^3 tg/ts
        m[kMapCZ * sc * NT] = make_float2(__fdividef(ds * ds * ds, ts), az);
        m[kMapPX * sc * NT] = make_float2(fmaf(-tanx1c, az, ax), fmaf(tanx2c, az, -ax));
        m[kMapPY * sc * NT] = make_float2(fmaf(-tany1c, az, ay), fmaf(tany2c, az, -ay));
      }
      for (int pc0 = 0; pc0 < nmem; pc0 += MC) {
        // the chunk's members kept for this tile (warp w, round k: word k NW + w)
#pragma unroll 4
        for (int k = 0; k < MC / NT; ++k) {
          const int wi = k * NW + warp;
          const int p = pc0 + 32 * wi + lane;
          bool keep = false;
          if (p < nmem) {
            const int4 mi = __ldg(mem + p);
            const int sl = (mi.y & 0xFFFFFF) - s0;
            const int lo = max(mi.z, ixi_lo), hi = min(mi.w, ixi_hi);
            if (sl >= 0 && sl < ns && lo <= hi) {
              if (uni) {
                const float2 sp = __ldg(srcpos + s0 + sl), gp = __ldg(grppos + __ldg(memgrp + p));
                const bool cov = tile_covers(s_tg, sp) && tile_covers(s_tg, gp);
                keep = cov && tile_keep(sp, gp, box);
                // dropped by the dip bound: its in-aperture points still count
                if (cov && !keep) cdrop += s_col[hi - ixi_lo + 1] - s_col[lo - ixi_lo];
              } else {
                keep = true;  // several cells in the tile: every point decides alone
              }
            }
          }
          const unsigned bits = __ballot_sync(0xffffffffu, keep);
          if (lane == 0) s_mask[wi] = bits;
        }
        __syncthreads();
        if (act) {
          // kept members in order: word w of the mask, remaining bits mw
          int w = 0;
          unsigned mw = s_mask[0];
          auto next = [&]() -> int {
            while (mw == 0) {
              if (++w >= NT) return -1;
              mw = s_mask[w];
            }
            const int b = __ffs(mw) - 1;
            mw &= mw - 1;
            return pc0 + 32 * w + b;
          };
          int nxt = next();
          int gn = nxt >= 0 ? __ldg(memgrp + nxt) : -1;
          int cur = -1;
          float agx = 0.f, agy = 0.f, agz = 0.f, qx1 = 0.f, qx2 = 0.f, qy1 = 0.f, qy2 = 0.f;
          float tg = 0.f, qg = 0.f, gfac = 0.f;
          bool rok = false;  // the current receiver has table values at this point
          while (nxt >= 0) {
            const int g = gn;
            if (g != cur) {
              cur = g;
              // receiver terms, once per receiver position
              const float2 gp = __ldg(grppos + g);
              rok = lookup_tq(pc, dt, ttt, dq, qqq, tqp, a.nxi1, a.nzi1, gp.x, gp.y, tg, qg);
              const float dgx = gp.x - x;
              const float rdg = rsqrtf(dgx * dgx + gp.y * gp.y + z2);  // 1 / dg
              agx = dgx * rdg, agy = gp.y * rdg, agz = z * rdg;
              // dip-test thresholds of this receiver (NaN: no table value,
              // every member fails)
              qx1 = rok ? fmaf(tanx1c, agz, -agx) : NAN;
              qx2 = fmaf(-tanx2c, agz, agx);
              qy1 = fmaf(tany1c, agz, -agy);
              qy2 = fmaf(-tany2c, agz, agy);
              gfac = tg * rdg * rdg * rdg;  // receiver factor of (ds/dg)^3 tg/ts
              qg *= inv_dts;                // t* in bins
            }
            // up to U kept members of this receiver group
            int pm[U];
            pm[0] = nxt;
            nxt = next();
            gn = nxt >= 0 ? __ldg(memgrp + nxt) : -1;
#pragma unroll
            for (int u = 1; u < U; ++u) {
              if (gn == g) {
                pm[u] = nxt;
                nxt = next();
                gn = nxt >= 0 ? __ldg(memgrp + nxt) : -1;
              } else {
                pm[u] = -1;
              }
            }
            // Phase 1, without branches, for all U: the member record, the
            // aperture check (counted), the source direction and the dip
            // test.  Phase 2: time/t* pick and weight of the members that
            // passed.  Then all panel gathers, then the sums (in member
            // order), so that U members' loads are in flight together.
            int4 mi[U];
#pragma unroll
            for (int u = 0; u < U; ++u)
              mi[u] = pm[u] >= 0 ? __ldg(mem + pm[u]) : make_int4(0, -1, 1, 0);
            bool on[U];
            int slv[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
              const int sl = (mi[u].y & 0xFFFFFF) - s0;
              const bool inr = (unsigned)sl < (unsigned)ns && ixi >= mi[u].z && ixi <= mi[u].w;
              slv[u] = inr ? sl : 0;
              const float2 *m = smap + (size_t)slv[u] * NT + tid;
              const float2 px = m[kMapPX * sc * NT], py = m[kMapPY * sc * NT];
              // source terms are NaN where the source has no table value
              cnt += (inr && rok && px.x == px.x) ? 1u : 0u;
              on[u] = inr && px.x > qx1 && px.y > qx2 && py.x > qy1 && py.y > qy2;
            }
            const T *pp[U];
            float fwt[U], fwb[U], fac[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
              pp[u] = panels;
              fwt[u] = fwb[u] = fac[u] = 0.0f;
              if (!on[u]) continue;
              on[u] = false;
              const float2 *m = smap + (size_t)slv[u] * NT + tid;
              const float2 tq = m[kMapTQ * sc * NT], cz = m[kMapCZ * sc * NT];
              const float2 px = m[kMapPX * sc * NT], py = m[kMapPY * sc * NT];
              const float ts = tq.x;
              // dip taper from the pair's test functions (ux - tanx1c uz and
              // the like, all > 0 here): (tanx - tanx1c) / (tanx1 - tanx1c) =
              // (ux - tanx1c uz) / ((tanx1 - tanx1c) uz) below tanx1, likewise
              // at the other three limits; of the two limits of an axis at
              // most one taper is active, so each axis takes the smaller ratio
              const float ruz = __fdividef(1.0f, cz.y + agz);
              const float ex = fminf((px.x - qx1) * iwx1, (px.y - qx2) * iwx2);
              const float ey = fminf((py.x - qy1) * iwy1, (py.y - qy2) * iwy2);
              const float wt = fminf(1.0f, ex * ruz) * fminf(1.0f, ey * ruz);
              const float t = ts + tg;
              const float ft = t * inv_dt1;
              const int it1 = (int)ft;
              if (!(it1 > 0 && it1 + 1 < a.nt)) continue;
              const float fb = fminf(fmaxf(tq.y + qg, 0.0f), (float)(a.nbins - 1));
              const int b0 = min((int)fb, a.nbins - 2);
              fwt[u] = ft - (float)it1;
              fwb[u] = fb - (float)b0;
              pp[u] = panels + (size_t)mi[u].x * pstride + (unsigned)(b0 * a.nt + it1);
              // w v (r + 1/r), v = 100 / t^2 (10^4 below 0.1 s), with one
              // reciprocal: w (r^2 + 1) * 100 / (r t^2)
              const float r = cz.x * gfac;
              const bool far = t > 0.1f;
              fac[u] = wt * fmaf(r, r, 1.0f) *
                       __fdividef(far ? 100.0f : 10000.0f, far ? r * t * t : r);
              if (std::is_same<T, __half>::value)  // 2^e from the record's exponent bits
                fac[u] *= __int_as_float((int)((((unsigned)mi[u].y >> 24) - 1u) << 23));
              on[u] = true;
              ++cimg;
            }
            float smp[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
              smp[u] = 0.0f;
              if (on[u]) {
                const T *q = pp[u];
                const float p00 = ld_sample<T>(q), p01 = ld_sample<T>(q + 1);
                const float p10 = ld_sample<T>(q + a.nt), p11 = ld_sample<T>(q + a.nt + 1);
                const float s0v = p00 + fwt[u] * (p01 - p00), s1v = p10 + fwt[u] * (p11 - p10);
                smp[u] = s0v + fwb[u] * (s1v - s0v);
              }
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
              if (!on[u]) continue;
              const float val = fac[u] * smp[u];
              if (comp) {
                const float y = val - cmp;
                const float tt = acc + y;
                cmp = (tt - acc) - y;
                acc = tt;
              } else {
                acc += val;
              }
            }
          }
        }
        __syncthreads();  // the mask is rewritten by the next chunk
      }
    }
    if (live) {
      img[(size_t)ixb * a.nzi + izi] = acc;
      if (comp) comp[(size_t)ixb * a.nzi + izi] = cmp;
    }
  }
  if (npt) add_counts(npt, s_cnt, cnt + cdrop, cdrop, cimg);
}

// Receiver (or source) lookup of a point in a uniform tile with paired
// (t, t*) tables: the tile's surface grid g, the point's two depth-node
// blocks pA, pB (the cell's data plus the point's offset inside a surface
// node's plane) and its depth weight c2.  The arithmetic of lookup_tq.
__device__ __forceinline__ bool lookup_uni(const TileGrid &g, const float2 *__restrict__ pA,
                                           const float2 *__restrict__ pB, float c2, int plane,
                                           float px, float py, float &t, float &q) {
  float fx, fy;
  if (!grid_pos(px, py, g.xc, g.rdx, g.rdy, g.hx, g.hy, g.nxs, g.nys, fx, fy)) return false;
  const int ix = min((int)fx, max(g.nxs - 2, 0));
  const int iy = min((int)fy, max(g.nys - 2, 0));
  const float wx = g.nxs > 1 ? __fsub_rn(fx, (float)ix) : 0.0f;
  const float wy = g.nys > 1 ? __fsub_rn(fy, (float)iy) : 0.0f;
  const int64_t sx = g.nxs > 1 ? plane : 0, sy = g.nys > 1 ? (int64_t)g.nxs * plane : 0;
  const int64_t off = (int64_t)(iy * g.nxs + ix) * plane;
  const float2 a = bilin2(pA, off, sx, sy, wx, wy);
  const float2 b = bilin2(pB, off, sx, sy, wx, wy);
  t = lerp(a.x, b.x, c2);
  q = lerp(a.y, b.y, c2);
  return true;
}

// Batched imaging, fast form: the same sums as k_image_batched for the tiles
// whose active points all read the same table cells of paired (t, t*)
// tables (with the tables' x-cells and depth cells aligned to the tile shape,
// every tile); any other tile is appended to defer[] (*ndefer of them) and
// left to k_image_batched.  The chunk's kept members are compacted in member
// order into shared memory (int4: trace, source slot | FP16 exponent bits,
// tile-local column range, receiver group), so that every point reads one
// broadcast record per member instead of scanning the keep mask and loading
// the member from global memory; the point-traces are counted per member in
// the keep pass (coverage is a tile-level test); lookups go through the
// tile's surface grid in shared memory and the point's two depth-node
// pointers.  Source terms are two float4 planes per (source, point):
// A = (T, t* / dtstar, CS = ds^3 / ts, AZ), B = (PX1, PX2, PY1, PY2).  One
// reciprocal per pair: inv = 1 / (uz r tt) gives both the taper's 1 / uz
// (r tt inv) and the weight's 1 / (r tt) (uz inv), tt = t^2 (0.01 below
// 0.1 s).  PK (two members per block): the two members' pick, weight and
// sample blend run as packed FP32 pairs (one f32x2 instruction for both
// members; minima, conversions and the sums stay scalar); every value that
// decides a pair -- t, t / dt1, the t* bin -- is the same IEEE add or
// multiply as in the scalar walk, so the same pairs are imaged.
template <int TZ, int TX, int MB, int U, int MW, bool PK, typename T>
__global__ void __launch_bounds__(TZ *TX, MB)
    k_image_batched_fast(float *__restrict__ img, float *__restrict__ comp, PhysImageArgs a,
                       const float *__restrict__ dips, const int *__restrict__ memgrp,
                       const float2 *__restrict__ grppos, const int4 *__restrict__ mem,
                       const int *__restrict__ nmem_ptr,
                       const float2 *__restrict__ srcpos, const int *__restrict__ nsrc_ptr,
                       const qpsdm_ttt_desc *__restrict__ dt, const float *__restrict__ ttt,
                       const qpsdm_ttt_desc *__restrict__ dq, const float *__restrict__ qqq,
                       const float2 *__restrict__ tqp, const T *__restrict__ panels,
                       int *__restrict__ tile_ctr, int ntz, int ntx, int sc,
                       unsigned long long *npt, int *__restrict__ defer,
                       int *__restrict__ ndefer) {
  constexpr int NT = TZ * TX, NW = NT / 32, MC = 32 * MW;
  static_assert(NT % 32 == 0 && MW % NW == 0, "whole warps, whole words per warp");
  const int nmem = *nmem_ptr;
  extern __shared__ float4 smap4[];  // [2][sc][NT]: plane A, plane B
  __shared__ int4 s_list[MC];        // the chunk's kept members, in member order
  __shared__ unsigned s_mask[MW];    // kept members of the chunk, one bit each
  __shared__ int s_wpos[MW + 1];     // kept members before word w (s_wpos[MW]: all)
  __shared__ int s_col[TX + 1];      // active points of the tile's columns (prefix sums)
  __shared__ float s_red[13][NW];
  __shared__ TileGrid s_tg;
  __shared__ TileBox s_box;  // the tile's box and dip-limit ranges (keep pass only)
  __shared__ int s_tgw;
  __shared__ int s_tile;
  __shared__ unsigned long long s_cnt[3];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int lz = tid % TZ, lx = tid / TZ;
  const int nsrc = *nsrc_ptr;
  const float inv_dt1 = 1.0f / a.dt1, inv_dts = 1.0f / a.dtstar;
  const size_t pstride = (size_t)a.nbins * a.nt;
  float4 *const planeA = smap4, *const planeB = smap4 + (size_t)sc * NT;
  unsigned cnt = 0, cdrop = 0, cimg = 0;
  for (;;) {
    __syncthreads();
    if (tid == 0) {
      s_tile = atomicAdd(tile_ctr, 1);
      s_tgw = -1;
    }
    if (tid <= TX) s_col[tid] = 0;
    __syncthreads();
    const int tile = s_tile;
    if (tile >= ntz * ntx) break;
    const int iz0 = (tile % ntz) * TZ, ixb0 = (tile / ntz) * TX;
    const int izi = iz0 + lz;
    const int ixb = ixb0 + lx;
    const bool live = izi < a.nzi && ixb < a.nxb;
    const int ixi = ixb + a.ixstart;
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
      setup_cells(pc, ixi, z, a, dt, dq);
    }
    const bool act = live && pc.ok;
    const float tz = a.taperzone;
    const float tanx1c = tanx1 - tz * (1.0f + tanx1 * tanx1);
    const float tanx2c = tanx2 + tz * (1.0f + tanx2 * tanx2);
    const float tany1c = tany1 - tz * (1.0f + tany1 * tany1);
    const float tany2c = tany2 + tz * (1.0f + tany2 * tany2);
    const float iwx1 = 1.0f / (tanx1 - tanx1c), iwx2 = 1.0f / (tanx2c - tanx2);
    const float iwy1 = 1.0f / (tany1 - tany1c), iwy2 = 1.0f / (tany2c - tany2);
    const float z2 = z * z;
    const float x = ixi * a.dxi;
    {
      const float big = 3.0e38f;
      block_min<NW>(act ? tanx1c : big, s_red, 0);
      block_min<NW>(act ? -tanx1c : big, s_red, 1);
      block_min<NW>(act ? tanx2c : big, s_red, 2);
      block_min<NW>(act ? -tanx2c : big, s_red, 3);
      block_min<NW>(act ? tany1c : big, s_red, 4);
      block_min<NW>(act ? -tany1c : big, s_red, 5);
      block_min<NW>(act ? tany2c : big, s_red, 6);
      block_min<NW>(act ? -tany2c : big, s_red, 7);
      block_min<NW>(act ? (float)pc.cA : big, s_red, 8);
      block_min<NW>(act ? -(float)pc.cA : big, s_red, 9);
      block_min<NW>(act ? (float)pc.cB : big, s_red, 10);
      block_min<NW>(act ? -(float)pc.cB : big, s_red, 11);
      block_min<NW>(act ? (pc.same ? 0.0f : -1.0f) : big, s_red, 12);
      if (act) atomicAdd(&s_col[lx + 1], 1);
    }
    __syncthreads();
    if (tid == 0)
      for (int c = 1; c <= TX; ++c) s_col[c] += s_col[c - 1];
    bool uni;
    {
      TileBox box;
      float r[13];
#pragma unroll
      for (int k = 0; k < 13; ++k) {
        r[k] = s_red[k][0];
#pragma unroll
        for (int w = 1; w < NW; ++w) r[k] = fminf(r[k], s_red[k][w]);
      }
      box.t1lo = r[0], box.t1hi = -r[1], box.t2lo = r[2], box.t2hi = -r[3];
      box.u1lo = r[4], box.u1hi = -r[5], box.u2lo = r[6], box.u2hi = -r[7];
      float tmax = 1.0f;
#pragma unroll
      for (int k = 0; k < 8; ++k) tmax = fmaxf(tmax, fabsf(r[k]));
      box.margin = -1e-4f * tmax;
      const int ncol = min(TX, a.nxb - ixb0), nrow = min(TZ, a.nzi - iz0);
      box.x0 = (ixb0 + a.ixstart) * a.dxi;
      box.x1 = (ixb0 + a.ixstart + ncol - 1) * a.dxi;
      box.z0 = iz0 * a.dzi;
      box.z1 = (iz0 + nrow - 1) * a.dzi;
      uni = r[8] == -r[9] && r[10] == -r[11] && r[12] == 0.0f;
      if (tid == 0) s_box = box;
      if (uni && act && atomicCAS(&s_tgw, -1, tid) == -1)
        s_tg = TileGrid{pc.xc, pc.rdx, pc.rdy, pc.hx, pc.hy, pc.nxs, pc.nys};
    }
    __syncthreads();
    if (s_col[TX] == 0) continue;
    if (!uni) {  // left to k_image_batched
      if (tid == 0) defer[atomicAdd(ndefer, 1)] = tile;
      continue;
    }
    const int ixi_lo = ixb0 + a.ixstart, ixi_hi = ixi_lo + min(TX, a.nxb - ixb0) - 1;
    const int plane = a.nxi1 * a.nzi1;
    const float2 *ptA = tqp, *ptB = tqp;
    if (act) {
      ptA = tqp + pc.tA + pc.offA;
      ptB = tqp + pc.tB + pc.offB;
    }
    const float c2 = pc.c2;

    for (int s0 = 0; s0 < nsrc; s0 += sc) {
      const int ns = min(sc, nsrc - s0);
      for (int s = 0; s < ns && act; ++s) {
        const float2 sp = srcpos[s0 + s];
        float ts, qs;
        float4 *mA = planeA + (size_t)s * NT + tid, *mB = planeB + (size_t)s * NT + tid;
        if (!lookup_uni(s_tg, ptA, ptB, c2, plane, sp.x, sp.y, ts, qs)) {
          // no table value: NaN fails every member's dip test
          *mA = make_float4(NAN, 0.0f, 0.0f, NAN);
          *mB = make_float4(NAN, NAN, NAN, NAN);
          continue;
        }
        const float dsx = sp.x - x;
        const float ds = sqrtf(dsx * dsx + sp.y * sp.y + z2);
        const float rds = __fdividef(1.0f, ds);
        const float ax = dsx * rds, ay = sp.y * rds, az = z * rds;
        *mA = make_float4(ts, qs * inv_dts, __fdividef(ds * ds * ds, ts), az);
        *mB = make_float4(fmaf(-tanx1c, az, ax), fmaf(tanx2c, az, -ax), fmaf(-tany1c, az, ay),
                          fmaf(tany2c, az, -ay));
      }
      for (int pc0 = 0; pc0 < nmem; pc0 += MC) {
        // keep pass: one bit per member of the chunk
#pragma unroll 4
        for (int k = 0; k < MW / NW; ++k) {
          const int wi = k * NW + warp;
          const int p = pc0 + 32 * wi + lane;
          bool keep = false;
          if (p < nmem) {
            const int4 mi = __ldg(mem + p);
            const int sl = (mi.y & 0xFFFFFF) - s0;
            const int lo = max(mi.z, ixi_lo), hi = min(mi.w, ixi_hi);
            if (sl >= 0 && sl < ns && lo <= hi) {
              const float2 sp = __ldg(srcpos + s0 + sl), gp = __ldg(grppos + __ldg(memgrp + p));
              if (tile_covers(s_tg, sp) && tile_covers(s_tg, gp)) {
                // every active point of columns lo..hi is a point-trace
                const unsigned n = s_col[hi - ixi_lo + 1] - s_col[lo - ixi_lo];
                cnt += n;
                keep = tile_keep(sp, gp, s_box);
                if (!keep) cdrop += n;
              }
            }
          }
          const unsigned bits = __ballot_sync(0xffffffffu, keep);
          if (lane == 0) s_mask[wi] = bits;
        }
        __syncthreads();
        if (warp == 0) {  // exclusive prefix of the words' kept counts
          int run = 0;
          for (int w0 = 0; w0 < MW; w0 += 32) {
            const int w = w0 + lane;
            int c = w < MW ? __popc(s_mask[w]) : 0;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
              const int v = __shfl_up_sync(0xffffffffu, c, off);
              if (lane >= off) c += v;
            }
            if (w < MW) s_wpos[w + 1] = run + c;
            run += __shfl_sync(0xffffffffu, c, 31);
          }
          if (lane == 0) s_wpos[0] = 0;
        }
        __syncthreads();
        // the kept members' records, in member order
#pragma unroll 4
        for (int k = 0; k < MW / NW; ++k) {
          const int wi = k * NW + warp;
          const unsigned bits = s_mask[wi];
          if (!((bits >> lane) & 1u)) continue;
          const int p = pc0 + 32 * wi + lane;
          const int4 mi = __ldg(mem + p);
          const int sl = (mi.y & 0xFFFFFF) - s0;
          const int lo = max(mi.z, ixi_lo) - ixi_lo, hi = min(mi.w, ixi_hi) - ixi_lo;
          s_list[s_wpos[wi] + __popc(bits & ((1u << lane) - 1u))] =
              make_int4(mi.x, sl | (int)((unsigned)mi.y & 0xFF000000u), (lo << 16) | hi,
                        __ldg(memgrp + p));
        }
        __syncthreads();
        const int nkept = s_wpos[MW];
        if (act && nkept > 0) {
          int cur = -1;
          float agz = 0.f, qx1 = 0.f, qx2 = 0.f, qy1 = 0.f, qy2 = 0.f;
          float tg = 0.f, qg = 0.f, gfac = 0.f;
          for (int k = 0; k < nkept;) {
            int4 rec[U];
            rec[0] = s_list[k];
            const int g = rec[0].w;
            if (g != cur) {
              cur = g;
              // receiver terms, once per receiver position (a kept member's
              // receiver lies on the tile's surface grid)
              const float2 gp = __ldg(grppos + g);
              const bool rok = lookup_uni(s_tg, ptA, ptB, c2, plane, gp.x, gp.y, tg, qg);
              const float dgx = gp.x - x;
              const float rdg = rsqrtf(dgx * dgx + gp.y * gp.y + z2);
              const float agx = dgx * rdg, agy = gp.y * rdg;
              agz = z * rdg;
              qx1 = rok ? fmaf(tanx1c, agz, -agx) : NAN;
              qx2 = fmaf(-tanx2c, agz, agx);
              qy1 = fmaf(tany1c, agz, -agy);
              qy2 = fmaf(-tany2c, agz, agy);
              gfac = tg * rdg * rdg * rdg;
              qg *= inv_dts;
            }
            // up to U kept members of this receiver group
            bool val[U];
            val[0] = true;
            ++k;
#pragma unroll
            for (int u = 1; u < U; ++u) {
              rec[u] = k < nkept ? s_list[k] : make_int4(0, 0, 0, -1);
              val[u] = rec[u].w == g;
              if (val[u]) ++k;
            }
            if constexpr (PK) {
              static_assert(U == 2, "packed walk: two members per block");
              bool on[2];
              float4 A[2], B[2];
#pragma unroll
              for (int u = 0; u < 2; ++u) {
                const int lo = rec[u].z >> 16, hi = rec[u].z & 0xFFFF;
                const bool inr = val[u] && (unsigned)(lx - lo) <= (unsigned)(hi - lo);
                B[u] = planeB[(size_t)(rec[u].y & 0xFF) * NT + tid];
                on[u] = inr && B[u].x > qx1 && B[u].y > qx2 && B[u].z > qy1 && B[u].w > qy2;
              }
              if (!(on[0] || on[1])) continue;
#pragma unroll
              for (int u = 0; u < 2; ++u) A[u] = planeA[(size_t)(rec[u].y & 0xFF) * NT + tid];
              const unsigned long long Ax = f2_pack(A[0].x, A[1].x), Ay = f2_pack(A[0].y, A[1].y);
              const unsigned long long Az = f2_pack(A[0].z, A[1].z), Aw = f2_pack(A[0].w, A[1].w);
              const unsigned long long uz = f2_add(Aw, f2_pack(agz, agz));
              const float2 ex1 = f2_unpack(f2_mul(f2_sub(f2_pack(B[0].x, B[1].x), f2_pack(qx1, qx1)),
                                                  f2_pack(iwx1, iwx1)));
              const float2 ex2 = f2_unpack(f2_mul(f2_sub(f2_pack(B[0].y, B[1].y), f2_pack(qx2, qx2)),
                                                  f2_pack(iwx2, iwx2)));
              const float2 ey1 = f2_unpack(f2_mul(f2_sub(f2_pack(B[0].z, B[1].z), f2_pack(qy1, qy1)),
                                                  f2_pack(iwy1, iwy1)));
              const float2 ey2 = f2_unpack(f2_mul(f2_sub(f2_pack(B[0].w, B[1].w), f2_pack(qy2, qy2)),
                                                  f2_pack(iwy2, iwy2)));
              const unsigned long long t = f2_add(Ax, f2_pack(tg, tg));
              const unsigned long long ft = f2_mul(t, f2_pack(inv_dt1, inv_dt1));
              const float2 ftv = f2_unpack(ft), tv = f2_unpack(t);
              const float2 fbr = f2_unpack(f2_add(Ay, f2_pack(qg, qg)));
              const int it0 = (int)ftv.x, it1v = (int)ftv.y;
              on[0] = on[0] && it0 > 0 && it0 + 1 < a.nt;
              on[1] = on[1] && it1v > 0 && it1v + 1 < a.nt;
              const float fb0 = fminf(fmaxf(fbr.x, 0.0f), (float)(a.nbins - 1));
              const float fb1 = fminf(fmaxf(fbr.y, 0.0f), (float)(a.nbins - 1));
              const int b00 = min((int)fb0, a.nbins - 2), b01 = min((int)fb1, a.nbins - 2);
              const unsigned long long fwt = f2_sub(ft, f2_pack((float)it0, (float)it1v));
              const unsigned long long fwb =
                  f2_sub(f2_pack(fb0, fb1), f2_pack((float)b00, (float)b01));
              // w v (r + 1/r) = w (r^2 + 1) 100 / (r tt), tt = t^2 (0.01 below 0.1 s)
              const unsigned long long r = f2_mul(Az, f2_pack(gfac, gfac));
              const float2 t2 = f2_unpack(f2_mul(t, t));
              const unsigned long long rtt =
                  f2_mul(r, f2_pack(tv.x > 0.1f ? t2.x : 0.01f, tv.y > 0.1f ? t2.y : 0.01f));
              const float2 den = f2_unpack(f2_mul(uz, rtt));
              const unsigned long long inv =
                  f2_pack(__fdividef(1.0f, den.x), __fdividef(1.0f, den.y));
              const unsigned long long ruz = f2_mul(rtt, inv);
              const float2 exr = f2_unpack(f2_mul(f2_pack(fminf(ex1.x, ex2.x), fminf(ex1.y, ex2.y)), ruz));
              const float2 eyr = f2_unpack(f2_mul(f2_pack(fminf(ey1.x, ey2.x), fminf(ey1.y, ey2.y)), ruz));
              const unsigned long long wt = f2_mul(f2_pack(fminf(1.0f, exr.x), fminf(1.0f, exr.y)),
                                                   f2_pack(fminf(1.0f, eyr.x), fminf(1.0f, eyr.y)));
              unsigned long long fac = f2_mul(f2_mul(wt, f2_fma(r, r, f2_pack(1.0f, 1.0f))),
                                              f2_mul(f2_mul(f2_pack(100.0f, 100.0f), uz), inv));
              if (std::is_same<T, __half>::value)  // 2^e from the records' exponent bits
                fac = f2_mul(fac, f2_pack(
                    __int_as_float((int)((((unsigned)rec[0].y >> 24) - 1u) << 23)),
                    __int_as_float((int)((((unsigned)rec[1].y >> 24) - 1u) << 23))));
              // samples (index clamped into the panel; loads only for imaged members)
              const T *q0 = panels + (size_t)rec[0].x * pstride +
                            (unsigned)(b00 * a.nt + min(max(it0, 0), a.nt - 2));
              const T *q1 = panels + (size_t)rec[1].x * pstride +
                            (unsigned)(b01 * a.nt + min(max(it1v, 0), a.nt - 2));
              float s00 = 0.f, s01 = 0.f, s10 = 0.f, s11 = 0.f;
              float u00 = 0.f, u01 = 0.f, u10 = 0.f, u11 = 0.f;
              if (on[0]) {
                s00 = ld_sample<T>(q0);
                s01 = ld_sample<T>(q0 + 1);
                s10 = ld_sample<T>(q0 + a.nt);
                s11 = ld_sample<T>(q0 + a.nt + 1);
              }
              if (on[1]) {
                u00 = ld_sample<T>(q1);
                u01 = ld_sample<T>(q1 + 1);
                u10 = ld_sample<T>(q1 + a.nt);
                u11 = ld_sample<T>(q1 + a.nt + 1);
              }
              const unsigned long long p00 = f2_pack(s00, u00), p01 = f2_pack(s01, u01);
              const unsigned long long p10 = f2_pack(s10, u10), p11 = f2_pack(s11, u11);
              const unsigned long long sa = f2_fma(fwt, f2_sub(p01, p00), p00);
              const unsigned long long sb = f2_fma(fwt, f2_sub(p11, p10), p10);
              const float2 v = f2_unpack(f2_mul(fac, f2_fma(fwb, f2_sub(sb, sa), sa)));
#pragma unroll
              for (int u = 0; u < 2; ++u) {
                if (!on[u]) continue;
                ++cimg;
                const float vu = u ? v.y : v.x;
                if (comp) {
                  const float y = vu - cmp;
                  const float tt = acc + y;
                  cmp = (tt - acc) - y;
                  acc = tt;
                } else {
                  acc += vu;
                }
              }
              continue;
            }
            bool on[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
              const int lo = rec[u].z >> 16, hi = rec[u].z & 0xFFFF;
              const bool inr = val[u] && (unsigned)(lx - lo) <= (unsigned)(hi - lo);
              const float4 B = planeB[(size_t)(rec[u].y & 0xFF) * NT + tid];
              on[u] = inr && B.x > qx1 && B.y > qx2 && B.z > qy1 && B.w > qy2;
            }
            const T *pp[U];
            float fwt[U], fwb[U], fac[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
              pp[u] = panels;
              fwt[u] = fwb[u] = fac[u] = 0.0f;
              if (!on[u]) continue;
              on[u] = false;
              const float4 A = planeA[(size_t)(rec[u].y & 0xFF) * NT + tid];
              const float4 B = planeB[(size_t)(rec[u].y & 0xFF) * NT + tid];
              const float uz = A.w + agz;
              const float ex = fminf((B.x - qx1) * iwx1, (B.y - qx2) * iwx2);
              const float ey = fminf((B.z - qy1) * iwy1, (B.w - qy2) * iwy2);
              const float t = A.x + tg;
              const float ft = t * inv_dt1;
              const int it1 = (int)ft;
              if (!(it1 > 0 && it1 + 1 < a.nt)) continue;
              const float fb = fminf(fmaxf(A.y + qg, 0.0f), (float)(a.nbins - 1));
              const int b0 = min((int)fb, a.nbins - 2);
              fwt[u] = ft - (float)it1;
              fwb[u] = fb - (float)b0;
              pp[u] = panels + (size_t)rec[u].x * pstride + (unsigned)(b0 * a.nt + it1);
              // w v (r + 1/r) = w (r^2 + 1) 100 / (r tt), tt = t^2 (0.01 below 0.1 s)
              const float r = A.z * gfac;
              const float rtt = r * (t > 0.1f ? t * t : 0.01f);
              const float inv = __fdividef(1.0f, uz * rtt);
              const float ruz = rtt * inv;
              const float wt = fminf(1.0f, ex * ruz) * fminf(1.0f, ey * ruz);
              fac[u] = wt * fmaf(r, r, 1.0f) * (100.0f * uz * inv);
              if (std::is_same<T, __half>::value)  // 2^e from the record's exponent bits
                fac[u] *= __int_as_float((int)((((unsigned)rec[u].y >> 24) - 1u) << 23));
              on[u] = true;
              ++cimg;
            }
            float smp[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
              smp[u] = 0.0f;
              if (on[u]) {
                const T *q = pp[u];
                const float p00 = ld_sample<T>(q), p01 = ld_sample<T>(q + 1);
                const float p10 = ld_sample<T>(q + a.nt), p11 = ld_sample<T>(q + a.nt + 1);
                const float s0v = p00 + fwt[u] * (p01 - p00), s1v = p10 + fwt[u] * (p11 - p10);
                smp[u] = s0v + fwb[u] * (s1v - s0v);
              }
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
              if (!on[u]) continue;
              const float v = fac[u] * smp[u];
              if (comp) {
                const float y = v - cmp;
                const float tt = acc + y;
                cmp = (tt - acc) - y;
                acc = tt;
              } else {
                acc += v;
              }
            }
          }
        }
        __syncthreads();  // s_mask, s_wpos and s_list are rewritten by the next chunk
      }
    }
    if (live) {
      img[(size_t)ixb * a.nzi + izi] = acc;
      if (comp) comp[(size_t)ixb * a.nzi + izi] = cmp;
    }
  }
  if (npt) add_counts(npt, s_cnt, cnt, cdrop, cimg);
}

static int batched_alloc(PhysicsState *s, const qpsdm_static_params &p) {
  const int n = p.max_batch;
  bool ok = true;
  for (GroupSet &g : s->sets) {
    for (int i = 0; i < 2; ++i) {
      ok &= cudaMalloc(&g.d_key[i], sizeof(unsigned long long) * n) == cudaSuccess;
      ok &= cudaMalloc(&g.d_val[i], sizeof(int) * n) == cudaSuccess;
    }
    ok &= cudaMalloc(&g.d_ukey, sizeof(unsigned long long) * n) == cudaSuccess;
    ok &= cudaMalloc(&g.d_count, sizeof(int) * n) == cudaSuccess;
    ok &= cudaMalloc(&g.d_off, sizeof(int) * n) == cudaSuccess;
    ok &= cudaMalloc(&g.d_nruns, sizeof(int)) == cudaSuccess;
    ok &= cudaMalloc(&g.d_srcflag, sizeof(int) * n) == cudaSuccess;
    ok &= cudaMalloc(&g.d_sid, sizeof(int) * n) == cudaSuccess;
    ok &= cudaMalloc(&g.d_srcpos, sizeof(float2) * n) == cudaSuccess;
    ok &= cudaMalloc(&g.d_mem, sizeof(int4) * n) == cudaSuccess;
    ok &= cudaMalloc(&g.d_grppos, sizeof(float2) * n) == cudaSuccess;
    ok &= cudaMalloc(&g.d_memgrp, sizeof(int) * n) == cudaSuccess;
    ok &= cudaMalloc(&g.d_tile_ctr, sizeof(int)) == cudaSuccess;
    ok &= cudaMalloc(&g.d_ndefer, sizeof(int)) == cudaSuccess;
    ok &= cudaMalloc(&g.d_nmem, sizeof(int)) == cudaSuccess;
  }
  if (!ok) return QPSDM_ENOMEM;
  GroupSet &g0 = s->sets[0];
  size_t b1 = 0, b2 = 0, b3 = 0, b4 = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, b1, g0.d_key[0], g0.d_key[1], g0.d_val[0],
                                  g0.d_val[1], n);
  cub::DeviceRunLengthEncode::Encode(nullptr, b2, g0.d_key[1], g0.d_ukey, g0.d_count,
                                     g0.d_nruns, n);
  cub::DeviceScan::ExclusiveSum(nullptr, b3, g0.d_count, g0.d_off, n);
  cub::DeviceScan::InclusiveSum(nullptr, b4, g0.d_srcflag, g0.d_sid, n);
  s->cub_bytes = std::max(std::max(b1, b2), std::max(b3, b4));
  for (GroupSet &g : s->sets)
    if (cudaMalloc(&g.d_cub, s->cub_bytes) != cudaSuccess) return QPSDM_ENOMEM;
  if (cudaStreamCreateWithFlags(&s->aux, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->ev_join, cudaEventDisableTiming) != cudaSuccess)
    return QPSDM_ECUDA;
  select_set(s, 0);
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, dev);
  if (p.tile_z > 0) s->tile_z = p.tile_z;
  if (p.tile_x > 0) s->tile_x = p.tile_x;
  s->forced_variant = p.variant;
  return QPSDM_OK;
}

// One line of the brick as the image kernels see it.
struct LineView {
  const int *ints;
  const float *geom;
  const float *dips;
  float *img;
  float *comp;
  const PhysicsState::LineTab *tab;
  const qpsdm_line_params *l;
};

// Launch variants of the batched kernel: image tile (depth x cdps, one
// thread per point; a warp spans min(TZ, 32) depths), the minimum resident
// blocks per SM the register allocation is held to, the sources per
// shared-memory chunk (more sources per chunk: fewer passes over the receiver
// groups, more shared memory per block) and the members per block U.  The
// autotuner times them all on the first batch and keeps the fastest.  (U = 8
// was slower everywhere tried: the extra registers cost more occupancy than
// the extra loads in flight gain.)
// Variants from 13 on are the fast form (k_image_batched_fast, with
// k_image_batched over the tiles it leaves) with mw words of 32 members per
// chunk; cl = 2: the walk on packed FP32 pairs.
struct BatchedVariant {
  int tz, tx, mb, sc, u, cl, mw;
};
static const BatchedVariant kVariants[] = {
    {32, 8, 2, 8, 4, 0, 0},   {32, 4, 4, 8, 4, 0, 0},   {32, 4, 6, 8, 4, 0, 0},
    {64, 4, 3, 8, 4, 0, 0},   {32, 4, 3, 16, 4, 0, 0},  {8, 16, 4, 8, 4, 0, 0},
    {4, 32, 4, 8, 4, 0, 0},   {16, 8, 4, 8, 4, 0, 0},   {8, 16, 4, 16, 4, 0, 0},
    {16, 8, 3, 16, 4, 0, 0},  {8, 16, 5, 8, 4, 0, 0},   {8, 16, 5, 16, 4, 0, 0},
    {16, 8, 5, 8, 4, 0, 0},   {8, 16, 5, 8, 4, 1, 16},  {8, 16, 4, 8, 4, 1, 32},
    {16, 8, 5, 8, 4, 1, 16},  {32, 4, 5, 8, 4, 1, 16},  {8, 16, 4, 16, 4, 1, 16},
    {16, 8, 4, 8, 4, 1, 32},  {8, 16, 6, 8, 2, 1, 8},   {8, 16, 6, 8, 4, 1, 8},
    {16, 8, 6, 8, 2, 1, 8},   {8, 16, 5, 8, 2, 1, 16},  {8, 16, 6, 8, 2, 2, 8},
    {8, 16, 5, 8, 2, 2, 8},
};
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);
static_assert(kNumVariants <= 32, "tune_ms holds 32 timings");

// The original kernel over every tile of the image, or (tile_list) over the
// *ntile_list tiles of a list, with one persistent CTA per SM.
template <int TZ, int TX, int MB, int U, typename T>
static int launch_batched_tile(PhysicsState *s, const PhysImageArgs &a, const PhysicsBatch &b,
                               const LineView &v, float *img, float *comp,
                               unsigned long long *npt, int sc, cudaStream_t st,
                               const int *tile_list = nullptr,
                               const int *ntile_list = nullptr) {
  const int ntz = (a.nzi + TZ - 1) / TZ, ntx = (a.nxb + TX - 1) / TX;
  const size_t smem = sizeof(float2) * kMapN * (size_t)sc * TZ * TX;
  auto kern = k_image_batched<TZ, TX, MB, U, T>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return QPSDM_ECUDA;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, TZ * TX, smem);
  const int grid = tile_list ? std::max(1, s->num_sms)
                             : std::max(1, std::min(ntz * ntx, std::max(per_sm, 1) * s->num_sms));
  cudaMemsetAsync(s->d_tile_ctr, 0, sizeof(int), st);
  kern<<<grid, TZ * TX, smem, st>>>(img, comp, a, v.dips, s->d_memgrp, s->d_grppos, s->d_mem,
                                    s->d_nmem, s->d_srcpos, s->d_sid + (b.ntr - 1), v.tab->dt,
                                    v.tab->ttt, v.tab->dq, v.tab->qqq,
                                    v.tab->paired ? v.tab->tq : nullptr, (const T *)s->d_panels,
                                    s->d_tile_ctr, ntz, ntx, sc, npt, tile_list, ntile_list);
  return cudaGetLastError() == cudaSuccess ? QPSDM_OK : QPSDM_ECUDA;
}

// The fast form over the image's uniform tiles, then the original kernel
// (same tile shape, MBO blocks per SM) over the tiles it left; with unpaired
// tables the original kernel takes every tile.
template <int TZ, int TX, int MB, int U, int MW, int MBO, typename T, bool PK = false>
static int launch_batched_fast(PhysicsState *s, const PhysImageArgs &a, const PhysicsBatch &b,
                               const LineView &v, float *img, float *comp,
                               unsigned long long *npt, int sc, cudaStream_t st) {
  if (!v.tab->paired)
    return launch_batched_tile<TZ, TX, MBO, 4, T>(s, a, b, v, img, comp, npt, sc, st);
  const int ntz = (a.nzi + TZ - 1) / TZ, ntx = (a.nxb + TX - 1) / TX;
  if ((size_t)ntz * ntx > s->defer_cap) return QPSDM_EINVAL;  // cannot happen: sized per offset
  const size_t smem = sizeof(float4) * 2 * (size_t)sc * TZ * TX;
  auto kern = k_image_batched_fast<TZ, TX, MB, U, MW, PK, T>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return QPSDM_ECUDA;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, TZ * TX, smem);
  const int grid = std::max(1, std::min(ntz * ntx, std::max(per_sm, 1) * s->num_sms));
  cudaMemsetAsync(s->d_tile_ctr, 0, sizeof(int), st);
  cudaMemsetAsync(s->d_ndefer, 0, sizeof(int), st);
  kern<<<grid, TZ * TX, smem, st>>>(img, comp, a, v.dips, s->d_memgrp, s->d_grppos, s->d_mem,
                                    s->d_nmem, s->d_srcpos, s->d_sid + (b.ntr - 1), v.tab->dt,
                                    v.tab->ttt, v.tab->dq, v.tab->qqq, v.tab->tq,
                                    (const T *)s->d_panels, s->d_tile_ctr, ntz, ntx, sc, npt,
                                    s->d_defer, s->d_ndefer);
  if (cudaGetLastError() != cudaSuccess) return QPSDM_ECUDA;
  return launch_batched_tile<TZ, TX, MBO, 4, T>(s, a, b, v, img, comp, npt, sc, st, s->d_defer,
                                                s->d_ndefer);
}

template <typename T>
static int launch_variant(int vi, PhysicsState *s, const PhysImageArgs &a, const PhysicsBatch &b,
                          const LineView &v, float *img, float *comp, unsigned long long *npt,
                          cudaStream_t st) {
  const int sc = kVariants[vi].sc;
  switch (vi) {
    case 13: return launch_batched_fast<8, 16, 5, 4, 16, 4, T>(s, a, b, v, img, comp, npt, sc, st);
    case 14: return launch_batched_fast<8, 16, 4, 4, 32, 4, T>(s, a, b, v, img, comp, npt, sc, st);
    case 15: return launch_batched_fast<16, 8, 5, 4, 16, 4, T>(s, a, b, v, img, comp, npt, sc, st);
    case 16: return launch_batched_fast<32, 4, 5, 4, 16, 4, T>(s, a, b, v, img, comp, npt, sc, st);
    case 17: return launch_batched_fast<8, 16, 4, 4, 16, 4, T>(s, a, b, v, img, comp, npt, sc, st);
    case 18: return launch_batched_fast<16, 8, 4, 4, 32, 4, T>(s, a, b, v, img, comp, npt, sc, st);
    case 19: return launch_batched_fast<8, 16, 6, 2, 8, 4, T>(s, a, b, v, img, comp, npt, sc, st);
    case 20: return launch_batched_fast<8, 16, 6, 4, 8, 4, T>(s, a, b, v, img, comp, npt, sc, st);
    case 21: return launch_batched_fast<16, 8, 6, 2, 8, 4, T>(s, a, b, v, img, comp, npt, sc, st);
    case 22: return launch_batched_fast<8, 16, 5, 2, 16, 4, T>(s, a, b, v, img, comp, npt, sc, st);
    case 23: return launch_batched_fast<8, 16, 6, 2, 8, 4, T, true>(s, a, b, v, img, comp, npt, sc, st);
    case 24: return launch_batched_fast<8, 16, 5, 2, 8, 4, T, true>(s, a, b, v, img, comp, npt, sc, st);
    case 0: return launch_batched_tile<32, 8, 2, 4, T>(s, a, b, v, img, comp, npt, sc, st);
    case 1: return launch_batched_tile<32, 4, 4, 4, T>(s, a, b, v, img, comp, npt, sc, st);
    case 2: return launch_batched_tile<32, 4, 6, 4, T>(s, a, b, v, img, comp, npt, sc, st);
    case 3: return launch_batched_tile<64, 4, 3, 4, T>(s, a, b, v, img, comp, npt, sc, st);
    case 4: return launch_batched_tile<32, 4, 3, 4, T>(s, a, b, v, img, comp, npt, sc, st);
    case 5: return launch_batched_tile<8, 16, 4, 4, T>(s, a, b, v, img, comp, npt, sc, st);
    case 6: return launch_batched_tile<4, 32, 4, 4, T>(s, a, b, v, img, comp, npt, sc, st);
    case 7: return launch_batched_tile<16, 8, 4, 4, T>(s, a, b, v, img, comp, npt, sc, st);
    case 8: return launch_batched_tile<8, 16, 4, 4, T>(s, a, b, v, img, comp, npt, sc, st);
    case 9: return launch_batched_tile<16, 8, 3, 4, T>(s, a, b, v, img, comp, npt, sc, st);
    case 10:
    case 11: return launch_batched_tile<8, 16, 5, 4, T>(s, a, b, v, img, comp, npt, sc, st);
    case 12: return launch_batched_tile<16, 8, 5, 4, T>(s, a, b, v, img, comp, npt, sc, st);
    default: return QPSDM_EINVAL;
  }
}

// Tuning results shared by the engines of a process:
// (device, nzi, nxb, dtype, nbins) -> variant.
static std::mutex g_tune_mu;
static std::map<std::tuple<int, int, int, int, int>, int> g_tune;

// Picks the variant for this image shape: an explicit tile from the static
// parameters, a cached result, or a timing of every variant on this batch
// into a scratch image (synchronous; happens on the first batch only).
template <typename T>
static int choose_variant(PhysicsState *s, const PhysImageArgs &a, const PhysicsBatch &b,
                          const LineView &v, cudaStream_t st) {
  if (s->variant >= 0) return s->variant;
  if (s->forced_variant > 0 && s->forced_variant <= kNumVariants)
    return s->variant = s->forced_variant - 1;
  if (s->tile_z > 0 && s->tile_x > 0) {
    for (int i = 0; i < kNumVariants; ++i)
      if (kVariants[i].tz == s->tile_z && kVariants[i].tx == s->tile_x) return s->variant = i;
  }
  int dev = 0;
  cudaGetDevice(&dev);
  const auto key = std::make_tuple(dev, a.nzi, a.nxb, s->dtype, s->nbins);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) return s->variant = it->second;
  }
  float *scratch = s->d_tune;
  const size_t n = (size_t)a.nxb * a.nzi;
  if (!scratch || s->tune_cap < n) return s->variant = 2;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int best = 2;
  float best_ms = 1e30f;
  for (int i = 0; i < kNumVariants; ++i) {
    cudaMemsetAsync(scratch, 0, sizeof(float) * n, st);
    cudaEventRecord(e0, st);
    const int rc = launch_variant<T>(i, s, a, b, v, scratch, nullptr, nullptr, st);
    cudaEventRecord(e1, st);
    if (rc || cudaEventSynchronize(e1) != cudaSuccess) continue;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    s->tune_ms[i] = ms;
    if (ms < best_ms) {
      best_ms = ms;
      best = i;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaGetLastError();
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[key] = best;
  return s->variant = best;
}

template <typename T>
static int launch_batched_image(PhysicsState *s, const PhysImageArgs &a, const PhysicsBatch &b,
                                const LineView &v, cudaStream_t st) {
  const int vi = choose_variant<T>(s, a, b, v, st);
  return launch_variant<T>(vi, s, a, b, v, v.img, v.comp, b.d_npt, st);
}

// Grouping of one batch (all on the stream, nothing read back).
static int batched_group(PhysicsState *s, const qpsdm_static_params &p, const LineView &v,
                         const PhysicsBatch &b, cudaStream_t st) {
  const qpsdm_line_params &l = *v.l;
  const int n = b.ntr, blk = 256, grd = (n + blk - 1) / blk;
  cudaMemsetAsync(s->d_nmem, 0, sizeof(int), st);
  k_batch_keys<<<grd, blk, 0, st>>>(b.d_rec, b.rec_bytes, b.big_endian, n, v.ints, v.geom,
                                    s->d_key[0], s->d_val[0], s->d_srcflag, s->d_nmem);
  size_t tb = s->cub_bytes;
  if (cub::DeviceScan::InclusiveSum(s->d_cub, tb, s->d_srcflag, s->d_sid, n, st) != cudaSuccess)
    return QPSDM_ECUDA;
  tb = s->cub_bytes;
  if (cub::DeviceRadixSort::SortPairs(s->d_cub, tb, s->d_key[0], s->d_key[1], s->d_val[0],
                                      s->d_val[1], n, 0, 64, st) != cudaSuccess)
    return QPSDM_ECUDA;
  cudaMemsetAsync(s->d_count, 0, sizeof(int) * n, st);
  tb = s->cub_bytes;
  if (cub::DeviceRunLengthEncode::Encode(s->d_cub, tb, s->d_key[1], s->d_ukey, s->d_count,
                                         s->d_nruns, n, st) != cudaSuccess)
    return QPSDM_ECUDA;
  tb = s->cub_bytes;
  if (cub::DeviceScan::ExclusiveSum(s->d_cub, tb, s->d_count, s->d_off, n, st) != cudaSuccess)
    return QPSDM_ECUDA;
  k_batch_groups<<<grd, blk, 0, st>>>(s->d_ukey, s->d_nruns, s->d_grppos, n);
  k_batch_memgrp<<<grd, blk, 0, st>>>(s->d_off, s->d_nruns, s->d_memgrp, n);
  k_batch_members<<<grd, blk, 0, st>>>(b.d_rec, b.rec_bytes, b.big_endian, n, s->d_val[1],
                                       v.ints, s->d_sid, s->d_srcflag, p.scaled, l.fxi, l.cyi,
                                       s->dtype == QPSDM_PANEL_FP16 ? s->d_pscale : nullptr,
                                       s->d_mem, s->d_srcpos);
  return cudaGetLastError() == cudaSuccess ? QPSDM_OK : QPSDM_ECUDA;
}

// Any line of the brick accepted the trace: its panels are needed.
__global__ void k_any_line(const int *__restrict__ ints, size_t ints_ls, int nlines, int ntr,
                           unsigned long long mask, int *__restrict__ any) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ntr) return;
  int a = 0;
  for (int il = 0; il < nlines; ++il)
    if (il >= 64 || ((mask >> il) & 1ull))
      a |= ints[il * ints_ls + (size_t)i * kGateInts] == kAccepted;
  any[i] = a ? kAccepted : 0;
}

// Forward spectra and t*-binned panels of the traces whose status is kAccepted.
static int run_panels(PhysicsState *s, const qpsdm_static_params &p, const PhysicsBatch &b,
                      const int *status, int sstride, cudaStream_t st, std::string *err) {
  FftPlan pf, pi;
  int rc = fft_plan(p.nfft, &pf, err);
  if (rc) return rc;
  rc = fft_plan(p.nffti, &pi, err);
  if (rc) return rc;
  const int ntr = b.ntr;
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  // persistent grids: as many CTAs as fit on the GPU, at most one per trace
  auto grid_of = [&](const void *kern, size_t smem) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, smem);
    return std::max(1, std::min(ntr, std::max(per_sm, 1) * std::max(nsm, 1)));
  };
  size_t sm = fft_smem_bytes(pf.m);
  if ((rc = fft_set_smem_attr((const void *)k_phys_fwd, sm))) return rc;
  const bool fp16 = s->dtype == QPSDM_PANEL_FP16;
  k_phys_fwd<<<grid_of((const void *)k_phys_fwd, sm), 256, sm, st>>>(
      b.d_rec, b.rec_bytes, b.big_endian, status, sstride, ntr, p.ntl, p.dt, b.d_taper200, pf,
      s->d_spec, s->d_fmax, fp16 ? s->d_pscale : nullptr);
  const int nk = p.nfft / 2 + 1;
  sm = fft_smem_bytes(pi.m) + sizeof(float2) * (size_t)nk;
  switch (s->dtype) {
    case QPSDM_PANEL_FP32: {
      const void *k = (const void *)k_phys_panels<float>;
      if ((rc = fft_set_smem_attr(k, sm))) return rc;
      k_phys_panels<float><<<grid_of(k, sm), 256, sm, st>>>(
          status, sstride, ntr, s->d_spec, nk, s->d_filter, pi, s->nbins,
          (float *)s->d_panels, nullptr);
      break;
    }
    case QPSDM_PANEL_BF16: {
      const void *k = (const void *)k_phys_panels<__nv_bfloat16>;
      if ((rc = fft_set_smem_attr(k, sm))) return rc;
      k_phys_panels<__nv_bfloat16><<<grid_of(k, sm), 256, sm, st>>>(
          status, sstride, ntr, s->d_spec, nk, s->d_filter, pi, s->nbins,
          (__nv_bfloat16 *)s->d_panels, nullptr);
      break;
    }
    default: {
      const void *k = (const void *)k_phys_panels<__half>;
      if ((rc = fft_set_smem_attr(k, sm))) return rc;
      k_phys_panels<__half><<<grid_of(k, sm), 256, sm, st>>>(
          status, sstride, ntr, s->d_spec, nk, s->d_filter, pi, s->nbins,
          (__half *)s->d_panels, s->d_pscale);
    }
  }
  return cudaGetLastError() == cudaSuccess ? QPSDM_OK : QPSDM_ECUDA;
}

static PhysImageArgs image_args(const PhysicsState *s, const qpsdm_static_params &p,
                                const qpsdm_line_params &l, const qpsdm_offset_params &o,
                                size_t nxz) {
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
  a.nxz = nxz;
  a.xfast = s->form == QPSDM_FORM_BATCHED;
  return a;
}

template <typename T>
static void launch_plain(const PhysImageArgs &a, const PhysicsBatch &b, const LineView &v,
                         const T *panels, const float *pscale, cudaStream_t st) {
  dim3 block(kPhysBz, kPhysBx);
  dim3 grid((a.nzi + kPhysBz - 1) / kPhysBz, (a.nxb + kPhysBx - 1) / kPhysBx);
  k_image_plain<T><<<grid, block, 0, st>>>(v.img, v.comp, a, v.dips, v.ints, v.geom, b.ntr,
                                           v.tab->dt, v.tab->ttt, v.tab->dq, v.tab->qqq,
                                           panels, pscale, b.d_npt);
}

int physics_process(PhysicsState *s, const qpsdm_static_params &p,
                    const qpsdm_line_params *lines, const qpsdm_offset_params &o,
                    const PhysicsBatch &b, cudaStream_t st, std::string *err) {
  if (s->ntabs < b.nlines) {
    if (err) *err = "physics mode: set_line without tables";
    return QPSDM_ESTATE;
  }
  const size_t nimg = (size_t)(o.ixend - o.ixstart) * p.nzi;
  auto view = [&](int il) {
    LineView v;
    v.ints = b.d_ints + il * b.ints_ls;
    v.geom = b.d_geom + il * b.geom_ls;
    v.dips = b.d_dips + (size_t)il * 4 * b.nxz;
    v.img = b.d_img + il * b.img_ls;
    v.comp = p.kahan ? s->d_comp + il * nimg : nullptr;
    v.tab = &s->tabs[il];
    v.l = &lines[il];
    return v;
  };
  int rc = QPSDM_OK;
  if (s->form == QPSDM_FORM_PLAIN) {
    // as the reference: each line preprocesses its accepted traces again
    for (int il = 0; il < b.nlines && !rc; ++il) {
      if (!batch_line_on(b, il)) continue;
      const LineView v = view(il);
      b.prof->begin(QPSDM_K_PRE, st);
      rc = run_panels(s, p, b, v.ints, kGateInts, st, err);
      b.prof->end(st);
      if (rc) break;
      const PhysImageArgs a = image_args(s, p, lines[il], o, b.nxz);
      b.prof->begin(QPSDM_K_IMAGE, st);
      if (s->dtype == QPSDM_PANEL_FP32)
        launch_plain<float>(a, b, v, (const float *)s->d_panels, s->d_pscale, st);
      else if (s->dtype == QPSDM_PANEL_BF16)
        launch_plain<__nv_bfloat16>(a, b, v, (const __nv_bfloat16 *)s->d_panels, s->d_pscale,
                                    st);
      else
        launch_plain<__half>(a, b, v, (const __half *)s->d_panels, s->d_pscale, st);
      b.prof->end(st);
      if (cudaGetLastError() != cudaSuccess) rc = QPSDM_ECUDA;
    }
    if (rc && err && err->empty()) *err = "physics launch failed";
    return rc;
  }
  // batched: panels once for every trace any line accepted, shared by the brick
  b.prof->begin(QPSDM_K_PRE, st);
  k_any_line<<<(b.ntr + 255) / 256, 256, 0, st>>>(b.d_ints, b.ints_ls, b.nlines, b.ntr,
                                                  b.line_mask, s->d_any);
  rc = run_panels(s, p, b, s->d_any, 1, st, err);
  b.prof->end(st);
  if (rc) return rc;
  // Lines alternate between the engine's stream (grouping set 0) and the
  // second stream (set 1), which starts after the panels; the engine's stream
  // waits for the second one before returning, so the next batch (which
  // rewrites the panels) and any read of the image come after every line.
  int nactive = 0;
  for (int il = 0; il < b.nlines; ++il) nactive += batch_line_on(b, il);
  const bool forked = nactive > 1;
  if (forked && (cudaEventRecord(s->ev_fork, st) != cudaSuccess ||
                 cudaStreamWaitEvent(s->aux, s->ev_fork, 0) != cudaSuccess))
    return QPSDM_ECUDA;
  int nrun = 0;
  for (int il = 0; il < b.nlines && !rc; ++il) {
    if (!batch_line_on(b, il)) continue;
    const int set = nrun++ & 1;
    cudaStream_t ss = set ? s->aux : st;
    select_set(s, set);
    const LineView v = view(il);
    b.prof->begin(QPSDM_K_OTHER, ss);
    rc = batched_group(s, p, v, b, ss);
    b.prof->end(ss);
    if (rc) {
      if (err) *err = "batched grouping failed";
      break;
    }
    const PhysImageArgs a = image_args(s, p, lines[il], o, b.nxz);
    b.prof->begin(QPSDM_K_IMAGE, ss);
    if (s->dtype == QPSDM_PANEL_FP32)
      rc = launch_batched_image<float>(s, a, b, v, ss);
    else if (s->dtype == QPSDM_PANEL_BF16)
      rc = launch_batched_image<__nv_bfloat16>(s, a, b, v, ss);
    else
      rc = launch_batched_image<__half>(s, a, b, v, ss);
    b.prof->end(ss);
    if (rc && err) *err = "batched image launch failed";
  }
  if (forked && (cudaEventRecord(s->ev_join, s->aux) != cudaSuccess ||
                 cudaStreamWaitEvent(st, s->ev_join, 0) != cudaSuccess) && !rc)
    rc = QPSDM_ECUDA;
  select_set(s, 0);
  return rc;
}

int physics_tuning(const PhysicsState *s, int *variant, int *tz, int *tx, int *mb,
                   float *times, int ntimes) {
  if (!s) return QPSDM_ESTATE;
  const int v = s->variant;
  if (variant) *variant = v;
  if (tz) *tz = v >= 0 ? kVariants[v].tz : 0;
  if (tx) *tx = v >= 0 ? kVariants[v].tx : 0;
  if (mb) *mb = v >= 0 ? kVariants[v].mb : 0;
  for (int i = 0; times && i < ntimes && i < kNumVariants; ++i) times[i] = s->tune_ms[i];
  return kNumVariants;
}

void physics_panels(const PhysicsState *s, void **d_panels, float **d_pscale) {
  *d_panels = s->d_panels;
  *d_pscale = s->d_pscale;
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
