// engine.cu -- the C ABI of include/qpsdm_engine.h.
//
// Replaces the reference's threading and per-trace launch structure
// (safe_queue + producer/consumer pthreads, src/queue.h:12-72,
// src/q-psdm.cu:1693-1738, :1862-2061, and one synchronous launch per trace
// in psdm_kernel, src/q-psdm.cu:2218-2243) with a single-GPU pipeline:
//
//   host records --memcpy--> pinned staging slot (2 slots)
//                --cudaMemcpyAsync on the copy stream--> device record slot
//                --event--> compute stream: gate -> spectra/panels -> image
//
// The copy of batch i+1 overlaps the kernels of batch i.  All device memory
// is allocated at create / set_line / begin_offset; submits allocate nothing.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "common.cuh"
#include "internal.h"
#include "physics.h"
#include "qpsdm_engine.h"

using namespace qpsdm;

struct qpsdm_engine {
  int device = 0;
  unsigned long long line_mask = ~0ull;  // lines of the brick the next batches feed
  qpsdm_static_params p{};
  std::string err;
  cudaStream_t s_comp = nullptr, s_copy = nullptr;
  cudaStream_t s_own = nullptr;  // the engine's own compute stream
  // per-slot events: staging slot reusable / device slot filled / device slot free
  cudaEvent_t ev_stage_free[2] = {}, ev_rec_ready[2] = {}, ev_rec_free[2] = {};
  int slot = 0;
  size_t rec_bytes = 0;
  int naztab = 0;
  // static device buffers
  int *d_iaztab = nullptr;
  float *d_taper200 = nullptr;
  uint8_t *d_rec[2] = {};
  uint8_t *h_stage[2] = {};
  int *d_cap[2] = {};  // per-trace aperture caps of the staged batch (2 ints each)
  int *h_cap[2] = {};
  int *d_ints = nullptr;
  float *d_geom = nullptr;
  unsigned *d_err = nullptr;
  unsigned long long *d_npt = nullptr;  // point-traces, decided per tile, imaged
  unsigned long long *d_nacc = nullptr;  // (trace, line) pairs the gate accepted
  // lines of the image brick
  bool line_set = false;
  std::vector<qpsdm_line_params> lines;
  int lines_cap = 0;     // lines the per-line buffers hold
  float *d_dips = nullptr;  // [line][4][nxi][nzi]
  size_t nxz = 0;
  // offset
  bool offset_set = false;
  qpsdm_offset_params off{};
  float *d_omega = nullptr;
  int omega_cap = 0;
  float *d_re = nullptr, *d_im = nullptr;
  size_t spec_cap = 0;
  float *d_img = nullptr;
  size_t img_cap = 0;
  // physics state (physics.cu)
  PhysicsState *phys = nullptr;
  KernelProfiler prof;
  // CUDA graphs of whole batches, keyed by (record buffer, aperture caps,
  // ntr, big_endian, line mask)
  struct GraphRec {
    cudaGraphExec_t exec;
    int64_t launches[4];
  };
  std::map<std::tuple<const void *, const void *, int, int, unsigned long long>, GraphRec>
      graphs;
  int64_t batches_run = 0;
  int64_t graph_replays = 0;
  // asynchronous image reads (qpsdm_get_image_async): a ring of outstanding
  // copies, ticket t in slot t % kReads
  static constexpr int kReads = 4;
  struct ImageRead {
    cudaEvent_t done = nullptr;
    float *host = nullptr;
    size_t n = 0;
    int scale = 0;
    float nsb = 1.0f;  // the offset group's nsb when the read was enqueued
    int64_t ticket = -1;
  };
  ImageRead reads[kReads];
  int64_t next_ticket = 0;
};

namespace {

int fail(qpsdm_engine *e, int code, const std::string &msg) {
  if (e) e->err = msg;
  return code;
}

int cuda_fail(qpsdm_engine *e, cudaError_t c, const char *what) {
  return fail(e, c == cudaErrorMemoryAllocation ? QPSDM_ENOMEM : QPSDM_ECUDA,
              std::string(what) + ": " + cudaGetErrorString(c));
}

#define CK(call)                                              \
  do {                                                        \
    cudaError_t _c = (call);                                  \
    if (_c != cudaSuccess) return cuda_fail(e, _c, #call);    \
  } while (0)

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int d) {
    cudaGetDevice(&prev);
    if (prev != d) cudaSetDevice(d);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

template <typename T>
int grow(qpsdm_engine *e, T **ptr, size_t *cap, size_t need) {
  if (*cap >= need && *ptr) return QPSDM_OK;
  if (*ptr) cudaFree(*ptr);
  *ptr = nullptr;
  *cap = 0;
  CK(cudaMalloc((void **)ptr, sizeof(T) * need));
  *cap = need;
  return QPSDM_OK;
}

void clear_graphs(qpsdm_engine *e);

// Taper factors of fetch_and_taper (src/psdmpkg.cc:221-228), computed on the
// host with the same float/double mix so the device multiplies by the same
// bits.
void taper_factors(float *c) {
  for (int it = 0; it < 200; ++it)
    c[it] = (float)(0.5 - 0.5 * cosf((float)(M_PI * it / 200.0)));
}

}  // namespace

extern "C" const char *qpsdm_last_error(const qpsdm_engine *e) {
  return e ? e->err.c_str() : "null engine";
}

extern "C" int qpsdm_engine_create(const qpsdm_static_params *p,
                                   const int *iaztab, int naztab, int device,
                                   qpsdm_engine **out) {
  if (!p || !out || !iaztab || naztab <= 0) return QPSDM_EINVAL;
  *out = nullptr;
  if (p->nfft <= 0 || p->nffti <= 0 || p->dt1 <= 0.0f)
    return QPSDM_EINVAL;  // qpsdm_static_params_init not called
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
    return QPSDM_ECUDA;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return QPSDM_ECUDA;
  if (prop.major != 10 || prop.minor != 0) return QPSDM_ENOKERNEL;

  qpsdm_engine *e = new qpsdm_engine;
  e->device = device;
  e->p = *p;
  DeviceGuard g(device);
  if (e->p.max_batch <= 0) e->p.max_batch = 4096;
  e->rec_bytes = (size_t)kSuHdr + 4 * (size_t)e->p.ntl;
  e->naztab = naztab;
  auto bail = [&](int rc) {
    *out = nullptr;
    std::string m = e->err;
    qpsdm_engine_destroy(e);
    return rc;
  };
#define CKC(call)                                          \
  do {                                                     \
    cudaError_t _c = (call);                               \
    if (_c != cudaSuccess) return bail(cuda_fail(e, _c, #call)); \
  } while (0)
  CKC(cudaStreamCreateWithFlags(&e->s_comp, cudaStreamNonBlocking));
  e->s_own = e->s_comp;
  CKC(cudaStreamCreateWithFlags(&e->s_copy, cudaStreamNonBlocking));
  for (int i = 0; i < 2; ++i) {
    CKC(cudaEventCreateWithFlags(&e->ev_stage_free[i], cudaEventDisableTiming));
    CKC(cudaEventCreateWithFlags(&e->ev_rec_ready[i], cudaEventDisableTiming));
    CKC(cudaEventCreateWithFlags(&e->ev_rec_free[i], cudaEventDisableTiming));
    CKC(cudaMalloc(&e->d_rec[i], e->rec_bytes * e->p.max_batch));
    CKC(cudaMallocHost(&e->h_stage[i], e->rec_bytes * e->p.max_batch));
    CKC(cudaMalloc(&e->d_cap[i], 2 * sizeof(int) * e->p.max_batch));
    CKC(cudaMallocHost(&e->h_cap[i], 2 * sizeof(int) * e->p.max_batch));
  }
  CKC(cudaMalloc(&e->d_iaztab, sizeof(int) * naztab));
  CKC(cudaMemcpy(e->d_iaztab, iaztab, sizeof(int) * naztab, cudaMemcpyHostToDevice));
  float tap[200];
  taper_factors(tap);
  CKC(cudaMalloc(&e->d_taper200, sizeof(tap)));
  CKC(cudaMemcpy(e->d_taper200, tap, sizeof(tap), cudaMemcpyHostToDevice));
  CKC(cudaMalloc(&e->d_ints, sizeof(int) * kGateInts * e->p.max_batch));
  CKC(cudaMalloc(&e->d_geom, sizeof(float) * kGateF * e->p.max_batch));
  CKC(cudaMalloc(&e->d_err, sizeof(unsigned)));
  CKC(cudaMemset(e->d_err, 0, sizeof(unsigned)));
  CKC(cudaMalloc(&e->d_npt, 3 * sizeof(unsigned long long)));
  CKC(cudaMemset(e->d_npt, 0, 3 * sizeof(unsigned long long)));
  CKC(cudaMalloc(&e->d_nacc, sizeof(unsigned long long)));
  CKC(cudaMemset(e->d_nacc, 0, sizeof(unsigned long long)));
  if (e->p.mode == QPSDM_MODE_PHYSICS) {
    int rc = physics_create(&e->phys, e->p, &e->err);
    if (rc) return bail(rc);
  } else if (e->p.mode != QPSDM_MODE_COMPAT) {
    return bail(fail(e, QPSDM_EINVAL, "unknown mode"));
  }
#undef CKC
  *out = e;
  return QPSDM_OK;
}

extern "C" int qpsdm_engine_destroy(qpsdm_engine *e) {
  if (!e) return QPSDM_OK;
  DeviceGuard g(e->device);
  if (e->s_comp) cudaStreamSynchronize(e->s_comp);
  if (e->s_copy) cudaStreamSynchronize(e->s_copy);
  clear_graphs(e);
  for (auto &r : e->reads)
    if (r.done) cudaEventDestroy(r.done);
  if (e->phys) physics_destroy(e->phys);
  for (int i = 0; i < 2; ++i) {
    if (e->ev_stage_free[i]) cudaEventDestroy(e->ev_stage_free[i]);
    if (e->ev_rec_ready[i]) cudaEventDestroy(e->ev_rec_ready[i]);
    if (e->ev_rec_free[i]) cudaEventDestroy(e->ev_rec_free[i]);
    if (e->d_rec[i]) cudaFree(e->d_rec[i]);
    if (e->h_stage[i]) cudaFreeHost(e->h_stage[i]);
    if (e->d_cap[i]) cudaFree(e->d_cap[i]);
    if (e->h_cap[i]) cudaFreeHost(e->h_cap[i]);
  }
  cudaFree(e->d_iaztab);
  cudaFree(e->d_taper200);
  cudaFree(e->d_ints);
  cudaFree(e->d_geom);
  cudaFree(e->d_err);
  cudaFree(e->d_npt);
  cudaFree(e->d_nacc);
  cudaFree(e->d_dips);
  cudaFree(e->d_omega);
  cudaFree(e->d_re);
  cudaFree(e->d_im);
  cudaFree(e->d_img);
  if (e->s_own) cudaStreamDestroy(e->s_own);
  if (e->s_copy) cudaStreamDestroy(e->s_copy);
  delete e;
  return QPSDM_OK;
}

extern "C" int qpsdm_set_lines(qpsdm_engine *e, const qpsdm_line_params *l, int nlines) {
  if (!e || !l || nlines <= 0) return QPSDM_EINVAL;
  for (int il = 0; il < nlines; ++il)
    if (!l[il].dipx1 || !l[il].dipx2 || !l[il].dipy1 || !l[il].dipy2)
      return fail(e, QPSDM_EINVAL, "dip fields are required");
  DeviceGuard g(e->device);
  CK(cudaStreamSynchronize(e->s_comp));
  e->nxz = (size_t)e->p.nxi * e->p.nzi;
  if (nlines > e->lines_cap) {  // per-line dip fields and gate results
    cudaFree(e->d_dips);
    cudaFree(e->d_ints);
    cudaFree(e->d_geom);
    e->d_dips = nullptr;
    e->d_ints = nullptr;
    e->d_geom = nullptr;
    e->lines_cap = 0;
    CK(cudaMalloc(&e->d_dips, sizeof(float) * 4 * e->nxz * nlines));
    CK(cudaMalloc(&e->d_ints, sizeof(int) * kGateInts * (size_t)e->p.max_batch * nlines));
    CK(cudaMalloc(&e->d_geom, sizeof(float) * kGateF * (size_t)e->p.max_batch * nlines));
    e->lines_cap = nlines;
  }
  for (int il = 0; il < nlines; ++il) {
    const float *f[4] = {l[il].dipx1, l[il].dipx2, l[il].dipy1, l[il].dipy2};
    for (int i = 0; i < 4; ++i)
      CK(cudaMemcpy(e->d_dips + (size_t)il * 4 * e->nxz + i * e->nxz, f[i],
                    sizeof(float) * e->nxz, cudaMemcpyHostToDevice));
  }
  if (e->p.mode == QPSDM_MODE_PHYSICS) {
    int rc = physics_set_lines(e->phys, e->p, l, nlines, e->s_comp, &e->err);
    if (rc) return rc;
  }
  e->lines.assign(l, l + nlines);
  clear_graphs(e);
  e->line_set = true;
  e->offset_set = false;
  return QPSDM_OK;
}

extern "C" int qpsdm_set_line(qpsdm_engine *e, const qpsdm_line_params *l) {
  return qpsdm_set_lines(e, l, 1);
}

extern "C" int qpsdm_begin_offset(qpsdm_engine *e, const qpsdm_offset_params *o) {
  if (!e || !o) return QPSDM_EINVAL;
  if (!e->line_set) return fail(e, QPSDM_ESTATE, "begin_offset before set_line");
  if (o->ixstart < 0 || o->ixend > e->p.nxi || o->ixend <= o->ixstart || o->nsb <= 0 ||
      o->nww <= 0 || o->nf1 < 0 || o->nf1 + o->nww > o->nsb / 2 + 1)
    return fail(e, QPSDM_EINVAL, "bad offset parameters");
  DeviceGuard g(e->device);
  CK(cudaStreamSynchronize(e->s_comp));
  // -i*w frequencies accumulated in float as psdm_kernel does (w += dw).
  std::vector<float> om(o->nww);
  float w = o->nf1 * o->dw;
  for (int iw = 0; iw < o->nww; ++iw, w += o->dw) om[iw] = w;
  size_t ocap = e->omega_cap;
  int rc = grow(e, &e->d_omega, &ocap, (size_t)o->nww);
  if (rc) return rc;
  e->omega_cap = (int)ocap;
  CK(cudaMemcpy(e->d_omega, om.data(), sizeof(float) * o->nww, cudaMemcpyHostToDevice));
  size_t need = (size_t)e->p.max_batch * 2 * o->nww;
  size_t cap_re = e->spec_cap, cap_im = e->spec_cap;
  if ((rc = grow(e, &e->d_re, &cap_re, need))) return rc;
  if ((rc = grow(e, &e->d_im, &cap_im, need))) return rc;
  e->spec_cap = cap_re;
  const size_t nimg = (size_t)(o->ixend - o->ixstart) * e->p.nzi * e->lines.size();
  const bool realloc_img = e->img_cap < nimg;
  if ((rc = grow(e, &e->d_img, &e->img_cap, nimg))) return rc;
  if (o->zero_image || realloc_img || !e->offset_set)
    CK(cudaMemsetAsync(e->d_img, 0, sizeof(float) * nimg, e->s_comp));
  CK(cudaMemsetAsync(e->d_npt, 0, 3 * sizeof(unsigned long long), e->s_comp));
  CK(cudaMemsetAsync(e->d_nacc, 0, sizeof(unsigned long long), e->s_comp));
  if (e->p.mode == QPSDM_MODE_PHYSICS) {
    rc = physics_begin_offset(e->phys, e->p, *o, (int)e->lines.size(), e->s_comp, &e->err);
    if (rc) return rc;
  }
  e->off = *o;
  clear_graphs(e);
  e->offset_set = true;
  return QPSDM_OK;
}

namespace {

// Kernels of one batch whose records are in device memory.
int process_batch(qpsdm_engine *e, const uint8_t *d_rec, const int *d_cap, int ntr, int be) {
  const int nlines = (int)e->lines.size();
  const int nxb = e->off.ixend - e->off.ixstart;
  const size_t ints_ls = (size_t)kGateInts * e->p.max_batch;  // per-line strides
  const size_t geom_ls = (size_t)kGateF * e->p.max_batch;
  const size_t img_ls = (size_t)nxb * e->p.nzi;
  auto line_on = [&](int il) { return il >= 64 || ((e->line_mask >> il) & 1ull); };
  // gate every line of the brick (src/q-psdm.cu:2107-2171 for each line's cyi)
  for (int il = 0; il < nlines; ++il) {
    if (!line_on(il)) continue;
    const qpsdm_line_params &ln = e->lines[il];
    GateArgs g{};
    g.scaled = e->p.scaled;
    g.fxi = ln.fxi;
    g.cyi = ln.cyi;
    g.fxv1 = e->p.fxv1;
    g.fyv1 = e->p.fyv1;
    g.exv1 = e->p.exv1;
    g.eyv1 = e->p.eyv1;
    g.dxi = e->p.dxi;
    g.dyi = e->p.dyi;
    g.eps = e->p.eps;
    g.nzi = e->p.nzi;
    g.ixstart = e->off.ixstart;
    g.ixend = e->off.ixend;
    g.naztab = e->naztab;
    g.iaztab = e->d_iaztab;
    g.cap = d_cap;
    memcpy(g.az[0], e->off.aznx1, sizeof(int) * QPSDM_NAZ);
    memcpy(g.az[1], e->off.aznx2, sizeof(int) * QPSDM_NAZ);
    memcpy(g.az[2], e->off.azny1, sizeof(int) * QPSDM_NAZ);
    memcpy(g.az[3], e->off.azny2, sizeof(int) * QPSDM_NAZ);
    e->prof.begin(QPSDM_K_GATE, e->s_comp);
    int rc = launch_gate(d_rec, (int)e->rec_bytes, ntr, be, g, e->d_ints + il * ints_ls,
                         e->d_geom + il * geom_ls, e->d_err, e->d_nacc, e->s_comp);
    e->prof.end(e->s_comp);
    if (rc) return fail(e, rc, "gate launch failed");
  }
  if (e->p.mode == QPSDM_MODE_COMPAT) {
    // the reference preprocesses and images each trace once per line
    for (int il = 0; il < nlines; ++il) {
      if (!line_on(il)) continue;
      const qpsdm_line_params &ln = e->lines[il];
      SpectraArgs a{};
      a.ntl = e->p.ntl;
      a.nsb = e->off.nsb;
      a.itb1 = e->off.itb1;
      a.itb2 = e->off.itb2;
      a.nf1 = e->off.nf1;
      a.nww = e->off.nww;
      a.dt = e->p.dt;
      a.taper200 = e->d_taper200;
      a.omega = e->d_omega;
      e->prof.begin(QPSDM_K_PRE, e->s_comp);
      int rc = launch_spectra(d_rec, (int)e->rec_bytes, ntr, be, e->d_ints + il * ints_ls, a,
                              e->d_re, e->d_im, e->s_comp);
      e->prof.end(e->s_comp);
      if (rc) return fail(e, rc, "spectra launch failed");
      CompatImageArgs c{};
      c.nzi = e->p.nzi;
      c.nxb = nxb;
      c.ixstart = e->off.ixstart;
      c.nt = e->p.nffti;
      c.dt1 = e->p.dt1;
      c.dxi = e->p.dxi;
      c.dzi = e->p.dzi;
      c.taperzone = e->p.taperzone;
      c.tcdp1 = ln.ttt_cdp1 - e->p.fci;
      c.tcdp2 = ln.ttt_cdp2 - e->p.fci;
      c.nxz = e->nxz;
      e->prof.begin(QPSDM_K_IMAGE, e->s_comp);
      rc = launch_image_compat(e->d_img + il * img_ls, c, e->d_dips + (size_t)il * 4 * e->nxz,
                               e->d_ints + il * ints_ls, e->d_geom + il * geom_ls, ntr,
                               e->d_npt, e->s_comp);
      e->prof.end(e->s_comp);
      if (rc) return fail(e, rc, "image launch failed");
    }
    return QPSDM_OK;
  }
  PhysicsBatch b{};
  b.d_rec = d_rec;
  b.rec_bytes = (int)e->rec_bytes;
  b.ntr = ntr;
  b.big_endian = be;
  b.nlines = nlines;
  b.d_ints = e->d_ints;
  b.ints_ls = ints_ls;
  b.d_geom = e->d_geom;
  b.geom_ls = geom_ls;
  b.d_taper200 = e->d_taper200;
  b.d_dips = e->d_dips;
  b.nxz = e->nxz;
  b.d_img = e->d_img;
  b.img_ls = img_ls;
  b.d_npt = e->d_npt;
  b.d_err = e->d_err;
  b.prof = &e->prof;
  b.line_mask = e->line_mask;
  return physics_process(e->phys, e->p, e->lines.data(), e->off, b, e->s_comp, &e->err);
}

void clear_graphs(qpsdm_engine *e) {
  for (auto &kv : e->graphs) cudaGraphExecDestroy(kv.second.exec);
  e->graphs.clear();
}

// One batch: replayed from a CUDA graph when use_graph is set and this
// (buffer, size) was seen before; captured on its second occurrence (the
// first runs eagerly so that plans, attributes and the autotuner settle).
int run_batch(qpsdm_engine *e, const uint8_t *d_rec, const int *d_cap, int ntr, int be) {
  const bool graphs = e->p.use_graph != 0;
  if (!graphs || e->batches_run == 0) {
    ++e->batches_run;
    return process_batch(e, d_rec, d_cap, ntr, be);
  }
  const auto key = std::make_tuple((const void *)d_rec, (const void *)d_cap, ntr, be,
                                   e->line_mask);
  auto it = e->graphs.find(key);
  if (it != e->graphs.end()) {
    CK(cudaGraphLaunch(it->second.exec, e->s_comp));
    for (int c = 0; c < 4; ++c) e->prof.launches[c] += it->second.launches[c];
    ++e->graph_replays;
    ++e->batches_run;
    return QPSDM_OK;
  }
  int64_t before[4];
  for (int c = 0; c < 4; ++c) before[c] = e->prof.launches[c];
  const bool prof_on = e->prof.on;
  e->prof.on = false;  // no timing events inside the graph
  CK(cudaStreamBeginCapture(e->s_comp, cudaStreamCaptureModeThreadLocal));
  const int rc = process_batch(e, d_rec, d_cap, ntr, be);
  cudaGraph_t g = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(e->s_comp, &g);
  e->prof.on = prof_on;
  if (rc || ce != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return rc ? rc : cuda_fail(e, ce, "cudaStreamEndCapture");
  }
  qpsdm_engine::GraphRec gr{};
  const cudaError_t ie = cudaGraphInstantiate(&gr.exec, g, 0);
  cudaGraphDestroy(g);
  if (ie != cudaSuccess) return cuda_fail(e, ie, "cudaGraphInstantiate");
  for (int c = 0; c < 4; ++c) gr.launches[c] = e->prof.launches[c] - before[c];
  e->graphs[key] = gr;
  CK(cudaGraphLaunch(gr.exec, e->s_comp));
  ++e->batches_run;
  return QPSDM_OK;
}

}  // namespace

namespace {

int submit_device(qpsdm_engine *e, const void *d_records, const int *d_aperture, int ntr,
                  int ns, int be) {
  if (!e || (!d_records && ntr > 0)) return QPSDM_EINVAL;
  if (!e->offset_set) return fail(e, QPSDM_ESTATE, "submit before begin_offset");
  if (ns != e->p.ntl)
    return fail(e, QPSDM_EINVAL, "trace ns differs from ntl (src/q-psdm.cu:915-921)");
  if (ntr < 0 || ntr > e->p.max_batch) return fail(e, QPSDM_EINVAL, "ntr outside [0, max_batch]");
  if (ntr == 0) return QPSDM_OK;
  DeviceGuard g(e->device);
  return run_batch(e, (const uint8_t *)d_records, d_aperture, ntr, be);
}

int submit_host(qpsdm_engine *e, const void *records, const int *aperture, int ntr, int ns,
                int be) {
  if (!e || (!records && ntr > 0)) return QPSDM_EINVAL;
  if (!e->offset_set) return fail(e, QPSDM_ESTATE, "submit before begin_offset");
  if (ns != e->p.ntl)
    return fail(e, QPSDM_EINVAL, "trace ns differs from ntl (src/q-psdm.cu:915-921)");
  if (ntr < 0) return fail(e, QPSDM_EINVAL, "negative ntr");
  DeviceGuard g(e->device);
  const uint8_t *src = (const uint8_t *)records;
  // Records already in page-locked memory are copied by DMA directly; others
  // go through the engine's pinned staging slots.
  cudaPointerAttributes pa;
  const bool pinned = cudaPointerGetAttributes(&pa, records) == cudaSuccess &&
                      pa.type == cudaMemoryTypeHost;
  cudaGetLastError();  // a pageable pointer may leave an error behind
  while (ntr > 0) {
    const int n = ntr < e->p.max_batch ? ntr : e->p.max_batch;
    const size_t bytes = e->rec_bytes * n;
    const int s = e->slot;
    CK(cudaEventSynchronize(e->ev_stage_free[s]));
    if (!pinned) memcpy(e->h_stage[s], src, bytes);
    if (aperture) memcpy(e->h_cap[s], aperture, 2 * sizeof(int) * n);
    CK(cudaStreamWaitEvent(e->s_copy, e->ev_rec_free[s], 0));
    CK(cudaMemcpyAsync(e->d_rec[s], pinned ? src : e->h_stage[s], bytes,
                       cudaMemcpyHostToDevice, e->s_copy));
    if (aperture)
      CK(cudaMemcpyAsync(e->d_cap[s], e->h_cap[s], 2 * sizeof(int) * n,
                         cudaMemcpyHostToDevice, e->s_copy));
    CK(cudaEventRecord(e->ev_stage_free[s], e->s_copy));
    // a caller's pinned buffer may be reused once the call returns
    if (pinned) CK(cudaEventSynchronize(e->ev_stage_free[s]));
    CK(cudaEventRecord(e->ev_rec_ready[s], e->s_copy));
    CK(cudaStreamWaitEvent(e->s_comp, e->ev_rec_ready[s], 0));
    int rc = run_batch(e, e->d_rec[s], aperture ? e->d_cap[s] : nullptr, n, be);
    if (rc) return rc;
    CK(cudaEventRecord(e->ev_rec_free[s], e->s_comp));
    e->slot ^= 1;
    src += bytes;
    if (aperture) aperture += 2 * n;
    ntr -= n;
  }
  return QPSDM_OK;
}

}  // namespace

extern "C" int qpsdm_submit_traces_device(qpsdm_engine *e, const void *d_records,
                                          int ntr, int ns, int be) {
  return submit_device(e, d_records, nullptr, ntr, ns, be);
}

extern "C" int qpsdm_submit_gathers_device(qpsdm_engine *e, const void *d_records,
                                           const int *d_aperture, int ntr, int ns, int be) {
  return submit_device(e, d_records, d_aperture, ntr, ns, be);
}

extern "C" int qpsdm_submit_gathers(qpsdm_engine *e, const void *records, const int *aperture,
                                    int ntr, int ns, int be) {
  return submit_host(e, records, aperture, ntr, ns, be);
}

extern "C" int qpsdm_submit_traces(qpsdm_engine *e, const void *records, int ntr,
                                   int ns, int be) {
  return submit_host(e, records, nullptr, ntr, ns, be);
}

extern "C" int qpsdm_set_line_mask(qpsdm_engine *e, unsigned long long mask) {
  if (!e) return QPSDM_EINVAL;
  if (mask == 0) return fail(e, QPSDM_EINVAL, "line mask selects no line");
  e->line_mask = mask;
  return QPSDM_OK;
}

extern "C" int qpsdm_fence(qpsdm_engine *e) {
  if (!e) return QPSDM_EINVAL;
  DeviceGuard g(e->device);
  CK(cudaStreamSynchronize(e->s_copy));
  CK(cudaStreamSynchronize(e->s_comp));
  unsigned herr = 0;
  CK(cudaMemcpy(&herr, e->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost));
  if (herr) {
    char b[96];
    snprintf(b, sizeof b, "device error word 0x%x (index clamped or masked)", herr);
    e->err = b;
  }
  return QPSDM_OK;
}

extern "C" int qpsdm_get_image(qpsdm_engine *e, float *host_img, int apply_nsb_scale) {
  if (!e || !host_img) return QPSDM_EINVAL;
  if (!e->offset_set) return fail(e, QPSDM_ESTATE, "get_image before begin_offset");
  int rc = qpsdm_fence(e);
  if (rc) return rc;
  DeviceGuard g(e->device);
  const size_t n = (size_t)(e->off.ixend - e->off.ixstart) * e->p.nzi * e->lines.size();
  if (e->p.mode == QPSDM_MODE_PHYSICS) {
    rc = physics_finalize_image(e->phys, e->d_img, n, e->s_comp, &e->err);
    if (rc) return rc;
    CK(cudaStreamSynchronize(e->s_comp));
  }
  CK(cudaMemcpy(host_img, e->d_img, sizeof(float) * n, cudaMemcpyDeviceToHost));
  if (apply_nsb_scale)
    for (size_t i = 0; i < n; ++i) host_img[i] /= e->off.nsb;  // src/q-psdm.cu:1761-1765
  return QPSDM_OK;
}

namespace {

// Waits for the read in ring slot r and applies its /nsb scale on the host.
int finish_read(qpsdm_engine *e, qpsdm_engine::ImageRead &r) {
  if (r.ticket < 0) return QPSDM_OK;
  CK(cudaEventSynchronize(r.done));
  if (r.scale)
    for (size_t i = 0; i < r.n; ++i) r.host[i] /= r.nsb;  // src/q-psdm.cu:1761-1765
  r.ticket = -1;
  return QPSDM_OK;
}

}  // namespace

extern "C" int qpsdm_get_image_async(qpsdm_engine *e, float *host_img, int apply_nsb_scale,
                                     int64_t *ticket) {
  if (!e || !host_img || !ticket) return QPSDM_EINVAL;
  if (!e->offset_set) return fail(e, QPSDM_ESTATE, "get_image_async before begin_offset");
  DeviceGuard g(e->device);
  cudaPointerAttributes pa;
  if (cudaPointerGetAttributes(&pa, host_img) != cudaSuccess ||
      pa.type != cudaMemoryTypeHost) {
    cudaGetLastError();
    return fail(e, QPSDM_EINVAL, "get_image_async needs page-locked host memory");
  }
  const size_t n = (size_t)(e->off.ixend - e->off.ixstart) * e->p.nzi * e->lines.size();
  qpsdm_engine::ImageRead &r = e->reads[e->next_ticket % qpsdm_engine::kReads];
  int rc = finish_read(e, r);  // the oldest read still in this slot
  if (rc) return rc;
  if (!r.done) CK(cudaEventCreateWithFlags(&r.done, cudaEventDisableTiming));
  if (e->p.mode == QPSDM_MODE_PHYSICS) {
    rc = physics_finalize_image(e->phys, e->d_img, n, e->s_comp, &e->err);
    if (rc) return rc;
  }
  CK(cudaMemcpyAsync(host_img, e->d_img, sizeof(float) * n, cudaMemcpyDeviceToHost,
                     e->s_comp));
  CK(cudaEventRecord(r.done, e->s_comp));
  r.host = host_img;
  r.n = n;
  r.scale = apply_nsb_scale != 0;
  r.nsb = (float)e->off.nsb;
  r.ticket = e->next_ticket;
  *ticket = e->next_ticket++;
  return QPSDM_OK;
}

extern "C" int qpsdm_image_wait(qpsdm_engine *e, int64_t ticket) {
  if (!e || ticket < 0 || ticket >= e->next_ticket) return QPSDM_EINVAL;
  DeviceGuard g(e->device);
  qpsdm_engine::ImageRead &r = e->reads[ticket % qpsdm_engine::kReads];
  if (r.ticket != ticket) return QPSDM_OK;  // finished already (or reused after finishing)
  return finish_read(e, r);
}

extern "C" int qpsdm_set_stream(qpsdm_engine *e, void *stream) {
  if (!e) return QPSDM_EINVAL;
  DeviceGuard g(e->device);
  CK(cudaStreamSynchronize(e->s_comp));
  e->s_comp = stream ? (cudaStream_t)stream : e->s_own;
  return QPSDM_OK;
}

extern "C" int qpsdm_profile_enable(qpsdm_engine *e, int on) {
  if (!e) return QPSDM_EINVAL;
  DeviceGuard g(e->device);
  CK(cudaStreamSynchronize(e->s_comp));
  e->prof.reset();
  e->prof.on = on != 0;
  return QPSDM_OK;
}

extern "C" int qpsdm_profile_get(qpsdm_engine *e, int cls, double *ms, int64_t *launches) {
  if (!e || cls < 0 || cls > 3) return QPSDM_EINVAL;
  DeviceGuard g(e->device);
  if (ms) *ms = e->prof.total_ms(cls);
  if (launches) *launches = e->prof.launches[cls];
  return QPSDM_OK;
}

extern "C" int qpsdm_tuning_info(qpsdm_engine *e, int *variant, int *tile_z, int *tile_x,
                                 int *min_blocks, float *ms, int nms) {
  if (!e) return QPSDM_EINVAL;
  if (!e->phys) return fail(e, QPSDM_ESTATE, "no physics state");
  return physics_tuning(e->phys, variant, tile_z, tile_x, min_blocks, ms, nms);
}

extern "C" int qpsdm_image_device_ptr(qpsdm_engine *e, float **d_img) {
  if (!e || !d_img) return QPSDM_EINVAL;
  *d_img = e->d_img;
  return QPSDM_OK;
}

extern "C" int qpsdm_get_counters(qpsdm_engine *e, int64_t *acc, int64_t *npt) {
  if (!e) return QPSDM_EINVAL;
  DeviceGuard g(e->device);
  CK(cudaStreamSynchronize(e->s_comp));
  unsigned long long v = 0, na = 0;
  CK(cudaMemcpy(&v, e->d_npt, sizeof(v), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(&na, e->d_nacc, sizeof(na), cudaMemcpyDeviceToHost));
  if (npt) *npt = (int64_t)v;
  if (acc) *acc = (int64_t)na;
  return QPSDM_OK;
}

extern "C" int qpsdm_get_stats(qpsdm_engine *e, int64_t *out, int n) {
  if (!e || (!out && n > 0) || n < 0) return QPSDM_EINVAL;
  DeviceGuard g(e->device);
  CK(cudaStreamSynchronize(e->s_comp));
  unsigned long long v[4] = {0, 0, 0, 0};
  CK(cudaMemcpy(&v[0], e->d_nacc, sizeof(v[0]), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(&v[1], e->d_npt, 3 * sizeof(v[0]), cudaMemcpyDeviceToHost));
  for (int i = 0; i < n && i < 4; ++i) out[i] = (int64_t)v[i];
  return 4;
}

extern "C" int qpsdm_panels_device_ptr(qpsdm_engine *e, void **d_panels, float **d_pscale) {
  if (!e || !d_panels || !d_pscale) return QPSDM_EINVAL;
  if (!e->phys) return fail(e, QPSDM_ESTATE, "panels exist in physics mode only");
  physics_panels(e->phys, d_panels, d_pscale);
  return QPSDM_OK;
}

extern "C" int qpsdm_spectra_device_ptr(qpsdm_engine *e, float **d_re, float **d_im) {
  if (!e || !d_re || !d_im) return QPSDM_EINVAL;
  *d_re = e->d_re;
  *d_im = e->d_im;
  return QPSDM_OK;
}

extern "C" int qpsdm_gate_device_ptr(qpsdm_engine *e, int **d_ints, float **d_geom) {
  if (!e || !d_ints || !d_geom) return QPSDM_EINVAL;
  *d_ints = e->d_ints;
  *d_geom = e->d_geom;
  return QPSDM_OK;
}
