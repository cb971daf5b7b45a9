/*
 * qpsdm_engine.h -- C ABI of the B200 Q-compensated Kirchhoff PSDM engine.
 *
 * This is the drop-in boundary for the imaging path of resetlla/q_psdm.  The
 * reference has no plugin API: its hot path sits behind the per-trace C++
 * call psdm_kernel(segy tr, ~75 scalars ...) (src/q-psdm.cu:252-283, body
 * :2063-2244), called by the consumer threads (src/q-psdm.cu:1928-2061),
 * with line state set up by qpsdm() (src/q-psdm.cu:1298-1376, :1495-1515,
 * :1653-1691) and tables loaded by get_ttt_all() (src/q-psdm.cu:2382-2622).
 * Each entry point below names the reference interface it replaces.
 *
 * Conventions
 *   - Plain C types and pointers; no CUDA or torch types in signatures.
 *     Streams are passed as void* (a cudaStream_t; NULL = the engine's own).
 *   - Every call returns an int status (QPSDM_OK == 0).  The library never
 *     exits the process; qpsdm_last_error() gives the message.
 *   - One engine handle per host thread; a handle is bound to one device.
 *   - Host pointers are read during the call (or, for the _async calls,
 *     until the next qpsdm_fence()).  Device pointers ("d_" prefix) must be
 *     memory of the engine's device.
 */
#ifndef QPSDM_ENGINE_H_
#define QPSDM_ENGINE_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QPSDM_ABI_VERSION 1
#define QPSDM_NAZ 18 /* azimuth sectors, src/q-psdm.cu:1177 */
#define QPSDM_SU_HDR_BYTES 240

enum {
  QPSDM_OK = 0,
  QPSDM_EINVAL = 1,   /* bad argument or size */
  QPSDM_ECUDA = 2,    /* CUDA runtime error */
  QPSDM_ENOMEM = 3,   /* device or pinned allocation failed */
  QPSDM_ESTATE = 4,   /* call out of order (e.g. submit before begin_offset) */
  QPSDM_ETIMEOUT = 5, /* a bounded device wait gave up */
  QPSDM_ENOTSUP = 6,
  QPSDM_ENOKERNEL = 7, /* no sm_100a image for this device */
  QPSDM_ESIZE = 8      /* request larger than a fixed built-in capacity */
};

enum { QPSDM_MODE_COMPAT = 0, QPSDM_MODE_PHYSICS = 1 };
enum { QPSDM_PANEL_FP32 = 0, QPSDM_PANEL_BF16 = 1, QPSDM_PANEL_FP16 = 2 };

typedef struct qpsdm_engine qpsdm_engine;

/* Traveltime / t* table descriptor, byte-identical to ttt_desc_t
 * (src/q-psdm.cu:103-109) and to the 16-byte records of Lxxx.{tidx,qidx}. */
typedef struct {
  int64_t idx; /* float offset of the cell's block in the data array */
  uint16_t nys, nxs, dys, dxs; /* local surface grid: nodes and spacing (m) */
} qpsdm_ttt_desc;

/* Line-independent parameters: mirrors CPUParamsNoLine
 * (src/q-psdm.cu:111-147) plus the engine's own options.
 * qpsdm_static_params_init() fills the derived members the way qpsdm()
 * does (src/q-psdm.cu:1201-1287). */
typedef struct {
  /* from the command line / par.dat */
  float dyi, dxi;  /* image line and cdp spacing (m) */
  int nxi, nzi;    /* image cdps per line, depth samples */
  int ntl;         /* samples per input trace */
  double scaled;   /* coordinate scale of the data (getscale(scalco)) */
  int fci;         /* first image cdp */
  float dzi;       /* image depth step (m) */
  float dt;        /* input sample interval (s) */
  float fc;        /* reference frequency (Hz) of the dispersion law */
  float f1, f3, f4;/* band: low cut, high-cut start and end (Hz) */
  float threshold; /* gain limit G (linear) */
  float contract, taperzone; /* degrees on input, radians after init */
  float fxv1, fyv1, exv1, eyv1; /* velocity-grid bbox padded +-2 km / +-1 km */
  float dzii;      /* table depth-node spacing (m) */
  /* derived by qpsdm_static_params_init */
  float eps;       /* azimuth table step, 0.001 */
  int nfft, nffti; /* npfar(ntl), npfar(2*ntl) */
  float dt1;       /* resampled interval 1/(nffti*df) */
  float df, dw;    /* 1/(nfft*dt), 2*pi*df */
  float lnG, coef1, coef2, coef3, coef4; /* gain-limit law */
  /* engine options */
  int mode;        /* QPSDM_MODE_* */
  int panel_dtype; /* QPSDM_PANEL_* (physics mode) */
  int nbins;       /* t* bins of the compensated panels (physics mode) */
  float dtstar;    /* t* bin spacing (s) */
  int max_batch;   /* largest ntr of one submit (sizes device buffers) */
  int kahan;       /* 1 = compensated FP32 image accumulation (physics) */
  int form;        /* physics: QPSDM_FORM_PLAIN or QPSDM_FORM_BATCHED */
  int use_graph;   /* batched form: replay each batch as a captured CUDA graph */
  int tile_z, tile_x; /* batched image tile (0 = autotuned) */
  int variant;     /* batched: launch variant + 1 of the autotuner's list (0 = tuned) */
  int reserved[3];
} qpsdm_static_params;

/* Physics forms.  PLAIN: one pass per trace in submission order with table
 * lookups per point-trace (source terms reused while consecutive traces share
 * a source).  BATCHED: traces of a batch grouped by receiver position and
 * source; a persistent kernel over image tiles builds the source terms once
 * per shot and tile, drops for the tile every trace whose dip test fails at
 * all its points (a conservative bound; the image and point-trace counts
 * are unchanged), and computes receiver terms once per receiver position; t*
 * panels computed once per trace and shared by every line of a brick
 * (qpsdm_set_lines).  FP16 panels are scaled per trace by a power of two
 * from a bound on the trace's filtered amplitude, so any data amplitude
 * stays inside FP16's range. */
enum { QPSDM_FORM_PLAIN = 0, QPSDM_FORM_BATCHED = 1 };

/* Per-line state: mirrors the line part of CPUParamsWithLine
 * (src/q-psdm.cu:149-179) and the line buffers of GPUParamsWithLine
 * (src/q-psdm.cu:195-213).  Replaces the per-line H2D block of qpsdm()
 * (src/q-psdm.cu:1463-1515) and get_ttt_all() (src/q-psdm.cu:2382-2622).
 * All pointers are host memory, copied during qpsdm_set_line, except the
 * table data ttt and qqq, which may also be memory of the engine's device
 * (tables built on the GPU, e.g. by qpsdm_surrogate_tables). */
typedef struct {
  double fxi, cyi;       /* x of the first image cdp, y of this line */
  const float *dipx1, *dipx2, *dipy1, *dipy2; /* [nxi][nzi] dip tangents */
  const int *nf3;        /* [nxi][nzi] high-cut bin (physics; may be NULL) */
  const float *q;        /* [nxi][nzi] dw/(2Q) field (may be NULL) */
  /* traveltime (ttt) and t* (qqq) tables in the reference layout */
  int nxg, nzg, nxi1, nzi1;
  int ttt_cdp1, ttt_cdp2; /* absolute cdp range of the tables */
  const qpsdm_ttt_desc *ttt_desc, *qqq_desc; /* [nxg*nzg], may be NULL in compat */
  const float *ttt, *qqq;                    /* table data */
  int64_t ttt_len, qqq_len;                  /* floats in ttt, qqq */
} qpsdm_line_params;

/* One offset group inside one x block: mirrors the per-offset members of
 * CPUParamsWithLine and the window split of qpsdm()
 * (src/q-psdm.cu:1593-1691).  qpsdm_offset_params_init() derives them. */
typedef struct {
  int ioffs;
  int ixstart, ixend;          /* image block [ixstart, ixend) */
  int itb1, itb2, nsb;         /* FFT windows */
  float tdstart1, tdstart2, tdmid;
  int nf1, nww, ncoef1;
  float df, dw;
  int aznx1[QPSDM_NAZ], aznx2[QPSDM_NAZ]; /* aperture (cdps) per azimuth */
  int azny1[QPSDM_NAZ], azny2[QPSDM_NAZ]; /* aperture (lines) per azimuth */
  int zero_image;              /* 1 = clear the block image (opcrp) */
} qpsdm_offset_params;

/* ---- parameter derivation (host only, no device work) -------------------*/

/* npfar(): smallest valid real prime-factor FFT length >= nmin
 * (src/fft.cc:491-494, get_opt_n_fftw src/fft.cc:3721). */
int qpsdm_npfar(int nmin);

/* Fills eps, nfft, nffti, dt1, df, dw, lnG, coef1..4 and converts contract
 * and taperzone to radians, as qpsdm() does (src/q-psdm.cu:1201-1287). */
int qpsdm_static_params_init(qpsdm_static_params *p);

/* Azimuth sector table (src/q-psdm.cu:1167-1193); writes up to cap ints,
 * returns the table length (2001 for eps = 0.001) or -1. */
int qpsdm_build_iaztab(float eps, int *iaztab, int cap);

/* Window split and bins of one offset group (src/q-psdm.cu:1593-1645). */
int qpsdm_offset_params_init(const qpsdm_static_params *p, int ixstart,
                             int ixend, qpsdm_offset_params *o);

/* ---- engine lifetime -----------------------------------------------------*/

/* Replaces the per-consumer set-up of qpsdm() (src/q-psdm.cu:1298-1376).
 * iaztab: naztab ints (host).  Allocates all device buffers for max_batch
 * traces up front. */
int qpsdm_engine_create(const qpsdm_static_params *p, const int *iaztab,
                        int naztab, int device, qpsdm_engine **out);
int qpsdm_engine_destroy(qpsdm_engine *e);
const char *qpsdm_last_error(const qpsdm_engine *e);

/* ---- line / offset state ---------------------------------------------------*/

/* Replaces get_ttt_all x2 + the dip/nf3/Q uploads of qpsdm()
 * (src/q-psdm.cu:1449-1515). */
int qpsdm_set_line(qpsdm_engine *e, const qpsdm_line_params *l);

/* A brick of nlines image lines imaged together: every submitted trace is
 * gated and imaged for each line (the reference's line loop,
 * src/q-psdm.cu:1427, run over the same traces), and the image becomes
 * [nlines][nxb][nzi].  In the batched physics form the compensated panels of
 * a trace are computed once and shared by all lines of the brick. */
int qpsdm_set_lines(qpsdm_engine *e, const qpsdm_line_params *lines, int nlines);

/* Replaces the per-offset set-up of qpsdm() (src/q-psdm.cu:1593-1691). */
int qpsdm_begin_offset(qpsdm_engine *e, const qpsdm_offset_params *o);

/* ---- traces --------------------------------------------------------------*/

/* Replaces producer -> queue -> consumer -> psdm_kernel for ntr traces
 * (src/q-psdm.cu:1862-2061, :2063-2244).  records: ntr SU records of
 * 240 + 4*ns bytes, host memory, big-endian on disk layout when
 * big_endian != 0 (as swaptr() decodes, src/segy.cc:6395) else native.
 * Copies through the engine's pinned staging ring and returns when the
 * host buffer may be reused; device work continues asynchronously. */
int qpsdm_submit_traces(qpsdm_engine *e, const void *records, int ntr, int ns,
                        int big_endian);

/* Same, records already resident in device memory (no copy). */
int qpsdm_submit_traces_device(qpsdm_engine *e, const void *d_records, int ntr,
                               int ns, int big_endian);

/* Shot gathers of uneven sizes and apertures in one submit: as
 * qpsdm_submit_traces(_device), with aperture[2*i], aperture[2*i+1] the
 * half-width in cdps and in lines of trace i's own aperture (the aperture its
 * gather was recorded with), which caps the offset group's azimuth tables:
 * trace i images columns cdpx - min(aznx1[iaz], aperture[2i]) ..
 * cdpx + min(aznx2[iaz], aperture[2i]) - 1 of the lines with
 * -min(azny2[iaz], aperture[2i+1]) <= cdpy <= min(azny1[iaz], aperture[2i+1])
 * (the reference's per-offset-group aperture test, src/q-psdm.cu:2147-2171,
 * per trace).  A batch of whole gathers is one persistent imaging launch.
 * aperture: host memory for qpsdm_submit_gathers (copied with the records),
 * device memory for qpsdm_submit_gathers_device (read when the batch runs; a
 * captured batch reads it again at every replay).  No counterpart in the
 * reference. */
int qpsdm_submit_gathers(qpsdm_engine *e, const void *records, const int *aperture, int ntr,
                         int ns, int big_endian);
int qpsdm_submit_gathers_device(qpsdm_engine *e, const void *d_records,
                                const int *d_aperture, int ntr, int ns, int big_endian);

/* Waits for all submitted work; returns QPSDM_ETIMEOUT / QPSDM_ECUDA on a
 * device-side error. */
int qpsdm_fence(qpsdm_engine *e);

/* Lines of the current brick (qpsdm_set_lines) that the following submits
 * feed: bit il selects line il (lines from 64 on always take every batch);
 * default all.  The reference reads, for each image line, only the data
 * lines within +-extxline of it (src/q-psdm.cu:1432-1435, :1882-1886); a
 * driver imaging a brick in one pass sets, before each data line's traces,
 * the image lines that data line belongs to.  No counterpart in the
 * reference, which images one line per pass. */
int qpsdm_set_line_mask(qpsdm_engine *e, unsigned long long mask);

/* Replaces the D2H + host sum + /nsb of qpsdm() (src/q-psdm.cu:1745-1765).
 * host_img: [nxb][nzi] floats (nxb = ixend - ixstart). */
int qpsdm_get_image(qpsdm_engine *e, float *host_img, int apply_nsb_scale);

/* The same read as qpsdm_get_image, enqueued instead of waited for, so that
 * a caller can overlap the next batch's host-to-device copy with this one's
 * kernels and still read every batch's result (the reference's D2H + host sum
 * + /nsb of src/q-psdm.cu:1745-1765, which it does once per offset group).
 * host_img: page-locked host memory (cudaMallocHost / cudaHostRegister) of
 * [lines][nxb][nzi] floats; the copy runs on the engine's compute stream
 * after every kernel of the submits so far and before those of any later
 * submit.  *ticket identifies it; qpsdm_image_wait(e, ticket) returns once
 * the image is in host_img (divided by nsb if apply_nsb_scale).  At most 4
 * reads are outstanding: a fifth first waits for the oldest.  host_img must
 * stay untouched until its wait returns. */
int qpsdm_get_image_async(qpsdm_engine *e, float *host_img, int apply_nsb_scale,
                          int64_t *ticket);
int qpsdm_image_wait(qpsdm_engine *e, int64_t ticket);

/* Device pointer of the block image [nxb][nzi] (FP32) for zero-copy use. */
int qpsdm_image_device_ptr(qpsdm_engine *e, float **d_img);

/* Runs the engine's kernels on `stream` (a cudaStream_t of the engine's
 * device) instead of its own stream; NULL restores the engine's stream.
 * Lets a caller order engine work with its own kernels, time it with its own
 * events, or capture it into a CUDA graph.  In the batched physics form the
 * lines of a brick alternate between this stream and an internal second
 * stream, which forks from this stream after the batch's panels and joins
 * it again before the submit's work ends, so everything a submit enqueues is
 * ordered before the stream's later work (and captured with it). */
int qpsdm_set_stream(qpsdm_engine *e, void *stream);

/* Kernel timing: with profiling on, every launch of the engine is bracketed
 * by CUDA events on the stream it runs on.  qpsdm_profile_get sums the
 * elapsed device time (ms) and launches of one kernel class since the last
 * enable (waits for the stream).  Kernel classes: */
enum { QPSDM_K_GATE = 0, QPSDM_K_PRE = 1, QPSDM_K_IMAGE = 2, QPSDM_K_OTHER = 3 };
int qpsdm_profile_enable(qpsdm_engine *e, int on);
int qpsdm_profile_get(qpsdm_engine *e, int kernel_class, double *total_ms,
                      int64_t *launches);

/* Batched physics form: the image-kernel variant the autotuner chose on the
 * first batch (tile depth x cdps, minimum resident blocks per SM) and the
 * timing of every variant (ms, up to nms values).  Returns the number of
 * variants, or a negative/error status.  No reference counterpart. */
int qpsdm_tuning_info(qpsdm_engine *e, int *variant, int *tile_z, int *tile_x,
                      int *min_blocks, float *ms, int nms);

/* Counters since begin_offset: traces accepted by the gate (summed over the
 * lines of the brick: a trace accepted by two lines counts twice; counted on
 * the device, so batches replayed from CUDA graphs count too) and point-traces
 * evaluated (one per image point inside a trace's aperture). */
int qpsdm_get_counters(qpsdm_engine *e, int64_t *traces_accepted,
                       int64_t *point_traces);

/* Counters since begin_offset, up to n of: [0] traces accepted by the gate,
 * [1] point-traces, [2] point-traces decided for a whole image tile by the
 * batched kernel (members whose dip test fails at every point of the tile;
 * 0 in the plain form), [3] point-traces imaged (past the dip test and the
 * time window; 0 in compat mode).  Returns the number of counters (4).  No
 * counterpart in the reference, which counts nothing. */
int qpsdm_get_stats(qpsdm_engine *e, int64_t *out, int n);

/* Per-trace spectra of the last submit (re, im: [ntr][2*nww], rejected
 * traces untouched), as psdm_kernel leaves them in red/imd
 * (src/q-psdm.cu:2186-2219).  Device pointers, valid until the next submit. */
int qpsdm_spectra_device_ptr(qpsdm_engine *e, float **d_re, float **d_im);

/* Physics mode: the t*-binned compensated panels of the last submit,
 * [ntr][nbins][nffti] in the engine's panel type (the plain form holds the
 * last image line's accepted traces, the batched form every trace some line
 * of the brick accepted), and for FP16 panels the per-trace sample
 * multipliers [ntr] (powers of two).  Device pointers, valid until the next
 * submit.  The panels stand where psdm_kernel leaves its spectra (red/imd,
 * src/q-psdm.cu:2186-2219). */
int qpsdm_panels_device_ptr(qpsdm_engine *e, void **d_panels, float **d_pscale);

/* Per-trace gate results of the last submit: [ntr][8] ints
 * (status, cdpx, cdpy, iaz, ixi1, ixi2, ntibeg, izimin) and [ntr][4] floats
 * (sx, sy, gx, gy relative to fxi, cyi).  Device pointers. */
int qpsdm_gate_device_ptr(qpsdm_engine *e, int **d_ints, float **d_geom);

/* ---- table generation (the files get_ttt_all reads) -----------------------*/

/* Gridded model: velocity (m/s) and 1/Q on [nz][ny][nx] nodes of spacing h
 * with origin (ox, oy) at the surface; (v0, kz) is the linear-gradient
 * background used to start each source analytically. */
typedef struct {
  int nx, ny, nz;
  float h, ox, oy;
  float v0, kz;
} qpsdm_eik_model;

/* Local grid of every source of a batch: nx x ny x nz nodes of spacing h. */
typedef struct {
  int nx, ny, nz;
  float h;
} qpsdm_eik_grid;

/* Traveltime T and t* of nsrc surface sources on their local grids
 * (d_T, d_tstar: [nsrc][nz][ny][nx]).  d_src: nsrc x (sx, sy, ox, oy) floats,
 * source position and local-grid origin in model coordinates.  d_work:
 * QPSDM_EIK_WORK_FLOATS(nsrc * nx*ny*nz) floats of scratch, 8-byte aligned.
 * First-order Godunov upwind updates relaxed until nothing changes (at most
 * max_iter sweeps), the analytic background held inside init_radius of the
 * source; t* is transported in FP64 and stored as float.  The
 * generator of the L<line>.ttt / .qqq data read by get_ttt_all
 * (src/q-psdm.cu:2382-2627); no counterpart of its own in the reference. */
#define QPSDM_EIK_WORK_FLOATS(n) (4 * (size_t)(n) + 4)
int qpsdm_eikonal_solve(const float *d_vel, const float *d_invq,
                        const qpsdm_eik_model *model, const float *d_src, int nsrc,
                        const qpsdm_eik_grid *grid, float init_radius, int max_iter,
                        float *d_work, float *d_T, float *d_tstar, void *stream);

/* Geometry of the line table being filled (reference layout). */
typedef struct {
  int nxi1, nzi1, nzg;
  float dxi, dzii;
  float x_cdp1; /* model x of the table's first cdp */
  float line_y; /* model y of the image line */
} qpsdm_eik_fill_geom;

/* Writes every table entry whose source is in this solved batch
 * (sources s0 .. s0+ns-1, d_src of the batch) by trilinear sampling of the
 * grids: entries of cell c are block c of the descriptors (d_cell_base:
 * ncell+1 prefix sums of block sizes), node_src maps (cell, surface node) to
 * the global source number (d_node_base: ncell+1 prefix sums of nodes). */
int qpsdm_eikonal_fill(const float *d_T, const float *d_tstar, const qpsdm_eik_grid *grid,
                       const float *d_src, int s0, int ns, const qpsdm_ttt_desc *d_desc,
                       const int64_t *d_cell_base, const int *d_node_base,
                       const int *d_node_src, int ncell, const qpsdm_eik_fill_geom *fg,
                       float *d_ttt, float *d_qqq, void *stream);

/* ---- standalone kernels (device pointers) ---------------------------------*/

/* Batched real-to-complex FFT, unnormalised, e^{-iwt} (the convention of
 * pfarc with isign = -1, src/fft.cc:1838-1910).  n: an npfar length.
 * d_in [batch][n] floats, d_out [batch][n/2+1] interleaved complex. */
int qpsdm_fft_r2c(const float *d_in, int n, int batch, float *d_out,
                  void *stream);

/* Batched complex-to-real inverse, unnormalised, e^{+iwt}
 * (pfacr with isign = +1, src/fft.cc:1768-1836). */
int qpsdm_fft_c2r(const float *d_in, int n, int batch, float *d_out,
                  void *stream);

/* Same transform and result as qpsdm_fft_r2c, for callers that may not
 * allocate device memory (a host framework whose own pool owns all of HBM,
 * or a latency-critical caller that cannot take the device synchronisation
 * an allocation may cause).  No counterpart in the reference.
 * Allocates nothing: its twiddle tables live in a fixed device array built
 * into the library (QPSDM_FFT_NOALLOC_MAX_N + 1 complex floats, 64 KiB per
 * GPU that loads the library, held until exit).  n above
 * QPSDM_FFT_NOALLOC_MAX_N returns QPSDM_ESIZE.  Every call shares that array:
 * calls that overlap on the GPU race and must be serialised.  The first call
 * on a device looks up the array's device address; make it before any
 * stream capture. */
#define QPSDM_FFT_NOALLOC_MAX_N 8192
int qpsdm_fft_r2c_noalloc(const float *d_in, int n, int batch, float *d_out,
                          void *stream);

/* ---------------------------------------------------------------------------
 * Learned traveltime / t* surrogate (no counterpart in the reference, which
 * reads precomputed tables only).
 *
 * A 5 -> 128 x 4 (SiLU) -> 2 multilayer perceptron: inputs (source x, source
 * y, point x, point y, point z), outputs two table corrections.  BF16 weights
 * and activations on the tcgen05 tensor cores, FP32 accumulation, FP32 master
 * weights and Adam moments.  Inputs are normalised on the device as
 * (raw - in_shift) * in_scale; the training loss is
 *   sum_s sum_j out_weight[j] (y_j - t_j)^2 / n.
 * The parameter vector (qpsdm_mlp_param_count() floats) is, in order:
 * W1 [128][16] (input columns 5..15 are padding, kept at zero), b1 [128],
 * W2 [128][128], b2, W3, b3, W4, b4, W5 [16][128] (rows 2..15 padding), b5 [16].
 * Training kernels write per-CTA gradient slices that are summed in a fixed
 * order: gradients and training are deterministic for a given launch size.
 * Device pointers: d_x [n][5], d_t [n][2], d_y [n][2] floats.
 * ------------------------------------------------------------------------- */
typedef struct qpsdm_mlp qpsdm_mlp;
int qpsdm_mlp_create(int device, qpsdm_mlp **out);
int qpsdm_mlp_destroy(qpsdm_mlp *h);
int qpsdm_mlp_param_count(void);
/* Replace the parameters (host array) and reset the Adam state. */
int qpsdm_mlp_set_params(qpsdm_mlp *h, const float *host_params);
int qpsdm_mlp_get_params(qpsdm_mlp *h, float *host_params);
int qpsdm_mlp_set_scaling(qpsdm_mlp *h, const float *in_shift,
                          const float *in_scale, const float *out_weight);
/* Loss and its gradient over all n samples (no update); host_grads
 * (param_count floats) and loss may be NULL.  Synchronises the stream. */
int qpsdm_mlp_gradients(qpsdm_mlp *h, const float *d_x, const float *d_t,
                        int n, float *host_grads, float *loss, void *stream);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8) on the n samples given; when
 * loss is not NULL the loss before the step is returned (synchronises). */
int qpsdm_mlp_train_step(qpsdm_mlp *h, const float *d_x, const float *d_t,
                         int n, float lr, float *loss, void *stream);
/* Inference, asynchronous on stream. */
int qpsdm_mlp_forward(qpsdm_mlp *h, const float *d_x, int n, float *d_y,
                      void *stream);
/* Synchronise; QPSDM_ETIMEOUT if a tensor-core wait gave up in any kernel
 * since the handle was created. */
int qpsdm_mlp_status(qpsdm_mlp *h);

/* ---- the surrogate and the tables ------------------------------------------
 * Outputs of the network are corrections (ms) to the linear-gradient
 * background: T = T_bg + y0 / 1000, t* = T_bg / q_ref + y1 / 1000, with T_bg
 * the exact traveltime of v = v0 + kz z from the surface point.  Coordinates
 * are model coordinates (x from the first image cdp, y of the eikonal model). */
typedef struct {
  float v0, kz;  /* background velocity law */
  float q_ref;   /* background t* = T_bg / q_ref of the network's targets */
  float q_bg;    /* constant Q of the background solves (d_T_bg, d_tstar_bg) */
} qpsdm_sur_background;

/* Training samples drawn from solved grids (qpsdm_eikonal_solve of ns
 * sources, d_src as there): nsamples uniform (source, node) pairs from the
 * hash of seed; d_x [n][5] = (sx, sy, x, y, z), d_t [n][2] = the corrections
 * (ms) of T and t*.  With the background's own solves on the same grids
 * (d_T_bg, d_tstar_bg, both or neither) the values are corrected as the
 * tables are: T = T_bg + T - T_bgsolve, t* = t* (T_bg / q_bg) / t*_bgsolve.
 * A set of sources x volume points is never materialised: each batch of
 * sources yields its samples while its grids are on the device.  No
 * counterpart in the reference (it reads precomputed tables). */
int qpsdm_eikonal_samples(const float *d_T, const float *d_tstar, const float *d_T_bg,
                          const float *d_tstar_bg, const qpsdm_eik_grid *grid,
                          const float *d_src, int ns, const qpsdm_sur_background *bg,
                          uint64_t seed, int nsamples, float *d_x, float *d_t, void *stream);

/* One image line's tables as the surrogate sees them (reference layout,
 * surface grid of a cell centred on its middle cdp and on the line). */
typedef struct {
  int nxg, nzg, nxi1, nzi1;
  int tcdp1;       /* first table cdp relative to the first image cdp */
  float dxi, dzii; /* cdp spacing, depth-node spacing (m) */
  float line_y;    /* model y of the line */
  float v0, kz, q_ref; /* the network's background */
} qpsdm_sur_line;

/* Table data of `line` between the lines line_lo <= line <= line_hi that
 * have table files (d_lo, d_hi: n floats each, device): d_out = d_lo c1 +
 * d_hi c2 with c2 = (line - line_lo) / (line_hi - line_lo), c1 = 1 - c2, in
 * float without fused multiply-adds -- the interpolation of get_ttt_all
 * (src/q-psdm.cu:2584-2596) on the device, bit for bit.  Asynchronous. */
int qpsdm_tables_lerp(const float *d_lo, const float *d_hi, int64_t n, int line, int line_lo,
                      int line_hi, float *d_out, void *stream);

/* Background correction of a line's eikonal tables in place: with d_ttt_bg,
 * d_qqq_bg the same line's tables from solves of the linear-gradient
 * background (v0, kz of ln, constant Q = q_bg) on the same grids,
 * T = T_bg + T - T_bgsolve and t* = t* (T_bg / q_bg) / t*_bgsolve, T_bg exact:
 * the first-order scheme's systematic error cancels.  Synchronises. */
int qpsdm_eikonal_correct(const qpsdm_sur_line *ln, const qpsdm_ttt_desc *desc, float *d_ttt,
                          float *d_qqq, const float *d_ttt_bg, const float *d_qqq_bg,
                          int64_t len, float q_bg, void *stream);

/* The network's traveltime error (ms) against the line's tables at every
 * surface node of every cell, the maximum over the node's points,
 * max-accumulated into d_node_err (float per node, cells in descriptor
 * order, nodes [iys][ixs]; clear it first: calls for several lines give the
 * maximum over them).  desc: host descriptors; d_ttt: len floats (device).
 * Synchronises the stream. */
int qpsdm_surrogate_gate(qpsdm_mlp *net, const qpsdm_sur_line *ln, const qpsdm_ttt_desc *desc,
                         const float *d_ttt, int64_t len, float *d_node_err, void *stream);

/* Tables of the line on the surface grids of fine_desc (same cells as
 * coarse_desc) from the network; in every coarse patch whose corner nodes
 * the network missed by more than gate_ms (d_node_err as written by
 * qpsdm_surrogate_gate) the fine values are the bilinear interpolation of
 * the coarse tables instead (the plain method keeps the last word on the
 * network's error).  gated_nodes (may be NULL): fine surface nodes of all
 * cells that kept the tables.  Replaces, for this line, the table lookup the
 * reference stages for its kernel (src/q-psdm.cu:2343-2357) with denser
 * tables.  Synchronises the stream. */
int qpsdm_surrogate_tables(qpsdm_mlp *net, const qpsdm_sur_line *ln,
                           const qpsdm_ttt_desc *coarse_desc, const float *d_cttt,
                           const float *d_cqqq, int64_t coarse_len, const float *d_node_err,
                           float gate_ms, const qpsdm_ttt_desc *fine_desc, float *d_fttt,
                           float *d_fqqq, int64_t fine_len, int64_t *gated_nodes, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* QPSDM_ENGINE_H_ */
