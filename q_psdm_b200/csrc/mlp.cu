// mlp.cu -- the learned traveltime / t* surrogate on 5th-generation tensor cores.
//
// Network: 5 inputs (padded to 16) -> 4 x 128 (SiLU) -> 2 outputs (padded to
// 16).  BF16 weights and activations, FP32 accumulation in tensor memory,
// FP32 master weights and Adam moments in global memory.
//
// Every layer is one 128-sample tcgen05 tile GEMM (tc.cuh): activations are
// the A operand ([sample][feature], K-major), weights [out][in] the B
// operand, the FP32 accumulator 128 TMEM columns.  A team of 8 warps owns a
// tile: warp w reads TMEM lane quarter (w mod 4) -- the quarter a warp may
// access is fixed by its warp index -- and column half (w / 4), so the
// epilogue of a layer (bias, SiLU, BF16 store) is spread over 256 threads.
//
// Inference: two teams per CTA work on two tiles at once, each with its own
// mbarrier, TMEM columns and activation buffer (a layer's output overwrites
// its input once the MMA that read it has completed), so one team's MMAs run
// while the other team is in its epilogue.  Each thread loads its inputs of
// the next tile while the current one is computed.
//
// Training: one team per CTA.  Backward re-computes what it needs (all
// activations do not fit in shared memory next to the weights) and forms
//   dW_l = dZ_l^T H_{l-1}   (A = dZ MN-major view, B = H MN-major view)
//   dH_{l-1} = dZ_l W_l      (A = dZ K-major, B = W MN-major view)
// Each CTA accumulates gradients into its own slice of a global buffer
// (plain read-modify-write, no atomics); bias gradients are reduced across
// a warp by a butterfly transpose-sum and across warps in a fixed order; a
// reduction over the slices in a fixed order and an Adam step follow, so
// training is deterministic.
//
// SiLU(z) = z sigma(z) = h + h tanh(h), h = z / 2, with the hardware FP32
// tanh (tanh.approx.f32, about 2^-11 relative, below the BF16 rounding of
// the stored activations).  (The packed f16x2 tanh would halve the
// special-function work of the epilogue, the inference kernel's limiter,
// but its error is no longer small against BF16.)
#include <cuda_bf16.h>
#include <math.h>

#include <vector>

#include "common.cuh"
#include "qpsdm_engine.h"
#include "tc.cuh"

namespace qpsdm {

constexpr int kH = 128, kIn = 16, kOut = 16, kTile = 128;
// FP32 parameter block offsets
constexpr int oW1 = 0, oB1 = oW1 + kH * kIn;
constexpr int oW2 = oB1 + kH, oB2 = oW2 + kH * kH;
constexpr int oW3 = oB2 + kH, oB3 = oW3 + kH * kH;
constexpr int oW4 = oB3 + kH, oB4 = oW4 + kH * kH;
constexpr int oW5 = oB4 + kH, oB5 = oW5 + kOut * kH;
constexpr int kParams = oB5 + kOut;  // 53776
constexpr int kSlice = kParams + 16;  // + loss sum and padding
// BF16 weight images in the core-matrix layout (bytes)
constexpr int sW1 = 0, sW2 = sW1 + kH * kIn * 2, sW3 = sW2 + kH * kH * 2;
constexpr int sW4 = sW3 + kH * kH * 2, sW5 = sW4 + kH * kH * 2;
constexpr int kWBytes = sW5 + kOut * kH * 2;  // 106496
constexpr int kTeam = 256;                    // threads of a team
constexpr int kXBytes = kTile * kIn * 2, kHBytes = kTile * kH * 2;
// biases in shared memory: half biases of layers 1-4 (the SiLU argument is
// h = (z + b) / 2), then b5
constexpr int kBiasBytes = (4 * kH + kOut) * 4;  // 2112
// training shared memory map
constexpr int sX = kWBytes;                   // [128][16] bf16
constexpr int sH0 = sX + kXBytes;             // [128][128] bf16
constexpr int sH1 = sH0 + kHBytes;
constexpr int sG = sH1 + kHBytes;             // dZ, [128][128] or [128][16]
constexpr int sBias = sG + kHBytes;
constexpr int sDb = sBias + kBiasBytes;       // fp32 bias-gradient partials [4 quarters][128]
constexpr int sLoss = sDb + 4 * kH * 4;       // fp32 loss partials [8 warps]
constexpr int kSmem = sLoss + 32;             // 214,112 bytes
// inference shared memory map: weights, biases, then per team X and H
constexpr int fBias = kWBytes;
constexpr int fTeam0 = fBias + 2304;
constexpr int kFwdSmem = fTeam0 + 2 * (kXBytes + kHBytes);  // 182,528 bytes

struct MlpTileArgs {
  float in_scale[5], in_shift[5];  // features = (raw - shift) * scale
  float w_out[2];                  // loss weights of the two outputs
  float inv_batch;
};

__device__ __forceinline__ float tanh_hw(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
// h = (z + b) / 2 -> SiLU(z + b)
__device__ __forceinline__ float silu_h(float h) { return fmaf(h, tanh_hw(h), h); }
// SiLU'(u) = s (1 + u (1 - s)), s = sigma(u) = (1 + tanh(u / 2)) / 2, h = u / 2
__device__ __forceinline__ float silu_grad_h(float h) {
  const float s = fmaf(0.5f, tanh_hw(h), 0.5f);
  return s * fmaf(2.0f * h, 1.0f - s, 1.0f);
}

// 8 bf16 of row r, columns c..c+7 of a K-major core-matrix buffer (rowlen K).
__device__ __forceinline__ void st_row8(uint8_t *buf, int r, int c, int K, const float *v) {
  __nv_bfloat162 p[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) p[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
  *reinterpret_cast<uint4 *>(buf + tc::kmaj_off(r, c, K)) = *reinterpret_cast<uint4 *>(p);
}

// A group of threads synchronised by its own named barrier.
struct Team {
  uint32_t id, nthr;
  __device__ __forceinline__ void sync() const {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthr) : "memory");
  }
  // true on every thread of the team if p is true on any
  __device__ __forceinline__ bool any(bool p) const {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred q, %2, %3, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)p), "r"(id), "r"(nthr)
        : "memory");
    return r != 0;
  }
};

// Position of a team thread: TMEM lane quarter, column half, tile row.
struct Role {
  int lane, quarter, half, row;
  uint32_t lane_base;  // TMEM address bits of the quarter's first lane
  __device__ __forceinline__ explicit Role(int t) {
    const int w = t >> 5;
    lane = t & 31;
    quarter = w & 3;
    half = w >> 2;
    row = quarter * 32 + lane;
    lane_base = (uint32_t)(quarter * 32) << 16;
  }
};

struct Gemm {
  Team team;
  uint64_t *bar;
  uint32_t phase;
  int *err;
  bool leader;
  // D (TMEM) = A * B^T.  a/b: core-matrix buffers with storage row length
  // a_len/b_len; *_mn = 1 reads the buffer transposed (MN-major).  K: the
  // reduction length.  Every team thread calls; the leader issues.  The
  // result is the same on every thread: false if the wait gave up.
  __device__ __forceinline__ bool run(uint32_t d, const uint8_t *a, int a_len, int a_mn,
                                      const uint8_t *b, int b_len, int b_mn, int N, int K) {
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    team.sync();
    tc::fence_after_sync();
    if (leader) {
      const uint32_t a_lbo = a_mn ? (a_len / 8) * 128 : 128, a_sbo = a_mn ? 128 : (a_len / 8) * 128;
      const uint32_t b_lbo = b_mn ? (b_len / 8) * 128 : 128, b_sbo = b_mn ? 128 : (b_len / 8) * 128;
      tc::gemm_issue(d, tc::smem_u32(a), a_lbo, a_sbo, a_mn ? 2 * a_lbo : 256, tc::smem_u32(b),
                     b_lbo, b_sbo, b_mn ? 2 * b_lbo : 256, tc::idesc_bf16(128, N, a_mn, b_mn), K,
                     false, bar);
    }
    const bool timed_out = !tc::mbar_wait(bar, phase, 1u << 30);
    phase ^= 1u;
    const bool ok = !team.any(timed_out);
    if (!ok && leader) atomicExch(err, 1);
    tc::fence_after_sync();
    return ok;
  }
};

// 64 accumulator columns [c0, c0+64) of this thread's row.
__device__ __forceinline__ void acc_ld64(uint32_t acc, const Role &ro, int c0, float *v) {
  uint32_t r[64];
#pragma unroll
  for (int k = 0; k < 4; ++k) tc::tmem_ld16_nowait(acc + ro.lane_base + c0 + 16 * k, r + 16 * k);
#pragma unroll
  for (int k = 0; k < 4; ++k) tc::tmem_wait_ld_dep16(r + 16 * k);
#pragma unroll
  for (int i = 0; i < 64; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void acc_ld16(uint32_t acc, const Role &ro, int c0, float *v) {
  tc::tmem_ld16(acc + ro.lane_base + c0, v);
}

// H = SiLU(acc + b) for this thread's 64 columns, into a [128][128] buffer.
__device__ __forceinline__ void epi_silu(uint32_t acc, const Role &ro, const float *hb,
                                         uint8_t *hout) {
  const int c0 = ro.half * 64;
  float v[64];
  acc_ld64(acc, ro, c0, v);
#pragma unroll
  for (int i = 0; i < 64; ++i) v[i] = silu_h(fmaf(0.5f, v[i], hb[c0 + i]));
#pragma unroll
  for (int k = 0; k < 8; ++k) st_row8(hout, ro.row, c0 + 8 * k, kH, v + 8 * k);
}

// Normalised features of one sample into the X tile (zero padding to 16).
__device__ __forceinline__ void put_raw(uint8_t *sx, int row, const float *raw, bool live,
                                        const MlpTileArgs &ta) {
  float v[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = 0.0f;
  if (live)
#pragma unroll
    for (int j = 0; j < 5; ++j) v[j] = (raw[j] - ta.in_shift[j]) * ta.in_scale[j];
  st_row8(sx, row, 0, kIn, v);
  st_row8(sx, row, 8, kIn, v + 8);
}
__device__ __forceinline__ void load_raw(const float *__restrict__ x, int s, bool live,
                                         float *raw) {
#pragma unroll
  for (int j = 0; j < 5; ++j) raw[j] = live ? __ldg(x + (size_t)s * 5 + j) : 0.0f;
}
__device__ __forceinline__ void put_x(uint8_t *sx, int row, const float *__restrict__ x, int s,
                                      bool live, const MlpTileArgs &ta) {
  float raw[5];
  load_raw(x, s, live, raw);
  put_raw(sx, row, raw, live, ta);
}

// Copy weights (bf16 images) and biases (half biases for layers 1-4).
__device__ __forceinline__ void load_weights(uint8_t *sm, float *bias,
                                             const uint8_t *__restrict__ wimg,
                                             const float *__restrict__ params) {
  const uint4 *src = reinterpret_cast<const uint4 *>(wimg);
  uint4 *dst = reinterpret_cast<uint4 *>(sm);
  for (int i = threadIdx.x; i < kWBytes / 16; i += blockDim.x) dst[i] = src[i];
  for (int i = threadIdx.x; i < kH; i += blockDim.x) {
    bias[i] = 0.5f * params[oB1 + i];
    bias[kH + i] = 0.5f * params[oB2 + i];
    bias[2 * kH + i] = 0.5f * params[oB3 + i];
    bias[3 * kH + i] = 0.5f * params[oB4 + i];
  }
  if (threadIdx.x < kOut) bias[4 * kH + threadIdx.x] = params[oB5 + threadIdx.x];
}

// ---------------------------------------------------------------------------
// inference: y[n][2] from x[n][5]; two teams of 256 threads per CTA
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(2 * kTeam, 1)
    k_mlp_forward(const uint8_t *__restrict__ wimg, const float *__restrict__ params,
                  const float *__restrict__ x, int nsamp, MlpTileArgs ta, float *__restrict__ y,
                  int *err) {
  extern __shared__ __align__(1024) uint8_t sm[];
  __shared__ uint64_t bars[2];
  __shared__ uint32_t tslot;
  const int tid = threadIdx.x, team_id = tid / kTeam, t = tid % kTeam;
  if (tid < 32) tc::tmem_alloc(&tslot, 256);
  if (tid == 0) {
    tc::mbar_init(&bars[0], 1);
    tc::mbar_init(&bars[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  float *bias = reinterpret_cast<float *>(sm + fBias);
  load_weights(sm, bias, wimg, params);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const Role ro(t);
  uint8_t *sx = sm + fTeam0 + team_id * (kXBytes + kHBytes), *sh = sx + kXBytes;
  const uint32_t acc = tslot + 128 * team_id;
  Gemm g{Team{1u + team_id, kTeam}, &bars[team_id], 0u, err, t == 0};
  const int ntiles = (nsamp + kTile - 1) / kTile;
  // this thread's inputs of its next tile, loaded one tile ahead
  float raw[5];
  {
    const int s0 = (2 * blockIdx.x + team_id) * kTile + ro.row;
    load_raw(x, s0, ro.half == 0 && s0 < nsamp, raw);
  }
  for (int tile = 2 * blockIdx.x + team_id; tile < ntiles; tile += 2 * gridDim.x) {
    const int s = tile * kTile + ro.row;
    const bool live = s < nsamp;
    if (ro.half == 0) {
      put_raw(sx, ro.row, raw, live, ta);
      const int sn = s + 2 * gridDim.x * kTile;
      load_raw(x, sn, sn < nsamp, raw);
    }
    if (!g.run(acc, sx, kIn, 0, sm + sW1, kIn, 0, kH, kIn)) break;
    epi_silu(acc, ro, bias, sh);
    bool ok = true;
    for (int l = 1; l < 4 && ok; ++l) {
      ok = g.run(acc, sh, kH, 0, sm + sW2 + (l - 1) * kH * kH * 2, kH, 0, kH, kH);
      if (ok) epi_silu(acc, ro, bias + l * kH, sh);
    }
    if (!ok || !g.run(acc, sh, kH, 0, sm + sW5, kH, 0, kOut, kH)) break;
    if (ro.half == 0) {
      float v[16];
      acc_ld16(acc, ro, 0, v);
      if (live) {
        y[(size_t)s * 2] = v[0] + bias[4 * kH];
        y[(size_t)s * 2 + 1] = v[1] + bias[4 * kH + 1];
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (tid < 32) tc::tmem_free(tslot, 256);
}

// ---------------------------------------------------------------------------
// training
// ---------------------------------------------------------------------------
// Butterfly transpose-sum of 64 per-lane values over the warp: afterwards
// lane l holds in v[0], v[1] the sums of columns 2l and 2l+1 (fixed order).
template <int O, int N>
__device__ __forceinline__ void xsum_step(float *v, int lane) {
  const bool up = (lane & O) != 0;
#pragma unroll
  for (int i = 0; i < N / 2; ++i) {
    const float send = up ? v[i] : v[i + N / 2];
    const float keep = up ? v[i + N / 2] : v[i];
    v[i] = keep + __shfl_xor_sync(0xffffffffu, send, O);
  }
}
__device__ __forceinline__ void xsum64(float *v, int lane) {
  xsum_step<16, 64>(v, lane);
  xsum_step<8, 32>(v, lane);
  xsum_step<4, 16>(v, lane);
  xsum_step<2, 8>(v, lane);
  xsum_step<1, 4>(v, lane);
}

// dZ = dH (acc1) * SiLU'(Z + b) (Z in acc0) into sG for this thread's 64
// columns; this warp's bias-gradient partials (its 32 rows) into
// sDb[quarter][column].
__device__ __forceinline__ void dz_epilogue(uint32_t acc0, uint32_t acc1, const Role &ro,
                                            const float *hb, uint8_t *sm, bool live) {
  const int c0 = ro.half * 64;
  float d[64];
  {
    float z[64];
    acc_ld64(acc0, ro, c0, z);
    acc_ld64(acc1, ro, c0, d);
#pragma unroll
    for (int i = 0; i < 64; ++i)
      d[i] = live ? d[i] * silu_grad_h(fmaf(0.5f, z[i], hb[c0 + i])) : 0.0f;
  }
#pragma unroll
  for (int k = 0; k < 8; ++k) st_row8(sm + sG, ro.row, c0 + 8 * k, kH, d + 8 * k);
  xsum64(d, ro.lane);
  float *db = reinterpret_cast<float *>(sm + sDb) + ro.quarter * kH + c0 + 2 * ro.lane;
  db[0] = d[0];
  db[1] = d[1];
}

// add the four quarters' bias partials (in order) to the gradient slice
__device__ __forceinline__ void flush_db(const Team &team, uint8_t *sm, float *gs, int off,
                                         int n) {
  team.sync();
  const float *db = reinterpret_cast<const float *>(sm + sDb);
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    gs[off + i] += ((db[i] + db[kH + i]) + db[2 * kH + i]) + db[3 * kH + i];
  team.sync();
}

// dW [128 out][128 in] tile (rows = TMEM lanes) into the slice, this
// thread's row and 64 columns.
__device__ __forceinline__ void add_grad128(uint32_t acc, const Role &ro, float *gs, int off) {
  const int c0 = ro.half * 64;
  float v[64];
  acc_ld64(acc, ro, c0, v);
  float4 *p = reinterpret_cast<float4 *>(gs + off + ro.row * kH + c0);
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    float4 q = p[k];
    q.x += v[4 * k];
    q.y += v[4 * k + 1];
    q.z += v[4 * k + 2];
    q.w += v[4 * k + 3];
    p[k] = q;
  }
}

// x: [n][5], t: [n][2]; grads: [gridDim.x][kSlice] (slice zeroed here)
__global__ void __launch_bounds__(kTeam, 1)
    k_mlp_grad(const uint8_t *__restrict__ wimg, const float *__restrict__ params,
               const float *__restrict__ x, const float *__restrict__ t, int nsamp,
               MlpTileArgs ta, float *__restrict__ grads, int *err) {
  extern __shared__ __align__(1024) uint8_t sm[];
  __shared__ uint64_t bar;
  __shared__ uint32_t tslot;
  const int tid = threadIdx.x;
  float *gs = grads + (size_t)blockIdx.x * kSlice;
  for (int i = tid; i < kSlice; i += blockDim.x) gs[i] = 0.0f;
  if (tid < 32) tc::tmem_alloc(&tslot, 256);
  if (tid == 0) {
    tc::mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  float *bias = reinterpret_cast<float *>(sm + sBias);
  load_weights(sm, bias, wimg, params);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t acc0 = tslot, acc1 = tslot + 128;
  const Role ro(tid);
  const Team team{1u, kTeam};
  Gemm g{team, &bar, 0u, err, tid == 0};
  float loss = 0.0f;
  const int ntiles = (nsamp + kTile - 1) / kTile;
  bool ok = true;
  for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const int s = tile * kTile + ro.row;
    const bool live = s < nsamp;
    if (ro.half == 0) put_x(sm + sX, ro.row, x, s, live, ta);
    // forward: H1 sH0, H2 sH1, H3 sH0, H4 sH1
    if (!(ok = g.run(acc0, sm + sX, kIn, 0, sm + sW1, kIn, 0, kH, kIn))) break;
    epi_silu(acc0, ro, bias, sm + sH0);
    if (!(ok = g.run(acc0, sm + sH0, kH, 0, sm + sW2, kH, 0, kH, kH))) break;
    epi_silu(acc0, ro, bias + kH, sm + sH1);
    if (!(ok = g.run(acc0, sm + sH1, kH, 0, sm + sW3, kH, 0, kH, kH))) break;
    epi_silu(acc0, ro, bias + 2 * kH, sm + sH0);
    if (!(ok = g.run(acc0, sm + sH0, kH, 0, sm + sW4, kH, 0, kH, kH))) break;
    epi_silu(acc0, ro, bias + 3 * kH, sm + sH1);
    if (!(ok = g.run(acc1, sm + sH1, kH, 0, sm + sW5, kH, 0, kOut, kH))) break;
    // loss and dZ5 = dY ([128][16] tile in sG, 2 live columns)
    if (ro.half == 0) {
      float v[16], d5[16];
      acc_ld16(acc1, ro, 0, v);
#pragma unroll
      for (int j = 0; j < 16; ++j) d5[j] = 0.0f;
      if (live) {
        const float e0 = v[0] + bias[4 * kH] - t[(size_t)s * 2];
        const float e1 = v[1] + bias[4 * kH + 1] - t[(size_t)s * 2 + 1];
        loss += ta.w_out[0] * e0 * e0 + ta.w_out[1] * e1 * e1;
        d5[0] = 2.0f * ta.w_out[0] * e0 * ta.inv_batch;
        d5[1] = 2.0f * ta.w_out[1] * e1 * ta.inv_batch;
      }
      st_row8(sm + sG, ro.row, 0, kOut, d5);
      st_row8(sm + sG, ro.row, 8, kOut, d5 + 8);
      float *db = reinterpret_cast<float *>(sm + sDb) + ro.quarter * kH;
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        float a = d5[j];
        for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        if (ro.lane == 0) db[j] = a;
      }
      if (ro.lane < kOut - 2) db[2 + ro.lane] = 0.0f;
    }
    flush_db(team, sm, gs, oB5, kOut);
    // layer 5: dW5^T = H4^T dZ5 (rows = in), dH4 = dZ5 W5
    if (!(ok = g.run(acc0, sm + sH1, kH, 1, sm + sG, kOut, 1, kOut, kTile))) break;
    if (ro.half == 0) {
      float v[16];
      acc_ld16(acc0, ro, 0, v);
#pragma unroll
      for (int j = 0; j < kOut; ++j) gs[oW5 + j * kH + ro.row] += v[j];
    }
    if (!(ok = g.run(acc1, sm + sG, kOut, 0, sm + sW5, kH, 1, kH, kOut))) break;
    // layer 4: Z4 = H3 W4^T (H3 still in sH0)
    if (!(ok = g.run(acc0, sm + sH0, kH, 0, sm + sW4, kH, 0, kH, kH))) break;
    dz_epilogue(acc0, acc1, ro, bias + 3 * kH, sm, live);
    flush_db(team, sm, gs, oB4, kH);
    if (!(ok = g.run(acc0, sm + sG, kH, 1, sm + sH0, kH, 1, kH, kTile))) break;
    add_grad128(acc0, ro, gs, oW4);
    if (!(ok = g.run(acc1, sm + sG, kH, 0, sm + sW4, kH, 1, kH, kH))) break;
    // layer 3: recompute H1 (sH1), H2 (sH0), Z3
    if (!(ok = g.run(acc0, sm + sX, kIn, 0, sm + sW1, kIn, 0, kH, kIn))) break;
    epi_silu(acc0, ro, bias, sm + sH1);
    if (!(ok = g.run(acc0, sm + sH1, kH, 0, sm + sW2, kH, 0, kH, kH))) break;
    epi_silu(acc0, ro, bias + kH, sm + sH0);
    if (!(ok = g.run(acc0, sm + sH0, kH, 0, sm + sW3, kH, 0, kH, kH))) break;
    dz_epilogue(acc0, acc1, ro, bias + 2 * kH, sm, live);
    flush_db(team, sm, gs, oB3, kH);
    if (!(ok = g.run(acc0, sm + sG, kH, 1, sm + sH0, kH, 1, kH, kTile))) break;
    add_grad128(acc0, ro, gs, oW3);
    if (!(ok = g.run(acc1, sm + sG, kH, 0, sm + sW3, kH, 1, kH, kH))) break;
    // layer 2: H1 in sH1, recompute Z2
    if (!(ok = g.run(acc0, sm + sH1, kH, 0, sm + sW2, kH, 0, kH, kH))) break;
    dz_epilogue(acc0, acc1, ro, bias + kH, sm, live);
    flush_db(team, sm, gs, oB2, kH);
    if (!(ok = g.run(acc0, sm + sG, kH, 1, sm + sH1, kH, 1, kH, kTile))) break;
    add_grad128(acc0, ro, gs, oW2);
    if (!(ok = g.run(acc1, sm + sG, kH, 0, sm + sW2, kH, 1, kH, kH))) break;
    // layer 1: recompute Z1 from X
    if (!(ok = g.run(acc0, sm + sX, kIn, 0, sm + sW1, kIn, 0, kH, kIn))) break;
    dz_epilogue(acc0, acc1, ro, bias, sm, live);
    flush_db(team, sm, gs, oB1, kH);
    if (!(ok = g.run(acc0, sm + sG, kH, 1, sm + sX, kIn, 1, kIn, kTile))) break;
    if (ro.half == 0) {
      float v[16];
      acc_ld16(acc0, ro, 0, v);
      float4 *p = reinterpret_cast<float4 *>(gs + oW1 + ro.row * kIn);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        float4 q = p[k];
        q.x += v[4 * k];
        q.y += v[4 * k + 1];
        q.z += v[4 * k + 2];
        q.w += v[4 * k + 3];
        p[k] = q;
      }
    }
  }
  // loss sum of this CTA, in warp order
  for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
  float *ls = reinterpret_cast<float *>(sm + sLoss);
  if (ro.lane == 0) ls[tid >> 5] = loss;
  tc::fence_before_sync();
  __syncthreads();
  if (tid == 0) {
    float a = 0.0f;
    for (int w = 0; w < kTeam / 32; ++w) a += ls[w];
    gs[kParams] = a * ta.inv_batch;
  }
  if (tid < 32) tc::tmem_free(tslot, 256);
}

// Sum the per-CTA slices in a fixed order.
__global__ void k_mlp_reduce(const float *__restrict__ grads, int nslice, float *__restrict__ g) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kSlice; i += gridDim.x * blockDim.x) {
    float s = 0.0f;
    for (int c = 0; c < nslice; ++c) s += grads[(size_t)c * kSlice + i];
    g[i] = s;
  }
}

// BF16 core-matrix images of the weights (pads stay zero).
__global__ void k_mlp_pack(const float *__restrict__ p, uint8_t *__restrict__ wimg) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kH * kIn + 3 * kH * kH + kOut * kH;
       i += gridDim.x * blockDim.x) {
    int base, off, K, r, k;
    if (i < kH * kIn) {
      base = sW1; off = oW1; K = kIn; r = i / K; k = i % K;
    } else if (i < kH * kIn + 3 * kH * kH) {
      const int j = i - kH * kIn, l = j / (kH * kH), e = j % (kH * kH);
      base = sW2 + l * kH * kH * 2;
      off = oW2 + l * (kH * kH + kH);
      K = kH;
      r = e / K;
      k = e % K;
    } else {
      const int e = i - kH * kIn - 3 * kH * kH;
      base = sW5; off = oW5; K = kH; r = e / K; k = e % K;
    }
    *reinterpret_cast<__nv_bfloat16 *>(wimg + base +
                                       ((r >> 3) * (K >> 3) * 128 + (k >> 3) * 128 + (r & 7) * 16 +
                                        (k & 7) * 2)) = __float2bfloat16_rn(p[off + r * K + k]);
  }
}

// Adam on the FP32 master weights; padded entries are kept at zero.
__global__ void k_mlp_adam(float *__restrict__ p, float *__restrict__ m, float *__restrict__ v,
                           const float *__restrict__ g, const float *__restrict__ mask, float lr,
                           float b1, float b2, float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kParams; i += gridDim.x * blockDim.x) {
    const float gi = g[i] * mask[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] = (p[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps)) * mask[i];
  }
}

}  // namespace qpsdm


// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
using namespace qpsdm;

struct qpsdm_mlp {
  int device = 0, nsm = 0;
  float *p = nullptr, *m = nullptr, *v = nullptr, *g = nullptr, *mask = nullptr;
  float *slices = nullptr;
  uint8_t *wimg = nullptr;
  int *err = nullptr;
  int64_t step = 0;
  MlpTileArgs ta{};
};

static int mlp_grid(const qpsdm_mlp *h, int nsamp) {
  const int ntiles = (nsamp + kTile - 1) / kTile;
  return ntiles < h->nsm ? ntiles : h->nsm;
}

extern "C" int qpsdm_mlp_create(int device, qpsdm_mlp **out) {
  if (!out) return QPSDM_EINVAL;
  *out = nullptr;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return QPSDM_ECUDA;
  if (prop.major != 10 || prop.minor != 0) return QPSDM_ENOKERNEL;
  cudaSetDevice(device);
  auto *h = new qpsdm_mlp;
  h->device = device;
  h->nsm = prop.multiProcessorCount;
  bool ok = cudaMalloc(&h->p, sizeof(float) * kParams) == cudaSuccess &&
            cudaMalloc(&h->m, sizeof(float) * kParams) == cudaSuccess &&
            cudaMalloc(&h->v, sizeof(float) * kParams) == cudaSuccess &&
            cudaMalloc(&h->g, sizeof(float) * kSlice) == cudaSuccess &&
            cudaMalloc(&h->mask, sizeof(float) * kParams) == cudaSuccess &&
            cudaMalloc(&h->slices, sizeof(float) * kSlice * h->nsm) == cudaSuccess &&
            cudaMalloc(&h->wimg, kWBytes) == cudaSuccess &&
            cudaMalloc(&h->err, sizeof(int)) == cudaSuccess;
  if (!ok) {
    qpsdm_mlp_destroy(h);
    return QPSDM_ENOMEM;
  }
  cudaMemset(h->p, 0, sizeof(float) * kParams);
  cudaMemset(h->m, 0, sizeof(float) * kParams);
  cudaMemset(h->v, 0, sizeof(float) * kParams);
  cudaMemset(h->wimg, 0, kWBytes);
  cudaMemset(h->err, 0, sizeof(int));
  // trainable entries: input columns 0..4 of W1, output rows 0..1 of W5 and b5
  std::vector<float> mk(kParams, 1.0f);
  for (int r = 0; r < kH; ++r)
    for (int k = 5; k < kIn; ++k) mk[oW1 + r * kIn + k] = 0.0f;
  for (int r = 2; r < kOut; ++r) {
    for (int k = 0; k < kH; ++k) mk[oW5 + r * kH + k] = 0.0f;
    mk[oB5 + r] = 0.0f;
  }
  cudaMemcpy(h->mask, mk.data(), sizeof(float) * kParams, cudaMemcpyHostToDevice);
  for (int j = 0; j < 5; ++j) h->ta.in_scale[j] = 1.0f;
  h->ta.w_out[0] = h->ta.w_out[1] = 1.0f;
  if (cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmem) !=
          cudaSuccess ||
      cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           kFwdSmem) != cudaSuccess) {
    qpsdm_mlp_destroy(h);
    return QPSDM_ECUDA;
  }
  *out = h;
  return QPSDM_OK;
}

extern "C" int qpsdm_mlp_destroy(qpsdm_mlp *h) {
  if (!h) return QPSDM_OK;
  cudaFree(h->p);
  cudaFree(h->m);
  cudaFree(h->v);
  cudaFree(h->g);
  cudaFree(h->mask);
  cudaFree(h->slices);
  cudaFree(h->wimg);
  cudaFree(h->err);
  delete h;
  return QPSDM_OK;
}

extern "C" int qpsdm_mlp_param_count(void) { return kParams; }

extern "C" int qpsdm_mlp_set_params(qpsdm_mlp *h, const float *host_params) {
  if (!h || !host_params) return QPSDM_EINVAL;
  cudaSetDevice(h->device);
  std::vector<float> p(host_params, host_params + kParams), mk(kParams);
  cudaMemcpy(mk.data(), h->mask, sizeof(float) * kParams, cudaMemcpyDeviceToHost);
  for (int i = 0; i < kParams; ++i) p[i] *= mk[i];
  if (cudaMemcpy(h->p, p.data(), sizeof(float) * kParams, cudaMemcpyHostToDevice) != cudaSuccess)
    return QPSDM_ECUDA;
  cudaMemset(h->m, 0, sizeof(float) * kParams);
  cudaMemset(h->v, 0, sizeof(float) * kParams);
  h->step = 0;
  k_mlp_pack<<<64, 256>>>(h->p, h->wimg);
  return cudaDeviceSynchronize() == cudaSuccess ? QPSDM_OK : QPSDM_ECUDA;
}

extern "C" int qpsdm_mlp_get_params(qpsdm_mlp *h, float *host_params) {
  if (!h || !host_params) return QPSDM_EINVAL;
  cudaSetDevice(h->device);
  return cudaMemcpy(host_params, h->p, sizeof(float) * kParams, cudaMemcpyDeviceToHost) ==
                 cudaSuccess
             ? QPSDM_OK
             : QPSDM_ECUDA;
}

extern "C" int qpsdm_mlp_set_scaling(qpsdm_mlp *h, const float *in_shift, const float *in_scale,
                                     const float *out_weight) {
  if (!h || !in_shift || !in_scale || !out_weight) return QPSDM_EINVAL;
  for (int j = 0; j < 5; ++j) {
    h->ta.in_shift[j] = in_shift[j];
    h->ta.in_scale[j] = in_scale[j];
  }
  h->ta.w_out[0] = out_weight[0];
  h->ta.w_out[1] = out_weight[1];
  return QPSDM_OK;
}

static int mlp_check_err(qpsdm_mlp *h) {
  int e = 0;
  if (cudaMemcpy(&e, h->err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    return QPSDM_ECUDA;
  return e ? QPSDM_ETIMEOUT : QPSDM_OK;
}

extern "C" int qpsdm_mlp_gradients(qpsdm_mlp *h, const float *d_x, const float *d_t, int n,
                                   float *host_grads, float *loss, void *stream) {
  if (!h || !d_x || !d_t || n <= 0) return QPSDM_EINVAL;
  cudaSetDevice(h->device);
  cudaStream_t st = (cudaStream_t)stream;
  MlpTileArgs ta = h->ta;
  ta.inv_batch = 1.0f / n;
  const int grid = mlp_grid(h, n);
  k_mlp_grad<<<grid, kTeam, kSmem, st>>>(h->wimg, h->p, d_x, d_t, n, ta, h->slices, h->err);
  k_mlp_reduce<<<64, 256, 0, st>>>(h->slices, grid, h->g);
  if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
    return QPSDM_ECUDA;
  int rc = mlp_check_err(h);
  if (rc) return rc;
  if (host_grads)
    cudaMemcpy(host_grads, h->g, sizeof(float) * kParams, cudaMemcpyDeviceToHost);
  if (loss) cudaMemcpy(loss, h->g + kParams, sizeof(float), cudaMemcpyDeviceToHost);
  return QPSDM_OK;
}

extern "C" int qpsdm_mlp_train_step(qpsdm_mlp *h, const float *d_x, const float *d_t, int n,
                                    float lr, float *loss, void *stream) {
  if (!h || !d_x || !d_t || n <= 0 || !(lr > 0.0f)) return QPSDM_EINVAL;
  cudaSetDevice(h->device);
  cudaStream_t st = (cudaStream_t)stream;
  MlpTileArgs ta = h->ta;
  ta.inv_batch = 1.0f / n;
  const int grid = mlp_grid(h, n);
  k_mlp_grad<<<grid, kTeam, kSmem, st>>>(h->wimg, h->p, d_x, d_t, n, ta, h->slices, h->err);
  k_mlp_reduce<<<64, 256, 0, st>>>(h->slices, grid, h->g);
  h->step += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.0f / (1.0f - powf(b1, (float)h->step));
  const float c2 = 1.0f / (1.0f - powf(b2, (float)h->step));
  k_mlp_adam<<<64, 256, 0, st>>>(h->p, h->m, h->v, h->g, h->mask, lr, b1, b2, 1e-8f, c1, c2);
  k_mlp_pack<<<64, 256, 0, st>>>(h->p, h->wimg);
  if (cudaGetLastError() != cudaSuccess) return QPSDM_ECUDA;
  if (loss) {
    if (cudaMemcpyAsync(loss, h->g + kParams, sizeof(float), cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return QPSDM_ECUDA;
    return mlp_check_err(h);
  }
  return QPSDM_OK;
}

extern "C" int qpsdm_mlp_forward(qpsdm_mlp *h, const float *d_x, int n, float *d_y,
                                 void *stream) {
  if (!h || !d_x || !d_y || n <= 0) return QPSDM_EINVAL;
  cudaSetDevice(h->device);
  const int pairs = ((n + kTile - 1) / kTile + 1) / 2;
  const int grid = pairs < h->nsm ? pairs : h->nsm;
  k_mlp_forward<<<grid, 2 * kTeam, kFwdSmem, (cudaStream_t)stream>>>(h->wimg, h->p, d_x, n,
                                                                     h->ta, d_y, h->err);
  return cudaGetLastError() == cudaSuccess ? QPSDM_OK : QPSDM_ECUDA;
}

extern "C" int qpsdm_mlp_status(qpsdm_mlp *h) {
  if (!h) return QPSDM_EINVAL;
  cudaSetDevice(h->device);
  if (cudaDeviceSynchronize() != cudaSuccess) return QPSDM_ECUDA;
  return mlp_check_err(h);
}
