// mlp.cu -- the learned traveltime / t* surrogate on 5th-generation tensor cores.
//
// Network: 5 inputs (padded to 16) -> 4 x 128 (SiLU) -> 2 outputs (padded to
// 16).  BF16 weights and activations, FP32 accumulation in tensor memory,
// FP32 master weights and Adam moments in global memory.
//
// One persistent CTA of 128 threads (a warpgroup) per SM walks 128-sample
// tiles.  Every layer is one tcgen05 tile GEMM (tc.cuh): activations are the
// A operand ([sample][feature], K-major), weights [out][in] the B operand.
// Backward re-computes what it needs (all activations do not fit in shared
// memory next to the weights) and forms
//   dW_l = dZ_l^T H_{l-1}   (A = dZ MN-major view, B = H MN-major view)
//   dH_{l-1} = dZ_l W_l      (A = dZ K-major, B = W MN-major view)
// Each CTA accumulates gradients into its own slice of a global buffer
// (plain read-modify-write, no atomics); a reduction over the slices in a
// fixed order and an Adam step follow, so training is deterministic.
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
// shared memory map
constexpr int sX = kWBytes;                   // [128][16] bf16
constexpr int sH0 = sX + kTile * kIn * 2;     // [128][128] bf16
constexpr int sH1 = sH0 + kTile * kH * 2;
constexpr int sG = sH1 + kTile * kH * 2;      // dZ, [128][128] or [128][16]
constexpr int sBias = sG + kTile * kH * 2;    // fp32 biases (4*128 + 16)
constexpr int sDb = sBias + (4 * kH + kOut) * 4;  // fp32 bias-gradient partials [4 warps][128]
constexpr int sLoss = sDb + 4 * kH * 4;       // fp32 loss partials [4 warps]
constexpr int kSmem = sLoss + 16;             // 214,096 bytes

struct MlpTileArgs {
  float in_scale[5], in_shift[5];  // features = (raw - shift) * scale
  float w_out[2];                  // loss weights of the two outputs
  float inv_batch;
};

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float silu_grad(float z) {
  const float s = 1.0f / (1.0f + __expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

// 8 bf16 of row r, columns c..c+7 of a K-major core-matrix buffer (rowlen K).
__device__ __forceinline__ void st_row8(uint8_t *buf, int r, int c, int K, const float *v) {
  __nv_bfloat162 p[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) p[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
  *reinterpret_cast<uint4 *>(buf + tc::kmaj_off(r, c, K)) = *reinterpret_cast<uint4 *>(p);
}

struct Gemm {
  uint64_t *bar;
  uint32_t phase;
  int *err;
  // D (TMEM) = A * B^T.  a/b: core-matrix buffers with storage row length
  // a_len/b_len; *_mn = 1 reads the buffer transposed (MN-major).  K: the
  // reduction length.  All threads call; thread 0 issues.
  __device__ bool run(uint32_t d, const uint8_t *a, int a_len, int a_mn, const uint8_t *b,
                      int b_len, int b_mn, int N, int K) {
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (threadIdx.x == 0) {
      const uint32_t a_lbo = a_mn ? (a_len / 8) * 128 : 128, a_sbo = a_mn ? 128 : (a_len / 8) * 128;
      const uint32_t b_lbo = b_mn ? (b_len / 8) * 128 : 128, b_sbo = b_mn ? 128 : (b_len / 8) * 128;
      tc::gemm_issue(d, tc::smem_u32(a), a_lbo, a_sbo, a_mn ? 2 * a_lbo : 256, tc::smem_u32(b),
                     b_lbo, b_sbo, b_mn ? 2 * b_lbo : 256, tc::idesc_bf16(128, N, a_mn, b_mn), K,
                     false, bar);
    }
    const bool timed_out = !tc::mbar_wait(bar, phase, 1u << 30);
    phase ^= 1u;
    // one decision for the whole CTA, so that every thread leaves together
    const bool ok = !__syncthreads_or(timed_out);
    if (!ok && threadIdx.x == 0) atomicExch(err, 1);
    tc::fence_after_sync();
    return ok;
  }
};

// Row r of the accumulator, 16 columns at col.
__device__ __forceinline__ void acc_row16(uint32_t acc, int col, float *v) {
  const int warp = threadIdx.x >> 5;
  tc::tmem_ld16(acc + ((uint32_t)(warp * 32) << 16) + col, v);
}

// Z = A W^T (acc) then H = SiLU(Z + b) into hout ([128][128] bf16).
__device__ __forceinline__ bool layer_fwd(Gemm &g, uint32_t acc, const uint8_t *a, int a_len,
                                          const uint8_t *w, const float *bias, uint8_t *hout) {
  if (!g.run(acc, a, a_len, 0, w, a_len, 0, kH, a_len)) return false;
  const int r = threadIdx.x;
  for (int c = 0; c < kH; c += 16) {
    float v[16];
    acc_row16(acc, c, v);
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = silu(v[j] + bias[c + j]);
    st_row8(hout, r, c, kH, v);
    st_row8(hout, r, c + 8, kH, v + 8);
  }
  return true;
}

// Forward of one tile from sX: H1..H4 alternate in sH0/sH1 (H4 in sH1),
// outputs y[2] of this thread's sample.
__device__ __forceinline__ bool forward(Gemm &g, uint32_t acc0, uint32_t acc1, uint8_t *sm,
                                        float y[2]) {
  const float *bias = reinterpret_cast<const float *>(sm + sBias);
  if (!layer_fwd(g, acc0, sm + sX, kIn, sm + sW1, bias + 0 * kH, sm + sH0)) return false;
  if (!layer_fwd(g, acc0, sm + sH0, kH, sm + sW2, bias + 1 * kH, sm + sH1)) return false;
  if (!layer_fwd(g, acc0, sm + sH1, kH, sm + sW3, bias + 2 * kH, sm + sH0)) return false;
  if (!layer_fwd(g, acc0, sm + sH0, kH, sm + sW4, bias + 3 * kH, sm + sH1)) return false;
  if (!g.run(acc1, sm + sH1, kH, 0, sm + sW5, kH, 0, kOut, kH)) return false;
  float v[16];
  acc_row16(acc1, 0, v);
  y[0] = v[0] + bias[4 * kH + 0];
  y[1] = v[1] + bias[4 * kH + 1];
  return true;
}

// Copy weights (bf16 images) and biases into shared memory.
__device__ __forceinline__ void load_weights(uint8_t *sm, const uint8_t *__restrict__ wimg,
                                             const float *__restrict__ params) {
  const uint4 *src = reinterpret_cast<const uint4 *>(wimg);
  uint4 *dst = reinterpret_cast<uint4 *>(sm);
  for (int i = threadIdx.x; i < kWBytes / 16; i += blockDim.x) dst[i] = src[i];
  float *bias = reinterpret_cast<float *>(sm + sBias);
  for (int i = threadIdx.x; i < kH; i += blockDim.x) {
    bias[i] = params[oB1 + i];
    bias[kH + i] = params[oB2 + i];
    bias[2 * kH + i] = params[oB3 + i];
    bias[3 * kH + i] = params[oB4 + i];
  }
  if (threadIdx.x < kOut) bias[4 * kH + threadIdx.x] = params[oB5 + threadIdx.x];
}

// Normalised features of sample r into the X tile (zero padding to 16).
__device__ __forceinline__ void put_x(uint8_t *sm, int r, const float *raw,
                                      const MlpTileArgs &ta, bool live) {
  float v[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = 0.0f;
  if (live)
#pragma unroll
    for (int j = 0; j < 5; ++j) v[j] = (raw[j] - ta.in_shift[j]) * ta.in_scale[j];
  st_row8(sm + sX, r, 0, kIn, v);
  st_row8(sm + sX, r, 8, kIn, v + 8);
}

// dZ = dH (acc1) * SiLU'(Z + b) (Z in acc0) into sG; bias-gradient partials
// of this warp's 32 samples into its own row of sDb (no atomics: the order
// of every sum is fixed).
__device__ __forceinline__ void dz_epilogue(uint32_t acc0, uint32_t acc1, const float *bias,
                                            uint8_t *sm, bool live) {
  const int r = threadIdx.x, lane = r & 31;
  float *db = reinterpret_cast<float *>(sm + sDb) + (r >> 5) * kH;
  for (int c = 0; c < kH; c += 16) {
    float z[16], d[16];
    acc_row16(acc0, c, z);
    acc_row16(acc1, c, d);
#pragma unroll
    for (int j = 0; j < 16; ++j) d[j] = live ? d[j] * silu_grad(z[j] + bias[c + j]) : 0.0f;
    st_row8(sm + sG, r, c, kH, d);
    st_row8(sm + sG, r, c + 8, kH, d + 8);
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      float s = d[j];
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (lane == 0) db[c + j] = s;
    }
  }
}

// this CTA's gradient slice: add a [rows][cols] accumulator tile (row = TMEM
// lane).  transpose: the accumulator holds W^T (rows = in, cols = out).
__device__ __forceinline__ void add_grad(uint32_t acc, int ncols, float *gs, int off,
                                         int row_len, bool transpose) {
  const int r = threadIdx.x;
  for (int c = 0; c < ncols; c += 16) {
    float v[16];
    acc_row16(acc, c, v);
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      float *p = transpose ? gs + off + (c + j) * row_len + r : gs + off + r * row_len + c + j;
      *p += v[j];
    }
  }
}

// add the four warps' bias partials (in warp order) to the gradient slice
__device__ __forceinline__ void flush_db(uint8_t *sm, float *gs, int off, int n) {
  __syncthreads();
  const float *db = reinterpret_cast<const float *>(sm + sDb);
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    gs[off + i] += ((db[i] + db[kH + i]) + db[2 * kH + i]) + db[3 * kH + i];
  __syncthreads();
}

// ---------------------------------------------------------------------------
// training: gradients of the weighted MSE over nsamp samples
// x: [n][5], t: [n][2]; grads: [gridDim.x][kSlice] (slice zeroed here)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128, 1)
    k_mlp_grad(const uint8_t *__restrict__ wimg, const float *__restrict__ params,
               const float *__restrict__ x, const float *__restrict__ t, int nsamp,
               MlpTileArgs ta, float *__restrict__ grads, int *err) {
  extern __shared__ __align__(1024) uint8_t sm[];
  __shared__ uint64_t bar;
  __shared__ uint32_t tslot;
  const int tid = threadIdx.x, warp = tid >> 5;
  float *gs = grads + (size_t)blockIdx.x * kSlice;
  for (int i = tid; i < kSlice; i += blockDim.x) gs[i] = 0.0f;
  if (warp == 0) tc::tmem_alloc(&tslot, 256);
  if (tid == 0) {
    tc::mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  load_weights(sm, wimg, params);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t acc0 = tslot, acc1 = tslot + 128;
  Gemm g{&bar, 0u, err};
  const float *bias = reinterpret_cast<const float *>(sm + sBias);
  float loss = 0.0f;
  const int ntiles = (nsamp + kTile - 1) / kTile;
  bool ok = true;
  for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const int s = tile * kTile + tid;
    const bool live = s < nsamp;
    float raw[5] = {0, 0, 0, 0, 0};
    if (live)
      for (int j = 0; j < 5; ++j) raw[j] = x[(size_t)s * 5 + j];
    put_x(sm, tid, raw, ta, live);
    const float tg0 = live ? t[(size_t)s * 2] : 0.0f, tg1 = live ? t[(size_t)s * 2 + 1] : 0.0f;
    float y[2];
    if (!(ok = forward(g, acc0, acc1, sm, y))) break;
    // loss and dZ5 = dY (2 live columns of a [128][16] tile in sG)
    float d5[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) d5[j] = 0.0f;
    if (live) {
      const float e0 = y[0] - tg0, e1 = y[1] - tg1;
      loss += ta.w_out[0] * e0 * e0 + ta.w_out[1] * e1 * e1;
      d5[0] = 2.0f * ta.w_out[0] * e0 * ta.inv_batch;
      d5[1] = 2.0f * ta.w_out[1] * e1 * ta.inv_batch;
    }
    st_row8(sm + sG, tid, 0, kOut, d5);
    st_row8(sm + sG, tid, 8, kOut, d5 + 8);
    {  // db5 partials of this warp (columns 0 and 1; the rest stay zero)
      float *db = reinterpret_cast<float *>(sm + sDb) + warp * kH;
      for (int j = 0; j < kOut; ++j) {
        float v = d5[j];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((tid & 31) == 0) db[j] = v;
      }
    }
    flush_db(sm, gs, oB5, kOut);
    // layer 5: dW5^T = H4^T dZ5 (rows = in), dH4 = dZ5 W5
    if (!(ok = g.run(acc0, sm + sH1, kH, 1, sm + sG, kOut, 1, kOut, kTile))) break;
    add_grad(acc0, kOut, gs, oW5, kH, true);
    if (!(ok = g.run(acc1, sm + sG, kOut, 0, sm + sW5, kH, 1, kH, kOut))) break;
    // layer 4: Z4 = H3 W4^T (H3 still in sH0)
    if (!(ok = g.run(acc0, sm + sH0, kH, 0, sm + sW4, kH, 0, kH, kH))) break;
    dz_epilogue(acc0, acc1, bias + 3 * kH, sm, live);
    flush_db(sm, gs, oB4, kH);
    if (!(ok = g.run(acc0, sm + sG, kH, 1, sm + sH0, kH, 1, kH, kTile))) break;
    add_grad(acc0, kH, gs, oW4, kH, false);
    if (!(ok = g.run(acc1, sm + sG, kH, 0, sm + sW4, kH, 1, kH, kH))) break;
    // layer 3: recompute H1 (sH1), H2 (sH0), Z3
    if (!(ok = layer_fwd(g, acc0, sm + sX, kIn, sm + sW1, bias, sm + sH1))) break;
    if (!(ok = layer_fwd(g, acc0, sm + sH1, kH, sm + sW2, bias + kH, sm + sH0))) break;
    if (!(ok = g.run(acc0, sm + sH0, kH, 0, sm + sW3, kH, 0, kH, kH))) break;
    dz_epilogue(acc0, acc1, bias + 2 * kH, sm, live);
    flush_db(sm, gs, oB3, kH);
    if (!(ok = g.run(acc0, sm + sG, kH, 1, sm + sH0, kH, 1, kH, kTile))) break;
    add_grad(acc0, kH, gs, oW3, kH, false);
    if (!(ok = g.run(acc1, sm + sG, kH, 0, sm + sW3, kH, 1, kH, kH))) break;
    // layer 2: H1 in sH1, recompute Z2
    if (!(ok = g.run(acc0, sm + sH1, kH, 0, sm + sW2, kH, 0, kH, kH))) break;
    dz_epilogue(acc0, acc1, bias + kH, sm, live);
    flush_db(sm, gs, oB2, kH);
    if (!(ok = g.run(acc0, sm + sG, kH, 1, sm + sH1, kH, 1, kH, kTile))) break;
    add_grad(acc0, kH, gs, oW2, kH, false);
    if (!(ok = g.run(acc1, sm + sG, kH, 0, sm + sW2, kH, 1, kH, kH))) break;
    // layer 1: recompute Z1 from X
    if (!(ok = g.run(acc0, sm + sX, kIn, 0, sm + sW1, kIn, 0, kH, kIn))) break;
    dz_epilogue(acc0, acc1, bias, sm, live);
    flush_db(sm, gs, oB1, kH);
    if (!(ok = g.run(acc0, sm + sG, kH, 1, sm + sX, kIn, 1, kIn, kTile))) break;
    add_grad(acc0, kIn, gs, oW1, kIn, false);
  }
  // loss sum of this CTA, in warp order
  for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
  float *ls = reinterpret_cast<float *>(sm + sLoss);
  if ((tid & 31) == 0) ls[warp] = loss;
  __syncthreads();
  if (tid == 0) gs[kParams] = (((ls[0] + ls[1]) + ls[2]) + ls[3]) * ta.inv_batch;
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_free(tslot, 256);
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

// ---------------------------------------------------------------------------
// inference: y[n][2] from x[n][5]
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128, 1)
    k_mlp_forward(const uint8_t *__restrict__ wimg, const float *__restrict__ params,
                  const float *__restrict__ x, int nsamp, MlpTileArgs ta, float *__restrict__ y,
                  int *err) {
  extern __shared__ __align__(1024) uint8_t sm[];
  __shared__ uint64_t bar;
  __shared__ uint32_t tslot;
  const int tid = threadIdx.x, warp = tid >> 5;
  if (warp == 0) tc::tmem_alloc(&tslot, 256);
  if (tid == 0) {
    tc::mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  load_weights(sm, wimg, params);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t acc0 = tslot, acc1 = tslot + 128;
  Gemm g{&bar, 0u, err};
  const int ntiles = (nsamp + kTile - 1) / kTile;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int s = tile * kTile + tid;
    const bool live = s < nsamp;
    float raw[5] = {0, 0, 0, 0, 0};
    if (live)
      for (int j = 0; j < 5; ++j) raw[j] = x[(size_t)s * 5 + j];
    put_x(sm, tid, raw, ta, live);
    float out[2];
    if (!forward(g, acc0, acc1, sm, out)) break;
    if (live) {
      y[(size_t)s * 2] = out[0];
      y[(size_t)s * 2 + 1] = out[1];
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_free(tslot, 256);
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
      cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmem) !=
          cudaSuccess) {
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
  k_mlp_grad<<<grid, 128, kSmem, st>>>(h->wimg, h->p, d_x, d_t, n, ta, h->slices, h->err);
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
  k_mlp_grad<<<grid, 128, kSmem, st>>>(h->wimg, h->p, d_x, d_t, n, ta, h->slices, h->err);
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
  k_mlp_forward<<<mlp_grid(h, n), 128, kSmem, (cudaStream_t)stream>>>(h->wimg, h->p, d_x, n,
                                                                      h->ta, d_y, h->err);
  return cudaGetLastError() == cudaSuccess ? QPSDM_OK : QPSDM_ECUDA;
}

extern "C" int qpsdm_mlp_status(qpsdm_mlp *h) {
  if (!h) return QPSDM_EINVAL;
  cudaSetDevice(h->device);
  if (cudaDeviceSynchronize() != cudaSuccess) return QPSDM_ECUDA;
  return mlp_check_err(h);
}
