// tc.cuh -- tcgen05 (5th-generation tensor core) building blocks for sm_100a.
//
// A 128 x N tile GEMM with BF16 operands in shared memory and the FP32
// accumulator in tensor memory (TMEM):
//   D[128][N] (+)= A[128][K] * B[N][K]^T      (A, B K-major or MN-major)
// issued by one thread as K/16 tcgen05.mma instructions, completed through
// tcgen05.commit on an mbarrier, read back by the four warps of a warpgroup
// with tcgen05.ld (warp w owns TMEM lanes 32w..32w+31 = rows of D).
//
// Shared-memory operand layout ("core matrices", no swizzle): a K-major
// matrix [R][K] of 16-bit elements is stored as 8 x 8 blocks of 128 bytes,
// row r of a block at 16 r bytes:
//   offset(r, k) = (r / 8) * SBO + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2,
//   SBO = (K / 8) * 128.
// Read K-major its descriptor has LBO = 128 (next 8-element K chunk) and
// SBO; the same bytes read MN-major (the transpose, [K][R]) have LBO = SBO
// and SBO = 128.  Every wait is bounded: on timeout the kernel records an
// error code and carries on, it never spins forever.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

namespace qpsdm {
namespace tc {

// --- encodings -------------------------------------------------------------
// Shared-memory matrix descriptor: start address, leading and stride byte
// offsets (all >> 4), descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: BF16 x BF16 -> F32, M x N, majors
// (0 = K-major, 1 = MN-major).
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, int a_mn, int b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// byte offset of element (r, k) of a K-major core-matrix operand with K columns
__device__ __forceinline__ uint32_t kmaj_off(int r, int k, int K) {
  return (uint32_t)((r >> 3) * (K >> 3) * 128 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// --- TMEM --------------------------------------------------------------------
// One full warp allocates / frees; the address lands in *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(slot)),
               "r"(ncols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}
__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// generic-proxy shared-memory writes become visible to the tensor core
__device__ __forceinline__ void fence_smem_to_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// --- mbarrier ----------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait for phase `parity` to complete: gives up after max_iter polls
// or limit_ns of wall time, whichever comes first; returns false on timeout.
__device__ __forceinline__ bool mbar_wait_for(uint64_t *bar, uint32_t parity, uint32_t max_iter,
                                              uint64_t limit_ns) {
  const uint32_t a = smem_u32(bar);
  const uint64_t t0 = globaltimer_ns();
  for (uint32_t i = 0; i < max_iter; ++i) {
    if ((i & 1023u) == 1023u && globaltimer_ns() - t0 > limit_ns) return false;
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
// the kernels' waits: 2 s
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t max_iter) {
  return mbar_wait_for(bar, parity, max_iter, 2000000000ull);
}

// --- MMA ---------------------------------------------------------------------
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}
// arrive on *bar once every MMA this thread issued before has completed
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// 16 consecutive FP32 columns, without waiting: several loads can be in
// flight before the wait.
__device__ __forceinline__ void tmem_ld16_nowait(uint32_t taddr, uint32_t *r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
// The wait, with 16 loaded registers as its operands so that no use of them
// can be scheduled before it (call once per group of 16; after the first the
// wait returns at once).
__device__ __forceinline__ void tmem_wait_ld_dep16(uint32_t *r) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]),
                 "+r"(r[6]), "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]),
                 "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15])
               :
               : "memory");
}

// D (TMEM, 128 lanes x N columns at d_tmem) (+)= A * B^T over K (multiple of
// 16).  A: 128 x K; B: N x K.  a_desc0/b_desc0 describe the first K = 16
// step; each further step advances the start addresses by a_step/b_step
// bytes.  Issued by the calling thread only; commits to *bar.
__device__ __forceinline__ void gemm_issue(uint32_t d_tmem, uint32_t a_saddr, uint32_t a_lbo,
                                           uint32_t a_sbo, uint32_t a_step, uint32_t b_saddr,
                                           uint32_t b_lbo, uint32_t b_sbo, uint32_t b_step,
                                           uint32_t idesc, int K, bool accumulate,
                                           uint64_t *bar) {
  for (int s = 0; s < K / 16; ++s) {
    const uint64_t ad = smem_desc(a_saddr + s * a_step, a_lbo, a_sbo);
    const uint64_t bd = smem_desc(b_saddr + s * b_step, b_lbo, b_sbo);
    mma_bf16(d_tmem, ad, bd, idesc, (accumulate || s > 0) ? 1u : 0u);
  }
  mma_commit(bar);
}

}  // namespace tc
}  // namespace qpsdm
