// tc_selftest.cu -- a single 128 x N x K tcgen05 tile GEMM, exported for the
// test suite (not part of the public C ABI): it checks the operand layouts,
// descriptors and TMEM read-back of tc.cuh against a reference GEMM.
#include <cuda_bf16.h>

#include "tc.cuh"
#include "qpsdm_engine.h"

namespace qpsdm {

// a: [128][K] (a_mn = 0) bf16 row-major; b: [N][K] bf16 row-major.
// a_mn / b_mn = 1 stores the operand transposed in shared memory and has the
// tensor core read it MN-major (the weight-gradient case of the MLP).
__global__ void __launch_bounds__(128) k_tc_gemm_test(const __nv_bfloat16 *__restrict__ a,
                                                      const __nv_bfloat16 *__restrict__ b,
                                                      float *__restrict__ d, int N, int K,
                                                      int a_mn, int b_mn, int *err) {
  extern __shared__ __align__(1024) uint8_t sm[];
  uint8_t *sa = sm;                       // 128 * K * 2 bytes
  uint8_t *sb = sm + 128 * K * 2;         // N * K * 2 bytes
  __shared__ uint64_t bar;
  __shared__ uint32_t tslot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t ncols = N <= 32 ? 32 : (N <= 64 ? 64 : (N <= 128 ? 128 : 256));
  if (warp == 0) tc::tmem_alloc(&tslot, ncols);
  if (tid == 0) {
    tc::mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // operands into the core-matrix layout
  for (int i = tid; i < 128 * K; i += 128) {
    const int r = i / K, k = i % K;
    const uint32_t off = a_mn ? tc::kmaj_off(k, r, 128) : tc::kmaj_off(r, k, K);
    *reinterpret_cast<__nv_bfloat16 *>(sa + off) = a[i];
  }
  for (int i = tid; i < N * K; i += 128) {
    const int r = i / K, k = i % K;
    const uint32_t off = b_mn ? tc::kmaj_off(k, r, N) : tc::kmaj_off(r, k, K);
    *reinterpret_cast<__nv_bfloat16 *>(sb + off) = b[i];
  }
  tc::fence_smem_to_async();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tslot;
  if (tid == 0) {
    // K-major: LBO 128, SBO (K/8)*128, step 256.  MN-major (stored as the
    // transpose with R = 128 or N columns): LBO = (R/8)*128, SBO 128, step 2*LBO.
    const uint32_t a_lbo = a_mn ? 16 * 128 : 128, a_sbo = a_mn ? 128 : (K / 8) * 128;
    const uint32_t a_step = a_mn ? 2 * a_lbo : 256;
    const uint32_t b_lbo = b_mn ? (N / 8) * 128 : 128, b_sbo = b_mn ? 128 : (K / 8) * 128;
    const uint32_t b_step = b_mn ? 2 * b_lbo : 256;
    tc::gemm_issue(tmem, tc::smem_u32(sa), a_lbo, a_sbo, a_step, tc::smem_u32(sb), b_lbo, b_sbo,
                   b_step, tc::idesc_bf16(128, N, a_mn, b_mn), K, false, &bar);
  }
  const bool ok = tc::mbar_wait(&bar, 0, 1u << 26);
  if (!ok && lane == 0) atomicExch(err, 1);
  tc::fence_after_sync();
  if (ok) {
    for (int c = 0; c < N; c += 16) {
      float v[16];
      tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + c, v);
      float *row = d + (size_t)(warp * 32 + lane) * N + c;
#pragma unroll
      for (int j = 0; j < 16; ++j) row[j] = v[j];
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_free(tmem, ncols);
}

// The failure path of the tensor-core kernels' bounded waits: a CTA holding
// TMEM waits on an mbarrier that nothing will arrive on (no MMA is issued, so
// nothing is in flight), gives up after limit_ns, records the timeout and
// still frees its TMEM and returns normally -- the context stays usable.
__global__ void __launch_bounds__(128) k_tc_wait_test(int *err, unsigned long long limit_ns) {
  __shared__ uint64_t bar;
  __shared__ uint32_t tslot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) tc::tmem_alloc(&tslot, 32);
  if (tid == 0) {
    tc::mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tslot;
  const bool ok = tc::mbar_wait_for(&bar, 0, 1u << 30, limit_ns);
  if (!ok && lane == 0) atomicExch(err, 1);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_free(tmem, 32);
}

}  // namespace qpsdm

// Test entry: runs k_tc_wait_test with a limit of limit_us microseconds,
// synchronises the stream and returns QPSDM_ETIMEOUT when the wait gave up.
extern "C" int qpsdm_internal_tc_wait_timeout(int limit_us, int *d_err, void *stream) {
  using namespace qpsdm;
  if (!d_err || limit_us <= 0 || limit_us > 1000000) return QPSDM_EINVAL;
  if (cudaMemsetAsync(d_err, 0, sizeof(int), (cudaStream_t)stream) != cudaSuccess)
    return QPSDM_ECUDA;
  k_tc_wait_test<<<1, 128, 0, (cudaStream_t)stream>>>(d_err, 1000ull * (unsigned)limit_us);
  if (cudaGetLastError() != cudaSuccess) return QPSDM_ECUDA;
  int h = 0;
  if (cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess ||
      cudaMemcpy(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    return QPSDM_ECUDA;
  return h ? QPSDM_ETIMEOUT : QPSDM_OK;
}

extern "C" int qpsdm_internal_tc_gemm(const void *d_a, const void *d_b, float *d_out, int N,
                                      int K, int a_mn, int b_mn, int *d_err, void *stream) {
  using namespace qpsdm;
  if (!d_a || !d_b || !d_out || !d_err) return QPSDM_EINVAL;
  if (N < 16 || N > 256 || N % 16 || K < 16 || K > 256 || K % 16) return QPSDM_EINVAL;
  const size_t smem = (size_t)(128 + N) * K * 2;
  if (smem > 200 * 1024) return QPSDM_EINVAL;
  if (cudaFuncSetAttribute(k_tc_gemm_test, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return QPSDM_ECUDA;
  k_tc_gemm_test<<<1, 128, smem, (cudaStream_t)stream>>>(
      (const __nv_bfloat16 *)d_a, (const __nv_bfloat16 *)d_b, d_out, N, K, a_mn, b_mn, d_err);
  return cudaGetLastError() == cudaSuccess ? QPSDM_OK : QPSDM_ECUDA;
}
