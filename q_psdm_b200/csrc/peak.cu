// peak.cu -- the FP32 FMA rate of the device, measured by a kernel of
// independent fused multiply-add chains (test and benchmark entry, not part
// of the public C ABI).  The imaging kernels are FP32-issue-bound gathers,
// so this is the ceiling their roofline is read against, beside cuBLAS SGEMM.
#include <cuda_runtime.h>

#include "qpsdm_engine.h"

namespace qpsdm {

// Every thread runs kChains independent chains x <- x * b + c for `iters`
// rounds (2 flop per FMA), so the FMA pipe never waits on a result: the
// chains hide the FMA latency and every issue slot can take an FMA.  b and c
// are kernel arguments, so the compiler cannot fold the chains; the sums are
// stored so that they are not removed.
constexpr int kChains = 16;

__global__ void __launch_bounds__(512, 4) k_fma_rate(float b, float c, int iters,
                                                  float *__restrict__ out) {
  float x[kChains];
#pragma unroll
  for (int i = 0; i < kChains; ++i) x[i] = (float)(threadIdx.x + i);
  for (int k = 0; k < iters; ++k) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
#pragma unroll
      for (int i = 0; i < kChains; ++i) x[i] = fmaf(x[i], b, c);
    }
  }
  float s = 0.0f;
#pragma unroll
  for (int i = 0; i < kChains; ++i) s += x[i];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace qpsdm

// Launches k_fma_rate on `stream` over `blocks` blocks of 512 threads with
// `iters` rounds; *flop receives the FP32 operations the launch performs
// (multiply and add of each FMA counted).  d_out holds blocks * 512 floats.
// The caller times the launch (CUDA events on the same stream).
extern "C" int qpsdm_internal_fma_rate(int blocks, int iters, float *d_out, double *flop,
                                       void *stream) {
  using namespace qpsdm;
  if (!d_out || !flop || blocks <= 0 || iters <= 0) return QPSDM_EINVAL;
  k_fma_rate<<<blocks, 512, 0, (cudaStream_t)stream>>>(1.0000001f, 1e-7f, iters, d_out);
  if (cudaGetLastError() != cudaSuccess) return QPSDM_ECUDA;
  *flop = 2.0 * kChains * 8 * (double)iters * blocks * 512;
  return QPSDM_OK;
}
