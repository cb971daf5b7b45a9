// fft.cu -- FFT plans (twiddle tables per device and length) and the
// standalone batched real transforms of the C ABI.
#include <cmath>
#include <map>
#include <mutex>
#include <utility>

#include "fft.cuh"
#include "internal.h"
#include "qpsdm_engine.h"

namespace qpsdm {

static std::mutex g_plan_mu;
static std::map<std::pair<int, int>, FftPlan> g_plans;

// Radices of m: powers of two as 4s (and one 2), nines as 3s, then 5,7,11,13.
static bool factor_radices(int m, FftPlan &p) {
  p.npass = 0;
  int r = m;
  while (r % 4 == 0 && p.npass < kFftMaxPass) { p.radix[p.npass++] = 4; r /= 4; }
  if (r % 2 == 0 && p.npass < kFftMaxPass) { p.radix[p.npass++] = 2; r /= 2; }
  const int odd[5] = {3, 5, 7, 11, 13};
  for (int q : odd)
    while (r % q == 0 && p.npass < kFftMaxPass) { p.radix[p.npass++] = q; r /= q; }
  return r == 1;
}

int fft_plan(int n, FftPlan *out, std::string *err) {
  if (n < 2 || (n & 1)) {
    if (err) *err = "FFT length must be even and >= 2";
    return QPSDM_EINVAL;
  }
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_plan_mu);
  auto key = std::make_pair(dev, n);
  auto it = g_plans.find(key);
  if (it != g_plans.end()) {
    *out = it->second;
    return QPSDM_OK;
  }
  FftPlan p{};
  p.n = n;
  p.m = n / 2;
  if (!factor_radices(p.m, p)) {
    if (err) *err = "FFT length " + std::to_string(n) + " has a factor outside {2,3,5,7,11,13}";
    return QPSDM_EINVAL;
  }
  if (fft_smem_bytes(p.m) > 200 * 1024) {
    if (err) *err = "FFT length too large for one CTA";
    return QPSDM_EINVAL;
  }
  std::vector<float2> h((size_t)p.m + (size_t)p.m + 1);
  for (int e = 0; e < p.m; ++e) {
    double a = -2.0 * M_PI * (double)e / (double)p.m;
    h[e] = make_float2((float)std::cos(a), (float)std::sin(a));
  }
  for (int k = 0; k <= p.m; ++k) {
    double a = -2.0 * M_PI * (double)k / (double)n;
    h[p.m + k] = make_float2((float)std::cos(a), (float)std::sin(a));
  }
  float2 *d = nullptr;
  if (cudaMalloc(&d, sizeof(float2) * h.size()) != cudaSuccess) {
    if (err) *err = "cudaMalloc of FFT twiddles failed";
    return QPSDM_ENOMEM;
  }
  cudaMemcpy(d, h.data(), sizeof(float2) * h.size(), cudaMemcpyHostToDevice);
  p.tw_m = d;
  p.tw_n = d + p.m;
  g_plans[key] = p;
  *out = p;
  return QPSDM_OK;
}

// Stage both twiddle tables into shared memory after the two work buffers.
__device__ __forceinline__ void stage_twiddles(const FftPlan &p, float2 *s_twm,
                                               float2 *s_twn) {
  for (int i = threadIdx.x; i < p.m; i += blockDim.x) s_twm[i] = p.tw_m[i];
  for (int i = threadIdx.x; i <= p.m; i += blockDim.x) s_twn[i] = p.tw_n[i];
}

__global__ void __launch_bounds__(256) k_rfft_batch(const float *__restrict__ in,
                                                    float2 *__restrict__ out,
                                                    FftPlan p) {
  extern __shared__ float2 sm[];
  float2 *b0 = sm, *b1 = sm + p.m, *twm = sm + 2 * p.m, *twn = sm + 3 * p.m;
  const float *x = in + (size_t)blockIdx.x * p.n;
  stage_twiddles(p, twm, twn);
  for (int j = threadIdx.x; j < p.m; j += blockDim.x)
    b0[j] = make_float2(x[2 * j], x[2 * j + 1]);
  __syncthreads();
  int cur = fft_complex_smem(b0, b1, p, twm, false);
  const float2 *Z = cur ? b1 : b0;
  float2 *y = out + (size_t)blockIdx.x * (p.m + 1);
  for (int k = threadIdx.x; k <= p.m; k += blockDim.x) y[k] = rfft_bin(Z, twn, p.m, k);
}

__global__ void __launch_bounds__(256) k_irfft_batch(const float2 *__restrict__ in,
                                                     float *__restrict__ out,
                                                     FftPlan p) {
  extern __shared__ float2 sm[];
  float2 *b0 = sm, *b1 = sm + p.m, *twm = sm + 2 * p.m, *twn = sm + 3 * p.m;
  const float2 *X = in + (size_t)blockIdx.x * (p.m + 1);
  stage_twiddles(p, twm, twn);
  __syncthreads();
  for (int k = threadIdx.x; k < p.m; k += blockDim.x) b0[k] = irfft_pre(X, twn, p.m, k);
  __syncthreads();
  int cur = fft_complex_smem(b0, b1, p, twm, true);
  const float2 *z = cur ? b1 : b0;
  float *y = out + (size_t)blockIdx.x * p.n;
  for (int j = threadIdx.x; j < p.m; j += blockDim.x) {
    y[2 * j] = 2.0f * z[j].x;
    y[2 * j + 1] = 2.0f * z[j].y;
  }
}

int fft_set_smem_attr(const void *kernel, size_t bytes) {
  if (bytes > 48 * 1024)
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)bytes) == cudaSuccess
               ? QPSDM_OK
               : QPSDM_ECUDA;
  return QPSDM_OK;
}

}  // namespace qpsdm

using namespace qpsdm;

extern "C" int qpsdm_fft_r2c(const float *d_in, int n, int batch, float *d_out,
                             void *stream) {
  if (!d_in || !d_out || batch < 0) return QPSDM_EINVAL;
  if (batch == 0) return QPSDM_OK;
  FftPlan p;
  int rc = fft_plan(n, &p, nullptr);
  if (rc) return rc;
  size_t sm = fft_smem_bytes(p.m);
  if ((rc = fft_set_smem_attr((const void *)k_rfft_batch, sm))) return rc;
  k_rfft_batch<<<batch, 256, sm, (cudaStream_t)stream>>>(d_in, (float2 *)d_out, p);
  return cudaGetLastError() == cudaSuccess ? QPSDM_OK : QPSDM_ECUDA;
}

extern "C" int qpsdm_fft_c2r(const float *d_in, int n, int batch, float *d_out,
                             void *stream) {
  if (!d_in || !d_out || batch < 0) return QPSDM_EINVAL;
  if (batch == 0) return QPSDM_OK;
  FftPlan p;
  int rc = fft_plan(n, &p, nullptr);
  if (rc) return rc;
  size_t sm = fft_smem_bytes(p.m);
  if ((rc = fft_set_smem_attr((const void *)k_irfft_batch, sm))) return rc;
  k_irfft_batch<<<batch, 256, sm, (cudaStream_t)stream>>>((const float2 *)d_in, d_out, p);
  return cudaGetLastError() == cudaSuccess ? QPSDM_OK : QPSDM_ECUDA;
}

// ---------------------------------------------------------------------------
// Allocation-free batched real FFT.
//
// Some callers of this library must not allocate device memory: a host
// framework that owns every byte of HBM through its own pool and forbids
// cudaMalloc behind its back, or a latency-critical caller that cannot take
// the implicit device synchronisation a cudaMalloc may cause.  qpsdm_fft_r2c
// allocates its twiddle tables on the first use of each length; this variant
// keeps them in one fixed file-scope device array instead, which every GPU
// that loads the library holds until the process exits.
//
// The array is shared by every call on a device and keeps the last call's
// twiddles; each call first rewrites the part it uses with a small kernel on
// its own stream (cos and sin of the angles in double precision, rounded once
// to float), so nothing needs clearing and no host buffer is involved.  Calls
// that overlap on the GPU (concurrent streams) race on the array and must be
// serialised by the caller.  The first call on a device looks up the array's
// device address (cudaGetSymbolAddress); make that first call before any
// stream capture.
// ---------------------------------------------------------------------------
namespace qpsdm {

constexpr int kNoAllocMaxDevices = 64;
// m twiddles + (m + 1) split twiddles, m = n / 2 <= QPSDM_FFT_NOALLOC_MAX_N / 2
static __device__ __align__(256) float2 g_noalloc_twiddles[QPSDM_FFT_NOALLOC_MAX_N + 1];
static std::mutex g_noalloc_mu;
static float2 *g_noalloc_dev_ptr[kNoAllocMaxDevices];

// Device address of g_noalloc_twiddles on the current device; set up once per
// device with that device current.  In host code the array's name is only a
// host-side stand-in, never a usable device address.
static int noalloc_twiddle_ptr(float2 **out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices)
    return QPSDM_ECUDA;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_dev_ptr[dev]) {
    void *ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_noalloc_twiddles) != cudaSuccess || !ptr)
      return QPSDM_ECUDA;
    g_noalloc_dev_ptr[dev] = (float2 *)ptr;
  }
  *out = g_noalloc_dev_ptr[dev];
  return QPSDM_OK;
}

// Twiddles of length n = 2m into tw: exp(-2 pi i e / m) for e < m, then
// exp(-2 pi i k / n) for k <= m (the layout of FftPlan's tw_m, tw_n).
__global__ void k_noalloc_twiddles(float2 *__restrict__ tw, int m) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 2 * m + 1) return;
  const double turns = i < m ? -2.0 * (double)i / (double)m : -(double)(i - m) / (double)m;
  double sn, cs;
  sincospi(turns, &sn, &cs);
  tw[i] = make_float2((float)cs, (float)sn);
}

}  // namespace qpsdm

extern "C" int qpsdm_fft_r2c_noalloc(const float *d_in, int n, int batch,
                                     float *d_out, void *stream) {
  if (!d_in || !d_out || batch < 0) return QPSDM_EINVAL;
  if (n > QPSDM_FFT_NOALLOC_MAX_N) return QPSDM_ESIZE;
  if (n < 2 || (n & 1)) return QPSDM_EINVAL;
  if (batch == 0) return QPSDM_OK;
  FftPlan p{};
  p.n = n;
  p.m = n / 2;
  if (!factor_radices(p.m, p)) return QPSDM_EINVAL;
  float2 *tw = nullptr;
  int rc = noalloc_twiddle_ptr(&tw);
  if (rc) return rc;
  // this length's twiddles into the shared array, on the caller's stream
  const int ntw = 2 * p.m + 1;
  k_noalloc_twiddles<<<(ntw + 255) / 256, 256, 0, (cudaStream_t)stream>>>(tw, p.m);
  p.tw_m = tw;
  p.tw_n = tw + p.m;
  const size_t sm = fft_smem_bytes(p.m);
  if ((rc = fft_set_smem_attr((const void *)k_rfft_batch, sm))) return rc;
  k_rfft_batch<<<batch, 256, sm, (cudaStream_t)stream>>>(d_in, (float2 *)d_out, p);
  return cudaGetLastError() == cudaSuccess ? QPSDM_OK : QPSDM_ECUDA;
}
