// common.cuh -- shared device/host helpers of the q-psdm B200 engine.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define QPSDM_HD __host__ __device__ __forceinline__

namespace qpsdm {

// ---- SU record field access (offsets: src/segy.cc:53-80) -------------------
constexpr int kSuHdr = 240;
constexpr int kOffScalco = 70;  // int16
constexpr int kOffSx = 72, kOffSy = 76, kOffGx = 80, kOffGy = 84;  // int32
constexpr int kOffNs = 114;     // uint16

__device__ __forceinline__ uint32_t bswap32(uint32_t v) { return __byte_perm(v, 0, 0x0123); }

__device__ __forceinline__ int32_t su_i32(const uint8_t *rec, int off, int be) {
  uint32_t v = (uint32_t)rec[off] | ((uint32_t)rec[off + 1] << 8) |
               ((uint32_t)rec[off + 2] << 16) | ((uint32_t)rec[off + 3] << 24);
  return (int32_t)(be ? bswap32(v) : v);
}

// Sample it of a record whose samples start at rec + 240; records are
// 4-byte aligned (240 + 4*ns bytes each).
__device__ __forceinline__ float su_sample(const uint8_t *rec, int it, int be) {
  uint32_t v = reinterpret_cast<const uint32_t *>(rec + kSuHdr)[it];
  return __uint_as_float(be ? bswap32(v) : v);
}

// ---- complex helpers -------------------------------------------------------
QPSDM_HD float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
QPSDM_HD float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
QPSDM_HD float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
QPSDM_HD float2 cconj(float2 a) { return make_float2(a.x, -a.y); }

// ---- gate output layout ----------------------------------------------------
// ints per trace: status, cdpx, cdpy, iaz, ixi1, ixi2, ntibeg, izimin
constexpr int kGateInts = 8;
constexpr int kGateF = 4;  // sx, sy, gx, gy relative to (fxi, cyi)
enum GateStatus { kRejBbox = 0, kRejY = 1, kRejCols = 2, kAccepted = 3 };

// Device-side error word bits (host reads it at fence time).
enum DevErr : unsigned {
  kErrNone = 0,
  kErrIaz = 1u << 0,     // azimuth index outside the table (clamped)
  kErrTable = 1u << 1,   // table index outside the table (masked)
  kErrNs = 1u << 2,      // record ns differs from ntl
};

}  // namespace qpsdm
