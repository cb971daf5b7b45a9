// fft.cuh -- batched mixed-radix FFT in shared memory (sm_100a).
//
// Replaces the reference's host PFA FFT (pfarc/pfacr, src/fft.cc:1768-1910,
// behind the fftw-style shim src/fft.cc:3721-3773).  Written from the
// mathematics, not from fft.cc: a Stockham autosort transform (Govindaraju et
// al., "High performance discrete Fourier transforms on graphics processors",
// SC 2008) with one pass per radix, so any length whose factors are in
// {2,3,4,5,7,11,13} works; every npfar() length qualifies (its half-length is
// a product of {2,4,8,16},{3,9},5,7,11,13).  Real transforms of length n use
// one complex transform of length m = n/2 plus a split step.
//
// One CTA transforms one signal held in shared memory (two ping-pong buffers
// of m complex floats plus the m twiddles).  Twiddles are tables made on the
// host in double precision and rounded once to float.
#pragma once

#include "common.cuh"

namespace qpsdm {

constexpr int kFftMaxPass = 12;

struct FftPlan {
  int n;  // real length (even)
  int m;  // complex length n/2
  int npass;
  int radix[kFftMaxPass];
  const float2 *tw_m;  // [m]    exp(-2 pi i e / m)
  const float2 *tw_n;  // [m+1]  exp(-2 pi i k / n)
};

// Shared-memory bytes one CTA needs for a plan (2 buffers + m twiddles +
// m+1 split twiddles).
QPSDM_HD size_t fft_smem_bytes(int m) { return sizeof(float2) * (size_t)(4 * m + 1); }

// One Stockham pass of radix P over m points: in -> out.
// Butterfly j (0 <= j < m/P) reads in[j + r*m/P], twiddles input r by
// W_{Ns*P}^{k*r} with k = j mod Ns, does a P-point DFT and writes
// out[(j/Ns)*Ns*P + k + r*Ns].  Ns is the product of the radices already done.
template <int P>
__device__ __forceinline__ void stockham_pass(const float2 *__restrict__ in,
                                              float2 *__restrict__ out, int m,
                                              int Ns, const float2 *twm,
                                              bool inverse) {
  const int nb = m / P;
  const int twstride = m / (Ns * P);
  const int rootstride = m / P;
  float2 w[P];
#pragma unroll
  for (int e = 0; e < P; ++e) {
    float2 t = twm[e * rootstride];
    w[e] = inverse ? cconj(t) : t;
  }
  // j / Ns as a multiply-high: magic = ceil(2^32 / Ns) is exact for
  // j, Ns < 2^16 (the error j * (magic - 2^32/Ns) / 2^32 < 2^-16 <= 1/Ns).
  const unsigned magic =
      Ns > 1 ? (unsigned)((0x100000000ull + (unsigned)Ns - 1) / (unsigned)Ns) : 0u;
  for (int j = threadIdx.x; j < nb; j += blockDim.x) {
    float2 v[P];
#pragma unroll
    for (int r = 0; r < P; ++r) v[r] = in[j + r * nb];
    const int jq = Ns > 1 ? (int)__umulhi((unsigned)j, magic) : j;
    const int k = j - jq * Ns;
    if (Ns > 1) {
      // k * r * twstride < Ns * P * (m / (Ns * P)) = m: no reduction needed
#pragma unroll
      for (int r = 1; r < P; ++r) {
        float2 t = twm[k * r * twstride];
        v[r] = cmul(v[r], inverse ? cconj(t) : t);
      }
    }
    float2 o[P];
    if (P == 2) {
      o[0] = cadd(v[0], v[1]);
      o[1] = csub(v[0], v[1]);
    } else if (P == 4) {
      float2 a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
      float2 c = cadd(v[1], v[3]), d = csub(v[1], v[3]);
      // forward: W4 = -i; d * (-i) = (d.y, -d.x)
      float2 dm = inverse ? make_float2(-d.y, d.x) : make_float2(d.y, -d.x);
      o[0] = cadd(a, c);
      o[2] = csub(a, c);
      o[1] = cadd(b, dm);
      o[3] = csub(b, dm);
    } else if (P & 1) {
      // Odd P: pair inputs r and P-r.  With s_r = v_r + v_{P-r},
      // d_r = v_r - v_{P-r}, C_k = v_0 + sum_r s_r cos(2 pi r k / P) and
      // S_k = sum_r d_r sin(2 pi r k / P), the forward outputs are
      // o_k = C_k - i S_k and o_{P-k} = C_k + i S_k (signs swap for the
      // inverse): a quarter of the real multiplies of the direct sum.
      constexpr int H = (P - 1) / 2;
      float2 s[H + 1], d[H + 1];
      float2 o0 = v[0];
#pragma unroll
      for (int r = 1; r <= H; ++r) {
        s[r] = cadd(v[r], v[P - r]);
        d[r] = csub(v[r], v[P - r]);
        o0 = cadd(o0, s[r]);
      }
      o[0] = o0;
#pragma unroll
      for (int k = 1; k <= H; ++k) {
        float2 c = v[0], sn = make_float2(0.f, 0.f);
#pragma unroll
        for (int r = 1; r <= H; ++r) {
          const float cs = w[(r * k) % P].x;    // cos(2 pi r k / P)
          const float sv = -w[(r * k) % P].y;   // sin(2 pi r k / P) (forward table)
          c.x += s[r].x * cs;
          c.y += s[r].y * cs;
          sn.x += d[r].x * sv;
          sn.y += d[r].y * sv;
        }
        // -i*S = (S.y, -S.x); the inverse table is conjugated, which flips sv
        o[k] = make_float2(c.x + sn.y, c.y - sn.x);
        o[P - k] = make_float2(c.x - sn.y, c.y + sn.x);
      }
    } else {
#pragma unroll
      for (int q = 0; q < P; ++q) {
        float2 acc = v[0];
#pragma unroll
        for (int r = 1; r < P; ++r) {
          float2 t = w[(r * q) % P];
          acc.x += v[r].x * t.x - v[r].y * t.y;
          acc.y += v[r].x * t.y + v[r].y * t.x;
        }
        o[q] = acc;
      }
    }
    const int base = jq * Ns * P + k;
#pragma unroll
    for (int r = 0; r < P; ++r) out[base + r * Ns] = o[r];
  }
}

// Full complex transform of m points held in buf[0]; buf[1] is scratch.
// Returns the buffer index (0 or 1) holding the result.  Unnormalised.
// Ends with a __syncthreads().
__device__ __forceinline__ int fft_complex_smem(float2 *buf0, float2 *buf1,
                                                const FftPlan &p,
                                                const float2 *twm,
                                                bool inverse) {
  float2 *src = buf0, *dst = buf1;
  int Ns = 1, cur = 0;
  for (int ip = 0; ip < p.npass; ++ip) {
    const int P = p.radix[ip];
    switch (P) {
      case 2: stockham_pass<2>(src, dst, p.m, Ns, twm, inverse); break;
      case 3: stockham_pass<3>(src, dst, p.m, Ns, twm, inverse); break;
      case 4: stockham_pass<4>(src, dst, p.m, Ns, twm, inverse); break;
      case 5: stockham_pass<5>(src, dst, p.m, Ns, twm, inverse); break;
      case 7: stockham_pass<7>(src, dst, p.m, Ns, twm, inverse); break;
      case 11: stockham_pass<11>(src, dst, p.m, Ns, twm, inverse); break;
      case 13: stockham_pass<13>(src, dst, p.m, Ns, twm, inverse); break;
      default: break;
    }
    __syncthreads();
    Ns *= P;
    float2 *t = src;
    src = dst;
    dst = t;
    cur ^= 1;
  }
  return cur;
}

// Split step of a real forward transform: Z = FFT_m(x[2j] + i x[2j+1]);
// X[k] = E + W_n^k O with E = (Z[k] + conj Z[m-k])/2,
// O = -i (Z[k] - conj Z[m-k])/2, for 0 <= k <= m.
__device__ __forceinline__ float2 rfft_bin(const float2 *Z, const float2 *twn,
                                           int m, int k) {
  float2 a = Z[k == m ? 0 : k];
  float2 b = cconj(Z[k == 0 ? 0 : m - k]);
  float2 e = make_float2(0.5f * (a.x + b.x), 0.5f * (a.y + b.y));
  float2 d = make_float2(0.5f * (a.x - b.x), 0.5f * (a.y - b.y));
  float2 o = make_float2(d.y, -d.x);  // -i * d
  return cadd(e, cmul(twn[k], o));
}

// Inverse of the split: from X[k] (0 <= k <= m) build Z[k] for 0 <= k < m
// such that the unnormalised inverse complex transform of Z gives
// y[2j] + i y[2j+1] = (n x[2j] + i n x[2j+1]) / 2.
__device__ __forceinline__ float2 irfft_pre(const float2 *X, const float2 *twn,
                                            int m, int k) {
  float2 a = X[k];
  float2 b = cconj(X[m - k]);
  float2 e = make_float2(0.5f * (a.x + b.x), 0.5f * (a.y + b.y));
  float2 d = make_float2(0.5f * (a.x - b.x), 0.5f * (a.y - b.y));
  float2 o = cmul(d, cconj(twn[k]));  // d / W_n^k
  return make_float2(e.x - o.y, e.y + o.x);  // e + i o
}

}  // namespace qpsdm
