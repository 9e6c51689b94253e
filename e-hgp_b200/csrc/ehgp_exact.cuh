// Exact arithmetic for the geometric stages (sm_100a device code).
//
// Representation: every canonical coordinate x of a cloud is an exact integer
// X = x * 2^S at one per-cloud scale S (the largest number of fractional bits
// over all coordinates), provided |X| < 2^124 for every coordinate; a cloud
// outside that range makes the exact stages return EHGP_ERR_NUMERIC_RANGE.
// Squared distances are then exact integers D = sum (Xa - Xb)^2 < 2^252 at
// scale 2^(2S), so comparisons of any two squared distances of the cloud are
// integer comparisons.
//
// Every predicate is first evaluated in FP64 with a rigorous relative error
// band; only candidates inside the band are decided with the multi-limb
// integers below (the reference's cascade fp64 filter -> exact,
// include/morsehgp3d/exact/fp64_interval.hpp, expansion.hpp, integer.hpp).
#pragma once

#include <stdint.h>

namespace ehgp {

// Relative error band of an FP64 squared distance fl(fl(dx^2)+fl(dy^2)+fl(dz^2))
// with dx = fl(xa - xb): each term carries at most 3 roundings and the sum 2
// more, so |fl(d) - d| <= 6u d + O(u^2) with u = 2^-53; 16u leaves room for
// the second-order terms and for comparing two such values.
constexpr double kDistRelErr = 16.0 * 1.1102230246251565e-16;

// ---- fixed-width two's-complement integers ------------------------------------
template <int N>
struct WInt {
  uint64_t w[N];

  __host__ __device__ static WInt zero() {
    WInt r;
    for (int i = 0; i < N; ++i) r.w[i] = 0;
    return r;
  }
  __host__ __device__ static WInt from_i128(__int128 v) {
    WInt r;
    r.w[0] = (uint64_t)v;
    r.w[1] = (uint64_t)((unsigned __int128)v >> 64);
    const uint64_t ext = v < 0 ? ~uint64_t{0} : 0;
    for (int i = 2; i < N; ++i) r.w[i] = ext;
    return r;
  }
  __host__ __device__ bool negative() const { return (w[N - 1] >> 63) != 0; }
  __host__ __device__ bool is_zero() const {
    for (int i = 0; i < N; ++i)
      if (w[i]) return false;
    return true;
  }
  __host__ __device__ int sign() const { return negative() ? -1 : (is_zero() ? 0 : 1); }
};

template <int N>
__host__ __device__ inline WInt<N> wadd(const WInt<N>& a, const WInt<N>& b) {
  WInt<N> r;
  unsigned __int128 c = 0;
  for (int i = 0; i < N; ++i) {
    c += (unsigned __int128)a.w[i] + b.w[i];
    r.w[i] = (uint64_t)c;
    c >>= 64;
  }
  return r;
}

template <int N>
__host__ __device__ inline WInt<N> wneg(const WInt<N>& a) {
  WInt<N> r;
  unsigned __int128 c = 1;
  for (int i = 0; i < N; ++i) {
    c += (unsigned __int128)(~a.w[i]);
    r.w[i] = (uint64_t)c;
    c >>= 64;
  }
  return r;
}

template <int N>
__host__ __device__ inline WInt<N> wsub(const WInt<N>& a, const WInt<N>& b) {
  return wadd(a, wneg(b));
}

// Signed product truncated to N limbs (caller guarantees no overflow).
template <int N>
__host__ __device__ inline WInt<N> wmul(const WInt<N>& a, const WInt<N>& b) {
  const bool na = a.negative(), nb = b.negative();
  const WInt<N> ua = na ? wneg(a) : a, ub = nb ? wneg(b) : b;
  WInt<N> r = WInt<N>::zero();
  for (int i = 0; i < N; ++i) {
    if (ua.w[i] == 0) continue;
    unsigned __int128 c = 0;
    for (int j = 0; i + j < N; ++j) {
      c += (unsigned __int128)ua.w[i] * ub.w[j] + r.w[i + j];
      r.w[i + j] = (uint64_t)c;
      c >>= 64;
    }
  }
  return (na != nb) ? wneg(r) : r;
}

template <int N>
__host__ __device__ inline int wcmp(const WInt<N>& a, const WInt<N>& b) {
  const bool na = a.negative(), nb = b.negative();
  if (na != nb) return na ? -1 : 1;
  for (int i = N - 1; i >= 0; --i)
    if (a.w[i] != b.w[i]) return a.w[i] < b.w[i] ? -1 : 1;
  return 0;
}

// ---- cloud scale ------------------------------------------------------------------
// Exact fixed-point value of a canonical binary64 word at scale S: x * 2^S.
// Valid when the cloud's scale check passed (see CloudScale).
__host__ __device__ inline int ctz64(uint64_t v) {
#ifdef __CUDA_ARCH__
  return __ffsll((long long)v) - 1;
#else
  return __builtin_ctzll(v);
#endif
}

__host__ __device__ inline __int128 fixed_of(uint64_t bits, int S) {
  const uint64_t ex = (bits >> 52) & 0x7ff, fr = bits & ((uint64_t{1} << 52) - 1);
  if (ex == 0 && fr == 0) return 0;
  uint64_t m = ex ? (fr | (uint64_t{1} << 52)) : fr;
  int e = ex ? (int)ex - 1075 : -1074;
  const int tz = ctz64(m);  // x = (m >> tz) * 2^(e + tz) with an odd significand
  m >>= tz;
  e += tz;
  const int sh = e + S;  // >= 0: S is at least the fractional bit count of x
  __int128 v = (__int128)m << sh;
  return (bits >> 63) ? -v : v;
}

// Exact squared distance of two points at scale 2^(2S) (< 2^252).
__host__ __device__ inline WInt<4> exact_dist2(const __int128* a, const __int128* b) {
  WInt<4> s = WInt<4>::zero();
  for (int i = 0; i < 3; ++i) {
    const WInt<4> d = WInt<4>::from_i128(a[i] - b[i]);
    s = wadd(s, wmul(d, d));
  }
  return s;
}

}  // namespace ehgp
