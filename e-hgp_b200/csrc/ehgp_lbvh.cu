// Canonical point cloud + exact Morton LBVH on sm_100a.
//
// Reference semantics (Ludwig-H/E-HGP, morsehgp3d/):
//  * PointIds = ranks in lexicographic binary64 total order, -0 -> +0,
//    duplicates rejected: src/cpu/spatial/point_cloud.cpp:40-94.
//  * exact global frame with least-PointId extremum witnesses:
//    exact_morton_frame, src/cpu/spatial/lbvh.cpp:107-155.
//  * exact quantiser q = floor(2^21 (x-l)/(u-l)), x=u -> 2^21-1, l=u -> 0:
//    quantized_coordinate_from_bits, lbvh.cpp:237-296.
//  * interleave x->3i+2, y->3i+1, z->3i: interleaved_morton_code, lbvh.cpp:78-91.
//  * stable (code, PointId) leaf order: lbvh.cpp:93-100,512.
//  * top-down split at the highest differing bit, midpoint for equal codes,
//    strict left/right postorder numbering: find_split / build_range,
//    lbvh.cpp:831-906.
//  * AABB witnesses: extremal PointId per axis, ties -> least PointId:
//    lower_witness / upper_witness, lbvh.cpp:46-76.
//
// B200 design: the top-down recursion is replaced by
//  (1) a Karras (2012) binary radix tree over the UNIQUE Morton codes -- its
//      splits are exactly find_split's, because a highest-differing-bit split
//      always falls on a boundary between equal-code groups;
//  (2) one balanced midpoint subtree per equal-code group (find_split's
//      collision rule), built by one thread per group;
//  (3) postorder indices from the closed form idx = 2*end - 2 - r, where r is
//      the number of right turns on the root path (a node's subtree over k
//      leaves holds 2k-1 nodes, so everything left of `begin` takes 2*begin - r
//      slots); children follow as right = idx-1, left = idx - 2*(end - split);
//  (4) witnesses reduced bottom-up with one arrival counter per node (the
//      (key, PointId) minimum is associative, so the order of merges cannot
//      change the result).
// No level-synchronous launches and no host synchronisation inside the build.
#include "ehgp_internal.cuh"

#include <cstdio>
#include <cstring>

namespace ehgp {
namespace {

constexpr int kThreads = 256;

__host__ __device__ inline uint32_t blocks_for(uint64_t n, int threads = kThreads) {
  uint64_t b = (n + threads - 1) / threads;
  return b == 0 ? 1u : (uint32_t)b;
}

// ---- exact arithmetic helpers (error-free transformations) -----------------
// Knuth's TwoSum and the FMA TwoProduct; the _rn intrinsics keep the compiler
// from contracting or reassociating them.
__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = __dadd_rn(a, b);
  const double bb = __dsub_rn(s, a);
  e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
}
__device__ __forceinline__ void two_diff(double a, double b, double& s, double& e) {
  two_sum(a, -b, s, e);
}
__device__ __forceinline__ void two_prod(double a, double b, double& p, double& e) {
  p = __dmul_rn(a, b);
  e = __fma_rn(a, b, -p);
}

// Exact sign of a sum of `count` doubles (count <= 8) by Shewchuk's
// Grow-Expansion (J. R. Shewchuk, "Adaptive Precision Floating-Point
// Arithmetic and Fast Robust Geometric Predicates", 1997, sec. 2.6): the
// expansion is nonoverlapping and ordered by magnitude, so its sign is the
// sign of its largest nonzero component.
__device__ int exact_sum_sign(const double* terms, int count) {
  double h[8];
  int len = 0;
  for (int t = 0; t < count; ++t) {
    double q = terms[t];
    for (int i = 0; i < len; ++i) {
      double s, e;
      two_sum(q, h[i], s, e);
      h[i] = e;
      q = s;
    }
    h[len++] = q;
  }
  for (int i = len - 1; i >= 0; --i) {
    if (h[i] > 0.0) return 1;
    if (h[i] < 0.0) return -1;
  }
  return 0;
}

// sign(2^21 * (x - l) - q * (u - l)), exact for finite inputs.  Returns 2 when
// an intermediate overflowed.
__device__ int quantizer_residual_sign(double dh, double dl, double eh, double el, double q) {
  double terms[6];
  terms[0] = dh * 2097152.0;
  terms[1] = dl * 2097152.0;
  double p1, e1, p2, e2;
  two_prod(q, eh, p1, e1);
  two_prod(q, el, p2, e2);
  terms[2] = -p1;
  terms[3] = -e1;
  terms[4] = -p2;
  terms[5] = -e2;
  for (int i = 0; i < 6; ++i)
    if (!isfinite(terms[i])) return 2;
  return exact_sum_sign(terms, 6);
}

// Exact sign of c0*v0 + c1*v1 + c2*v2 for small integers |c| <= 2^22 and any
// finite doubles, in a 2304-bit two's-complement accumulator.  Every finite
// binary64 is m * 2^e with |m| < 2^53 and -1074 <= e <= 971, so after
// aligning at the smallest exponent a term needs at most 2045 + 75 bits.
// Used only when the FP64 expansion route overflows (coordinates near
// +-DBL_MAX), so its cost does not matter.
__device__ int wide_sign3(const long long* c, const double* v) {
  constexpr int kLimbs = 36;
  uint64_t acc[kLimbs];
  for (int i = 0; i < kLimbs; ++i) acc[i] = 0;
  int emin = 100000;
  long long m[3];
  int e[3];
  for (int t = 0; t < 3; ++t) {
    const uint64_t bits = (uint64_t)__double_as_longlong(v[t]);
    const uint64_t ex = (bits >> 52) & 0x7ff, fr = bits & ((uint64_t{1} << 52) - 1);
    m[t] = (long long)(ex ? (fr | (uint64_t{1} << 52)) : fr);
    e[t] = ex ? (int)ex - 1075 : -1074;
    if (bits >> 63) m[t] = -m[t];
    if (m[t] != 0 && c[t] != 0) emin = min(emin, e[t]);
  }
  for (int t = 0; t < 3; ++t) {
    if (m[t] == 0 || c[t] == 0) continue;
    const bool neg = (m[t] < 0) != (c[t] < 0);
    const unsigned __int128 mag =
        (unsigned __int128)(uint64_t)(m[t] < 0 ? -m[t] : m[t]) * (uint64_t)(c[t] < 0 ? -c[t] : c[t]);
    const int shift = e[t] - emin;
    const int limb = shift >> 6, bit = shift & 63;
    // mag << bit spans up to three limbs
    uint64_t w[3];
    w[0] = (uint64_t)mag << bit;
    w[1] = bit ? (uint64_t)(mag >> (64 - bit)) : (uint64_t)(mag >> 64);
    w[2] = bit ? (uint64_t)(mag >> (128 - bit)) : 0;
    if (bit == 0) w[2] = 0;
    unsigned __int128 carry = 0;
    if (!neg) {
      for (int i = limb; i < kLimbs; ++i) {
        const uint64_t add = (i - limb < 3) ? w[i - limb] : 0;
        const unsigned __int128 s = (unsigned __int128)acc[i] + add + carry;
        acc[i] = (uint64_t)s;
        carry = s >> 64;
        if (i - limb >= 2 && carry == 0) break;
      }
    } else {
      uint64_t borrow = 0;
      for (int i = limb; i < kLimbs; ++i) {
        const uint64_t sub = (i - limb < 3) ? w[i - limb] : 0;
        const unsigned __int128 d = (unsigned __int128)acc[i] - sub - borrow;
        acc[i] = (uint64_t)d;
        borrow = (uint64_t)(d >> 64) & 1u;
        if (i - limb >= 2 && borrow == 0) break;
      }
    }
  }
  if (acc[kLimbs - 1] >> 63) return -1;
  for (int i = 0; i < kLimbs; ++i)
    if (acc[i]) return 1;
  return 0;
}

// sign(2^21 (x - l) - q (u - l)) = sign(2^21 x + (q - 2^21) l - q u), exact.
__device__ int quantizer_wide_sign(double x, double l, double u, long long q) {
  const long long c[3] = {(long long)kMortonGrid, q - (long long)kMortonGrid, -q};
  const double v[3] = {x, l, u};
  return wide_sign3(c, v);
}

// floor(2^21 (x - l) / (u - l)) exactly (quantized_coordinate_from_bits,
// src/cpu/spatial/lbvh.cpp:237-296).  The FP64 estimate is within one of the
// true floor; the exact residual sign then moves it to the unique q with
// 2^21 D - q E >= 0 > 2^21 D - (q+1) E.  Residual signs come from a
// double-double expansion, or from the wide accumulator when an intermediate
// would overflow binary64.
__device__ uint32_t quantize_axis(uint64_t xb, uint64_t lb, uint64_t ub, uint32_t* err) {
  if (lb == ub) return 0u;
  if (xb == ub) return (uint32_t)(kMortonGrid - 1);
  const double x = __longlong_as_double((long long)xb);
  const double l = __longlong_as_double((long long)lb);
  const double u = __longlong_as_double((long long)ub);
  double dh, dl, eh, el;
  two_diff(x, l, dh, dl);
  two_diff(u, l, eh, el);
  bool wide = !isfinite(dh) || !isfinite(eh) || fabs(dh) > 0x1p1000 || fabs(eh) > 0x1p1000;
  double t;
  if (!wide) {
    t = floor((dh / eh) * 2097152.0);
  } else {
    const double hd = __dsub_rn(x * 0.5, l * 0.5), he = __dsub_rn(u * 0.5, l * 0.5);
    t = floor((hd / he) * 2097152.0);
  }
  if (!(t == t)) t = 0.0;
  int64_t q = (int64_t)fmax(0.0, fmin(t, (double)(kMortonGrid - 1)));
  for (int it = 0; it < 16; ++it) {
    int s0 = wide ? 2 : quantizer_residual_sign(dh, dl, eh, el, (double)q);
    if (s0 == 2) { wide = true; s0 = quantizer_wide_sign(x, l, u, q); }
    if (s0 < 0) { --q; continue; }
    if (q + 1 <= (int64_t)kMortonGrid - 1) {
      int s1 = wide ? 2 : quantizer_residual_sign(dh, dl, eh, el, (double)(q + 1));
      if (s1 == 2) { wide = true; s1 = quantizer_wide_sign(x, l, u, q + 1); }
      if (s1 >= 0) { ++q; continue; }
    }
    return (uint32_t)q;
  }
  atomicOr(err, kErrInternal);
  return (uint32_t)q;
}

// 21-bit lane spread for 3-way interleaving (bit i -> bit 3i).
__host__ __device__ __forceinline__ uint64_t spread3(uint64_t v) {
  v &= 0x1fffffull;
  v = (v | (v << 32)) & 0x1f00000000ffffull;
  v = (v | (v << 16)) & 0x1f0000ff0000ffull;
  v = (v | (v << 8)) & 0x100f00f00f00f00full;
  v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
  v = (v | (v << 2)) & 0x1249249249249249ull;
  return v;
}

__device__ __forceinline__ uint64_t canonical_bits(uint64_t bits, uint32_t* err) {
  if ((bits & 0x7ff0000000000000ull) == 0x7ff0000000000000ull) {
    atomicOr(err, kErrNonFinite);
    return 0;
  }
  return bits == 0x8000000000000000ull ? 0ull : bits;
}

// ---- stage 1: canonical words --------------------------------------------------
__global__ void __launch_bounds__(kThreads)
k_canon_prep_f64(uint32_t n, const double* __restrict__ xyz, uint64_t* __restrict__ cin,
                 uint32_t* __restrict__ vals, uint32_t* __restrict__ err) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const uint64_t b = (uint64_t)__double_as_longlong(xyz[3ull * i + a]);
    cin[(uint64_t)a * n + i] = canonical_bits(b, err);
  }
  vals[i] = i;
}

__global__ void __launch_bounds__(kThreads)
k_canon_prep_f32(uint32_t n, const float* __restrict__ xyz, uint64_t* __restrict__ cin,
                 uint32_t* __restrict__ vals, uint32_t* __restrict__ err) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double widened = (double)xyz[3ull * i + a];  // exact widening
    cin[(uint64_t)a * n + i] = canonical_bits((uint64_t)__double_as_longlong(widened), err);
  }
  vals[i] = i;
}

// ---- stage 2: canonical cloud by PointId + duplicate check -------------------------
__global__ void __launch_bounds__(kThreads)
k_canon_finish(uint32_t n, const uint32_t* __restrict__ vals0, const uint32_t* __restrict__ vals1,
               const uint32_t* __restrict__ state, int passes, const uint64_t* __restrict__ cin,
               double* __restrict__ px, double* __restrict__ py, double* __restrict__ pz,
               uint32_t* __restrict__ source_index, uint32_t* __restrict__ err) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t* sorted = radix_result(state, passes, vals0, vals1);
  const uint32_t s = sorted[i];
  const uint64_t bx = cin[s], by = cin[(uint64_t)n + s], bz = cin[2ull * n + s];
  px[i] = __longlong_as_double((long long)bx);
  py[i] = __longlong_as_double((long long)by);
  pz[i] = __longlong_as_double((long long)bz);
  source_index[i] = s;
  if (i > 0) {
    const uint32_t t = sorted[i - 1];
    if (cin[t] == bx && cin[(uint64_t)n + t] == by && cin[2ull * n + t] == bz) atomicOr(err, kErrDuplicate);
  }
}

// ---- stage 3: exact frame (extrema + least-PointId witnesses) -----------------------
struct KeyId {
  uint64_t key;
  uint32_t id;
};
__device__ __forceinline__ bool lower_better(const KeyId& a, const KeyId& b) {  // a strictly better than b
  return a.key < b.key || (a.key == b.key && a.id < b.id);
}
__device__ __forceinline__ bool upper_better(const KeyId& a, const KeyId& b) {
  return a.key > b.key || (a.key == b.key && a.id < b.id);
}

constexpr int kFrameBlocks = kLbvhFrameBlocks;

__global__ void __launch_bounds__(kThreads)
k_frame(uint32_t n, const double* __restrict__ px, const double* __restrict__ py, const double* __restrict__ pz,
        unsigned long long* __restrict__ partial, uint32_t* __restrict__ done, uint64_t* __restrict__ frame) {
  KeyId lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    lo[a] = {~0ull, kInvalid32};
    hi[a] = {0ull, kInvalid32};
  }
  const double* P[3] = {px, py, pz};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    for (int a = 0; a < 3; ++a) {
      const KeyId k{order_key((uint64_t)__double_as_longlong(P[a][i])), i};
      if (lower_better(k, lo[a]) || lo[a].id == kInvalid32) lo[a] = k;
      if (upper_better(k, hi[a]) || hi[a].id == kInvalid32) hi[a] = k;
    }
  }
  // warp reduce
  for (int off = 16; off > 0; off >>= 1) {
    for (int a = 0; a < 3; ++a) {
      KeyId o;
      o.key = __shfl_down_sync(0xffffffffu, lo[a].key, off);
      o.id = __shfl_down_sync(0xffffffffu, lo[a].id, off);
      if (o.id != kInvalid32 && (lo[a].id == kInvalid32 || lower_better(o, lo[a]))) lo[a] = o;
      o.key = __shfl_down_sync(0xffffffffu, hi[a].key, off);
      o.id = __shfl_down_sync(0xffffffffu, hi[a].id, off);
      if (o.id != kInvalid32 && (hi[a].id == kInvalid32 || upper_better(o, hi[a]))) hi[a] = o;
    }
  }
  __shared__ KeyId s_lo[kThreads / 32][3], s_hi[kThreads / 32][3];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0)
    for (int a = 0; a < 3; ++a) { s_lo[warp][a] = lo[a]; s_hi[warp][a] = hi[a]; }
  __syncthreads();
  __shared__ bool is_last;
  if (threadIdx.x == 0) {
    for (int w = 1; w < kThreads / 32; ++w)
      for (int a = 0; a < 3; ++a) {
        if (s_lo[w][a].id != kInvalid32 && (lo[a].id == kInvalid32 || lower_better(s_lo[w][a], lo[a]))) lo[a] = s_lo[w][a];
        if (s_hi[w][a].id != kInvalid32 && (hi[a].id == kInvalid32 || upper_better(s_hi[w][a], hi[a]))) hi[a] = s_hi[w][a];
      }
    unsigned long long* my = partial + 12ull * blockIdx.x;
    for (int a = 0; a < 3; ++a) {
      my[a] = lo[a].key; my[3 + a] = lo[a].id;
      my[6 + a] = hi[a].key; my[9 + a] = hi[a].id;
    }
    __threadfence();
    const uint32_t ticket = atomicAdd(done, 1u);
    is_last = (ticket == gridDim.x - 1);
  }
  __syncthreads();
  if (!is_last || threadIdx.x != 0) return;
  __threadfence();
  KeyId L[3], H[3];
  for (int a = 0; a < 3; ++a) { L[a] = {~0ull, kInvalid32}; H[a] = {0ull, kInvalid32}; }
  for (uint32_t b = 0; b < gridDim.x; ++b) {
    const unsigned long long* pb = partial + 12ull * b;
    for (int a = 0; a < 3; ++a) {
      const KeyId l{__ldcg(pb + a), (uint32_t)__ldcg(pb + 3 + a)};
      const KeyId h{__ldcg(pb + 6 + a), (uint32_t)__ldcg(pb + 9 + a)};
      if (l.id != kInvalid32 && (L[a].id == kInvalid32 || lower_better(l, L[a]))) L[a] = l;
      if (h.id != kInvalid32 && (H[a].id == kInvalid32 || upper_better(h, H[a]))) H[a] = h;
    }
  }
  for (int a = 0; a < 3; ++a) {
    frame[a] = (uint64_t)__double_as_longlong(P[a][L[a].id]);
    frame[3 + a] = (uint64_t)__double_as_longlong(P[a][H[a].id]);
    frame[6 + a] = L[a].id;
    frame[9 + a] = H[a].id;
  }
  *done = 0;  // re-arm for the next call
}

// ---- stage 4: exact Morton codes ----------------------------------------------------
__global__ void __launch_bounds__(kThreads)
k_morton(uint32_t n, const double* __restrict__ px, const double* __restrict__ py, const double* __restrict__ pz,
         const uint64_t* __restrict__ frame, uint64_t* __restrict__ code, uint32_t* __restrict__ vals,
         uint32_t* __restrict__ err) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t qx = quantize_axis((uint64_t)__double_as_longlong(px[i]), frame[0], frame[3], err);
  const uint32_t qy = quantize_axis((uint64_t)__double_as_longlong(py[i]), frame[1], frame[4], err);
  const uint32_t qz = quantize_axis((uint64_t)__double_as_longlong(pz[i]), frame[2], frame[5], err);
  code[i] = (spread3(qx) << 2) | (spread3(qy) << 1) | spread3(qz);
  vals[i] = i;
}

// ---- stage 5: leaves, equal-code groups -------------------------------------------
__global__ void __launch_bounds__(kThreads)
k_leaves(uint32_t n, const uint32_t* __restrict__ vals0, const uint32_t* __restrict__ vals1,
         const uint32_t* __restrict__ state, int passes, const uint64_t* __restrict__ code,
         uint32_t* __restrict__ leaf_pid, uint64_t* __restrict__ leaf_code, uint32_t* __restrict__ head) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t* sorted = radix_result(state, passes, vals0, vals1);
  const uint32_t p = sorted[i];
  const uint64_t c = code[p];
  leaf_pid[i] = p;
  leaf_code[i] = c;
  head[i] = (i == 0 || code[sorted[i - 1]] != c) ? 1u : 0u;
}

// Inclusive scan of u32 in three launches (block scan, scan of block sums,
// add).  Blocks of 1024 elements.
constexpr int kScanThreads = kLbvhScanThreads;

__device__ __forceinline__ uint32_t block_inclusive_scan(uint32_t v, uint32_t* s_warp) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, v, off);
    if (lane >= off) v += t;
  }
  if (lane == 31) s_warp[warp] = v;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = (lane < (int)(blockDim.x >> 5)) ? s_warp[lane] : 0u;
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, w, off);
      if (lane >= off) w += t;
    }
    s_warp[lane] = w;
  }
  __syncthreads();
  if (warp > 0) v += s_warp[warp - 1];
  __syncthreads();
  return v;
}

__global__ void __launch_bounds__(kScanThreads)
k_scan_blocks(uint32_t n, uint32_t* __restrict__ data, uint32_t* __restrict__ sums) {
  __shared__ uint32_t s_warp[32];
  const uint32_t i = blockIdx.x * kScanThreads + threadIdx.x;
  const uint32_t v = i < n ? data[i] : 0u;
  const uint32_t inc = block_inclusive_scan(v, s_warp);
  if (i < n) data[i] = inc;
  if (threadIdx.x == kScanThreads - 1) sums[blockIdx.x] = inc;
}

__global__ void __launch_bounds__(kScanThreads)
k_scan_sums(uint32_t count, uint32_t* __restrict__ sums) {
  __shared__ uint32_t s_warp[32];
  __shared__ uint32_t s_last;
  uint32_t carry = 0;
  for (uint32_t base = 0; base < count; base += kScanThreads) {
    const uint32_t i = base + threadIdx.x;
    const uint32_t v = i < count ? sums[i] : 0u;
    const uint32_t inc = block_inclusive_scan(v, s_warp);
    if (i < count) sums[i] = inc + carry;
    if (threadIdx.x == kScanThreads - 1) s_last = inc;
    __syncthreads();
    carry += s_last;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kScanThreads)
k_scan_add(uint32_t n, uint32_t* __restrict__ data, const uint32_t* __restrict__ sums) {
  const uint32_t i = blockIdx.x * kScanThreads + threadIdx.x;
  if (i < n && blockIdx.x > 0) data[i] += sums[blockIdx.x - 1];
}

__global__ void __launch_bounds__(kThreads)
k_groups(uint32_t n, const uint32_t* __restrict__ scan, const uint64_t* __restrict__ leaf_code,
         uint32_t* __restrict__ gstart, uint64_t* __restrict__ gcode, uint32_t* __restrict__ stats) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t g = scan[i] - 1u;
  if (i == 0 || scan[i - 1] != scan[i]) {
    gstart[g] = i;
    gcode[g] = leaf_code[i];
  }
  if (i == n - 1) {
    gstart[g + 1] = n;
    stats[0] = g + 1;  // m = number of distinct codes
  }
}

// ---- stage 6: Karras radix tree over the m distinct codes ----------------------------
__device__ __forceinline__ int delta(const uint64_t* __restrict__ k, int m, int i, int j) {
  if (j < 0 || j >= m) return -1;
  return __clzll((long long)(k[i] ^ k[j]));
}

constexpr uint32_t kGroupBit = 0x80000000u;
constexpr uint32_t kRightBit = 0x80000000u;

__global__ void __launch_bounds__(kThreads)
k_karras(const uint32_t* __restrict__ stats, const uint64_t* __restrict__ gcode,
         uint32_t* __restrict__ top_left, uint32_t* __restrict__ top_right, uint32_t* __restrict__ top_split,
         uint32_t* __restrict__ top_gmin, uint32_t* __restrict__ top_gmax,
         uint32_t* __restrict__ parent_int, uint32_t* __restrict__ parent_grp) {
  const int m = (int)stats[0];
  const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= m - 1) return;
  const int d = (delta(gcode, m, i, i + 1) - delta(gcode, m, i, i - 1)) >= 0 ? 1 : -1;
  const int dmin = delta(gcode, m, i, i - d);
  int lmax = 2;
  while (delta(gcode, m, i, i + lmax * d) > dmin) lmax <<= 1;
  int l = 0;
  for (int t = lmax >> 1; t >= 1; t >>= 1)
    if (delta(gcode, m, i, i + (l + t) * d) > dmin) l += t;
  const int j = i + l * d;
  const int dnode = delta(gcode, m, i, j);
  int s = 0;
  for (int div = 2;; div <<= 1) {
    const int t = (l + div - 1) / div;
    if (delta(gcode, m, i, i + (s + t) * d) > dnode) s += t;
    if (t <= 1) break;
  }
  const int gamma = i + s * d + (d < 0 ? -1 : 0);
  const int lo = min(i, j), hi = max(i, j);
  top_split[i] = (uint32_t)gamma;
  top_gmin[i] = (uint32_t)lo;
  top_gmax[i] = (uint32_t)hi;
  if (lo == gamma) {
    top_left[i] = kGroupBit | (uint32_t)gamma;
    parent_grp[gamma] = (uint32_t)i;
  } else {
    top_left[i] = (uint32_t)gamma;
    parent_int[gamma] = (uint32_t)i;
  }
  if (hi == gamma + 1) {
    top_right[i] = kGroupBit | (uint32_t)(gamma + 1);
    parent_grp[gamma + 1] = (uint32_t)i | kRightBit;
  } else {
    top_right[i] = (uint32_t)(gamma + 1);
    parent_int[gamma + 1] = (uint32_t)i | kRightBit;
  }
  if (i == 0) parent_int[0] = kInvalid32;
}

// ---- stage 7: postorder index of every top-tree node ---------------------------------
// Top node t: t < m-1 is internal node t, otherwise group g = t - (m-1).
__global__ void __launch_bounds__(kThreads)
k_top_index(uint32_t n, const uint32_t* __restrict__ stats, const uint32_t* __restrict__ gstart,
            const uint32_t* __restrict__ top_split, const uint32_t* __restrict__ top_gmin,
            const uint32_t* __restrict__ top_gmax, const uint32_t* __restrict__ parent_int,
            const uint32_t* __restrict__ parent_grp, uint32_t* __restrict__ n_left, uint32_t* __restrict__ n_right,
            uint32_t* __restrict__ n_begin, uint32_t* __restrict__ n_end, uint32_t* __restrict__ n_parent,
            uint32_t* __restrict__ grp_root_idx, uint32_t* __restrict__ grp_depth, uint32_t* __restrict__ err) {
  const uint32_t m = stats[0];
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2 * m - 1) return;
  const bool is_group = t >= m - 1;
  uint32_t b, e, up;
  if (is_group) {
    const uint32_t g = t - (m - 1);
    b = gstart[g];
    e = gstart[g + 1];
    up = (m == 1) ? kInvalid32 : parent_grp[g];
  } else {
    b = gstart[top_gmin[t]];
    e = gstart[top_gmax[t] + 1];
    up = parent_int[t];
  }
  // walk to the root counting right turns and depth
  uint32_t right_turns = 0, depth = 0, cur = up;
  const uint32_t self_right = (up != kInvalid32 && (up & kRightBit)) ? 1u : 0u;
  while (cur != kInvalid32) {
    if (cur & kRightBit) ++right_turns;
    ++depth;
    const uint32_t p = cur & ~kRightBit;
    cur = parent_int[p];
    if (depth > 2 * n + 64) { atomicOr(err, kErrInternal); return; }
  }
  const uint32_t idx = 2 * e - 2 - right_turns;
  uint32_t pidx = kInvalid32;
  if (up != kInvalid32) {
    const uint32_t p = up & ~kRightBit;
    const uint32_t pe = gstart[top_gmax[p] + 1];
    pidx = 2 * pe - 2 - (right_turns - self_right);
    if (pidx >= 2 * n - 1) { atomicOr(err, kErrInternal); return; }
  }
  if (idx >= 2 * n - 1 || e > n || b >= e) { atomicOr(err, kErrInternal); return; }
  if (is_group) {
    const uint32_t g = t - (m - 1);
    grp_root_idx[g] = idx;
    grp_depth[g] = depth;
    n_parent[idx] = pidx;
  } else {
    const uint32_t split = gstart[top_split[t] + 1];
    n_begin[idx] = b;
    n_end[idx] = e;
    n_right[idx] = idx - 1;
    n_left[idx] = idx - 2 * (e - split);
    n_parent[idx] = pidx;
  }
}

// ---- stage 8: midpoint subtree of every equal-code group -----------------------------
__device__ __forceinline__ uint64_t axis_key(const double* __restrict__ P, uint32_t id) {
  return order_key((uint64_t)__double_as_longlong(P[id]));
}

__global__ void __launch_bounds__(kThreads)
k_group_subtrees(uint32_t n, const uint32_t* __restrict__ stats, const uint32_t* __restrict__ gstart,
                 const uint32_t* __restrict__ grp_root_idx, const uint32_t* __restrict__ grp_depth,
                 const uint32_t* __restrict__ leaf_pid, const double* __restrict__ px,
                 const double* __restrict__ py, const double* __restrict__ pz, uint32_t* __restrict__ n_left,
                 uint32_t* __restrict__ n_right, uint32_t* __restrict__ n_begin, uint32_t* __restrict__ n_end,
                 uint32_t* __restrict__ n_parent, uint32_t* __restrict__ n_lo, uint32_t* __restrict__ n_hi,
                 uint32_t* __restrict__ gstats, uint32_t* __restrict__ err) {
  const uint32_t m = stats[0];
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= m) return;
  const uint32_t N2 = 2 * n;  // stride of the witness planes
  const double* P[3] = {px, py, pz};
  const uint32_t s = gstart[g], c = gstart[g + 1] - s;
  if (c >= 2) {
    atomicAdd(&gstats[2], 1u);
    atomicMax(&gstats[3], c);
  }
  struct Item { uint32_t b, e, idx, depth; };
  Item stack[72];
  int top = 0;
  stack[top++] = {s, s + c, grp_root_idx[g], grp_depth[g]};
  uint32_t max_depth = 0;
  while (top > 0) {
    const Item it = stack[--top];
    if (it.idx >= 2 * n - 1 || it.e > n || it.b >= it.e) { atomicOr(err, kErrInternal); return; }
    max_depth = max(max_depth, it.depth);
    n_begin[it.idx] = it.b;
    n_end[it.idx] = it.e;
    // witnesses by direct scan of the (small) range
    for (int a = 0; a < 3; ++a) {
      uint32_t lo = leaf_pid[it.b], hi = lo;
      uint64_t klo = axis_key(P[a], lo), khi = klo;
      for (uint32_t q = it.b + 1; q < it.e; ++q) {
        const uint32_t id = leaf_pid[q];
        const uint64_t k = axis_key(P[a], id);
        if (k < klo || (k == klo && id < lo)) { klo = k; lo = id; }
        if (k > khi || (k == khi && id < hi)) { khi = k; hi = id; }
      }
      n_lo[(uint64_t)a * N2 + it.idx] = lo;
      n_hi[(uint64_t)a * N2 + it.idx] = hi;
    }
    if (it.e - it.b == 1) {
      n_left[it.idx] = kInvalid32;
      n_right[it.idx] = kInvalid32;
      continue;
    }
    const uint32_t split = it.b + (it.e - it.b) / 2;
    const uint32_t ridx = it.idx - 1, lidx = it.idx - 2 * (it.e - split);
    n_left[it.idx] = lidx;
    n_right[it.idx] = ridx;
    n_parent[lidx] = it.idx;
    n_parent[ridx] = it.idx;
    if (top + 2 > 72) { atomicOr(err, kErrInternal); return; }
    stack[top++] = {split, it.e, ridx, it.depth + 1};
    stack[top++] = {it.b, split, lidx, it.depth + 1};
  }
  atomicMax(&gstats[1], max_depth);
}

// ---- stage 9: bottom-up witnesses over the top tree -------------------------------------
__global__ void __launch_bounds__(kThreads)
k_bottom_up(uint32_t n, const uint32_t* __restrict__ stats, const uint32_t* __restrict__ grp_root_idx,
            const uint32_t* __restrict__ n_left, const uint32_t* __restrict__ n_right,
            const uint32_t* __restrict__ n_parent, const double* __restrict__ px, const double* __restrict__ py,
            const double* __restrict__ pz, uint32_t* n_lo, uint32_t* n_hi, uint32_t* __restrict__ n_flag,
            uint32_t* __restrict__ err) {
  const uint32_t m = stats[0];
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= m) return;
  const uint32_t N2 = 2 * n;
  const double* P[3] = {px, py, pz};
  uint32_t cur = grp_root_idx[g];
  for (uint32_t step = 0; step < 2 * n + 64; ++step) {
    const uint32_t p = n_parent[cur];
    if (p == kInvalid32) return;
    if (p >= 2 * n - 1) { atomicOr(err, kErrInternal); return; }
    __threadfence();
    if (atomicAdd(&n_flag[p], 1u) == 0u) return;  // first arrival: the sibling finishes
    __threadfence();
    const uint32_t l = n_left[p], r = n_right[p];
    if (l >= 2 * n - 1 || r >= 2 * n - 1) { atomicOr(err, kErrInternal); return; }
    for (int a = 0; a < 3; ++a) {
      const uint32_t ll = __ldcg(n_lo + (uint64_t)a * N2 + l), rl = __ldcg(n_lo + (uint64_t)a * N2 + r);
      const uint32_t lh = __ldcg(n_hi + (uint64_t)a * N2 + l), rh = __ldcg(n_hi + (uint64_t)a * N2 + r);
      const uint64_t kll = axis_key(P[a], ll), krl = axis_key(P[a], rl);
      const uint64_t klh = axis_key(P[a], lh), krh = axis_key(P[a], rh);
      const uint32_t lo = (krl < kll || (krl == kll && rl < ll)) ? rl : ll;
      const uint32_t hi = (krh > klh || (krh == klh && rh < lh)) ? rh : lh;
      __stcg(n_lo + (uint64_t)a * N2 + p, lo);
      __stcg(n_hi + (uint64_t)a * N2 + p, hi);
    }
    cur = p;
  }
  atomicOr(err, kErrInternal);
}

// ---- stage 10: export in the reference's snapshot layout --------------------------------
__global__ void __launch_bounds__(kThreads)
k_export(uint32_t n, const uint32_t* __restrict__ leaf_pid, const uint64_t* __restrict__ leaf_code,
         const uint32_t* __restrict__ n_left, const uint32_t* __restrict__ n_right,
         const uint32_t* __restrict__ n_begin, const uint32_t* __restrict__ n_end,
         const uint32_t* __restrict__ n_lo, const uint32_t* __restrict__ n_hi,
         const uint32_t* __restrict__ source_index, ehgp_lbvh_leaf* __restrict__ leaves,
         ehgp_lbvh_node* __restrict__ nodes, uint64_t* __restrict__ src64, int want_leaves, int want_nodes,
         int want_src) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t N2 = 2 * n;
  if (want_nodes && i < 2 * n - 1) {
    ehgp_lbvh_node r;
    for (int a = 0; a < 3; ++a) {
      r.lower_point_ids[a] = n_lo[(uint64_t)a * N2 + i];
      r.upper_point_ids[a] = n_hi[(uint64_t)a * N2 + i];
    }
    const uint32_t l = n_left[i], rr = n_right[i];
    r.left_child = l == kInvalid32 ? EHGP_INVALID_NODE_INDEX : l;
    r.right_child = rr == kInvalid32 ? EHGP_INVALID_NODE_INDEX : rr;
    r.leaf_begin = n_begin[i];
    r.leaf_end = n_end[i];
    nodes[i] = r;
  }
  if (i < n) {
    if (want_leaves) leaves[i] = ehgp_lbvh_leaf{leaf_code[i], leaf_pid[i]};
    if (want_src) src64[i] = source_index[i];
  }
}

}  // namespace

cudaError_t lbvh_alloc(Ctx& ctx) {
  const uint64_t n = ctx.max_points;
  LbvhBuffers& b = ctx.lb;
  cudaError_t e = cudaSuccess;
#define EHGP_ALLOC(ptr, bytes) \
  if ((e = ctx_alloc(ctx, (void**)&(ptr), (bytes))) != cudaSuccess) return e
  EHGP_ALLOC(b.xyz_in, 3 * n * sizeof(double));
  EHGP_ALLOC(b.xyz_in_f32, 3 * n * sizeof(float));
  EHGP_ALLOC(b.cin, 3 * n * sizeof(uint64_t));
  EHGP_ALLOC(b.px, n * sizeof(double));
  EHGP_ALLOC(b.py, n * sizeof(double));
  EHGP_ALLOC(b.pz, n * sizeof(double));
  EHGP_ALLOC(b.source_index, n * sizeof(uint32_t));
  EHGP_ALLOC(b.code, n * sizeof(uint64_t));
  EHGP_ALLOC(b.vals0, n * sizeof(uint32_t));
  EHGP_ALLOC(b.vals1, n * sizeof(uint32_t));
  EHGP_ALLOC(b.leaf_pid, n * sizeof(uint32_t));
  EHGP_ALLOC(b.leaf_code, n * sizeof(uint64_t));
  EHGP_ALLOC(b.group_of, n * sizeof(uint32_t));
  EHGP_ALLOC(b.block_sums, lbvh_scan_block_sums(n) * sizeof(uint32_t));
  EHGP_ALLOC(b.gstart, (n + 1) * sizeof(uint32_t));
  EHGP_ALLOC(b.gcode, n * sizeof(uint64_t));
  EHGP_ALLOC(b.top_left, n * sizeof(uint32_t));
  EHGP_ALLOC(b.top_right, n * sizeof(uint32_t));
  EHGP_ALLOC(b.top_parent_int, n * sizeof(uint32_t));
  EHGP_ALLOC(b.top_parent_grp, n * sizeof(uint32_t));
  EHGP_ALLOC(b.grp_root_idx, n * sizeof(uint32_t));
  EHGP_ALLOC(b.grp_depth, n * sizeof(uint32_t));
  // top_split/gmin/gmax share one allocation of 3n
  uint32_t* topx = nullptr;
  EHGP_ALLOC(topx, 3 * n * sizeof(uint32_t));
  b.n_flag = nullptr;
  EHGP_ALLOC(b.n_left, 2 * n * sizeof(uint32_t));
  EHGP_ALLOC(b.n_right, 2 * n * sizeof(uint32_t));
  EHGP_ALLOC(b.n_begin, 2 * n * sizeof(uint32_t));
  EHGP_ALLOC(b.n_end, 2 * n * sizeof(uint32_t));
  EHGP_ALLOC(b.n_parent, 2 * n * sizeof(uint32_t));
  EHGP_ALLOC(b.n_lo, 3 * 2 * n * sizeof(uint32_t));
  EHGP_ALLOC(b.n_hi, 3 * 2 * n * sizeof(uint32_t));
  EHGP_ALLOC(b.n_flag, 2 * n * sizeof(uint32_t));
  EHGP_ALLOC(b.frame, 12 * sizeof(uint64_t));
  EHGP_ALLOC(b.frame_partial, 12 * kFrameBlocks * sizeof(unsigned long long));
  EHGP_ALLOC(b.frame_done, sizeof(uint32_t));
  EHGP_ALLOC(b.stats, 8 * sizeof(uint32_t));
  b.export_bytes = (2 * n) * sizeof(ehgp_lbvh_node) + n * sizeof(ehgp_lbvh_leaf) + n * sizeof(uint64_t);
  EHGP_ALLOC(b.export_buf, b.export_bytes);
  ctx.lb_top_split = topx;
  ctx.lb_top_gmin = topx + n;
  ctx.lb_top_gmax = topx + 2 * n;
  const uint32_t tiles = (uint32_t)((n + kRadixTile - 1) / kRadixTile);
  ctx.radix.max_tiles = tiles;
  EHGP_ALLOC(ctx.radix.counts, 256ull * tiles * sizeof(uint32_t));
  EHGP_ALLOC(ctx.radix.state, kRadixStateWords * sizeof(uint32_t));
#undef EHGP_ALLOC
  return cudaMemsetAsync(b.frame_done, 0, sizeof(uint32_t), ctx.stream);
}

uint64_t lbvh_enqueue(Ctx& ctx, uint32_t n, int input_kind) {
  LbvhBuffers& b = ctx.lb;
  cudaStream_t st = ctx.stream;
  uint64_t launches = 0;
  const uint32_t nb = blocks_for(n);
  if (input_kind == 1)
    k_canon_prep_f32<<<nb, kThreads, 0, st>>>(n, b.xyz_in_f32, b.cin, b.vals0, ctx.d_err);
  else
    k_canon_prep_f64<<<nb, kThreads, 0, st>>>(n, b.xyz_in, b.cin, b.vals0, ctx.d_err);
  ++launches;
  // lexicographic (x, y, z): least-significant stage first
  const IndirectKey canon_stages[3] = {{b.cin + 2ull * n, 1}, {b.cin + (uint64_t)n, 1}, {b.cin, 1}};
  const int canon_bits[3] = {64, 64, 64};
  const int p1 = radix_sort_indirect(st, n, b.vals0, b.vals1, canon_stages, canon_bits, 3, ctx.radix, &launches);
  k_canon_finish<<<nb, kThreads, 0, st>>>(n, b.vals0, b.vals1, ctx.radix.state, p1, b.cin, b.px, b.py, b.pz,
                                           b.source_index, ctx.d_err);
  ++launches;
  const uint32_t fb = min(blocks_for(n), (uint32_t)kFrameBlocks);
  k_frame<<<fb, kThreads, 0, st>>>(n, b.px, b.py, b.pz, b.frame_partial, b.frame_done, b.frame);
  k_morton<<<nb, kThreads, 0, st>>>(n, b.px, b.py, b.pz, b.frame, b.code, b.vals0, ctx.d_err);
  launches += 2;
  const IndirectKey morton_stage[1] = {{b.code, 0}};
  const int morton_bits[1] = {64};
  const int p2 = radix_sort_indirect(st, n, b.vals0, b.vals1, morton_stage, morton_bits, 1, ctx.radix, &launches);
  k_leaves<<<nb, kThreads, 0, st>>>(n, b.vals0, b.vals1, ctx.radix.state, p2, b.code, b.leaf_pid, b.leaf_code,
                                     b.group_of);
  const uint32_t sb = (n + kScanThreads - 1) / kScanThreads;
  k_scan_blocks<<<sb, kScanThreads, 0, st>>>(n, b.group_of, b.block_sums);
  k_scan_sums<<<1, kScanThreads, 0, st>>>(sb, b.block_sums);
  k_scan_add<<<sb, kScanThreads, 0, st>>>(n, b.group_of, b.block_sums);
  cudaMemsetAsync(b.stats, 0, 8 * sizeof(uint32_t), st);
  k_groups<<<nb, kThreads, 0, st>>>(n, b.group_of, b.leaf_code, b.gstart, b.gcode, b.stats);
  launches += 5;
  k_karras<<<blocks_for(n > 1 ? n - 1 : 1), kThreads, 0, st>>>(b.stats, b.gcode, b.top_left, b.top_right,
                                                               ctx.lb_top_split, ctx.lb_top_gmin, ctx.lb_top_gmax,
                                                               b.top_parent_int, b.top_parent_grp);
  k_top_index<<<blocks_for(2ull * n), kThreads, 0, st>>>(n, b.stats, b.gstart, ctx.lb_top_split, ctx.lb_top_gmin,
                                                        ctx.lb_top_gmax, b.top_parent_int, b.top_parent_grp,
                                                        b.n_left, b.n_right, b.n_begin, b.n_end, b.n_parent,
                                                        b.grp_root_idx, b.grp_depth, ctx.d_err);
  k_group_subtrees<<<nb, kThreads, 0, st>>>(n, b.stats, b.gstart, b.grp_root_idx, b.grp_depth, b.leaf_pid, b.px,
                                             b.py, b.pz, b.n_left, b.n_right, b.n_begin, b.n_end, b.n_parent,
                                             b.n_lo, b.n_hi, b.stats, ctx.d_err);
  cudaMemsetAsync(b.n_flag, 0, 2ull * n * sizeof(uint32_t), st);
  k_bottom_up<<<nb, kThreads, 0, st>>>(n, b.stats, b.grp_root_idx, b.n_left, b.n_right, b.n_parent, b.px, b.py,
                                        b.pz, b.n_lo, b.n_hi, b.n_flag, ctx.d_err);
  launches += 4;
  return launches;
}

cudaError_t lbvh_export(Ctx& ctx, uint32_t n, const ehgp_lbvh_out* out) {
  LbvhBuffers& b = ctx.lb;
  cudaStream_t st = ctx.stream;
  char* base = (char*)b.export_buf;
  ehgp_lbvh_node* d_nodes = (ehgp_lbvh_node*)base;
  ehgp_lbvh_leaf* d_leaves = (ehgp_lbvh_leaf*)(base + 2ull * ctx.max_points * sizeof(ehgp_lbvh_node));
  uint64_t* d_src = (uint64_t*)((char*)d_leaves + ctx.max_points * sizeof(ehgp_lbvh_leaf));
  const int wl = out->leaves != nullptr, wn = out->nodes != nullptr, ws = out->source_index != nullptr;
  if (wl || wn || ws) {
    k_export<<<blocks_for(2ull * n), kThreads, 0, st>>>(n, b.leaf_pid, b.leaf_code, b.n_left, b.n_right, b.n_begin,
                                                        b.n_end, b.n_lo, b.n_hi, b.source_index, d_leaves, d_nodes,
                                                        d_src, wl, wn, ws);
    ctx.last_launches += 1;
  }
  cudaError_t e;
  if (wn && (e = cudaMemcpyAsync(out->nodes, d_nodes, (2ull * n - 1) * sizeof(ehgp_lbvh_node),
                                 cudaMemcpyDeviceToHost, st)) != cudaSuccess)
    return e;
  if (wl && (e = cudaMemcpyAsync(out->leaves, d_leaves, n * sizeof(ehgp_lbvh_leaf), cudaMemcpyDeviceToHost, st)) !=
                cudaSuccess)
    return e;
  if (ws && (e = cudaMemcpyAsync(out->source_index, d_src, n * sizeof(uint64_t), cudaMemcpyDeviceToHost, st)) !=
                cudaSuccess)
    return e;
  uint64_t frame[12];
  if ((e = cudaMemcpyAsync(frame, b.frame, sizeof(frame), cudaMemcpyDeviceToHost, st)) != cudaSuccess) return e;
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
  if (out->root_aabb_bits) std::memcpy(out->root_aabb_bits, frame, 6 * sizeof(uint64_t));
  if (out->root_node_index) *out->root_node_index = 2ull * n - 2;
  if (out->counters) {
    out->counters->point_count = n;
    out->counters->node_count = 2ull * n - 1;
    out->counters->maximum_depth = ctx.h_status[2];
    out->counters->morton_collision_group_count = ctx.h_status[3];
    out->counters->maximum_morton_collision_size = ctx.h_status[4];
  }
  return cudaSuccess;
}

}  // namespace ehgp
