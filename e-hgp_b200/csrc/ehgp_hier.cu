// Direct Morse hierarchy on sm_100a: terminal facade, Morse event journal,
// saddle arm seeds, strict-arm descent, frozen-root quotient and the batched
// hyper-Kruskal forest journal.
//
// Reference semantics (Ludwig-H/E-HGP, morsehgp3d/):
//  facade   src/cpu/hierarchy/direct_support_terminal.cpp:68-300 — accepted events of
//           arity 2-4 ordered by (exact level, closed rank, interior ids, support ids);
//           birth_order = rank if rank <= K_eff, saddle_order = rank - 1 if 2 <= rank <= K_eff + 1;
//  journal  src/cpu/hierarchy/direct_morse_event_journal.cpp:260-400 — n singleton births
//           (order 1, level 0) plus one role per order, batches of equal (order, exact level);
//  seeds    src/cpu/hierarchy/direct_saddle_arm_seed_journal.cpp:380-420 — one family per
//           saddle role, one arm F_u = (I u U) \ {u} per support point u;
//  forest   src/cpu/hierarchy/direct_morse_forest_journal.cpp:1042-2150 — per batch, strict
//           arms resolved against the pre-batch locator, transitive carrier quotient,
//           q_R = 0 reduced birth, 1 continuation, >= 2 multifusion, then unions and births.
//
// B200 design:
//  * events are assembled, given a rigorous FP64 level interval and sorted on the device
//    (LSD radix over the level bits); only runs whose intervals overlap are settled exactly
//    on the host (2304-bit level comparisons), so the facade order is exact;
//  * a stable partition by closed rank gives every order's births and saddle families in
//    facade order at once; births are hashed by facet on the device;
//  * each strict arm descends on its own thread: exact facet miniball (FP64 Welzl, then
//    exact verification, exhaustive exact enumeration as the fallback), LBVH ball query at
//    the miniball centre, exact top-k with the cutoff shell settled by 832-bit distance
//    comparisons, the strict level decrease certified, until the facet hits a birth;
//    the terminal facet does not depend on the locator state (a descent chain only
//    reaches a minimum, and minima of lower level are bound before the arm's batch), so
//    every arm of every batch descends in one launch;
//  * the order-by-order hyper-Kruskal pass over the resolved arms is host code with
//    incremental carrier counts.
#include "ehgp_internal.cuh"
#include "ehgp_exact.cuh"
#include "ehgp_sphere.cuh"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <atomic>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <numeric>
#include <thread>
#include <vector>

#include <sys/mman.h>
#if defined(__x86_64__)
#include <immintrin.h>
#endif

namespace ehgp {

struct HierState;

namespace {

constexpr double kU = 1.1102230246251565e-16;
constexpr double kFilt = 64.0 * kU;
constexpr double kTiny = 1e-300;
constexpr int kMaxFacet = 10;
constexpr int kT = 256;              // threads per block of the elementwise kernels
constexpr int kCandCap = 64;         // ball-query candidates per descent step
constexpr int kDStack = 96;          // LBVH traversal stack per descent thread (depth <= 63 + log2 n + 1)
constexpr uint32_t kSortQueueMin = 1u << 15;  // descent queues at least this long are sorted spatially
constexpr int kDescentSteps = 512;   // descent steps per arm

// Slow-path counters of the descent (read back per call): [0] exhaustive miniball
// enumerations, [1] exact hull signs, [2] exact closed-ball sides, [3] exact level
// conversions, [4] exact band orders, [5] exact cutoff comparisons, [6] strictness
// checks on a cutoff equal to the level.
__device__ unsigned long long g_descent_slow[8];
// LBVH nodes visited by the descent's ball queries, striped over 64 counters by block
// (one atomic per step, spread to keep a single address from serialising them).
constexpr int kVisitStripes = 64;
__device__ unsigned long long g_descent_visits[kVisitStripes];
__device__ __forceinline__ void slow(int i) { atomicAdd(&g_descent_slow[i], 1ull); }

// Descent status per arm.
enum ArmStatus : uint8_t {
  kArmOk = 0,
  kArmUnresolved = 1,   // canonical top-k choice equals the facet
  kArmPlateau = 2,      // no strict level decrease
  kArmCapacity = 3,     // ball query or traversal capacity
  kArmSteps = 4,        // step budget
  kArmInternal = 5,     // no miniball or inconsistent top-k
};

__host__ __device__ inline uint32_t nblk(uint64_t n, int t) {
  const uint64_t b = (n + t - 1) / t;
  return b == 0 ? 1u : (uint32_t)b;
}

// Device layouts of the support records (ehgp_pairs.cu, ehgp_higher.cu).
struct PairRecD {
  uint32_t u, v, interior, shell, witness;
  uint32_t ids[9];
  uint32_t pad[2];
};
struct HigherRecD {
  uint32_t size;
  uint32_t ids[4];
  uint32_t interior, shell, witness;
  uint32_t iids[8];
};
struct EvRec {
  uint32_t size, ids[4], nint, rank, iids[9];
};
static_assert(sizeof(EvRec) == 64 && sizeof(PairRecD) == 64 && sizeof(HigherRecD) == 64, "64-byte records");

__device__ __forceinline__ TNode load_node(const TNode* __restrict__ tn, uint32_t i) {
  const float4* p = reinterpret_cast<const float4*>(tn + i);
  const float4 a = __ldg(p), b = __ldg(p + 1);
  TNode t;
  t.lo[0] = a.x; t.lo[1] = a.y; t.lo[2] = a.z; t.left = __float_as_uint(a.w);
  t.hi[0] = b.x; t.hi[1] = b.y; t.hi[2] = b.z; t.right = __float_as_uint(b.w);
  return t;
}

__host__ __device__ inline double wdbl(const W& x, int shift) {  // x 2^-shift, relative error ~1e-15
  const bool neg = x.negative();
  const W a = neg ? wneg(x) : x;
  int t = 12;
  while (t > 0 && a.w[t] == 0) --t;
  double v = 0.0;
  for (int i = t; i >= 0 && i >= t - 2; --i) v += ldexp((double)a.w[i], 64 * i - shift);
  return neg ? -v : v;
}

// ---- FP64 circumsphere with uniform error bounds ---------------------------------
// Same bounds as the support kernels: with every difference coordinate bounded by
// M, |computed - exact| <= 64 u m with m of A: 1 (pair), 18 M^4 (triangle), 6 M^3
// (tetrahedron) and of each N coordinate: M (pair), 36 M^5, 18 M^4.
struct FSphere {
  double ax, ay, az;   // ids[0]
  double A, Nx, Ny, Nz;
  double eA, eN;       // error bounds of A and of each N coordinate
  double M;            // difference coordinate bound
};

__device__ void fsphere(const double* __restrict__ px, const double* __restrict__ py, const double* __restrict__ pz,
                        const uint32_t* ids, int size, FSphere& s) {
  s.ax = px[ids[0]];
  s.ay = py[ids[0]];
  s.az = pz[ids[0]];
  double e[3][3];
  double M = 0.0;
  for (int j = 1; j < size; ++j) {
    e[j - 1][0] = px[ids[j]] - s.ax;
    e[j - 1][1] = py[ids[j]] - s.ay;
    e[j - 1][2] = pz[ids[j]] - s.az;
    M = fmax(M, fmax(fabs(e[j - 1][0]), fmax(fabs(e[j - 1][1]), fabs(e[j - 1][2]))));
  }
  M *= (1.0 + 1e-15);
  s.M = M;
  const double M2 = M * M;
  if (size == 1) {
    s.A = 1.0; s.Nx = s.Ny = s.Nz = 0.0; s.eA = 0.0; s.eN = 0.0;
  } else if (size == 2) {
    s.A = 1.0; s.Nx = e[0][0]; s.Ny = e[0][1]; s.Nz = e[0][2];
    s.eA = 0.0; s.eN = 2.0 * kU * M + kTiny;
  } else if (size == 3) {
    const double G11 = (e[0][0] * e[0][0] + e[0][1] * e[0][1]) + e[0][2] * e[0][2];
    const double G22 = (e[1][0] * e[1][0] + e[1][1] * e[1][1]) + e[1][2] * e[1][2];
    const double G12 = (e[0][0] * e[1][0] + e[0][1] * e[1][1]) + e[0][2] * e[1][2];
    const double f1 = G22 * (G11 - G12), f2 = G11 * (G22 - G12);
    s.A = G11 * G22 - G12 * G12;
    s.Nx = f1 * e[0][0] + f2 * e[1][0];
    s.Ny = f1 * e[0][1] + f2 * e[1][1];
    s.Nz = f1 * e[0][2] + f2 * e[1][2];
    s.eA = kFilt * 18.0 * M2 * M2 + kTiny;
    s.eN = kFilt * 36.0 * M2 * M2 * M + kTiny;
  } else {
    const double* e1 = e[0];
    const double* e2 = e[1];
    const double* e3 = e[2];
    const double c23x = e2[1] * e3[2] - e2[2] * e3[1], c23y = e2[2] * e3[0] - e2[0] * e3[2], c23z = e2[0] * e3[1] - e2[1] * e3[0];
    const double c31x = e3[1] * e1[2] - e3[2] * e1[1], c31y = e3[2] * e1[0] - e3[0] * e1[2], c31z = e3[0] * e1[1] - e3[1] * e1[0];
    const double c12x = e1[1] * e2[2] - e1[2] * e2[1], c12y = e1[2] * e2[0] - e1[0] * e2[2], c12z = e1[0] * e2[1] - e1[1] * e2[0];
    const double q1 = (e1[0] * e1[0] + e1[1] * e1[1]) + e1[2] * e1[2];
    const double q2 = (e2[0] * e2[0] + e2[1] * e2[1]) + e2[2] * e2[2];
    const double q3 = (e3[0] * e3[0] + e3[1] * e3[1]) + e3[2] * e3[2];
    s.A = (e1[0] * c23x + e1[1] * c23y) + e1[2] * c23z;
    s.Nx = (q1 * c23x + q2 * c31x) + q3 * c12x;
    s.Ny = (q1 * c23y + q2 * c31y) + q3 * c12y;
    s.Nz = (q1 * c23z + q2 * c31z) + q3 * c12z;
    s.eA = kFilt * 6.0 * M2 * M + kTiny;
    s.eN = kFilt * 18.0 * M2 * M2 + kTiny;
  }
}

// Rigorous interval [lo, hi] of the squared radius |N|^2 / (4 A^2); false when A is not
// bounded away from 0 in FP64.
__device__ bool flevel(const FSphere& s, double& lo, double& hi) {
  const double nn = sqrt(s.Nx * s.Nx + s.Ny * s.Ny + s.Nz * s.Nz);
  const double en = s.eN * 1.7320508075688772;
  const double alo = fabs(s.A) - s.eA, ahi = fabs(s.A) + s.eA;
  if (!(alo > 0.0)) return false;
  const double nlo = fmax(nn - en, 0.0), nhi = nn + en;
  lo = nlo * nlo / (4.0 * ahi * ahi) * (1.0 - 1e-14);
  hi = nhi * nhi / (4.0 * alo * alo) * (1.0 + 1e-14);
  return isfinite(hi);
}

// Exact squared radius converted to FP64 (for ill-conditioned supports): 36-limb free.
__device__ void exact_level_fp(const Cloud& c, const uint32_t* ids, int size, double& lo, double& hi) {
  W A;
  WV N;
  exact_sphere(c, ids, size, A, N);
  // scale both to moderate magnitude: |N|^2 / (4A^2) 2^-2S
  int ta = 12, tn = 12;
  const W aa = A.negative() ? wneg(A) : A;
  while (ta > 0 && aa.w[ta] == 0) --ta;
  const W* comp[3] = {&N.x, &N.y, &N.z};
  int tmax = 0;
  for (int k = 0; k < 3; ++k) {
    const W v = comp[k]->negative() ? wneg(*comp[k]) : *comp[k];
    int t = 12;
    while (t > 0 && v.w[t] == 0) --t;
    tmax = max(tmax, t);
  }
  tn = tmax;
  const int sa = 64 * ta, sn = 64 * tn;
  const double a = wdbl(A, sa);
  const double nx = wdbl(N.x, sn), ny = wdbl(N.y, sn), nz = wdbl(N.z, sn);
  const double r = (nx * nx + ny * ny + nz * nz) / (4.0 * a * a);
  const double L = ldexp(r, 2 * sn - 2 * sa - 2 * c.S);
  lo = L * (1.0 - 1e-13);
  hi = L * (1.0 + 1e-13);
}

// ---- 1. events -------------------------------------------------------------------
__global__ void k_ev_build(uint32_t np, uint32_t nh, const PairRecD* __restrict__ pr, const HigherRecD* __restrict__ hr,
                           const double* __restrict__ px, const double* __restrict__ py,
                           const double* __restrict__ pz, const int* __restrict__ cloud_scale, EvRec* __restrict__ ev,
                           double* __restrict__ lmid, double* __restrict__ lerr, uint64_t* __restrict__ key,
                           uint32_t* __restrict__ diag) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np + nh) return;
  EvRec r;
  uint32_t shell;
  if (i < np) {
    const PairRecD p = pr[i];
    r.size = 2;
    r.ids[0] = p.u;
    r.ids[1] = p.v;
    r.ids[2] = r.ids[3] = 0;
    r.nint = p.interior;
    for (int j = 0; j < 9; ++j) r.iids[j] = j < (int)p.interior ? p.ids[j] : kInvalid32;
    shell = p.shell;
  } else {
    const HigherRecD h = hr[i - np];
    r.size = h.size;
    for (int j = 0; j < 4; ++j) r.ids[j] = h.ids[j];
    r.nint = h.interior;
    for (int j = 0; j < 9; ++j) r.iids[j] = j < 8 && j < (int)h.interior ? h.iids[j] : kInvalid32;
    shell = h.shell;
  }
  r.rank = r.nint + r.size;
  ev[i] = r;
  if (shell != r.size) {  // relevant extra-shell diagnostic: excluded from the facade
    atomicAdd(diag, 1u);
    key[i] = ~uint64_t{0};
    lmid[i] = INFINITY;
    lerr[i] = 0.0;
    return;
  }
  FSphere s;
  fsphere(px, py, pz, r.ids, (int)r.size, s);
  double lo, hi;
  if (r.size == 2) {
    const double d2 = (s.Nx * s.Nx + s.Ny * s.Ny) + s.Nz * s.Nz;
    lo = 0.25 * d2 * (1.0 - 8.0 * kU);
    hi = 0.25 * d2 * (1.0 + 8.0 * kU);
  } else if (!flevel(s, lo, hi) || hi - lo > 1e-9 * hi) {
    const Cloud c{px, py, pz, cloud_scale[0]};
    exact_level_fp(c, r.ids, (int)r.size, lo, hi);
  }
  const double mid = 0.5 * (lo + hi);
  lmid[i] = mid;
  lerr[i] = 0.5 * (hi - lo) + 1e-15 * mid;
  key[i] = dbits(mid);
}

__global__ void k_ev_gather(uint32_t m, const uint32_t* __restrict__ v0, const uint32_t* __restrict__ v1,
                            const uint32_t* __restrict__ state, int passes, const EvRec* __restrict__ ev,
                            const double* __restrict__ lmid, const double* __restrict__ lerr, EvRec* __restrict__ out,
                            double* __restrict__ omid, double* __restrict__ oerr, uint32_t* __restrict__ perm) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const uint32_t s = radix_result(state, passes, v0, v1)[i];
  out[i] = ev[s];
  omid[i] = lmid[s];
  oerr[i] = lerr[s];
  perm[i] = s;
}

// ---- scans (block-local then across blocks) -----------------------------------------
struct OpMax {
  __device__ double operator()(double a, double b) const { return fmax(a, b); }
};
struct OpMin {
  __device__ double operator()(double a, double b) const { return fmin(a, b); }
};

// Inclusive prefix max of hi[i] = mid + err (forward) and suffix min of lo = mid - err
// (backward), chunked: one block per 1024 items, then a sequential pass over blocks.
template <class Op>
__global__ void k_scan_blocks(uint32_t m, const double* __restrict__ mid, const double* __restrict__ err, double sgn,
                              int reverse, double* __restrict__ out, double* __restrict__ bsum, Op op, double ident) {
  __shared__ double sh[1024];
  const uint32_t base = blockIdx.x * 1024u;
  for (uint32_t t = threadIdx.x; t < 1024; t += blockDim.x) {
    const uint32_t j = base + t;
    double v = ident;
    if (j < m) {
      const uint32_t idx = reverse ? m - 1 - j : j;
      v = mid[idx] + sgn * err[idx];
    }
    sh[t] = v;
  }
  __syncthreads();
  for (uint32_t off = 1; off < 1024; off <<= 1) {
    double add[4];
    int c = 0;
    for (uint32_t t = threadIdx.x; t < 1024; t += blockDim.x) add[c++] = t >= off ? sh[t - off] : ident;
    __syncthreads();
    c = 0;
    for (uint32_t t = threadIdx.x; t < 1024; t += blockDim.x) {
      sh[t] = op(sh[t], add[c++]);
    }
    __syncthreads();
  }
  for (uint32_t t = threadIdx.x; t < 1024; t += blockDim.x) {
    const uint32_t j = base + t;
    if (j < m) out[reverse ? m - 1 - j : j] = sh[t];
  }
  if (threadIdx.x == 0) bsum[blockIdx.x] = sh[1023];
}

template <class Op>
__global__ void k_scan_carry(uint32_t nb, double* __restrict__ bsum, Op op, double ident) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  double run = ident;
  for (uint32_t b = 0; b < nb; ++b) {
    const double v = bsum[b];
    bsum[b] = run;  // exclusive carry
    run = op(run, v);
  }
}

template <class Op>
__global__ void k_scan_apply(uint32_t m, int reverse, double* __restrict__ out, const double* __restrict__ bsum,
                             Op op) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  const uint32_t idx = reverse ? m - 1 - j : j;
  out[idx] = op(out[idx], bsum[j / 1024u]);
}

// A boundary between facade positions p - 1 and p is certain when every level
// interval before it lies strictly below every one after it.
__global__ void k_uncertain(uint32_t m, const double* __restrict__ pre_hi, const double* __restrict__ suf_lo,
                            uint32_t* __restrict__ list, uint32_t cap, uint32_t* __restrict__ count) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p == 0 || p >= m) return;
  if (pre_hi[p - 1] < suf_lo[p]) return;
  const uint32_t at = atomicAdd(count, 1u);
  if (at < cap) list[at] = p;
}

__global__ void k_iota(uint32_t m, uint32_t* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) out[i] = i;
}

// ---- exact order inside the runs that the FP64 level intervals leave open ----------
// A run is a maximal range [lo, hi] of facade positions whose intervals overlap.  Each member
// gets its exact level key once (|N|^2 and A^2 of its circumsphere, 2304-bit integers; the
// level is |N|^2 / (4 A^2)), then one thread per run merge-sorts the run's positions by
// (exact level, closed rank, interior ids, support ids) and writes the records back in that
// order with their equal-level flags.
__global__ void k_tie_keys(uint32_t cnt, const uint32_t* __restrict__ pos, const EvRec* __restrict__ ev, Cloud c,
                           WL* __restrict__ knum, WL* __restrict__ ka2) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= cnt) return;
  const EvRec r = ev[pos[i]];
  W A;
  WV N;
  exact_sphere(c, r.ids, (int)r.size, A, N);
  const WL x = widen<36>(N.x), y = widen<36>(N.y), z = widen<36>(N.z), a = widen<36>(A);
  knum[i] = wadd(wadd(wmul(x, x), wmul(y, y)), wmul(z, z));
  ka2[i] = wmul(a, a);
}

__device__ int tie_level_cmp(const WL* knum, const WL* ka2, uint32_t i, uint32_t j) {
  return wcmp(wmul(knum[i], ka2[j]), wmul(knum[j], ka2[i]));
}

__device__ bool tie_less(const WL* knum, const WL* ka2, const EvRec* rec, uint32_t i, uint32_t j) {
  const int s = tie_level_cmp(knum, ka2, i, j);
  if (s != 0) return s < 0;
  const EvRec& a = rec[i];
  const EvRec& b = rec[j];
  if (a.rank != b.rank) return a.rank < b.rank;
  const uint32_t m = min(a.nint, b.nint);
  for (uint32_t t = 0; t < m; ++t)
    if (a.iids[t] != b.iids[t]) return a.iids[t] < b.iids[t];
  if (a.nint != b.nint) return a.nint < b.nint;
  const uint32_t ms = min(a.size, b.size);
  for (uint32_t t = 0; t < ms; ++t)
    if (a.ids[t] != b.ids[t]) return a.ids[t] < b.ids[t];
  return a.size < b.size;
}

// rec[i]: copy of the member's record (members of run r are run_off[r] .. run_off[r + 1] - 1,
// at facade positions run_lo[r] ...); idx / tmp: scratch of the member count.
__global__ void k_tie_sort(uint32_t nruns, const uint32_t* __restrict__ run_off, const uint32_t* __restrict__ run_lo,
                           const WL* __restrict__ knum, const WL* __restrict__ ka2, const EvRec* __restrict__ rec,
                           uint32_t* __restrict__ idx, uint32_t* __restrict__ tmp, EvRec* __restrict__ ev,
                           uint8_t* __restrict__ eqprev) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nruns) return;
  const uint32_t b = run_off[r], L = run_off[r + 1] - b;
  for (uint32_t t = 0; t < L; ++t) idx[b + t] = b + t;
  // bottom-up merge sort (stable) of the member indices
  uint32_t* src = idx + b;
  uint32_t* dst = tmp + b;
  for (uint32_t w = 1; w < L; w <<= 1) {
    for (uint32_t lo = 0; lo < L; lo += 2 * w) {
      const uint32_t mid = min(lo + w, L), hi = min(lo + 2 * w, L);
      uint32_t i = lo, j = mid, o = lo;
      while (i < mid && j < hi) dst[o++] = tie_less(knum, ka2, rec, src[j], src[i]) ? src[j++] : src[i++];
      while (i < mid) dst[o++] = src[i++];
      while (j < hi) dst[o++] = src[j++];
    }
    uint32_t* t = src;
    src = dst;
    dst = t;
  }
  const uint32_t p0 = run_lo[r];
  for (uint32_t t = 0; t < L; ++t) {
    ev[p0 + t] = rec[src[t]];
    if (t > 0) eqprev[p0 + t] = tie_level_cmp(knum, ka2, src[t - 1], src[t]) == 0 ? 1 : 0;
  }
}

// Gathers the facade records of the uncertain runs (the member copies of the tie sort).
__global__ void k_run_gather(uint32_t cnt, const uint32_t* __restrict__ idx, const EvRec* __restrict__ ev,
                             EvRec* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < cnt) out[i] = ev[idx[i]];
}

// Support records of facade events: out[5i] = size, out[5i + 1..4] = ids (unused 0); an
// index of kInvalid32 (level 0) or past the facade gives size 0.
__global__ void k_event_supports(uint32_t m, const uint32_t* __restrict__ idx, const EvRec* __restrict__ ev,
                                 uint32_t nev, uint32_t* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const uint32_t e = idx[i];
  const bool ok = e < nev;
  out[5ull * i] = ok ? ev[e].size : 0u;
  for (int j = 0; j < 4; ++j) out[5ull * i + 1 + j] = ok && (uint32_t)j < ev[e].size ? ev[e].ids[j] : 0u;
}

// ---- 2. level classes, rank partition, births -----------------------------------
__global__ void k_level_class(uint32_t m, const uint8_t* __restrict__ eqprev, uint32_t* __restrict__ flag) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < m) flag[p] = (p == 0 || !eqprev[p]) ? 1u : 0u;
}

// Inclusive prefix sum of 32-bit flags (block-local, then carries).
__global__ void k_sum_blocks(uint32_t m, const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                             uint32_t* __restrict__ bsum) {
  __shared__ uint32_t sh[1024];
  const uint32_t base = blockIdx.x * 1024u;
  for (uint32_t t = threadIdx.x; t < 1024; t += blockDim.x) sh[t] = base + t < m ? in[base + t] : 0u;
  __syncthreads();
  for (uint32_t off = 1; off < 1024; off <<= 1) {
    uint32_t add[4];
    int c = 0;
    for (uint32_t t = threadIdx.x; t < 1024; t += blockDim.x) add[c++] = t >= off ? sh[t - off] : 0u;
    __syncthreads();
    c = 0;
    for (uint32_t t = threadIdx.x; t < 1024; t += blockDim.x) sh[t] += add[c++];
    __syncthreads();
  }
  for (uint32_t t = threadIdx.x; t < 1024; t += blockDim.x)
    if (base + t < m) out[base + t] = sh[t];
  if (threadIdx.x == 0) bsum[blockIdx.x] = sh[1023];
}

__global__ void k_sum_carry(uint32_t nb, uint32_t* __restrict__ bsum) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  uint32_t run = 0;
  for (uint32_t b = 0; b < nb; ++b) {
    const uint32_t v = bsum[b];
    bsum[b] = run;
    run += v;
  }
}

__global__ void k_sum_apply(uint32_t m, uint32_t* __restrict__ out, const uint32_t* __restrict__ bsum, int minus1) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < m) out[j] = out[j] + bsum[j / 1024u] - (minus1 ? 1u : 0u);
}

// Rank keys for the stable partition; the rank histogram is summed per block in shared
// memory (16 bins) before one global add per bin.
__global__ void k_rank_key(uint32_t m, const EvRec* __restrict__ ev, uint64_t* __restrict__ key,
                           uint32_t* __restrict__ iota, uint32_t* __restrict__ hist) {
  __shared__ uint32_t bins[16];
  if (threadIdx.x < 16) bins[threadIdx.x] = 0;
  __syncthreads();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) {
    const uint32_t r = ev[i].rank;
    key[i] = r;
    iota[i] = i;
    atomicAdd(&bins[r < 15 ? r : 15], 1u);
  }
  __syncthreads();
  if (threadIdx.x < 16 && bins[threadIdx.x]) atomicAdd(&hist[threadIdx.x], bins[threadIdx.x]);
}

__global__ void k_rank_gather(uint32_t m, const uint32_t* __restrict__ v0, const uint32_t* __restrict__ v1,
                              const uint32_t* __restrict__ state, int passes, uint32_t* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) out[i] = radix_result(state, passes, v0, v1)[i];
}

__host__ __device__ inline uint32_t facet_hash(const uint32_t* ids, int k) {
  uint64_t h = 0x9E3779B97F4A7C15ull ^ (uint64_t)k;
  for (int i = 0; i < k; ++i) {
    h ^= ids[i];
    h *= 0xFF51AFD7ED558CCDull;
    h ^= h >> 33;
  }
  h *= 0xC4CEB9FE1A85EC53ull;
  h ^= h >> 33;
  return (uint32_t)h;
}

__device__ __forceinline__ int event_facet(const EvRec& e, uint32_t* F) {  // I u U, ascending
  int k = 0;
  for (uint32_t j = 0; j < e.nint; ++j) F[k++] = e.iids[j];
  for (uint32_t j = 0; j < e.size; ++j) F[k++] = e.ids[j];
  for (int a = 1; a < k; ++a) {
    const uint32_t x = F[a];
    int b = a;
    while (b > 0 && F[b - 1] > x) { F[b] = F[b - 1]; --b; }
    F[b] = x;
  }
  return k;
}

// Births of orders >= 2: handle = n + position in the rank partition; facets stored
// (10 words, unused = kInvalid32) and hashed (open addressing, handle per slot).
__global__ void k_birth_insert(uint32_t nb, uint32_t n, uint32_t birth_base, const uint32_t* __restrict__ rank_order,
                               const EvRec* __restrict__ ev, uint32_t* __restrict__ bfac, uint32_t* __restrict__ slots,
                               uint32_t mask, uint32_t* __restrict__ err) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  const uint32_t fi = rank_order[birth_base + b];
  uint32_t F[kMaxFacet + 1];
  const int k = event_facet(ev[fi], F);
  uint32_t* out = bfac + (uint64_t)b * kMaxFacet;
  for (int j = 0; j < kMaxFacet; ++j) out[j] = j < k ? F[j] : kInvalid32;
  const uint32_t h = n + b;
  uint32_t s = facet_hash(F, k) & mask;
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    const uint32_t prev = atomicCAS(&slots[s], kInvalid32, h);
    if (prev == kInvalid32) return;
    s = (s + 1) & mask;
  }
  atomicOr(err, kErrCapacity);
}

// Rank-partition views read by the host pass in sequence: level class and support size
// of the event at each rank position.
__global__ void k_rank_info(uint32_t m, const uint32_t* __restrict__ rank_order, const EvRec* __restrict__ ev,
                            const uint32_t* __restrict__ lclass, uint32_t* __restrict__ cls_rp,
                            uint32_t* __restrict__ size_rp) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const uint32_t fi = rank_order[i];
  cls_rp[i] = lclass[fi];
  size_rp[i] = ev[fi].size;
}

// One arm seed per support point of every saddle family (families = rank positions
// fam_lo.. in journal order; arm_off = exclusive sum of their support sizes).
__global__ void k_arm_expand(uint32_t nfam, uint32_t fam_lo, const uint32_t* __restrict__ rank_order,
                             const EvRec* __restrict__ ev, const uint32_t* __restrict__ arm_off,
                             uint32_t* __restrict__ arm_family, uint8_t* __restrict__ arm_local,
                             uint32_t* __restrict__ arm_removed) {
  const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nfam) return;
  const EvRec& e = ev[rank_order[fam_lo + f]];
  const uint32_t o = arm_off[f];
  for (uint32_t j = 0; j < e.size; ++j) {
    arm_family[o + j] = f;
    arm_local[o + j] = (uint8_t)j;
    arm_removed[o + j] = e.ids[j];
  }
}

// ---- 3. strict-arm descent ----------------------------------------------------------
struct DescentParams {
  uint32_t n, root;
  const TNode* tn;
  const double* px;
  const double* py;
  const double* pz;
  int S;
  const uint32_t* slots;
  uint32_t mask;
  const uint32_t* bfac;
  uint32_t nbirths;
};

__device__ uint32_t probe_facet(const DescentParams& d, const uint32_t* F, int k) {
  if (k == 1) return F[0];  // order-one births are the singletons, handle = PointId
  uint32_t s = facet_hash(F, k) & d.mask;
  for (uint32_t probe = 0; probe <= d.mask; ++probe) {
    const uint32_t h = __ldg(d.slots + s);
    if (h == kInvalid32) return kInvalid32;
    const uint32_t* f = d.bfac + (uint64_t)(h - d.n) * kMaxFacet;
    bool eq = true;
    for (int j = 0; j < kMaxFacet && eq; ++j) eq = __ldg(f + j) == (j < k ? F[j] : kInvalid32);
    if (eq) return h;
    s = (s + 1) & d.mask;
  }
  return kInvalid32;
}

// Exact closed-ball membership of w in the circumsphere of T (side <= 0), FP64 first.
__device__ bool inside_closed(const Cloud& c, const FSphere& fs, const uint32_t* T, int ts, uint32_t w) {
  const double x = c.px[w] - fs.ax, y = c.py[w] - fs.ay, z = c.pz[w] - fs.az;
  const double Mp = fmax(fs.M, fmax(fabs(x), fmax(fabs(y), fabs(z)))) * (1.0 + 1e-15);
  const double q = (x * x + y * y) + z * z;
  const double v = fs.A * q - ((x * fs.Nx + y * fs.Ny) + z * fs.Nz);
  const double M2 = fs.M * fs.M, M4 = M2 * M2;
  const double Am = ts <= 2 ? 1.0 : (ts == 3 ? 18.0 * M4 : 6.0 * M2 * fs.M);
  const double Nm = ts == 1 ? 0.0 : (ts == 2 ? fs.M : (ts == 3 ? 36.0 * M4 * fs.M : 18.0 * M4));
  const double bnd = kFilt * (Am * 3.0 * Mp * Mp + 3.0 * Mp * Nm) + kTiny;
  const int sa = fs.A > fs.eA ? 1 : (fs.A < -fs.eA ? -1 : 0);
  if (sa != 0) {
    if (v * sa < -bnd) return true;
    if (v * sa > bnd) return false;
  }
  slow(2);
  W A;
  WV N;
  exact_sphere(c, T, ts, A, N);
  const WV dq = c.wdiff(w, T[0]);
  const int sd = wsub(wmul(A, wdot(dq, dq)), wdot(dq, N)).sign() * A.sign();
  return sd <= 0;
}

// Exact: the circumcentre of T lies in the closed convex hull of T and T is affinely independent.
__device__ bool hull_centre(const Cloud& c, const uint32_t* T, int ts) {
  if (ts <= 2) return ts == 1 || T[0] != T[1];
  // FP64 signs with the uniform bounds of the support kernels, exact when undecided
  double e[3][3], M = 0.0;
  for (int j = 1; j < ts; ++j) {
    e[j - 1][0] = c.px[T[j]] - c.px[T[0]];
    e[j - 1][1] = c.py[T[j]] - c.py[T[0]];
    e[j - 1][2] = c.pz[T[j]] - c.pz[T[0]];
    M = fmax(M, fmax(fabs(e[j - 1][0]), fmax(fabs(e[j - 1][1]), fabs(e[j - 1][2]))));
  }
  M *= (1.0 + 1e-15);
  const double M2 = M * M;
  int sg[5];
  bool undecided = false;
  auto fs = [&](double v, double b) {
    const int r = v > b ? 1 : (v < -b ? -1 : 2);
    undecided |= r == 2;
    return r;
  };
  if (ts == 3) {
    const double G11 = (e[0][0] * e[0][0] + e[0][1] * e[0][1]) + e[0][2] * e[0][2];
    const double G22 = (e[1][0] * e[1][0] + e[1][1] * e[1][1]) + e[1][2] * e[1][2];
    const double G12 = (e[0][0] * e[1][0] + e[0][1] * e[1][1]) + e[0][2] * e[1][2];
    sg[0] = fs(G12, kFilt * 3.0 * M2 + kTiny);
    sg[1] = fs(G11 - G12, kFilt * 6.0 * M2 + kTiny);
    sg[2] = fs(G22 - G12, kFilt * 6.0 * M2 + kTiny);
    sg[3] = fs(G11 * G22 - G12 * G12, kFilt * 18.0 * M2 * M2 + kTiny);
    if (undecided) { slow(1); tri_signs_exact(c, T, sg); }
    return sg[3] != 0 && sg[0] >= 0 && sg[1] >= 0 && sg[2] >= 0;
  }
  const double* e1 = e[0];
  const double* e2 = e[1];
  const double* e3 = e[2];
  const double c23x = e2[1] * e3[2] - e2[2] * e3[1], c23y = e2[2] * e3[0] - e2[0] * e3[2], c23z = e2[0] * e3[1] - e2[1] * e3[0];
  const double c31x = e3[1] * e1[2] - e3[2] * e1[1], c31y = e3[2] * e1[0] - e3[0] * e1[2], c31z = e3[0] * e1[1] - e3[1] * e1[0];
  const double c12x = e1[1] * e2[2] - e1[2] * e2[1], c12y = e1[2] * e2[0] - e1[0] * e2[2], c12z = e1[0] * e2[1] - e1[1] * e2[0];
  const double q1 = (e1[0] * e1[0] + e1[1] * e1[1]) + e1[2] * e1[2];
  const double q2 = (e2[0] * e2[0] + e2[1] * e2[1]) + e2[2] * e2[2];
  const double q3 = (e3[0] * e3[0] + e3[1] * e3[1]) + e3[2] * e3[2];
  const double detE = (e1[0] * c23x + e1[1] * c23y) + e1[2] * c23z;
  const double Nx = (q1 * c23x + q2 * c31x) + q3 * c12x;
  const double Ny = (q1 * c23y + q2 * c31y) + q3 * c12y;
  const double Nz = (q1 * c23z + q2 * c31z) + q3 * c12z;
  const double l1 = (Nx * c23x + Ny * c23y) + Nz * c23z;
  const double l2 = (Nx * c31x + Ny * c31y) + Nz * c31z;
  const double l3 = (Nx * c12x + Ny * c12y) + Nz * c12z;
  const double l0 = (2.0 * detE) * detE - ((l1 + l2) + l3);
  const double M6 = M2 * M2 * M2;
  sg[0] = fs(detE, kFilt * 6.0 * M2 * M + kTiny);
  sg[1] = fs(l0, kFilt * 396.0 * M6 + kTiny);
  sg[2] = fs(l1, kFilt * 108.0 * M6 + kTiny);
  sg[3] = fs(l2, kFilt * 108.0 * M6 + kTiny);
  sg[4] = fs(l3, kFilt * 108.0 * M6 + kTiny);
  if (undecided) { slow(1); quad_signs_exact(c, T, sg); }
  return sg[0] != 0 && sg[1] >= 0 && sg[2] >= 0 && sg[3] >= 0 && sg[4] >= 0;
}

struct Mini {
  uint32_t T[4];
  int ts;
  FSphere fs;
};

__device__ bool verify_mini(const Cloud& c, const uint32_t* F, int k, Mini& mb) {
  if (!hull_centre(c, mb.T, mb.ts)) return false;
  fsphere(c.px, c.py, c.pz, mb.T, mb.ts, mb.fs);
  for (int i = 0; i < k; ++i) {
    bool sup = false;
    for (int j = 0; j < mb.ts; ++j) sup |= mb.T[j] == F[i];
    if (!sup && !inside_closed(c, mb.fs, mb.T, mb.ts, F[i])) return false;
  }
  return true;
}

// Exact miniball of the facet F (1..10 points): FP64 Welzl proposes the support,
// exact predicates verify it; exhaustive exact enumeration of 1..4-subsets when the
// proposal fails (build_exact_facet_miniball, hierarchy/facet_miniball.hpp:86-102).
__device__ __noinline__ bool facet_miniball(const Cloud& c, const uint32_t* F, int k, Mini& mb) {
  double P[kMaxFacet][3];
  for (int i = 0; i < k; ++i) {
    P[i][0] = c.px[F[i]] - c.px[F[0]];
    P[i][1] = c.py[F[i]] - c.py[F[0]];
    P[i][2] = c.pz[F[i]] - c.pz[F[0]];
  }
  double cx = 0, cy = 0, cz = 0, r2 = 0;
  int T[4] = {0, 0, 0, 0}, ts = 1;
  bool fp_ok = true;
  auto out = [&](int i) {
    const double dx = P[i][0] - cx, dy = P[i][1] - cy, dz = P[i][2] - cz;
    return dx * dx + dy * dy + dz * dz > r2 * (1.0 + 1e-10) + 1e-300;
  };
  auto set_ball = [&](const int* idx, int s) {
    T[0] = idx[0]; T[1] = s > 1 ? idx[1] : 0; T[2] = s > 2 ? idx[2] : 0; T[3] = s > 3 ? idx[3] : 0;
    ts = s;
    const double* a = P[idx[0]];
    if (s == 1) { cx = a[0]; cy = a[1]; cz = a[2]; r2 = 0; return; }
    double e[3][3];
    for (int j = 1; j < s; ++j)
      for (int t = 0; t < 3; ++t) e[j - 1][t] = P[idx[j]][t] - a[t];
    double A, N0, N1, N2;
    if (s == 2) {
      A = 1.0; N0 = e[0][0]; N1 = e[0][1]; N2 = e[0][2];
    } else if (s == 3) {
      const double G11 = e[0][0] * e[0][0] + e[0][1] * e[0][1] + e[0][2] * e[0][2];
      const double G22 = e[1][0] * e[1][0] + e[1][1] * e[1][1] + e[1][2] * e[1][2];
      const double G12 = e[0][0] * e[1][0] + e[0][1] * e[1][1] + e[0][2] * e[1][2];
      A = G11 * G22 - G12 * G12;
      const double f1 = G22 * (G11 - G12), f2 = G11 * (G22 - G12);
      N0 = f1 * e[0][0] + f2 * e[1][0]; N1 = f1 * e[0][1] + f2 * e[1][1]; N2 = f1 * e[0][2] + f2 * e[1][2];
    } else {
      const double* e1 = e[0]; const double* e2 = e[1]; const double* e3 = e[2];
      const double c23[3] = {e2[1] * e3[2] - e2[2] * e3[1], e2[2] * e3[0] - e2[0] * e3[2], e2[0] * e3[1] - e2[1] * e3[0]};
      const double c31[3] = {e3[1] * e1[2] - e3[2] * e1[1], e3[2] * e1[0] - e3[0] * e1[2], e3[0] * e1[1] - e3[1] * e1[0]};
      const double c12[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
      const double q1 = e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2];
      const double q2 = e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2];
      const double q3 = e3[0] * e3[0] + e3[1] * e3[1] + e3[2] * e3[2];
      A = e1[0] * c23[0] + e1[1] * c23[1] + e1[2] * c23[2];
      N0 = q1 * c23[0] + q2 * c31[0] + q3 * c12[0];
      N1 = q1 * c23[1] + q2 * c31[1] + q3 * c12[1];
      N2 = q1 * c23[2] + q2 * c31[2] + q3 * c12[2];
    }
    if (!(fabs(A) > 0.0)) { fp_ok = false; A = 1e-300; }
    const double inv = 0.5 / A;
    cx = a[0] + N0 * inv; cy = a[1] + N1 * inv; cz = a[2] + N2 * inv;
    r2 = (N0 * N0 + N1 * N1 + N2 * N2) * inv * inv;
  };
  int idx[4];
  idx[0] = 0;
  set_ball(idx, 1);
  for (int i = 1; i < k && fp_ok; ++i) {
    if (!out(i)) continue;
    idx[0] = i;
    set_ball(idx, 1);
    for (int j = 0; j < i && fp_ok; ++j) {
      if (!out(j)) continue;
      idx[0] = i; idx[1] = j;
      set_ball(idx, 2);
      for (int l = 0; l < j && fp_ok; ++l) {
        if (!out(l)) continue;
        idx[0] = i; idx[1] = j; idx[2] = l;
        set_ball(idx, 3);
        for (int m = 0; m < l && fp_ok; ++m) {
          if (!out(m)) continue;
          idx[0] = i; idx[1] = j; idx[2] = l; idx[3] = m;
          set_ball(idx, 4);
        }
      }
    }
  }
  if (fp_ok) {
    mb.ts = ts;
    for (int j = 0; j < ts; ++j) mb.T[j] = F[T[j]];
    // canonical support order (ascending ids) for the exact data
    for (int a = 1; a < ts; ++a) {
      const uint32_t x = mb.T[a];
      int b = a;
      while (b > 0 && mb.T[b - 1] > x) { mb.T[b] = mb.T[b - 1]; --b; }
      mb.T[b] = x;
    }
    if (verify_mini(c, F, k, mb)) return true;
  }
  // exhaustive exact enumeration
  slow(0);
  for (int s = (k == 1 ? 1 : 2); s <= 4 && s <= k; ++s) {
    int id[4] = {0, 1, 2, 3};
    while (true) {
      mb.ts = s;
      for (int j = 0; j < s; ++j) mb.T[j] = F[id[j]];
      if (verify_mini(c, F, k, mb)) return true;
      int p = s - 1;
      while (p >= 0 && id[p] == k - s + p) --p;
      if (p < 0) break;
      ++id[p];
      for (int q = p + 1; q < s; ++q) id[q] = id[q - 1] + 1;
    }
  }
  return false;
}

// Exact canonical top-k choice at the miniball centre of F.  Returns the status; on
// success G holds k ascending ids and *cut_below is 1 when the cutoff lies strictly
// below beta(F), 0 when it equals it.
__device__ __noinline__ int topk_choice(const DescentParams& d, const Cloud& c, const Mini& mb, int k, uint32_t* G,
                                        int* cut_below, uint32_t* visits) {
  const FSphere& fs = mb.fs;
  double llo, lhi;
  if (!flevel(fs, llo, lhi)) { slow(3); exact_level_fp(c, mb.T, mb.ts, llo, lhi); }
  // FP64 centre and its error: c~ = a + N / (2A)
  const double inv = 0.5 / fs.A;
  const double ox = fs.Nx * inv, oy = fs.Ny * inv, oz = fs.Nz * inv;
  const double cx = fs.ax + ox, cy = fs.ay + oy, cz = fs.az + oz;
  const double on = sqrt(ox * ox + oy * oy + oz * oz);
  const double nn = sqrt(fs.Nx * fs.Nx + fs.Ny * fs.Ny + fs.Nz * fs.Nz);
  const double relA = fs.eA / fmax(fabs(fs.A) - fs.eA, 1e-300);
  const double relN = fs.eN * 1.7320508075688772 / fmax(nn, 1e-300);
  double dc = on * (relA + relN) * 1.01 + 4.0 * kU * (fabs(cx) + fabs(cy) + fabs(cz)) + kTiny;
  if (!(relA < 0.5) || !isfinite(dc)) dc = 2.0 * sqrt(lhi) + 1e-300;  // centre not trusted: widen the ball
  const double R = sqrt(lhi) * (1.0 + 1e-12) + dc;
  const double R2 = R * R * (1.0 + 1e-12);
  const double ed = 2.0 * R * dc + dc * dc + 8.0 * kU * R2 + kTiny;
  // ball query
  uint32_t cid[kCandCap];
  double cd[kCandCap];
  int cnt = 0;
  uint32_t stack[kDStack];
  int top = 0;
  stack[top++] = d.root;
  // The nearest kCandCap points within R, sorted by FP64 squared distance; a farther point
  // is dropped when the list is full.  Only the points up to the band around the k-th
  // distance matter, so the traversal is pruned at the current k-th distance + 2 ed (it
  // can only decrease), and the dropped points are checked to lie beyond the band below.
  double R2_eff = R2;
  bool dropped = false;
  // The node prune runs in binary32 (the FP64 pipe is the step's tighter unit): qf is the
  // binary32 rounding of the centre and dqf its distance from it, rounded up (exact in binary64).
  // Each axis gap to a node box is lowered by the rounding of the subtraction (a relative
  // 2^-22) and by dqf, clamped at 0; the sum of squares is lowered by a relative 2^-20 and
  // compared with R2_eff rounded up.  The bound never exceeds the exact one, so the prune skips
  // only boxes that hold no point within R2_eff (the FP64 prune skips at least those; the
  // leaves decide membership in FP64 as before).  Far from the origin the FP64 prune stays.
  const double qv[3] = {cx, cy, cz};
  const bool f32 = fabs(cx) < 0x1p60 && fabs(cy) < 0x1p60 && fabs(cz) < 0x1p60 && R2 < 0x1p100;
  float qf[3], dqf[3];
  for (int a = 0; a < 3; ++a) {
    qf[a] = (float)qv[a];
    dqf[a] = __double2float_ru(fabs(qv[a] - (double)qf[a]));
  }
  float R2f = __double2float_ru(R2_eff);
  while (top > 0) {
    const uint32_t node = stack[--top];
    const TNode t = load_node(d.tn, node);
    ++*visits;
    if (t.left == kInvalid32) {
      const uint32_t q = t.right;
      const double dx = c.px[q] - cx, dy = c.py[q] - cy, dz = c.pz[q] - cz;
      const double dd = dx * dx + dy * dy + dz * dz;
      if (dd > R2_eff) continue;
      if (cnt == kCandCap) {
        if (dd >= cd[kCandCap - 1]) { dropped = true; continue; }
        --cnt;
        dropped = true;
      }
      int j = cnt++;
      while (j > 0 && cd[j - 1] > dd) { cd[j] = cd[j - 1]; cid[j] = cid[j - 1]; --j; }
      cd[j] = dd;
      cid[j] = q;
      if (cnt >= k) {
        R2_eff = fmin(R2, (cd[k - 1] + 2.0 * ed) * (1.0 + 1e-12));
        R2f = __double2float_ru(R2_eff);
      }
      continue;
    }
    if (f32) {
      float lbf = 0.f;
      for (int a = 0; a < 3; ++a) {
        const float g0 = fmaxf(fmaxf(t.lo[a] - qf[a], qf[a] - t.hi[a]), 0.f);
        const float g = fmaxf(g0 * (1.f - 0x1p-22f) - dqf[a], 0.f);
        lbf += g * g;
      }
      if (lbf * (1.f - 0x1p-20f) > R2f) continue;
    } else {
      double lb = 0.0;
      for (int a = 0; a < 3; ++a) {
        const double g = fmax(fmax((double)t.lo[a] - qv[a], qv[a] - (double)t.hi[a]), 0.0);
        lb += g * g;
      }
      if (lb * (1.0 - 1e-6) > R2_eff) continue;
    }
    if (top + 2 > kDStack) return kArmCapacity;
    stack[top++] = t.left;
    stack[top++] = t.right;
  }
  if (cnt < k) return kArmInternal;
  // partition around the k-th approximate distance
  const double tk = cd[k - 1];
  // every dropped point is at least as far as the last kept one: it must lie past the band
  if (dropped && !(cd[cnt - 1] > tk + 2.0 * ed)) return kArmCapacity;
  int below = 0, band0 = -1, band1 = -1;
  for (int i = 0; i < cnt; ++i) {
    if (cd[i] < tk - 2.0 * ed) below = i + 1;
    else if (cd[i] <= tk + 2.0 * ed) { if (band0 < 0) band0 = i; band1 = i; }
  }
  int nsel = 0;
  for (int i = 0; i < below; ++i) G[nsel++] = cid[i];
  uint32_t cut_point;
  if (band0 == band1) {  // the k-th is isolated
    G[nsel++] = cid[band0];
    cut_point = cid[band0];
  } else {
    // The band usually holds support points of F's miniball, which lie exactly on
    // its sphere: relate every band member to beta(F) (support points are equal to it
    // by construction; others by FP64, exact when undecided).  When the cutoff is
    // beta(F) the choice needs no mutual order of the members below it.
    const int nb = band1 - band0 + 1;
    uint32_t* B = cid + band0;
    int rel[kCandCap];
    int n_lo = 0, n_eq = 0, n_hi = 0;
    for (int t = 0; t < nb; ++t) {
      bool sup = false;
      for (int j = 0; j < mb.ts; ++j) sup |= mb.T[j] == B[t];
      int r;
      if (sup) r = 0;
      else if (cd[band0 + t] + ed < llo) r = -1;
      else if (cd[band0 + t] - ed > lhi) r = 1;
      else {
        slow(5);
        r = dist_cmp_exact(c, mb.T, mb.ts, B[t], mb.T[0]);
      }
      rel[t] = r;
      n_lo += r < 0;
      n_eq += r == 0;
      n_hi += r > 0;
    }
    const int need = k - below;  // >= 1
    if (need > n_lo && need <= n_lo + n_eq) {
      // cutoff = beta(F): the lower members, then the least ids at beta(F)
      for (int t = 0; t < nb; ++t)
        if (rel[t] < 0) G[nsel++] = B[t];
      uint32_t eq[kCandCap];
      int ne = 0;
      for (int t = 0; t < nb; ++t)
        if (rel[t] == 0) eq[ne++] = B[t];
      for (int a = 1; a < ne; ++a) {
        const uint32_t x = eq[a];
        int b = a;
        while (b > 0 && eq[b - 1] > x) { eq[b] = eq[b - 1]; --b; }
        eq[b] = x;
      }
      for (int t = 0; nsel < k; ++t) G[nsel++] = eq[t];
      cut_point = mb.T[0];
    } else {
      // exact order of the band by (distance, id)
      slow(4);
      for (int a = 1; a < nb; ++a) {
        const uint32_t x = B[a];
        int b = a;
        while (b > 0) {
          const int s = dist_cmp_exact(c, mb.T, mb.ts, B[b - 1], x);
          if (s < 0 || (s == 0 && B[b - 1] < x)) break;
          B[b] = B[b - 1];
          --b;
        }
        B[b] = x;
      }
      cut_point = B[need - 1];
      // strictly below the cutoff, then the least ids of the shell
      int j = 0;
      while (j < nb && dist_cmp_exact(c, mb.T, mb.ts, B[j], cut_point) < 0) G[nsel++] = B[j++];
      while (nsel < k) G[nsel++] = B[j++];  // shell members in id order
    }
  }
  for (int a = 1; a < k; ++a) {
    const uint32_t x = G[a];
    int b = a;
    while (b > 0 && G[b - 1] > x) { G[b] = G[b - 1]; --b; }
    G[b] = x;
  }
  // cutoff versus beta(F) = |T0 - centre|^2
  bool on_sphere = false;
  for (int j = 0; j < mb.ts; ++j) on_sphere |= mb.T[j] == cut_point;
  if (on_sphere) {
    *cut_below = 0;
  } else {
    // FP64 first: the cutoff's approximate distance against the radius interval
    const double dcut = band0 == band1 ? cd[band0] : tk + 2.0 * ed;  // upper bound of the cutoff's FP distance
    if (dcut + ed < llo) {
      *cut_below = 1;
    } else {
      slow(5);
      const int s = dist_cmp_exact(c, mb.T, mb.ts, cut_point, mb.T[0]);
      if (s > 0) return kArmInternal;
      *cut_below = s < 0 ? 1 : 0;
    }
  }
  return kArmOk;
}

// Facet of arm a: F_u = (I u U) \ {u}, ascending.
__device__ __forceinline__ int arm_facet(const EvRec& e, uint32_t removed, uint32_t* F) {
  int k = event_facet(e, F);
  int w = 0;
  for (int j = 0; j < k; ++j)
    if (F[j] != removed) F[w++] = F[j];
  return w;
}

// First probe of every arm: most arms are themselves a birth facet of their order.
// Misses are queued with their facet for the descent steps.
__global__ void k_arm_probe(DescentParams d, uint32_t a0, uint32_t narms,
                            const uint32_t* __restrict__ fam_event /* rank_order + fam_lo */,
                            const uint32_t* __restrict__ arm_family, const uint8_t* __restrict__ arm_local,
                            const EvRec* __restrict__ ev, uint32_t* __restrict__ term, uint8_t* __restrict__ status,
                            uint32_t* __restrict__ q_arm, uint32_t* __restrict__ q_fac, uint32_t* __restrict__ q_count) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= narms) return;
  const uint32_t a = a0 + i;
  const EvRec e = ev[fam_event[arm_family[a]]];
  uint32_t F[kMaxFacet + 1];
  const int k = arm_facet(e, e.ids[arm_local[a]], F);
  const uint32_t h = probe_facet(d, F, k);
  term[a] = h;
  status[a] = kArmOk;
  if (h != kInvalid32) return;
  const uint32_t slot = atomicAdd(q_count, 1u);
  q_arm[slot] = a;
  for (int j = 0; j < kMaxFacet; ++j) q_fac[(uint64_t)slot * kMaxFacet + j] = j < k ? F[j] : kInvalid32;
}

// One strict descent step for every queued arm: exact miniball of F, exact canonical
// top-k choice G at its centre, certified beta(G) < beta(F); G is probed and either
// binds the arm or is queued for the next step.
// Blocks per SM the descent step's register budget is sized for: 8 x 128 threads gives 64
// registers and 32 warps per SM; the spills cost less than the latency they hide (measured at
// 50k: 3 blocks 246 ms, 4 222, 6 188, 8 172, 10 168, 12 176).
#ifndef EHGP_STEP_BLOCKS_PER_SM
#define EHGP_STEP_BLOCKS_PER_SM 8
#endif
// Sort keys of a descent queue: the top 24 bits of the Morton code of each facet's least
// point, so that a warp's threads descend from nearby facets (shared traversal paths,
// less divergence).  The order of processing never changes a result.
__global__ void k_queue_keys(uint32_t m, const uint32_t* __restrict__ in_fac, const uint64_t* __restrict__ code,
                             uint64_t* __restrict__ key, uint32_t* __restrict__ val) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  key[i] = code[in_fac[(uint64_t)i * kMaxFacet]] >> 39;
  val[i] = i;
}

__global__ void __launch_bounds__(128, EHGP_STEP_BLOCKS_PER_SM)
k_arm_step(DescentParams d, uint32_t m, const uint32_t* __restrict__ in_arm, const uint32_t* __restrict__ in_fac,
           const uint32_t* __restrict__ rstate, int passes, const uint32_t* __restrict__ v0,
           const uint32_t* __restrict__ v1, uint32_t* __restrict__ out_arm, uint32_t* __restrict__ out_fac,
           uint32_t* __restrict__ out_count, uint32_t* __restrict__ term, uint8_t* __restrict__ status,
           unsigned long long* __restrict__ stats) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= m) return;
  // queue entry: in Morton order of the facets when the queue was sorted (passes >= 0)
  const uint32_t i = passes >= 0 ? radix_result(rstate, passes, v0, v1)[t] : t;
  const uint32_t a = in_arm[i];
  uint32_t F[kMaxFacet];
  int k = 0;
  for (int j = 0; j < kMaxFacet; ++j) {
    F[j] = in_fac[(uint64_t)i * kMaxFacet + j];
    k += F[j] != kInvalid32;
  }
  const Cloud c{d.px, d.py, d.pz, d.S};
  auto fail = [&](int why) {  // stats[3] counts failed arms
    status[a] = (uint8_t)why;
    atomicAdd(stats + 3, 1ull);
  };
  Mini mb;
  if (!facet_miniball(c, F, k, mb)) { fail(kArmInternal); return; }
  uint32_t G[kMaxFacet];
  int cut_below = 0;
  uint32_t visits = 0;
  const int s = topk_choice(d, c, mb, k, G, &cut_below, &visits);
  atomicAdd(&g_descent_visits[blockIdx.x % kVisitStripes], (unsigned long long)visits);
  if (s != kArmOk) { fail(s); return; }
  bool same = true;
  for (int j = 0; j < k; ++j) same &= G[j] == F[j];
  if (same) { fail(kArmUnresolved); return; }
  if (!cut_below) {  // beta(G) <= cutoff = beta(F): the decrease must be strict
    slow(6);
    Mini mg;
    if (!facet_miniball(c, G, k, mg)) { fail(kArmInternal); return; }
    double glo, ghi, flo, fhi;
    if (!flevel(mg.fs, glo, ghi)) exact_level_fp(c, mg.T, mg.ts, glo, ghi);
    if (!flevel(mb.fs, flo, fhi)) exact_level_fp(c, mb.T, mb.ts, flo, fhi);
    if (!(ghi < flo) && level_cmp_exact(c, mg.T, mg.ts, mb.T, mb.ts) >= 0) { fail(kArmPlateau); return; }
    atomicAdd(stats + 2, 1ull);
  }
  atomicAdd(stats, 1ull);
  const uint32_t h = probe_facet(d, G, k);
  if (h != kInvalid32) {
    term[a] = h;
    return;
  }
  const uint32_t slot = atomicAdd(out_count, 1u);
  out_arm[slot] = a;
  for (int j = 0; j < kMaxFacet; ++j) out_fac[(uint64_t)slot * kMaxFacet + j] = j < k ? G[j] : kInvalid32;
}

}  // namespace

// ---- host state ---------------------------------------------------------------------
// Streaming (non-temporal) store of one record of 4-byte words: the forest records are
// written once and read at copy-out, so they bypass the caches that hold the union-find
// arrays.  stream_fence() orders them before a release that publishes them.
template <class T>
inline void nt_store(T& dst, const T& v) {
  static_assert(sizeof(T) % 4 == 0, "records of 4-byte words");
#if defined(__x86_64__)
  if (sizeof(T) % 16 == 0 && (reinterpret_cast<uintptr_t>(&dst) & 15) == 0) {  // whole 16-byte stores
    __m128i* d = reinterpret_cast<__m128i*>(&dst);
    for (size_t i = 0; i < sizeof(T) / 16; ++i) {
      __m128i w;
      std::memcpy(&w, reinterpret_cast<const char*>(&v) + 16 * i, 16);
      _mm_stream_si128(d + i, w);
    }
    return;
  }
  const int* s = reinterpret_cast<const int*>(&v);
  int* d = reinterpret_cast<int*>(&dst);
  for (size_t i = 0; i < sizeof(T) / 4; ++i) _mm_stream_si32(d + i, s[i]);
#else
  dst = v;
#endif
}
inline void stream_fence() {
#if defined(__x86_64__)
  _mm_sfence();
#endif
}

constexpr uint32_t kUnborn = 0xFFFFFFFEu;  // HierDsu::rroot of a handle not yet born

struct HierDsu {
  uint32_t parent, rroot;  // rroot: the component's reduced root (at roots), kUnborn before the birth
};

// Anonymous mapping advised for transparent huge pages: the union-find array is read at
// random, and 2 MB pages keep its translations in the TLB.  Capacity is kept across calls.
struct HugeBuf {
  void* p = nullptr;
  size_t bytes = 0;
  HugeBuf() = default;
  HugeBuf(const HugeBuf&) = delete;
  HugeBuf& operator=(const HugeBuf&) = delete;
  ~HugeBuf() {
    if (p) munmap(p, bytes);
  }
  bool ensure(size_t need) {
    if (need <= bytes) return true;
    if (p) munmap(p, bytes);
    p = nullptr;
    bytes = 0;
    const size_t align = size_t{2} << 20, b = (need + align - 1) / align * align;
    void* q = mmap(nullptr, b, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS, -1, 0);
    if (q == MAP_FAILED) return false;
    madvise(q, b, MADV_HUGEPAGE);
    p = q;
    bytes = b;
    return true;
  }
};

// Growable storage of plain C records that keeps its capacity across calls and leaves new
// storage uninitialised; n counts the records in use.  Writers stay within the capacity
// reserved up front (fits() reports an overrun, which is never written).
template <class T>
struct Arena {
  std::unique_ptr<T[]> p;
  uint64_t cap = 0, n = 0;
  void reset(uint64_t need) {
    if (need > cap) {
      p.reset(new T[need]);
      cap = need;
    }
    n = 0;
  }
  uint64_t size() const { return n; }
  bool fits() const { return n <= cap; }
  T& operator[](uint64_t i) { return p[i]; }
  const T& operator[](uint64_t i) const { return p[i]; }
  T* begin() { return p.get(); }
  T* end() { return p.get() + n; }
  void push_back(const T& x) {
    if (n < cap) p[n] = x;
    ++n;
  }
  template <class It>
  void append(It first, It last) {
    for (; first != last; ++first) push_back(*first);
  }
};

struct HierOrderOut {  // one order's journal and forest arenas, local indices
  Arena<ehgp_journal_batch> jb;
  Arena<ehgp_role_record> roles;
  Arena<ehgp_family_record> fam;
  Arena<ehgp_forest_node> nodes;
  Arena<uint32_t> children;
  Arena<ehgp_forest_birth> births;
  Arena<ehgp_forest_binding> bindings;
  Arena<ehgp_forest_saddle> saddles;
  Arena<ehgp_forest_group> groups;
  Arena<ehgp_forest_batch> fb;
  Arena<ehgp_forest_root> roots;
  Arena<uint32_t> node_cls;  // level class of each node (kInvalid32: an order-one birth node)
  Arena<uint32_t> fam_res;   // resulting root of each family's atomic group (local node id)
  Arena<uint32_t> v_res;     // vertical maps from this order: each node's carrier-saddle root one order down
  Arena<uint32_t> v_cls;     // and its own level class
  int status = EHGP_OK;
  const char* msg = "";
  double ms = 0;
};

struct HierOff {
  uint32_t jb, role, fam, node, child, birth, bind, sad, grp, root, vert;
};

struct HierState {
  std::vector<void*> allocs;
  uint64_t cap_events = 0, cap_arms = 0, cap_births = 0, cap_slots = 0;
  // device
  EvRec* ev_raw = nullptr;
  EvRec* ev = nullptr;          // facade order
  double* lmid_raw = nullptr;
  double* lerr_raw = nullptr;
  double* lmid = nullptr;
  double* lerr = nullptr;
  uint64_t* key = nullptr;
  uint64_t* key2 = nullptr;     // key-value sort scratch
  uint32_t* order0 = nullptr;
  uint32_t* order1 = nullptr;
  uint32_t* perm = nullptr;
  double* pre_hi = nullptr;
  double* suf_lo = nullptr;
  double* bsum = nullptr;
  uint32_t* ubsum = nullptr;
  uint32_t* uncertain = nullptr;
  uint8_t* eqprev = nullptr;
  uint32_t* lclass = nullptr;   // level class per facade index
  uint32_t* rank_order = nullptr;
  uint32_t* counters = nullptr; // [0] diag, [1] uncertain, [2] err, [3..18] rank histogram
  uint32_t* radix_counts = nullptr;
  uint32_t* bfac = nullptr;
  uint32_t* slots = nullptr;
  uint32_t* fam_event = nullptr;
  uint32_t* arm_family = nullptr;
  uint8_t* arm_local = nullptr;
  uint32_t* term = nullptr;
  uint8_t* arm_status = nullptr;
  unsigned long long* dstats = nullptr;
  uint32_t* qcount = nullptr;   // [0] first-probe misses, [1], [2] step outputs (ping-pong)
  uint32_t* q_arm[2] = {nullptr, nullptr};
  uint32_t* q_fac[2] = {nullptr, nullptr};
  uint64_t q_cap = 0;
  cudaEvent_t ev_block = nullptr;  // blocking-sync event: the descent loop waits without spinning a core
  uint32_t first_misses = 0, descent_rounds = 0;
  unsigned long long slow[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  unsigned long long visits[kVisitStripes] = {};  // ball-query node visits of the descent steps
  // host results
  uint32_t n = 0, K = 0, keff = 0;
  int S = 0;
  uint64_t events = 0, diagnostics = 0;
  std::vector<HierOrderOut> outs;     // per-order arenas (capacity kept across calls)
  HugeBuf dsu;
  uint64_t pin_m = 0, pin_arms = 0;   // pinned host views of the last call
  uint32_t* p_rank = nullptr;
  uint32_t* p_cls = nullptr;
  uint32_t* p_armoff = nullptr;
  uint32_t* p_term = nullptr;
  uint8_t* p_stat = nullptr;
  uint32_t* d_cls_rp = nullptr;       // device views (event capacity)
  uint32_t* d_size_rp = nullptr;
  uint32_t* d_armoff = nullptr;
  uint32_t* d_removed = nullptr;
  // exact order of the facade's tie runs on the device (capacities kept across calls)
  WL* tie_num = nullptr;   // [tie_cap] |N|^2 of each run member
  WL* tie_a2 = nullptr;    // [tie_cap] A^2
  uint32_t* tie_idx = nullptr;
  uint32_t* tie_tmp = nullptr;
  uint32_t* tie_pos = nullptr;
  uint32_t* run_off = nullptr;
  uint32_t* run_lo = nullptr;
  uint64_t tie_cap = 0, run_cap = 0;
  // The result stays in the per-order arenas (local indices); off[k] holds the global
  // offsets of order k's records, off[keff + 1] the totals.  Records take their global
  // indices when they are copied out.  An empty `off` means no result.
  std::vector<HierOff> off;
  uint64_t arm_seeds = 0;  // d_removed holds the removed point of each arm seed
  std::vector<std::vector<ehgp_vertical_assignment>> vert;  // per source order, global node ids
  uint32_t decision = EHGP_ERR_NOT_BUILT;
  double ms_device = 0, ms_forest = 0, ms_descent = 0, ms_orders = 0;
  double ms_host[4] = {0, 0, 0, 0};  // exact facade ties, order passes, (unused), vertical maps
  uint64_t descent_steps = 0, arms = 0, exact_boundaries = 0;
  cudaEvent_t ev_step[2] = {nullptr, nullptr};  // around each descent-step launch
  double ms_steps = 0;                          // summed k_arm_step launch times
  uint64_t step_launches = 0;
  // Schedule of the host forest pass and of the descent parts (results never depend on it):
  // single-role batches per published chunk, arms per descent part, host pool threads
  // (0: every hardware thread).
  uint32_t chunk_batches = 1u << 14, part_arms = 1u << 22, pool_threads = 0;
};

void hier_free(Ctx& ctx) {
  if (!ctx.hier) return;
  for (void* p : ctx.hier->allocs) cudaFree(p);
  for (void* p : {(void*)ctx.hier->q_arm[0], (void*)ctx.hier->q_arm[1], (void*)ctx.hier->q_fac[0],
                  (void*)ctx.hier->q_fac[1]})
    if (p) cudaFree(p);
  for (void* p : {(void*)ctx.hier->p_rank, (void*)ctx.hier->p_cls, (void*)ctx.hier->p_armoff,
                  (void*)ctx.hier->p_term, (void*)ctx.hier->p_stat})
    if (p) cudaFreeHost(p);
  if (ctx.hier->ev_block) cudaEventDestroy(ctx.hier->ev_block);
  for (void* q : {(void*)ctx.hier->tie_num, (void*)ctx.hier->tie_a2, (void*)ctx.hier->tie_idx,
                  (void*)ctx.hier->tie_tmp, (void*)ctx.hier->tie_pos, (void*)ctx.hier->run_off,
                  (void*)ctx.hier->run_lo})
    if (q) cudaFree(q);
  for (cudaEvent_t ev : ctx.hier->ev_step)
    if (ev) cudaEventDestroy(ev);
  delete ctx.hier;
  ctx.hier = nullptr;
}

namespace {

template <class T>
cudaError_t halloc(HierState& h, T** p, uint64_t count) {
  void* q = nullptr;
  const cudaError_t e = cudaMalloc(&q, count * sizeof(T) + 16);
  if (e != cudaSuccess) return e;
  h.allocs.push_back(q);
  *p = (T*)q;
  return cudaSuccess;
}

void hfree_all(HierState& h) {
  for (void* p : h.allocs) cudaFree(p);
  h.allocs.clear();
  h.qcount = nullptr;
  h.cap_events = h.cap_arms = h.cap_births = h.cap_slots = 0;
}

cudaError_t ensure_events(HierState& h, uint64_t m) {
  if (m <= h.cap_events && h.cap_events) return cudaSuccess;
  hfree_all(h);
  const uint64_t cap = m + m / 8 + 1024;
  cudaError_t e;
#define HA(p, c) if ((e = halloc(h, &(p), (c))) != cudaSuccess) return e
  HA(h.ev_raw, cap);
  HA(h.ev, cap);
  HA(h.lmid_raw, cap);
  HA(h.lerr_raw, cap);
  HA(h.lmid, cap);
  HA(h.lerr, cap);
  HA(h.key, cap);
  HA(h.key2, cap);
  HA(h.order0, cap);
  HA(h.order1, cap);
  HA(h.perm, cap);
  HA(h.pre_hi, cap);
  HA(h.suf_lo, cap);
  HA(h.bsum, cap / 1024 + 2);
  HA(h.ubsum, cap / 1024 + 2);
  HA(h.uncertain, 1u << 20);
  HA(h.eqprev, cap);
  HA(h.lclass, cap);
  HA(h.rank_order, cap);
  HA(h.counters, 32);
  HA(h.radix_counts, 256ull * ((cap + kRadixTile - 1) / kRadixTile) + 256);
  HA(h.bfac, cap * kMaxFacet);
  HA(h.fam_event, cap);
  HA(h.d_cls_rp, cap);
  HA(h.d_size_rp, cap);
  HA(h.d_armoff, cap + 1);
  HA(h.dstats, 4);
  const uint64_t arms = 4 * cap;
  HA(h.arm_family, arms);
  HA(h.arm_local, arms);
  HA(h.term, arms);
  HA(h.arm_status, arms);
  HA(h.d_removed, arms);
  uint64_t slots = 1;
  while (slots < 2 * cap + 1024) slots <<= 1;
  HA(h.slots, slots);
#undef HA
  h.cap_events = cap;
  h.cap_arms = arms;
  h.cap_slots = slots;
  return cudaSuccess;
}


void scan_minmax(cudaStream_t st, uint32_t m, const double* mid, const double* err, double* out, double* bsum,
                 bool forward_max, uint64_t* launches) {
  const uint32_t nb = nblk(m, 1024);
  if (forward_max) {
    k_scan_blocks<<<nb, 256, 0, st>>>(m, mid, err, 1.0, 0, out, bsum, OpMax{}, -INFINITY);
    k_scan_carry<<<1, 1, 0, st>>>(nb, bsum, OpMax{}, -INFINITY);
    k_scan_apply<<<nblk(m, kT), kT, 0, st>>>(m, 0, out, bsum, OpMax{});
  } else {
    k_scan_blocks<<<nb, 256, 0, st>>>(m, mid, err, -1.0, 1, out, bsum, OpMin{}, INFINITY);
    k_scan_carry<<<1, 1, 0, st>>>(nb, bsum, OpMin{}, INFINITY);
    k_scan_apply<<<nblk(m, kT), kT, 0, st>>>(m, 1, out, bsum, OpMin{});
  }
  *launches += 3;
}

}  // namespace

int hier_run(Ctx& ctx, uint32_t K) {
  if (!ctx.hier) ctx.hier = new HierState();
  HierState& h = *ctx.hier;
  const uint32_t n = (uint32_t)ctx.built_n;
  cudaStream_t st = ctx.stream;
  LbvhBuffers& b = ctx.lb;
  GeomBuffers& g = ctx.gb;
  uint64_t launches = 0;
  h.decision = EHGP_ERR_NOT_BUILT;
  h.off.clear();
  h.arm_seeds = 0;
  h.n = n;
  h.K = K;
  h.keff = K < n ? K : n;
  if (K == 0 || K > 10) return abi_fail(&ctx, EHGP_ERR_INVALID_ARGUMENT, "K_max must be in [1, 10]");
  // supports for this K
  uint32_t np = 0, nh = 0;
  if (!(ctx.pb.K == K && ctx.pb.resident)) {  // pair supports of this cloud and K
    const int s = pairs_run(ctx, K, &np);
    if (s != EHGP_OK) return s;
  }
  np = ctx.pb.count;
  if (ctx.hb.K != K) {
    const int s = higher_run(ctx, K, &nh);
    if (s != EHGP_OK) return s;
  }
  nh = ctx.hb.count;
  const auto t0 = std::chrono::steady_clock::now();
  cudaEventRecord(ctx.ev0, st);
  const uint64_t total = (uint64_t)np + nh;
  cudaError_t e = ensure_events(h, total + 1);
  if (e != cudaSuccess) return abi_fail(&ctx, EHGP_ERR_OUT_OF_MEMORY, "hierarchy buffers do not fit the device");
  cudaMemsetAsync(h.counters, 0, 32 * sizeof(uint32_t), st);
  cudaMemsetAsync(h.dstats, 0, 4 * sizeof(unsigned long long), st);
  {
    const unsigned long long zero[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    cudaMemcpyToSymbolAsync(g_descent_slow, zero, sizeof(zero), 0, cudaMemcpyHostToDevice, st);
    static const unsigned long long zv[kVisitStripes] = {};
    cudaMemcpyToSymbolAsync(g_descent_visits, zv, sizeof(zv), 0, cudaMemcpyHostToDevice, st);
  }
  if (total)
    k_ev_build<<<nblk(total, kT), kT, 0, st>>>(np, nh, (const PairRecD*)ctx.pb.sorted, (const HigherRecD*)ctx.hb.sorted,
                                                b.px, b.py, b.pz, g.scale, h.ev_raw, h.lmid_raw, h.lerr_raw, h.key,
                                                h.counters);
  ++launches;
  uint32_t hc[2] = {0, 0};
  cudaMemcpyAsync(hc, h.counters, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return abi_cuda_fail(&ctx, e, "hierarchy events");
  h.diagnostics = hc[0];
  const uint32_t m = (uint32_t)(total - hc[0]);
  h.events = m;
  // facade order by the FP64 level midpoints (diagnostics sort last)
  RadixScratch rs{h.radix_counts, ctx.radix.state, (uint32_t)((h.cap_events + kRadixTile - 1) / kRadixTile)};
  if (total) {
    k_iota<<<nblk(total, kT), kT, 0, st>>>((uint32_t)total, h.order0);
    ++launches;
    // facade order: the event keys (FP64 level midpoints, diagnostics last) move with the indices
    const int passes = radix_sort_kv(st, (uint32_t)total, h.order0, h.order1, h.key, h.key2, 64, rs, &launches);
    k_ev_gather<<<nblk(total, kT), kT, 0, st>>>((uint32_t)total, h.order0, h.order1, ctx.radix.state, passes, h.ev_raw,
                                                 h.lmid_raw, h.lerr_raw, h.ev, h.lmid, h.lerr, h.perm);
    ++launches;
  }
  int scale_h[4];
  cudaMemcpyAsync(scale_h, g.scale, sizeof(scale_h), cudaMemcpyDeviceToHost, st);
  cudaMemsetAsync(h.eqprev, 0, m + 1, st);
  uint32_t unc = 0;
  if (m > 1) {
    scan_minmax(st, m, h.lmid, h.lerr, h.pre_hi, h.bsum, true, &launches);
    scan_minmax(st, m, h.lmid, h.lerr, h.suf_lo, h.bsum, false, &launches);
    k_uncertain<<<nblk(m, kT), kT, 0, st>>>(m, h.pre_hi, h.suf_lo, h.uncertain, 1u << 20, h.counters + 1);
    ++launches;
    cudaMemcpyAsync(&unc, h.counters + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
  }
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return abi_cuda_fail(&ctx, e, "hierarchy facade order");
  h.S = scale_h[0];
  if (unc > (1u << 20)) return abi_fail(&ctx, EHGP_ERR_CAPACITY, "too many uncertain level boundaries in the facade");
  double ms_ties = 0;
  if (unc) {
    const auto tt0 = std::chrono::steady_clock::now();
    std::vector<uint32_t> list(unc);
    cudaMemcpy(list.data(), h.uncertain, unc * sizeof(uint32_t), cudaMemcpyDeviceToHost);
    std::sort(list.begin(), list.end());
    // maximal runs of positions whose order the FP64 intervals leave open: a run starts one
    // before its first uncertain boundary (that boundary before it is certain)
    std::vector<uint32_t> run_off, run_lo, idx;
    for (size_t i = 0; i < list.size();) {
      const uint32_t s0 = list[i] - 1;
      uint32_t s1 = list[i];
      size_t j = i + 1;
      while (j < list.size() && list[j] == s1 + 1) s1 = list[j++];
      run_off.push_back((uint32_t)idx.size());
      run_lo.push_back(s0);
      for (uint32_t t = s0; t <= s1; ++t) idx.push_back(t);
      i = j;
    }
    run_off.push_back((uint32_t)idx.size());
    const uint32_t cnt = (uint32_t)idx.size(), nruns = (uint32_t)run_lo.size();
    // settled on the device: exact level keys per member, then a merge sort per run
    if (h.tie_cap < cnt || h.run_cap < nruns + 1) {
      for (void* q : {(void*)h.tie_num, (void*)h.tie_a2, (void*)h.tie_idx, (void*)h.tie_tmp, (void*)h.tie_pos,
                      (void*)h.run_off, (void*)h.run_lo})
        if (q) cudaFree(q);
      h.tie_num = h.tie_a2 = nullptr;
      h.tie_idx = h.tie_tmp = h.tie_pos = h.run_off = h.run_lo = nullptr;
      h.tie_cap = h.run_cap = 0;
      const uint64_t tc = cnt + cnt / 4 + 64, rc = nruns + nruns / 4 + 64;
      if (cudaMalloc(&h.tie_num, tc * sizeof(WL)) != cudaSuccess || cudaMalloc(&h.tie_a2, tc * sizeof(WL)) != cudaSuccess ||
          cudaMalloc(&h.tie_idx, tc * 4) != cudaSuccess || cudaMalloc(&h.tie_tmp, tc * 4) != cudaSuccess ||
          cudaMalloc(&h.tie_pos, tc * 4) != cudaSuccess || cudaMalloc(&h.run_off, rc * 4) != cudaSuccess ||
          cudaMalloc(&h.run_lo, rc * 4) != cudaSuccess) {
        cudaGetLastError();
        return abi_fail(&ctx, EHGP_ERR_OUT_OF_MEMORY, "the facade tie runs do not fit the device");
      }
      h.tie_cap = tc;
      h.run_cap = rc;
    }
    // members' records are copied (ev_raw is free between the facade gather and the level
    // classes) so that the sort writes the facade in place
    cudaMemcpyAsync(h.tie_pos, idx.data(), (uint64_t)cnt * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(h.run_off, run_off.data(), (uint64_t)(nruns + 1) * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(h.run_lo, run_lo.data(), (uint64_t)nruns * 4, cudaMemcpyHostToDevice, st);
    k_run_gather<<<nblk(cnt, kT), kT, 0, st>>>(cnt, h.tie_pos, h.ev, h.ev_raw);
    const Cloud dc{b.px, b.py, b.pz, h.S};
    k_tie_keys<<<nblk(cnt, 128), 128, 0, st>>>(cnt, h.tie_pos, h.ev, dc, h.tie_num, h.tie_a2);
    k_tie_sort<<<nblk(nruns, 64), 64, 0, st>>>(nruns, h.run_off, h.run_lo, h.tie_num, h.tie_a2, h.ev_raw, h.tie_idx,
                                               h.tie_tmp, h.ev, h.eqprev);
    launches += 3;
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return abi_cuda_fail(&ctx, e, "facade tie runs");
    ms_ties = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tt0).count();
  }
  // level classes
  if (m) {
    uint32_t* flag = h.order1;  // scratch
    k_level_class<<<nblk(m, kT), kT, 0, st>>>(m, h.eqprev, flag);
    const uint32_t nb = nblk(m, 1024);
    k_sum_blocks<<<nb, 256, 0, st>>>(m, flag, h.lclass, h.ubsum);
    k_sum_carry<<<1, 1, 0, st>>>(nb, h.ubsum);
    k_sum_apply<<<nblk(m, kT), kT, 0, st>>>(m, h.lclass, h.ubsum, 1);
    launches += 4;
  }
  // stable partition by closed rank
  uint32_t hist[16] = {0};
  int rpasses = 0;
  if (m) {
    k_rank_key<<<nblk(m, kT), kT, 0, st>>>(m, h.ev, h.key, h.order0, h.counters + 3);
    const IndirectKey stages[1] = {{h.key, 0}};
    const int bits[1] = {8};
    rpasses = radix_sort_indirect(st, m, h.order0, h.order1, stages, bits, 1, rs, &launches);
    k_rank_gather<<<nblk(m, kT), kT, 0, st>>>(m, h.order0, h.order1, ctx.radix.state, rpasses, h.rank_order);
    launches += 2;
    cudaMemcpyAsync(hist, h.counters + 3, 16 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
  }
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return abi_cuda_fail(&ctx, e, "hierarchy facade");
  if (h.diagnostics) {
    h.decision = EHGP_ERR_DEGENERATE;
    return abi_fail(&ctx, EHGP_ERR_DEGENERATE,
                    "relevant extra-shell diagnostics: the Morse event journal is not built");
  }
  const uint32_t keff = h.keff;
  // rank segments: rb[r] = first position of rank r in rank_order
  uint64_t rb[18] = {0};
  for (int r = 0; r < 16; ++r) rb[r + 1] = rb[r] + hist[r];
  // births (orders 2..keff): handle n + (position - rb[2])
  const uint64_t nb_higher = rb[keff + 1 > 16 ? 16 : keff + 1] - rb[2];
  if (nb_higher) {
    cudaMemsetAsync(h.slots, 0xff, h.cap_slots * sizeof(uint32_t), st);
    k_birth_insert<<<nblk(nb_higher, kT), kT, 0, st>>>((uint32_t)nb_higher, n, (uint32_t)rb[2], h.rank_order, h.ev,
                                                       h.bfac, h.slots, (uint32_t)(h.cap_slots - 1), h.counters + 2);
    ++launches;
  }
  // families: saddle events of ranks 2..keff+1 in rank-partition order; arms per support point
  const uint64_t fam_lo = rb[2], fam_hi = rb[std::min<uint32_t>(keff + 2, 16)];
  const uint64_t nfam = fam_hi - fam_lo;
  uint64_t narms = 0;
  if (m) {
    k_rank_info<<<nblk(m, kT), kT, 0, st>>>(m, h.rank_order, h.ev, h.lclass, h.d_cls_rp, h.d_size_rp);
    ++launches;
  }
  if (nfam) {  // arm offsets: inclusive sum of the family sizes into d_armoff + 1
    const uint32_t nb = nblk(nfam, 1024);
    k_sum_blocks<<<nb, 256, 0, st>>>((uint32_t)nfam, h.d_size_rp + fam_lo, h.d_armoff + 1, h.ubsum);
    k_sum_carry<<<1, 1, 0, st>>>(nb, h.ubsum);
    k_sum_apply<<<nblk(nfam, kT), kT, 0, st>>>((uint32_t)nfam, h.d_armoff + 1, h.ubsum, 0);
    cudaMemsetAsync(h.d_armoff, 0, sizeof(uint32_t), st);
    launches += 3;
    uint32_t na = 0;
    cudaMemcpyAsync(&na, h.d_armoff + nfam, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return abi_cuda_fail(&ctx, e, "arm offsets");
    narms = na;
  }
  if (narms > h.cap_arms) return abi_fail(&ctx, EHGP_ERR_CAPACITY, "strict arms exceed the hierarchy buffers");
  // pinned host views
  if (h.pin_m < m + 1 || h.pin_arms < narms + 1) {
    for (void* p : {(void*)h.p_rank, (void*)h.p_cls, (void*)h.p_armoff, (void*)h.p_term, (void*)h.p_stat})
      if (p) cudaFreeHost(p);
    h.p_rank = h.p_cls = h.p_armoff = h.p_term = nullptr;
    h.p_stat = nullptr;
    const uint64_t pm = (m + 1) + (m + 1) / 8, pa = (narms + 1) + (narms + 1) / 8;
    if (cudaMallocHost(&h.p_rank, pm * 4) != cudaSuccess || cudaMallocHost(&h.p_cls, pm * 4) != cudaSuccess ||
        cudaMallocHost(&h.p_armoff, pm * 4) != cudaSuccess || cudaMallocHost(&h.p_term, pa * 4) != cudaSuccess ||
        cudaMallocHost(&h.p_stat, pa) != cudaSuccess) {
      h.pin_m = h.pin_arms = 0;
      return abi_fail(&ctx, EHGP_ERR_OUT_OF_MEMORY, "pinned host buffers for the hierarchy");
    }
    h.pin_m = pm;
    h.pin_arms = pa;
  }
  const uint32_t* rank_order = h.p_rank;
  const uint32_t* cls_rp = h.p_cls;
  const uint32_t* arm_off = h.p_armoff;
  const uint32_t* term = h.p_term;
  const uint8_t* astat = h.p_stat;
  if (m) {
    cudaMemcpyAsync(h.p_rank, h.rank_order, (uint64_t)m * 4, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(h.p_cls, h.d_cls_rp, (uint64_t)m * 4, cudaMemcpyDeviceToHost, st);
  }
  if (nfam) cudaMemcpyAsync(h.p_armoff, h.d_armoff, (nfam + 1) * 4, cudaMemcpyDeviceToHost, st);
  if (narms) {
    k_arm_expand<<<nblk(nfam, kT), kT, 0, st>>>((uint32_t)nfam, (uint32_t)fam_lo, h.rank_order, h.ev, h.d_armoff,
                                               h.arm_family, h.arm_local, h.d_removed);
    ++launches;
  }
  // the facade, rank partition, births and arm seeds are complete: the descent runs order
  // by order below, overlapped with the host forest pass
  uint32_t herr = 0;
  cudaMemcpyAsync(&herr, h.counters + 2, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return abi_cuda_fail(&ctx, e, "strict-arm seeds");
  if (herr) return abi_fail(&ctx, EHGP_ERR_CAPACITY, "the birth facet table is full");
  if (narms) {
    if (!h.qcount && (e = halloc(h, &h.qcount, 4)) != cudaSuccess)
      return abi_fail(&ctx, EHGP_ERR_OUT_OF_MEMORY, "descent queue");
    if (h.q_cap < narms) {  // worst case: every arm misses
      for (void* p : {(void*)h.q_arm[0], (void*)h.q_arm[1], (void*)h.q_fac[0], (void*)h.q_fac[1]})
        if (p) cudaFree(p);
      h.q_arm[0] = h.q_arm[1] = h.q_fac[0] = h.q_fac[1] = nullptr;
      const uint64_t qc = narms + narms / 8 + 1024;
      if (cudaMalloc(&h.q_arm[0], qc * 4) != cudaSuccess || cudaMalloc(&h.q_arm[1], qc * 4) != cudaSuccess ||
          cudaMalloc(&h.q_fac[0], qc * 4 * kMaxFacet) != cudaSuccess ||
          cudaMalloc(&h.q_fac[1], qc * 4 * kMaxFacet) != cudaSuccess)
        return abi_fail(&ctx, EHGP_ERR_OUT_OF_MEMORY, "descent queue buffers do not fit the device");
      h.q_cap = qc;
    }
  }
  h.arms = narms;
  h.exact_boundaries = unc;
  // ---- host: journal, seeds and the forest journal ------------------------------------
  // Orders are independent (their handles, components and nodes never meet), so each
  // order runs on its own host thread with local indices; records take the global offsets
  // the reference's single pass would give when they are copied out.
  const auto t1 = std::chrono::steady_clock::now();
  const uint64_t birth_count = n + nb_higher;
  // union-find state packed per birth handle: one cache line touch per arm
  if (!h.dsu.ensure(birth_count * sizeof(HierDsu)))  // each order initialises its own handle range
    return abi_fail(&ctx, EHGP_ERR_OUT_OF_MEMORY, "the union-find array does not fit host memory");
  HierDsu* dsu = static_cast<HierDsu*>(h.dsu.p);
  // per-order arenas and union-find state persist across calls (no page faults when warm)
  if (h.outs.size() < keff + 1) h.outs.resize(keff + 1);
  auto& outs = h.outs;
  for (uint32_t k = 1; k <= keff; ++k) {
    HierOrderOut& o = outs[k];
    o.status = EHGP_OK;
    o.msg = "";
  }
  const auto t_init = std::chrono::steady_clock::now();
  // Each order runs a lean sequential core (union-find over its batches; it writes the arm
  // bindings in place and handles multi-role batches whole) and publishes chunks of
  // single-role batches with the running counters at their start; a shared pool of host
  // threads rebuilds those batches' journal and forest records from the bindings while the
  // cores go on.  Record positions and contents equal those of one sequential pass.
  struct Cnt {
    uint64_t bi, si;
    uint32_t jb, role, birth, sad, grp, node, child, count;
    uint64_t carriers, reduced;
  };
  const uint32_t kChunkBatches = h.chunk_batches;
  constexpr uint32_t kSnapBlock = 4096;
  struct Progress {
    std::vector<std::unique_ptr<Cnt[]>> blocks;  // published chunk starts, kSnapBlock per block
    std::atomic<uint32_t> published{0}, claimed{0}, replayed{0};
    std::atomic<int> done{0}, bad{0};
    // vertical maps from this order (k >= 2): parallel gathers, then one sweep
    std::atomic<uint32_t> va_claimed{0}, va_done{0};
    std::atomic<int> vb_claimed{0}, vb_done{0}, vstat{EHGP_OK};
  };
  std::vector<Progress> prog(keff + 1);
  auto order_range = [&](uint32_t k, uint64_t& b_lo, uint64_t& b_hi, uint64_t& s_lo, uint64_t& s_hi,
                         uint64_t& arm_lo, uint64_t& arm_hi) {
    b_lo = k == 1 ? 0 : rb[k];
    b_hi = k == 1 ? 0 : rb[k + 1];
    s_lo = rb[k + 1];
    s_hi = rb[k + 2 > 16 ? 16 : k + 2];
    arm_lo = s_hi > s_lo ? arm_off[s_lo - fam_lo] : 0;
    arm_hi = s_hi > s_lo ? arm_off[s_hi - fam_lo] : 0;
  };
  // fam_lim[k]: saddle positions below it have their terminal handles on the host (the
  // descent of an order arrives in parts cut at batch boundaries); stop_all ends waits
  std::unique_ptr<std::atomic<uint64_t>[]> fam_lim(new std::atomic<uint64_t>[keff + 1]);
  for (uint32_t k = 0; k <= keff; ++k) fam_lim[k].store(0);
  std::atomic<int> stop_all{0};
  // This order's union-find handles: every one a root, not yet born (done by the order's
  // thread while the device descends its first part).
  auto init_dsu = [&](uint32_t k) {
    const uint64_t h_lo = k == 1 ? 0 : n + (rb[k] - rb[2]), h_hi = k == 1 ? n : n + (rb[k + 1] - rb[2]);
    for (uint64_t i = h_lo; i < h_hi; ++i) dsu[i] = {(uint32_t)i, kUnborn};
  };
  auto run_core = [&](uint32_t k, HierOrderOut& o) {
    const auto to0 = std::chrono::steady_clock::now();
    Progress& pg = prog[k];
    auto fail_o = [&](const char* m) {
      o.status = EHGP_ERR_DEGENERATE;
      o.msg = m;
    };
    auto find = [&](uint32_t x) {  // path halving; roots follow the least-handle union rule alone
      while (dsu[x].parent != x) {
        dsu[x].parent = dsu[dsu[x].parent].parent;
        x = dsu[x].parent;
      }
      return x;
    };
    uint64_t b_lo, b_hi, s_lo, s_hi, arm_lo, arm_hi;
    order_range(k, b_lo, b_hi, s_lo, s_hi, arm_lo, arm_hi);
    const uint64_t births_k = k == 1 ? n : b_hi - b_lo, fams_k = s_hi - s_lo, arms_k = arm_hi - arm_lo;
    const uint64_t h_lo = k == 1 ? 0 : n + (rb[k] - rb[2]), h_hi = h_lo + births_k;  // this order's handles
    // capacities are upper bounds (one batch holds at least one role; a group at least one
    // saddle; a multifusion's children are distinct prior roots of its arms' carriers)
    o.jb.reset(births_k + fams_k);
    o.fb.reset(births_k + fams_k);
    o.roles.reset(births_k + fams_k);
    o.fam.reset(fams_k);
    o.saddles.reset(fams_k);
    o.groups.reset(fams_k);
    o.births.reset(births_k);
    o.bindings.reset(arms_k);
    o.nodes.reset((k == 1 ? n : 0) + fams_k);
    o.children.reset(arms_k);
    o.roots.reset(births_k);
    o.node_cls.reset((k == 1 ? n : 0) + fams_k);
    o.fam_res.reset(fams_k);
    // this order's union-find handles
    pg.blocks.clear();
    // chunks <= batches / kChunkBatches + multi-role batches + 1 <= batches + 1
    pg.blocks.resize((births_k + fams_k + 1) / kSnapBlock + 2);
    Cnt c{b_lo, s_lo, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    uint32_t nchunk = 0;
    Cnt open = c;  // start of the chunk being filled
    auto close_chunk = [&] {
      if (open.count == 0) return;
      const uint32_t blk = nchunk / kSnapBlock;
      if (!pg.blocks[blk]) pg.blocks[blk].reset(new Cnt[kSnapBlock]);
      pg.blocks[blk][nchunk % kSnapBlock] = open;
      ++nchunk;
      stream_fence();  // the chunk's bindings
      pg.published.store(nchunk, std::memory_order_release);
    };
    auto reopen = [&] {
      open = c;
      open.count = 0;
    };
    struct Role {
      uint32_t proj, role, fi, pos;
    };
    struct Arm {
      uint32_t seed, carrier, prior;
    };
    struct Plan {
      uint32_t c_off, c_cnt, p_off, p_cnt, s_off, s_cnt, kind, created, result;
    };
    std::vector<Role> batch_roles;
    std::vector<uint32_t> fam_pos, fam_local, arm_b_off, cars, qp, plan_of, plan_car, plan_prior, plan_sad, tmp,
        new_births;
    std::vector<Arm> arms_b;
    std::vector<Plan> plans;
    std::vector<ehgp_forest_node> gnodes;
    uint64_t& bi = c.bi;
    uint64_t& si = c.si;
    uint64_t& carriers = c.carriers;
    uint64_t& reduced = c.reduced;
    bool singles = k == 1;
    uint64_t lim = 0;  // saddle positions below lim have their terminal handles
    auto core = [&]() {
      while (singles || bi < b_hi || si < s_hi) {
        uint32_t cls = kInvalid32, lev = kInvalid32;
        if (!singles) {
          const uint32_t cls_b = bi < b_hi ? cls_rp[bi] : kInvalid32;
          const uint32_t cls_s = si < s_hi ? cls_rp[si] : kInvalid32;
          if (cls_s <= cls_b && si >= lim) {  // the batch holds saddles: wait for their part of the descent
            while ((lim = fam_lim[k].load(std::memory_order_acquire)) <= si) {
              if (stop_all.load(std::memory_order_acquire)) {
                fail_o("the strict-arm descent stopped");
                return;
              }
              std::this_thread::sleep_for(std::chrono::microseconds(20));
            }
          }
          cls = std::min(cls_b, cls_s);
          lev = cls_b <= cls_s ? rank_order[bi] : rank_order[si];
          // single-role batches (almost every batch off ties): union-find only here
          const bool one_b = cls_b == cls && !(bi + 1 < b_hi && cls_rp[bi + 1] == cls) && cls_s != cls;
          const bool one_s = cls_s == cls && !(si + 1 < s_hi && cls_rp[si + 1] == cls) && cls_b != cls;
          if (one_b) {
            const uint32_t handle = n + (uint32_t)(bi - rb[2]);
            dsu[handle].rroot = kInvalid32;
            ++carriers;
            ++c.jb; ++c.role; ++c.birth;
            ++bi;
            if (++open.count == kChunkBatches) { close_chunk(); reopen(); }
            continue;
          }
          if (one_s) {
            const uint32_t pos = (uint32_t)(si - fam_lo), fidx = (uint32_t)(si - s_lo);
            const uint32_t a0 = arm_off[pos], a1 = arm_off[pos + 1];
            uint32_t dc[4], pr[4];
            int ndc = 0, np = 0;
            for (uint32_t a = a0; a < a1; ++a) {
              // two-stage prefetch: the arm's record 64 arms ahead, its parent's 32 ahead
              if (a + 64 < arm_hi) __builtin_prefetch(&dsu[term[a + 64] < birth_count ? term[a + 64] : 0]);
              if (a + 32 < arm_hi && term[a + 32] >= h_lo && term[a + 32] < h_hi) __builtin_prefetch(&dsu[dsu[term[a + 32]].parent]);
              if (term[a] < h_lo || term[a] >= h_hi || dsu[term[a]].rroot == kUnborn) {
                fail_o("a strict arm descended to a minimum that is not yet born");
                return;
              }
              const uint32_t c0 = find(term[a]);
              const uint32_t p0 = dsu[c0].rroot;
              nt_store(o.bindings[a - arm_lo], ehgp_forest_binding{a, fidx, c0, p0});
              bool dup = false;
              for (int t = 0; t < ndc; ++t) dup |= dc[t] == c0;
              if (dup) continue;
              int j = ndc++;
              while (j > 0 && dc[j - 1] > c0) { dc[j] = dc[j - 1]; --j; }
              dc[j] = c0;
              if (p0 != kInvalid32) {
                int q = np++;
                while (q > 0 && pr[q - 1] > p0) { pr[q] = pr[q - 1]; --q; }
                pr[q] = p0;
                if ((q > 0 && pr[q - 1] == p0) || (q + 1 < np && pr[q + 1] == p0)) {
                  fail_o("a frozen carrier class repeats a reduced root");
                  return;
                }
              }
            }
            uint32_t result;
            if (np == 1) {
              result = pr[0];
            } else {
              if (np == 0 && k == 1) {
                fail_o("an order-one group has no root");
                return;
              }
              result = c.node++;
              if (np >= 2) c.child += (uint32_t)np;
            }
            // commit: the distinct carriers are pre-batch roots; the least survives
            for (int t = 1; t < ndc; ++t) dsu[dc[t]].parent = dc[0];
            carriers -= (uint64_t)(ndc - 1);
            dsu[dc[0]].rroot = result;
            reduced = reduced - (uint64_t)np + 1;
            ++c.jb; ++c.role; ++c.sad; ++c.grp;
            ++si;
            if (++open.count == kChunkBatches) { close_chunk(); reopen(); }
            continue;
          }
        }
        // a multi-role batch, whole: the arenas' counts follow the core's counters
        close_chunk();
        o.jb.n = c.jb; o.fb.n = c.jb; o.roles.n = c.role; o.fam.n = (uint32_t)(si - s_lo); o.births.n = c.birth;
        o.bindings.n = si < s_hi ? arm_off[si - fam_lo] - arm_lo : arms_k;
        o.saddles.n = c.sad; o.groups.n = c.grp; o.nodes.n = c.node; o.children.n = c.child;
        const uint32_t bidx = (uint32_t)o.jb.size();
        ehgp_journal_batch jb{k, lev, (uint32_t)o.roles.size(), 0, 0, 0};
        ehgp_forest_batch fb{};
        fb.order = k;
        fb.level_event = lev;
        fb.pre_carriers = (uint32_t)carriers;
        fb.pre_roots = (uint32_t)reduced;
        batch_roles.clear();
        if (singles) {
          for (uint32_t p = 0; p < n; ++p) batch_roles.push_back({p, 0, kInvalid32, p});
        } else {
          while (bi < b_hi && cls_rp[bi] == cls) {
            batch_roles.push_back({n + rank_order[bi], 0, rank_order[bi], (uint32_t)(bi - rb[2])});
            ++bi;
          }
          const size_t nbr = batch_roles.size();
          while (si < s_hi && cls_rp[si] == cls) {
            batch_roles.push_back({n + rank_order[si], 1, rank_order[si], (uint32_t)(si - fam_lo)});
            ++si;
          }
          if (nbr && nbr < batch_roles.size())
            std::inplace_merge(batch_roles.begin(), batch_roles.begin() + nbr, batch_roles.end(),
                               [](const Role& x, const Role& y) { return x.proj < y.proj; });
        }
        singles = false;
        // journal roles and saddle families
        fam_pos.clear();
        fam_local.clear();
        for (size_t q = 0; q < batch_roles.size(); ++q) {
          const Role& r = batch_roles[q];
          const uint32_t ridx = (uint32_t)o.roles.size();
          o.roles.push_back({bidx, r.proj, r.role});
          if (r.role == 0) {
            ++jb.birth_roles;
            continue;
          }
          ++jb.saddle_roles;
          // arm seeds follow the rank partition: the family at position p owns seeds arm_off[p]..
          fam_local.push_back((uint32_t)o.fam.size());
          o.fam.push_back({r.fi, r.proj, ridx, bidx, k, arm_off[r.pos], arm_off[r.pos + 1] - arm_off[r.pos]});
          fam_pos.push_back(r.pos);
        }
        jb.role_count = (uint32_t)batch_roles.size();
        o.jb.push_back(jb);
        // arms resolved against the pre-batch components
        arms_b.clear();
        arm_b_off.clear();
        for (uint32_t q = 0; q < fam_pos.size(); ++q) {
          const uint32_t fpos = fam_pos[q];
          arm_b_off.push_back((uint32_t)arms_b.size());
          for (uint64_t a = arm_off[fpos]; a < arm_off[fpos + 1]; ++a) {
            // two-stage prefetch: the arm's record 64 arms ahead, its parent's 32 ahead
            if (a + 64 < arm_hi) __builtin_prefetch(&dsu[term[a + 64] < birth_count ? term[a + 64] : 0]);
            if (a + 32 < arm_hi && term[a + 32] >= h_lo && term[a + 32] < h_hi) __builtin_prefetch(&dsu[dsu[term[a + 32]].parent]);
            if (term[a] < h_lo || term[a] >= h_hi || dsu[term[a]].rroot == kUnborn) {
              fail_o("a strict arm descended to a minimum that is not yet born");
              return;
            }
            const uint32_t c0 = find(term[a]);
            arms_b.push_back({(uint32_t)a, c0, dsu[c0].rroot});
          }
        }
        arm_b_off.push_back((uint32_t)arms_b.size());
        // frozen-root quotient: transitive carrier classes, ordered by least carrier
        plans.clear();
        plan_car.clear();
        plan_prior.clear();
        plan_sad.clear();
        if (!fam_pos.empty()) {
          cars.clear();
          for (const Arm& a : arms_b) cars.push_back(a.carrier);
          std::sort(cars.begin(), cars.end());
          cars.erase(std::unique(cars.begin(), cars.end()), cars.end());
          const uint32_t nc = (uint32_t)cars.size();
          auto qi = [&](uint32_t x) { return (uint32_t)(std::lower_bound(cars.begin(), cars.end(), x) - cars.begin()); };
          qp.resize(nc);
          std::iota(qp.begin(), qp.end(), 0u);
          auto qf = [&](uint32_t x) {
            while (qp[x] != x) x = qp[x] = qp[qp[x]];
            return x;
          };
          for (uint32_t q = 0; q + 1 < arm_b_off.size(); ++q) {
            const uint32_t a0 = qf(qi(arms_b[arm_b_off[q]].carrier));
            for (uint32_t a = arm_b_off[q] + 1; a < arm_b_off[q + 1]; ++a) {
              const uint32_t x = qf(a0), y = qf(qi(arms_b[a].carrier));
              if (x != y) qp[std::max(x, y)] = std::min(x, y);
            }
          }
          plan_of.assign(nc, kInvalid32);
          for (uint32_t i = 0; i < nc; ++i) {
            const uint32_t r0 = qf(i);
            if (plan_of[r0] == kInvalid32) {
              plan_of[r0] = (uint32_t)plans.size();
              plans.push_back({0, 0, 0, 0, 0, 0, 0, kInvalid32, 0});
            }
          }
          for (uint32_t i = 0; i < nc; ++i) {
            Plan& p = plans[plan_of[qf(i)]];
            ++p.c_cnt;
            if (dsu[cars[i]].rroot != kInvalid32) ++p.p_cnt;
          }
          for (uint32_t q = 0; q + 1 < arm_b_off.size(); ++q) ++plans[plan_of[qf(qi(arms_b[arm_b_off[q]].carrier))]].s_cnt;
          uint32_t co = 0, po = 0, so = 0;
          for (Plan& p : plans) {
            p.c_off = co; p.p_off = po; p.s_off = so;
            co += p.c_cnt; po += p.p_cnt; so += p.s_cnt;
            p.c_cnt = p.p_cnt = p.s_cnt = 0;
          }
          plan_car.resize(co);
          plan_prior.resize(po);
          plan_sad.resize(so);
          for (uint32_t i = 0; i < nc; ++i) {
            Plan& p = plans[plan_of[qf(i)]];
            plan_car[p.c_off + p.c_cnt++] = cars[i];
            if (dsu[cars[i]].rroot != kInvalid32) plan_prior[p.p_off + p.p_cnt++] = dsu[cars[i]].rroot;
          }
          for (uint32_t q = 0; q + 1 < arm_b_off.size(); ++q) {
            Plan& p = plans[plan_of[qf(qi(arms_b[arm_b_off[q]].carrier))]];
            plan_sad[p.s_off + p.s_cnt++] = q;
          }
          uint32_t pending = 0;
          for (Plan& p : plans) {
            uint32_t* pr = plan_prior.data() + p.p_off;
            std::sort(pr, pr + p.p_cnt);
            if (std::adjacent_find(pr, pr + p.p_cnt) != pr + p.p_cnt) {
              fail_o("a frozen carrier class repeats a reduced root");
              return;
            }
            if (p.p_cnt == 1) {
              p.kind = 1;
              p.created = kInvalid32;
              p.result = pr[0];
            } else {
              if (p.p_cnt == 0 && k == 1) {
                fail_o("an order-one group has no root");
                return;
              }
              p.kind = p.p_cnt == 0 ? 0 : 2;
              p.created = (uint32_t)o.nodes.size() + pending++;
              p.result = p.created;
            }
          }
        }
        fb.saddle_offset = (uint32_t)o.saddles.size();
        fb.group_offset = (uint32_t)o.groups.size();
        gnodes.clear();
        for (const Plan& p : plans) {
          const uint32_t g_soff = (uint32_t)o.saddles.size();
          const uint32_t gidx = (uint32_t)o.groups.size();
          for (uint32_t t = 0; t < p.s_cnt; ++t) {
            const uint32_t q = plan_sad[p.s_off + t];
            const uint32_t fidx = fam_local[q];
            const uint32_t arm_o = (uint32_t)o.bindings.size();
            tmp.clear();
            uint32_t nprior = 0;
            for (uint32_t a = arm_b_off[q]; a < arm_b_off[q + 1]; ++a) {
              const Arm& am = arms_b[a];
              o.bindings.push_back({am.seed, fidx, am.carrier, am.prior});
              tmp.push_back(am.carrier);
            }
            std::sort(tmp.begin(), tmp.end());
            tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
            for (uint32_t c0 : tmp) nprior += dsu[c0].rroot != kInvalid32;  // carriers are pre-batch roots
            o.saddles.push_back({fidx, o.fam[fidx].event, bidx, arm_o, arm_b_off[q + 1] - arm_b_off[q],
                                 (uint32_t)tmp.size(), (uint32_t)tmp.size() - nprior, nprior, gidx});
          }
          const uint32_t ccnt = p.kind == 2 ? p.p_cnt : 0u;
          o.groups.push_back({bidx, g_soff, (uint32_t)o.saddles.size() - g_soff, p.c_cnt, p.c_cnt - p.p_cnt, p.p_cnt,
                              (uint32_t)o.children.size(), ccnt, p.created, p.result, p.kind});
          if (p.kind != 1)
            gnodes.push_back({k, lev, p.kind == 0 ? 1u : 2u, (uint32_t)o.children.size(), ccnt, kInvalid32, gidx});
          if (p.kind == 2)
            o.children.append(plan_prior.begin() + p.p_off, plan_prior.begin() + p.p_off + p.p_cnt);
        }
        o.nodes.append(gnodes.begin(), gnodes.end());
        // births of this batch (hidden from this batch's arms); handles are global
        fb.birth_offset = (uint32_t)o.births.size();
        new_births.clear();
        for (const Role& r : batch_roles) {
          if (r.role != 0) continue;
          const uint32_t handle = k == 1 ? r.proj : n + r.pos;
          uint32_t node = kInvalid32;
          if (k == 1) {
            node = (uint32_t)o.nodes.size();
            o.nodes.push_back({1, kInvalid32, 0, (uint32_t)o.children.size(), 0, handle, kInvalid32});
          }
          o.births.push_back({r.proj, bidx, k, handle, node});
          new_births.push_back(handle);
        }
        // commit: unions (least handle survives), reduced roots, then births
        for (const Plan& p : plans) {
          uint32_t r0 = find(plan_car[p.c_off]);
          uint32_t had_reduced = dsu[r0].rroot != kInvalid32;
          for (uint32_t i = 1; i < p.c_cnt; ++i) {
            const uint32_t r1 = find(plan_car[p.c_off + i]);
            if (r1 == r0) continue;
            had_reduced += dsu[r1].rroot != kInvalid32;
            const uint32_t lo = std::min(r0, r1), hi = std::max(r0, r1);
            dsu[hi].parent = lo;
            r0 = lo;
            --carriers;
          }
          dsu[r0].rroot = p.result;
          reduced = reduced - had_reduced + 1;
        }
        for (size_t t = 0; t < new_births.size(); ++t) {
          const uint32_t hnd = new_births[t];
          dsu[hnd].rroot = k == 1 ? o.births[fb.birth_offset + t].order_one_node : kInvalid32;
          ++carriers;
          if (k == 1) ++reduced;
        }
        fb.birth_count = (uint32_t)new_births.size();
        fb.saddle_count = (uint32_t)o.saddles.size() - fb.saddle_offset;
        fb.group_count = (uint32_t)o.groups.size() - fb.group_offset;
        fb.post_carriers = (uint32_t)carriers;
        fb.post_roots = (uint32_t)reduced;
        o.fb.push_back(fb);
        for (uint64_t i = c.node; i < o.nodes.n && i < o.nodes.cap; ++i)
          o.node_cls[i] = o.nodes[i].level_event == kInvalid32 ? kInvalid32 : cls;
        for (uint64_t sd = c.sad; sd < o.saddles.n && sd < o.saddles.cap; ++sd)
          o.fam_res[o.saddles[sd].family] = o.groups[o.saddles[sd].group].result_node;
        c.jb = (uint32_t)o.jb.n; c.role = (uint32_t)o.roles.n; c.birth = (uint32_t)o.births.n;
        c.sad = (uint32_t)o.saddles.n; c.grp = (uint32_t)o.groups.n; c.node = (uint32_t)o.nodes.n;
        c.child = (uint32_t)o.children.n;
        reopen();
      }
    };
    core();
    if (o.status == EHGP_OK) {
      close_chunk();
      o.jb.n = c.jb; o.fb.n = c.jb; o.roles.n = c.role; o.fam.n = fams_k; o.births.n = c.birth; o.bindings.n = arms_k;
      o.saddles.n = c.sad; o.groups.n = c.grp; o.nodes.n = c.node; o.children.n = c.child;
      if (!o.jb.fits() || !o.roles.fits() || !o.nodes.fits() || !o.children.fits() || !o.groups.fits() ||
          !o.saddles.fits() || !o.births.fits() || !o.fb.fits() || !o.fam.fits() || !o.bindings.fits())
        fail_o("internal: a forest arena bound was exceeded");
    }
    if (o.status == EHGP_OK) {
      // final roots of this order (local node ids)
      for (uint64_t hnd = h_lo; hnd < h_hi; ++hnd)
        if (dsu[hnd].parent == hnd && dsu[hnd].rroot != kInvalid32 && dsu[hnd].rroot != kUnborn)
          o.roots.push_back({k, (uint32_t)hnd, dsu[hnd].rroot});
      std::sort(o.roots.begin(), o.roots.end(),
                [](const ehgp_forest_root& x, const ehgp_forest_root& y) { return x.node < y.node; });
    }
    o.v_res.reset(o.nodes.n);
    o.v_cls.reset(o.nodes.n);
    o.ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - to0).count();
    stream_fence();
    pg.done.store(1, std::memory_order_release);
  };
  // Rebuilds the records of one published chunk of single-role batches.
  auto replay = [&](uint32_t k, uint32_t j) {
    HierOrderOut& o = outs[k];
    Progress& pg = prog[k];
    Cnt c = pg.blocks[j / kSnapBlock][j % kSnapBlock];
    uint64_t b_lo, b_hi, s_lo, s_hi, arm_lo, arm_hi;
    order_range(k, b_lo, b_hi, s_lo, s_hi, arm_lo, arm_hi);
    (void)b_lo;
    (void)arm_hi;
    for (uint32_t t = 0; t < c.count; ++t) {
      const uint32_t cls_b = c.bi < b_hi ? cls_rp[c.bi] : kInvalid32;
      const uint32_t cls_s = c.si < s_hi ? cls_rp[c.si] : kInvalid32;
      const uint32_t cls = std::min(cls_b, cls_s);
      const uint32_t lev = cls_b <= cls_s ? rank_order[c.bi] : rank_order[c.si];
      const bool one_b = cls_b == cls && !(c.bi + 1 < b_hi && cls_rp[c.bi + 1] == cls) && cls_s != cls;
      const bool one_s = cls_s == cls && !(c.si + 1 < s_hi && cls_rp[c.si + 1] == cls) && cls_b != cls;
      const uint32_t bidx = c.jb;
      if (one_b) {
        const uint32_t pos = (uint32_t)(c.bi - rb[2]), fi = rank_order[c.bi];
        nt_store(o.jb[bidx], ehgp_journal_batch{k, lev, c.role, 1, 1, 0});
        nt_store(o.roles[c.role], ehgp_role_record{bidx, n + fi, 0});
        nt_store(o.births[c.birth], ehgp_forest_birth{n + fi, bidx, k, n + pos, kInvalid32});
        nt_store(o.fb[bidx], ehgp_forest_batch{k, lev, c.birth, 1, c.sad, 0, c.grp, 0, (uint32_t)c.carriers,
                                               (uint32_t)c.reduced, (uint32_t)(c.carriers + 1), (uint32_t)c.reduced});
        ++c.carriers;
        ++c.jb; ++c.role; ++c.birth;
        ++c.bi;
        continue;
      }
      if (!one_s) {
        pg.bad.store(1);
        return;
      }
      const uint32_t pos = (uint32_t)(c.si - fam_lo), fi = rank_order[c.si], fidx = (uint32_t)(c.si - s_lo);
      const uint32_t a0 = arm_off[pos], a1 = arm_off[pos + 1];
      const uint32_t ridx = c.role;
      nt_store(o.jb[bidx], ehgp_journal_batch{k, lev, ridx, 1, 0, 1});
      nt_store(o.roles[ridx], ehgp_role_record{bidx, n + fi, 1});
      nt_store(o.fam[fidx], ehgp_family_record{fi, n + fi, ridx, bidx, k, a0, a1 - a0});
      uint32_t dc[4], pr[4];
      int ndc = 0, np = 0;
      for (uint32_t a = a0; a < a1; ++a) {
        const ehgp_forest_binding& bd = o.bindings[a - arm_lo];
        bool dup = false;
        for (int q = 0; q < ndc; ++q) dup |= dc[q] == bd.carrier;
        if (dup) continue;
        dc[ndc++] = bd.carrier;
        if (bd.prior_root != kInvalid32) {
          int q = np++;
          while (q > 0 && pr[q - 1] > bd.prior_root) { pr[q] = pr[q - 1]; --q; }
          pr[q] = bd.prior_root;
        }
      }
      const uint32_t kind = np == 1 ? 1u : np == 0 ? 0u : 2u;
      const uint32_t created = kind == 1 ? kInvalid32 : c.node;
      const uint32_t result = kind == 1 ? pr[0] : created;
      const uint32_t ccnt = kind == 2 ? (uint32_t)np : 0u;
      nt_store(o.saddles[c.sad], ehgp_forest_saddle{fidx, fi, bidx, a0 - (uint32_t)arm_lo, a1 - a0, (uint32_t)ndc,
                                                    (uint32_t)(ndc - np), (uint32_t)np, c.grp});
      nt_store(o.groups[c.grp], ehgp_forest_group{bidx, c.sad, 1, (uint32_t)ndc, (uint32_t)(ndc - np), (uint32_t)np,
                                                  c.child, ccnt, created, result, kind});
      o.fam_res[fidx] = result;
      if (kind != 1) {
        o.node_cls[c.node] = cls;
        o.nodes[c.node++] = {k, lev, kind == 0 ? 1u : 2u, c.child, ccnt, kInvalid32, c.grp};
      }
      for (uint32_t q = 0; q < ccnt; ++q) o.children[c.child + q] = pr[q];
      c.child += ccnt;
      nt_store(o.fb[bidx], ehgp_forest_batch{k, lev, c.birth, 0, c.sad, 1, c.grp, 1, (uint32_t)c.carriers,
                                             (uint32_t)c.reduced, (uint32_t)(c.carriers - (uint64_t)(ndc - 1)),
                                             (uint32_t)(c.reduced - (uint64_t)np + 1)});
      c.carriers -= (uint64_t)(ndc - 1);
      c.reduced = c.reduced - (uint64_t)np + 1;
      ++c.jb; ++c.role; ++c.sad; ++c.grp;
      ++c.si;
    }
  };
  // ---- vertical maps: each reduced node of order k >= 2 at level a maps, on the closed
  // cut at a, to the root of order k - 1 whose component contains it.  A carrier birth of
  // the node's group is an event of rank k; that event is a saddle of order k - 1, whose
  // group's resulting root (level <= a) is climbed through multifusion parents of level <= a
  // (the contract serializer's assignment, reference/morsehgp3d_oracle/serialization.py:1040-1099).
  // They run in the same pool as soon as orders k and k - 1 are complete: chunks of source
  // nodes gather their targets in parallel, then one offline sweep per order climbs them
  // (node ids grow with level in both forests, so the target forest's parent links are
  // united in id order as the source levels rise; the image is one find with path compression).
  constexpr uint32_t kVChunk = 1u << 15;
  if (h.vert.size() < keff + 1) h.vert.resize(keff + 1);
  auto vcls = [](const HierOrderOut& o, uint32_t node) -> int64_t {
    const uint32_t c = o.node_cls[node];
    return c == kInvalid32 ? -1 : (int64_t)c;
  };
  auto complete = [&](uint32_t k) {
    Progress& pg = prog[k];
    return pg.done.load(std::memory_order_acquire) &&
           pg.replayed.load(std::memory_order_acquire) == pg.published.load(std::memory_order_acquire);
  };
  auto v_gather = [&](uint32_t k, uint32_t chunk) {
    HierOrderOut& src = outs[k];
    const HierOrderOut& tgt = outs[k - 1];
    const uint64_t h_lo = n + (rb[k] - rb[2]);  // first birth handle of order k
    const uint64_t i_hi = std::min<uint64_t>(src.nodes.size(), (uint64_t)(chunk + 1) * kVChunk);
    for (uint64_t i = (uint64_t)chunk * kVChunk; i < i_hi; ++i) {
      const ehgp_forest_node& nd = src.nodes[i];
      const ehgp_forest_group& g = src.groups[nd.atomic_group];
      const uint64_t carrier = src.bindings[src.saddles[g.saddle_offset].arm_offset].carrier;
      // the carrier's birth (rank k) and its saddle family of order k - 1 share the rank
      // segment position, so the family's local index is carrier - h_lo
      const uint64_t f = carrier - h_lo;
      if (carrier < h_lo || f >= tgt.fam.size()) {
        prog[k].vstat.store(EHGP_ERR_DEGENERATE);
        src.v_res[i] = kInvalid32;
        continue;
      }
      src.v_res[i] = tgt.fam_res[f];
      src.v_cls[i] = src.node_cls[i];
    }
  };
  auto v_sweep = [&](uint32_t k) {
    const HierOrderOut& src = outs[k];
    const HierOrderOut& tgt = outs[k - 1];
    std::vector<ehgp_vertical_assignment>& vo = h.vert[k];
    vo.clear();
    if (prog[k].vstat.load() != EHGP_OK) return;
    const uint32_t t_n = (uint32_t)tgt.nodes.size();
    std::vector<uint32_t> up(t_n);
    std::iota(up.begin(), up.end(), 0u);
    auto find_up = [&](uint32_t x) {
      while (up[x] != x) {
        up[x] = up[up[x]];
        x = up[x];
      }
      return x;
    };
    uint32_t sweep = 0;  // next target node whose child links are not yet united
    for (uint64_t i = 0; i < src.nodes.size(); ++i) {
      const uint32_t R = src.v_res[i];
      const int64_t lev = vcls(src, (uint32_t)i);
      if (R >= t_n || vcls(tgt, R) > lev) {
        prog[k].vstat.store(EHGP_ERR_DEGENERATE);
        return;
      }
      while (sweep < t_n && vcls(tgt, sweep) <= lev) {
        const ehgp_forest_node& p = tgt.nodes[sweep];
        if (p.kind == 2)
          for (uint32_t c = 0; c < p.child_count; ++c) up[find_up(tgt.children[p.child_offset + c])] = sweep;
        ++sweep;
      }
      vo.push_back({(uint32_t)i, find_up(R), k, src.nodes[i].level_event});  // local ids; offsets at copy-out
    }
  };
  // One step of vertical work (a gather chunk or a sweep) if one is ready; `pending` is
  // cleared while some vertical map is unfinished.
  auto vertical_step = [&](bool& pending) {
    for (uint32_t k = keff; k >= 2; --k) {
      Progress& pg = prog[k];
      if (pg.vb_done.load(std::memory_order_acquire)) continue;
      pending = false;
      if (!complete(k) || !complete(k - 1)) continue;
      if (outs[k].status != EHGP_OK || outs[k - 1].status != EHGP_OK || prog[k].bad.load() || prog[k - 1].bad.load()) {
        int z = 0;
        if (pg.vb_claimed.compare_exchange_strong(z, 1)) pg.vb_done.store(1, std::memory_order_release);
        continue;
      }
      const uint32_t na = (uint32_t)((outs[k].nodes.size() + kVChunk - 1) / kVChunk);
      uint32_t c = pg.va_claimed.load(std::memory_order_relaxed);
      while (c < na) {
        if (pg.va_claimed.compare_exchange_weak(c, c + 1)) {
          v_gather(k, c);
          pg.va_done.fetch_add(1, std::memory_order_acq_rel);
          return true;
        }
      }
      if (pg.va_done.load(std::memory_order_acquire) == na) {
        int z = 0;
        if (pg.vb_claimed.compare_exchange_strong(z, 1)) {
          v_sweep(k);
          pg.vb_done.store(1, std::memory_order_release);
          return true;
        }
      }
    }
    return false;
  };
  // claims and replays published chunks, highest order first, then the vertical maps, until
  // every core is done and every chunk and map is finished
  auto work = [&] {
    uint32_t idle = 0;  // idle rounds: a short spin, then 50 us sleeps (the cores need the CPUs)
    for (;;) {
      bool did = false, all = true;
      for (uint32_t k = keff; k >= 1; --k) {
        Progress& pg = prog[k];
        const int done = pg.done.load(std::memory_order_acquire);
        const uint32_t pub = pg.published.load(std::memory_order_acquire);
        uint32_t cl = pg.claimed.load(std::memory_order_relaxed);
        while (cl < pub) {
          if (pg.claimed.compare_exchange_weak(cl, cl + 1)) {
            replay(k, cl);  // published chunks are complete even when the core stops later
            stream_fence();
            pg.replayed.fetch_add(1, std::memory_order_acq_rel);
            did = true;
            break;
          }
        }
        if (!done || pg.claimed.load(std::memory_order_relaxed) < pg.published.load(std::memory_order_acquire))
          all = false;
        if (did) break;
      }
      if (!did && vertical_step(all)) did = true;
      if (did) {
        idle = 0;
        continue;
      }
      if (all) return;
      if (++idle < 64) std::this_thread::yield();
      else std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
  };
  // The strict-arm descent runs order by order, highest first, on this thread; an order's
  // union-find core starts as soon as its terminal handles are on the host, while the
  // device descends the lower orders.  ready[k]: 0 waiting, 1 go, 2 stopped.
  std::unique_ptr<std::atomic<int>[]> ready(new std::atomic<int>[keff + 1]);
  for (uint32_t k = 0; k <= keff; ++k) ready[k].store(0);
  int dstatus = EHGP_OK;
  const char* dmsg = "";
  cudaError_t dcuda = cudaSuccess;
  {
    const uint32_t hw = h.pool_threads ? h.pool_threads : std::max(1u, std::thread::hardware_concurrency());
    const uint32_t extra = hw > keff + 1 ? std::min(hw - keff - 1, 32u) : 0u;  // one CPU for this thread
    std::vector<std::thread> pool;
    for (uint32_t k = 1; k <= keff; ++k)
      pool.emplace_back([&, k] {
        init_dsu(k);
        int r;
        while ((r = ready[k].load(std::memory_order_acquire)) == 0) std::this_thread::sleep_for(std::chrono::microseconds(20));
        if (r == 1) {
          run_core(k, outs[k]);
        } else {
          outs[k].status = EHGP_ERR_DEGENERATE;
          outs[k].msg = "the strict-arm descent stopped";
          prog[k].done.store(1, std::memory_order_release);
        }
        work();
      });
    for (uint32_t i = 0; i < extra; ++i) pool.emplace_back(work);
    // descent, order by order; the host thread sleeps in its waits (the cores need the CPUs)
    if (!h.ev_block && cudaEventCreateWithFlags(&h.ev_block, cudaEventBlockingSync | cudaEventDisableTiming) != cudaSuccess)
      h.ev_block = nullptr;
    auto wait_stream = [&]() -> cudaError_t {
      if (!h.ev_block) return cudaStreamSynchronize(st);
      cudaError_t r = cudaEventRecord(h.ev_block, st);
      return r == cudaSuccess ? cudaEventSynchronize(h.ev_block) : r;
    };
    const DescentParams dp{n, 2 * n - 2, g.tnodes, b.px, b.py, b.pz, h.S, h.slots, (uint32_t)(h.cap_slots - 1), h.bfac,
                           (uint32_t)nb_higher};
    uint32_t misses = 0, max_rounds = 0;
    unsigned long long failed_before = 0;
    h.descent_steps = 0;
    h.ms_steps = 0;
    h.step_launches = 0;
    for (cudaEvent_t& ev : h.ev_step)
      if (!ev && cudaEventCreate(&ev) != cudaSuccess) ev = nullptr;
    cudaEventRecord(ctx.evk0, st);
    uint32_t k = keff;
    auto stop = [&](int status, const char* msg) {
      dstatus = status;
      dmsg = msg;
    };
    const uint32_t kPartArms = h.part_arms;  // arms per part of an order's descent (about)
    std::vector<uint64_t> plo(keff + 1);
    for (uint32_t j = 1; j <= keff; ++j) plo[j] = rb[j + 1];
    // Descends the next part of order k (cut at a batch boundary after about kPartArms arms)
    // and publishes it to the order's core; false on a failure.
    auto part = [&](uint32_t k) -> bool {
      const uint64_t s_hi = rb[k + 2 > 16 ? 16 : k + 2];
      uint64_t& p_lo = plo[k];
      // the part ends at a batch boundary after about kPartArms arms
      uint64_t p_hi = p_lo;
      {
        uint64_t lo = p_lo, hi = s_hi;  // first position whose arms reach the budget
        const uint64_t goal = (uint64_t)arm_off[p_lo - fam_lo] + kPartArms;
        while (lo < hi) {
          const uint64_t mid = (lo + hi) / 2;
          if ((uint64_t)arm_off[mid + 1 - fam_lo] >= goal) hi = mid; else lo = mid + 1;
        }
        p_hi = std::min<uint64_t>(lo + 1, s_hi);
        while (p_hi < s_hi && cls_rp[p_hi] == cls_rp[p_hi - 1]) ++p_hi;
      }
      const uint32_t a_lo = arm_off[p_lo - fam_lo], a_hi = arm_off[p_hi - fam_lo];
      if (a_hi > a_lo) {
        const uint32_t na = a_hi - a_lo;
        cudaMemsetAsync(h.qcount, 0, 4 * sizeof(uint32_t), st);
        k_arm_probe<<<nblk(na, kT), kT, 0, st>>>(dp, a_lo, na, h.rank_order + fam_lo, h.arm_family, h.arm_local,
                                                 h.ev, h.term, h.arm_status, h.q_arm[0], h.q_fac[0], h.qcount);
        ++launches;
        uint32_t pending = 0;
        cudaMemcpyAsync(&pending, h.qcount, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
        if ((dcuda = wait_stream()) != cudaSuccess) return false;
        misses += pending;
        int cur = 0;
        uint32_t rounds = 0;
        while (pending) {
          if (++rounds > (uint32_t)kDescentSteps) {
            stop(EHGP_ERR_DEGENERATE, "a strict arm descent exceeded its step budget");
            break;
          }
          uint32_t* oc = h.qcount + 1 + (1 - cur);
          cudaMemsetAsync(oc, 0, sizeof(uint32_t), st);
          if (h.ev_step[0]) cudaEventRecord(h.ev_step[0], st);
          int spasses = -1;  // large queues run in Morton order of their facets
          if (pending >= kSortQueueMin && pending <= h.cap_events) {
            k_queue_keys<<<nblk(pending, kT), kT, 0, st>>>(pending, h.q_fac[cur], b.code, h.key, h.order0);
            ++launches;
            spasses = radix_sort_kv(st, pending, h.order0, h.order1, h.key, h.key2, 24, rs, &launches);
          }
          k_arm_step<<<nblk(pending, 128), 128, 0, st>>>(dp, pending, h.q_arm[cur], h.q_fac[cur], ctx.radix.state,
                                                         spasses, h.order0, h.order1, h.q_arm[1 - cur],
                                                         h.q_fac[1 - cur], oc, h.term, h.arm_status, h.dstats);
          if (h.ev_step[1]) cudaEventRecord(h.ev_step[1], st);
          ++launches;
          ++h.step_launches;
          cudaMemcpyAsync(&pending, oc, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
          if ((dcuda = wait_stream()) != cudaSuccess) break;
          if (h.ev_step[0] && h.ev_step[1]) {
            float sm = 0.f;
            if (cudaEventElapsedTime(&sm, h.ev_step[0], h.ev_step[1]) == cudaSuccess) h.ms_steps += sm;
          }
          cur = 1 - cur;
        }
        if (dcuda != cudaSuccess || dstatus != EHGP_OK) return false;
        max_rounds = std::max(max_rounds, rounds);
        unsigned long long dst[4] = {0, 0, 0, 0};
        cudaMemcpyAsync(h.p_term + a_lo, h.term + a_lo, (uint64_t)na * sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(dst, h.dstats, sizeof(dst), cudaMemcpyDeviceToHost, st);
        if ((dcuda = wait_stream()) != cudaSuccess) return false;
        h.descent_steps = dst[0];
        if (dst[3] > failed_before) {  // an arm of this part failed: report the first one
          failed_before = dst[3];
          if ((dcuda = cudaMemcpy(h.p_stat + a_lo, h.arm_status + a_lo, na, cudaMemcpyDeviceToHost)) != cudaSuccess)
            return false;
          static const char* msg[] = {"", "a strict arm descent is unresolved", "a strict arm descent met a plateau",
                                      "a strict arm descent exceeded its ball-query capacity",
                                      "a strict arm descent exceeded its step budget",
                                      "a strict arm descent found no consistent exact miniball or top-k"};
          for (uint32_t a = a_lo; a < a_hi; ++a)
            if (astat[a] != kArmOk) {
              stop(astat[a] == kArmCapacity ? EHGP_ERR_CAPACITY : EHGP_ERR_DEGENERATE,
                   msg[astat[a] < 6 ? astat[a] : 5]);
              break;
            }
          if (dstatus != EHGP_OK) return false;
        }
      }
      fam_lim[k].store(p_hi, std::memory_order_release);
      ready[k].store(1, std::memory_order_release);
      p_lo = p_hi;
      return true;
    };
    // The first parts of the four largest orders first, so that their cores start early; then
    // each order's remaining parts, highest order first.
    bool dok = true;
    for (k = keff; dok && k >= 1 && k + 4 > keff; --k)
      if (plo[k] < rb[k + 2 > 16 ? 16 : k + 2]) dok = part(k);
    for (k = keff; dok && k >= 1; --k) {
      const uint64_t s_hi = rb[k + 2 > 16 ? 16 : k + 2];
      while (dok && plo[k] < s_hi) dok = part(k);
      if (!dok) break;
      fam_lim[k].store(s_hi, std::memory_order_release);
      ready[k].store(1, std::memory_order_release);
    }
    if (dcuda != cudaSuccess || dstatus != EHGP_OK) stop_all.store(1, std::memory_order_release);
    // orders left waiting after a failure stop without running
    for (uint32_t j = 1; j <= keff; ++j) {
      int expect = 0;
      ready[j].compare_exchange_strong(expect, 2);
    }
    cudaEventRecord(ctx.evk1, st);
    cudaMemcpyFromSymbolAsync(h.slow, g_descent_slow, sizeof(h.slow), 0, cudaMemcpyDeviceToHost, st);
    cudaMemcpyFromSymbolAsync(h.visits, g_descent_visits, sizeof(h.visits), 0, cudaMemcpyDeviceToHost, st);
    cudaEventRecord(ctx.ev1, st);
    if (dcuda == cudaSuccess) dcuda = cudaStreamSynchronize(st);
    h.first_misses = misses;
    h.descent_rounds = max_rounds;
    for (auto& t : pool) t.join();
    for (uint32_t j = 1; j <= keff; ++j)
      if (outs[j].status == EHGP_OK && prog[j].bad.load()) {
        outs[j].status = EHGP_ERR_DEGENERATE;
        outs[j].msg = "internal: a forest chunk replay disagrees with its core";
      }
  }
  if (dcuda != cudaSuccess) return abi_cuda_fail(&ctx, dcuda, "strict-arm descent");
  {
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx.ev0, ctx.ev1);
    h.ms_device = ms;
    if (narms) {
      cudaEventElapsedTime(&ms, ctx.evk0, ctx.evk1);
      ctx.kernel_ms = ms;
      h.ms_descent = ms;
    }
  }
  if (dstatus != EHGP_OK) {
    h.decision = (uint32_t)dstatus;
    return abi_fail(&ctx, dstatus, dmsg);
  }
  const auto t_orders = std::chrono::steady_clock::now();
  for (uint32_t k = 1; k <= keff; ++k)
    if (outs[k].status != EHGP_OK) return abi_fail(&ctx, outs[k].status, outs[k].msg);
  h.ms_orders = 0;
  for (uint32_t k = 1; k <= keff; ++k) h.ms_orders = std::max(h.ms_orders, outs[k].ms);
  // global offsets of each order's records (the reference's single pass emits orders in turn)
  std::vector<HierOff> off(keff + 2);
  off[1] = HierOff{0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (uint32_t k = 1; k <= keff; ++k) {
    const HierOrderOut& o = outs[k];
    const HierOff& a = off[k];
    off[k + 1] = {a.jb + (uint32_t)o.jb.size(),         a.role + (uint32_t)o.roles.size(),
                  a.fam + (uint32_t)o.fam.size(),       a.node + (uint32_t)o.nodes.size(),
                  a.child + (uint32_t)o.children.size(), a.birth + (uint32_t)o.births.size(),
                  a.bind + (uint32_t)o.bindings.size(), a.sad + (uint32_t)o.saddles.size(),
                  a.grp + (uint32_t)o.groups.size(),    a.root + (uint32_t)o.roots.size(), 0u};
  }
  const auto t_merge = std::chrono::steady_clock::now();
  {
    uint32_t vtot = 0;
    for (uint32_t k = 1; k <= keff; ++k) {
      if (k >= 2 && prog[k].vstat.load() != EHGP_OK)
        return abi_fail(&ctx, prog[k].vstat.load(), "a reduced node has no lower-order image through its carrier saddle");
      off[k].vert = vtot;
      if (k >= 2) vtot += (uint32_t)h.vert[k].size();
    }
    off[keff + 1].vert = vtot;
  }
  const auto t2 = std::chrono::steady_clock::now();
  h.ms_forest = std::chrono::duration<double, std::milli>(t2 - t1).count();
  {
    using msd = std::chrono::duration<double, std::milli>;
    h.ms_host[0] = ms_ties;
    h.ms_host[1] = msd(t_orders - t_init).count();
    h.ms_host[2] = msd(t_merge - t_orders).count();
    h.ms_host[3] = msd(t2 - t_merge).count();
  }
  (void)t0;
  ctx.last_launches = launches;
  ctx.last_ms = h.ms_device + h.ms_forest;
  h.off = std::move(off);
  h.arm_seeds = narms;
  h.decision = EHGP_OK;
  return EHGP_OK;
}

}  // namespace ehgp

extern "C" {

int ehgp_hierarchy(ehgp_ctx* ctx, uint32_t K, ehgp_hier_counts* counts) {
  if (!ctx) return EHGP_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(ctx->mutex);
  ctx->last_error.clear();
  if (ctx->poisoned) return ehgp::abi_fail(ctx, EHGP_ERR_POISONED, "the context is poisoned by an earlier CUDA failure");
  if (ctx->built_n == 0) return ehgp::abi_fail(ctx, EHGP_ERR_NOT_BUILT, "ehgp_hierarchy needs a resident LBVH");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return ehgp::abi_cuda_fail(ctx, e, "cudaSetDevice");
  if (!ctx->geom_ready) {
    ehgp::geom_prepare(*ctx, (uint32_t)ctx->built_n);
    if ((e = cudaGetLastError()) != cudaSuccess) return ehgp::abi_cuda_fail(ctx, e, "traversal preparation");
  }
  if (!ctx->scale_valid)
    return ehgp::abi_fail(ctx, EHGP_ERR_NUMERIC_RANGE, "the cloud exceeds the exact fixed-point range");
  cudaMemsetAsync(ctx->d_err, 0, sizeof(uint32_t), ctx->stream);
  const int s = ehgp::hier_run(*ctx, K);
  if (counts) {
    std::memset(counts, 0, sizeof(*counts));
    if (ctx->hier) {
      const ehgp::HierState& h = *ctx->hier;
      counts->events = h.events;
      counts->diagnostics = h.diagnostics;
      if (!h.off.empty()) {
        const ehgp::HierOff& t = h.off.back();
        counts->journal_batches = t.jb;
        counts->role_records = t.role;
        counts->families = t.fam;
        counts->arm_seeds = h.arm_seeds;
        counts->birth_records = t.birth;
        counts->nodes = t.node;
        counts->children = t.child;
        counts->arm_bindings = t.bind;
        counts->saddle_records = t.sad;
        counts->atomic_groups = t.grp;
        counts->final_roots = t.root;
        counts->vertical_assignments = t.vert;
      }
      counts->k_eff = h.keff;
    }
    counts->decision = (uint32_t)s;
  }
  return s;
}

int ehgp_hier_schedule(ehgp_ctx* ctx, uint32_t chunk_batches, uint32_t part_arms, uint32_t host_threads) {
  if (!ctx) return EHGP_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(ctx->mutex);
  if (!ctx->hier) ctx->hier = new ehgp::HierState();
  ehgp::HierState& h = *ctx->hier;
  h.chunk_batches = chunk_batches ? chunk_batches : 1u << 14;
  h.part_arms = part_arms ? part_arms : 1u << 22;
  h.pool_threads = host_threads;
  return EHGP_OK;
}

int ehgp_hier_copy(ehgp_ctx* ctx, const ehgp_hier_out* out) {
  if (!ctx || !out) return EHGP_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(ctx->mutex);
  if (!ctx->hier) return ehgp::abi_fail(ctx, EHGP_ERR_NOT_BUILT, "no hierarchy result is resident");
  const ehgp::HierState& h = *ctx->hier;
  if (out->events && h.events) {
    const cudaError_t e = cudaMemcpy(out->events, h.ev, h.events * sizeof(ehgp::EvRec), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return ehgp::abi_cuda_fail(ctx, e, "facade copy");
  }
  if (h.off.empty()) return EHGP_OK;
  if (out->arm_removed && h.arm_seeds) {
    const cudaError_t e = cudaMemcpy(out->arm_removed, h.d_removed, h.arm_seeds * 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return ehgp::abi_cuda_fail(ctx, e, "arm seed copy");
  }
  // Each order's arenas go to their global offsets with local indices shifted, in chunks
  // spread over the host cores.
  using ehgp::HierOff;
  const uint32_t keff = (uint32_t)h.off.size() - 2;
  std::vector<std::function<void()>> tasks;
  constexpr uint64_t kChunk = 1u << 18;
  auto shift = [](uint32_t v, uint32_t d) { return v == ehgp::kInvalid32 ? v : v + d; };
  auto add = [&](void* dst_base, uint64_t count, auto&& one) {
    if (!dst_base) return;
    for (uint64_t lo = 0; lo < count; lo += kChunk) {
      const uint64_t hi = std::min(count, lo + kChunk);
      tasks.emplace_back([=] {
        for (uint64_t i = lo; i < hi; ++i) one(i);
      });
    }
  };
  for (uint32_t k = 1; k <= keff; ++k) {
    const ehgp::HierOrderOut& o = h.outs[k];
    const HierOff f = h.off[k];
    add(out->journal_batches, o.jb.size(), [&o, f, out](uint64_t i) {
      ehgp_journal_batch x = o.jb[i];
      x.role_offset += f.role;
      ehgp::nt_store(out->journal_batches[f.jb + i], x);
    });
    add(out->batches, o.fb.size(), [&o, f, out](uint64_t i) {
      ehgp_forest_batch y = o.fb[i];
      y.birth_offset += f.birth;
      y.saddle_offset += f.sad;
      y.group_offset += f.grp;
      ehgp::nt_store(out->batches[f.jb + i], y);
    });
    add(out->roles, o.roles.size(), [&o, f, out](uint64_t i) {
      ehgp_role_record x = o.roles[i];
      x.batch += f.jb;
      ehgp::nt_store(out->roles[f.role + i], x);
    });
    add(out->families, o.fam.size(), [&o, f, out](uint64_t i) {
      ehgp_family_record x = o.fam[i];
      x.role_record += f.role;
      x.batch += f.jb;
      ehgp::nt_store(out->families[f.fam + i], x);
    });
    add(out->nodes, o.nodes.size(), [&o, f, out, shift](uint64_t i) {
      ehgp_forest_node x = o.nodes[i];
      x.child_offset += f.child;
      x.atomic_group = shift(x.atomic_group, f.grp);
      ehgp::nt_store(out->nodes[f.node + i], x);
    });
    add(out->children, o.children.size(), [&o, f, out](uint64_t i) { out->children[f.child + i] = o.children[i] + f.node; });
    add(out->births, o.births.size(), [&o, f, out, shift](uint64_t i) {
      ehgp_forest_birth x = o.births[i];
      x.batch += f.jb;
      x.order_one_node = shift(x.order_one_node, f.node);
      ehgp::nt_store(out->births[f.birth + i], x);
    });
    add(out->bindings, o.bindings.size(), [&o, f, out, shift](uint64_t i) {
      ehgp_forest_binding x = o.bindings[i];
      x.family += f.fam;
      x.prior_root = shift(x.prior_root, f.node);
      ehgp::nt_store(out->bindings[f.bind + i], x);
    });
    add(out->saddles, o.saddles.size(), [&o, f, out](uint64_t i) {
      ehgp_forest_saddle x = o.saddles[i];
      x.family += f.fam;
      x.batch += f.jb;
      x.arm_offset += f.bind;
      x.group += f.grp;
      ehgp::nt_store(out->saddles[f.sad + i], x);
    });
    add(out->groups, o.groups.size(), [&o, f, out, shift](uint64_t i) {
      ehgp_forest_group x = o.groups[i];
      x.batch += f.jb;
      x.saddle_offset += f.sad;
      x.child_offset += f.child;
      x.created_node = shift(x.created_node, f.node);
      x.result_node = shift(x.result_node, f.node);
      ehgp::nt_store(out->groups[f.grp + i], x);
    });
    add(out->roots, o.roots.size(), [&o, f, out](uint64_t i) {
      ehgp_forest_root x = o.roots[i];
      x.node += f.node;
      ehgp::nt_store(out->roots[f.root + i], x);
    });
    if (k >= 2 && k < h.vert.size()) {
      const std::vector<ehgp_vertical_assignment>& v = h.vert[k];
      const uint32_t tnode = h.off[k - 1].node;
      add(out->vertical, v.size(), [&v, f, tnode, out](uint64_t i) {
        ehgp_vertical_assignment x = v[i];
        x.source_node += f.node;
        x.target_node += tnode;
        ehgp::nt_store(out->vertical[f.vert + i], x);
      });
    }
  }
  if (!tasks.empty()) {
    const uint32_t hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    const uint32_t nt = (uint32_t)std::min<uint64_t>(hw, tasks.size());
    std::atomic<uint64_t> next{0};
    auto work = [&] {
      for (uint64_t t; (t = next.fetch_add(1)) < tasks.size();) tasks[t]();
      ehgp::stream_fence();  // the streaming stores are complete before the join
    };
    std::vector<std::thread> pool;
    for (uint32_t i = 1; i < nt; ++i) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
  }
  return EHGP_OK;
}

int ehgp_hier_stats(const ehgp_ctx* ctx, double* ms, uint64_t* stats) {
  if (!ctx || !ctx->hier) return EHGP_ERR_INVALID_ARGUMENT;
  const ehgp::HierState& h = *ctx->hier;
  if (ms) {
    ms[0] = h.ms_device;
    ms[1] = h.ms_descent;
    ms[2] = h.ms_forest;
    ms[3] = h.ms_orders;
    for (int i = 0; i < 4; ++i) ms[4 + i] = h.ms_host[i];
    for (uint32_t k = 1; k <= 16; ++k) ms[7 + k] = k < h.outs.size() ? h.outs[k].ms : 0.0;
  }
  if (stats) {
    stats[0] = h.arms;
    stats[1] = h.descent_steps;
    stats[2] = h.exact_boundaries;
    stats[3] = h.events;
    stats[4] = h.first_misses;
    stats[5] = h.descent_rounds;
    for (int i = 0; i < 7; ++i) stats[6 + i] = h.slow[i];
    uint64_t v = 0;
    for (int i = 0; i < ehgp::kVisitStripes; ++i) v += h.visits[i];
    stats[13] = v;
    stats[14] = h.step_launches;
  }
  if (ms) ms[24] = h.ms_steps;
  return EHGP_OK;
}

int ehgp_event_supports(ehgp_ctx* ctx, const uint32_t* events, uint64_t count, uint32_t* out) {
  if (!ctx || (count && (!events || !out))) return EHGP_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(ctx->mutex);
  if (!ctx->hier || ctx->hier->decision != EHGP_OK || !ctx->hier->order0 || !ctx->hier->ev_raw)
    return ehgp::abi_fail(ctx, EHGP_ERR_NOT_BUILT, "ehgp_event_supports needs a hierarchy result");
  ehgp::HierState& h = *ctx->hier;
  cudaStream_t st = ctx->stream;
  // chunks through the facade's scratch (index: order0, output: ev_raw), free after the call
  const uint64_t chunk = std::min<uint64_t>(h.cap_events, (h.cap_events * sizeof(ehgp::EvRec)) / 20);
  for (uint64_t b0 = 0; b0 < count; b0 += chunk) {
    const uint32_t m = (uint32_t)std::min<uint64_t>(chunk, count - b0);
    cudaMemcpyAsync(h.order0, events + b0, (uint64_t)m * 4, cudaMemcpyHostToDevice, st);
    ehgp::k_event_supports<<<ehgp::nblk(m, ehgp::kT), ehgp::kT, 0, st>>>(m, h.order0, h.ev, (uint32_t)h.events,
                                                                        (uint32_t*)h.ev_raw);
    cudaMemcpyAsync(out + 5 * b0, h.ev_raw, (uint64_t)m * 20, cudaMemcpyDeviceToHost, st);
    const cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return ehgp::abi_cuda_fail(ctx, e, "facade event supports");
  }
  return EHGP_OK;
}

int ehgp_event_level(ehgp_ctx* ctx, uint64_t event, uint64_t* num, uint64_t* den, int32_t* scale) {
  if (!ctx || !num || !den) return EHGP_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(ctx->mutex);
  if (!ctx->hier || event >= ctx->hier->events)
    return ehgp::abi_fail(ctx, EHGP_ERR_INVALID_ARGUMENT, "no such facade event");
  const ehgp::HierState& h = *ctx->hier;
  ehgp::EvRec r;
  cudaError_t ce = cudaMemcpy(&r, h.ev + event, sizeof r, cudaMemcpyDeviceToHost);
  if (ce != cudaSuccess) return ehgp::abi_cuda_fail(ctx, ce, "facade event copy");
  if (r.size < 2 || r.size > 4) return ehgp::abi_fail(ctx, EHGP_ERR_INVALID_ARGUMENT, "no such facade event");
  // the support's coordinates only (the cloud stays on the device)
  double sx[4], sy[4], sz[4];
  uint32_t local[4];
  for (uint32_t j = 0; j < r.size; ++j) {
    if ((ce = cudaMemcpy(sx + j, ctx->lb.px + r.ids[j], 8, cudaMemcpyDeviceToHost)) != cudaSuccess ||
        (ce = cudaMemcpy(sy + j, ctx->lb.py + r.ids[j], 8, cudaMemcpyDeviceToHost)) != cudaSuccess ||
        (ce = cudaMemcpy(sz + j, ctx->lb.pz + r.ids[j], 8, cudaMemcpyDeviceToHost)) != cudaSuccess)
      return ehgp::abi_cuda_fail(ctx, ce, "support coordinates");
    local[j] = j;
  }
  const ehgp::Cloud c{sx, sy, sz, h.S};
  ehgp::W A;
  ehgp::WV N;
  ehgp::exact_sphere(c, local, (int)r.size, A, N);
  using WL = ehgp::WL;
  const WL x = ehgp::widen<36>(N.x), y = ehgp::widen<36>(N.y), z = ehgp::widen<36>(N.z), a = ehgp::widen<36>(A);
  const WL nn = ehgp::wadd(ehgp::wadd(ehgp::wmul(x, x), ehgp::wmul(y, y)), ehgp::wmul(z, z));
  const WL dd = ehgp::wmul(ehgp::wmul(a, a), WL::from_i128(4));
  for (int i = 0; i < 36; ++i) {
    num[i] = nn.w[i];
    den[i] = dd.w[i];
  }
  if (scale) *scale = h.S;
  return EHGP_OK;
}

}  // extern "C"
