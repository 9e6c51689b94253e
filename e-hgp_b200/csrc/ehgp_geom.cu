// Exact k-nearest neighbours and Boruvka EMST over the resident LBVH (sm_100a).
//
// Reference semantics (Ludwig-H/E-HGP, morsehgp3d/):
//  * top-k partition: the k-th smallest exact squared distance is the cutoff,
//    every point strictly below it, the COMPLETE equality shell at it, and the
//    canonical choice = strict points + least shell PointIds:
//    TopKPartition::from_evaluated_neighbors, src/cpu/spatial/brute_force.cpp:319-384;
//    order (squared distance, PointId): exact_neighbor_less,
//    src/cpu/spatial/exact_query.hpp:54-61; LBVH traversal prunes only on
//    strict bounds: lbvh_top_k, include/morsehgp3d/spatial/lbvh.hpp:424-450.
//  * Boruvka: per round, labels frozen to the least PointId of each component,
//    LBVH nodes tagged uniform/mixed, every component's minimum outgoing edge by
//    kappa = (squared length, u, v) with u < v, contraction through the least
//    PointId: build_exact_lbvh_boruvka, include/morsehgp3d/hierarchy/boruvka.hpp:1-140,
//    src/cpu/hierarchy/boruvka.cpp; output order (squared_length, u, v).
//
// B200 design: one thread per query in Morton order (neighbouring threads walk
// neighbouring subtrees), binary32 outward-rounded boxes for pruning, FP64
// distances with a rigorous relative band, exact integer squared distances at
// the cloud's fixed-point scale only for candidates inside the band.
// Component minima are reduced with a 64-bit atomicMin on the FP64 distance
// bits, then an exact compare-and-swap among the few candidates inside the band.
// Contraction is a lock-free union-find that always hooks the larger root
// under the smaller one, so every root is the least PointId of its component.
#include "ehgp_internal.cuh"
#include "ehgp_exact.cuh"

#include <cstring>
#include <vector>

namespace ehgp {
namespace {

constexpr int kThreads = 256;
constexpr int kStack = 128;
constexpr int kKnnMax = 11;
constexpr int kKnnCap = 48;
constexpr double kTiny = 1e-290;

__host__ __device__ inline uint32_t nblocks(uint64_t n, int t = kThreads) {
  const uint64_t b = (n + t - 1) / t;
  return b == 0 ? 1u : (uint32_t)b;
}

__device__ __forceinline__ uint64_t dbits(double v) { return (uint64_t)__double_as_longlong(v); }

// a < b with certainty despite FP64 rounding of both (kDistRelErr each).
__device__ __forceinline__ bool fp_surely_less(double a, double b) {
  return b > kTiny && a < b * (1.0 - 2.0 * kDistRelErr);
}

__device__ __forceinline__ double dist2_fp(double ax, double ay, double az, double bx, double by, double bz) {
  const double dx = ax - bx, dy = ay - by, dz = az - bz;
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

// Lower bound of the squared distance from q to a binary32 box (outward
// rounded); deflated so that it never exceeds the exact bound.
__device__ __forceinline__ double box_lb(const TNode& t, double qx, double qy, double qz) {
  const double dx = fmax(fmax((double)t.lo[0] - qx, qx - (double)t.hi[0]), 0.0);
  const double dy = fmax(fmax((double)t.lo[1] - qy, qy - (double)t.hi[1]), 0.0);
  const double dz = fmax(fmax((double)t.lo[2] - qz, qz - (double)t.hi[2]), 0.0);
  return (dx * dx + dy * dy + dz * dz) * (1.0 - 4.0 * kDistRelErr);
}

__device__ __forceinline__ TNode load_node(const TNode* __restrict__ tn, uint32_t i) {
  const float4* p = reinterpret_cast<const float4*>(tn + i);
  const float4 a = __ldg(p), b = __ldg(p + 1);
  TNode t;
  t.lo[0] = a.x; t.lo[1] = a.y; t.lo[2] = a.z; t.left = __float_as_uint(a.w);
  t.hi[0] = b.x; t.hi[1] = b.y; t.hi[2] = b.z; t.right = __float_as_uint(b.w);
  return t;
}

struct Fix3 {
  __int128 v[3];
};
__device__ __forceinline__ Fix3 fixed_point(const double* px, const double* py, const double* pz, uint32_t id,
                                            int S) {
  Fix3 f;
  f.v[0] = fixed_of(dbits(px[id]), S);
  f.v[1] = fixed_of(dbits(py[id]), S);
  f.v[2] = fixed_of(dbits(pz[id]), S);
  return f;
}

// ---- preparation -----------------------------------------------------------------
__global__ void __launch_bounds__(kThreads)
k_tnodes(uint32_t n, const uint32_t* __restrict__ n_left, const uint32_t* __restrict__ n_right,
         const uint32_t* __restrict__ n_begin, const uint32_t* __restrict__ n_lo, const uint32_t* __restrict__ n_hi,
         const uint32_t* __restrict__ leaf_pid, const double* __restrict__ px, const double* __restrict__ py,
         const double* __restrict__ pz, TNode* __restrict__ tn, uint32_t* __restrict__ leaf_node) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 2 * n - 1) return;
  const uint32_t N2 = 2 * n;
  const double* P[3] = {px, py, pz};
  TNode t;
  for (int a = 0; a < 3; ++a) {
    t.lo[a] = __double2float_rd(P[a][n_lo[(uint64_t)a * N2 + i]]);
    t.hi[a] = __double2float_ru(P[a][n_hi[(uint64_t)a * N2 + i]]);
  }
  const uint32_t l = n_left[i];
  if (l == kInvalid32) {
    const uint32_t b = n_begin[i];
    t.left = kInvalid32;
    t.right = leaf_pid[b];
    leaf_node[b] = i;
  } else {
    t.left = l;
    t.right = n_right[i];
  }
  tn[i] = t;
}

// Cloud scale: S = the largest number of fractional bits of any coordinate;
// valid when every |x| * 2^S < 2^124.
__global__ void __launch_bounds__(kThreads)
k_scale(uint32_t n, const double* __restrict__ px, const double* __restrict__ py, const double* __restrict__ pz,
        int* __restrict__ scale) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* P[3] = {px, py, pz};
  int frac = -100000, high = -100000;
  for (int a = 0; a < 3; ++a) {
    const uint64_t b = dbits(P[a][i]);
    const uint64_t ex = (b >> 52) & 0x7ff, fr = b & ((uint64_t{1} << 52) - 1);
    if (ex == 0 && fr == 0) continue;
    const uint64_t m = ex ? (fr | (uint64_t{1} << 52)) : fr;
    const int e = ex ? (int)ex - 1075 : -1074;
    frac = max(frac, -(e + (int)__ffsll((long long)m) - 1));  // fractional bits of x
    high = max(high, e + 64 - (int)__clzll((long long)m));    // bit length of |x| relative to 2^0
  }
  atomicMax(scale + 0, frac);
  atomicMax(scale + 1, high);
}

// ---- exact k nearest neighbours ------------------------------------------------------
__global__ void __launch_bounds__(kThreads)
k_knn(uint32_t n, uint32_t k, uint32_t root, const TNode* __restrict__ tn, const uint32_t* __restrict__ leaf_pid,
      const double* __restrict__ px, const double* __restrict__ py, const double* __restrict__ pz,
      const int* __restrict__ scale, uint32_t* __restrict__ out_ids, uint32_t* __restrict__ out_meta,
      uint64_t* __restrict__ out_cut, uint32_t* __restrict__ err) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t p = leaf_pid[i];
  const double qx = px[p], qy = py[p], qz = pz[p];
  double cd[kKnnCap];
  uint32_t cid[kKnnCap];
  int cnt = 0;
  uint32_t stack[kStack];
  int top = 0;
  stack[top++] = root;
  const double band = 1.0 + 2.0 * kDistRelErr;
  while (top > 0) {
    const uint32_t node = stack[--top];
    const TNode t = load_node(tn, node);
    const double thr = (cnt >= (int)k) ? cd[k - 1] * band : INFINITY;
    if (t.left == kInvalid32) {
      const uint32_t q = t.right;
      if (q == p) continue;
      const double d = dist2_fp(qx, qy, qz, px[q], py[q], pz[q]);
      if (d > thr && d > kTiny) continue;
      if (cnt == kKnnCap) { atomicOr(err, kErrCapacity); return; }
      int j = cnt++;
      while (j > 0 && (cd[j - 1] > d || (cd[j - 1] == d && cid[j - 1] > q))) {
        cd[j] = cd[j - 1];
        cid[j] = cid[j - 1];
        --j;
      }
      cd[j] = d;
      cid[j] = q;
      if (cnt > (int)k) {  // drop the tail outside the band of the k-th
        const double lim = cd[k - 1] * band;
        while (cnt > (int)k && cd[cnt - 1] > lim && cd[cnt - 1] > kTiny) --cnt;
      }
      continue;
    }
    if (box_lb(t, qx, qy, qz) > thr) continue;
    const TNode L = load_node(tn, t.left), R = load_node(tn, t.right);
    const double lb_l = box_lb(L, qx, qy, qz), lb_r = box_lb(R, qx, qy, qz);
    if (top + 2 > kStack) { atomicOr(err, kErrCapacity); return; }
    // push the far child first so that the near child is visited first
    if (lb_l <= lb_r) {
      if (lb_r <= thr) stack[top++] = t.right;
      if (lb_l <= thr) stack[top++] = t.left;
    } else {
      if (lb_l <= thr) stack[top++] = t.left;
      if (lb_r <= thr) stack[top++] = t.right;
    }
  }
  if (cnt < (int)k) { atomicOr(err, kErrInternal); return; }
  // exact refinement: order the band candidates by (exact squared distance, id)
  if (!scale[2]) { atomicOr(err, kErrNumericRange); return; }
  const int S = scale[0];
  const Fix3 fq = fixed_point(px, py, pz, p, S);
  WInt<4> D[kKnnCap];
  for (int j = 0; j < cnt; ++j) {
    const Fix3 f = fixed_point(px, py, pz, cid[j], S);
    D[j] = exact_dist2(fq.v, f.v);
  }
  for (int a = 1; a < cnt; ++a) {
    const WInt<4> dv = D[a];
    const uint32_t iv = cid[a];
    int j = a;
    while (j > 0) {
      const int c = wcmp(D[j - 1], dv);
      if (c < 0 || (c == 0 && cid[j - 1] < iv)) break;
      D[j] = D[j - 1];
      cid[j] = cid[j - 1];
      --j;
    }
    D[j] = dv;
    cid[j] = iv;
  }
  const WInt<4> cut = D[k - 1];
  uint32_t strict = 0, shell = 0;
  for (int j = 0; j < cnt; ++j) {
    const int c = wcmp(D[j], cut);
    if (c < 0) ++strict;
    else if (c == 0) ++shell;
  }
  for (uint32_t j = 0; j < k; ++j) out_ids[(uint64_t)p * k + j] = cid[j];
  out_meta[2ull * p] = strict;
  out_meta[2ull * p + 1] = shell;
  for (int w = 0; w < 4; ++w) out_cut[4ull * p + w] = cut.w[w];
}

// ---- Boruvka EMST -----------------------------------------------------------------------
__global__ void k_bv_init(uint32_t n, uint32_t* __restrict__ labels, uint32_t* __restrict__ uf) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    labels[i] = i;
    uf[i] = i;
  }
}

// uniform-label tags of every node, bottom-up (one arrival counter per node)
__global__ void __launch_bounds__(kThreads)
k_bv_node_labels(uint32_t n, const uint32_t* __restrict__ leaf_node, const uint32_t* __restrict__ leaf_pid,
                 const uint32_t* __restrict__ labels, const uint32_t* __restrict__ n_parent,
                 const uint32_t* __restrict__ n_left, const uint32_t* __restrict__ n_right, uint32_t* nlabel,
                 uint32_t* __restrict__ nflag, uint32_t* __restrict__ err) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t cur = leaf_node[i];
  __stcg(nlabel + cur, labels[leaf_pid[i]]);
  for (uint32_t step = 0; step < 2 * n + 64; ++step) {
    const uint32_t p = n_parent[cur];
    if (p == kInvalid32) return;
    __threadfence();
    if (atomicAdd(&nflag[p], 1u) == 0u) return;
    __threadfence();
    const uint32_t a = __ldcg(nlabel + n_left[p]), b = __ldcg(nlabel + n_right[p]);
    __stcg(nlabel + p, (a == b) ? a : kInvalid32);
    cur = p;
  }
  atomicOr(err, kErrInternal);
}

// kappa order of two candidate edges (p1,q1) and (p2,q2) with FP64 lengths.
__device__ bool kappa_less(uint32_t p1, uint32_t q1, double d1, uint32_t p2, uint32_t q2, double d2,
                           const double* px, const double* py, const double* pz, int S) {
  if (fp_surely_less(d1, d2)) return true;
  if (fp_surely_less(d2, d1)) return false;
  const Fix3 a = fixed_point(px, py, pz, p1, S), b = fixed_point(px, py, pz, q1, S);
  const Fix3 c = fixed_point(px, py, pz, p2, S), d = fixed_point(px, py, pz, q2, S);
  const int cmp = wcmp(exact_dist2(a.v, b.v), exact_dist2(c.v, d.v));
  if (cmp != 0) return cmp < 0;
  const uint32_t u1 = min(p1, q1), v1 = max(p1, q1), u2 = min(p2, q2), v2 = max(p2, q2);
  return u1 < u2 || (u1 == u2 && v1 < v2);
}

__global__ void __launch_bounds__(kThreads)
k_bv_nearest(uint32_t n, uint32_t root, const TNode* __restrict__ tn, const uint32_t* __restrict__ leaf_pid,
             const uint32_t* __restrict__ labels, const uint32_t* __restrict__ nlabel,
             const double* __restrict__ px, const double* __restrict__ py, const double* __restrict__ pz,
             const int* __restrict__ scale, uint32_t* __restrict__ best_q, double* __restrict__ best_d,
             uint32_t* __restrict__ err) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t p = leaf_pid[i];
  const uint32_t my = labels[p];
  const double qx = px[p], qy = py[p], qz = pz[p];
  const int S = scale[0];
  uint32_t bq = kInvalid32;
  double bd = INFINITY;
  uint32_t stack[kStack];
  int top = 0;
  stack[top++] = root;
  const double band = 1.0 + 2.0 * kDistRelErr;
  while (top > 0) {
    const uint32_t node = stack[--top];
    if (__ldg(nlabel + node) == my) continue;  // whole subtree inside my component
    const TNode t = load_node(tn, node);
    const double thr = (bq == kInvalid32) ? INFINITY : fmax(bd * band, kTiny);
    if (t.left == kInvalid32) {
      const uint32_t q = t.right;
      const double d = dist2_fp(qx, qy, qz, px[q], py[q], pz[q]);
      if (d > thr) continue;
      if (bq == kInvalid32 || kappa_less(p, q, d, p, bq, bd, px, py, pz, S)) {
        bq = q;
        bd = d;
      }
      continue;
    }
    if (box_lb(t, qx, qy, qz) > thr) continue;
    const TNode L = load_node(tn, t.left), R = load_node(tn, t.right);
    const double lb_l = box_lb(L, qx, qy, qz), lb_r = box_lb(R, qx, qy, qz);
    if (top + 2 > kStack) { atomicOr(err, kErrCapacity); return; }
    if (lb_l <= lb_r) {
      if (lb_r <= thr) stack[top++] = t.right;
      if (lb_l <= thr) stack[top++] = t.left;
    } else {
      if (lb_l <= thr) stack[top++] = t.left;
      if (lb_r <= thr) stack[top++] = t.right;
    }
  }
  best_q[p] = bq;
  best_d[p] = bd;
}

__global__ void __launch_bounds__(kThreads)
k_bv_comp_fpmin(uint32_t n, const uint32_t* __restrict__ labels, const uint32_t* __restrict__ best_q,
                const double* __restrict__ best_d, unsigned long long* __restrict__ comp_dbits) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n || best_q[p] == kInvalid32) return;
  atomicMin(comp_dbits + labels[p], (unsigned long long)dbits(best_d[p]));
}

__global__ void __launch_bounds__(kThreads)
k_bv_comp_exact(uint32_t n, const uint32_t* __restrict__ labels, const uint32_t* __restrict__ best_q,
                const double* __restrict__ best_d, const unsigned long long* __restrict__ comp_dbits,
                uint32_t* __restrict__ comp_best, const double* __restrict__ px, const double* __restrict__ py,
                const double* __restrict__ pz, const int* __restrict__ scale, uint32_t* __restrict__ err) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n || best_q[p] == kInvalid32) return;
  const uint32_t c = labels[p];
  const double m = __longlong_as_double((long long)comp_dbits[c]);
  const double d = best_d[p];
  if (fp_surely_less(m, d)) return;  // cannot be the component minimum
  const int S = scale[0];
  const uint32_t q = best_q[p];
  uint32_t cur = atomicAdd(comp_best + c, 0u);
  for (int it = 0; it < 1 << 20; ++it) {
    if (cur != kInvalid32) {
      const uint32_t cq = best_q[cur];
      if (!kappa_less(p, q, d, cur, cq, best_d[cur], px, py, pz, S)) return;
    }
    const uint32_t seen = atomicCAS(comp_best + c, cur, p);
    if (seen == cur) return;
    cur = seen;
  }
  atomicOr(err, kErrTimeout);
}

__device__ uint32_t uf_find(uint32_t* uf, uint32_t x) {
  for (int it = 0; it < 1 << 22; ++it) {
    const uint32_t p = __ldcg(uf + x);
    if (p == x) return x;
    const uint32_t gp = __ldcg(uf + p);
    if (gp != p) atomicCAS(uf + x, p, gp);  // path halving, benign under races
    x = gp;
  }
  return x;
}

__global__ void __launch_bounds__(kThreads)
k_bv_accept(uint32_t n, uint32_t round, const uint32_t* __restrict__ labels, const uint32_t* __restrict__ comp_best,
            const uint32_t* __restrict__ best_q, uint32_t* __restrict__ uf, uint32_t* __restrict__ counters,
            uint32_t* __restrict__ minima, uint32_t minima_cap, uint32_t* __restrict__ edge_u,
            uint32_t* __restrict__ edge_v, uint32_t* __restrict__ err) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n || labels[c] != c) return;  // one thread per frozen component
  const uint32_t p = comp_best[c];
  if (p == kInvalid32) return;           // the single final component
  const uint32_t q = best_q[p];
  const uint32_t c2 = labels[q];
  const uint32_t mi = atomicAdd(counters + 1, 1u);
  if (mi < minima_cap) {
    minima[4ull * mi] = round;
    minima[4ull * mi + 1] = c;
    minima[4ull * mi + 2] = p;
    minima[4ull * mi + 3] = q;
  } else {
    atomicOr(err, kErrCapacity);
  }
  const uint32_t p2 = comp_best[c2];
  const uint32_t q2 = (p2 == kInvalid32) ? kInvalid32 : best_q[p2];
  const bool mutual = (p2 == q && q2 == p);
  if (!(mutual && c > c2)) {
    const uint32_t e = atomicAdd(counters + 2, 1u);
    if (e < n - 1) {
      edge_u[e] = min(p, q);
      edge_v[e] = max(p, q);
    } else {
      atomicOr(err, kErrInternal);
    }
  }
  // lock-free union: hook the larger root under the smaller one
  uint32_t a = c, b = c2;
  for (int it = 0; it < 1 << 20; ++it) {
    a = uf_find(uf, a);
    b = uf_find(uf, b);
    if (a == b) return;
    if (a > b) { const uint32_t t = a; a = b; b = t; }
    if (atomicCAS(uf + b, b, a) == b) return;
  }
  atomicOr(err, kErrTimeout);
}

__global__ void __launch_bounds__(kThreads)
k_bv_relabel(uint32_t n, uint32_t* __restrict__ labels, uint32_t* __restrict__ uf, uint32_t* __restrict__ counters) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const uint32_t r = uf_find(uf, labels[p]);
  labels[p] = r;
  if (r == p) atomicAdd(counters, 1u);
}

__global__ void __launch_bounds__(kThreads)
k_bv_edge_keys(uint32_t m, const uint32_t* __restrict__ eu, const uint32_t* __restrict__ ev,
               const double* __restrict__ px, const double* __restrict__ py, const double* __restrict__ pz,
               uint64_t* __restrict__ ku, uint64_t* __restrict__ kv, uint64_t* __restrict__ kd,
               uint32_t* __restrict__ order) {
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= m) return;
  const uint32_t u = eu[e], v = ev[e];
  ku[e] = u;
  kv[e] = v;
  kd[e] = dbits(dist2_fp(px[u], py[u], pz[u], px[v], py[v], pz[v]));
  order[e] = e;
}

__global__ void __launch_bounds__(kThreads)
k_bv_gather(uint32_t m, const uint32_t* __restrict__ vals0, const uint32_t* __restrict__ vals1,
            const uint32_t* __restrict__ state, int passes, const uint32_t* __restrict__ eu,
            const uint32_t* __restrict__ ev, const double* __restrict__ px, const double* __restrict__ py,
            const double* __restrict__ pz, const int* __restrict__ scale, uint32_t* __restrict__ su,
            uint32_t* __restrict__ sv, uint64_t* __restrict__ sD) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const uint32_t e = radix_result(state, passes, vals0, vals1)[i];
  const uint32_t u = eu[e], v = ev[e];
  su[i] = u;
  sv[i] = v;
  const int S = scale[0];
  const Fix3 a = fixed_point(px, py, pz, u, S), b = fixed_point(px, py, pz, v, S);
  const WInt<4> D = exact_dist2(a.v, b.v);
  for (int w = 0; w < 4; ++w) sD[4ull * i + w] = D.w[w];
}

__device__ __forceinline__ bool fp_ambiguous(double a, double b) {
  return !fp_surely_less(a, b) && !fp_surely_less(b, a);
}

__device__ __forceinline__ int edge_cmp(const uint64_t* D, const uint32_t* u, const uint32_t* v, uint32_t i,
                                        uint32_t j) {
  for (int w = 3; w >= 0; --w)
    if (D[4ull * i + w] != D[4ull * j + w]) return D[4ull * i + w] < D[4ull * j + w] ? -1 : 1;
  if (u[i] != u[j]) return u[i] < u[j] ? -1 : 1;
  if (v[i] != v[j]) return v[i] < v[j] ? -1 : 1;
  return 0;
}

// Marks adjacent pairs of the FP64 radix order whose lengths are within the
// rounding band of each other (amb[i] = pair (i, i+1) is ambiguous).
__global__ void __launch_bounds__(kThreads)
k_bv_mark_runs(uint32_t m, const double* __restrict__ px, const double* __restrict__ py,
               const double* __restrict__ pz, const uint32_t* __restrict__ su, const uint32_t* __restrict__ sv,
               uint32_t* __restrict__ amb) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  if (i + 1 >= m) { amb[i] = 0; return; }
  const double a = dist2_fp(px[su[i]], py[su[i]], pz[su[i]], px[sv[i]], py[sv[i]], pz[sv[i]]);
  const double b = dist2_fp(px[su[i + 1]], py[su[i + 1]], pz[su[i + 1]], px[sv[i + 1]], py[sv[i + 1]],
                            pz[sv[i + 1]]);
  amb[i] = fp_ambiguous(a, b) ? 1u : 0u;
}

// Re-sorts, exactly, every maximal run of mutually adjacent ambiguous edges
// (the FP64 radix order is exact elsewhere).  Runs are disjoint and found
// from the read-only marks, so threads never race.
__global__ void __launch_bounds__(kThreads)
k_bv_fix_runs(uint32_t m, const uint32_t* __restrict__ amb, uint32_t* __restrict__ su, uint32_t* __restrict__ sv,
              uint64_t* __restrict__ sD, uint32_t* __restrict__ err) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i + 1 >= m) return;
  if (!amb[i]) return;
  if (i > 0 && amb[i - 1]) return;  // not the start of its run
  uint32_t end = i + 1;
  while (end + 1 < m && amb[end]) {
    ++end;
    if (end - i > 4096) { atomicOr(err, kErrCapacity); return; }
  }
  // insertion sort of [i, end] by (D, u, v)
  for (uint32_t a = i + 1; a <= end; ++a) {
    uint32_t j = a;
    while (j > i && edge_cmp(sD, su, sv, j - 1, j) > 0) {
      for (int w = 0; w < 4; ++w) {
        const uint64_t t = sD[4ull * j + w];
        sD[4ull * j + w] = sD[4ull * (j - 1) + w];
        sD[4ull * (j - 1) + w] = t;
      }
      const uint32_t tu = su[j], tv = sv[j];
      su[j] = su[j - 1]; sv[j] = sv[j - 1];
      su[j - 1] = tu; sv[j - 1] = tv;
      --j;
    }
  }
}

}  // namespace

cudaError_t geom_alloc(Ctx& ctx) {
  const uint64_t n = ctx.max_points;
  GeomBuffers& g = ctx.gb;
  cudaError_t e = cudaSuccess;
#define EHGP_ALLOC(ptr, bytes) \
  if ((e = ctx_alloc(ctx, (void**)&(ptr), (bytes))) != cudaSuccess) return e
  EHGP_ALLOC(g.tnodes, 2 * n * sizeof(TNode));
  EHGP_ALLOC(g.leaf_node, n * sizeof(uint32_t));
  EHGP_ALLOC(g.scale, 4 * sizeof(int));
  EHGP_ALLOC(g.knn_ids, n * kKnnMax * sizeof(uint32_t));
  EHGP_ALLOC(g.knn_meta, 2 * n * sizeof(uint32_t));
  EHGP_ALLOC(g.knn_cut, 4 * n * sizeof(uint64_t));
  EHGP_ALLOC(g.labels, n * sizeof(uint32_t));
  EHGP_ALLOC(g.nlabel, 2 * n * sizeof(uint32_t));
  EHGP_ALLOC(g.nflag, 2 * n * sizeof(uint32_t));
  EHGP_ALLOC(g.best_q, n * sizeof(uint32_t));
  EHGP_ALLOC(g.best_d, n * sizeof(double));
  EHGP_ALLOC(g.comp_dbits, n * sizeof(unsigned long long));
  EHGP_ALLOC(g.comp_best, n * sizeof(uint32_t));
  EHGP_ALLOC(g.uf, n * sizeof(uint32_t));
  EHGP_ALLOC(g.counters, 8 * sizeof(uint32_t));
  EHGP_ALLOC(g.minima, 4 * 2 * n * sizeof(uint32_t));
  EHGP_ALLOC(g.edge_u, n * sizeof(uint32_t));
  EHGP_ALLOC(g.edge_v, n * sizeof(uint32_t));
  EHGP_ALLOC(g.key_u, n * sizeof(uint64_t));
  EHGP_ALLOC(g.key_v, n * sizeof(uint64_t));
  EHGP_ALLOC(g.key_d, n * sizeof(uint64_t));
  EHGP_ALLOC(g.order0, n * sizeof(uint32_t));
  EHGP_ALLOC(g.order1, n * sizeof(uint32_t));
  EHGP_ALLOC(g.edge_D, 4 * n * sizeof(uint64_t));
  EHGP_ALLOC(g.sorted_u, n * sizeof(uint32_t));
  EHGP_ALLOC(g.sorted_v, n * sizeof(uint32_t));
#undef EHGP_ALLOC
  return cudaSuccess;
}

uint64_t geom_prepare(Ctx& ctx, uint32_t n) {
  LbvhBuffers& b = ctx.lb;
  GeomBuffers& g = ctx.gb;
  cudaStream_t st = ctx.stream;
  k_tnodes<<<nblocks(2ull * n), kThreads, 0, st>>>(n, b.n_left, b.n_right, b.n_begin, b.n_lo, b.n_hi, b.leaf_pid,
                                                    b.px, b.py, b.pz, g.tnodes, g.leaf_node);
  const int init[4] = {-100000, -100000, 0, 0};
  cudaMemcpyAsync(g.scale, init, sizeof(init), cudaMemcpyHostToDevice, st);
  k_scale<<<nblocks(n), kThreads, 0, st>>>(n, b.px, b.py, b.pz, g.scale);
  int sc[4];
  cudaMemcpyAsync(sc, g.scale, sizeof(sc), cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  const int S = sc[0] < 0 ? 0 : sc[0];
  const bool valid = (sc[1] + S) < 124;
  const int fin[4] = {S, sc[1], valid ? 1 : 0, 0};
  cudaMemcpyAsync(g.scale, fin, sizeof(fin), cudaMemcpyHostToDevice, st);
  cudaStreamSynchronize(st);
  ctx.scale_S = S;
  ctx.scale_valid = valid;
  ctx.geom_ready = true;
  return 2;
}

}  // namespace ehgp

using ehgp::Ctx;

namespace {

int begin_stage(Ctx* ctx, const char* what) {
  if (ctx->poisoned) return ehgp::abi_fail(ctx, EHGP_ERR_POISONED, "the context is poisoned by an earlier CUDA failure");
  if (ctx->built_n == 0) return ehgp::abi_fail(ctx, EHGP_ERR_NOT_BUILT, what);
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return ehgp::abi_cuda_fail(ctx, e, "cudaSetDevice");
  if (!ctx->geom_ready) {
    ehgp::geom_prepare(*ctx, (uint32_t)ctx->built_n);
    if ((e = cudaGetLastError()) != cudaSuccess) return ehgp::abi_cuda_fail(ctx, e, "traversal preparation");
  }
  if ((e = cudaMemsetAsync(ctx->d_err, 0, sizeof(uint32_t), ctx->stream)) != cudaSuccess)
    return ehgp::abi_cuda_fail(ctx, e, "cudaMemsetAsync");
  return EHGP_OK;
}

int finish_stage(Ctx* ctx, const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return ehgp::abi_cuda_fail(ctx, e, what);
  cudaMemcpyAsync(ctx->h_status, ctx->d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream);
  if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return ehgp::abi_cuda_fail(ctx, e, what);
  return ehgp::abi_device_status(ctx, ctx->h_status[0]);
}

// Runs the Boruvka rounds and the exact (squared length, u, v) edge order on
// the device; leaves sorted edges in gb.sorted_u/sorted_v/edge_D.
int emst_run(Ctx* ctx) {
  using namespace ehgp;
  const uint32_t n = (uint32_t)ctx->built_n;
  GeomBuffers& g = ctx->gb;
  LbvhBuffers& b = ctx->lb;
  cudaStream_t st = ctx->stream;
  const uint32_t root = 2 * n - 2;
  uint64_t launches = 0;
  cudaEventRecord(ctx->ev0, st);
  cudaMemsetAsync(g.counters, 0, 8 * sizeof(uint32_t), st);
  k_bv_init<<<nblocks(n), kThreads, 0, st>>>(n, g.labels, g.uf);
  ++launches;
  uint32_t components = n, round = 0;
  while (components > 1) {
    if (round > 64) return abi_fail(ctx, EHGP_ERR_CUDA, "Boruvka did not converge");
    cudaMemsetAsync(g.nflag, 0, 2ull * n * sizeof(uint32_t), st);
    k_bv_node_labels<<<nblocks(n), kThreads, 0, st>>>(n, g.leaf_node, b.leaf_pid, g.labels, b.n_parent, b.n_left,
                                                       b.n_right, g.nlabel, g.nflag, ctx->d_err);
    k_bv_nearest<<<nblocks(n), kThreads, 0, st>>>(n, root, g.tnodes, b.leaf_pid, g.labels, g.nlabel, b.px, b.py,
                                                   b.pz, g.scale, g.best_q, g.best_d, ctx->d_err);
    cudaMemsetAsync(g.comp_dbits, 0xff, n * sizeof(unsigned long long), st);
    cudaMemsetAsync(g.comp_best, 0xff, n * sizeof(uint32_t), st);
    k_bv_comp_fpmin<<<nblocks(n), kThreads, 0, st>>>(n, g.labels, g.best_q, g.best_d, g.comp_dbits);
    k_bv_comp_exact<<<nblocks(n), kThreads, 0, st>>>(n, g.labels, g.best_q, g.best_d, g.comp_dbits, g.comp_best,
                                                      b.px, b.py, b.pz, g.scale, ctx->d_err);
    k_bv_accept<<<nblocks(n), kThreads, 0, st>>>(n, round, g.labels, g.comp_best, g.best_q, g.uf, g.counters,
                                                  g.minima, 2 * n, g.edge_u, g.edge_v, ctx->d_err);
    cudaMemsetAsync(g.counters, 0, sizeof(uint32_t), st);
    k_bv_relabel<<<nblocks(n), kThreads, 0, st>>>(n, g.labels, g.uf, g.counters);
    launches += 6;
    cudaMemcpyAsync(ctx->h_status, ctx->d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(ctx->h_status + 1, g.counters, 3 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return abi_cuda_fail(ctx, e, "Boruvka round");
    if (ctx->h_status[0]) return abi_device_status(ctx, ctx->h_status[0]);
    const uint32_t next = ctx->h_status[1];
    if (next >= components) return abi_fail(ctx, EHGP_ERR_CUDA, "a Boruvka round did not contract");
    components = next;
    ++round;
  }
  const uint32_t m = n - 1;
  ctx->emst_rounds = round;
  ctx->emst_minima = ctx->h_status[2];
  if (n > 1) {
    if (ctx->h_status[3] != m) return abi_fail(ctx, EHGP_ERR_CUDA, "Boruvka accepted a wrong number of edges");
    k_bv_edge_keys<<<nblocks(m), kThreads, 0, st>>>(m, g.edge_u, g.edge_v, b.px, b.py, b.pz, g.key_u, g.key_v,
                                                     g.key_d, g.order0);
    const IndirectKey stages[3] = {{g.key_v, 0}, {g.key_u, 0}, {g.key_d, 0}};
    const int bits[3] = {32, 32, 64};
    const int passes = radix_sort_indirect(st, m, g.order0, g.order1, stages, bits, 3, ctx->radix, &launches);
    k_bv_gather<<<nblocks(m), kThreads, 0, st>>>(m, g.order0, g.order1, ctx->radix.state, passes, g.edge_u,
                                                  g.edge_v, b.px, b.py, b.pz, g.scale, g.sorted_u, g.sorted_v,
                                                  g.edge_D);
    // the radix ping-pong buffer order1 is free after the gather: reuse it for the marks
    k_bv_mark_runs<<<nblocks(m), kThreads, 0, st>>>(m, b.px, b.py, b.pz, g.sorted_u, g.sorted_v, g.order1);
    k_bv_fix_runs<<<nblocks(m), kThreads, 0, st>>>(m, g.order1, g.sorted_u, g.sorted_v, g.edge_D, ctx->d_err);
    launches += 4;
  }
  cudaEventRecord(ctx->ev1, st);
  const int s = finish_stage(ctx, "EMST");
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  ctx->last_ms = ms;
  ctx->last_launches = launches;
  if (s == EHGP_OK) ctx->emst_ready = true;
  return s;
}

}  // namespace

extern "C" {

int ehgp_cloud_scale(ehgp_ctx* ctx, int32_t* scale_exponent, int32_t* valid) {
  if (!ctx) return EHGP_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(ctx->mutex);
  if (!ctx->geom_ready) {
    const int s = begin_stage(ctx, "ehgp_cloud_scale needs a resident LBVH (ehgp_lbvh_build)");
    if (s != EHGP_OK) return s;
  }
  if (scale_exponent) *scale_exponent = ctx->scale_S;
  if (valid) *valid = ctx->scale_valid ? 1 : 0;
  return EHGP_OK;
}

int ehgp_knn(ehgp_ctx* ctx, uint32_t k, const ehgp_knn_out* out) {
  if (!ctx) return EHGP_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(ctx->mutex);
  ctx->last_error.clear();
  int s = begin_stage(ctx, "ehgp_knn needs a resident LBVH (ehgp_lbvh_build)");
  if (s != EHGP_OK) return s;
  const uint32_t n = (uint32_t)ctx->built_n;
  if (!out || k == 0 || k > ehgp::kKnnMax || k >= n)
    return ehgp::abi_fail(ctx, EHGP_ERR_INVALID_ARGUMENT, "the requested rank is outside the eligible point set");
  if (!ctx->scale_valid)
    return ehgp::abi_fail(ctx, EHGP_ERR_NUMERIC_RANGE, "the cloud exceeds the exact fixed-point range");
  ehgp::GeomBuffers& g = ctx->gb;
  ehgp::LbvhBuffers& b = ctx->lb;
  cudaEventRecord(ctx->ev0, ctx->stream);
  ehgp::k_knn<<<ehgp::nblocks(n), ehgp::kThreads, 0, ctx->stream>>>(n, k, 2 * n - 2, g.tnodes, b.leaf_pid, b.px,
                                                                     b.py, b.pz, g.scale, g.knn_ids, g.knn_meta,
                                                                     g.knn_cut, ctx->d_err);
  cudaEventRecord(ctx->ev1, ctx->stream);
  s = finish_stage(ctx, "k-NN");
  if (s != EHGP_OK) return s;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  ctx->last_ms = ms;
  ctx->last_launches = 1;
  cudaError_t e = cudaSuccess;
  if (out->ids) e = cudaMemcpy(out->ids, g.knn_ids, (uint64_t)n * k * sizeof(uint32_t), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && out->meta) e = cudaMemcpy(out->meta, g.knn_meta, 2ull * n * sizeof(uint32_t), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && out->cutoff_num)
    e = cudaMemcpy(out->cutoff_num, g.knn_cut, 4ull * n * sizeof(uint64_t), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return ehgp::abi_cuda_fail(ctx, e, "k-NN copy");
  return EHGP_OK;
}

int ehgp_emst(ehgp_ctx* ctx, const ehgp_emst_out* out) {
  if (!ctx) return EHGP_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(ctx->mutex);
  ctx->last_error.clear();
  int s = begin_stage(ctx, "ehgp_emst needs a resident LBVH (ehgp_lbvh_build)");
  if (s != EHGP_OK) return s;
  if (!ctx->scale_valid)
    return ehgp::abi_fail(ctx, EHGP_ERR_NUMERIC_RANGE, "the cloud exceeds the exact fixed-point range");
  s = emst_run(ctx);
  if (s != EHGP_OK || !out) return s;
  const uint64_t n = ctx->built_n, m = n - 1;
  ehgp::GeomBuffers& g = ctx->gb;
  cudaError_t e = cudaSuccess;
  if (m && out->u) e = cudaMemcpy(out->u, g.sorted_u, m * sizeof(uint32_t), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && m && out->v) e = cudaMemcpy(out->v, g.sorted_v, m * sizeof(uint32_t), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && m && out->squared_length_num)
    e = cudaMemcpy(out->squared_length_num, g.edge_D, 4 * m * sizeof(uint64_t), cudaMemcpyDeviceToHost);
  if (out->rounds) *out->rounds = ctx->emst_rounds;
  if (out->minima_count) *out->minima_count = ctx->emst_minima;
  if (e == cudaSuccess && out->minima && out->minima_capacity) {
    const uint64_t c = ctx->emst_minima < out->minima_capacity ? ctx->emst_minima : out->minima_capacity;
    e = cudaMemcpy(out->minima, g.minima, 4 * c * sizeof(uint32_t), cudaMemcpyDeviceToHost);
  }
  if (e != cudaSuccess) return ehgp::abi_cuda_fail(ctx, e, "EMST copy");
  return EHGP_OK;
}

}  // extern "C"
