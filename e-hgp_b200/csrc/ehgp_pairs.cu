// Pair critical-sphere supports (rank <= s_max) on sm_100a.
//
// Reference semantics (Ludwig-H/E-HGP, morsehgp3d/):
//  build_exact_pair_support_stream (include/morsehgp3d/hierarchy/pair_support_stream.hpp:415)
//  with its leaf rule classify_leaf_pair / classify_sparse_closed_ball
//  (src/cpu/hierarchy/pair_support_stream.cpp:1781-2094):
//   * the sphere of a pair (u, v) is its diametral sphere: centre (u + v) / 2,
//     squared level |u - v|^2 / 4;
//   * w is strictly inside iff (w - u).(w - v) < 0, on the sphere iff = 0;
//   * the pair is relevant iff its strict interior count I <= s_max - 2, where
//     s_max = min(min(K, n) + 1, n);
//   * a shell of exactly {u, v} gives an event (closed rank I + 2), a larger
//     shell gives an extra-shell diagnostic with the complete shell count and
//     the least extra shell PointId;
//   * records are in (u, v) order (event_less, pair_support_stream.cpp:120-130).
//
// B200 design (replacing the reference's CPU frontier of node pairs with BigInt
// bounds, pair_support_stream.cpp:1518-2249):
//  * every point u owns a witness list W_u = its 32 nearest other points
//    (FP64 order); R_u^2 is the 32nd squared distance;
//  * one thread per u, in Morton order, walks the LBVH over partners v that
//    follow u in Morton order (each unordered pair is visited once);
//  * a subtree B of partners is pruned when at least s_max - 1 witnesses w of
//    u satisfy max_{v in B} (w - u).(w - v) < 0 with certainty (binary32
//    bound with a conservative margin): every pair (u, v in B) then has more
//    than s_max - 2 strict interior points;
//  * a leaf pair whose sphere lies in the strict 32-NN ball of u or of v
//    (|u - v| < R_u: every point of the closed diametral ball is within |u - v|
//    of u) is classified from that witness list alone; any other leaf pair
//    runs an exact closed-ball query over the LBVH with early rejection;
//  * every side decision is FP64 with a rigorous error bound, then exact
//    integers at the cloud scale inside the bound.
#include "ehgp_internal.cuh"
#include "ehgp_exact.cuh"

#include <cstring>

namespace ehgp {
namespace {

constexpr int kThreads = 128;
constexpr int kStack = 128;
constexpr int kW = 64;           // witnesses per point (two per lane)
constexpr int kMaxInterior = 9;  // s_max - 2 for K >= 10

__host__ __device__ inline uint32_t nblocks(uint64_t n, int t = kThreads) {
  const uint64_t b = (n + t - 1) / t;
  return b == 0 ? 1u : (uint32_t)b;
}

__device__ __forceinline__ uint64_t dbits(double v) { return (uint64_t)__double_as_longlong(v); }

__device__ __forceinline__ TNode load_node(const TNode* __restrict__ tn, uint32_t i) {
  const float4* p = reinterpret_cast<const float4*>(tn + i);
  const float4 a = __ldg(p), b = __ldg(p + 1);
  TNode t;
  t.lo[0] = a.x; t.lo[1] = a.y; t.lo[2] = a.z; t.left = __float_as_uint(a.w);
  t.hi[0] = b.x; t.hi[1] = b.y; t.hi[2] = b.z; t.right = __float_as_uint(b.w);
  return t;
}

__device__ __forceinline__ double d2fp(double ax, double ay, double az, double bx, double by, double bz) {
  const double dx = ax - bx, dy = ay - by, dz = az - bz;
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

__device__ __forceinline__ double box_lb(const TNode& t, double qx, double qy, double qz) {
  const double dx = fmax(fmax((double)t.lo[0] - qx, qx - (double)t.hi[0]), 0.0);
  const double dy = fmax(fmax((double)t.lo[1] - qy, qy - (double)t.hi[1]), 0.0);
  const double dz = fmax(fmax((double)t.lo[2] - qz, qz - (double)t.hi[2]), 0.0);
  return (dx * dx + dy * dy + dz * dz) * (1.0 - 4.0 * kDistRelErr);
}

__device__ __forceinline__ double box_ub(const TNode& t, double qx, double qy, double qz) {
  const double dx = fmax(fabs((double)t.lo[0] - qx), fabs((double)t.hi[0] - qx));
  const double dy = fmax(fabs((double)t.lo[1] - qy), fabs((double)t.hi[1] - qy));
  const double dz = fmax(fabs((double)t.lo[2] - qz), fabs((double)t.hi[2] - qz));
  return (dx * dx + dy * dy + dz * dz) * (1.0 + 4.0 * kDistRelErr);
}

// ---- 32 nearest neighbours (FP64 order; witnesses, no exactness needed) --------
__global__ void __launch_bounds__(kThreads)
k_witness_knn(uint32_t n, uint32_t kw, uint32_t root, const TNode* __restrict__ tn,
              const uint32_t* __restrict__ leaf_pid, const double* __restrict__ px, const double* __restrict__ py,
              const double* __restrict__ pz, uint32_t* __restrict__ W, double* __restrict__ R2,
              uint32_t* __restrict__ err) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t p = leaf_pid[i];
  const double qx = px[p], qy = py[p], qz = pz[p];
  double cd[kW];
  uint32_t cid[kW];
  int cnt = 0;
  uint32_t stack[kStack];
  int top = 0;
  stack[top++] = root;
  while (top > 0) {
    const uint32_t node = stack[--top];
    const TNode t = load_node(tn, node);
    const double thr = (cnt >= (int)kw) ? cd[kw - 1] : INFINITY;
    if (t.left == kInvalid32) {
      const uint32_t q = t.right;
      if (q == p) continue;
      const double d = d2fp(qx, qy, qz, px[q], py[q], pz[q]);
      if (d >= thr) continue;
      int j = (cnt < (int)kw) ? cnt++ : (int)kw - 1;
      while (j > 0 && cd[j - 1] > d) {
        cd[j] = cd[j - 1];
        cid[j] = cid[j - 1];
        --j;
      }
      cd[j] = d;
      cid[j] = q;
      continue;
    }
    if (box_lb(t, qx, qy, qz) > thr) continue;
    const TNode L = load_node(tn, t.left), R = load_node(tn, t.right);
    const double ll = box_lb(L, qx, qy, qz), lr = box_lb(R, qx, qy, qz);
    if (top + 2 > kStack) { atomicOr(err, kErrCapacity); return; }
    if (ll <= lr) {
      if (lr <= thr) stack[top++] = t.right;
      if (ll <= thr) stack[top++] = t.left;
    } else {
      if (ll <= thr) stack[top++] = t.left;
      if (lr <= thr) stack[top++] = t.right;
    }
  }
  for (int j = 0; j < kW; ++j) W[(uint64_t)p * kW + j] = j < cnt ? cid[j] : kInvalid32;
  // witness radius: every point strictly closer than R2 is in W (R2 = +inf when W is all other points)
  R2[p] = (cnt >= (int)kw && n - 1 > kw) ? cd[kw - 1] : INFINITY;
}

// ---- exact side of w relative to the diametral sphere of (u, v) ---------------------
struct Pt {
  double x, y, z;
};
__device__ __forceinline__ Pt point(const double* px, const double* py, const double* pz, uint32_t i) {
  return Pt{px[i], py[i], pz[i]};
}

// sign((w - u).(w - v)): -1 strictly inside, 0 on the sphere, +1 outside.
__device__ int diametral_side(const Pt& w, const Pt& u, const Pt& v, uint32_t iw, uint32_t iu, uint32_t iv,
                              const double* px, const double* py, const double* pz, int S) {
  const double t0 = (w.x - u.x) * (w.x - v.x), t1 = (w.y - u.y) * (w.y - v.y), t2 = (w.z - u.z) * (w.z - v.z);
  const double acc = t0 + t1 + t2;
  const double bound = 16.0 * 1.1102230246251565e-16 * (fabs(t0) + fabs(t1) + fabs(t2)) + 1e-300;
  if (acc > bound) return 1;
  if (acc < -bound) return -1;
  const double* P[3] = {px, py, pz};
  WInt<4> s = WInt<4>::zero();
  for (int a = 0; a < 3; ++a) {
    const __int128 xw = fixed_of(dbits(P[a][iw]), S), xu = fixed_of(dbits(P[a][iu]), S),
                   xv = fixed_of(dbits(P[a][iv]), S);
    s = wadd(s, wmul(WInt<4>::from_i128(xw - xu), WInt<4>::from_i128(xw - xv)));
  }
  return s.sign();
}

struct PairRec {
  uint32_t u, v, interior, shell, witness;
  uint32_t ids[kMaxInterior];
  uint32_t pad[2];
};
static_assert(sizeof(PairRec) == 64, "pair record is one 64-byte line");

// ---- warp-per-point enumeration ---------------------------------------------------
// One warp owns one point u; lane l holds witnesses l and l + 32 of W_u.
constexpr int kWarpsPerBlock = kThreads / 32;
constexpr int kQueue = 256;  // warp-cooperative ball-query frontier (power of two)

struct WarpShared {
  uint32_t stack[kStack];
  uint32_t queue[kQueue];
  uint32_t ids[kMaxInterior + 64];
};

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Appends the ids of flagged lanes (two flags per lane) to sh.ids[base...];
// returns the number appended.  Writes only while the total stays <= cap.
__device__ __forceinline__ uint32_t warp_append(WarpShared& sh, uint32_t base, bool f0, uint32_t id0, bool f1,
                                                uint32_t id1, uint32_t cap) {
  const uint32_t b0 = __ballot_sync(0xffffffffu, f0), b1 = __ballot_sync(0xffffffffu, f1);
  const uint32_t c0 = __popc(b0), total = c0 + __popc(b1);
  if (base + total <= cap) {
    const uint32_t lt = lanemask_lt();
    if (f0) sh.ids[base + __popc(b0 & lt)] = id0;
    if (f1) sh.ids[base + c0 + __popc(b1 & lt)] = id1;
  }
  return total;
}

struct WarpBall {
  uint32_t interior;
  uint32_t shell;    // extra shell points
  uint32_t witness;  // least extra shell id
  bool rejected;
};

// Classifies the two candidates of every lane (w0, w1; kInvalid32 = none).
__device__ __forceinline__ void warp_classify(WarpBall& b, WarpShared& sh, uint32_t w0, uint32_t w1, uint32_t iu,
                                              uint32_t iv, const Pt& u, const Pt& v, const double* px,
                                              const double* py, const double* pz, int S, uint32_t cap) {
  int s0 = 1, s1 = 1;
  if (w0 != kInvalid32 && w0 != iu && w0 != iv)
    s0 = diametral_side(point(px, py, pz, w0), u, v, w0, iu, iv, px, py, pz, S);
  if (w1 != kInvalid32 && w1 != iu && w1 != iv)
    s1 = diametral_side(point(px, py, pz, w1), u, v, w1, iu, iv, px, py, pz, S);
  const uint32_t added = warp_append(sh, b.interior, s0 < 0, w0, s1 < 0, w1, cap);
  b.interior += added;
  if (b.interior > cap) b.rejected = true;
  const uint32_t sb0 = __ballot_sync(0xffffffffu, s0 == 0), sb1 = __ballot_sync(0xffffffffu, s1 == 0);
  b.shell += __popc(sb0) + __popc(sb1);
  const uint32_t mw = min(s0 == 0 ? w0 : kInvalid32, s1 == 0 ? w1 : kInvalid32);
  b.witness = min(b.witness, __reduce_min_sync(0xffffffffu, mw));
}

// Warp-cooperative exact closed-ball query over the LBVH (breadth-first over
// the subtrees that straddle the sphere, 32 nodes per step), early rejection.
__device__ void warp_ball_query(WarpBall& b, WarpShared& sh, uint32_t iu, uint32_t iv, const Pt& u, const Pt& v,
                                uint32_t root, const TNode* tn, const uint32_t* leaf_pid, const uint32_t* n_begin,
                                const uint32_t* n_end, const double* px, const double* py, const double* pz, int S,
                                uint32_t cap, uint32_t* err, unsigned long long& nodes_seen) {
  const uint32_t lane = threadIdx.x & 31u;
  const double mx = 0.5 * (u.x + v.x), my = 0.5 * (u.y + v.y), mz = 0.5 * (u.z + v.z);
  const double r2 = 0.25 * d2fp(u.x, u.y, u.z, v.x, v.y, v.z);
  const double r2_hi = r2 * (1.0 + 8.0 * kDistRelErr) + 1e-300, r2_lo = r2 * (1.0 - 8.0 * kDistRelErr);
  uint32_t head = 0, tail = 1;
  if (lane == 0) sh.queue[0] = root;
  __syncwarp();
  while (head < tail && !b.rejected) {
    const uint32_t batch = min(tail - head, 32u);
    nodes_seen += batch;
    uint32_t node = kInvalid32;
    if (lane < batch) node = sh.queue[(head + lane) & (kQueue - 1)];
    __syncwarp();
    uint32_t leafw = kInvalid32, bulk_b = 0, bulk_e = 0;
    bool expand = false;
    TNode t;
    if (node != kInvalid32) {
      t = load_node(tn, node);
      if (t.left == kInvalid32) {
        leafw = t.right;
      } else if (box_lb(t, mx, my, mz) <= r2_hi) {
        if (box_ub(t, mx, my, mz) < r2_lo) {
          bulk_b = n_begin[node];
          bulk_e = n_end[node];
        } else {
          expand = true;
        }
      }
    }
    warp_classify(b, sh, leafw, kInvalid32, iu, iv, u, v, px, py, pz, S, cap);
    // whole subtrees strictly inside
    uint32_t bulk_total = bulk_e - bulk_b;
    for (int off = 16; off > 0; off >>= 1) bulk_total += __shfl_xor_sync(0xffffffffu, bulk_total, off);
    if (bulk_total) {
      if (b.interior + bulk_total > cap) {
        b.rejected = true;
      } else {
        // append the ids lane by lane (at most cap of them in total)
        uint32_t before = bulk_e - bulk_b;
        for (int off = 1; off < 32; off <<= 1) {
          const uint32_t t2 = __shfl_up_sync(0xffffffffu, before, off);
          if ((int)lane >= off) before += t2;
        }
        before -= (bulk_e - bulk_b);
        for (uint32_t q = bulk_b; q < bulk_e; ++q) sh.ids[b.interior + before + (q - bulk_b)] = leaf_pid[q];
        b.interior += bulk_total;
      }
    }
    // children of straddling subtrees
    const uint32_t eb = __ballot_sync(0xffffffffu, expand);
    const uint32_t pushes = 2 * __popc(eb);
    if (tail - head - batch + pushes > kQueue) {
      if (lane == 0) atomicOr(err, kErrCapacity);
      b.rejected = true;
      break;
    }
    if (expand) {
      const uint32_t at = tail + 2 * __popc(eb & lanemask_lt());
      sh.queue[at & (kQueue - 1)] = t.left;
      sh.queue[(at + 1) & (kQueue - 1)] = t.right;
    }
    __syncwarp();
    head += batch;
    tail += pushes;
  }
  __syncwarp();
}

__global__ void __launch_bounds__(kThreads)
k_pairs(uint32_t n, uint32_t cap, uint32_t root, const TNode* __restrict__ tn, const uint32_t* __restrict__ leaf_pid,
        const uint32_t* __restrict__ n_begin, const uint32_t* __restrict__ n_end, const double* __restrict__ px,
        const double* __restrict__ py, const double* __restrict__ pz, const int* __restrict__ scale,
        const uint32_t* __restrict__ W, const double* __restrict__ R2, PairRec* __restrict__ out,
        uint32_t out_cap, uint32_t* __restrict__ counters, unsigned long long* __restrict__ stats,
        uint32_t* __restrict__ err) {
  __shared__ WarpShared shared[kWarpsPerBlock];
  // work counters (identical in every lane; lane 0 publishes them)
  unsigned long long visits = 0, local_pairs = 0, ball_queries = 0, ball_nodes = 0, emitted = 0;
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  const uint32_t pos = blockIdx.x * kWarpsPerBlock + warp;
  if (pos >= n) return;  // uniform per warp
  WarpShared& sh = shared[warp];
  const uint32_t iu = leaf_pid[pos];
  const Pt u = point(px, py, pz, iu);
  const int S = scale[0];
  const double r2u = R2[iu];
  // this lane's two witnesses of u
  const uint32_t w0 = W[(uint64_t)iu * kW + lane], w1 = W[(uint64_t)iu * kW + 32 + lane];
  float ax0 = 0.f, ay0 = 0.f, az0 = 0.f, ax1 = 0.f, ay1 = 0.f, az1 = 0.f;
  if (w0 != kInvalid32) { ax0 = (float)(px[w0] - u.x); ay0 = (float)(py[w0] - u.y); az0 = (float)(pz[w0] - u.z); }
  if (w1 != kInvalid32) { ax1 = (float)(px[w1] - u.x); ay1 = (float)(py[w1] - u.y); az1 = (float)(pz[w1] - u.z); }
  const uint32_t nw = __popc(__ballot_sync(0xffffffffu, w0 != kInvalid32)) +
                      __popc(__ballot_sync(0xffffffffu, w1 != kInvalid32));
  const uint32_t need = cap + 1;
  uint32_t top = 0;
  if (lane == 0) sh.stack[0] = root;
  top = 1;
  __syncwarp();
  const double lo = 1.0 - 4.0 * kDistRelErr, hi = 1.0 + 4.0 * kDistRelErr;
  while (top > 0) {
    const uint32_t node = sh.stack[top - 1];
    --top;
    __syncwarp();
    if (n_end[node] <= pos + 1) continue;  // every partner precedes u in Morton order
    const TNode t = load_node(tn, node);
    ++visits;
    if (t.left != kInvalid32) {
      if (nw >= need) {
        const float lx = (float)((double)t.lo[0] - u.x), ly = (float)((double)t.lo[1] - u.y),
                    lz = (float)((double)t.lo[2] - u.z);
        const float hx = (float)((double)t.hi[0] - u.x), hy = (float)((double)t.hi[1] - u.y),
                    hz = (float)((double)t.hi[2] - u.z);
        // max over v in box of (w-u).(w-v) = sum_i a_i (a_i - (a_i >= 0 ? lo_i : hi_i)), a = w - u
        auto inside = [&](float ax, float ay, float az, bool valid) {
          const float tx = ax * (ax - (ax >= 0.f ? lx : hx));
          const float ty = ay * (ay - (ay >= 0.f ? ly : hy));
          const float tz = az * (az - (az >= 0.f ? lz : hz));
          const float mag = fabsf(tx) + fabsf(ty) + fabsf(tz) + ax * ax + ay * ay + az * az;
          return valid && (tx + ty + tz < -1e-5f * mag);
        };
        const uint32_t cnt = __popc(__ballot_sync(0xffffffffu, inside(ax0, ay0, az0, w0 != kInvalid32))) +
                             __popc(__ballot_sync(0xffffffffu, inside(ax1, ay1, az1, w1 != kInvalid32)));
        if (cnt >= need) continue;
      }
      if (top + 2 > kStack) {
        if (lane == 0) atomicOr(err, kErrCapacity);
        return;
      }
      if (lane == 0) {
        sh.stack[top] = t.right;
        sh.stack[top + 1] = t.left;
      }
      top += 2;
      __syncwarp();
      continue;
    }
    const uint32_t iv = t.right;
    const Pt v = point(px, py, pz, iv);
    const double d2 = d2fp(u.x, u.y, u.z, v.x, v.y, v.z);
    WarpBall b{0u, 0u, kInvalid32, false};
    if (d2 * hi < r2u * lo) {
      ++local_pairs;
      warp_classify(b, sh, w0, w1, iu, iv, u, v, px, py, pz, S, cap);
    } else if (d2 * hi < R2[iv] * lo) {
      ++local_pairs;
      const uint32_t v0 = W[(uint64_t)iv * kW + lane], v1 = W[(uint64_t)iv * kW + 32 + lane];
      warp_classify(b, sh, v0, v1, iu, iv, u, v, px, py, pz, S, cap);
    } else {
      // witnesses of u strictly inside this one sphere: enough of them rejects
      // the pair without a global query
      auto strictly_inside = [&](uint32_t w, float ax, float ay, float az) {
        if (w == kInvalid32 || w == iv) return false;
        const double dx = (double)ax, dy = (double)ay, dz = (double)az;  // w - u (binary32-rounded)
        const double vx = v.x - u.x, vy = v.y - u.y, vz = v.z - u.z;
        // (w-u).(w-v) = |a|^2 - a.(v-u); margin covers the binary32 rounding of a
        const double aa = dx * dx + dy * dy + dz * dz, av = dx * vx + dy * vy + dz * vz;
        return aa - av < -1e-5 * (aa + fabs(dx * vx) + fabs(dy * vy) + fabs(dz * vz));
      };
      const uint32_t inside = __popc(__ballot_sync(0xffffffffu, strictly_inside(w0, ax0, ay0, az0))) +
                              __popc(__ballot_sync(0xffffffffu, strictly_inside(w1, ax1, ay1, az1)));
      if (inside >= need) continue;
      ++ball_queries;
      warp_ball_query(b, sh, iu, iv, u, v, root, tn, leaf_pid, n_begin, n_end, px, py, pz, S, cap, err, ball_nodes);
    }
    __syncwarp();
    if (b.rejected || b.interior > cap) continue;
    ++emitted;
    if (lane == 0) {
      const uint32_t slot = atomicAdd(counters, 1u);
      if (slot < out_cap) {
        PairRec r;
        r.u = min(iu, iv);
        r.v = max(iu, iv);
        r.interior = b.interior;
        r.shell = b.shell + 2;
        r.witness = b.witness;
        for (uint32_t j = 0; j < kMaxInterior; ++j) r.ids[j] = j < b.interior ? sh.ids[j] : kInvalid32;
        for (uint32_t a = 1; a < b.interior; ++a) {  // ascending interior ids
          const uint32_t x = r.ids[a];
          uint32_t j = a;
          while (j > 0 && r.ids[j - 1] > x) { r.ids[j] = r.ids[j - 1]; --j; }
          r.ids[j] = x;
        }
        r.pad[0] = r.pad[1] = 0;
        out[slot] = r;
      }
    }
    __syncwarp();
  }
  if (lane == 0) {
    atomicAdd(stats + 0, visits);
    atomicAdd(stats + 1, local_pairs);
    atomicAdd(stats + 2, ball_queries);
    atomicAdd(stats + 3, ball_nodes);
    atomicAdd(stats + 4, emitted);
  }
}

__global__ void __launch_bounds__(256)
k_pair_keys(uint32_t m, const PairRec* __restrict__ recs, uint64_t* __restrict__ key, uint32_t* __restrict__ order) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  key[i] = ((uint64_t)recs[i].u << 32) | recs[i].v;
  order[i] = i;
}

__global__ void __launch_bounds__(256)
k_pair_gather(uint32_t m, const uint32_t* __restrict__ vals0, const uint32_t* __restrict__ vals1,
              const uint32_t* __restrict__ state, int passes, const PairRec* __restrict__ recs,
              PairRec* __restrict__ sorted, const double* __restrict__ px, const double* __restrict__ py,
              const double* __restrict__ pz, const int* __restrict__ scale, uint64_t* __restrict__ levelD) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const PairRec r = recs[radix_result(state, passes, vals0, vals1)[i]];
  sorted[i] = r;
  const int S = scale[0];
  __int128 a[3], b[3];
  const double* P[3] = {px, py, pz};
  for (int k = 0; k < 3; ++k) {
    a[k] = fixed_of(dbits(P[k][r.u]), S);
    b[k] = fixed_of(dbits(P[k][r.v]), S);
  }
  const WInt<4> D = exact_dist2(a, b);
  for (int w = 0; w < 4; ++w) levelD[4ull * i + w] = D.w[w];
}

}  // namespace

// Bytes of each record buffer for `c` records: raw, sorted, key, order0, order1, levelD, radix counts.
static void pair_record_bytes(uint64_t c, uint64_t* b) {
  b[0] = c * sizeof(PairRec);
  b[1] = c * sizeof(PairRec);
  b[2] = c * sizeof(uint64_t);
  b[3] = c * sizeof(uint32_t);
  b[4] = c * sizeof(uint32_t);
  b[5] = c * 4 * sizeof(uint64_t);
  b[6] = 256ull * ((c + kRadixTile - 1) / kRadixTile) * sizeof(uint32_t);
}

cudaError_t pairs_records_alloc(Ctx& ctx, uint64_t capacity) {
  PairBuffers& p = ctx.pb;
  void** bufs[7] = {&p.raw, &p.sorted, (void**)&p.key, (void**)&p.order0, (void**)&p.order1, (void**)&p.levelD,
                    (void**)&p.radix_counts};
  uint64_t old_b[7], new_b[7];
  pair_record_bytes(p.capacity, old_b);
  pair_record_bytes(capacity, new_b);
  for (int i = 0; i < 7; ++i) {
    ctx_free(ctx, *bufs[i], old_b[i]);
    *bufs[i] = nullptr;
  }
  p.capacity = 0;
  for (int i = 0; i < 7; ++i) {
    const cudaError_t e = ctx_alloc(ctx, bufs[i], new_b[i]);
    if (e != cudaSuccess) {
      for (int j = 0; j < i; ++j) {
        ctx_free(ctx, *bufs[j], new_b[j]);
        *bufs[j] = nullptr;
      }
      return e;
    }
  }
  p.capacity = (uint32_t)capacity;
  return cudaSuccess;
}

cudaError_t pairs_alloc(Ctx& ctx) {
  const uint64_t n = ctx.max_points;
  PairBuffers& p = ctx.pb;
  cudaError_t e = cudaSuccess;
#define EHGP_ALLOC(ptr, bytes) \
  if ((e = ctx_alloc(ctx, (void**)&(ptr), (bytes))) != cudaSuccess) return e
  EHGP_ALLOC(p.W, n * kW * sizeof(uint32_t));
  EHGP_ALLOC(p.R2, n * sizeof(double));
  EHGP_ALLOC(p.counters, 8 * sizeof(uint32_t));
  EHGP_ALLOC(p.stats, 8 * sizeof(unsigned long long));
#undef EHGP_ALLOC
  // records: about 38 per point in lattices and uniform clouds; grown on demand
  return pairs_records_alloc(ctx, 48 * n + 1024);
}

// Witness lists + pair enumeration + (u, v) sort.  Returns the record count
// (or a status through ctx on failure).
int pairs_run(Ctx& ctx, uint32_t K, uint32_t* out_count) {
  const uint32_t n = (uint32_t)ctx.built_n;
  PairBuffers& p = ctx.pb;
  LbvhBuffers& b = ctx.lb;
  GeomBuffers& g = ctx.gb;
  cudaStream_t st = ctx.stream;
  const uint32_t keff = K < n ? K : n;
  const uint32_t smax = (keff + 1 < n) ? keff + 1 : n;
  *out_count = 0;
  p.count = 0;
  p.resident = false;
  ++ctx.pair_runs;
  if (smax < 2 || n < 2) {
    p.K = K;
    p.resident = true;
    return EHGP_OK;
  }
  const uint32_t cap = smax - 2;
  if (cap > (uint32_t)kMaxInterior) return abi_fail(&ctx, EHGP_ERR_INVALID_ARGUMENT, "K above 10 is not supported");
  const uint32_t root = 2 * n - 2;
  const uint32_t kw = (n - 1 < (uint32_t)kW) ? n - 1 : (uint32_t)kW;
  uint64_t launches = 0;
  cudaEventRecord(ctx.ev0, st);
  k_witness_knn<<<nblocks(n), kThreads, 0, st>>>(n, kw, root, g.tnodes, b.leaf_pid, b.px, b.py, b.pz, p.W, p.R2,
                                                  ctx.d_err);
  ++launches;
  uint32_t hc[2] = {0, 0};
  cudaError_t e = cudaSuccess;
  // count -> allocate -> emit: the enumeration counts every record and writes those that fit;
  // when the count exceeds the buffer, the buffer grows to it and the enumeration runs again
  for (int attempt = 0; attempt < 2; ++attempt) {
    cudaMemsetAsync(p.counters, 0, 8 * sizeof(uint32_t), st);
    cudaMemsetAsync(p.stats, 0, 8 * sizeof(unsigned long long), st);
    cudaEventRecord(ctx.evk0, st);
    k_pairs<<<nblocks(n, kWarpsPerBlock), kThreads, 0, st>>>(n, cap, root, g.tnodes, b.leaf_pid, b.n_begin, b.n_end,
                                                             b.px, b.py, b.pz, g.scale, p.W, p.R2, (PairRec*)p.raw,
                                                             p.capacity, p.counters, p.stats, ctx.d_err);
    cudaEventRecord(ctx.evk1, st);
    ++launches;
    unsigned long long hs[8];
    cudaMemcpyAsync(hc, p.counters, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(hc + 1, ctx.d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(hs, p.stats, sizeof(hs), cudaMemcpyDeviceToHost, st);
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return abi_cuda_fail(&ctx, e, "pair enumeration");
    {
      float kms = 0.f;
      cudaEventElapsedTime(&kms, ctx.evk0, ctx.evk1);
      ctx.kernel_ms = kms;
      for (int i = 0; i < 8; ++i) ctx.kernel_stats[i] = hs[i];
    }
    if (hc[1]) return abi_device_status(&ctx, hc[1]);
    if (hc[0] <= p.capacity) break;
    if (attempt == 1 || (uint64_t)hc[0] >= 0xffff0000ull)
      return abi_fail(&ctx, EHGP_ERR_CAPACITY, "pair-support records exceed 32-bit record indices");
    if ((e = pairs_records_alloc(ctx, grown_capacity(hc[0]))) != cudaSuccess) {
      cudaGetLastError();
      return abi_fail(&ctx, EHGP_ERR_OUT_OF_MEMORY, "the pair-support records do not fit the device");
    }
    ++ctx.regrowths;
  }
  const uint32_t m = hc[0];
  if (m) {
    k_pair_keys<<<(m + 255) / 256, 256, 0, st>>>(m, (const PairRec*)p.raw, p.key, p.order0);
    RadixScratch rs{p.radix_counts, ctx.radix.state, (uint32_t)((p.capacity + kRadixTile - 1) / kRadixTile)};
    const IndirectKey stage[1] = {{p.key, 0}};
    const int bits[1] = {64};
    const int passes = radix_sort_indirect(st, m, p.order0, p.order1, stage, bits, 1, rs, &launches);
    k_pair_gather<<<(m + 255) / 256, 256, 0, st>>>(m, p.order0, p.order1, ctx.radix.state, passes,
                                                    (const PairRec*)p.raw, (PairRec*)p.sorted, b.px, b.py, b.pz,
                                                    g.scale, p.levelD);
    launches += 2;
  }
  cudaEventRecord(ctx.ev1, st);
  cudaMemcpyAsync(hc + 1, ctx.d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return abi_cuda_fail(&ctx, e, "pair sort");
  if (hc[1]) return abi_device_status(&ctx, hc[1]);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ctx.ev0, ctx.ev1);
  ctx.last_ms = ms;
  ctx.last_launches = launches;
  p.count = m;
  p.K = K;
  p.witness_ready = true;
  p.resident = true;
  *out_count = m;
  return EHGP_OK;
}

}  // namespace ehgp

extern "C" {

int ehgp_pairs(ehgp_ctx* ctx, uint32_t K, const ehgp_pairs_out* out) {
  if (!ctx) return EHGP_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(ctx->mutex);
  ctx->last_error.clear();
  if (ctx->poisoned) return ehgp::abi_fail(ctx, EHGP_ERR_POISONED, "the context is poisoned by an earlier CUDA failure");
  if (ctx->built_n == 0) return ehgp::abi_fail(ctx, EHGP_ERR_NOT_BUILT, "ehgp_pairs needs a resident LBVH");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return ehgp::abi_cuda_fail(ctx, e, "cudaSetDevice");
  if (!ctx->geom_ready) {
    ehgp::geom_prepare(*ctx, (uint32_t)ctx->built_n);
    if ((e = cudaGetLastError()) != cudaSuccess) return ehgp::abi_cuda_fail(ctx, e, "traversal preparation");
  }
  if (!ctx->scale_valid)
    return ehgp::abi_fail(ctx, EHGP_ERR_NUMERIC_RANGE, "the cloud exceeds the exact fixed-point range");
  cudaMemsetAsync(ctx->d_err, 0, sizeof(uint32_t), ctx->stream);
  uint32_t m = 0;
  const int s = ehgp::pairs_run(*ctx, K, &m);
  if (s != EHGP_OK) return s;
  if (out && out->count) *out->count = m;
  if (out && out->records && m) {
    if (out->capacity < m) return ehgp::abi_fail(ctx, EHGP_ERR_CAPACITY, "the output capacity is below the record count");
    e = cudaMemcpy(out->records, ctx->pb.sorted, (uint64_t)m * 64, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && out->level_num)
      e = cudaMemcpy(out->level_num, ctx->pb.levelD, (uint64_t)m * 32, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return ehgp::abi_cuda_fail(ctx, e, "pair copy");
  }
  return EHGP_OK;
}

}  // extern "C"
