// Triple and quad critical-sphere supports (rank <= s_max) on sm_100a.
//
// Reference semantics (Ludwig-H/E-HGP, morsehgp3d/):
//  build_exact_higher_support_stream (include/morsehgp3d/hierarchy/higher_support_stream.hpp:544),
//  leaf rule classify_terminal_support (src/cpu/hierarchy/higher_support_stream.cpp:1992-2110)
//  with exact::analyze_circumcenter_support (include/morsehgp3d/exact/support.hpp:41,474-479):
//   * only MINIMAL supports count: affinely independent, circumcentre strictly
//     inside the convex hull of the support (for a triangle: three acute
//     angles; for a tetrahedron: four positive barycentric coordinates);
//   * relevant iff interior + size <= s_max; an event iff the exact shell is
//     the support itself, else an extra-shell diagnostic;
//   * records ordered by (size, support ids) (support_record_less, :84-95).
//
// B200 design (replacing the reference's CPU branch-and-bound over LBVH node
// triples/quads with interval Gram/Cramer bounds):
//  1. Direction table.  Any sphere through a point a is the tangent ball
//     B(a + r u, r); a point p lies strictly inside it as soon as
//     r > rho_p(u) = |p - a| / (2 cos angle(u, p - a)), and tangent balls with the
//     same u are nested.  A relevant sphere of size >= 3 has at most s_max - 3
//     strict interior points, so r <= the (s_max-2)-th smallest rho_p(u).  Over
//     642 sampled directions s (covering angle delta), caps shrunk by delta give
//     a bound rho_s(a) valid in the whole cone of s, further capped by the AABB
//     support function (a well-centred sphere has a support point p with
//     (p - a).u >= r).  See k_dirtable for the derivation.
//  2. Candidate set C(a): the points whose lowest threshold in some cone is at
//     most rho_s(a).  It holds every support, shell and interior point of every
//     relevant sphere through a, and enough interior points of every other
//     well-centred sphere to reject it.  Every support is enumerated once, by
//     its least PointId a, from C(a), and classified exactly against C(a).
//  3. Exact predicates: FP64 with a tracked error bound, then 832-bit integers
//     at the cloud scale inside the bound.
#include "ehgp_internal.cuh"
#include "ehgp_exact.cuh"

#include <array>
#include <cmath>
#include <cstring>
#include <vector>

namespace ehgp {
namespace {

constexpr int kMaxNb = 1024;    // neighbour list capacity per point
constexpr int kDirs = 642;      // direction samples (icosphere, 3 subdivisions)
constexpr int kWarps = 4;       // warps per block
constexpr int kThreads = 32 * kWarps;
constexpr int kQueue = 1024;
constexpr int kMaxInteriorH = 8;  // s_max - 3 for K = 10
constexpr double kU = 1.1102230246251565e-16;

__host__ __device__ inline uint32_t nblocks(uint64_t n, int t) {
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

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// ---- FP64 values with a magnitude bound (error <= 64 u m) -------------------------
struct Fm {
  double v, m;
};
__device__ __forceinline__ Fm operator+(Fm a, Fm b) { return {a.v + b.v, a.m + b.m}; }
__device__ __forceinline__ Fm operator-(Fm a, Fm b) { return {a.v - b.v, a.m + b.m}; }
__device__ __forceinline__ Fm operator*(Fm a, Fm b) { return {a.v * b.v, a.m * b.m}; }
__device__ __forceinline__ int fm_sign(Fm x) {
  const double bound = 64.0 * kU * x.m + 1e-300;
  return x.v > bound ? 1 : (x.v < -bound ? -1 : 2);
}
struct FV {
  Fm x, y, z;
};
__device__ __forceinline__ Fm dot(const FV& a, const FV& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ FV cross(const FV& a, const FV& b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ FV scale(Fm s, const FV& a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ FV add(const FV& a, const FV& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }

struct P3 {
  double x, y, z;
};
__device__ __forceinline__ FV fdiff(const P3& p, const P3& q) {
  return {{p.x - q.x, fabs(p.x) + fabs(q.x)}, {p.y - q.y, fabs(p.y) + fabs(q.y)}, {p.z - q.z, fabs(p.z) + fabs(q.z)}};
}

// ---- exact versions (832-bit integers at the cloud scale) --------------------------
using W = WInt<13>;
struct WV {
  W x, y, z;
};
__device__ __forceinline__ W wdot(const WV& a, const WV& b) {
  return wadd(wadd(wmul(a.x, b.x), wmul(a.y, b.y)), wmul(a.z, b.z));
}
__device__ __forceinline__ WV wcross(const WV& a, const WV& b) {
  return {wsub(wmul(a.y, b.z), wmul(a.z, b.y)), wsub(wmul(a.z, b.x), wmul(a.x, b.z)),
          wsub(wmul(a.x, b.y), wmul(a.y, b.x))};
}
__device__ __forceinline__ WV wscale(const W& s, const WV& a) { return {wmul(s, a.x), wmul(s, a.y), wmul(s, a.z)}; }
__device__ __forceinline__ WV wvadd(const WV& a, const WV& b) { return {wadd(a.x, b.x), wadd(a.y, b.y), wadd(a.z, b.z)}; }

struct Cloud {
  const double* px;
  const double* py;
  const double* pz;
  int S;
  __device__ P3 p(uint32_t i) const { return P3{px[i], py[i], pz[i]}; }
  __device__ WV wdiff(uint32_t i, uint32_t j) const {
    return {W::from_i128(fixed_of(dbits(px[i]), S) - fixed_of(dbits(px[j]), S)),
            W::from_i128(fixed_of(dbits(py[i]), S) - fixed_of(dbits(py[j]), S)),
            W::from_i128(fixed_of(dbits(pz[i]), S) - fixed_of(dbits(pz[j]), S))};
  }
};

// A support's side polynomial: side(w) = sgn * sign(A |p|^2 - p.N), p = w - a.
struct Sphere {
  uint32_t ids[4];
  int size;
  int status;  // 0 minimal, 1 boundary reduced, 2 exterior centre, 3 dependent, 4 undecided in FP
  Fm A;
  FV N;
  int sgn;
  double r2_lo, r2_hi;  // FP bounds of the squared radius (valid when status == 0)
};

__device__ void radius_bounds(Sphere& s) {
  // r^2 = |N|^2 / (4 A^2) with |error| of every quantity <= 64 u m
  const double g = 64.0 * kU;
  const double a_lo = fabs(s.A.v) - g * s.A.m, a_hi = fabs(s.A.v) + g * s.A.m;
  double n_lo = 0, n_hi = 0;
  const Fm c[3] = {s.N.x, s.N.y, s.N.z};
  for (int i = 0; i < 3; ++i) {
    const double lo = fmax(fabs(c[i].v) - g * c[i].m, 0.0), hi = fabs(c[i].v) + g * c[i].m;
    n_lo += lo * lo;
    n_hi += hi * hi;
  }
  if (a_lo <= 0) {
    s.r2_lo = 0;
    s.r2_hi = INFINITY;
  } else {
    s.r2_lo = n_lo / (4 * a_hi * a_hi) * (1 - 1e-12);
    s.r2_hi = n_hi / (4 * a_lo * a_lo) * (1 + 1e-12);
  }
}

// Status of a triangle: minimal iff its three angles are acute.
__device__ int tri_status(const Cloud& c, const uint32_t* id, Sphere& s) {
  const P3 a = c.p(id[0]), b = c.p(id[1]), d = c.p(id[2]);
  const FV e1 = fdiff(b, a), e2 = fdiff(d, a);
  const Fm G11 = dot(e1, e1), G12 = dot(e1, e2), G22 = dot(e2, e2);
  const Fm db = G11 - G12, dc = G22 - G12;
  const Fm detG = G11 * G22 - G12 * G12;
  int sa = fm_sign(G12), sb = fm_sign(db), sc = fm_sign(dc), sd = fm_sign(detG);
  if (sa == 2 || sb == 2 || sc == 2 || sd == 2) {
    const WV w1 = c.wdiff(id[1], id[0]), w2 = c.wdiff(id[2], id[0]);
    const W g11 = wdot(w1, w1), g12 = wdot(w1, w2), g22 = wdot(w2, w2);
    sa = g12.sign();
    sb = wsub(g11, g12).sign();
    sc = wsub(g22, g12).sign();
    sd = wsub(wmul(g11, g22), wmul(g12, g12)).sign();
  }
  if (sd == 0) return 3;
  if (sa < 0 || sb < 0 || sc < 0) return 2;
  if (sa == 0 || sb == 0 || sc == 0) return 1;
  s.A = detG;
  s.N = add(scale(G22 * db, e1), scale(G11 * dc, e2));
  s.sgn = 1;
  return 0;
}

// Status of a tetrahedron: minimal iff the four barycentric coordinates of its
// circumcentre are positive.
__device__ int quad_status(const Cloud& c, const uint32_t* id, Sphere& s) {
  const P3 a = c.p(id[0]);
  const FV e1 = fdiff(c.p(id[1]), a), e2 = fdiff(c.p(id[2]), a), e3 = fdiff(c.p(id[3]), a);
  const FV c23 = cross(e2, e3), c31 = cross(e3, e1), c12 = cross(e1, e2);
  const Fm detE = dot(e1, c23);
  const FV N = add(add(scale(dot(e1, e1), c23), scale(dot(e2, e2), c31)), scale(dot(e3, e3), c12));
  const Fm l1 = dot(N, c23), l2 = dot(N, c31), l3 = dot(N, c12);
  const Fm l0 = Fm{2.0, 0.0} * detE * detE - (l1 + l2 + l3);
  int sd = fm_sign(detE), s0 = fm_sign(l0), s1 = fm_sign(l1), s2 = fm_sign(l2), s3 = fm_sign(l3);
  if (sd == 2 || s0 == 2 || s1 == 2 || s2 == 2 || s3 == 2) {
    const WV w1 = c.wdiff(id[1], id[0]), w2 = c.wdiff(id[2], id[0]), w3 = c.wdiff(id[3], id[0]);
    const WV x23 = wcross(w2, w3), x31 = wcross(w3, w1), x12 = wcross(w1, w2);
    const W de = wdot(w1, x23);
    const WV nn = wvadd(wvadd(wscale(wdot(w1, w1), x23), wscale(wdot(w2, w2), x31)), wscale(wdot(w3, w3), x12));
    const W m1 = wdot(nn, x23), m2 = wdot(nn, x31), m3 = wdot(nn, x12);
    const W two = W::from_i128(2);
    const W m0 = wsub(wmul(two, wmul(de, de)), wadd(wadd(m1, m2), m3));
    sd = de.sign();
    s0 = m0.sign(); s1 = m1.sign(); s2 = m2.sign(); s3 = m3.sign();
  }
  if (sd == 0) return 3;
  if (s0 < 0 || s1 < 0 || s2 < 0 || s3 < 0) return 2;
  if (s0 == 0 || s1 == 0 || s2 == 0 || s3 == 0) return 1;
  s.A = detE;
  s.N = N;
  s.sgn = sd;
  return 0;
}

// Exact side of w: -1 strictly inside, 0 on the sphere, +1 outside.
__device__ int sphere_side(const Cloud& c, const Sphere& s, uint32_t w) {
  const FV p = fdiff(c.p(w), c.p(s.ids[0]));
  const int fs = fm_sign(s.A * dot(p, p) - dot(p, s.N));
  if (fs != 2) return fs * s.sgn;
  const WV q = c.wdiff(w, s.ids[0]);
  W val;
  if (s.size == 3) {
    const WV w1 = c.wdiff(s.ids[1], s.ids[0]), w2 = c.wdiff(s.ids[2], s.ids[0]);
    const W g11 = wdot(w1, w1), g12 = wdot(w1, w2), g22 = wdot(w2, w2);
    const W detG = wsub(wmul(g11, g22), wmul(g12, g12));
    const WV n = wvadd(wscale(wmul(g22, wsub(g11, g12)), w1), wscale(wmul(g11, wsub(g22, g12)), w2));
    val = wsub(wmul(detG, wdot(q, q)), wdot(q, n));
  } else {
    const WV w1 = c.wdiff(s.ids[1], s.ids[0]), w2 = c.wdiff(s.ids[2], s.ids[0]), w3 = c.wdiff(s.ids[3], s.ids[0]);
    const WV x23 = wcross(w2, w3), x31 = wcross(w3, w1), x12 = wcross(w1, w2);
    const W de = wdot(w1, x23);
    const WV nn = wvadd(wvadd(wscale(wdot(w1, w1), x23), wscale(wdot(w2, w2), x31)), wscale(wdot(w3, w3), x12));
    val = wsub(wmul(de, wdot(q, q)), wdot(q, nn));
  }
  return val.sign() * s.sgn;
}

// ---- 1. neighbour lists ------------------------------------------------------------------
// Every point within the gather radius of a (FP64 superset); overflow sets
// count = kMaxNb + 1.
__global__ void __launch_bounds__(kThreads)
k_gather(uint32_t n, uint32_t root, const TNode* __restrict__ tn, const uint32_t* __restrict__ leaf_pid,
         const uint32_t* __restrict__ n_begin, const uint32_t* __restrict__ n_end, const double* __restrict__ px,
         const double* __restrict__ py, const double* __restrict__ pz, const double* __restrict__ gather_r2,
         const uint8_t* __restrict__ todo, uint32_t* __restrict__ nb, uint32_t* __restrict__ nbc) {
  __shared__ uint32_t queue[kWarps][kQueue];
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  const uint32_t pos = blockIdx.x * kWarps + warp;
  if (pos >= n) return;
  const uint32_t a = leaf_pid[pos];
  if (!todo[a]) return;
  const double ax = px[a], ay = py[a], az = pz[a];
  const double R2 = gather_r2[a] * (1.0 + 32.0 * kU);
  uint32_t* out = nb + (uint64_t)a * kMaxNb;
  uint32_t count = 0, head = 0, tail = 1;
  bool overflow = false;
  if (lane == 0) queue[warp][0] = root;
  __syncwarp();
  while (head < tail && !overflow) {
    const uint32_t batch = min(tail - head, 32u);
    uint32_t node = kInvalid32;
    if (lane < batch) node = queue[warp][(head + lane) & (kQueue - 1)];
    __syncwarp();
    bool take = false, expand = false;
    uint32_t pid = kInvalid32, bb = 0, be = 0;
    TNode t;
    if (node != kInvalid32) {
      t = load_node(tn, node);
      if (t.left == kInvalid32) {
        pid = t.right;
        const double dx = px[pid] - ax, dy = py[pid] - ay, dz = pz[pid] - az;
        take = pid != a && dx * dx + dy * dy + dz * dz <= R2;
      } else {
        const double lx = fmax(fmax((double)t.lo[0] - ax, ax - (double)t.hi[0]), 0.0);
        const double ly = fmax(fmax((double)t.lo[1] - ay, ay - (double)t.hi[1]), 0.0);
        const double lz = fmax(fmax((double)t.lo[2] - az, az - (double)t.hi[2]), 0.0);
        if ((lx * lx + ly * ly + lz * lz) * (1.0 - 16.0 * kU) <= R2) {
          const double ux = fmax(fabs((double)t.lo[0] - ax), fabs((double)t.hi[0] - ax));
          const double uy = fmax(fabs((double)t.lo[1] - ay), fabs((double)t.hi[1] - ay));
          const double uz = fmax(fabs((double)t.lo[2] - az), fabs((double)t.hi[2] - az));
          if ((ux * ux + uy * uy + uz * uz) * (1.0 + 16.0 * kU) < R2) {
            bb = n_begin[node];
            be = n_end[node];
          } else {
            expand = true;
          }
        }
      }
    }
    // single points
    const uint32_t tb = __ballot_sync(0xffffffffu, take);
    if (take) {
      const uint32_t at = count + __popc(tb & lanemask_lt());
      if (at < kMaxNb) out[at] = pid;
    }
    count += __popc(tb);
    // whole subtrees inside the radius (a itself may be in them)
    uint32_t bulk = be - bb;
    uint32_t before = bulk;
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t x = __shfl_up_sync(0xffffffffu, before, off);
      if ((int)lane >= off) before += x;
    }
    uint32_t total = __shfl_sync(0xffffffffu, before, 31);
    before -= bulk;
    // a's own leaf inside a bulk range: count the lanes holding it
    bool holds_a = false;
    uint32_t skip_before = 0;
    {
      // positions are Morton positions; a sits at position pos
      holds_a = (bulk > 0 && pos >= bb && pos < be);
      const uint32_t hb = __ballot_sync(0xffffffffu, holds_a);
      skip_before = __popc(hb & lanemask_lt());
      total -= __popc(hb);
    }
    uint32_t w = count + before - skip_before;
    for (uint32_t q = bb; q < be; ++q) {
      if (q == pos) continue;
      if (w < kMaxNb) out[w] = leaf_pid[q];
      ++w;
    }
    count += total;
    if (count > kMaxNb) overflow = true;
    const uint32_t eb = __ballot_sync(0xffffffffu, expand);
    const uint32_t pushes = 2 * __popc(eb);
    if (tail - head - batch + pushes > kQueue) { overflow = true; break; }
    if (expand) {
      const uint32_t at = tail + 2 * __popc(eb & lanemask_lt());
      queue[warp][at & (kQueue - 1)] = t.left;
      queue[warp][(at + 1) & (kQueue - 1)] = t.right;
    }
    __syncwarp();
    head += batch;
    tail += pushes;
  }
  if (lane == 0) nbc[a] = overflow ? (uint32_t)kMaxNb + 1 : count;
}

// ---- 2. direction table and candidate set --------------------------------------------
// For owner a and sampled direction s (cone of half-angle delta):
//   rho_shr_p(s) = |p - a| / (2 cos(angle(s, p - a) + delta))  >= rho_p(u) for u in the cone
//   rho_lo_p(s)  = |p - a| / (2 cos(max(angle(s, p - a) - delta, 0)))  <= rho_p(u)
//   rho_s(a)     = min((s_max - 2)-th smallest rho_shr_p(s), ext_s)
// where ext_s bounds the AABB support function over the cone.  A relevant
// sphere through a with centre direction u in the cone of s has
// r <= rho_(s_max-2)(u) <= rho_s(a), so each of its support, shell and strictly
// interior points p has rho_lo_p(s) <= rho_p(u) <= r <= rho_s(a): the candidate
// set C(a) = {p : rho_lo_p(s) <= rho_s(a) for some s} holds them all.  A
// well-centred sphere through a that is NOT relevant has r <= ext_s and at
// least s_max - 2 points with rho_p(u) < r whose thresholds are the smallest at
// u; those lie in C(a) too, so classifying against C(a) rejects it.
// The neighbour list (points within the gather radius L, sorted by distance)
// certifies rho_s when rho_s <= L / 2: every unlisted point has rho >= L / 2.
constexpr int kDirWarps = 2;
constexpr int kMaxCand = 256;  // candidate-set capacity per point

struct CertParams {
  const float* dirs;  // [kDirs * 3] unit vectors
  double delta;       // covering angle of the directions (radians)
  double lo[3], hi[3];  // cloud AABB
  uint32_t need;        // s_max - 2
};

__global__ void __launch_bounds__(32 * kDirWarps)
k_dirtable(uint32_t n, CertParams cp, const uint32_t* __restrict__ leaf_pid, uint32_t* __restrict__ nb,
           const uint32_t* __restrict__ nbc, const double* __restrict__ px, const double* __restrict__ py,
           const double* __restrict__ pz, const double* __restrict__ gather_r2, uint8_t* __restrict__ todo,
           uint32_t* __restrict__ cand, uint32_t* __restrict__ candc, double* __restrict__ need_r) {
  __shared__ float4 rel[kDirWarps][kMaxNb];  // x, y, z, |p - a| (binary32 copies; margins below)
  __shared__ uint32_t ids[kDirWarps][kMaxNb];
  __shared__ uint32_t mark[kDirWarps][kMaxNb / 32];
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  const uint32_t pos = blockIdx.x * kDirWarps + warp;
  if (pos >= n) return;
  const uint32_t a = leaf_pid[pos];
  if (!todo[a]) return;
  const uint32_t m = nbc[a];
  if (m > (uint32_t)kMaxNb) {
    if (lane == 0) need_r[a] = INFINITY;
    return;
  }
  const double ax = px[a], ay = py[a], az = pz[a];
  for (uint32_t i = lane; i < m; i += 32) {
    const uint32_t p = nb[(uint64_t)a * kMaxNb + i];
    const double x = px[p] - ax, y = py[p] - ay, z = pz[p] - az;
    rel[warp][i] = make_float4((float)x, (float)y, (float)z, (float)sqrt(x * x + y * y + z * z));
    ids[warp][i] = p;
  }
  for (uint32_t i = lane; i < (uint32_t)kMaxNb / 32; i += 32) mark[warp][i] = 0;
  __syncwarp();
  // sort by distance (odd-even merge sort over a power-of-two padding, in shared memory)
  uint32_t P = 1;
  while (P < m) P <<= 1;
  for (uint32_t i = m + lane; i < P; i += 32) {
    rel[warp][i] = make_float4(0.f, 0.f, 0.f, INFINITY);
    ids[warp][i] = kInvalid32;
  }
  __syncwarp();
  for (uint32_t k = 2; k <= P; k <<= 1) {
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      for (uint32_t i = lane; i < P; i += 32) {
        const uint32_t l = i ^ j;
        if (l > i) {
          const bool up = (i & k) == 0;
          const float4 x = rel[warp][i], y = rel[warp][l];
          if ((x.w > y.w) == up) {
            rel[warp][i] = y;
            rel[warp][l] = x;
            const uint32_t t = ids[warp][i];
            ids[warp][i] = ids[warp][l];
            ids[warp][l] = t;
          }
        }
      }
      __syncwarp();
    }
  }
  // distances are binary32: thresholds carry a relative margin of 1e-5 in the safe direction
  const double L2 = sqrt(gather_r2[a]) * (1.0 - 1e-9);  // list covers |p - a| <= L
  const double half_L = 0.5 * L2;
  const double cd = cos(cp.delta), sdl = sin(cp.delta);
  const double A[3] = {ax, ay, az};
  double worst_needed = 0.0;  // largest certified rho_s (the list must cover 2 rho_s)
  bool ok = true;
  for (int d = lane; d < kDirs; d += 32) {
    const double s0 = cp.dirs[3 * d], s1 = cp.dirs[3 * d + 1], s2 = cp.dirs[3 * d + 2];
    // AABB support bound over the cone
    double ext = 0.0;
    const double sv[3] = {s0, s1, s2};
    for (int k = 0; k < 3; ++k) {
      const double up = cp.hi[k] - A[k], dn = cp.lo[k] - A[k];
      const double t1 = sv[k] - cp.delta, t2 = sv[k] + cp.delta;
      const double f1 = t1 >= 0 ? up * t1 : dn * t1, f2 = t2 >= 0 ? up * t2 : dn * t2;
      ext += fmax(f1, f2);
    }
    ext *= (1.0 + 1e-12);
    // the centre of a well-centred sphere lies in conv(S), inside the AABB: r is at most
    // the distance at which the ray a + r u leaves the AABB, maximised over the cone
    // axis by axis (min over axes of the per-axis maxima bounds the max of the min)
    for (int k = 0; k < 3; ++k) {
      const double t1 = sv[k] - cp.delta, t2 = sv[k] + cp.delta;
      if (t1 <= 0.0 && t2 >= 0.0) continue;  // the cone crosses this axis' zero: no bound
      const double g = t1 > 0.0 ? (cp.hi[k] - A[k]) / t1 : (A[k] - cp.lo[k]) / (-t2);
      ext = fmin(ext, g * (1.0 + 1e-12));
    }
    // the `need` smallest shrunk thresholds (early exit: rho_shr >= |p - a| / 2)
    double best[16];
    uint32_t cnt = 0;
    for (uint32_t i = 0; i < m; ++i) {
      const float4 r = rel[warp][i];
      const double dist = (double)r.w;
      const double kth = cnt >= cp.need ? best[cp.need - 1] : INFINITY;
      if (0.5 * dist * (1.0 - 1e-5) > fmin(kth, ext)) break;
      const double c = (s0 * r.x + s1 * r.y + s2 * r.z) / dist;
      // upper bound of the angle (cosine lowered by the binary32 margin) -> cos(angle + delta) lowered
      const double cs = fmax(-1.0, c - 1e-5), sn = sqrt(fmax(0.0, 1.0 - cs * cs));
      const double cshr = cs * cd - sn * sdl;
      if (cshr <= 1e-9) continue;
      const double rho = dist / (2.0 * cshr) * (1.0 + 1e-5);
      if (cnt < cp.need) {
        uint32_t j = cnt++;
        while (j > 0 && best[j - 1] > rho) { best[j] = best[j - 1]; --j; }
        best[j] = rho;
      } else if (rho < best[cp.need - 1]) {
        uint32_t j = cp.need - 1;
        while (j > 0 && best[j - 1] > rho) { best[j] = best[j - 1]; --j; }
        best[j] = rho;
      }
    }
    const double kth = cnt >= cp.need ? best[cp.need - 1] : INFINITY;
    const double rho_s = fmin(kth, ext);
    // certified when every unlisted point (rho >= L/2) cannot lower it
    if (!(rho_s <= half_L)) ok = false;
    worst_needed = fmax(worst_needed, rho_s);
    // mark the candidates of this cone: rho_lo_p(s) <= rho_s (rho_lo >= |p - a| / 2)
    for (uint32_t i = 0; i < m; ++i) {
      const float4 r = rel[warp][i];
      const double dist = (double)r.w;
      if (0.5 * dist * (1.0 - 1e-5) > rho_s) break;
      const double c = (s0 * r.x + s1 * r.y + s2 * r.z) / dist;
      // lower bound of the angle (cosine raised by the margin) -> cos(max(angle - delta, 0)) raised
      const double cs = fmin(1.0, c + 1e-5);
      const double sn = sqrt(fmax(0.0, 1.0 - cs * cs));
      const double clo = (cs >= cd) ? 1.0 : cs * cd + sn * sdl;
      if (clo <= 0.0) continue;
      const double rho_lo = dist / (2.0 * clo) * (1.0 - 1e-5);
      if (rho_lo <= rho_s * (1.0 + 1e-9)) atomicOr(&mark[warp][i >> 5], 1u << (i & 31));
    }
  }
  ok = __all_sync(0xffffffffu, ok);
  for (int off = 16; off > 0; off >>= 1) worst_needed = fmax(worst_needed, __shfl_xor_sync(0xffffffffu, worst_needed, off));
  __syncwarp();
  if (!ok) {  // the list must grow to 2 rho_s (with room)
    if (lane == 0) need_r[a] = worst_needed;
    return;
  }
  // compact the candidate set in distance order
  uint32_t c = 0;
  uint32_t* out = cand + (uint64_t)a * kMaxCand;
  bool overflow = false;
  for (uint32_t base = 0; base < m; base += 32) {
    const uint32_t i = base + lane;
    const bool f = i < m && ((mark[warp][i >> 5] >> (i & 31)) & 1u);
    const uint32_t b = __ballot_sync(0xffffffffu, f);
    if (f) {
      const uint32_t at = c + __popc(b & lanemask_lt());
      if (at < (uint32_t)kMaxCand) out[at] = ids[warp][i];
    }
    c += __popc(b);
  }
  overflow = c > (uint32_t)kMaxCand;
  if (lane == 0) {
    candc[a] = overflow ? (uint32_t)kMaxCand + 1 : c;
    need_r[a] = worst_needed;
    todo[a] = overflow ? 2 : 0;  // 2: candidate set too large (reported)
  }
}

// ---- 3. owner-local enumeration ---------------------------------------------------------
struct HigherRec {
  uint32_t size;
  uint32_t ids[4];
  uint32_t interior, shell, witness;
  uint32_t iids[kMaxInteriorH];
};
static_assert(sizeof(HigherRec) == 64, "higher-support record is one 64-byte line");

struct Ctl {
  uint32_t smax;
  uint32_t cap;  // record capacity
};

// Classifies every point of the candidate set (support excluded) against s;
// false when the interior exceeds icap.
__device__ bool classify_set(const Cloud& c, const Sphere& s, const uint32_t* set, uint32_t m, uint32_t icap,
                             HigherRec& r) {
  r.interior = 0;
  r.shell = (uint32_t)s.size;
  r.witness = kInvalid32;
  for (uint32_t i = 0; i < m; ++i) {
    const uint32_t w = set[i];
    if (w == s.ids[1] || w == s.ids[2] || (s.size == 4 && w == s.ids[3])) continue;
    const int sd = sphere_side(c, s, w);
    if (sd < 0) {
      if (r.interior >= icap) return false;
      r.iids[r.interior++] = w;
    } else if (sd == 0) {
      ++r.shell;
      r.witness = min(r.witness, w);
    }
  }
  return true;
}

__device__ void emit(HigherRec& r, const Sphere& s, HigherRec* out, uint32_t out_cap, uint32_t* counter) {
  r.size = (uint32_t)s.size;
  for (int i = 0; i < 4; ++i) r.ids[i] = i < s.size ? s.ids[i] : 0u;
  for (int i = 1; i < s.size; ++i) {  // support ids ascending
    const uint32_t x = r.ids[i];
    int j = i;
    while (j > 0 && r.ids[j - 1] > x) { r.ids[j] = r.ids[j - 1]; --j; }
    r.ids[j] = x;
  }
  for (uint32_t i = 1; i < r.interior; ++i) {  // interior ids ascending
    const uint32_t x = r.iids[i];
    uint32_t j = i;
    while (j > 0 && r.iids[j - 1] > x) { r.iids[j] = r.iids[j - 1]; --j; }
    r.iids[j] = x;
  }
  for (uint32_t i = r.interior; i < (uint32_t)kMaxInteriorH; ++i) r.iids[i] = kInvalid32;
  const uint32_t slot = atomicAdd(counter, 1u);
  if (slot < out_cap) out[slot] = r;
}

__device__ __forceinline__ void decode_pair(uint64_t t, uint32_t& lo, uint32_t& hi) {
  uint32_t i = (uint32_t)((sqrt(8.0 * (double)t + 1.0) - 1.0) / 2.0);
  while ((uint64_t)(i + 1) * i / 2 > t) --i;
  while ((uint64_t)(i + 2) * (i + 1) / 2 <= t) ++i;
  lo = (uint32_t)(t - (uint64_t)(i + 1) * i / 2);
  hi = i + 1;
}

__global__ void __launch_bounds__(kThreads)
k_higher(uint32_t n, Ctl ctl, const uint32_t* __restrict__ leaf_pid, const uint32_t* __restrict__ cand,
         const uint32_t* __restrict__ candc, const double* __restrict__ px, const double* __restrict__ py,
         const double* __restrict__ pz, const int* __restrict__ cloud_scale, HigherRec* __restrict__ out,
         uint32_t* __restrict__ counter, unsigned long long* __restrict__ stats, uint32_t* __restrict__ err) {
  __shared__ uint32_t set[kWarps][kMaxCand];  // C(a): classification set
  __shared__ uint32_t sup[kWarps][kMaxCand];  // C(a) with ids > a: support candidates
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  const uint32_t pos = blockIdx.x * kWarps + warp;
  if (pos >= n) return;
  const uint32_t a = leaf_pid[pos];
  const Cloud c{px, py, pz, cloud_scale[0]};
  const uint32_t m = candc[a];
  if (m > (uint32_t)kMaxCand) return;  // reported by the host
  uint32_t mc = 0;
  for (uint32_t base = 0; base < m; base += 32) {
    const uint32_t i = base + lane;
    const uint32_t p = i < m ? cand[(uint64_t)a * kMaxCand + i] : kInvalid32;
    if (i < m) set[warp][i] = p;
    const bool f = i < m && p > a;
    const uint32_t b = __ballot_sync(0xffffffffu, f);
    if (f) sup[warp][mc + __popc(b & lanemask_lt())] = p;
    mc += __popc(b);
  }
  __syncwarp();
  unsigned long long tested = 0, classified = 0, emitted = 0;
  const uint64_t P2 = (uint64_t)mc * (mc - 1) / 2;
  // --- triples (a, b, c): lanes over candidate pairs
  if (ctl.smax >= 3) {
    const uint32_t icap = ctl.smax - 3;
    for (uint64_t t = lane; t < P2; t += 32) {
      uint32_t j, k;
      decode_pair(t, j, k);
      Sphere s;
      s.size = 3;
      s.ids[0] = a;
      s.ids[1] = sup[warp][j];
      s.ids[2] = sup[warp][k];
      ++tested;
      if (tri_status(c, s.ids, s) != 0) continue;
      ++classified;
      HigherRec r;
      if (!classify_set(c, s, set[warp], m, icap, r)) continue;
      ++emitted;
      emit(r, s, out, ctl.cap, counter);
    }
  }
  // --- quads (a, b, c, d): lanes over pairs (b, c), inner loop over d
  if (ctl.smax >= 4) {
    const uint32_t icap = ctl.smax - 4;
    for (uint64_t t = lane; t < P2; t += 32) {
      uint32_t j, k;
      decode_pair(t, j, k);
      for (uint32_t l = k + 1; l < mc; ++l) {
        Sphere s;
        s.size = 4;
        s.ids[0] = a;
        s.ids[1] = sup[warp][j];
        s.ids[2] = sup[warp][k];
        s.ids[3] = sup[warp][l];
        ++tested;
        if (quad_status(c, s.ids, s) != 0) continue;
        ++classified;
        HigherRec r;
        if (!classify_set(c, s, set[warp], m, icap, r)) continue;
        ++emitted;
        emit(r, s, out, ctl.cap, counter);
      }
    }
  }
  for (int off = 16; off > 0; off >>= 1) {
    tested += __shfl_xor_sync(0xffffffffu, tested, off);
    classified += __shfl_xor_sync(0xffffffffu, classified, off);
    emitted += __shfl_xor_sync(0xffffffffu, emitted, off);
  }
  if (lane == 0) {
    atomicAdd(stats + 0, tested);
    atomicAdd(stats + 1, classified);
    atomicAdd(stats + 2, emitted);
    atomicAdd(stats + 3, (unsigned long long)m);
    atomicAdd(stats + 4, (unsigned long long)mc);
  }
}

__global__ void k_higher_keys(uint32_t m, const HigherRec* __restrict__ recs, uint64_t* __restrict__ khi,
                              uint64_t* __restrict__ klo, uint32_t* __restrict__ order) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const HigherRec& r = recs[i];
  // (size, id0, id1, id2, id3) with ids < 2^31: size - 3 in bit 62 of khi
  khi[i] = ((uint64_t)(r.size - 3) << 62) | ((uint64_t)r.ids[0] << 31) | r.ids[1];
  klo[i] = ((uint64_t)r.ids[2] << 31) | r.ids[3];
  order[i] = i;
}

__global__ void k_higher_gather(uint32_t m, const uint32_t* __restrict__ v0, const uint32_t* __restrict__ v1,
                                const uint32_t* __restrict__ state, int passes, const HigherRec* __restrict__ recs,
                                HigherRec* __restrict__ sorted) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) sorted[i] = recs[radix_result(state, passes, v0, v1)[i]];
}

__global__ void k_gather_init(uint32_t n, const double* __restrict__ R2w, double* __restrict__ gr2,
                              uint8_t* __restrict__ todo, double factor2) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  gr2[i] = R2w[i] * factor2;
  todo[i] = 1;
}

// Points whose direction table is not yet certified: cover 2 rho_max with room.
__global__ void k_gather_grow(uint32_t n, double* __restrict__ gr2, const uint8_t* __restrict__ todo,
                              const double* __restrict__ need_r) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || todo[i] != 1) return;
  const double want = 4.0 * need_r[i] * need_r[i] * 1.1;
  gr2[i] = fmax(gr2[i] * 1.44, isfinite(want) ? want : gr2[i] * 4.0);
}

// Icosphere directions and their covering angle (max angular circumradius of a face).
void icosphere(std::vector<float>& dirs, double& delta) {
  const double t = (1.0 + std::sqrt(5.0)) / 2.0;
  std::vector<std::array<double, 3>> v = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0}, {0, -1, t}, {0, 1, t},
                                          {0, -1, -t}, {0, 1, -t}, {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
  std::vector<std::array<int, 3>> f = {{0, 11, 5}, {0, 5, 1}, {0, 1, 7}, {0, 7, 10}, {0, 10, 11}, {1, 5, 9}, {5, 11, 4},
                                       {11, 10, 2}, {10, 7, 6}, {7, 1, 8}, {3, 9, 4}, {3, 4, 2}, {3, 2, 6}, {3, 6, 8},
                                       {3, 8, 9}, {4, 9, 5}, {2, 4, 11}, {6, 2, 10}, {8, 6, 7}, {9, 8, 1}};
  auto norm = [](std::array<double, 3> p) {
    const double l = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
    return std::array<double, 3>{p[0] / l, p[1] / l, p[2] / l};
  };
  for (auto& p : v) p = norm(p);
  for (int level = 0; level < 3; ++level) {
    std::vector<std::array<int, 3>> nf;
    std::vector<std::pair<std::pair<int, int>, int>> mid;
    auto midpoint = [&](int i, int j) {
      const auto key = std::make_pair(std::min(i, j), std::max(i, j));
      for (auto& e : mid)
        if (e.first == key) return e.second;
      v.push_back(norm({(v[i][0] + v[j][0]) / 2, (v[i][1] + v[j][1]) / 2, (v[i][2] + v[j][2]) / 2}));
      mid.push_back({key, (int)v.size() - 1});
      return (int)v.size() - 1;
    };
    for (auto& tri : f) {
      const int a = midpoint(tri[0], tri[1]), b = midpoint(tri[1], tri[2]), c = midpoint(tri[2], tri[0]);
      nf.push_back({tri[0], a, c});
      nf.push_back({tri[1], b, a});
      nf.push_back({tri[2], c, b});
      nf.push_back({a, b, c});
    }
    f = nf;
  }
  // covering angle: every direction is within the circumradius of its face
  delta = 0.0;
  for (auto& tri : f) {
    const auto& A = v[tri[0]];
    const auto& B = v[tri[1]];
    const auto& C = v[tri[2]];
    std::array<double, 3> u{B[0] - A[0], B[1] - A[1], B[2] - A[2]}, w{C[0] - A[0], C[1] - A[1], C[2] - A[2]};
    std::array<double, 3> nrm{u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2], u[0] * w[1] - u[1] * w[0]};
    nrm = norm(nrm);
    if (nrm[0] * A[0] + nrm[1] * A[1] + nrm[2] * A[2] < 0) nrm = {-nrm[0], -nrm[1], -nrm[2]};
    for (const auto* P : {&A, &B, &C}) {
      const double cosang = nrm[0] * (*P)[0] + nrm[1] * (*P)[1] + nrm[2] * (*P)[2];
      delta = std::max(delta, std::acos(std::min(1.0, cosang)));
    }
  }
  delta *= 1.05;  // margin for the binary32 rounding of the stored directions
  dirs.clear();
  for (auto& p : v)
    for (int k = 0; k < 3; ++k) dirs.push_back((float)p[k]);
}

}  // namespace

cudaError_t higher_alloc(Ctx& ctx) {
  const uint64_t n = ctx.max_points;
  HigherBuffers& h = ctx.hb;
  cudaError_t e = cudaSuccess;
  h.capacity = (uint32_t)(512 * n + 4096);  // ~225 supports per point in lattices, more with ties
#define EHGP_ALLOC(ptr, bytes) \
  if ((e = ctx_alloc(ctx, (void**)&(ptr), (bytes))) != cudaSuccess) return e
  EHGP_ALLOC(h.nb, n * kMaxNb * sizeof(uint32_t));
  EHGP_ALLOC(h.nbc, n * sizeof(uint32_t));
  EHGP_ALLOC(h.cand, n * kMaxCand * sizeof(uint32_t));
  EHGP_ALLOC(h.candc, n * sizeof(uint32_t));
  EHGP_ALLOC(h.gather_r2, n * sizeof(double));
  EHGP_ALLOC(h.rcap, n * sizeof(double));
  EHGP_ALLOC(h.todo, n * sizeof(uint8_t));
  EHGP_ALLOC(h.raw, (uint64_t)h.capacity * sizeof(HigherRec));
  EHGP_ALLOC(h.sorted, (uint64_t)h.capacity * sizeof(HigherRec));
  EHGP_ALLOC(h.khi, (uint64_t)h.capacity * sizeof(uint64_t));
  EHGP_ALLOC(h.klo, (uint64_t)h.capacity * sizeof(uint64_t));
  EHGP_ALLOC(h.order0, (uint64_t)h.capacity * sizeof(uint32_t));
  EHGP_ALLOC(h.order1, (uint64_t)h.capacity * sizeof(uint32_t));
  EHGP_ALLOC(h.counters, 8 * sizeof(uint32_t));
  EHGP_ALLOC(h.stats, 8 * sizeof(unsigned long long));
  EHGP_ALLOC(h.radix_counts, 256ull * ((h.capacity + kRadixTile - 1) / kRadixTile) * sizeof(uint32_t));
  std::vector<float> dirs;
  double delta = 0;
  icosphere(dirs, delta);
  if (dirs.size() != 3 * (size_t)kDirs) return cudaErrorInvalidValue;
  EHGP_ALLOC(h.dirs, dirs.size() * sizeof(float));
#undef EHGP_ALLOC
  h.delta = delta;
  return cudaMemcpy(h.dirs, dirs.data(), dirs.size() * sizeof(float), cudaMemcpyHostToDevice);
}

int higher_run(Ctx& ctx, uint32_t K, uint32_t* out_count) {
  const uint32_t n = (uint32_t)ctx.built_n;
  HigherBuffers& h = ctx.hb;
  PairBuffers& p = ctx.pb;
  LbvhBuffers& b = ctx.lb;
  GeomBuffers& g = ctx.gb;
  cudaStream_t st = ctx.stream;
  const uint32_t keff = K < n ? K : n;
  const uint32_t smax = (keff + 1 < n) ? keff + 1 : n;
  *out_count = 0;
  h.count = 0;
  if (smax < 3 || n < 3) return EHGP_OK;
  if (smax - 3 > (uint32_t)kMaxInteriorH) return abi_fail(&ctx, EHGP_ERR_INVALID_ARGUMENT, "K above 10 is not supported");
  if (!p.witness_ready) {  // the witness radii come from the pair stage
    uint32_t pc = 0;
    const int s = pairs_run(ctx, K, &pc);
    if (s != EHGP_OK) return s;
  }
  const uint32_t root = 2 * n - 2;
  uint64_t launches = 0;
  cudaEventRecord(ctx.ev0, st);
  k_gather_init<<<nblocks(n, 256), 256, 0, st>>>(n, p.R2, h.gather_r2, h.todo, 1.6 * 1.6);
  launches += 1;
  CertParams cp;
  {
    uint64_t fr[12];
    cudaMemcpyAsync(fr, b.frame, sizeof(fr), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    for (int k = 0; k < 3; ++k) {
      std::memcpy(&cp.lo[k], &fr[k], 8);
      std::memcpy(&cp.hi[k], &fr[3 + k], 8);
    }
  }
  cp.dirs = h.dirs;
  cp.delta = h.delta;
  cp.need = smax - 2;
  if (cp.need > 16) return abi_fail(&ctx, EHGP_ERR_INVALID_ARGUMENT, "K above 10 is not supported");
  uint32_t pending = n, overflowed = 0;
  std::vector<uint8_t> todo(n);
  for (int round = 0; round < 6 && pending > 0; ++round) {
    k_gather<<<nblocks(n, kWarps), kThreads, 0, st>>>(n, root, g.tnodes, b.leaf_pid, b.n_begin, b.n_end, b.px, b.py,
                                                      b.pz, h.gather_r2, h.todo, h.nb, h.nbc);
    k_dirtable<<<nblocks(n, kDirWarps), 32 * kDirWarps, 0, st>>>(n, cp, b.leaf_pid, h.nb, h.nbc, b.px, b.py, b.pz,
                                                                  h.gather_r2, h.todo, h.cand, h.candc, h.rcap);
    launches += 2;
    cudaMemcpyAsync(todo.data(), h.todo, n, cudaMemcpyDeviceToHost, st);
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return abi_cuda_fail(&ctx, e, "higher-support certificate");
    pending = overflowed = 0;
    for (uint32_t i = 0; i < n; ++i) {
      pending += todo[i] == 1;
      overflowed += todo[i] == 2;
    }
    if (overflowed) break;
    if (pending) {
      k_gather_grow<<<nblocks(n, 256), 256, 0, st>>>(n, h.gather_r2, h.todo, h.rcap);
      ++launches;
    }
  }
  if (pending || overflowed) {
    std::vector<uint32_t> cnt(n), cc(n);
    std::vector<double> need(n), gr(n);
    cudaMemcpy(cnt.data(), h.nbc, 4ull * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(cc.data(), h.candc, 4ull * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(need.data(), h.rcap, 8ull * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(gr.data(), h.gather_r2, 8ull * n, cudaMemcpyDeviceToHost);
    uint32_t i = 0;
    while (i < n && todo[i] == 0) ++i;
    char msg[320];
    snprintf(msg, sizeof msg,
             "a certified neighbourhood exceeds its capacity (%u points pending, %u over %d candidates): e.g. "
             "PointId %u with %u neighbours, %u candidates, radius bound %.6g, gather radius %.6g",
             pending, overflowed, kMaxCand, i, i < n ? cnt[i] : 0u, i < n ? cc[i] : 0u, i < n ? need[i] : 0.0,
             i < n ? std::sqrt(gr[i]) : 0.0);
    return abi_fail(&ctx, EHGP_ERR_CAPACITY, msg);
  }
  cudaMemsetAsync(h.counters, 0, 8 * sizeof(uint32_t), st);
  cudaMemsetAsync(h.stats, 0, 8 * sizeof(unsigned long long), st);
  Ctl ctl{smax, h.capacity};
  cudaEventRecord(ctx.evk0, st);
  k_higher<<<nblocks(n, kWarps), kThreads, 0, st>>>(n, ctl, b.leaf_pid, h.cand, h.candc, b.px, b.py, b.pz, g.scale,
                                                    (HigherRec*)h.raw, h.counters, h.stats, ctx.d_err);
  cudaEventRecord(ctx.evk1, st);
  ++launches;
  uint32_t hc[2];
  unsigned long long hs[8];
  cudaMemcpyAsync(hc, h.counters, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(hc + 1, ctx.d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(hs, h.stats, sizeof(hs), cudaMemcpyDeviceToHost, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return abi_cuda_fail(&ctx, e, "higher-support enumeration");
  if (hc[1]) return abi_device_status(&ctx, hc[1]);
  if (hc[0] > h.capacity) return abi_fail(&ctx, EHGP_ERR_CAPACITY, "higher-support records exceed the buffer");
  {
    float kms = 0;
    cudaEventElapsedTime(&kms, ctx.evk0, ctx.evk1);
    h.kernel_ms = kms;
    for (int i = 0; i < 8; ++i) h.stats_host[i] = hs[i];
  }
  const uint32_t m = hc[0];
  if (m) {
    k_higher_keys<<<nblocks(m, 256), 256, 0, st>>>(m, (const HigherRec*)h.raw, h.khi, h.klo, h.order0);
    RadixScratch rs{h.radix_counts, ctx.radix.state, (uint32_t)((h.capacity + kRadixTile - 1) / kRadixTile)};
    const IndirectKey stages[2] = {{h.klo, 0}, {h.khi, 0}};
    const int bits[2] = {64, 64};
    const int passes = radix_sort_indirect(st, m, h.order0, h.order1, stages, bits, 2, rs, &launches);
    k_higher_gather<<<nblocks(m, 256), 256, 0, st>>>(m, h.order0, h.order1, ctx.radix.state, passes,
                                                     (const HigherRec*)h.raw, (HigherRec*)h.sorted);
    launches += 2;
  }
  cudaEventRecord(ctx.ev1, st);
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return abi_cuda_fail(&ctx, e, "higher-support sort");
  float ms = 0;
  cudaEventElapsedTime(&ms, ctx.ev0, ctx.ev1);
  ctx.last_ms = ms;
  ctx.last_launches = launches;
  h.count = m;
  h.K = K;
  *out_count = m;
  return EHGP_OK;
}

}  // namespace ehgp

extern "C" {

int ehgp_higher(ehgp_ctx* ctx, uint32_t K, const ehgp_higher_out* out) {
  if (!ctx) return EHGP_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(ctx->mutex);
  ctx->last_error.clear();
  if (ctx->poisoned) return ehgp::abi_fail(ctx, EHGP_ERR_POISONED, "the context is poisoned by an earlier CUDA failure");
  if (ctx->built_n == 0) return ehgp::abi_fail(ctx, EHGP_ERR_NOT_BUILT, "ehgp_higher needs a resident LBVH");
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
  const int s = ehgp::higher_run(*ctx, K, &m);
  if (s != EHGP_OK) return s;
  if (out && out->count) *out->count = m;
  if (out && out->records && m) {
    if (out->capacity < m) return ehgp::abi_fail(ctx, EHGP_ERR_CAPACITY, "the output capacity is below the record count");
    e = cudaMemcpy(out->records, ctx->hb.sorted, (uint64_t)m * 64, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return ehgp::abi_cuda_fail(ctx, e, "higher-support copy");
  }
  return EHGP_OK;
}

int ehgp_higher_stats(const ehgp_ctx* ctx, double* kernel_ms, uint64_t* stats, uint32_t count) {
  if (!ctx) return EHGP_ERR_INVALID_ARGUMENT;
  if (kernel_ms) *kernel_ms = ctx->hb.kernel_ms;
  for (uint32_t i = 0; stats && i < count && i < 8; ++i) stats[i] = ctx->hb.stats_host[i];
  return EHGP_OK;
}

}  // extern "C"
