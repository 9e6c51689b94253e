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

#include <type_traits>
#include "ehgp_exact.cuh"
#include "ehgp_sphere.cuh"

#include <algorithm>
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

// ---- FP64 filters with per-tuple uniform error bounds ------------------------------
// Every coordinate difference p - a is one correctly rounded subtraction, so
// |fl(p - a) - (p - a)| <= u |p - a|.  For a polynomial evaluated in binary64 with
// at most ~15 roundings on any path, |computed - exact| <= 64 u m where m is the
// value of the same polynomial with every input replaced by an upper bound of its
// magnitude and every subtraction by an addition.  With all difference
// coordinates bounded by M (M >= max |coordinate| (1 + 2u)) that gives, per
// coordinate or scalar:
//   dot(e, e')          3 M^2        cross(e, e')       2 M^2
//   triangle  G12 3 M^2, G11 - G12 6 M^2, detG 18 M^4, N 36 M^5
//   tetra     detE 6 M^3, N 18 M^4, l_i = N.(e_j x e_k) 108 M^6, l_0 396 M^6
//   side      A q - p.N with |p| <= Mp:  A_m 3 Mp^2 + 3 Mp N_m
// 1e-300 absolute covers underflow.  An undecided sign goes to the exact path.
constexpr double kFilt = 64.0 * kU;
constexpr double kTiny = 1e-300;

__device__ __forceinline__ int fsign(double v, double bound) { return v > bound ? 1 : (v < -bound ? -1 : 2); }

struct SetPt {
  double x, y, z, q;  // fl(p - a) and fl(|fl(p - a)|^2) = (x x + y y) + z z
};

__device__ __forceinline__ double ptmax(const SetPt& p) { return fmax(fabs(p.x), fmax(fabs(p.y), fabs(p.z))); }

// A minimal support waiting for classification: side(w) = sgn * sign(A q - p.N)
// with p = fl(w - a), q = fl(|p|^2); the FP value is decided outside +-bnd.
struct QEntry {
  double A, Nx, Ny, Nz, bnd;
  uint32_t ids[4];  // ids[0] = owner a; ids[3] = kInvalid32 for a triangle
  int16_t size, sgn;
  float cut;  // candidates (sorted by distance from a) with |p - a|^2 above cut lie outside
};
static_assert(sizeof(QEntry) == 64, "queue entries are 64 bytes");

// The exact fallbacks take their ids by value and return the signs packed two bits each
// (sign + 1), so that no array of the hot path needs an address (and local memory).
__device__ __noinline__ uint32_t tri_signs_packed(Cloud c, uint32_t i0, uint32_t i1, uint32_t i2) {
  const uint32_t id[3] = {i0, i1, i2};
  int sg[4];
  tri_signs_exact(c, id, sg);
  uint32_t r = 0;
  for (int k = 0; k < 4; ++k) r |= (uint32_t)(sg[k] + 1) << (2 * k);
  return r;
}
__device__ __noinline__ uint32_t quad_signs_packed(Cloud c, uint32_t i0, uint32_t i1, uint32_t i2, uint32_t i3) {
  const uint32_t id[4] = {i0, i1, i2, i3};
  int sg[5];
  quad_signs_exact(c, id, sg);
  uint32_t r = 0;
  for (int k = 0; k < 5; ++k) r |= (uint32_t)(sg[k] + 1) << (2 * k);
  return r;
}
__device__ __forceinline__ int packed_sign(uint32_t p, int k) { return (int)((p >> (2 * k)) & 3u) - 1; }

// Triangle (a, a + e1, a + e2): minimal iff its three angles are acute.
// Returns 0 minimal (E filled), 1 boundary reduced, 2 obtuse, 3 collinear; *adm is
// false when the circumradius certainly exceeds rmax (no relevant tetrahedron
// has this face: its circumsphere contains the face's circumcircle).
__device__ int tri_eval(const Cloud& c, const SetPt& e1, const SetPt& e2, uint32_t i0, uint32_t i1, uint32_t i2,
                        double Mp, double rmax2,
                        QEntry& E, double& eA, double& eN, bool& adm) {
  const double M = fmax(ptmax(e1), ptmax(e2)) * (1.0 + 1e-15), M2 = M * M;
  const double G11 = e1.q, G22 = e2.q, G12 = (e1.x * e2.x + e1.y * e2.y) + e1.z * e2.z;
  const double db = G11 - G12, dc = G22 - G12;
  const double detG = G11 * G22 - G12 * G12;
  const double bG = kFilt * 3.0 * M2 + kTiny, bD = kFilt * 6.0 * M2 + kTiny, b4 = kFilt * 18.0 * M2 * M2 + kTiny;
  int sg0 = fsign(G12, bG), sg1 = fsign(db, bD), sg2 = fsign(dc, bD), sg3 = fsign(detG, b4);
  if (sg0 == 2 || sg1 == 2 || sg2 == 2 || sg3 == 2) {
    const uint32_t pk = tri_signs_packed(c, i0, i1, i2);
    sg0 = packed_sign(pk, 0);
    sg1 = packed_sign(pk, 1);
    sg2 = packed_sign(pk, 2);
    sg3 = packed_sign(pk, 3);
  }
  if (sg3 == 0) {
    adm = false;
    return 3;
  }
  {  // r^2 = G11 G22 |b - c|^2 / (4 detG): lower bound against rmax^2
    const double bc = G11 + G22 - 2.0 * G12, ebc = kFilt * 12.0 * M2 + kTiny;
    const double num = fmax(G11 - bG, 0.0) * fmax(G22 - bG, 0.0) * fmax(bc - ebc, 0.0);
    const double den = 4.0 * (detG + b4);
    adm = !(num * (1.0 - 1e-12) > rmax2 * den * (1.0 + 1e-9));
  }
  if (sg0 < 0 || sg1 < 0 || sg2 < 0) return 2;
  if (sg0 == 0 || sg1 == 0 || sg2 == 0) return 1;
  const double f1 = G22 * db, f2 = G11 * dc;
  E.A = detG;
  E.Nx = f1 * e1.x + f2 * e2.x;
  E.Ny = f1 * e1.y + f2 * e2.y;
  E.Nz = f1 * e1.z + f2 * e2.z;
  const double Am = 18.0 * M2 * M2, Nm = 36.0 * M2 * M2 * M;
  E.bnd = kFilt * (Am * 3.0 * Mp * Mp + 3.0 * Mp * Nm) + kTiny;
  E.sgn = 1;
  E.size = 3;
  eA = kFilt * Am + kTiny;
  eN = kFilt * Nm + kTiny;
  return 0;
}

// Tetrahedron (a, a + e1, a + e2, a + e3): minimal iff the four barycentric
// coordinates l_i / (2 detE^2) of its circumcentre are positive.
__device__ int quad_eval(const Cloud& c, const SetPt& e1, const SetPt& e2, const SetPt& e3, uint32_t i0, uint32_t i1,
                         uint32_t i2, uint32_t i3,
                         double Mp, QEntry& E, double& eA, double& eN) {
  const double M = fmax(fmax(ptmax(e1), ptmax(e2)), ptmax(e3)) * (1.0 + 1e-15), M2 = M * M, M3 = M2 * M;
  const double c23x = e2.y * e3.z - e2.z * e3.y, c23y = e2.z * e3.x - e2.x * e3.z, c23z = e2.x * e3.y - e2.y * e3.x;
  const double c31x = e3.y * e1.z - e3.z * e1.y, c31y = e3.z * e1.x - e3.x * e1.z, c31z = e3.x * e1.y - e3.y * e1.x;
  const double c12x = e1.y * e2.z - e1.z * e2.y, c12y = e1.z * e2.x - e1.x * e2.z, c12z = e1.x * e2.y - e1.y * e2.x;
  const double detE = (e1.x * c23x + e1.y * c23y) + e1.z * c23z;
  const double Nx = (e1.q * c23x + e2.q * c31x) + e3.q * c12x;
  const double Ny = (e1.q * c23y + e2.q * c31y) + e3.q * c12y;
  const double Nz = (e1.q * c23z + e2.q * c31z) + e3.q * c12z;
  const double l1 = (Nx * c23x + Ny * c23y) + Nz * c23z;
  const double l2 = (Nx * c31x + Ny * c31y) + Nz * c31z;
  const double l3 = (Nx * c12x + Ny * c12y) + Nz * c12z;
  const double l0 = (2.0 * detE) * detE - ((l1 + l2) + l3);
  const double M6 = M3 * M3;
  const double bE = kFilt * 6.0 * M3 + kTiny, bl = kFilt * 108.0 * M6 + kTiny, b0 = kFilt * 396.0 * M6 + kTiny;
  int sg0 = fsign(detE, bE), sg1 = fsign(l0, b0), sg2 = fsign(l1, bl), sg3 = fsign(l2, bl), sg4 = fsign(l3, bl);
  if (sg0 == 2 || sg1 == 2 || sg2 == 2 || sg3 == 2 || sg4 == 2) {
    const uint32_t pk = quad_signs_packed(c, i0, i1, i2, i3);
    sg0 = packed_sign(pk, 0);
    sg1 = packed_sign(pk, 1);
    sg2 = packed_sign(pk, 2);
    sg3 = packed_sign(pk, 3);
    sg4 = packed_sign(pk, 4);
  }
  if (sg0 == 0) return 3;
  if (sg1 < 0 || sg2 < 0 || sg3 < 0 || sg4 < 0) return 2;
  if (sg1 == 0 || sg2 == 0 || sg3 == 0 || sg4 == 0) return 1;
  const double Am = 6.0 * M3, Nm = 18.0 * M2 * M2;
  E.A = detE;
  E.Nx = Nx;
  E.Ny = Ny;
  E.Nz = Nz;
  E.bnd = kFilt * (Am * 3.0 * Mp * Mp + 3.0 * Mp * Nm) + kTiny;
  E.sgn = sg0;
  E.size = 4;
  eA = kFilt * Am + kTiny;
  eN = kFilt * Nm + kTiny;
  return 0;
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
  if (todo[a] != 1) return;
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
constexpr int kDirThreads = 128;  // one block per point: four warps share its sorted list
constexpr int kMaxCand = 256;     // candidate-set capacity per point
constexpr int kLargeCand = 1024;  // large sets: staged whole in shared memory with their face mask
constexpr int kHugeCand = 4096;   // huge sets: staged in shared memory, face mask in global scratch
constexpr int kMegaCand = 16384;  // larger sets: set and face mask in global scratch (one per block)
constexpr int kMaxNeed = kMaxInteriorH + 1;  // s_max - 2 for K = 10

struct CertParams {
  const float* dirs;  // [kDirs * 3] unit vectors
  double delta;       // covering angle of the directions (radians)
  double lo[3], hi[3];  // cloud AABB
  uint32_t need;        // s_max - 2
};

// Largest (s_k +- delta)-weighted excursion from a along axis k inside the cloud AABB:
// sum over k bounds the support of the AABB over a cone of directions around s.
__device__ __forceinline__ double cone_ext(const CertParams& cp, double sk, double ak, int k) {
  const double up = cp.hi[k] - ak, dn = cp.lo[k] - ak;
  const double t1 = sk - cp.delta, t2 = sk + cp.delta;
  const double f1 = t1 >= 0 ? up * t1 : dn * t1, f2 = t2 >= 0 ? up * t2 : dn * t2;
  return fmax(f1, f2);
}

// Distance along the cone (direction s, half-angle delta) at which a ray from a leaves the
// AABB across axis k; infinite when the cone crosses that axis' zero.
__device__ __forceinline__ double cone_exit(const CertParams& cp, double sk, double ak, int k) {
  const double t1 = sk - cp.delta, t2 = sk + cp.delta;
  if (t1 <= 0.0 && t2 >= 0.0) return INFINITY;
  const double g = t1 > 0.0 ? (cp.hi[k] - ak) / t1 : (ak - cp.lo[k]) / (-t2);
  return g * (1.0 + 1e-12);
}

// Bitonic sort of one value per lane, descending across the warp (lane 0 the largest).
__device__ __forceinline__ float warp_sort_desc(float v, uint32_t lane) {
#pragma unroll
  for (uint32_t k = 2; k <= 32; k <<= 1) {
#pragma unroll
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      const float o = __shfl_xor_sync(0xffffffffu, v, j);
      v = (((lane & j) == 0) == ((lane & k) == 0)) ? fmaxf(v, o) : fminf(v, o);
    }
  }
  return v;
}

// top holds the 32 largest values seen so far, descending across the warp; merges in one
// value per lane: the larger of top[j] and the j-th smallest new value forms a bitonic
// sequence that holds the 32 largest of both, and a bitonic merge orders it.
__device__ __forceinline__ float warp_top_merge(float top, float v, uint32_t lane) {
  const float s = warp_sort_desc(v, lane);
  float x = fmaxf(top, __shfl_sync(0xffffffffu, s, 31u - lane));
#pragma unroll
  for (uint32_t j = 16; j > 0; j >>= 1) {
    const float o = __shfl_xor_sync(0xffffffffu, x, j);
    x = ((lane & j) == 0) ? fmaxf(x, o) : fminf(x, o);
  }
  return x;
}

// register budget of the direction table: 10 blocks of 128 threads per SM (51 registers; its
// shared list is 20.6 KB per block); measured higher-stage wall at 50k 113.6 ms at 7, 111.7 at 10
#ifndef EHGP_DIRTABLE_BLOCKS_PER_SM
#define EHGP_DIRTABLE_BLOCKS_PER_SM 10
#endif
__global__ void __launch_bounds__(kDirThreads, EHGP_DIRTABLE_BLOCKS_PER_SM)
k_dirtable(uint32_t n, uint32_t list_cap, CertParams cp, const uint32_t* __restrict__ leaf_pid, uint32_t* __restrict__ nb,
           const uint32_t* __restrict__ nbc, const double* __restrict__ px, const double* __restrict__ py,
           const double* __restrict__ pz, const double* __restrict__ gather_r2, uint8_t* __restrict__ todo,
           uint32_t* __restrict__ cand, uint32_t* __restrict__ candc, double* __restrict__ need_r,
           float* __restrict__ rho_tab) {
  __shared__ float4 rel[kMaxNb];  // unit direction of p - a and |p - a| (binary32; margins below)
  __shared__ uint32_t ids[kMaxNb];
  __shared__ uint32_t mark[kMaxNb / 32];
  __shared__ double worst_w[kDirThreads / 32];
  const uint32_t t = threadIdx.x, warp = t >> 5, lane = t & 31u;
  const uint32_t pos = blockIdx.x;
  if (pos >= n) return;
  const uint32_t a = leaf_pid[pos];
  if (todo[a] != 1) return;
  const uint32_t m = nbc[a];
  if (m > list_cap) {  // more neighbours than a list holds: the large-neighbourhood path
    if (t == 0) todo[a] = 3;
    return;
  }
  const double ax = px[a], ay = py[a], az = pz[a];
  for (uint32_t i = t; i < m; i += kDirThreads) {
    const uint32_t p = nb[(uint64_t)a * kMaxNb + i];
    const double x = px[p] - ax, y = py[p] - ay, z = pz[p] - az;
    const double dd = sqrt(x * x + y * y + z * z);
    const double inv = dd > 0.0 ? 1.0 / dd : 0.0;
    rel[i] = make_float4((float)(x * inv), (float)(y * inv), (float)(z * inv), (float)dd);  // unit direction, |p - a|
    ids[i] = p;
  }
  if (t < (uint32_t)kMaxNb / 32) mark[t] = 0;
  // sort by distance (bitonic network over a power-of-two padding, in shared memory)
  uint32_t P = 1;
  while (P < m) P <<= 1;
  for (uint32_t i = m + t; i < P; i += kDirThreads) {
    rel[i] = make_float4(0.f, 0.f, 0.f, INFINITY);
    ids[i] = kInvalid32;
  }
  __syncthreads();
  for (uint32_t k = 2; k <= P; k <<= 1) {
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      for (uint32_t i = t; i < P; i += kDirThreads) {
        const uint32_t l = i ^ j;
        if (l > i) {
          const bool up = (i & k) == 0;
          const float4 x = rel[i], y = rel[l];
          if ((x.w > y.w) == up) {
            rel[i] = y;
            rel[l] = x;
            const uint32_t tmp = ids[i];
            ids[i] = ids[l];
            ids[l] = tmp;
          }
        }
      }
      __syncthreads();
    }
  }
  // the sorted list keeps 1 / |p - a| in .w from here on (binary32)
  for (uint32_t i = t; i < P; i += kDirThreads) {
    float4 r = rel[i];
    r.w = i < m ? 1.0f / r.w : 0.0f;
    rel[i] = r;
  }
  __syncthreads();
  // distances are binary32: thresholds carry a relative margin of 1e-5 in the safe direction
  const double L2 = sqrt(gather_r2[a]) * (1.0 - 1e-9);  // list covers |p - a| <= L
  const double half_L = 0.5 * L2;
  const double cd = cos(cp.delta), sdl = sin(cp.delta);
  const float cdf = (float)cd, sdlf = (float)sdl;
  const uint32_t need = cp.need;
  double worst_needed = 0.0;  // largest certified rho_s (the list must cover 2 rho_s)
  bool ok = true;
  // Each warp takes batches of 32 directions; lane j prepares direction j of the batch, then
  // the warp scans the sorted list for one direction at a time, 32 points per step.
  for (uint32_t dbase = warp * 32u; dbase < (uint32_t)kDirs; dbase += kDirThreads) {
    const uint32_t dl = dbase + lane;
    float s0f = 0.f, s1f = 0.f, s2f = 0.f;
    double ext_c = 0.0;
    if (dl < (uint32_t)kDirs) {
      const double s0 = cp.dirs[3 * dl], s1 = cp.dirs[3 * dl + 1], s2 = cp.dirs[3 * dl + 2];
      s0f = (float)s0;
      s1f = (float)s1;
      s2f = (float)s2;
      // AABB support bound over the cone
      const double ext = cone_ext(cp, s0, ax, 0) + cone_ext(cp, s1, ay, 1) + cone_ext(cp, s2, az, 2);
      // the centre of a well-centred sphere lies in conv(S), inside the AABB: r is at most
      // the distance at which the ray a + r u leaves the AABB, maximised over the cone
      // axis by axis (min over axes of the per-axis maxima bounds the max of the min)
      const double exit_r = fmin(fmin(cone_exit(cp, s0, ax, 0), cone_exit(cp, s1, ay, 1)), cone_exit(cp, s2, az, 2));
      ext_c = fmin(ext * (1.0 + 1e-12), exit_r);
    }
    const uint32_t nd = min(32u, (uint32_t)kDirs - dbase);
    float my_rho = 0.f;
    for (uint32_t jd = 0; jd < nd; ++jd) {
      const float u0 = __shfl_sync(0xffffffffu, s0f, jd), u1 = __shfl_sync(0xffffffffu, s1f, jd),
                  u2 = __shfl_sync(0xffffffffu, s2f, jd);
      const double ext_d = __shfl_sync(0xffffffffu, ext_c, jd);
      // The `need` smallest shrunk thresholds, kept as the `need` largest lower bounds of
      // 1 / rho_shr (binary32, no divides):  1/rho_p(u) >= 2 cos(angle + delta) / |p - a|.
      // Every binary32 rounding (about 1e-7 relative) is covered by the 1e-5 margins and the
      // 1e-6 absolute slack on the cosines, always in the safe direction.  The scan stops at
      // the first step whose nearest point has rho >= |p - a| / 2 > min(kth, ext); points
      // past that bound can neither enter the `need` largest nor lower min(kth, ext).
      const float inv_ext = 1.0f / __double2float_ru(ext_d);
      float top = 0.0f;  // lane j: the j-th largest lower bound so far
      float thr = 0.0f;  // top[need - 1]
      for (uint32_t base = 0; base < m; base += 32) {
        const uint32_t i = base + lane;
        const float lim = 0.5f * (1.0f - 1e-5f) * fmaxf(thr, inv_ext);
        const float4 r = i < m ? rel[i] : make_float4(0.f, 0.f, 0.f, 0.f);  // r.w = 1 / |p - a|
        if (lim > __shfl_sync(0xffffffffu, r.w, 0)) break;
        float inv = 0.0f;
        if (i < m && !(lim > r.w)) {
          const float c = u0 * r.x + u1 * r.y + u2 * r.z;
          const float cs = fmaxf(-1.0f, c - 1e-5f);  // cosine of an upper bound of the angle
          const float sn = sqrtf(fmaxf(0.0f, (1.0f - cs) * (1.0f + cs)));
          const float cshr = cs * cdf - sn * sdlf - 1e-6f;  // lower bound of cos(angle + delta)
          if (cshr > 1e-6f) inv = 2.0f * cshr * r.w * (1.0f - 1e-5f);  // lower bound of 1 / rho_p(u)
        }
        if (__any_sync(0xffffffffu, inv > thr)) {
          top = warp_top_merge(top, inv, lane);
          thr = __shfl_sync(0xffffffffu, top, need - 1);
        }
      }
      const double kth = thr > 0.0f ? (1.0 / (double)thr) * (1.0 + 1e-12) : INFINITY;
      const double rho_s = fmin(kth, ext_d);
      const float rho_sf = __double2float_ru(rho_s);  // per-cone bound, rounded up
      if (lane == jd) my_rho = rho_sf;
      // certified when every unlisted point (rho >= L/2) cannot lower it
      if (!(rho_s <= half_L)) ok = false;
      worst_needed = fmax(worst_needed, rho_s);
      // mark the candidates of this cone: rho_lo_p(s) <= rho_s, i.e. 2 cos(max(angle - delta, 0)) rho_s >= |p - a|;
      // rho_lo >= |p - a| / 2 > rho_s stops the scan (monotone along the sorted list)
      for (uint32_t base = 0; base < m; base += 32) {
        const uint32_t i = base + lane;
        const float4 r = i < m ? rel[i] : make_float4(0.f, 0.f, 0.f, 0.f);
        const bool stop = !(i < m) || (0.5f * (1.0f - 1e-5f) > rho_sf * r.w);
        if (__shfl_sync(0xffffffffu, stop, 0)) break;
        bool f = false;
        if (!stop) {
          const float c = u0 * r.x + u1 * r.y + u2 * r.z;
          const float cs = fminf(1.0f, c + 1e-5f);  // cosine of a lower bound of the angle
          const float sn = sqrtf(fmaxf(0.0f, (1.0f - cs) * (1.0f + cs)));
          const float clo = (cs >= cdf) ? 1.0f : cs * cdf + sn * sdlf + 1e-6f;  // upper bound of cos(max(angle - delta, 0))
          f = clo > 0.0f && 2.0f * clo * rho_sf * r.w * (1.0f + 2e-5f) >= 1.0f;
        }
        const uint32_t bits = __ballot_sync(0xffffffffu, f);
        if (lane == 0 && bits) atomicOr(&mark[base >> 5], bits);
      }
    }
    if (lane < nd) rho_tab[(uint64_t)a * kDirs + dl] = my_rho;
  }
  for (int off = 16; off > 0; off >>= 1) worst_needed = fmax(worst_needed, __shfl_xor_sync(0xffffffffu, worst_needed, off));
  if (lane == 0) worst_w[warp] = worst_needed;
  ok = __syncthreads_and(ok);  // also publishes mark[] and worst_w[]
#pragma unroll
  for (int w = 0; w < kDirThreads / 32; ++w) worst_needed = fmax(worst_needed, worst_w[w]);
  if (!ok) {  // the list must grow to 2 rho_s (with room)
    if (t == 0) need_r[a] = worst_needed;
    return;
  }
  if (warp != 0) return;
  // compact the candidate set in distance order
  uint32_t c = 0;
  uint32_t* out = cand + (uint64_t)a * kMaxCand;
  for (uint32_t base = 0; base < m; base += 32) {
    const uint32_t i = base + lane;
    const bool f = i < m && ((mark[i >> 5] >> (i & 31)) & 1u);
    const uint32_t b = __ballot_sync(0xffffffffu, f);
    if (f) {
      const uint32_t at = c + __popc(b & lanemask_lt());
      if (at < (uint32_t)kMaxCand) out[at] = ids[i];
    }
    c += __popc(b);
  }
  const bool overflow = c > (uint32_t)kMaxCand;
  if (lane == 0) {
    candc[a] = overflow ? (uint32_t)kMaxCand + 1 : c;
    need_r[a] = worst_needed;
    todo[a] = overflow ? 4 : 0;  // 4: certified, candidate set above kMaxCand (k_cand_large)
  }
}



// ---- 2b. large neighbourhoods ------------------------------------------------------------
// Owners whose gather radius holds more than kMaxNb points (edges of dense clusters whose
// bounds reach into a sparse background, points near the hull) take this path, with the
// same certificate: their neighbour lists are counted, allocated in one arena and written
// (one thread per owner, depth first, whole subtrees inside the radius taken as ranges); a
// block per owner then stages its list in chunks and keeps, per direction, the `need` largest
// lower bounds of 1 / rho_shr with every neighbour seen (the list is not sorted, so there is
// no early exit), marks the candidates and writes C(a) sorted by binary32 distance.
constexpr int kBigStack = 128;    // traversal stack: the LBVH is at most 63 + log2(n) + 1 deep
constexpr int kBigThreads = 256;  // one block of eight warps per large owner
constexpr int kBigChunk = 2048;   // neighbours staged per step

__global__ void __launch_bounds__(128)
k_gather_big(uint32_t nbig, const uint32_t* __restrict__ big, uint32_t root, const TNode* __restrict__ tn,
             const uint32_t* __restrict__ leaf_pid, const uint32_t* __restrict__ n_begin,
             const uint32_t* __restrict__ n_end, const double* __restrict__ px, const double* __restrict__ py,
             const double* __restrict__ pz, const double* __restrict__ gather_r2, const uint64_t* __restrict__ off,
             uint32_t* __restrict__ arena, uint32_t* __restrict__ cnt, uint32_t* __restrict__ err) {
  // one warp per owner: every lane takes the same walk (warp-uniform branches, broadcast loads);
  // lane 0 appends single leaves, and a whole subtree inside the radius is copied by the 32
  // lanes; the list keeps the order of one thread's walk
  const uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31u;
  if (i >= nbig) return;
  const uint32_t a = big[i];
  const double ax = px[a], ay = py[a], az = pz[a];
  const double R2 = gather_r2[a] * (1.0 + 32.0 * kU);
  const uint64_t cap = arena ? off[i + 1] - off[i] : 0;
  uint32_t* out = arena ? arena + off[i] : nullptr;
  uint64_t c = 0;
  uint32_t stack[kBigStack];
  int top = 0;
  stack[top++] = root;
  while (top > 0) {
    const uint32_t node = stack[--top];
    const TNode t = load_node(tn, node);
    if (t.left == kInvalid32) {
      const uint32_t pid = t.right;
      const double dx = px[pid] - ax, dy = py[pid] - ay, dz = pz[pid] - az;
      if (pid != a && dx * dx + dy * dy + dz * dz <= R2) {
        if (lane == 0 && c < cap) out[c] = pid;
        ++c;
      }
      continue;
    }
    const double lx = fmax(fmax((double)t.lo[0] - ax, ax - (double)t.hi[0]), 0.0);
    const double ly = fmax(fmax((double)t.lo[1] - ay, ay - (double)t.hi[1]), 0.0);
    const double lz = fmax(fmax((double)t.lo[2] - az, az - (double)t.hi[2]), 0.0);
    if ((lx * lx + ly * ly + lz * lz) * (1.0 - 16.0 * kU) > R2) continue;
    const double ux = fmax(fabs((double)t.lo[0] - ax), fabs((double)t.hi[0] - ax));
    const double uy = fmax(fabs((double)t.lo[1] - ay), fabs((double)t.hi[1] - ay));
    const double uz = fmax(fabs((double)t.lo[2] - az), fabs((double)t.hi[2] - az));
    if ((ux * ux + uy * uy + uz * uz) * (1.0 + 16.0 * kU) < R2) {  // the whole subtree is inside
      const uint32_t q_hi = n_end[node];
      for (uint32_t q0 = n_begin[node]; q0 < q_hi; q0 += 32) {
        const uint32_t q = q0 + lane;
        const uint32_t pid = q < q_hi ? leaf_pid[q] : kInvalid32;
        const bool keep = q < q_hi && pid != a;
        const uint32_t bal = __ballot_sync(0xffffffffu, keep);
        const uint64_t pos = c + __popc(bal & lanemask_lt());
        if (keep && pos < cap) out[pos] = pid;
        c += __popc(bal);
      }
      continue;
    }
    if (top + 2 > kBigStack) {
      if (lane == 0) atomicOr(err, kErrCapacity);
      return;
    }
    stack[top++] = t.right;
    stack[top++] = t.left;
  }
  if (lane != 0) return;
  if (!arena) cnt[i] = (uint32_t)c;
  else if (c != cap) atomicOr(err, kErrInternal);
}

// Dynamic shared memory of k_dirtable_big.
constexpr size_t kBigSmem = (size_t)kBigChunk * 16 + (size_t)kDirs * kMaxNeed * 4 + (size_t)kDirs * 4 + 16 +
                            (size_t)kDirs * 8 + (size_t)kMaxCand * 8;

__global__ void __launch_bounds__(kBigThreads)
k_dirtable_big(uint32_t nbig, CertParams cp, const uint32_t* __restrict__ big, const uint64_t* __restrict__ off,
               const uint32_t* __restrict__ arena, const double* __restrict__ px, const double* __restrict__ py,
               const double* __restrict__ pz, const double* __restrict__ gather_r2, uint8_t* __restrict__ todo,
               uint32_t* __restrict__ cand, uint32_t* __restrict__ candc, double* __restrict__ need_r,
               float* __restrict__ rho_tab) {
  extern __shared__ __align__(16) unsigned char smem[];
  float4* rel = reinterpret_cast<float4*>(smem);               // [kBigChunk] unit direction, 1 / |p - a|
  float* topt = reinterpret_cast<float*>(rel + kBigChunk);     // [kDirs][kMaxNeed] descending
  float* rho = topt + kDirs * kMaxNeed;                        // [kDirs] certified per-cone bounds
  double* ext = reinterpret_cast<double*>(reinterpret_cast<uintptr_t>(rho + kDirs + 3) & ~uintptr_t(7));  // [kDirs]
  uint32_t* cid = reinterpret_cast<uint32_t*>(ext + kDirs);    // [kMaxCand]
  float* cds = reinterpret_cast<float*>(cid + kMaxCand);       // [kMaxCand] binary32 |p - a|
  __shared__ double s_worst[kBigThreads / 32];
  __shared__ float s_rmax[kBigThreads / 32];
  __shared__ uint32_t s_c;
  const uint32_t t = threadIdx.x, warp = t >> 5, lane = t & 31u;
  if (blockIdx.x >= nbig) return;
  const uint32_t a = big[blockIdx.x];
  const uint64_t m = off[blockIdx.x + 1] - off[blockIdx.x];
  const uint32_t* list = arena + off[blockIdx.x];
  const double ax = px[a], ay = py[a], az = pz[a];
  const double L2 = sqrt(gather_r2[a]) * (1.0 - 1e-9);  // the list covers |p - a| <= L
  const double half_L = 0.5 * L2;
  const double cd = cos(cp.delta), sdl = sin(cp.delta);
  const float cdf = (float)cd, sdlf = (float)sdl;
  const uint32_t need = cp.need;
  for (uint32_t d = t; d < (uint32_t)kDirs; d += kBigThreads) {
    const double s0 = cp.dirs[3 * d], s1 = cp.dirs[3 * d + 1], s2 = cp.dirs[3 * d + 2];
    const double e = cone_ext(cp, s0, ax, 0) + cone_ext(cp, s1, ay, 1) + cone_ext(cp, s2, az, 2);
    const double exit_r = fmin(fmin(cone_exit(cp, s0, ax, 0), cone_exit(cp, s1, ay, 1)), cone_exit(cp, s2, az, 2));
    ext[d] = fmin(e * (1.0 + 1e-12), exit_r);
    for (uint32_t j = 0; j < (uint32_t)kMaxNeed; ++j) topt[d * kMaxNeed + j] = 0.0f;
  }
  if (t == 0) s_c = 0;
  __syncthreads();
  // 1. per cone, the `need` largest lower bounds of 1 / rho_shr over the whole list
  for (uint64_t base = 0; base < m; base += kBigChunk) {
    const uint32_t cnt = (uint32_t)min((uint64_t)kBigChunk, m - base);
    for (uint32_t j = t; j < cnt; j += kBigThreads) {
      const uint32_t p = list[base + j];
      const double x = px[p] - ax, y = py[p] - ay, z = pz[p] - az;
      const double dd = sqrt(x * x + y * y + z * z);
      const double inv = dd > 0.0 ? 1.0 / dd : 0.0;
      const float df = (float)dd;
      rel[j] = make_float4((float)(x * inv), (float)(y * inv), (float)(z * inv), 1.0f / df);
    }
    __syncthreads();
    for (uint32_t d = warp; d < (uint32_t)kDirs; d += kBigThreads / 32) {
      const float u0 = cp.dirs[3 * d], u1 = cp.dirs[3 * d + 1], u2 = cp.dirs[3 * d + 2];
      const float inv_ext = 1.0f / __double2float_ru(ext[d]);
      float top = lane < need ? topt[d * kMaxNeed + lane] : 0.0f;
      float thr = __shfl_sync(0xffffffffu, top, need - 1);
      for (uint32_t sb = 0; sb < cnt; sb += 32) {
        const uint32_t j = sb + lane;
        const float lim = 0.5f * (1.0f - 1e-5f) * fmaxf(thr, inv_ext);
        const float4 r = j < cnt ? rel[j] : make_float4(0.f, 0.f, 0.f, 0.f);
        float inv = 0.0f;
        if (j < cnt && !(lim > r.w)) {
          const float c = u0 * r.x + u1 * r.y + u2 * r.z;
          const float cs = fmaxf(-1.0f, c - 1e-5f);
          const float sn = sqrtf(fmaxf(0.0f, (1.0f - cs) * (1.0f + cs)));
          const float cshr = cs * cdf - sn * sdlf - 1e-6f;
          if (cshr > 1e-6f) inv = 2.0f * cshr * r.w * (1.0f - 1e-5f);
        }
        if (__any_sync(0xffffffffu, inv > thr)) {
          top = warp_top_merge(top, inv, lane);
          thr = __shfl_sync(0xffffffffu, top, need - 1);
        }
      }
      if (lane < need) topt[d * kMaxNeed + lane] = top;
    }
    __syncthreads();
  }
  // certified per-cone bounds (same rule as the list path)
  double worst = 0.0;
  float rmax = 0.0f;
  bool ok = true;
  for (uint32_t d = t; d < (uint32_t)kDirs; d += kBigThreads) {
    const float thr = topt[d * kMaxNeed + need - 1];
    const double kth = thr > 0.0f ? (1.0 / (double)thr) * (1.0 + 1e-12) : INFINITY;
    const double rho_s = fmin(kth, ext[d]);
    const float rho_sf = __double2float_ru(rho_s);
    rho[d] = rho_sf;
    rho_tab[(uint64_t)a * kDirs + d] = rho_sf;
    if (!(rho_s <= half_L)) ok = false;
    worst = fmax(worst, rho_s);
    rmax = fmaxf(rmax, rho_sf);
  }
  for (int o = 16; o > 0; o >>= 1) {
    worst = fmax(worst, __shfl_xor_sync(0xffffffffu, worst, o));
    rmax = fmaxf(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
  }
  if (lane == 0) {
    s_worst[warp] = worst;
    s_rmax[warp] = rmax;
  }
  ok = __syncthreads_and(ok);
  for (int w = 0; w < kBigThreads / 32; ++w) {
    worst = fmax(worst, s_worst[w]);
    rmax = fmaxf(rmax, s_rmax[w]);
  }
  if (!ok) {  // the list must grow to 2 rho_s (with room); the owner stays on this path
    if (t == 0) need_r[a] = worst;
    return;
  }
  // 2. candidates: rho_lo_p(s) <= rho_s for some cone s
  for (uint64_t j = t; j < m; j += kBigThreads) {
    const uint32_t p = list[j];
    const double x = px[p] - ax, y = py[p] - ay, z = pz[p] - az;
    const double dd = sqrt(x * x + y * y + z * z);
    const double inv = dd > 0.0 ? 1.0 / dd : 0.0;
    const float df = (float)dd;
    const float rw = 1.0f / df;
    if (0.5f * (1.0f - 1e-5f) > rmax * rw) continue;  // beyond 2 rho_s of every cone
    const float r0 = (float)(x * inv), r1 = (float)(y * inv), r2 = (float)(z * inv);
    bool f = false;
    for (uint32_t d = 0; d < (uint32_t)kDirs && !f; ++d) {
      const float rho_sf = rho[d];
      if (0.5f * (1.0f - 1e-5f) > rho_sf * rw) continue;
      const float c = cp.dirs[3 * d] * r0 + cp.dirs[3 * d + 1] * r1 + cp.dirs[3 * d + 2] * r2;
      const float cs = fminf(1.0f, c + 1e-5f);
      const float sn = sqrtf(fmaxf(0.0f, (1.0f - cs) * (1.0f + cs)));
      const float clo = (cs >= cdf) ? 1.0f : cs * cdf + sn * sdlf + 1e-6f;
      f = clo > 0.0f && 2.0f * clo * rho_sf * rw * (1.0f + 2e-5f) >= 1.0f;
    }
    if (f) {
      const uint32_t at = atomicAdd(&s_c, 1u);
      if (at < (uint32_t)kMaxCand) {
        cid[at] = p;
        cds[at] = df;
      }
    }
  }
  __syncthreads();
  const uint32_t c = s_c;
  if (c > (uint32_t)kMaxCand) {
    if (t == 0) {
      candc[a] = (uint32_t)kMaxCand + 1;
      need_r[a] = worst;
      todo[a] = 4;  // certified, candidate set above kMaxCand (k_cand_large)
    }
    return;
  }
  // 3. C(a) in binary32 distance order (bitonic over kMaxCand slots)
  for (uint32_t j = c + t; j < (uint32_t)kMaxCand; j += kBigThreads) {
    cds[j] = INFINITY;
    cid[j] = kInvalid32;
  }
  __syncthreads();
  for (uint32_t k = 2; k <= (uint32_t)kMaxCand; k <<= 1)
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      for (uint32_t x = t; x < (uint32_t)kMaxCand; x += kBigThreads) {
        const uint32_t y = x ^ j;
        if (y > x) {
          const bool up = (x & k) == 0;
          const float dx = cds[x], dy = cds[y];
          if ((dx > dy) == up) {
            cds[x] = dy;
            cds[y] = dx;
            const uint32_t tmp = cid[x];
            cid[x] = cid[y];
            cid[y] = tmp;
          }
        }
      }
      __syncthreads();
    }
  for (uint32_t j = t; j < c; j += kBigThreads) cand[(uint64_t)a * kMaxCand + j] = cid[j];
  if (t == 0) {
    candc[a] = c;
    need_r[a] = worst;
    todo[a] = 0;
  }
}

// ---- 2c. large candidate sets -------------------------------------------------------------
// Owners certified with more than kMaxCand candidates: their candidate sets are counted and
// then written, sorted by binary32 distance, into an arena (count -> allocate -> write), from
// the certified per-cone bounds rho_tab and the owner's neighbour list (the per-point list,
// or the large-neighbourhood arena); the candidate rule is the one of the direction tables.
constexpr int kCandThreads = 256;

template <bool kFromArena>
__global__ void __launch_bounds__(kCandThreads)
k_cand_large(uint32_t nown, const uint32_t* __restrict__ owners, const uint32_t* __restrict__ nb,
             const uint32_t* __restrict__ nbc, const uint64_t* __restrict__ loff, const uint32_t* __restrict__ larena,
             CertParams cp, const double* __restrict__ px, const double* __restrict__ py,
             const double* __restrict__ pz, const float* __restrict__ rho_tab, const uint64_t* __restrict__ coff,
             uint32_t* __restrict__ carena, uint32_t* __restrict__ ccnt, float* __restrict__ dist_scratch) {
  // counting pass: carena == nullptr, ccnt[i] receives the count; writing pass: the sorted
  // set goes to carena + coff[i] when its count equals ccnt[i]
  __shared__ float rho[kDirs];
  __shared__ float s_rmax[kCandThreads / 32];
  __shared__ uint32_t s_c;
  __shared__ float s_cds[kHugeCand];
  __shared__ uint32_t s_cid[kHugeCand];
  const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
  const uint32_t i = blockIdx.x;
  if (i >= nown) return;
  const uint32_t a = owners[i];
  // the set is gathered and sorted in shared memory up to kHugeCand entries, above that in
  // its own slot of the arena (kMegaCand at most), with the distances in `dist_scratch`
  const bool in_arena = carena != nullptr && ccnt[i] > (uint32_t)kHugeCand;
  float* cds = in_arena ? dist_scratch + coff[i] : s_cds;
  uint32_t* cid = in_arena ? carena + coff[i] : s_cid;
  const uint32_t cap = in_arena ? (uint32_t)kMegaCand : (uint32_t)kHugeCand;
  const uint32_t* list = kFromArena ? larena + loff[i] : nb + (uint64_t)a * kMaxNb;
  const uint64_t m = kFromArena ? loff[i + 1] - loff[i] : nbc[a];
  const double ax = px[a], ay = py[a], az = pz[a];
  const float cdf = (float)cos(cp.delta), sdlf = (float)sin(cp.delta);
  float rmax = 0.0f;
  for (uint32_t d = t; d < (uint32_t)kDirs; d += kCandThreads) {
    rho[d] = rho_tab[(uint64_t)a * kDirs + d];
    rmax = fmaxf(rmax, rho[d]);
  }
  for (int o = 16; o > 0; o >>= 1) rmax = fmaxf(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
  if (lane == 0) s_rmax[warp] = rmax;
  if (t == 0) s_c = 0;
  __syncthreads();
  for (int w = 0; w < kCandThreads / 32; ++w) rmax = fmaxf(rmax, s_rmax[w]);
  const bool write = carena != nullptr;
  for (uint64_t j = t; j < m; j += kCandThreads) {
    const uint32_t p = list[j];
    const double x = px[p] - ax, y = py[p] - ay, z = pz[p] - az;
    const double dd = sqrt(x * x + y * y + z * z);
    const double inv = dd > 0.0 ? 1.0 / dd : 0.0;
    const float df = (float)dd;
    const float rw = 1.0f / df;
    if (0.5f * (1.0f - 1e-5f) > rmax * rw) continue;
    const float r0 = (float)(x * inv), r1 = (float)(y * inv), r2 = (float)(z * inv);
    bool f = false;
    for (uint32_t d = 0; d < (uint32_t)kDirs && !f; ++d) {
      const float rho_sf = rho[d];
      if (0.5f * (1.0f - 1e-5f) > rho_sf * rw) continue;
      const float c = cp.dirs[3 * d] * r0 + cp.dirs[3 * d + 1] * r1 + cp.dirs[3 * d + 2] * r2;
      const float cs = fminf(1.0f, c + 1e-5f);
      const float sn = sqrtf(fmaxf(0.0f, (1.0f - cs) * (1.0f + cs)));
      const float clo = (cs >= cdf) ? 1.0f : cs * cdf + sn * sdlf + 1e-6f;
      f = clo > 0.0f && 2.0f * clo * rho_sf * rw * (1.0f + 2e-5f) >= 1.0f;
    }
    if (f) {
      const uint32_t at = atomicAdd(&s_c, 1u);
      if (write && at < cap && at < ccnt[i]) {
        cid[at] = p;
        cds[at] = df;
      }
    }
  }
  __syncthreads();
  const uint32_t c = s_c;
  if (!write) {
    if (t == 0) ccnt[i] = c;
    return;
  }
  if (c != ccnt[i] || c > cap) return;  // the counting pass gave the same count
  if (in_arena) {  // sorted in place (odd-even transposition: the slot holds exactly c entries)
    for (uint32_t r = 0; r < c; ++r) {
      for (uint32_t x = 2 * t + (r & 1); x + 1 < c; x += 2 * kCandThreads) {
        const float dx = cds[x], dy = cds[x + 1];
        if (dx > dy) {
          cds[x] = dy;
          cds[x + 1] = dx;
          const uint32_t tmp = cid[x];
          cid[x] = cid[x + 1];
          cid[x + 1] = tmp;
        }
      }
      __syncthreads();
    }
    return;
  }
  uint32_t P = 32;
  while (P < c) P <<= 1;
  for (uint32_t j = c + t; j < P; j += kCandThreads) {
    cds[j] = INFINITY;
    cid[j] = kInvalid32;
  }
  __syncthreads();
  for (uint32_t k = 2; k <= P; k <<= 1)
    for (uint32_t jj = k >> 1; jj > 0; jj >>= 1) {
      for (uint32_t x = t; x < P; x += kCandThreads) {
        const uint32_t y = x ^ jj;
        if (y > x) {
          const bool up = (x & k) == 0;
          const float dx = cds[x], dy = cds[y];
          if ((dx > dy) == up) {
            cds[x] = dy;
            cds[y] = dx;
            const uint32_t tmp = cid[x];
            cid[x] = cid[y];
            cid[y] = tmp;
          }
        }
      }
      __syncthreads();
    }
  for (uint32_t j = t; j < c; j += kCandThreads) carena[coff[i] + j] = cid[j];
}

// ---- 3. owner-local enumeration ---------------------------------------------------------
// One warp per owner a.  C(a) is staged in shared memory as rounded differences
// p - a; the support candidates are C(a) with ids > a.  Lanes test triangles
// (pairs j < k) and tetrahedra (triples j < k < l, load-balanced over the pairs
// whose three a-faces pass the circumradius bound) for minimality; a minimal
// support whose circumradius certainly exceeds the radius bound of the cone
// holding its centre direction is dropped, the others are classified against
// C(a) by the whole warp, 32 points per step, with ballot counts and an early
// exit once the interior exceeds s_max - size.
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

#ifndef EHGP_HIGHER_OWNER_WARPS
#define EHGP_HIGHER_OWNER_WARPS 8
#endif
#ifndef EHGP_HIGHER_BLOCKS_PER_SM
#define EHGP_HIGHER_BLOCKS_PER_SM 4
#endif
// warps per owner block in k_higher (they share its staged candidate set), and the blocks per
// SM its register budget is sized for: 65536 / (256 threads x 4 blocks) = 64 per thread, 32 warps
// per SM (measured at 50k: 8 x 4 blocks 60.1 ms, 8 x 3 63.5, 8 x 2 81.4; earlier builds 4 x 4
// 83, 4 x 5 82, 12 x 2 83, 8 x 3 77)
constexpr int kHOwnerWarps = EHGP_HIGHER_OWNER_WARPS;
constexpr int kHBlocksPerSM = EHGP_HIGHER_BLOCKS_PER_SM;
constexpr int kCube = 32;       // cube-map cells per face edge for centre directions
constexpr int kCellDirs = 8;    // direction slots per cell (0xffff = unused)

struct HigherTables {
  const float* dirs;       // [kDirs * 3]
  const uint16_t* cells;   // [6 * kCube * kCube * kCellDirs]
  const float* rho;        // [n * kDirs] per-cone radius bounds, by PointId
  double cos_lim;          // cos(delta) raised by a margin: inside the cone for sure
};

template <int KC>
struct OwnerSmemT {  // one owner's staged candidate set (at most KC), shared by the block's warps
  uint32_t sid[KC];
  SetPt spt[KC];
  uint16_t supi[KC];
  float rho[kDirs];
};
// The face mask sits beside it: adm[j * (KC / 32) + w] bit k (j < k): face (a, j, k) within the bound.
using OwnerSmem = OwnerSmemT<kMaxCand>;

struct WarpQueue {  // one warp's queued supports
  uint32_t iids[kMaxInteriorH];
  QEntry q[32];
};

__device__ __forceinline__ int cube_cell(double ux, double uy, double uz) {
  const double ax = fabs(ux), ay = fabs(uy), az = fabs(uz);
  int face;
  double s, t;
  if (ax >= ay && ax >= az) {
    face = ux > 0 ? 0 : 1; s = uy / ax; t = uz / ax;
  } else if (ay >= az) {
    face = uy > 0 ? 2 : 3; s = ux / ay; t = uz / ay;
  } else {
    face = uz > 0 ? 4 : 5; s = ux / az; t = uy / az;
  }
  const int i = min(kCube - 1, max(0, (int)floor((s + 1.0) * 0.5 * kCube)));
  const int j = min(kCube - 1, max(0, (int)floor((t + 1.0) * 0.5 * kCube)));
  return (face * kCube + i) * kCube + j;
}

// True when the sphere's circumradius certainly exceeds the bound of a cone
// that certainly holds its centre direction: no relevant support.
__device__ bool cone_rejects(const QEntry& E, double eA, double eN, const float* rho, const HigherTables& tb) {
  const double nn = sqrt(E.Nx * E.Nx + E.Ny * E.Ny + E.Nz * E.Nz);
  const double en = eN * 1.7320508075688772;
  if (!(en <= 1e-7 * nn)) return false;  // direction not well determined
  const double r_lo = (nn - en) / (2.0 * (fabs(E.A) + eA)) * (1.0 - 1e-12);
  // centre offset N / (2A); the sign of A is the certified orientation sgn
  const double inv = (E.sgn > 0 ? 1.0 : -1.0) / nn;
  const double ux = E.Nx * inv, uy = E.Ny * inv, uz = E.Nz * inv;
  const uint16_t* cl = tb.cells + (uint64_t)cube_cell(ux, uy, uz) * kCellDirs;
  double bound = INFINITY;
  for (int i = 0; i < kCellDirs; ++i) {
    const uint32_t s = cl[i];
    if (s == 0xffffu) break;
    const double cs = (double)tb.dirs[3 * s] * ux + (double)tb.dirs[3 * s + 1] * uy + (double)tb.dirs[3 * s + 2] * uz;
    if (cs >= tb.cos_lim) bound = fmin(bound, (double)rho[s]);
  }
  return r_lo > bound * (1.0 + 1e-9);
}

// Every point of the closed ball lies within its diameter of a: |p - a|^2 <= 4 r^2 = |N|^2 / A^2.
// The cut adds 2e-5 for the FP64 values of A and N (relative errors below 1e-7 when the cut
// is used at all) and for the binary32 distances that order C(a); otherwise no cut.
__device__ float sphere_cut(const QEntry& E, double eA, double eN) {
  const double nn2 = E.Nx * E.Nx + E.Ny * E.Ny + E.Nz * E.Nz;
  if (!(eA <= 1e-7 * fabs(E.A)) || !(3.0 * eN * eN <= 1e-14 * nn2)) return INFINITY;
  return __double2float_ru(nn2 / (E.A * E.A) * (1.0 + 2e-5));
}

// Classifies the queued supports against C(a) with the whole warp and emits the relevant ones.
template <int KC, typename Count>
__device__ __forceinline__ void classify_queue(const OwnerSmemT<KC>& S, WarpQueue& Q, uint32_t qn, uint32_t m, const Cloud& c,
                               uint32_t smax, HigherRec* out, uint32_t cap, uint32_t* counter, uint32_t lane,
                               Count& emitted) {
  for (uint32_t e = 0; e < qn; ++e) {
    const QEntry E = Q.q[e];
    const uint32_t icap = smax - (uint32_t)E.size;
    uint32_t interior = 0, shell = (uint32_t)E.size, wit = kInvalid32;
    bool reject = false;
    for (uint32_t base = 0; base < m; base += 32) {
      // C(a) is sorted by distance from a: the rest of it lies beyond the sphere's diameter
      if (S.spt[base].q > (double)E.cut) break;
      const uint32_t i = base + lane;
      int sd = 1;
      uint32_t w = kInvalid32;
      if (i < m) {
        w = S.sid[i];
        if (w != E.ids[1] && w != E.ids[2] && w != E.ids[3]) {
          const SetPt p = S.spt[i];
          const double v = E.A * p.q - ((p.x * E.Nx + p.y * E.Ny) + p.z * E.Nz);
          sd = fsign(v, E.bnd);
          if (sd == 2) sd = side_exact(c, Q.q[e].ids, E.size, w);  // the queue entry's ids (shared memory)
          sd *= E.sgn;
        }
      }
      const uint32_t bi = __ballot_sync(0xffffffffu, sd < 0), bs = __ballot_sync(0xffffffffu, sd == 0);
      if (sd < 0) {
        const uint32_t at = interior + __popc(bi & lanemask_lt());
        if (at < icap) Q.iids[at] = w;
      }
      interior += __popc(bi);
      if (interior > icap) {
        reject = true;
        break;
      }
      if (bs) {
        shell += __popc(bs);
        wit = min(wit, __reduce_min_sync(0xffffffffu, sd == 0 ? w : kInvalid32));
      }
    }
    __syncwarp();
    if (!reject) {  // warp-uniform: the record is written by 16 lanes, one word each
      uint32_t slot = 0;
      if (lane == 0) {
        for (uint32_t i = 1; i < interior; ++i) {  // interior ids ascending, in place
          const uint32_t x = Q.iids[i];
          uint32_t j = i;
          while (j > 0 && Q.iids[j - 1] > x) {
            Q.iids[j] = Q.iids[j - 1];
            --j;
          }
          Q.iids[j] = x;
        }
        slot = atomicAdd(counter, 1u);
        ++emitted;
      }
      slot = __shfl_sync(0xffffffffu, slot, 0);
      __syncwarp();
      // support ids ascending (a triangle's fourth slot sorts last and is written as 0)
      uint32_t s0 = E.ids[0], s1 = E.ids[1], s2 = E.ids[2], s3 = E.size == 4 ? E.ids[3] : kInvalid32;
      auto cswap = [](uint32_t& x, uint32_t& y) {
        const uint32_t lo = min(x, y), hi = max(x, y);
        x = lo;
        y = hi;
      };
      cswap(s0, s1);
      cswap(s2, s3);
      cswap(s0, s2);
      cswap(s1, s3);
      cswap(s1, s2);
      if (E.size != 4) s3 = 0u;
      if (slot < cap && lane < 16) {
        uint32_t v;
        if (lane == 0) v = (uint32_t)E.size;
        else if (lane == 1) v = s0;
        else if (lane == 2) v = s1;
        else if (lane == 3) v = s2;
        else if (lane == 4) v = s3;
        else if (lane == 5) v = interior;
        else if (lane == 6) v = shell;
        else if (lane == 7) v = wit;
        else v = lane - 8 < interior ? Q.iids[lane - 8] : kInvalid32;
        reinterpret_cast<uint32_t*>(out + slot)[lane] = v;
      }
    }
    __syncwarp();
  }
}

__device__ __forceinline__ void decode_pair(uint64_t t, uint32_t& lo, uint32_t& hi) {
  uint32_t i = (uint32_t)((sqrt(8.0 * (double)t + 1.0) - 1.0) / 2.0);
  while ((uint64_t)(i + 1) * i / 2 > t) --i;
  while ((uint64_t)(i + 2) * (i + 1) / 2 <= t) ++i;
  lo = (uint32_t)(t - (uint64_t)(i + 1) * i / 2);
  hi = i + 1;
}

// Position of the r-th (0-based) set bit of x; x has more than r set bits.
__device__ __forceinline__ uint32_t select_bit(uint32_t x, uint32_t r) {
  uint32_t pos = 0;
  for (int w = 16; w > 0; w >>= 1) {
    const uint32_t cnt = __popc(x & ((1u << w) - 1u));
    if (r >= cnt) {
      r -= cnt;
      x >>= w;
      pos += w;
    }
  }
  return pos;
}

// Parts of one owner's enumeration that a block runs (higher_owner's `phases`): the
// triangles with the face mask, the tetrahedra, clearing the mask first, the owner's counters.
constexpr uint32_t kPhTri = 1, kPhTet = 2, kPhClear = 4, kPhStats = 8, kPhAll = 15;

// Enumeration of owner a over its candidate set clist[0..m) (m <= KC, sorted by binary32
// distance from a), by the whole block; adm holds KC * KC / 32 words (shared or global).
// The block runs the pairs [t_lo, t_hi) of the support candidates (the triangles (a, j, k) and
// the tetrahedra whose first two candidates are the pair), so one owner can be split over
// blocks: all triangles (which complete the face mask) before any tetrahedron.
template <int KC>
__device__ __forceinline__ void higher_owner(uint32_t a, const uint32_t* __restrict__ clist, uint32_t m,
                                             OwnerSmemT<KC>& S, uint32_t* adm, WarpQueue* wq, const Ctl& ctl,
                                             const HigherTables& tb, const double* __restrict__ px,
                                             const double* __restrict__ py, const double* __restrict__ pz,
                                             const int* __restrict__ cloud_scale, HigherRec* __restrict__ out,
                                             uint32_t* __restrict__ counter, unsigned long long* __restrict__ stats,
                                             uint64_t t_lo = 0, uint64_t t_hi = ~0ull, uint32_t phases = kPhAll) {
  constexpr uint32_t kWords = KC / 32;
  __shared__ double s_Mp;
  __shared__ uint32_t s_mc;
  __shared__ float s_rmax[kHOwnerWarps];
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  WarpQueue& Q = wq[warp];
  const Cloud c{px, py, pz, cloud_scale[0]};
  const double ax = px[a], ay = py[a], az = pz[a];
  // warp 0 stages C(a) (and the support candidates, ids above a); the block clears the
  // face mask and loads the cone bounds
  uint32_t mc = 0;
  double Mp = 0.0;
  for (uint32_t base = 0; warp == 0 && base < m; base += 32) {
    const uint32_t i = base + lane;
    const uint32_t p = i < m ? clist[i] : kInvalid32;
    if (i < m) {
      SetPt s;
      s.x = px[p] - ax;
      s.y = py[p] - ay;
      s.z = pz[p] - az;
      s.q = (s.x * s.x + s.y * s.y) + s.z * s.z;
      S.sid[i] = p;
      S.spt[i] = s;
      Mp = fmax(Mp, ptmax(s));
    }
    const bool f = i < m && p > a;
    const uint32_t b = __ballot_sync(0xffffffffu, f);
    if (f) S.supi[mc + __popc(b & lanemask_lt())] = (uint16_t)i;
    mc += __popc(b);
  }
  float rmax = 0.f;
  for (uint32_t d = threadIdx.x; d < (uint32_t)kDirs; d += 32 * kHOwnerWarps) {
    const float r = tb.rho[(uint64_t)a * kDirs + d];
    S.rho[d] = r;
    rmax = fmaxf(rmax, r);
  }
  if (phases & kPhClear)
    for (uint32_t i = threadIdx.x; i < (uint32_t)KC * kWords; i += 32 * kHOwnerWarps) adm[i] = 0u;
  for (int off = 16; off > 0; off >>= 1) {
    Mp = fmax(Mp, __shfl_xor_sync(0xffffffffu, Mp, off));
    rmax = fmaxf(rmax, __shfl_xor_sync(0xffffffffu, rmax, off));
  }
  if (lane == 0) s_rmax[warp] = rmax;
  if (threadIdx.x == 0) {
    s_Mp = Mp * (1.0 + 1e-15);
    s_mc = mc;
  }
  __syncthreads();
  Mp = s_Mp;
  mc = s_mc;
  rmax = s_rmax[0];
  for (int w = 1; w < kHOwnerWarps; ++w) rmax = fmaxf(rmax, s_rmax[w]);
  const double rmax2 = (double)rmax * (double)rmax * (1.0 + 1e-12);
  // per-lane work counters: 32-bit where a block's share of an owner cannot reach 2^32 (sets of
  // up to 1,024 candidates, or a chunk of pairs), else 64-bit (registers are the scarce unit)
  using Count = typename std::conditional<(KC <= 1024), uint32_t, unsigned long long>::type;
  Count tested = 0, minimal = 0, pruned = 0, classified = 0, emitted = 0, admitted = 0;
  const uint64_t P2 = min((uint64_t)mc * (mc - 1) / 2, t_hi);
  // --- triangles (a, j, k); also the face bound adm(j, k) for the tetrahedra
  for (uint64_t t0 = t_lo + 32 * warp; (phases & kPhTri) && t0 < P2; t0 += 32 * kHOwnerWarps) {
    const uint64_t t = t0 + lane;
    bool push = false;
    QEntry E;
    if (t < P2) {
      uint32_t j, k;
      decode_pair(t, j, k);
      const uint32_t ij = S.supi[j], ik = S.supi[k];
      E.ids[0] = a;
      E.ids[1] = S.sid[ij];
      E.ids[2] = S.sid[ik];
      E.ids[3] = kInvalid32;
      double eA, eN;
      bool face_ok;
      ++tested;
      const int st = tri_eval(c, S.spt[ij], S.spt[ik], E.ids[0], E.ids[1], E.ids[2], Mp, rmax2, E, eA, eN, face_ok);
      if (face_ok) {
        atomicOr(&adm[j * kWords + (k >> 5)], 1u << (k & 31));
        ++admitted;
      }
      if (st == 0 && ctl.smax >= 3) {
        ++minimal;
        if (cone_rejects(E, eA, eN, S.rho, tb)) ++pruned;
        else {
          push = true;
          E.cut = sphere_cut(E, eA, eN);
        }
      }
    }
    const uint32_t b = __ballot_sync(0xffffffffu, push);
    if (push) Q.q[__popc(b & lanemask_lt())] = E;
    __syncwarp();
    classified += __popc(b);
    classify_queue(S, Q, __popc(b), m, c, ctl.smax, out, ctl.cap, counter, lane, emitted);
  }
  if ((phases & kPhTri) && (phases & kPhTet)) __syncthreads();  // the face mask is complete
  // --- tetrahedra (a, j, k, l), j < k < l with adm(j,k), adm(j,l), adm(k,l)
  if (ctl.smax >= 4 && (phases & kPhTet)) {
    for (uint64_t t0 = t_lo + 32 * warp; t0 < P2; t0 += 32 * kHOwnerWarps) {
      const uint64_t t = t0 + lane;
      uint32_t j = 0, k = 0, cnt = 0;
      if (t < P2) {
        decode_pair(t, j, k);
        if ((adm[j * kWords + (k >> 5)] >> (k & 31)) & 1u) {
          const uint32_t w0 = (k + 1) >> 5;
          for (uint32_t w = w0; w < kWords; ++w) {
            uint32_t bits = adm[j * kWords + w] & adm[k * kWords + w];
            if (w == w0) bits &= ((k + 1) & 31) ? (0xffffffffu << ((k + 1) & 31)) : 0xffffffffu;
            cnt += __popc(bits);
          }
        }
      }
      uint32_t incl = cnt;
      for (int off = 1; off < 32; off <<= 1) {
        const uint32_t x = __shfl_up_sync(0xffffffffu, incl, off);
        if ((int)lane >= off) incl += x;
      }
      const uint32_t excl = incl - cnt, total = __shfl_sync(0xffffffffu, incl, 31);
      for (uint32_t q0 = 0; q0 < total; q0 += 32) {
        const uint32_t q = q0 + lane;
        // owner lane: the largest o with excl_o <= q
        uint32_t o = 0;
        for (uint32_t step = 16; step > 0; step >>= 1) {
          const uint32_t v = __shfl_sync(0xffffffffu, excl, o + step);
          if (v <= q) o += step;
        }
        const uint32_t oj = __shfl_sync(0xffffffffu, j, o), ok = __shfl_sync(0xffffffffu, k, o);
        const uint32_t oe = __shfl_sync(0xffffffffu, excl, o);
        bool push = false;
        QEntry E;
        if (q < total) {
          uint32_t r = q - oe, l = 0;
          const uint32_t w0 = (ok + 1) >> 5;
          for (uint32_t w = w0; w < kWords; ++w) {
            uint32_t bits = adm[oj * kWords + w] & adm[ok * kWords + w];
            if (w == w0) bits &= ((ok + 1) & 31) ? (0xffffffffu << ((ok + 1) & 31)) : 0xffffffffu;
            const uint32_t pc = __popc(bits);
            if (r < pc) {
              l = w * 32 + select_bit(bits, r);
              break;
            }
            r -= pc;
          }
          const uint32_t ij = S.supi[oj], ik = S.supi[ok], il = S.supi[l];
          E.ids[0] = a;
          E.ids[1] = S.sid[ij];
          E.ids[2] = S.sid[ik];
          E.ids[3] = S.sid[il];
          double eA, eN;
          ++tested;
          if (quad_eval(c, S.spt[ij], S.spt[ik], S.spt[il], E.ids[0], E.ids[1], E.ids[2], E.ids[3], Mp, E, eA, eN) == 0) {
            ++minimal;
            if (cone_rejects(E, eA, eN, S.rho, tb)) ++pruned;
            else {
              push = true;
              E.cut = sphere_cut(E, eA, eN);
            }
          }
        }
        const uint32_t b = __ballot_sync(0xffffffffu, push);
        if (push) Q.q[__popc(b & lanemask_lt())] = E;
        __syncwarp();
        classified += __popc(b);
        classify_queue(S, Q, __popc(b), m, c, ctl.smax, out, ctl.cap, counter, lane, emitted);
      }
    }
  }
  for (int off = 16; off > 0; off >>= 1) {
    tested += __shfl_xor_sync(0xffffffffu, tested, off);
    minimal += __shfl_xor_sync(0xffffffffu, minimal, off);
    pruned += __shfl_xor_sync(0xffffffffu, pruned, off);
    admitted += __shfl_xor_sync(0xffffffffu, admitted, off);
  }
  if (lane == 0) {
    atomicAdd(stats + 0, (unsigned long long)tested);
    atomicAdd(stats + 1, (unsigned long long)classified);
    atomicAdd(stats + 2, (unsigned long long)emitted);
    if (warp == 0 && (phases & kPhStats)) {
      atomicAdd(stats + 3, (unsigned long long)m);
      atomicAdd(stats + 4, (unsigned long long)mc);
    }
    atomicAdd(stats + 5, (unsigned long long)minimal);
    atomicAdd(stats + 6, (unsigned long long)pruned);
    atomicAdd(stats + 7, (unsigned long long)admitted);
  }
}

__global__ void __launch_bounds__(32 * kHOwnerWarps, kHBlocksPerSM)
k_higher(uint32_t n, Ctl ctl, HigherTables tb, const uint32_t* __restrict__ leaf_pid, const uint32_t* __restrict__ cand,
         const uint32_t* __restrict__ candc, const double* __restrict__ px, const double* __restrict__ py,
         const double* __restrict__ pz, const int* __restrict__ cloud_scale, HigherRec* __restrict__ out,
         uint32_t* __restrict__ counter, unsigned long long* __restrict__ stats) {
  __shared__ OwnerSmem S;
  __shared__ uint32_t adm[kMaxCand * (kMaxCand / 32)];
  __shared__ WarpQueue wq[kHOwnerWarps];
  const uint32_t pos = blockIdx.x;
  if (pos >= n) return;
  const uint32_t a = leaf_pid[pos];
  const uint32_t m = candc[a];
  if (m > (uint32_t)kMaxCand) return;  // a large candidate set (k_higher_large)
  higher_owner<kMaxCand>(a, cand + (uint64_t)a * kMaxCand, m, S, adm, wq, ctl, tb, px, py, pz, cloud_scale, out,
                         counter, stats);
}

// Owners whose candidate set exceeds kMaxCand: the same enumeration with the set staged in
// dynamic shared memory (at most KC candidates) and the face mask in shared memory (KC <= 1024)
// or in a per-block global scratch; blocks loop over the owners.
// Placement of a large owner's staged set and face mask: kMode 0 both in shared memory,
// 1 the set in shared memory and the mask in global scratch, 2 both in global scratch.
template <int KC>
constexpr size_t large_set_bytes() {
  return (sizeof(OwnerSmemT<KC>) + 15) / 16 * 16;
}
template <int KC>
constexpr size_t large_adm_bytes() {
  return (size_t)KC * (KC / 32) * 4;
}
template <int KC, int kMode>
constexpr size_t large_smem() {
  return sizeof(WarpQueue) * kHOwnerWarps + (kMode <= 1 ? large_set_bytes<KC>() : 0) +
         (kMode == 0 ? large_adm_bytes<KC>() : 0);
}
template <int KC, int kMode>
constexpr size_t large_scratch_bytes() {  // per block
  return (kMode >= 1 ? large_adm_bytes<KC>() : 0) + (kMode == 2 ? large_set_bytes<KC>() : 0);
}

template <int KC, int kMode>
__global__ void __launch_bounds__(32 * kHOwnerWarps, 1)
k_higher_large(uint32_t nown, const uint32_t* __restrict__ owners, const uint64_t* __restrict__ coff,
               const uint32_t* __restrict__ carena, Ctl ctl, HigherTables tb, const double* __restrict__ px,
               const double* __restrict__ py, const double* __restrict__ pz, const int* __restrict__ cloud_scale,
               HigherRec* __restrict__ out, uint32_t* __restrict__ counter, unsigned long long* __restrict__ stats,
               unsigned char* __restrict__ scratch) {
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned char* mine = scratch + (uint64_t)blockIdx.x * large_scratch_bytes<KC, kMode>();
  WarpQueue* wq = reinterpret_cast<WarpQueue*>(smem);
  unsigned char* after_q = smem + sizeof(WarpQueue) * kHOwnerWarps;
  OwnerSmemT<KC>& S = *reinterpret_cast<OwnerSmemT<KC>*>(kMode <= 1 ? after_q : mine + large_adm_bytes<KC>());
  uint32_t* adm = reinterpret_cast<uint32_t*>(kMode == 0 ? after_q + large_set_bytes<KC>() : mine);
  for (uint32_t i = blockIdx.x; i < nown; i += gridDim.x) {
    const uint32_t m = (uint32_t)(coff[i + 1] - coff[i]);
    if (m <= (uint32_t)KC)
      higher_owner<KC>(owners[i], carena + coff[i], m, S, adm, wq, ctl, tb, px, py, pz, cloud_scale, out, counter,
                       stats);
    __syncthreads();  // the next owner restages the shared set
  }
}

// Owners with up to KC candidates split over blocks: block w runs pair chunk
// w - chunk_off[i] (kSplitPairs pairs) of owner i, the last i with chunk_off[i] <= w.  Phase
// kPhTri (with kPhStats on each owner's first chunk) fills the owners' face masks in global
// memory (adm_all, KC * KC / 32 words per owner, zero on entry); the next launch, kPhTet,
// reads them complete.  An owner's work is its O(m^2) pairs and their tetrahedra, so the
// large sets spread over every SM instead of one block each.
// pairs per chunk: small chunks keep the tetrahedron launch balanced (its chunks differ widely
// in admissible tetrahedra); measured on 3k/8k/20k mixtures and a 20k clustered cloud, k_higher
// 46/116/67/153 ms at 8,192, 29/67/60/93 at 2,048, 28/61/59/90 at 1,024, 29/61/61/92 at 512
constexpr uint32_t kSplitPairs = 1024;
template <int KC>
__global__ void __launch_bounds__(32 * kHOwnerWarps, 2)
k_higher_split(uint32_t nown, const uint32_t* __restrict__ owners, const uint64_t* __restrict__ coff,
               const uint32_t* __restrict__ carena, const uint32_t* __restrict__ chunk_off, uint32_t phase, Ctl ctl,
               HigherTables tb, const double* __restrict__ px, const double* __restrict__ py,
               const double* __restrict__ pz, const int* __restrict__ cloud_scale, HigherRec* __restrict__ out,
               uint32_t* __restrict__ counter, unsigned long long* __restrict__ stats, uint32_t* __restrict__ adm_all) {
  extern __shared__ __align__(16) unsigned char smem[];
  WarpQueue* wq = reinterpret_cast<WarpQueue*>(smem);
  OwnerSmemT<KC>& S = *reinterpret_cast<OwnerSmemT<KC>*>(smem + sizeof(WarpQueue) * kHOwnerWarps);
  const uint32_t w = blockIdx.x;
  uint32_t lo = 0, hi = nown;  // the owner: last i with chunk_off[i] <= w
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) / 2;
    if (chunk_off[mid] <= w) lo = mid;
    else hi = mid;
  }
  const uint32_t i = lo, c = w - chunk_off[i];
  const uint32_t m = (uint32_t)(coff[i + 1] - coff[i]);
  if (m > (uint32_t)KC) return;
  const uint32_t ph = phase == kPhTri ? (c == 0 ? kPhTri | kPhStats : kPhTri) : kPhTet;
  higher_owner<KC>(owners[i], carena + coff[i], m, S, adm_all + (uint64_t)i * KC * (KC / 32), wq, ctl, tb, px, py,
                   pz, cloud_scale, out, counter, stats, (uint64_t)c * kSplitPairs, (uint64_t)(c + 1) * kSplitPairs,
                   ph);
}
template <int KC>
constexpr size_t split_smem() {
  return sizeof(WarpQueue) * kHOwnerWarps + large_set_bytes<KC>();
}

// ---- single predicate evaluations (the product kernels' own filters and exact paths) ------
// For the reference's predicate fixtures: one device thread evaluates one predicate on
// PointIds of the resident cloud with the helpers the enumeration uses (FP64 with the
// uniform error bounds, then the fixed-width exact integers).  out[0] the result, out[1] 1 when
// an FP64 filter decided it (0 when the exact path did).
__device__ uint32_t g_pred_ids[16];
__device__ int32_t g_pred_out[2];

__global__ void k_predicate(uint32_t pred, uint32_t count, const double* __restrict__ px,
                            const double* __restrict__ py, const double* __restrict__ pz,
                            const int* __restrict__ cloud_scale) {
  const Cloud c{px, py, pz, cloud_scale[0]};
  uint32_t ids[16];
  for (uint32_t i = 0; i < count && i < 16; ++i) ids[i] = g_pred_ids[i];
  int32_t res = 0, fp = 0;
  auto setpt = [&](uint32_t p, uint32_t a) {
    SetPt s;
    s.x = px[p] - px[a];
    s.y = py[p] - py[a];
    s.z = pz[p] - pz[a];
    s.q = (s.x * s.x + s.y * s.y) + s.z * s.z;
    return s;
  };
  auto status = [&](const uint32_t* sup, int size, QEntry& E, double& eA, double& eN) -> int {
    if (size == 1) return 0;
    if (size == 2) return sup[0] == sup[1] ? 3 : 0;
    const SetPt e1 = setpt(sup[1], sup[0]), e2 = setpt(sup[2], sup[0]);
    double Mp = fmax(ptmax(e1), ptmax(e2));
    E.ids[0] = sup[0];
    E.ids[1] = sup[1];
    E.ids[2] = sup[2];
    E.ids[3] = size == 4 ? sup[3] : kInvalid32;
    if (size == 3) {
      bool adm;
      return tri_eval(c, e1, e2, sup[0], sup[1], sup[2], Mp * (1.0 + 1e-15), INFINITY, E, eA, eN, adm);
    }
    const SetPt e3 = setpt(sup[3], sup[0]);
    Mp = fmax(Mp, ptmax(e3));
    return quad_eval(c, e1, e2, e3, sup[0], sup[1], sup[2], sup[3], Mp * (1.0 + 1e-15), E, eA, eN);
  };
  if (pred == 1) {  // side of the last id against the support sphere of the others
    const int size = (int)count - 1;
    const uint32_t w = ids[size];
    QEntry E;
    double eA = 0, eN = 0;
    const int st = size >= 3 ? status(ids, size, E, eA, eN) : -1;
    if (st == 0) {  // a minimal support: the enumeration's classification
      const SetPt p = setpt(w, ids[0]);
      const double v = E.A * p.q - ((p.x * E.Nx + p.y * E.Ny) + p.z * E.Nz);
      int sd = fsign(v, E.bnd);
      fp = sd != 2;
      if (sd == 2) sd = side_exact(c, ids, size, w);
      res = sd * E.sgn;
    } else {  // any other support sphere: exact (orientation of A from its exact sign)
      W A;
      WV N;
      exact_sphere(c, ids, size, A, N);
      res = A.sign() == 0 ? 2 : side_exact(c, ids, size, w) * (A.sign() < 0 ? -1 : 1);  // 2: no sphere
    }
  } else if (pred == 2) {  // status of a 1- to 4-point support: 0 minimal, 1 boundary, 2 exterior, 3 dependent
    QEntry E;
    double eA = 0, eN = 0;
    res = status(ids, (int)count, E, eA, eN);
  } else if (pred == 3) {  // sign of level(left) - level(right); ids: left size, left ids, right ids
    const int s1 = (int)ids[0];
    res = level_cmp_exact(c, ids + 1, s1, ids + 1 + s1, (int)count - 1 - s1);
  } else if (pred == 4) {  // sign of |ids[1] - ids[0]|^2 - |ids[2] - ids[0]|^2
    res = dist_cmp_exact(c, ids, 1, ids[1], ids[2]);
  }
  g_pred_out[0] = res;
  g_pred_out[1] = fp;
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
  if (i >= n || (todo[i] != 1 && todo[i] != 3)) return;
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

// Cube-map cells over the sphere of directions (the same face/cell mapping as
// cube_cell): each cell lists the directions nearest to its centre that lie
// within delta + the cell's angular radius, so that the direction covering any
// u in the cell is listed.  The device re-checks every listed cone, so a short
// list only costs pruning, never correctness.
void cube_cells(const std::vector<float>& dirs, double delta, std::vector<uint16_t>& cells) {
  cells.assign((size_t)6 * kCube * kCube * kCellDirs, (uint16_t)0xffff);
  auto vec = [](int face, double s, double t) {
    std::array<double, 3> p{};
    switch (face) {
      case 0: p = {1, s, t}; break;
      case 1: p = {-1, s, t}; break;
      case 2: p = {s, 1, t}; break;
      case 3: p = {s, -1, t}; break;
      case 4: p = {s, t, 1}; break;
      default: p = {s, t, -1}; break;
    }
    const double l = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
    return std::array<double, 3>{p[0] / l, p[1] / l, p[2] / l};
  };
  auto angle = [](const std::array<double, 3>& x, const std::array<double, 3>& y) {
    return std::acos(std::max(-1.0, std::min(1.0, x[0] * y[0] + x[1] * y[1] + x[2] * y[2])));
  };
  const size_t nd = dirs.size() / 3;
  for (int face = 0; face < 6; ++face)
    for (int i = 0; i < kCube; ++i)
      for (int j = 0; j < kCube; ++j) {
        const double s0 = -1.0 + 2.0 * i / kCube, s1 = -1.0 + 2.0 * (i + 1) / kCube;
        const double t0 = -1.0 + 2.0 * j / kCube, t1 = -1.0 + 2.0 * (j + 1) / kCube;
        const auto ctr = vec(face, 0.5 * (s0 + s1), 0.5 * (t0 + t1));
        double eps = 0;
        for (double s : {s0, s1})
          for (double t : {t0, t1}) eps = std::max(eps, angle(ctr, vec(face, s, t)));
        std::vector<std::pair<double, uint16_t>> near;
        for (size_t d = 0; d < nd; ++d) {
          const std::array<double, 3> dv{dirs[3 * d], dirs[3 * d + 1], dirs[3 * d + 2]};
          const double g = angle(ctr, dv);
          if (g <= delta + eps + 1e-6) near.push_back({g, (uint16_t)d});
        }
        std::sort(near.begin(), near.end());
        uint16_t* out = &cells[((size_t)(face * kCube + i) * kCube + j) * kCellDirs];
        for (size_t q = 0; q < near.size() && q < (size_t)kCellDirs; ++q) out[q] = near[q].second;
      }
}

}  // namespace

// Bytes of each record buffer for `c` records: raw, sorted, khi, klo, order0, order1, radix counts.
static void higher_record_bytes(uint64_t c, uint64_t* b) {
  b[0] = c * sizeof(HigherRec);
  b[1] = c * sizeof(HigherRec);
  b[2] = c * sizeof(uint64_t);
  b[3] = c * sizeof(uint64_t);
  b[4] = c * sizeof(uint32_t);
  b[5] = c * sizeof(uint32_t);
  b[6] = 256ull * ((c + kRadixTile - 1) / kRadixTile) * sizeof(uint32_t);
}

cudaError_t higher_records_alloc(Ctx& ctx, uint64_t capacity) {
  HigherBuffers& h = ctx.hb;
  void** bufs[7] = {&h.raw, &h.sorted, (void**)&h.khi, (void**)&h.klo, (void**)&h.order0, (void**)&h.order1,
                    (void**)&h.radix_counts};
  uint64_t old_b[7], new_b[7];
  higher_record_bytes(h.capacity, old_b);
  higher_record_bytes(capacity, new_b);
  for (int i = 0; i < 7; ++i) {
    ctx_free(ctx, *bufs[i], old_b[i]);
    *bufs[i] = nullptr;
  }
  h.capacity = 0;
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
  h.capacity = (uint32_t)capacity;
  return cudaSuccess;
}

cudaError_t higher_alloc(Ctx& ctx) {
  const uint64_t n = ctx.max_points;
  HigherBuffers& h = ctx.hb;
  cudaError_t e = cudaSuccess;
  // records: about 200 per point in uniform clouds and 450 in jittered lattices; the buffer
  // starts below that and grows on demand (count -> allocate -> emit)
  if ((e = higher_records_alloc(ctx, 128 * n + 4096)) != cudaSuccess) return e;
#define EHGP_ALLOC(ptr, bytes) \
  if ((e = ctx_alloc(ctx, (void**)&(ptr), (bytes))) != cudaSuccess) return e
  EHGP_ALLOC(h.nb, n * kMaxNb * sizeof(uint32_t));
  EHGP_ALLOC(h.nbc, n * sizeof(uint32_t));
  EHGP_ALLOC(h.cand, n * kMaxCand * sizeof(uint32_t));
  EHGP_ALLOC(h.candc, n * sizeof(uint32_t));
  EHGP_ALLOC(h.gather_r2, n * sizeof(double));
  EHGP_ALLOC(h.rcap, n * sizeof(double));
  EHGP_ALLOC(h.todo, n * sizeof(uint8_t));
  EHGP_ALLOC(h.counters, 8 * sizeof(uint32_t));
  EHGP_ALLOC(h.stats, 8 * sizeof(unsigned long long));
  std::vector<float> dirs;
  double delta = 0;
  icosphere(dirs, delta);
  if (dirs.size() != 3 * (size_t)kDirs) return cudaErrorInvalidValue;
  std::vector<uint16_t> cells;
  cube_cells(dirs, delta, cells);
  EHGP_ALLOC(h.dirs, dirs.size() * sizeof(float));
  EHGP_ALLOC(h.cells, cells.size() * sizeof(uint16_t));
  EHGP_ALLOC(h.rho, n * kDirs * sizeof(float));
#undef EHGP_ALLOC
  h.delta = delta;
  h.cos_lim = std::cos(delta) + 1e-6;
  if ((e = cudaMemcpy(h.cells, cells.data(), cells.size() * sizeof(uint16_t), cudaMemcpyHostToDevice)) != cudaSuccess)
    return e;
  return cudaMemcpy(h.dirs, dirs.data(), dirs.size() * sizeof(float), cudaMemcpyHostToDevice);
}

// Grows a device array of ctx to hold `need` elements of `elem` bytes (contents dropped).
template <class T>
cudaError_t grow_array(Ctx& ctx, T*& ptr, uint64_t& cap, uint64_t need, uint64_t elem) {
  if (cap >= need && ptr) return cudaSuccess;
  ctx_free(ctx, ptr, cap * elem);
  ptr = nullptr;
  cap = 0;
  const uint64_t c = need + need / 4 + 256;
  const cudaError_t e = ctx_alloc(ctx, (void**)&ptr, c * elem);
  if (e == cudaSuccess) cap = c;
  return e;
}

// Neighbour lists of the owners in `big` (their current gather radii) into the arena:
// counted, the arena grown to fit, then written (count -> allocate -> write); off receives
// the prefix offsets (also on the device in h.big_off).
int gather_big_lists(Ctx& ctx, uint32_t root, const std::vector<uint32_t>& big, std::vector<uint64_t>& off,
                     uint64_t* launches) {
  HigherBuffers& h = ctx.hb;
  LbvhBuffers& b = ctx.lb;
  GeomBuffers& g = ctx.gb;
  cudaStream_t st = ctx.stream;
  const uint32_t nb = (uint32_t)big.size();
  cudaError_t e = cudaSuccess;
  if (h.big_cap < nb) {
    uint64_t c1 = h.big_cap, c2 = h.big_cap, c3 = h.big_cap;
    if ((e = grow_array(ctx, h.big_ids, c1, nb, 4)) != cudaSuccess ||
        (e = grow_array(ctx, h.big_off, c2, nb + 1, 8)) != cudaSuccess ||
        (e = grow_array(ctx, h.big_cnt, c3, nb, 4)) != cudaSuccess) {
      cudaGetLastError();
      h.big_cap = 0;
      return abi_fail(&ctx, EHGP_ERR_OUT_OF_MEMORY, "the large-neighbourhood owners do not fit the device");
    }
    h.big_cap = std::min(c1, std::min(c2 - 1, c3));
  }
  cudaMemcpyAsync(h.big_ids, big.data(), (uint64_t)nb * 4, cudaMemcpyHostToDevice, st);
  k_gather_big<<<nblocks((uint64_t)nb * 32, 128), 128, 0, st>>>(nb, h.big_ids, root, g.tnodes, b.leaf_pid, b.n_begin, b.n_end, b.px,
                                                 b.py, b.pz, h.gather_r2, nullptr, nullptr, h.big_cnt, ctx.d_err);
  ++*launches;
  std::vector<uint32_t> cnt(nb);
  uint32_t err = 0;
  cudaMemcpyAsync(cnt.data(), h.big_cnt, (uint64_t)nb * 4, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(&err, ctx.d_err, 4, cudaMemcpyDeviceToHost, st);
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return abi_cuda_fail(&ctx, e, "large neighbourhoods");
  if (err) return abi_device_status(&ctx, err);
  off.assign(nb + 1, 0);
  for (uint32_t i = 0; i < nb; ++i) off[i + 1] = off[i] + cnt[i];
  if ((e = grow_array(ctx, h.big_arena, h.arena_cap, off[nb], 4)) != cudaSuccess) {
    cudaGetLastError();
    return abi_fail(&ctx, EHGP_ERR_OUT_OF_MEMORY, "the large neighbourhoods do not fit the device");
  }
  cudaMemcpyAsync(h.big_off, off.data(), (uint64_t)(nb + 1) * 8, cudaMemcpyHostToDevice, st);
  k_gather_big<<<nblocks((uint64_t)nb * 32, 128), 128, 0, st>>>(nb, h.big_ids, root, g.tnodes, b.leaf_pid, b.n_begin, b.n_end, b.px,
                                                 b.py, b.pz, h.gather_r2, h.big_off, h.big_arena, h.big_cnt,
                                                 ctx.d_err);
  ++*launches;
  return EHGP_OK;
}

// One round of the large-neighbourhood path for the owners in `big`: their lists, then the
// certified direction tables and candidate sets.
int higher_big_round(Ctx& ctx, const CertParams& cp, uint32_t root, const std::vector<uint32_t>& big,
                     std::vector<uint64_t>& off, uint64_t* launches) {
  HigherBuffers& h = ctx.hb;
  LbvhBuffers& b = ctx.lb;
  cudaStream_t st = ctx.stream;
  const uint32_t nb = (uint32_t)big.size();
  int s = gather_big_lists(ctx, root, big, off, launches);
  if (s != EHGP_OK) return s;
  // the attribute is per function and device: set on every round (cheap)
  cudaError_t e = cudaFuncSetAttribute(k_dirtable_big, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBigSmem);
  if (e != cudaSuccess) return abi_cuda_fail(&ctx, e, "large-neighbourhood shared memory");
  k_dirtable_big<<<nb, kBigThreads, kBigSmem, st>>>(nb, cp, h.big_ids, h.big_off, h.big_arena, b.px, b.py, b.pz,
                                                     h.gather_r2, h.todo, h.cand, h.candc, h.rcap, h.rho);
  ++*launches;
  uint32_t err = 0;
  cudaMemcpyAsync(&err, ctx.d_err, 4, cudaMemcpyDeviceToHost, st);
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return abi_cuda_fail(&ctx, e, "large neighbourhoods");
  if (err) return abi_device_status(&ctx, err);
  h.big_owners += nb;
  h.big_entries += off[nb];
  return EHGP_OK;
}

// Candidate sets above kMaxCand (owners certified with todo = 4): counted and written, sorted,
// into cand_arena; owners in arena order in large_ids (the n_large sets of at most kLargeCand
// first, then the n_huge sets of at most kHugeCand), prefix offsets in large_off.  lsmall:
// owners certified on their per-point list; lbig: owners certified on the large path (their
// lists are gathered again at the same radius).
int higher_large_candidates(Ctx& ctx, const CertParams& cp, uint32_t root, const std::vector<uint32_t>& lsmall,
                            const std::vector<uint32_t>& lbig, uint64_t* launches) {
  HigherBuffers& h = ctx.hb;
  LbvhBuffers& b = ctx.lb;
  cudaStream_t st = ctx.stream;
  const uint32_t ns = (uint32_t)lsmall.size(), nb = (uint32_t)lbig.size(), nt = ns + nb;
  cudaError_t e = cudaSuccess;
  std::vector<uint64_t> boff;
  if (nb) {
    const int s = gather_big_lists(ctx, root, lbig, boff, launches);
    if (s != EHGP_OK) return s;
  }
  if (h.large_cap < nt) {
    uint64_t c1 = h.large_cap, c2 = h.large_cap, c3 = h.large_cap, c4 = h.large_cap;
    if ((e = grow_array(ctx, h.large_ids, c1, nt, 4)) != cudaSuccess ||
        (e = grow_array(ctx, h.large_off, c2, nt + 1, 8)) != cudaSuccess ||
        (e = grow_array(ctx, h.large_cnt, c3, nt, 4)) != cudaSuccess ||
        (e = grow_array(ctx, h.large_dst, c4, nt, 8)) != cudaSuccess) {
      cudaGetLastError();
      h.large_cap = 0;
      return abi_fail(&ctx, EHGP_ERR_OUT_OF_MEMORY, "the large candidate sets do not fit the device");
    }
    h.large_cap = std::min(std::min(c1, c2 - 1), std::min(c3, c4));
  }
  // launch order: the per-point-list owners, then the large-path owners (as gathered)
  std::vector<uint32_t> launch(lsmall);
  launch.insert(launch.end(), lbig.begin(), lbig.end());
  cudaMemcpyAsync(h.large_ids, launch.data(), (uint64_t)nt * 4, cudaMemcpyHostToDevice, st);
  if (ns)
    k_cand_large<false><<<ns, kCandThreads, 0, st>>>(ns, h.large_ids, h.nb, h.nbc, nullptr, nullptr, cp, b.px, b.py,
                                                     b.pz, h.rho, nullptr, nullptr, h.large_cnt, nullptr);
  if (nb)
    k_cand_large<true><<<nb, kCandThreads, 0, st>>>(nb, h.large_ids + ns, h.nb, h.nbc, h.big_off, h.big_arena, cp,
                                                    b.px, b.py, b.pz, h.rho, nullptr, nullptr, h.large_cnt + ns,
                                                    nullptr);
  *launches += (ns ? 1 : 0) + (nb ? 1 : 0);
  std::vector<uint32_t> cnt(nt);
  cudaMemcpyAsync(cnt.data(), h.large_cnt, (uint64_t)nt * 4, cudaMemcpyDeviceToHost, st);
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return abi_cuda_fail(&ctx, e, "large candidate sets");
  // arena order: sets of at most kLargeCand, then kHugeCand, then kMegaCand
  auto cls = [](uint32_t c) { return c <= (uint32_t)kLargeCand ? 0 : c <= (uint32_t)kHugeCand ? 1 : 2; };
  std::vector<uint32_t> ord;
  for (uint32_t j = 0; j < nt; ++j)
    if (cnt[j] > (uint32_t)kMegaCand) {
      char msg[200];
      snprintf(msg, sizeof msg, "a certified candidate set holds %u points, above the %d this build stages (PointId %u)",
               cnt[j], kMegaCand, launch[j]);
      return abi_fail(&ctx, EHGP_ERR_CAPACITY, msg);
    }
  for (int pass = 0; pass < 3; ++pass)
    for (uint32_t j = 0; j < nt; ++j)
      if (cls(cnt[j]) == pass) ord.push_back(j);
  std::vector<uint64_t> dst(nt), pre(nt + 1, 0);
  std::vector<uint32_t> ids(nt);
  uint32_t per[3] = {0, 0, 0};
  for (uint32_t q = 0; q < nt; ++q) {
    const uint32_t j = ord[q];
    dst[j] = pre[q];
    pre[q + 1] = pre[q] + cnt[j];
    ids[q] = launch[j];
    ++per[cls(cnt[j])];
  }
  if ((e = grow_array(ctx, h.cand_arena, h.carena_cap, pre[nt], 4)) != cudaSuccess ||
      (per[2] && (e = grow_array(ctx, h.cand_dist, h.cdist_cap, pre[nt], 4)) != cudaSuccess)) {
    cudaGetLastError();
    return abi_fail(&ctx, EHGP_ERR_OUT_OF_MEMORY, "the large candidate sets do not fit the device");
  }
  cudaMemcpyAsync(h.large_dst, dst.data(), (uint64_t)nt * 8, cudaMemcpyHostToDevice, st);
  if (ns)
    k_cand_large<false><<<ns, kCandThreads, 0, st>>>(ns, h.large_ids, h.nb, h.nbc, nullptr, nullptr, cp, b.px, b.py,
                                                     b.pz, h.rho, h.large_dst, h.cand_arena, h.large_cnt, h.cand_dist);
  if (nb)
    k_cand_large<true><<<nb, kCandThreads, 0, st>>>(nb, h.large_ids + ns, h.nb, h.nbc, h.big_off, h.big_arena, cp,
                                                    b.px, b.py, b.pz, h.rho, h.large_dst + ns, h.cand_arena,
                                                    h.large_cnt + ns, h.cand_dist);
  *launches += (ns ? 1 : 0) + (nb ? 1 : 0);
  // the enumeration reads owners in arena order; the sets of at most kLargeCand and of at
  // most kHugeCand run split into chunks of their candidate pairs: chunk prefixes of the
  // first tier in split_off[0 .. per[0]], of the second in split_off[per[0] + 1 ..]
  std::vector<uint32_t> chunk_off((uint64_t)per[0] + per[1] + 2, 0);
  for (int tier = 0; tier < 2; ++tier) {
    const uint32_t q0 = tier ? per[0] : 0, cnt_t = per[tier];
    uint32_t* co = chunk_off.data() + (tier ? per[0] + 1 : 0);
    for (uint32_t q = 0; q < cnt_t; ++q) {
      const uint64_t mq = pre[q0 + q + 1] - pre[q0 + q], pairs = mq * (mq > 0 ? mq - 1 : 0) / 2;
      co[q + 1] = co[q] + (uint32_t)std::max<uint64_t>(1, (pairs + kSplitPairs - 1) / kSplitPairs);
    }
  }
  if ((e = grow_array(ctx, h.split_off, h.split_cap, chunk_off.size(), 4)) != cudaSuccess) {
    cudaGetLastError();
    return abi_fail(&ctx, EHGP_ERR_OUT_OF_MEMORY, "the large candidate sets do not fit the device");
  }
  cudaMemcpyAsync(h.split_off, chunk_off.data(), chunk_off.size() * 4, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(h.large_ids, ids.data(), (uint64_t)nt * 4, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(h.large_off, pre.data(), (uint64_t)(nt + 1) * 8, cudaMemcpyHostToDevice, st);
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return abi_cuda_fail(&ctx, e, "large candidate sets");
  h.n_large = per[0];
  h.split_chunks = chunk_off[per[0]];
  h.split_chunks_huge = chunk_off[(uint64_t)per[0] + 1 + per[1]];
  h.n_huge = per[1];
  h.n_mega = per[2];
  h.large_entries = pre[nt];
  return EHGP_OK;
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
  ++ctx.higher_runs;
  if (smax < 3 || n < 3) {
    h.K = K;
    return EHGP_OK;
  }
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
  if (cp.need < 1 || cp.need > (uint32_t)kMaxNeed) return abi_fail(&ctx, EHGP_ERR_INVALID_ARGUMENT, "K above 10 is not supported");
  uint32_t pending = n, overflowed = 0;
  std::vector<uint8_t> todo(n);
  std::vector<uint32_t> big;
  std::vector<uint64_t> big_off;
  std::vector<uint8_t> was_big(n, 0);
  h.big_owners = h.big_entries = 0;
  h.n_large = h.n_huge = h.n_mega = 0;
  h.large_entries = 0;
  // todo: 0 certified, 1 pending on the list path, 2 candidate set too large, 3 pending on
  // the large-neighbourhood path
  for (int round = 0; round < 8 && pending > 0; ++round) {
    k_gather<<<nblocks(n, kWarps), kThreads, 0, st>>>(n, root, g.tnodes, b.leaf_pid, b.n_begin, b.n_end, b.px, b.py,
                                                      b.pz, h.gather_r2, h.todo, h.nb, h.nbc);
    const uint32_t list_cap = h.list_cap < (uint32_t)kMaxNb ? h.list_cap : (uint32_t)kMaxNb;
    k_dirtable<<<n, kDirThreads, 0, st>>>(n, list_cap, cp, b.leaf_pid, h.nb, h.nbc, b.px, b.py, b.pz, h.gather_r2, h.todo,
                                          h.cand, h.candc, h.rcap, h.rho);
    launches += 2;
    cudaMemcpyAsync(todo.data(), h.todo, n, cudaMemcpyDeviceToHost, st);
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return abi_cuda_fail(&ctx, e, "higher-support certificate");
    big.clear();
    for (uint32_t i = 0; i < n; ++i)
      if (todo[i] == 3) {
        big.push_back(i);
        was_big[i] = 1;
      }
    if (!big.empty()) {
      const int s = higher_big_round(ctx, cp, root, big, big_off, &launches);
      if (s != EHGP_OK) return s;
      cudaMemcpyAsync(todo.data(), h.todo, n, cudaMemcpyDeviceToHost, st);
      if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return abi_cuda_fail(&ctx, e, "higher-support certificate");
    }
    pending = overflowed = 0;
    for (uint32_t i = 0; i < n; ++i) {
      pending += todo[i] == 1 || todo[i] == 3;
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
  {  // candidate sets above kMaxCand
    std::vector<uint32_t> lsmall, lbig;
    for (uint32_t i = 0; i < n; ++i)
      if (todo[i] == 4) (was_big[i] ? lbig : lsmall).push_back(i);
    if (!lsmall.empty() || !lbig.empty()) {
      const int s = higher_large_candidates(ctx, cp, root, lsmall, lbig, &launches);
      if (s != EHGP_OK) return s;
    }
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx.device);
  if (h.n_mega) {  // per-block scratch of the mega-set kernel (staged set and face mask)
    const uint64_t bm = std::min<uint64_t>(h.n_mega, (uint64_t)sms);
    const uint64_t need = bm * large_scratch_bytes<kMegaCand, 2>();
    if (grow_array(ctx, h.adm_scratch, h.adm_words, (need + 3) / 4, 4) != cudaSuccess) {
      cudaGetLastError();
      return abi_fail(&ctx, EHGP_ERR_OUT_OF_MEMORY, "the scratch of the huge candidate sets does not fit the device");
    }
  }
  if ((h.n_large || h.n_huge) &&
      (grow_array(ctx, h.split_adm, h.split_adm_words,
                       std::max((uint64_t)h.n_large * kLargeCand * (kLargeCand / 32),
                                (uint64_t)h.n_huge * kHugeCand * (kHugeCand / 32)),
                       4)) != cudaSuccess) {
    cudaGetLastError();
    return abi_fail(&ctx, EHGP_ERR_OUT_OF_MEMORY, "the face masks of the large candidate sets do not fit the device");
  }
  if (h.n_large || h.n_huge || h.n_mega) {
    cudaError_t ea = cudaFuncSetAttribute(k_higher_split<kLargeCand>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)split_smem<kLargeCand>());
    if (ea == cudaSuccess)
      ea = cudaFuncSetAttribute(k_higher_split<kHugeCand>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)split_smem<kHugeCand>());
    if (ea == cudaSuccess)
      ea = cudaFuncSetAttribute(k_higher_large<kMegaCand, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)large_smem<kMegaCand, 2>());
    if (ea != cudaSuccess) return abi_cuda_fail(&ctx, ea, "large candidate sets shared memory");
  }
  uint32_t hc[2];
  cudaError_t e = cudaSuccess;
  const HigherTables tb{h.dirs, h.cells, h.rho, h.cos_lim};
  // count -> allocate -> emit: the enumeration counts every record and writes those that fit;
  // when the count exceeds the buffer, the buffer grows to it and the enumeration runs again
  for (int attempt = 0; attempt < 2; ++attempt) {
    cudaMemsetAsync(h.counters, 0, 8 * sizeof(uint32_t), st);
    cudaMemsetAsync(h.stats, 0, 8 * sizeof(unsigned long long), st);
    const Ctl ctl{smax, h.capacity};
    cudaEventRecord(ctx.evk0, st);
    k_higher<<<n, 32 * kHOwnerWarps, 0, st>>>(n, ctl, tb, b.leaf_pid, h.cand, h.candc, b.px, b.py, b.pz, g.scale,
                                              (HigherRec*)h.raw, h.counters, h.stats);
    ++launches;
    if (h.n_large) {  // split over chunks of pairs: the triangles (face masks), then the tetrahedra
      cudaMemsetAsync(h.split_adm, 0, (uint64_t)h.n_large * kLargeCand * (kLargeCand / 32) * 4, st);
      for (const uint32_t phase : {kPhTri, kPhTet}) {
        k_higher_split<kLargeCand><<<h.split_chunks, 32 * kHOwnerWarps, split_smem<kLargeCand>(), st>>>(
            h.n_large, h.large_ids, h.large_off, h.cand_arena, h.split_off, phase, ctl, tb, b.px, b.py, b.pz, g.scale,
            (HigherRec*)h.raw, h.counters, h.stats, h.split_adm);
        ++launches;
      }
    }
    if (h.n_huge) {
      const uint32_t o = h.n_large;
      cudaMemsetAsync(h.split_adm, 0, (uint64_t)h.n_huge * kHugeCand * (kHugeCand / 32) * 4, st);
      for (const uint32_t phase : {kPhTri, kPhTet}) {
        k_higher_split<kHugeCand><<<h.split_chunks_huge, 32 * kHOwnerWarps, split_smem<kHugeCand>(), st>>>(
            h.n_huge, h.large_ids + o, h.large_off + o, h.cand_arena, h.split_off + o + 1, phase, ctl, tb, b.px, b.py,
            b.pz, g.scale, (HigherRec*)h.raw, h.counters, h.stats, h.split_adm);
        ++launches;
      }
    }
    if (h.n_mega) {
      const uint32_t o = h.n_large + h.n_huge;
      k_higher_large<kMegaCand, 2><<<std::min<uint32_t>(h.n_mega, (uint32_t)sms), 32 * kHOwnerWarps,
                                     large_smem<kMegaCand, 2>(), st>>>(
          h.n_mega, h.large_ids + o, h.large_off + o, h.cand_arena, ctl, tb, b.px, b.py, b.pz, g.scale,
          (HigherRec*)h.raw, h.counters, h.stats, (unsigned char*)h.adm_scratch);
      ++launches;
    }
    cudaEventRecord(ctx.evk1, st);
    unsigned long long hs[8];
    cudaMemcpyAsync(hc, h.counters, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(hc + 1, ctx.d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(hs, h.stats, sizeof(hs), cudaMemcpyDeviceToHost, st);
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return abi_cuda_fail(&ctx, e, "higher-support enumeration");
    if (hc[1]) return abi_device_status(&ctx, hc[1]);
    {
      float kms = 0;
      cudaEventElapsedTime(&kms, ctx.evk0, ctx.evk1);
      h.kernel_ms = kms;
      for (int i = 0; i < 8; ++i) h.stats_host[i] = hs[i];
    }
    if (hc[0] <= h.capacity) break;
    if (attempt == 1 || (uint64_t)hc[0] >= 0xffff0000ull)
      return abi_fail(&ctx, EHGP_ERR_CAPACITY, "higher-support records exceed 32-bit record indices");
    if ((e = higher_records_alloc(ctx, grown_capacity(hc[0]))) != cudaSuccess) {
      cudaGetLastError();
      return abi_fail(&ctx, EHGP_ERR_OUT_OF_MEMORY, "the higher-support records do not fit the device");
    }
    ++ctx.regrowths;
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

int ehgp_predicate_eval(ehgp_ctx* ctx, uint32_t predicate, const uint32_t* ids, uint32_t count, int32_t* out) {
  if (!ctx || !ids || !out || predicate < 1 || predicate > 4 || count == 0 || count > 16)
    return EHGP_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(ctx->mutex);
  ctx->last_error.clear();
  if (ctx->poisoned) return ehgp::abi_fail(ctx, EHGP_ERR_POISONED, "the context is poisoned by an earlier CUDA failure");
  if (ctx->built_n == 0) return ehgp::abi_fail(ctx, EHGP_ERR_NOT_BUILT, "ehgp_predicate_eval needs a resident cloud");
  for (uint32_t i = 0; i < count; ++i)
    if (ids[i] >= ctx->built_n && !(predicate == 3 && i == 0)) return EHGP_ERR_INVALID_ARGUMENT;
  const uint32_t need = predicate == 1 ? 2 : predicate == 2 ? 1 : predicate == 3 ? 3 : 3;
  if (count < need || (predicate == 1 && count > 5) || (predicate == 2 && count > 4) || (predicate == 4 && count != 3) ||
      (predicate == 3 && (ids[0] < 1 || ids[0] > 4 || count - 1 - ids[0] < 1 || count - 1 - ids[0] > 4)))
    return EHGP_ERR_INVALID_ARGUMENT;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return ehgp::abi_cuda_fail(ctx, e, "cudaSetDevice");
  if (!ctx->geom_ready) {
    ehgp::geom_prepare(*ctx, (uint32_t)ctx->built_n);
    if ((e = cudaGetLastError()) != cudaSuccess) return ehgp::abi_cuda_fail(ctx, e, "traversal preparation");
  }
  if (!ctx->scale_valid)
    return ehgp::abi_fail(ctx, EHGP_ERR_NUMERIC_RANGE, "the cloud exceeds the exact fixed-point range");
  cudaStream_t st = ctx->stream;
  cudaMemcpyToSymbolAsync(ehgp::g_pred_ids, ids, count * sizeof(uint32_t), 0, cudaMemcpyHostToDevice, st);
  ehgp::k_predicate<<<1, 1, 0, st>>>(predicate, count, ctx->lb.px, ctx->lb.py, ctx->lb.pz, ctx->gb.scale);
  cudaMemcpyFromSymbolAsync(out, ehgp::g_pred_out, 2 * sizeof(int32_t), 0, cudaMemcpyDeviceToHost, st);
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return ehgp::abi_cuda_fail(ctx, e, "predicate evaluation");
  return EHGP_OK;
}

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
  const ehgp::HigherBuffers& h = ctx->hb;
  const uint64_t more[6] = {h.big_owners, h.big_entries, h.n_large, h.n_huge, h.n_mega, h.large_entries};
  for (uint32_t i = 8; stats && i < count && i < 14; ++i) stats[i] = more[i - 8];
  return EHGP_OK;
}

}  // extern "C"
