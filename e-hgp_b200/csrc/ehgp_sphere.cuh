// Exact sphere predicates shared by the support and hierarchy stages.
//
// Every coordinate is an integer X = x 2^S at the cloud scale (|X| < 2^124), so
// the circumsphere data of a 1- to 4-point support are integers:
//   point a:                 A = 1, N = 0
//   pair a, a+e:             A = 1, N = e
//   triangle a, a+e1, a+e2:  A = det G,  N = G22 (G11 - G12) e1 + G11 (G22 - G12) e2
//   tetrahedron a, a+e1..e3: A = det E,  N = |e1|^2 e2 x e3 + |e2|^2 e3 x e1 + |e3|^2 e1 x e2
// with centre a + N / (2A) and squared radius |N|^2 / (4 A^2).  832-bit words hold
// every side polynomial A |p|^2 - p.N and distance comparison from one centre;
// level comparisons |N1|^2 A2^2 vs |N2|^2 A1^2 need 2304 bits.  These are the
// slow paths behind FP64 filters and are kept out of line.  Host and device
// share them (the host settles rare exact level ties).
#pragma once

#include <string.h>

#include "ehgp_exact.cuh"

namespace ehgp {
namespace {

__host__ __device__ inline uint64_t dbits(double v) {
  uint64_t b;
  memcpy(&b, &v, sizeof b);
  return b;
}

using W = WInt<13>;
using WL = WInt<36>;
struct WV {
  W x, y, z;
};
__host__ __device__ inline W wdot(const WV& a, const WV& b) {
  return wadd(wadd(wmul(a.x, b.x), wmul(a.y, b.y)), wmul(a.z, b.z));
}
__host__ __device__ inline WV wcross(const WV& a, const WV& b) {
  return {wsub(wmul(a.y, b.z), wmul(a.z, b.y)), wsub(wmul(a.z, b.x), wmul(a.x, b.z)),
          wsub(wmul(a.x, b.y), wmul(a.y, b.x))};
}
__host__ __device__ inline WV wscale(const W& s, const WV& a) { return {wmul(s, a.x), wmul(s, a.y), wmul(s, a.z)}; }
__host__ __device__ inline WV wvadd(const WV& a, const WV& b) { return {wadd(a.x, b.x), wadd(a.y, b.y), wadd(a.z, b.z)}; }

template <int M, int N>
__host__ __device__ inline WInt<M> widen(const WInt<N>& a) {
  WInt<M> r;
  const uint64_t ext = a.negative() ? ~uint64_t{0} : 0;
  for (int i = 0; i < M; ++i) r.w[i] = i < N ? a.w[i] : ext;
  return r;
}

struct Cloud {
  const double* px;
  const double* py;
  const double* pz;
  int S;
  __host__ __device__ WV wdiff(uint32_t i, uint32_t j) const {
    return {W::from_i128(fixed_of(dbits(px[i]), S) - fixed_of(dbits(px[j]), S)),
            W::from_i128(fixed_of(dbits(py[i]), S) - fixed_of(dbits(py[j]), S)),
            W::from_i128(fixed_of(dbits(pz[i]), S) - fixed_of(dbits(pz[j]), S))};
  }
};

// Exact signs of a triangle: G12, G11 - G12, G22 - G12, det G.
__host__ __device__ __noinline__ void tri_signs_exact(const Cloud& c, const uint32_t* id, int* sg) {
  const WV w1 = c.wdiff(id[1], id[0]), w2 = c.wdiff(id[2], id[0]);
  const W g11 = wdot(w1, w1), g12 = wdot(w1, w2), g22 = wdot(w2, w2);
  sg[0] = g12.sign();
  sg[1] = wsub(g11, g12).sign();
  sg[2] = wsub(g22, g12).sign();
  sg[3] = wsub(wmul(g11, g22), wmul(g12, g12)).sign();
}

// Exact signs of a tetrahedron: det E, then the barycentric numerators l0..l3 of its circumcentre.
__host__ __device__ __noinline__ void quad_signs_exact(const Cloud& c, const uint32_t* id, int* sg) {
  const WV w1 = c.wdiff(id[1], id[0]), w2 = c.wdiff(id[2], id[0]), w3 = c.wdiff(id[3], id[0]);
  const WV x23 = wcross(w2, w3), x31 = wcross(w3, w1), x12 = wcross(w1, w2);
  const WV nn = wvadd(wvadd(wscale(wdot(w1, w1), x23), wscale(wdot(w2, w2), x31)), wscale(wdot(w3, w3), x12));
  const W de = wdot(w1, x23);
  const W m1 = wdot(nn, x23), m2 = wdot(nn, x31), m3 = wdot(nn, x12);
  const W two = W::from_i128(2);
  const W m0 = wsub(wmul(two, wmul(de, de)), wadd(wadd(m1, m2), m3));
  sg[0] = de.sign();
  sg[1] = m0.sign();
  sg[2] = m1.sign();
  sg[3] = m2.sign();
  sg[4] = m3.sign();
}

// Integer circumsphere data (A, N) of a 1- to 4-point support, relative to ids[0].
__host__ __device__ __noinline__ void exact_sphere(const Cloud& c, const uint32_t* ids, int size, W& A, WV& N) {
  if (size <= 2) {
    A = W::from_i128(1);
    N = size == 2 ? c.wdiff(ids[1], ids[0]) : WV{W::zero(), W::zero(), W::zero()};
  } else if (size == 3) {
    const WV w1 = c.wdiff(ids[1], ids[0]), w2 = c.wdiff(ids[2], ids[0]);
    const W g11 = wdot(w1, w1), g12 = wdot(w1, w2), g22 = wdot(w2, w2);
    A = wsub(wmul(g11, g22), wmul(g12, g12));
    N = wvadd(wscale(wmul(g22, wsub(g11, g12)), w1), wscale(wmul(g11, wsub(g22, g12)), w2));
  } else {
    const WV w1 = c.wdiff(ids[1], ids[0]), w2 = c.wdiff(ids[2], ids[0]), w3 = c.wdiff(ids[3], ids[0]);
    const WV x23 = wcross(w2, w3), x31 = wcross(w3, w1), x12 = wcross(w1, w2);
    A = wdot(w1, x23);
    N = wvadd(wvadd(wscale(wdot(w1, w1), x23), wscale(wdot(w2, w2), x31)), wscale(wdot(w3, w3), x12));
  }
}

// Exact sign of the side polynomial A |w - a|^2 - (w - a).N (before the orientation sign).
__host__ __device__ __noinline__ int side_exact(const Cloud& c, const uint32_t* ids, int size, uint32_t w) {
  W A;
  WV N;
  exact_sphere(c, ids, size, A, N);
  const WV q = c.wdiff(w, ids[0]);
  return wsub(wmul(A, wdot(q, q)), wdot(q, N)).sign();
}

// Exact sign of |p - centre|^2 - |q - centre|^2 for the circumcentre of a 1- to 4-point support.
__host__ __device__ __noinline__ int dist_cmp_exact(const Cloud& c, const uint32_t* ids, int size, uint32_t p,
                                                    uint32_t q) {
  W A;
  WV N;
  exact_sphere(c, ids, size, A, N);
  const WV dp = c.wdiff(p, ids[0]), dq = c.wdiff(q, ids[0]);
  const WV pq = c.wdiff(p, q);
  // 2A (|p-c|^2 - |q-c|^2) = 2A (|p-a|^2 - |q-a|^2) - 2 (p-q).N; sign divided by sign(A)
  const W v = wsub(wmul(A, wsub(wdot(dp, dp), wdot(dq, dq))), wdot(pq, N));
  return v.sign() * A.sign();
}

// Exact sign of level(support 1) - level(support 2), levels |N|^2 / (4 A^2).
__host__ __device__ __noinline__ int level_cmp_exact(const Cloud& c, const uint32_t* ids1, int s1, const uint32_t* ids2,
                                                     int s2) {
  W A1, A2;
  WV N1, N2;
  exact_sphere(c, ids1, s1, A1, N1);
  exact_sphere(c, ids2, s2, A2, N2);
  auto sq = [](const WV& v) {  // |v|^2 in 2304 bits (|N| < 2^632)
    const WL x = widen<36>(v.x), y = widen<36>(v.y), z = widen<36>(v.z);
    return wadd(wadd(wmul(x, x), wmul(y, y)), wmul(z, z));
  };
  const WL n1 = sq(N1), n2 = sq(N2);
  const WL a1 = widen<36>(A1), a2 = widen<36>(A2);
  return wcmp(wmul(n1, wmul(a2, a2)), wmul(n2, wmul(a1, a1)));
}

}  // namespace
}  // namespace ehgp
