// ORACLE — test infrastructure only, never the product path.
//
// A CPU restatement, in plain C++, of the reference's algorithm for each stage
// of the MorseHGP3D product path (Ludwig-H/E-HGP, morsehgp3d/), written for
// clarity over speed.  Only tests/, the smoke check and bench.py's CPU
// baseline may load it, and only as the checker.  Exact arithmetic uses the
// arbitrary-precision integer of oracle/boost_shim.
//
// Pinning: tests check this restatement against the reference's own code
// compiled here (oracle/_ref, built by oracle/Makefile) and against the
// committed golden vectors in tests/golden/.
#include <boost/multiprecision/cpp_int.hpp>

#include <algorithm>
#include <cmath>
#include <array>
#include <cstdint>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace {

using Big = boost::multiprecision::cpp_int;
using u64 = std::uint64_t;

// exact::canonicalize_binary64_bits / binary64_total_order_key
// (include/morsehgp3d/exact/binary64.hpp:17-29)
u64 canonical(u64 bits) {
  if ((bits & 0x7ff0000000000000ull) == 0x7ff0000000000000ull)
    throw std::invalid_argument("binary64 coordinates must be finite");
  return bits == 0x8000000000000000ull ? 0ull : bits;
}
u64 order_key(u64 bits) { return (bits >> 63) ? ~bits : (bits ^ (u64{1} << 63)); }

u64 bits_of(double v) {
  u64 b;
  std::memcpy(&b, &v, 8);
  return b;
}

struct Cloud {
  std::vector<std::array<u64, 3>> bits;  // canonical words by PointId
  std::vector<u64> source;               // input index by PointId
};

// CanonicalPointCloud::rejecting_duplicates (src/cpu/spatial/point_cloud.cpp:40-94):
// PointId = rank in lexicographic order of the three total-order keys.
Cloud canonical_cloud(const double* xyz, u64 n) {
  if (n == 0) throw std::invalid_argument("a canonical point cloud cannot be empty");
  std::vector<std::array<u64, 3>> keys(n);
  std::vector<std::array<u64, 3>> words(n);
  for (u64 i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) {
      words[i][a] = canonical(bits_of(xyz[3 * i + a]));
      keys[i][a] = order_key(words[i][a]);
    }
  std::vector<u64> order(n);
  for (u64 i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](u64 l, u64 r) { return keys[l] < keys[r]; });
  for (u64 i = 1; i < n; ++i)
    if (keys[order[i - 1]] == keys[order[i]])
      throw std::invalid_argument("a canonical point cloud cannot contain duplicate geometric points");
  Cloud c;
  c.bits.resize(n);
  c.source = order;
  for (u64 p = 0; p < n; ++p) c.bits[p] = words[order[p]];
  return c;
}

// A finite binary64 value as significand * 2^exponent (lbvh.cpp:162-186).
struct Dyadic {
  long long sig;
  int exp;
};
Dyadic decode(u64 bits) {
  const u64 e = (bits >> 52) & 0x7ff, f = bits & ((u64{1} << 52) - 1);
  Dyadic d{(long long)f, -1074};
  if (e != 0) {
    d.sig = (long long)(f | (u64{1} << 52));
    d.exp = (int)e - 1075;
  }
  if (bits >> 63) d.sig = -d.sig;
  return d;
}

// quantized_coordinate_from_bits (src/cpu/spatial/lbvh.cpp:237-296): the
// exact floor(2^21 (x - l) / (u - l)) with the two boundary rules.
u64 quantize(u64 x, u64 l, u64 u) {
  if (l == u) return 0;
  if (x == u) return (u64{1} << 21) - 1;
  const Dyadic dx = decode(x), dl = decode(l), du = decode(u);
  int emin = 0;
  bool have = false;
  for (const Dyadic& d : {dl, dx, du})
    if (d.sig != 0) {
      emin = have ? std::min(emin, d.exp) : d.exp;
      have = true;
    }
  auto aligned = [&](const Dyadic& d) {
    Big v = d.sig;
    if (d.sig != 0) v <<= (unsigned)(d.exp - emin);
    return v;
  };
  const Big L = aligned(dl), X = aligned(dx), U = aligned(du);
  const Big q = (Big(u64{1} << 21) * (X - L)) / (U - L);
  return q.convert_to<u64>();
}

// interleaved_morton_code (src/cpu/spatial/lbvh.cpp:78-91)
u64 interleave(u64 qx, u64 qy, u64 qz) {
  u64 code = 0;
  for (int b = 0; b < 21; ++b) {
    code |= ((qx >> b) & 1) << (3 * b + 2);
    code |= ((qy >> b) & 1) << (3 * b + 1);
    code |= ((qz >> b) & 1) << (3 * b);
  }
  return code;
}

struct Node {
  u64 lo[3], hi[3], left, right, begin, end;
};

struct Lbvh {
  std::vector<std::pair<u64, u64>> leaves;  // (code, PointId)
  std::vector<Node> nodes;                   // postorder
  u64 max_depth = 0, collision_groups = 0, max_collision = 0;
  std::array<u64, 6> root_aabb{};
};

// MortonLbvhIndex::build (src/cpu/spatial/lbvh.cpp:484-549) with find_split
// (:831-860), build_range (:862-906) and the witness rules (:46-76).
Lbvh build_lbvh(const Cloud& c) {
  const u64 n = c.bits.size();
  auto key = [&](u64 id, int a) { return order_key(c.bits[id][a]); };
  Lbvh t;
  // exact frame: first extremum in PointId order wins (lbvh.cpp:107-155)
  std::array<u64, 3> lo_id{}, hi_id{};
  for (u64 p = 1; p < n; ++p)
    for (int a = 0; a < 3; ++a) {
      if (key(p, a) < key(lo_id[a], a)) lo_id[a] = p;
      if (key(p, a) > key(hi_id[a], a)) hi_id[a] = p;
    }
  for (int a = 0; a < 3; ++a) {
    t.root_aabb[a] = c.bits[lo_id[a]][a];
    t.root_aabb[3 + a] = c.bits[hi_id[a]][a];
  }
  t.leaves.resize(n);
  for (u64 p = 0; p < n; ++p) {
    u64 q[3];
    for (int a = 0; a < 3; ++a) q[a] = quantize(c.bits[p][a], t.root_aabb[a], t.root_aabb[3 + a]);
    t.leaves[p] = {interleave(q[0], q[1], q[2]), p};
  }
  std::sort(t.leaves.begin(), t.leaves.end());
  for (u64 b = 0; b < n;) {
    u64 e = b + 1;
    while (e < n && t.leaves[e].first == t.leaves[b].first) ++e;
    if (e - b > 1) {
      ++t.collision_groups;
      t.max_collision = std::max(t.max_collision, e - b);
    }
    b = e;
  }
  auto split = [&](u64 b, u64 e) -> u64 {
    const u64 f = t.leaves[b].first, l = t.leaves[e - 1].first;
    if (f == l) return b + (e - b) / 2;
    const int hb = 63 - __builtin_clzll(f ^ l);
    u64 lo = b + 1, hi = e;
    while (lo < hi) {
      const u64 mid = lo + (hi - lo) / 2;
      if (((t.leaves[mid].first >> hb) & 1) == 0) lo = mid + 1;
      else hi = mid;
    }
    return lo;
  };
  std::function<u64(u64, u64, u64)> rec = [&](u64 b, u64 e, u64 depth) -> u64 {
    t.max_depth = std::max(t.max_depth, depth);
    Node nd{};
    nd.begin = b;
    nd.end = e;
    if (e - b == 1) {
      for (int a = 0; a < 3; ++a) nd.lo[a] = nd.hi[a] = t.leaves[b].second;
      nd.left = nd.right = ~u64{0};
    } else {
      const u64 s = split(b, e);
      nd.left = rec(b, s, depth + 1);
      nd.right = rec(s, e, depth + 1);
      const Node& L = t.nodes[nd.left];
      const Node& R = t.nodes[nd.right];
      for (int a = 0; a < 3; ++a) {
        const u64 kl = key(L.lo[a], a), kr = key(R.lo[a], a);
        nd.lo[a] = (kr < kl || (kr == kl && R.lo[a] < L.lo[a])) ? R.lo[a] : L.lo[a];
        const u64 hl = key(L.hi[a], a), hr = key(R.hi[a], a);
        nd.hi[a] = (hr > hl || (hr == hl && R.hi[a] < L.hi[a])) ? R.hi[a] : L.hi[a];
      }
    }
    t.nodes.push_back(nd);
    return t.nodes.size() - 1;
  };
  rec(0, n, 0);
  return t;
}

// ---- exact geometry at one dyadic scale ------------------------------------------
// Every canonical coordinate as an integer numerator over 2^S (S = the largest
// fractional bit count); squared distances are then integers over 2^(2S).
struct FixedCloud {
  std::vector<std::array<Big, 3>> X;
  int S = 0;
};

FixedCloud fixed_cloud(const Cloud& c) {
  FixedCloud f;
  int S = 0;
  for (const auto& p : c.bits)
    for (int a = 0; a < 3; ++a) {
      const Dyadic d = decode(p[a]);
      if (d.sig == 0) continue;
      const long long m = d.sig < 0 ? -d.sig : d.sig;
      S = std::max(S, -(d.exp + __builtin_ctzll((u64)m)));
    }
  f.S = S;
  f.X.resize(c.bits.size());
  for (size_t i = 0; i < c.bits.size(); ++i)
    for (int a = 0; a < 3; ++a) {
      const Dyadic d = decode(c.bits[i][a]);
      Big v = d.sig;
      const int sh = d.exp + S;
      if (d.sig != 0) {
        if (sh >= 0) v <<= (unsigned)sh;
        else v /= (Big(1) << (unsigned)(-sh));  // exact: S bounds the fractional bits
      }
      f.X[i][a] = v;
    }
  return f;
}

Big dist2(const FixedCloud& f, u64 a, u64 b) {
  Big s = 0;
  for (int k = 0; k < 3; ++k) {
    const Big d = f.X[a][k] - f.X[b][k];
    s += d * d;
  }
  return s;
}

// reduced "num den" of N / 2^e
std::string reduced(Big N, int e) {
  while (e > 0 && N != 0 && (N % 2) == 0) {
    N /= 2;
    --e;
  }
  if (N == 0) e = 0;
  return N.str() + " " + (Big(1) << (unsigned)e).str();
}

// Brute-force exact top-k with exclusions {p}: the partition of
// TopKPartition::from_evaluated_neighbors (src/cpu/spatial/brute_force.cpp:319-384).
std::string knn_text(const Cloud& c, u64 k) {
  const FixedCloud f = fixed_cloud(c);
  const u64 n = c.bits.size();
  std::string s;
  std::vector<std::pair<Big, u64>> nb;
  for (u64 p = 0; p < n; ++p) {
    nb.clear();
    for (u64 q = 0; q < n; ++q)
      if (q != p) nb.emplace_back(dist2(f, p, q), q);
    std::sort(nb.begin(), nb.end());
    const Big cut = nb[k - 1].first;
    std::string strict, shell;
    for (const auto& [d, q] : nb) {
      if (d < cut) strict += std::to_string(q) + " ";
      else if (d == cut) shell += " " + std::to_string(q);
      else break;
    }
    s += strict + "|" + shell + " | " + reduced(cut, 2 * f.S) + "\n";
  }
  return s;
}

struct Edge {
  Big D;
  u64 u, v;
  bool operator<(const Edge& o) const {
    if (D != o.D) return D < o.D;
    if (u != o.u) return u < o.u;
    return v < o.v;
  }
};

struct MinDsu {  // union by least index (src/cpu/hierarchy/k1_forest.cpp:19-62)
  std::vector<u64> p;
  u64 count;
  explicit MinDsu(u64 n) : p(n), count(n) {
    for (u64 i = 0; i < n; ++i) p[i] = i;
  }
  u64 find(u64 x) {
    while (p[x] != x) x = p[x] = p[p[x]];
    return x;
  }
  bool unite(u64 a, u64 b) {
    a = find(a);
    b = find(b);
    if (a == b) return false;
    if (a > b) std::swap(a, b);
    p[b] = a;
    --count;
    return true;
  }
};

// Exact EMST + Boruvka rounds + compact k=1 forest, text format of
// ref_emst_forest (oracle/ref_driver.cpp).
//  * Boruvka rounds with labels frozen to least PointIds and kappa minima
//    (include/morsehgp3d/hierarchy/boruvka.hpp:1-140), O(n^2) per round;
//  * the compact forest of build_compact_k1_forest
//    (src/cpu/hierarchy/k1_forest.cpp:665-845): equal-length batches frozen
//    pre-batch, one merge node per connected group of >= 2 pre-batch
//    components, ordered by the group's least PointId, children ordered by
//    their least PointId, node ids n, n+1, ...
std::string emst_forest_text(const Cloud& c) {
  const FixedCloud f = fixed_cloud(c);
  const u64 n = c.bits.size();
  const int e2 = 2 * f.S;
  std::string s, minima_s;
  std::vector<u64> label(n);
  for (u64 i = 0; i < n; ++i) label[i] = i;
  std::vector<Edge> tree;
  u64 components = n, round = 0;
  while (components > 1) {
    std::vector<bool> has(n, false);
    std::vector<Edge> best(n);
    std::vector<u64> src(n);
    for (u64 p = 0; p < n; ++p)
      for (u64 q = 0; q < n; ++q) {
        if (label[q] == label[p]) continue;
        Edge e{dist2(f, p, q), std::min(p, q), std::max(p, q)};
        const u64 cp = label[p];
        if (!has[cp] || e < best[cp]) {
          has[cp] = true;
          best[cp] = e;
          src[cp] = p;
        }
      }
    std::vector<Edge> accepted;
    for (u64 cpn = 0; cpn < n; ++cpn)
      if (has[cpn]) {
        const Edge& e = best[cpn];
        minima_s += "M " + std::to_string(round) + " " + std::to_string(cpn) + " " + std::to_string(src[cpn]) + " " +
                    std::to_string(e.u) + " " + std::to_string(e.v) + " " + reduced(e.D, e2) + "\n";
        accepted.push_back(e);
      }
    std::sort(accepted.begin(), accepted.end());
    accepted.erase(std::unique(accepted.begin(), accepted.end(),
                               [](const Edge& a, const Edge& b) { return a.u == b.u && a.v == b.v; }),
                   accepted.end());
    MinDsu d(n);
    for (u64 p = 0; p < n; ++p) d.unite(p, label[p]);
    for (const Edge& e : accepted) {
      minima_s += "A " + std::to_string(round) + " " + std::to_string(e.u) + " " + std::to_string(e.v) + "\n";
      d.unite(e.u, e.v);
      tree.push_back(e);
    }
    for (u64 p = 0; p < n; ++p) label[p] = d.find(p);
    components = d.count;
    ++round;
  }
  std::sort(tree.begin(), tree.end());
  for (const Edge& e : tree)
    s += "E " + std::to_string(e.u) + " " + std::to_string(e.v) + " " + reduced(e.D, e2) + "\n";
  s += minima_s;
  // compact k=1 forest
  MinDsu comp(n);
  std::vector<u64> node_of(n), min_pt, cover;  // per root: current node id
  for (u64 i = 0; i < n; ++i) node_of[i] = i;
  std::string levels_s, nodes_s, child_s = "C", batches_s;
  u64 merge_count = 0, child_count_total = 0;
  auto coverage = [&](u64 id) { return id < n ? u64{1} : cover[id - n]; };
  for (size_t b = 0, level = 0; b < tree.size(); ++level) {
    size_t e = b + 1;
    while (e < tree.size() && tree[e].D == tree[b].D) ++e;
    levels_s += "L " + reduced(tree[b].D, e2 + 2) + "\n";
    const u64 pre = comp.count, node_off = merge_count;
    std::vector<u64> roots;
    for (size_t i = b; i < e; ++i) {
      roots.push_back(comp.find(tree[i].u));
      roots.push_back(comp.find(tree[i].v));
    }
    std::sort(roots.begin(), roots.end());
    roots.erase(std::unique(roots.begin(), roots.end()), roots.end());
    MinDsu local(roots.size());
    auto pos = [&](u64 r) { return (u64)(std::lower_bound(roots.begin(), roots.end(), r) - roots.begin()); };
    for (size_t i = b; i < e; ++i) local.unite(pos(comp.find(tree[i].u)), pos(comp.find(tree[i].v)));
    std::vector<std::vector<u64>> groups(roots.size());
    for (u64 li = 0; li < roots.size(); ++li) groups[local.find(li)].push_back(roots[li]);
    std::vector<std::pair<std::vector<u64>, u64>> pending;
    for (auto& g : groups) {
      if (g.empty()) continue;
      const u64 id = n + merge_count++;
      u64 cov = 0;
      for (u64 r : g) {
        child_s += " " + std::to_string(node_of[r]);
        cov += coverage(node_of[r]);
      }
      nodes_s += "N " + std::to_string(id) + " " + std::to_string(level) + " " + std::to_string(child_count_total) +
                 " " + std::to_string(g.size()) + " " + std::to_string(g.front()) + " " + std::to_string(cov) + "\n";
      child_count_total += g.size();
      cover.push_back(cov);
      pending.emplace_back(g, id);
    }
    for (size_t i = b; i < e; ++i) comp.unite(tree[i].u, tree[i].v);
    for (auto& [g, id] : pending) node_of[comp.find(g.front())] = id;
    batches_s += "B " + std::to_string(level) + " " + std::to_string(b) + " " + std::to_string(e - b) + " " +
                 std::to_string(node_off) + " " + std::to_string(merge_count - node_off) + " " + std::to_string(pre) +
                 " " + std::to_string(comp.count) + "\n";
    b = e;
  }
  s += levels_s + nodes_s + child_s + "\n" + batches_s + "R " + std::to_string(node_of[comp.find(0)]) + "\n";
  return s;
}

// Sign of (w - u).(w - v): w inside (<0), on (0) or outside (>0) the closed
// diametral ball of u, v.  FP64 with a forward error bound first, exact
// integers at the cloud scale when the bound does not decide.
int diametral_side(const Cloud& c, const FixedCloud& f, u64 w, u64 u, u64 v) {
  double acc = 0, mag = 0;
  for (int a = 0; a < 3; ++a) {
    double xw, xu, xv;
    std::memcpy(&xw, &c.bits[w][a], 8);
    std::memcpy(&xu, &c.bits[u][a], 8);
    std::memcpy(&xv, &c.bits[v][a], 8);
    const double t = (xw - xu) * (xw - xv);
    acc += t;
    mag += std::fabs(t);
  }
  const double bound = 16.0 * 1.1102230246251565e-16 * mag + 1e-300;
  if (acc > bound) return 1;
  if (acc < -bound) return -1;
  Big s = 0;
  for (int a = 0; a < 3; ++a) s += (f.X[w][a] - f.X[u][a]) * (f.X[w][a] - f.X[v][a]);
  return s < 0 ? -1 : (s > 0 ? 1 : 0);
}

std::string center_text(const FixedCloud& f, u64 u, u64 v) {
  Big num[3];
  for (int a = 0; a < 3; ++a) num[a] = f.X[u][a] + f.X[v][a];
  int e = f.S + 1;
  while (e > 0 && num[0] % 2 == 0 && num[1] % 2 == 0 && num[2] % 2 == 0) {
    for (auto& x : num) x /= 2;
    --e;
  }
  return num[0].str() + " " + num[1].str() + " " + num[2].str() + " " + (Big(1) << (unsigned)e).str();
}

// All relevant pair supports by brute force: the outcome of
// build_exact_pair_support_stream (include/morsehgp3d/hierarchy/pair_support_stream.hpp:415)
// with its leaf rule classify_leaf_pair / classify_sparse_closed_ball
// (src/cpu/hierarchy/pair_support_stream.cpp:1781-2094): relevant iff the strict
// interior count I <= s_max - 2, with s_max = min(min(K, n) + 1, n); a shell of
// exactly the two supports is an event, a larger shell a diagnostic carrying the
// complete shell count and the least extra shell PointId.
std::string pairs_text(const Cloud& c, u64 K) {
  const FixedCloud f = fixed_cloud(c);
  const u64 n = c.bits.size();
  const u64 keff = std::min(K, n);
  const u64 smax = std::min(keff + 1, n);
  std::string ev, dg;
  if (smax < 2) return "S complete\n";
  const u64 cap = smax - 2;
  std::vector<u64> interior;
  for (u64 u = 0; u < n; ++u)
    for (u64 v = u + 1; v < n; ++v) {
      interior.clear();
      u64 shell = 0, extra = ~u64{0};
      bool reject = false;
      for (u64 w = 0; w < n; ++w) {
        const int sd = (w == u || w == v) ? 0 : diametral_side(c, f, w, u, v);
        if (sd < 0) {
          interior.push_back(w);
          if (interior.size() > cap) {
            reject = true;
            break;
          }
        } else if (sd == 0) {
          ++shell;
          if (w != u && w != v) extra = std::min(extra, w);
        }
      }
      if (reject) continue;
      const u64 I = interior.size();
      const Big D = dist2(f, u, v);
      const std::string tail = reduced(D, 2 * f.S + 2) + " " + center_text(f, u, v) + " |";
      std::string ids;
      for (u64 w : interior) ids += " " + std::to_string(w);
      if (shell == 2)
        ev += "P " + std::to_string(u) + " " + std::to_string(v) + " " + std::to_string(I + 2) + " " +
              std::to_string(n - I - 2) + " " + tail + ids + "\n";
      else
        dg += "D " + std::to_string(u) + " " + std::to_string(v) + " " + std::to_string(shell) + " " +
              std::to_string(extra) + " " + std::to_string(I + 2) + " " + std::to_string(I + shell) + " " +
              std::to_string(n - I - shell) + " " + tail + ids + "\n";
    }
  return ev + dg + "S complete\n";
}

// ---- triples and quads ---------------------------------------------------------------
// A value with a bound m on the sum of absolute values of the terms that built
// it: after k roundings the FP64 error is at most k*u*m, so |v| > 64*u*m
// certifies the sign.
struct Fm {
  double v, m;
};
Fm operator+(Fm a, Fm b) { return {a.v + b.v, a.m + b.m}; }
Fm operator-(Fm a, Fm b) { return {a.v - b.v, a.m + b.m}; }
Fm operator*(Fm a, Fm b) { return {a.v * b.v, a.m * b.m}; }
int fm_sign(Fm x) {
  const double bound = 64.0 * 1.1102230246251565e-16 * x.m + 1e-300;
  return x.v > bound ? 1 : (x.v < -bound ? -1 : 2);  // 2 = undecided
}
using FV = std::array<Fm, 3>;
using BV = std::array<Big, 3>;
template <class T> T dot3(const std::array<T, 3>& a, const std::array<T, 3>& b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
template <class T> std::array<T, 3> cross3(const std::array<T, 3>& a, const std::array<T, 3>& b) {
  return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
template <class T> std::array<T, 3> scale3(const T& s, const std::array<T, 3>& a) { return {s * a[0], s * a[1], s * a[2]}; }
template <class T> std::array<T, 3> add3(const std::array<T, 3>& a, const std::array<T, 3>& b) {
  return {a[0] + b[0], a[1] + b[1], a[2] + b[2]};
}

FV fdiff(const Cloud& c, u64 p, u64 q) {  // p - q in FP64 with magnitudes
  FV r;
  for (int a = 0; a < 3; ++a) {
    double x, y;
    std::memcpy(&x, &c.bits[p][a], 8);
    std::memcpy(&y, &c.bits[q][a], 8);
    r[a] = {x - y, std::fabs(x) + std::fabs(y)};
  }
  return r;
}
BV bdiff(const FixedCloud& f, u64 p, u64 q) { return {f.X[p][0] - f.X[q][0], f.X[p][1] - f.X[q][1], f.X[p][2] - f.X[q][2]}; }

// Exact geometry of one 3- or 4-point support (the circumcenter analysis of
// exact::analyze_circumcenter_support, include/morsehgp3d/exact/support.hpp:41,474-479):
//  triangle: well-centred iff the three angles are acute ((b-a).(c-a) > 0 ...);
//            centre a + (G22(G11-G12) e1 + G11(G22-G12) e2) / (2 det G);
//  tetrahedron: centre a + N / (2 det E), N = |e1|^2 e2xe3 + |e2|^2 e3xe1 + |e3|^2 e1xe2,
//            barycentric signs of the centre from N.(e_j x e_k) and 2 det E^2 - sum.
// status: 0 minimal, 1 boundary reduced, 2 exterior centre, 3 affinely dependent.
struct SupportGeo {
  int status = 3;
  int size = 0;
  u64 ids[4]{};
  // side(w): val(w) = A * |p|^2 - p . Nv with p = w - ids[0]; sign multiplied by sgn
  Big A;
  BV Nv;
  int sgn = 1;
  FV fN;
  Fm fA{0, 0};
};

SupportGeo analyze(const Cloud& c, const FixedCloud& f, const u64* ids, int size) {
  SupportGeo g;
  g.size = size;
  for (int i = 0; i < size; ++i) g.ids[i] = ids[i];
  if (size == 3) {
    const BV e1 = bdiff(f, ids[1], ids[0]), e2 = bdiff(f, ids[2], ids[0]);
    const Big G11 = dot3(e1, e1), G12 = dot3(e1, e2), G22 = dot3(e2, e2);
    const Big detG = G11 * G22 - G12 * G12;
    if (detG == 0) return g;
    const Big da = G12, db = G11 - G12, dc = G22 - G12;
    if (da < 0 || db < 0 || dc < 0) { g.status = 2; return g; }
    if (da == 0 || db == 0 || dc == 0) { g.status = 1; return g; }
    g.status = 0;
    g.A = detG;
    g.Nv = add3(scale3(Big(G22 * db), e1), scale3(Big(G11 * dc), e2));
  } else {
    const BV e1 = bdiff(f, ids[1], ids[0]), e2 = bdiff(f, ids[2], ids[0]), e3 = bdiff(f, ids[3], ids[0]);
    const BV c23 = cross3(e2, e3), c31 = cross3(e3, e1), c12 = cross3(e1, e2);
    const Big detE = dot3(e1, c23);
    if (detE == 0) return g;
    const BV N = add3(add3(scale3(dot3(e1, e1), c23), scale3(dot3(e2, e2), c31)), scale3(dot3(e3, e3), c12));
    const Big l1 = dot3(N, c23), l2 = dot3(N, c31), l3 = dot3(N, c12);
    const Big l0 = 2 * detE * detE - (l1 + l2 + l3);
    if (l0 < 0 || l1 < 0 || l2 < 0 || l3 < 0) { g.status = 2; return g; }
    if (l0 == 0 || l1 == 0 || l2 == 0 || l3 == 0) { g.status = 1; return g; }
    g.status = 0;
    g.A = detE;
    g.Nv = N;
    g.sgn = detE < 0 ? -1 : 1;
  }
  return g;
}

// FP64 image of the side polynomial, for the filter.
void analyze_fp(const Cloud& c, SupportGeo& g) {
  const u64* ids = g.ids;
  if (g.size == 3) {
    const FV e1 = fdiff(c, ids[1], ids[0]), e2 = fdiff(c, ids[2], ids[0]);
    const Fm G11 = dot3(e1, e1), G12 = dot3(e1, e2), G22 = dot3(e2, e2);
    g.fA = G11 * G22 - G12 * G12;
    g.fN = add3(scale3(G22 * (G11 - G12), e1), scale3(G11 * (G22 - G12), e2));
  } else {
    const FV e1 = fdiff(c, ids[1], ids[0]), e2 = fdiff(c, ids[2], ids[0]), e3 = fdiff(c, ids[3], ids[0]);
    const FV c23 = cross3(e2, e3), c31 = cross3(e3, e1), c12 = cross3(e1, e2);
    g.fA = dot3(e1, c23);
    g.fN = add3(add3(scale3(dot3(e1, e1), c23), scale3(dot3(e2, e2), c31)), scale3(dot3(e3, e3), c12));
  }
}

// FP64-filtered status of a 3- or 4-point support with the same 64 u m bound: 0 minimal,
// 1 not minimal (boundary, exterior centre or dependent; which one does not matter to the
// enumeration), 2 undecided (the exact analysis settles it).  Only a cheaper route to
// analyze()'s status: a decided FP64 sign equals the exact sign.
int status_fp(const Cloud& c, const u64* ids, int size) {
  if (size == 3) {
    const FV e1 = fdiff(c, ids[1], ids[0]), e2 = fdiff(c, ids[2], ids[0]);
    const Fm G11 = dot3(e1, e1), G12 = dot3(e1, e2), G22 = dot3(e2, e2);
    const int sa = fm_sign(G12), sb = fm_sign(G11 - G12), sc = fm_sign(G22 - G12);
    if (sa == -1 || sb == -1 || sc == -1) return 1;  // an obtuse angle: exterior centre or dependent
    if (sa == 2 || sb == 2 || sc == 2) return 2;
    const int sd = fm_sign(G11 * G22 - G12 * G12);
    return sd == 1 ? 0 : 2;  // three acute angles: detG > 0 exactly
  }
  const FV e1 = fdiff(c, ids[1], ids[0]), e2 = fdiff(c, ids[2], ids[0]), e3 = fdiff(c, ids[3], ids[0]);
  const FV c23 = cross3(e2, e3), c31 = cross3(e3, e1), c12 = cross3(e1, e2);
  const Fm detE = dot3(e1, c23);
  const int sd = fm_sign(detE);
  if (sd == 2) return 2;
  if (sd == 0) return 1;
  const FV N = add3(add3(scale3(dot3(e1, e1), c23), scale3(dot3(e2, e2), c31)), scale3(dot3(e3, e3), c12));
  const Fm l1 = dot3(N, c23), l2 = dot3(N, c31), l3 = dot3(N, c12);
  const Fm two{2.0, 2.0};
  const Fm l0 = two * detE * detE - (l1 + l2 + l3);
  const int s[4] = {fm_sign(l0), fm_sign(l1), fm_sign(l2), fm_sign(l3)};
  bool und = false;
  for (int i = 0; i < 4; ++i) {
    if (s[i] == -1 || s[i] == 0) return 1;
    und |= s[i] == 2;
  }
  return und ? 2 : 0;
}

// Side of w against a support whose exact geometry may not be computed yet: the FP64
// filter first; the exact integers (analyze) only when it does not decide.
struct LazyGeo {
  const Cloud& c;
  const FixedCloud& f;
  SupportGeo g;
  bool exact = false;
  LazyGeo(const Cloud& c_, const FixedCloud& f_, const u64* ids, int size) : c(c_), f(f_) {
    g.size = size;
    for (int i = 0; i < size; ++i) g.ids[i] = ids[i];
    analyze_fp(c, g);
    // sign of A in FP64 (A = det G > 0 for a minimal triangle; det E for a tetrahedron)
    const int sa = fm_sign(g.fA);
    if (size == 3) g.sgn = 1;
    else if (sa == 1 || sa == -1) g.sgn = sa;
    else make_exact();
  }
  void make_exact() {
    if (exact) return;
    g = [&] { SupportGeo e = analyze(c, f, g.ids, g.size); analyze_fp(c, e); return e; }();
    exact = true;
  }
  int side(u64 w) {
    const FV p = fdiff(c, w, g.ids[0]);
    const int s = fm_sign(g.fA * dot3(p, p) - dot3(p, g.fN));
    if (s != 2) return s * g.sgn;
    make_exact();
    const BV q = bdiff(f, w, g.ids[0]);
    const Big val = g.A * dot3(q, q) - dot3(q, g.Nv);
    return (val < 0 ? -1 : (val > 0 ? 1 : 0)) * g.sgn;
  }
};

// Every minimal 3- and 4-point support with at most cap(size) strict interior points,
// enumerated by brute force over all tuples in (size, ids) order; emit(tid, geo, interior,
// shell, extra) runs for each on thread tid, its tuples' least id split over threads by
// `first` in strides, so a caller that keeps one buffer per least id restores the order.
template <class Emit>
void enumerate_higher(const Cloud& c, const FixedCloud& f, u64 smax, Emit&& emit) {
  const u64 n = c.bits.size();
  const unsigned hw = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
  std::vector<std::thread> pool;
  auto run = [&](unsigned tid) {
    std::vector<u64> interior;
    auto visit = [&](const u64* ids, int size) {
      if (smax < (u64)size) return;
      const int st = status_fp(c, ids, size);
      if (st == 1) return;
      if (st == 2 && analyze(c, f, ids, size).status != 0) return;
      LazyGeo lg(c, f, ids, size);
      const u64 cap = smax - size;
      interior.clear();
      u64 shell = size, extra = ~u64{0};
      for (u64 w = 0; w < n; ++w) {
        bool sup = false;
        for (int i = 0; i < size; ++i) sup |= (w == ids[i]);
        if (sup) continue;
        const int sd = lg.side(w);
        if (sd < 0) {
          interior.push_back(w);
          if (interior.size() > cap) return;
        } else if (sd == 0) {
          ++shell;
          extra = std::min(extra, w);
        }
      }
      lg.make_exact();
      emit(tid, lg.g, interior, shell, extra);
    };
    u64 ids[4];
    for (ids[0] = tid; ids[0] < n; ids[0] += hw)
      for (ids[1] = ids[0] + 1; ids[1] < n; ++ids[1])
        for (ids[2] = ids[1] + 1; ids[2] < n; ++ids[2]) {
          visit(ids, 3);
          for (ids[3] = ids[2] + 1; ids[3] < n; ++ids[3]) visit(ids, 4);
        }
  };
  for (unsigned t = 1; t < hw; ++t) pool.emplace_back(run, t);
  run(0);
  for (auto& t : pool) t.join();
}

int higher_side(const Cloud& c, const FixedCloud& f, const SupportGeo& g, u64 w) {
  const FV p = fdiff(c, w, g.ids[0]);
  const int s = fm_sign(g.fA * dot3(p, p) - dot3(p, g.fN));
  if (s != 2) return s * g.sgn;
  const BV q = bdiff(f, w, g.ids[0]);
  const Big val = g.A * dot3(q, q) - dot3(q, g.Nv);
  return (val < 0 ? -1 : (val > 0 ? 1 : 0)) * g.sgn;
}

std::string reduced_vec(BV num, Big den) {  // (num / den), common gcd removed
  if (den < 0) {
    den = -den;
    for (auto& x : num) x = -x;
  }
  Big g = den;
  for (const auto& x : num) {
    Big a = x < 0 ? Big(-x) : x, b = g;
    while (b != 0) {
      Big t = a % b;
      a = b;
      b = t;
    }
    g = a;
  }
  if (g == 0) g = 1;
  return Big(num[0] / g).str() + " " + Big(num[1] / g).str() + " " + Big(num[2] / g).str() + " " + Big(den / g).str();
}

std::string reduced_frac(Big num, Big den) {
  if (den < 0) { den = -den; num = -num; }
  Big a = num < 0 ? Big(-num) : num, b = den;
  while (b != 0) {
    Big t = a % b;
    a = b;
    b = t;
  }
  return Big(num / a).str() + " " + Big(den / a).str();
}

// Level and centre of a minimal support: centre = a + Nv / (k A) with k = 2.
std::string sphere_text(const FixedCloud& f, const SupportGeo& g) {
  const Big den = 2 * g.A;  // centre offset = Nv / den (both sizes)
  const Big two_S = Big(1) << (unsigned)f.S;
  const Big lev_num = dot3(g.Nv, g.Nv);
  const Big lev_den = den * den * (Big(1) << (unsigned)(2 * f.S));
  BV cnum;
  for (int a = 0; a < 3; ++a) cnum[a] = den * f.X[g.ids[0]][a] + g.Nv[a];
  return reduced_frac(lev_num, lev_den) + " " + reduced_vec(cnum, den * two_S);
}

// All relevant 3- and 4-point supports by brute force: the outcome of
// build_exact_higher_support_stream run to completion
// (include/morsehgp3d/hierarchy/higher_support_stream.hpp:544; leaf rule
// classify_terminal_support, src/cpu/hierarchy/higher_support_stream.cpp:1992-2110):
// only minimal (well-centred, affinely independent) supports; relevant iff
// interior + size <= s_max; event iff the shell is exactly the support.
std::string higher_text(const Cloud& c, u64 K) {
  const FixedCloud f = fixed_cloud(c);
  const u64 n = c.bits.size();
  const u64 keff = std::min(K, n), smax = std::min(keff + 1, n);
  // one buffer per (least id, size, event/diagnostic): concatenated in (size, ids) order
  std::vector<std::string> ev3(n), ev4(n), dg3(n), dg4(n);
  enumerate_higher(c, f, smax, [&](unsigned, const SupportGeo& g, const std::vector<u64>& interior, u64 shell,
                                   u64 extra) {
    const int size = g.size;
    const u64 I = interior.size();
    std::string head = std::to_string(size);
    for (int i = 0; i < size; ++i) head += " " + std::to_string(g.ids[i]);
    std::string idt;
    for (u64 w : interior) idt += " " + std::to_string(w);
    const std::string sph = sphere_text(f, g);
    const u64 a = g.ids[0];
    if (shell == (u64)size)
      (size == 3 ? ev3 : ev4)[a] += "H " + head + " " + std::to_string(I + size) + " " + std::to_string(n - I - size) +
                                    " " + sph + " |" + idt + "\n";
    else
      (size == 3 ? dg3 : dg4)[a] += "G " + head + " " + std::to_string(shell) + " " + std::to_string(extra) + " " +
                                    std::to_string(I + size) + " " + std::to_string(I + shell) + " " +
                                    std::to_string(n - I - shell) + " " + sph + " |" + idt + "\n";
  });
  // the stream orders records by (support size, ids): triples before quads
  std::string out;
  for (const auto* v : {&ev3, &ev4, &dg3, &dg4})
    for (const auto& x : *v) out += x;
  return out + "S complete\n";
}

// ---- direct hierarchy: facade, Morse event journal, arm seeds, forest journal --------
// A brute-force restatement of the reference's direct chain
//   build_exact_direct_support_terminal_facade (src/cpu/hierarchy/direct_support_terminal.cpp:68-300)
//   build_exact_direct_morse_event_journal     (src/cpu/hierarchy/direct_morse_event_journal.cpp:260-400)
//   build_exact_direct_saddle_arm_seed_journal (src/cpu/hierarchy/direct_saddle_arm_seed_journal.cpp:380-420)
//   build_exact_direct_morse_forest_journal    (src/cpu/hierarchy/direct_morse_forest_journal.cpp:1042-2150)
// with the descent closure of direct_sparse_facet_descent_{step,closure} restated
// as: a facet bound in the locator resolves to its birth handle; otherwise its
// exact miniball centre c_F gives the canonical top-k choice G (strictly closer
// points, then the least PointIds of the cutoff shell); G = F is unresolved, and
// beta(G) < beta(F) is required before the descent continues from G.
struct Rat {
  Big num, den;  // den > 0
};
bool rat_less(const Rat& a, const Rat& b) { return a.num * b.den < b.num * a.den; }
bool rat_eq(const Rat& a, const Rat& b) { return a.num * b.den == b.num * a.den; }
std::string rat_text(const Rat& r) { return reduced_frac(r.num, r.den); }

// A ball centred at X[ids0] + Nv / (2A) (cloud-scale integers); level in cloud units.
struct XBall {
  int size = 0;
  u64 ids[4]{};
  Big A;
  BV Nv;
  Rat level;
};

XBall ball_of(const Cloud& c, const FixedCloud& f, const u64* ids, int size, bool* minimal) {
  XBall b;
  b.size = size;
  for (int i = 0; i < size; ++i) b.ids[i] = ids[i];
  *minimal = true;
  if (size == 1) {
    b.A = 1;
    b.Nv = {Big(0), Big(0), Big(0)};
  } else if (size == 2) {
    b.A = 1;
    b.Nv = bdiff(f, ids[1], ids[0]);
  } else {
    SupportGeo g = analyze(c, f, ids, size);
    if (g.status != 0) {
      *minimal = false;
      return b;
    }
    b.A = g.A;
    b.Nv = g.Nv;
  }
  b.level = {dot3(b.Nv, b.Nv), 4 * b.A * b.A * (Big(1) << (unsigned)(2 * f.S))};
  return b;
}

// (2A)^2 2^(2S) |p - centre|^2 as an integer
Big scaled_dist(const FixedCloud& f, const XBall& b, u64 p) {
  Big s = 0;
  for (int a = 0; a < 3; ++a) {
    const Big t = 2 * b.A * (f.X[p][a] - f.X[b.ids[0]][a]) - b.Nv[a];
    s += t * t;
  }
  return s;
}

// Exact miniball of a facet of 1..10 points (build_exact_facet_miniball,
// include/morsehgp3d/hierarchy/facet_miniball.hpp:86-102): the enclosing ball of
// least radius among the circumspheres of 1- to 4-subsets with a relatively
// interior centre.
XBall facet_miniball(const Cloud& c, const FixedCloud& f, const std::vector<u64>& F) {
  const int k = (int)F.size();
  XBall best;
  bool have = false;
  u64 ids[4];
  auto consider = [&](int size) {
    bool minimal = false;
    XBall b = ball_of(c, f, ids, size, &minimal);
    if (!minimal) return;
    const Big r2 = dot3(b.Nv, b.Nv);  // (2A)^2 2^(2S) * level
    for (u64 w : F) {
      bool sup = false;
      for (int i = 0; i < size; ++i) sup |= ids[i] == w;
      if (sup) continue;
      if (scaled_dist(f, b, w) > r2) return;  // outside the closed ball
    }
    if (!have || rat_less(b.level, best.level)) {
      best = b;
      have = true;
    }
  };
  for (int i = 0; i < k; ++i) {
    ids[0] = F[i];
    if (k == 1) consider(1);
    for (int j = i + 1; j < k; ++j) {
      ids[1] = F[j];
      consider(2);
      for (int l = j + 1; l < k; ++l) {
        ids[2] = F[l];
        consider(3);
        for (int m = l + 1; m < k; ++m) {
          ids[3] = F[m];
          consider(4);
        }
      }
    }
  }
  if (!have) throw std::logic_error("a facet has no exact miniball");
  return best;
}

struct HEvent {
  int size = 0;
  u64 ids[4]{};
  std::vector<u64> interior;
  u64 rank = 0;
  Rat level;
  int birth = 0, saddle = 0;  // 0 = none
};

bool hevent_less(const HEvent& a, const HEvent& b) {
  if (!rat_eq(a.level, b.level)) return rat_less(a.level, b.level);
  if (a.rank != b.rank) return a.rank < b.rank;
  if (a.interior != b.interior) return a.interior < b.interior;
  const int m = std::min(a.size, b.size);
  for (int i = 0; i < m; ++i)
    if (a.ids[i] != b.ids[i]) return a.ids[i] < b.ids[i];
  return a.size < b.size;
}

std::string hierarchy_text(const Cloud& c, u64 K) {
  const FixedCloud f = fixed_cloud(c);
  const u64 n = c.bits.size();
  const u64 keff = std::min(K, n), smax = std::min(keff + 1, n);
  std::vector<HEvent> ev;
  u64 diagnostics = 0;
  // pair supports
  if (smax >= 2) {
    for (u64 u = 0; u < n; ++u)
      for (u64 v = u + 1; v < n; ++v) {
        HEvent e;
        e.size = 2;
        e.ids[0] = u;
        e.ids[1] = v;
        u64 shell = 2;
        bool reject = false;
        for (u64 w = 0; w < n && !reject; ++w) {
          if (w == u || w == v) continue;
          const int sd = diametral_side(c, f, w, u, v);
          if (sd < 0) {
            e.interior.push_back(w);
            reject = e.interior.size() > smax - 2;
          } else if (sd == 0) {
            ++shell;
          }
        }
        if (reject) continue;
        if (shell != 2) {
          ++diagnostics;
          continue;
        }
        bool minimal = false;
        e.level = ball_of(c, f, e.ids, 2, &minimal).level;
        ev.push_back(std::move(e));
      }
  }
  // triple and quad supports
  {
    std::vector<std::vector<HEvent>> per(std::max(1u, std::min(64u, std::thread::hardware_concurrency())));
    std::vector<u64> diag(per.size(), 0);
    enumerate_higher(c, f, smax, [&](unsigned tid, const SupportGeo& g, const std::vector<u64>& interior, u64 shell,
                                     u64) {
      if (shell != (u64)g.size) {
        ++diag[tid];
        return;
      }
      HEvent e;
      e.size = g.size;
      for (int i = 0; i < g.size; ++i) e.ids[i] = g.ids[i];
      e.interior = interior;
      bool minimal = false;
      e.level = ball_of(c, f, e.ids, g.size, &minimal).level;
      per[tid].push_back(std::move(e));
    });
    for (size_t t = 0; t < per.size(); ++t) {
      diagnostics += diag[t];
      for (auto& e : per[t]) ev.push_back(std::move(e));
    }
  }
  for (auto& e : ev) {
    e.rank = e.interior.size() + e.size;
    e.birth = e.rank <= keff ? (int)e.rank : 0;
    e.saddle = (e.rank >= 2 && e.rank - 1 <= keff) ? (int)(e.rank - 1) : 0;
  }
  std::sort(ev.begin(), ev.end(), hevent_less);
  std::string s;
  for (u64 i = 0; i < ev.size(); ++i) {
    const HEvent& e = ev[i];
    s += "F " + std::to_string(i) + " " + std::to_string(e.size);
    for (int j = 0; j < e.size; ++j) s += " " + std::to_string(e.ids[j]);
    s += " |";
    for (u64 w : e.interior) s += " " + std::to_string(w);
    s += " | " + std::to_string(e.rank) + " " + std::to_string(n - e.rank) + " " + rat_text(e.level) + " " +
         (e.birth ? std::to_string(e.birth) : std::string("-")) + " " +
         (e.saddle ? std::to_string(e.saddle) : std::string("-")) + "\n";
  }
  s += "X " + std::to_string(diagnostics) + "\n";
  if (diagnostics) {  // journal: no_journal_relevant_extra_shell_diagnostics; seeds and forest reject the source
    return s + "C\nD 4 3 4\n";
  }
  // Morse event journal: projections 0..n-1 are singletons, n + i the facade events
  struct Seed {
    u64 order;
    Rat level;
    u64 proj;
    int role;  // 0 birth, 1 saddle
  };
  std::vector<Seed> seeds;
  for (u64 p = 0; p < n; ++p) seeds.push_back({1, {Big(0), Big(1)}, p, 0});
  for (u64 i = 0; i < ev.size(); ++i) {
    if (ev[i].birth) seeds.push_back({(u64)ev[i].birth, ev[i].level, n + i, 0});
    if (ev[i].saddle) seeds.push_back({(u64)ev[i].saddle, ev[i].level, n + i, 1});
  }
  std::stable_sort(seeds.begin(), seeds.end(), [](const Seed& a, const Seed& b) {
    if (a.order != b.order) return a.order < b.order;
    if (!rat_eq(a.level, b.level)) return rat_less(a.level, b.level);
    if (a.proj != b.proj) return a.proj < b.proj;
    return a.role < b.role;
  });
  struct JBatch {
    u64 order;
    Rat level;
    u64 off, cnt, births, saddles;
  };
  std::vector<JBatch> jb;
  std::vector<u64> role_batch(seeds.size());
  for (u64 i = 0; i < seeds.size();) {
    u64 j = i;
    JBatch b{seeds[i].order, seeds[i].level, i, 0, 0, 0};
    while (j < seeds.size() && seeds[j].order == b.order && rat_eq(seeds[j].level, b.level)) {
      (seeds[j].role ? b.saddles : b.births)++;
      role_batch[j] = jb.size();
      ++j;
    }
    b.cnt = j - i;
    jb.push_back(b);
    i = j;
  }
  for (const auto& b : jb)
    s += "J " + std::to_string(&b - jb.data()) + " " + std::to_string(b.order) + " " + rat_text(b.level) + " " +
         std::to_string(b.off) + " " + std::to_string(b.cnt) + " " + std::to_string(b.births) + " " +
         std::to_string(b.saddles) + "\n";
  for (u64 i = 0; i < seeds.size(); ++i)
    s += "Q " + std::to_string(i) + " " + std::to_string(role_batch[i]) + " " + std::to_string(seeds[i].proj) + " " +
         std::to_string(seeds[i].role) + "\n";
  // saddle families and arm seeds
  auto facet_of = [&](u64 proj) {  // I u U sorted
    std::vector<u64> F;
    if (proj < n) {
      F.push_back(proj);
      return F;
    }
    const HEvent& e = ev[proj - n];
    F = e.interior;
    for (int j = 0; j < e.size; ++j) F.push_back(e.ids[j]);
    std::sort(F.begin(), F.end());
    return F;
  };
  struct Family {
    u64 event, proj, role, batch, order, arm_off, arm_cnt;
  };
  std::vector<Family> fam;
  std::vector<std::pair<u64, u64>> arms;  // (family, removed)
  for (u64 i = 0; i < seeds.size(); ++i) {
    if (seeds[i].role != 1) continue;
    const HEvent& e = ev[seeds[i].proj - n];
    fam.push_back({seeds[i].proj - n, seeds[i].proj, i, role_batch[i], seeds[i].order, arms.size(), (u64)e.size});
    for (int j = 0; j < e.size; ++j) arms.push_back({fam.size() - 1, e.ids[j]});
  }
  for (u64 i = 0; i < fam.size(); ++i)
    s += "Y " + std::to_string(i) + " " + std::to_string(fam[i].event) + " " + std::to_string(fam[i].proj) + " " +
         std::to_string(fam[i].role) + " " + std::to_string(fam[i].batch) + " " + std::to_string(fam[i].order) + " " +
         rat_text(jb[fam[i].batch].level) + " " + std::to_string(fam[i].arm_off) + " " +
         std::to_string(fam[i].arm_cnt) + "\n";
  for (u64 i = 0; i < arms.size(); ++i)
    s += "Z " + std::to_string(i) + " " + std::to_string(arms[i].first) + " " + std::to_string(arms[i].second) + "\n";
  auto arm_facet = [&](u64 a) {
    std::vector<u64> F = facet_of(fam[arms[a].first].proj);
    F.erase(std::find(F.begin(), F.end(), arms[a].second));
    return F;
  };
  // ---- forest journal
  u64 birth_count = 0;
  for (const auto& sd : seeds) birth_count += sd.role == 0;
  std::vector<u64> parent(birth_count), border(birth_count, 0);
  std::vector<long long> rroot(birth_count, -1);
  std::vector<char> active(birth_count, 0);
  for (u64 i = 0; i < birth_count; ++i) parent[i] = i;
  auto root = [&](u64 h) {
    while (parent[h] != h) h = parent[h];
    return h;
  };
  std::vector<std::vector<u64>> order_handles(keff + 2);  // born handles of each order
  auto count_roots = [&](u64 order, bool reduced) {
    u64 k = 0;
    for (u64 h : order_handles[order])
      if (active[h] && parent[h] == h && border[h] == order && (!reduced || rroot[h] >= 0)) ++k;
    return k;
  };
  std::map<std::vector<u64>, u64> locator;  // bound facet -> birth handle
  std::string N, C = "C", B, A, S, G, T, R;
  u64 nodes = 0, children = 0, births = 0, bindings = 0, saddles = 0, groups = 0;
  // The successor G of a facet F in a strict descent depends on the geometry alone, so it is
  // computed once per facet; where a descent stops depends on the locator at the call.
  std::map<std::vector<u64>, std::vector<u64>> successor;
  auto descend = [&](std::vector<u64> F) -> u64 {
    for (int guard = 0; guard < 100000; ++guard) {
      const auto hit = locator.find(F);
      if (hit != locator.end()) return hit->second;
      const auto memo = successor.find(F);
      if (memo != successor.end()) {
        F = memo->second;
        continue;
      }
      const XBall bf = facet_miniball(c, f, F);
      const u64 k = F.size();
      std::vector<std::pair<Big, u64>> d(n);
      for (u64 p = 0; p < n; ++p) d[p] = {scaled_dist(f, bf, p), p};
      std::nth_element(d.begin(), d.begin() + (k - 1), d.end(),
                       [](const auto& x, const auto& y) { return x.first < y.first; });
      const Big cut = d[k - 1].first;
      std::vector<u64> below, shell;
      for (const auto& x : d) {
        if (x.first < cut) below.push_back(x.second);
        else if (x.first == cut) shell.push_back(x.second);
      }
      std::sort(shell.begin(), shell.end());
      std::vector<u64> Gs = below;
      for (u64 i = 0; Gs.size() < k; ++i) Gs.push_back(shell[i]);
      std::sort(Gs.begin(), Gs.end());
      if (Gs == F) throw std::logic_error("a strict arm descent is unresolved");
      const XBall bg = facet_miniball(c, f, Gs);
      if (!rat_less(bg.level, bf.level)) throw std::logic_error("a strict arm descent met a plateau");
      successor.emplace(F, Gs);
      F = Gs;
    }
    throw std::logic_error("a strict arm descent did not terminate");
  };
  auto key_text = [](const std::vector<u64>& F) {
    std::string t = std::to_string(F.size());
    for (u64 x : F) t += " " + std::to_string(x);
    return t;
  };
  u64 fam_cursor = 0;
  for (u64 bi = 0; bi < jb.size(); ++bi) {
    const JBatch& jbat = jb[bi];
    const u64 pre_c = count_roots(jbat.order, false), pre_r = count_roots(jbat.order, true);
    const u64 fam_begin = fam_cursor;
    while (fam_cursor < fam.size() && fam[fam_cursor].batch == bi) ++fam_cursor;
    struct Arm {
      u64 seed, carrier;
      long long prior;
      std::vector<u64> key;
    };
    std::vector<std::vector<Arm>> sad;
    std::map<std::vector<u64>, std::pair<u64, long long>> resolved;
    for (u64 fi = fam_begin; fi < fam_cursor; ++fi) {
      std::vector<Arm> as;
      for (u64 a = fam[fi].arm_off; a < fam[fi].arm_off + fam[fi].arm_cnt; ++a) as.push_back({a, 0, -1, arm_facet(a)});
      sad.push_back(std::move(as));
    }
    for (auto& as : sad)
      for (auto& a : as) {
        auto it = resolved.find(a.key);
        if (it == resolved.end()) {
          const u64 h = root(descend(a.key));
          it = resolved.emplace(a.key, std::make_pair(h, rroot[h])).first;
        }
        a.carrier = it->second.first;
        a.prior = it->second.second;
      }
    // frozen-root quotient: transitive classes of carriers over the saddles
    std::map<u64, u64> qp;
    std::function<u64(u64)> qf = [&](u64 x) { return qp[x] == x ? x : (qp[x] = qf(qp[x])); };
    for (auto& as : sad)
      for (auto& a : as)
        if (!qp.count(a.carrier)) qp[a.carrier] = a.carrier;
    for (auto& as : sad)
      for (auto& a : as) {
        const u64 x = qf(as[0].carrier), y = qf(a.carrier);
        if (x != y) qp[std::max(x, y)] = std::min(x, y);
      }
    std::map<u64, std::vector<u64>> cls;  // least carrier -> carriers (sorted)
    for (auto& kv : qp) cls[qf(kv.first)].push_back(kv.first);
    struct Plan {
      std::vector<u64> carriers, priors, saddles;
      int kind;  // 0 reduced birth, 1 continuation, 2 multifusion
      long long created = -1;
      u64 result = 0;
    };
    std::vector<Plan> plans;
    std::map<u64, u64> plan_of;
    for (auto& kv : cls) {
      plan_of[kv.first] = plans.size();
      Plan p;
      p.carriers = kv.second;
      for (u64 h : p.carriers)
        if (rroot[h] >= 0) p.priors.push_back((u64)rroot[h]);
      std::sort(p.priors.begin(), p.priors.end());
      plans.push_back(std::move(p));
    }
    for (u64 si = 0; si < sad.size(); ++si) plans[plan_of[qf(sad[si][0].carrier)]].saddles.push_back(si);
    u64 pending_nodes = 0;
    for (auto& p : plans) {
      if (p.priors.size() == 1) {
        p.kind = 1;
        p.result = p.priors[0];
      } else {
        if (p.priors.empty() && jbat.order == 1) throw std::logic_error("an order-one group has no prior root");
        p.kind = p.priors.empty() ? 0 : 2;
        p.created = (long long)(nodes + pending_nodes++);
        p.result = (u64)p.created;
      }
    }
    const u64 s_off0 = saddles, g_off0 = groups;
    for (auto& p : plans) {
      const u64 g_s_off = saddles;
      for (u64 si : p.saddles) {
        const u64 fi = fam_begin + si;
        const u64 arm_off = bindings;
        std::vector<u64> cs, ps;
        for (auto& a : sad[si]) {
          A += "A " + std::to_string(bindings++) + " " + std::to_string(a.seed) + " " + std::to_string(fi) + " " +
               std::to_string(a.carrier) + " " + (a.prior >= 0 ? std::to_string(a.prior) : std::string("-")) +
               " | " + key_text(a.key) + "\n";
          cs.push_back(a.carrier);
          if (a.prior >= 0) ps.push_back((u64)a.prior);
        }
        std::sort(cs.begin(), cs.end());
        cs.erase(std::unique(cs.begin(), cs.end()), cs.end());
        std::sort(ps.begin(), ps.end());
        ps.erase(std::unique(ps.begin(), ps.end()), ps.end());
        S += "S " + std::to_string(saddles++) + " " + std::to_string(fi) + " " + std::to_string(fam[fi].event) + " " +
             std::to_string(bi) + " " + std::to_string(arm_off) + " " + std::to_string(sad[si].size()) + " " +
             std::to_string(cs.size()) + " " + std::to_string(cs.size() - ps.size()) + " " +
             std::to_string(ps.size()) + " " + std::to_string(groups) + "\n";
      }
      const u64 child_cnt = p.kind == 2 ? p.priors.size() : 0;
      G += "G " + std::to_string(groups) + " " + std::to_string(bi) + " " + std::to_string(g_s_off) + " " +
           std::to_string(saddles - g_s_off) + " " + std::to_string(p.carriers.size()) + " " +
           std::to_string(p.carriers.size() - p.priors.size()) + " " + std::to_string(p.priors.size()) + " " +
           std::to_string(children) + " " + std::to_string(child_cnt) + " " +
           (p.created >= 0 ? std::to_string(p.created) : std::string("-")) + " " + std::to_string(p.result) + " " +
           std::to_string(p.kind) + "\n";
      if (p.kind != 1)
        N += "N " + std::to_string(p.created) + " " + std::to_string(jbat.order) + " " + rat_text(jbat.level) + " " +
             std::to_string(p.kind == 0 ? 1 : 2) + " " + std::to_string(children) + " " + std::to_string(child_cnt) +
             " - " + std::to_string(groups) + "\n";
      if (p.kind == 2)
        for (u64 x : p.priors) C += " " + std::to_string(x);
      children += child_cnt;
      ++groups;
    }
    nodes += pending_nodes;
    // births of this batch (hidden from this batch's descents)
    struct Birth {
      u64 handle, order;
      long long node;
      std::vector<u64> key;
    };
    std::vector<Birth> nb;
    const u64 b_off0 = births;
    for (u64 r = jbat.off; r < jbat.off + jbat.cnt; ++r) {
      if (seeds[r].role != 0) continue;
      Birth b{births, jbat.order, -1, facet_of(seeds[r].proj)};
      if (jbat.order == 1) {
        b.node = (long long)nodes++;
        N += "N " + std::to_string(b.node) + " 1 " + rat_text(jbat.level) + " 0 " + std::to_string(children) +
             " 0 " + std::to_string(births) + " -\n";
      }
      B += "B " + std::to_string(births) + " " + std::to_string(seeds[r].proj) + " " + std::to_string(bi) + " " +
           std::to_string(jbat.order) + " " + std::to_string(births) + " " +
           (b.node >= 0 ? std::to_string(b.node) : std::string("-")) + " | " + key_text(b.key) + "\n";
      ++births;
      nb.push_back(std::move(b));
    }
    // commit: unions (least handle survives), reduced roots, then births
    for (auto& p : plans) {
      u64 r0 = root(p.carriers.front());
      for (u64 i = 1; i < p.carriers.size(); ++i) {
        const u64 r1 = root(p.carriers[i]);
        if (r1 == r0) continue;
        const u64 lo = std::min(r0, r1), hi = std::max(r0, r1);
        parent[hi] = lo;
        r0 = lo;
      }
      rroot[r0] = (long long)p.result;
    }
    for (auto& b : nb) {
      active[b.handle] = 1;
      border[b.handle] = b.order;
      order_handles[b.order].push_back(b.handle);
      rroot[b.handle] = b.node;
      locator[b.key] = b.handle;
    }
    T += "T " + std::to_string(bi) + " " + std::to_string(bi) + " " + std::to_string(jbat.order) + " " +
         rat_text(jbat.level) + " " + std::to_string(b_off0) + " " + std::to_string(births - b_off0) + " " +
         std::to_string(s_off0) + " " + std::to_string(saddles - s_off0) + " " + std::to_string(g_off0) + " " +
         std::to_string(groups - g_off0) + " " + std::to_string(pre_c) + " " + std::to_string(pre_r) + " " +
         std::to_string(count_roots(jbat.order, false)) + " " + std::to_string(count_roots(jbat.order, true)) + "\n";
  }
  std::vector<std::array<u64, 3>> fr;  // (order, node, handle)
  for (u64 h = 0; h < birth_count; ++h)
    if (active[h] && parent[h] == h && rroot[h] >= 0) fr.push_back({border[h], (u64)rroot[h], h});
  std::sort(fr.begin(), fr.end());
  for (u64 i = 0; i < fr.size(); ++i)
    R += "R " + std::to_string(i) + " " + std::to_string(fr[i][0]) + " " + std::to_string(fr[i][2]) + " " +
         std::to_string(fr[i][1]) + "\n";
  return s + N + C + "\n" + B + A + S + G + T + R + "D 5 5 13\n";
}

// Exact classification of given supports against every point of the cloud: the leaf rule
// of the pair stream (classify_sparse_closed_ball, src/cpu/hierarchy/pair_support_stream.cpp:1781-1952)
// and of the higher stream (classify_terminal_support, higher_support_stream.cpp:1992-2110),
// without any bound or pruning.  Per support (size, ids[4]): status (0 minimal, 1 not),
// strict interior count, complete shell count (support included), least extra shell
// PointId (or all ones), the first 10 strict interior ids ascending (unused all ones).
void classify_supports(const Cloud& c, const FixedCloud& f, const uint32_t* sup, u64 count, uint32_t* out) {
  const u64 n = c.bits.size();
  const unsigned hw = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
  auto run = [&](unsigned tid) {
    for (u64 i = tid; i < count; i += hw) {
      const uint32_t* r = sup + 5 * i;
      uint32_t* o = out + 14 * i;
      const int size = (int)r[0];
      u64 ids[4] = {r[1], r[2], r[3], r[4]};
      for (int j = 0; j < 14; ++j) o[j] = 0xffffffffu;
      o[0] = 1;
      if (size < 2 || size > 4) continue;
      bool ok = true;
      for (int j = 0; j < size; ++j) ok &= ids[j] < n;
      if (!ok) continue;
      std::unique_ptr<LazyGeo> lg;
      if (size >= 3) {
        if (analyze(c, f, ids, size).status != 0) continue;
        lg.reset(new LazyGeo(c, f, ids, size));
      }
      u64 I = 0, shell = (u64)size, extra = ~u64{0};
      for (u64 w = 0; w < n; ++w) {
        bool on = false;
        for (int j = 0; j < size; ++j) on |= w == ids[j];
        if (on) continue;
        const int sd = size == 2 ? diametral_side(c, f, w, ids[0], ids[1]) : lg->side(w);
        if (sd < 0) {
          if (I < 10) o[4 + I] = (uint32_t)w;
          ++I;
        } else if (sd == 0) {
          ++shell;
          extra = std::min(extra, w);
        }
      }
      o[0] = 0;
      o[1] = (uint32_t)I;
      o[2] = (uint32_t)shell;
      o[3] = extra == ~u64{0} ? 0xffffffffu : (uint32_t)extra;
    }
  };
  std::vector<std::thread> pool;
  for (unsigned t = 1; t < hw; ++t) pool.emplace_back(run, t);
  run(0);
  for (auto& t : pool) t.join();
}

u64 put_text(const std::string& s, char* buf, u64 cap) {
  if (s.size() + 1 > cap) return s.size() + 1;
  std::memcpy(buf, s.c_str(), s.size() + 1);
  return 0;
}

int report(const std::exception& e, char* err, u64 errlen, int code) {
  if (err && errlen) {
    std::strncpy(err, e.what(), errlen - 1);
    err[errlen - 1] = 0;
  }
  return code;
}

}  // namespace

extern "C" {

// Same outputs and layout as ref_lbvh_build in oracle/ref_driver.cpp.
int oracle_lbvh_build(const double* xyz, u64 n, u64* source_index, u64* leaves, u64* nodes, u64* counters,
                      u64* root_aabb, u64* root, char* err, u64 errlen) {
  try {
    const Cloud c = canonical_cloud(xyz, n);
    const Lbvh t = build_lbvh(c);
    if (source_index)
      for (u64 p = 0; p < n; ++p) source_index[p] = c.source[p];
    if (leaves)
      for (u64 i = 0; i < n; ++i) {
        leaves[2 * i] = t.leaves[i].first;
        leaves[2 * i + 1] = t.leaves[i].second;
      }
    if (nodes)
      for (u64 i = 0; i < t.nodes.size(); ++i) {
        const Node& nd = t.nodes[i];
        u64* r = nodes + 10 * i;
        for (int a = 0; a < 3; ++a) {
          r[a] = nd.lo[a];
          r[3 + a] = nd.hi[a];
        }
        r[6] = nd.left;
        r[7] = nd.right;
        r[8] = nd.begin;
        r[9] = nd.end;
      }
    if (counters) {
      counters[0] = n;
      counters[1] = 2 * n - 1;
      counters[2] = t.max_depth;
      counters[3] = t.collision_groups;
      counters[4] = t.max_collision;
    }
    if (root_aabb)
      for (int k = 0; k < 6; ++k) root_aabb[k] = t.root_aabb[k];
    if (root) *root = 2 * n - 2;
    return 0;
  } catch (const std::invalid_argument& e) {
    return report(e, err, errlen, 1);
  } catch (const std::exception& e) {
    return report(e, err, errlen, 2);
  }
}

int oracle_knn(const double* xyz, u64 n, u64 k, char* out, u64 cap, u64* needed, char* err, u64 errlen) {
  try {
    *needed = put_text(knn_text(canonical_cloud(xyz, n), k), out, cap);
    return 0;
  } catch (const std::exception& e) {
    return report(e, err, errlen, 1);
  }
}

int oracle_higher(const double* xyz, u64 n, u64 K, char* out, u64 cap, u64* needed, char* err, u64 errlen) {
  try {
    *needed = put_text(higher_text(canonical_cloud(xyz, n), K), out, cap);
    return 0;
  } catch (const std::exception& e) {
    return report(e, err, errlen, 1);
  }
}

int oracle_pairs(const double* xyz, u64 n, u64 K, char* out, u64 cap, u64* needed, char* err, u64 errlen) {
  try {
    *needed = put_text(pairs_text(canonical_cloud(xyz, n), K), out, cap);
    return 0;
  } catch (const std::exception& e) {
    return report(e, err, errlen, 1);
  }
}

int oracle_emst_forest(const double* xyz, u64 n, char* out, u64 cap, u64* needed, char* err, u64 errlen) {
  try {
    *needed = put_text(emst_forest_text(canonical_cloud(xyz, n)), out, cap);
    return 0;
  } catch (const std::exception& e) {
    return report(e, err, errlen, 1);
  }
}


int oracle_classify(const double* xyz, u64 n, const uint32_t* supports, u64 count, uint32_t* out, char* err,
                    u64 errlen) {
  try {
    const Cloud c = canonical_cloud(xyz, n);
    classify_supports(c, fixed_cloud(c), supports, count, out);
    return 0;
  } catch (const std::exception& e) {
    return report(e, err, errlen, 1);
  }
}

int oracle_hierarchy(const double* xyz, u64 n, u64 K, char* out, u64 cap, u64* needed, char* err, u64 errlen) {
  try {
    *needed = put_text(hierarchy_text(canonical_cloud(xyz, n), K), out, cap);
    return 0;
  } catch (const std::exception& e) {
    return report(e, err, errlen, 1);
  }
}

}  // extern "C"
