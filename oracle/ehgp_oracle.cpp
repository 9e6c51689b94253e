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
#include <stdexcept>
#include <string>
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
  std::string ev[2], dg[2];
  std::vector<u64> interior;
  auto visit = [&](const u64* ids, int size) {
    if (smax < (u64)size) return;
    SupportGeo g = analyze(c, f, ids, size);
    if (g.status != 0) return;
    analyze_fp(c, g);
    const u64 cap = smax - size;
    interior.clear();
    u64 shell = size, extra = ~u64{0};
    for (u64 w = 0; w < n; ++w) {
      bool sup = false;
      for (int i = 0; i < size; ++i) sup |= (w == ids[i]);
      if (sup) continue;
      const int sd = higher_side(c, f, g, w);
      if (sd < 0) {
        interior.push_back(w);
        if (interior.size() > cap) return;
      } else if (sd == 0) {
        ++shell;
        extra = std::min(extra, w);
      }
    }
    const u64 I = interior.size();
    std::string head = std::to_string(size);
    for (int i = 0; i < size; ++i) head += " " + std::to_string(ids[i]);
    std::string idt;
    for (u64 w : interior) idt += " " + std::to_string(w);
    const std::string sph = sphere_text(f, g);
    if (shell == (u64)size)
      ev[size - 3] += "H " + head + " " + std::to_string(I + size) + " " + std::to_string(n - I - size) + " " + sph +
                      " |" + idt + "\n";
    else
      dg[size - 3] += "G " + head + " " + std::to_string(shell) + " " + std::to_string(extra) + " " +
                      std::to_string(I + size) + " " + std::to_string(I + shell) + " " + std::to_string(n - I - shell) +
                      " " + sph + " |" + idt + "\n";
  };
  u64 ids[4];
  for (ids[0] = 0; ids[0] < n; ++ids[0])
    for (ids[1] = ids[0] + 1; ids[1] < n; ++ids[1])
      for (ids[2] = ids[1] + 1; ids[2] < n; ++ids[2]) {
        visit(ids, 3);
        for (ids[3] = ids[2] + 1; ids[3] < n; ++ids[3]) visit(ids, 4);
      }
  // the stream orders records by (support size, ids): triples before quads
  return ev[0] + ev[1] + dg[0] + dg[1] + "S complete\n";
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

}  // extern "C"
