// Test-oracle driver over the reference's own CPU code (Ludwig-H/E-HGP,
// morsehgp3d/src/cpu), compiled unmodified from its source tree against the
// project-written Boost shim in oracle/boost_shim.  Built by oracle/Makefile
// into oracle/_ref/libehgp_ref.so.  Test infrastructure only: it is the
// checker for the CUDA path and the timed reference CPU baseline, never part
// of the product path.
//
// Entry points are extern "C" with flat arrays so that Python tests can call
// them through ctypes.  Every function returns 0 on success, or a nonzero code
// with the reference's exception text copied into `err` (capacity errlen).
#include "morsehgp3d/exact/point.hpp"
#include "morsehgp3d/spatial/lbvh.hpp"
#include "morsehgp3d/spatial/point_cloud.hpp"

#include <chrono>
#include <cstdint>
#include <cstring>
#include <exception>
#include <span>
#include <stdexcept>
#include <string>
#include <vector>

namespace morsehgp3d::gpu {
// MortonLbvhIndex names this class a friend (include/morsehgp3d/spatial/lbvh.hpp:421);
// its real definition lives in the GPU sources, which are not linked here, so
// the oracle uses the name to read the private node array for comparison.
class SpatialLbvhContext {
 public:
  static void export_nodes(const spatial::MortonLbvhIndex& index, uint64_t* out) {
    for (std::size_t i = 0; i < index.nodes_.size(); ++i) {
      const auto& nd = index.nodes_[i];
      uint64_t* r = out + 10 * i;
      for (int a = 0; a < 3; ++a) {
        r[a] = nd.lower_point_ids[a];
        r[3 + a] = nd.upper_point_ids[a];
      }
      const uint64_t invalid = ~uint64_t{0};
      r[6] = nd.left_child == static_cast<std::size_t>(-1) ? invalid : nd.left_child;
      r[7] = nd.right_child == static_cast<std::size_t>(-1) ? invalid : nd.right_child;
      r[8] = nd.leaf_begin;
      r[9] = nd.leaf_end;
    }
  }
  static uint64_t root(const spatial::MortonLbvhIndex& index) { return index.root_index_; }
};
}  // namespace morsehgp3d::gpu

namespace {

using morsehgp3d::exact::CertifiedPoint3;
using morsehgp3d::spatial::CanonicalPointCloud;
using morsehgp3d::spatial::MortonLbvhIndex;

int report(const std::exception& e, char* err, uint64_t errlen, int code) {
  if (err && errlen) {
    std::strncpy(err, e.what(), errlen - 1);
    err[errlen - 1] = 0;
  }
  return code;
}

std::vector<CertifiedPoint3> points_from(const double* xyz, uint64_t n) {
  std::vector<CertifiedPoint3> pts;
  pts.reserve(n);
  for (uint64_t i = 0; i < n; ++i) pts.push_back(CertifiedPoint3::from_binary64(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]));
  return pts;
}

}  // namespace

extern "C" {

// CanonicalPointCloud::rejecting_duplicates + MortonLbvhIndex::build.
// Outputs (any may be null): source_index[n], leaves[2n] (code, id),
// nodes[10(2n-1)] in the MortonLbvhSnapshotNode field order, counters[5],
// root_aabb[6], root[1].  seconds[2]: canonicalisation and build wall time.
int ref_lbvh_build(const double* xyz, uint64_t n, uint64_t* source_index, uint64_t* leaves, uint64_t* nodes,
                   uint64_t* counters, uint64_t* root_aabb, uint64_t* root, double* seconds, char* err,
                   uint64_t errlen) {
  try {
    const auto pts = points_from(xyz, n);
    const auto t0 = std::chrono::steady_clock::now();
    const CanonicalPointCloud cloud = CanonicalPointCloud::rejecting_duplicates(pts);
    const auto t1 = std::chrono::steady_clock::now();
    const MortonLbvhIndex index = MortonLbvhIndex::build(cloud);
    const auto t2 = std::chrono::steady_clock::now();
    if (seconds) {
      seconds[0] = std::chrono::duration<double>(t1 - t0).count();
      seconds[1] = std::chrono::duration<double>(t2 - t1).count();
    }
    if (source_index)
      for (uint64_t p = 0; p < n; ++p) source_index[p] = cloud.source_index(p);
    if (leaves) {
      const auto lv = index.leaves();
      for (uint64_t i = 0; i < n; ++i) {
        leaves[2 * i] = lv[i].morton_code;
        leaves[2 * i + 1] = lv[i].point_id;
      }
    }
    if (nodes) morsehgp3d::gpu::SpatialLbvhContext::export_nodes(index, nodes);
    if (counters) {
      const auto& c = index.build_counters();
      counters[0] = c.point_count;
      counters[1] = c.node_count;
      counters[2] = c.maximum_depth;
      counters[3] = c.morton_collision_group_count;
      counters[4] = c.maximum_morton_collision_size;
    }
    if (root_aabb) {
      const auto& bb = index.root_aabb();
      for (int a = 0; a < 3; ++a) {
        root_aabb[a] = bb.lower_binary64_bits[a];
        root_aabb[3 + a] = bb.upper_binary64_bits[a];
      }
    }
    if (root) *root = morsehgp3d::gpu::SpatialLbvhContext::root(index);
    return 0;
  } catch (const std::invalid_argument& e) {
    return report(e, err, errlen, 1);
  } catch (const std::exception& e) {
    return report(e, err, errlen, 2);
  }
}

// MortonLbvhIndex::import_certified_snapshot (src/cpu/spatial/lbvh.cpp:551-829):
// the reference's own exhaustive validator of a device-built snapshot.  Returns
// 0 when the reference accepts every leaf, node, split, witness and counter.
int ref_lbvh_certify(const double* xyz, uint64_t n, const uint64_t* leaves, const uint64_t* nodes,
                     const uint64_t* counters, const uint64_t* root_aabb, uint64_t root, char* err,
                     uint64_t errlen) {
  try {
    const auto pts = points_from(xyz, n);
    const CanonicalPointCloud cloud = CanonicalPointCloud::rejecting_duplicates(pts);
    morsehgp3d::spatial::MortonLbvhSnapshot snap;
    snap.point_count = n;
    snap.root_node_index = root;
    for (int a = 0; a < 3; ++a) {
      snap.root_aabb.lower_binary64_bits[a] = root_aabb[a];
      snap.root_aabb.upper_binary64_bits[a] = root_aabb[3 + a];
    }
    snap.proposed_counters = {counters[0], counters[1], counters[2], counters[3], counters[4]};
    snap.leaves.resize(n);
    for (uint64_t i = 0; i < n; ++i) snap.leaves[i] = {leaves[2 * i], leaves[2 * i + 1]};
    snap.nodes.resize(2 * n - 1);
    for (uint64_t i = 0; i < 2 * n - 1; ++i) {
      auto& nd = snap.nodes[i];
      const uint64_t* r = nodes + 10 * i;
      for (int a = 0; a < 3; ++a) {
        nd.lower_point_ids[a] = r[a];
        nd.upper_point_ids[a] = r[3 + a];
      }
      nd.left_child = r[6];
      nd.right_child = r[7];
      nd.leaf_begin = r[8];
      nd.leaf_end = r[9];
    }
    const MortonLbvhIndex index = MortonLbvhIndex::import_certified_snapshot(cloud, snap);
    return index.ready() ? 0 : 3;
  } catch (const std::exception& e) {
    return report(e, err, errlen, 1);
  }
}

// Text-blob outputs below: one record per line, fields separated by spaces.
// Returns the number of bytes needed when `cap` is too small (nothing written).
static uint64_t put_text(const std::string& s, char* buf, uint64_t cap) {
  if (s.size() + 1 > cap) return s.size() + 1;
  std::memcpy(buf, s.c_str(), s.size() + 1);
  return 0;
}

// lbvh_top_k for every point p with exclusions {p}
// (include/morsehgp3d/spatial/lbvh.hpp:424).  Line p:
// "<strict ids (d,id) order> | <shell ids> | num den".
int ref_knn(const double* xyz, uint64_t n, uint64_t k, char* out, uint64_t cap, uint64_t* needed, double* seconds,
            char* err, uint64_t errlen) {
  try {
    using namespace morsehgp3d;
    const auto pts = points_from(xyz, n);
    const CanonicalPointCloud cloud = CanonicalPointCloud::rejecting_duplicates(pts);
    const MortonLbvhIndex index = MortonLbvhIndex::build(cloud);
    std::string s;
    const auto t0 = std::chrono::steady_clock::now();
    for (uint64_t p = 0; p < n; ++p) {
      const std::vector<spatial::PointId> ex{p};
      const auto exclusions = spatial::ExclusionSet::from_ids(ex, cloud, 9);
      const auto part = spatial::lbvh_top_k(index, cloud, cloud.point(p).exact(), k, exclusions);
      for (const auto& nb : part.strict_below()) s += std::to_string(nb.point_id) + " ";
      s += "|";
      for (const auto id : part.cutoff_shell_ids()) s += " " + std::to_string(id);
      s += " | " + part.cutoff_squared_distance().numerator_string() + " " +
           part.cutoff_squared_distance().denominator_string() + "\n";
    }
    if (seconds) seconds[0] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    *needed = put_text(s, out, cap);
    return 0;
  } catch (const std::exception& e) {
    return report(e, err, errlen, 1);
  }
}

}  // extern "C"

#include "morsehgp3d/hierarchy/boruvka.hpp"
#include "morsehgp3d/hierarchy/k1_forest.hpp"
#include "morsehgp3d/hierarchy/pair_support_stream.hpp"
#include "morsehgp3d/hierarchy/higher_support_stream.hpp"

namespace {

std::string center_text(const morsehgp3d::exact::ExactCenter3& c) {
  return c.numerator(0).str() + " " + c.numerator(1).str() + " " + c.numerator(2).str() + " " +
         c.denominator().str();
}

std::string ids_text(const std::vector<morsehgp3d::spatial::PointId>& ids) {
  std::string s;
  for (const auto id : ids) s += " " + std::to_string(id);
  return s;
}

morsehgp3d::hierarchy::ExactPairSupportStreamBudget unlimited_pair_budget() {
  morsehgp3d::hierarchy::ExactPairSupportStreamBudget b;
  const std::size_t big = std::size_t{1} << 62;
  b.maximum_work_unit_count = big;
  b.maximum_frontier_entry_count = big;
  b.maximum_auxiliary_frontier_entry_count = big;
  b.maximum_emitted_record_count = big;
  b.maximum_emitted_point_id_reference_count = big;
  b.maximum_global_closed_ball_query_count = big;
  b.maximum_point_classification_count = big;
  return b;
}

}  // namespace

extern "C" {

// build_exact_higher_support_stream (include/morsehgp3d/hierarchy/higher_support_stream.hpp:544)
// with an unlimited budget.  Lines in the stream's canonical (size, ids) order:
// "H size a b c [d] closed_rank exterior lnum lden cx cy cz cden | interior..."  (events)
// "G size a b c [d] shell witness min_rank observed exterior lnum lden cx cy cz cden | interior..."
// then "S complete|budget_exhausted".
int ref_higher(const double* xyz, uint64_t n, uint64_t K, char* out, uint64_t cap, uint64_t* needed, double* seconds,
               char* err, uint64_t errlen) {
  try {
    using namespace morsehgp3d;
    const auto pts = points_from(xyz, n);
    const CanonicalPointCloud cloud = CanonicalPointCloud::rejecting_duplicates(pts);
    const MortonLbvhIndex index = MortonLbvhIndex::build(cloud);
    hierarchy::ExactHigherSupportStreamBudget b;
    const std::size_t big = std::size_t{1} << 62;
    b.maximum_work_unit_count = big;
    b.maximum_frontier_entry_count = big;
    b.maximum_auxiliary_frontier_entry_count = big;
    b.maximum_emitted_record_count = big;
    b.maximum_emitted_point_id_reference_count = big;
    b.maximum_prune_receipt_count = big;
    b.maximum_global_closed_ball_query_count = big;
    b.maximum_point_classification_count = big;
    const auto t0 = std::chrono::steady_clock::now();
    const auto res = hierarchy::build_exact_higher_support_stream(index, cloud, K, b);
    if (seconds) seconds[0] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::string s;
    auto ids = [](const auto& r) {
      std::string t = std::to_string((int)r.support_size);
      for (int i = 0; i < r.support_size; ++i) t += " " + std::to_string(r.support_ids[i]);
      return t;
    };
    for (const auto& e : res.events)
      s += "H " + ids(e) + " " + std::to_string(e.closed_rank) + " " + std::to_string(e.exterior_count) + " " +
           e.squared_level.numerator_string() + " " + e.squared_level.denominator_string() + " " +
           center_text(e.center) + " |" + ids_text(e.interior_ids) + "\n";
    for (const auto& d : res.relevant_extra_shell_diagnostics)
      s += "G " + ids(d) + " " + std::to_string(d.shell_count) + " " + std::to_string(d.canonical_extra_shell_witness_id) +
           " " + std::to_string(d.minimum_possible_closed_rank) + " " + std::to_string(d.observed_closed_rank) + " " +
           std::to_string(d.exterior_count) + " " + d.squared_level.numerator_string() + " " +
           d.squared_level.denominator_string() + " " + center_text(d.center) + " |" + ids_text(d.interior_ids) +
           "\n";
    s += std::string("S ") +
         (res.status == hierarchy::ExactHigherSupportStreamStatus::complete ? "complete" : "budget_exhausted") + "\n";
    *needed = put_text(s, out, cap);
    return 0;
  } catch (const std::exception& e) {
    return report(e, err, errlen, 1);
  }
}

// build_exact_pair_support_stream (include/morsehgp3d/hierarchy/pair_support_stream.hpp:415)
// with an unlimited budget.  Lines, in the stream's canonical (u, v) order:
// "P u v closed_rank exterior lnum lden cx cy cz cden | interior..."  (events)
// "D u v shell witness min_rank observed exterior lnum lden cx cy cz cden | interior..."
// (relevant extra-shell diagnostics), then "S complete|budget_exhausted".
int ref_pairs(const double* xyz, uint64_t n, uint64_t K, char* out, uint64_t cap, uint64_t* needed, double* seconds,
              char* err, uint64_t errlen) {
  try {
    using namespace morsehgp3d;
    const auto pts = points_from(xyz, n);
    const CanonicalPointCloud cloud = CanonicalPointCloud::rejecting_duplicates(pts);
    const MortonLbvhIndex index = MortonLbvhIndex::build(cloud);
    const auto t0 = std::chrono::steady_clock::now();
    const auto res = hierarchy::build_exact_pair_support_stream(index, cloud, K, unlimited_pair_budget());
    if (seconds) seconds[0] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::string s;
    for (const auto& e : res.events)
      s += "P " + std::to_string(e.support_ids[0]) + " " + std::to_string(e.support_ids[1]) + " " +
           std::to_string(e.closed_rank) + " " + std::to_string(e.exterior_count) + " " +
           e.squared_level.numerator_string() + " " + e.squared_level.denominator_string() + " " +
           center_text(e.center) + " |" + ids_text(e.interior_ids) + "\n";
    for (const auto& d : res.relevant_extra_shell_diagnostics)
      s += "D " + std::to_string(d.support_ids[0]) + " " + std::to_string(d.support_ids[1]) + " " +
           std::to_string(d.shell_count) + " " + std::to_string(d.canonical_extra_shell_witness_id) + " " +
           std::to_string(d.minimum_possible_closed_rank) + " " + std::to_string(d.observed_closed_rank) + " " +
           std::to_string(d.exterior_count) + " " + d.squared_level.numerator_string() + " " +
           d.squared_level.denominator_string() + " " + center_text(d.center) + " |" + ids_text(d.interior_ids) +
           "\n";
    s += std::string("S ") +
         (res.status == hierarchy::ExactPairSupportStreamStatus::complete ? "complete" : "budget_exhausted") + "\n";
    *needed = put_text(s, out, cap);
    return 0;
  } catch (const std::exception& e) {
    return report(e, err, errlen, 1);
  }
}

// build_exact_lbvh_boruvka (include/morsehgp3d/hierarchy/boruvka.hpp:130) and
// build_compact_k1_forest on its edges (include/morsehgp3d/hierarchy/k1_forest.hpp:108).
// Lines: "E u v num den" (EMST, canonical order), "M round label source u v num den"
// (component minima), "A round u v" (accepted), "L num den" (forest levels),
// "N id level_index child_offset child_count min_point coverage" (merge nodes),
// "C child..." (child arena), "B level_index edge_off edge_cnt node_off node_cnt pre post",
// "R root".  seconds[0] = Boruvka, seconds[1] = forest.
int ref_emst_forest(const double* xyz, uint64_t n, char* out, uint64_t cap, uint64_t* needed, double* seconds,
                    char* err, uint64_t errlen) {
  try {
    using namespace morsehgp3d;
    const auto pts = points_from(xyz, n);
    const CanonicalPointCloud cloud = CanonicalPointCloud::rejecting_duplicates(pts);
    const MortonLbvhIndex index = MortonLbvhIndex::build(cloud);
    const auto t0 = std::chrono::steady_clock::now();
    const auto res = hierarchy::build_exact_lbvh_boruvka(index, cloud);
    const auto t1 = std::chrono::steady_clock::now();
    const auto forest = hierarchy::build_compact_k1_forest(n, res.emst_edges);
    const auto t2 = std::chrono::steady_clock::now();
    if (seconds) {
      seconds[0] = std::chrono::duration<double>(t1 - t0).count();
      seconds[1] = std::chrono::duration<double>(t2 - t1).count();
    }
    std::string s;
    for (const auto& e : res.emst_edges)
      s += "E " + std::to_string(e.u) + " " + std::to_string(e.v) + " " + e.squared_length.numerator_string() + " " +
           e.squared_length.denominator_string() + "\n";
    for (const auto& r : res.rounds) {
      for (const auto& m : r.component_minima)
        s += "M " + std::to_string(r.round_index) + " " + std::to_string(m.component_label) + " " +
             std::to_string(m.source_point_id) + " " + std::to_string(m.outgoing_edge.u) + " " +
             std::to_string(m.outgoing_edge.v) + " " + m.outgoing_edge.squared_length.numerator_string() + " " +
             m.outgoing_edge.squared_length.denominator_string() + "\n";
      for (const auto& a : r.accepted_edges)
        s += "A " + std::to_string(r.round_index) + " " + std::to_string(a.u) + " " + std::to_string(a.v) + "\n";
    }
    for (const auto& l : forest.levels) s += "L " + l.numerator_string() + " " + l.denominator_string() + "\n";
    for (const auto& nd : forest.merge_nodes)
      s += "N " + std::to_string(nd.id) + " " + std::to_string(nd.level_index) + " " +
           std::to_string(nd.child_offset) + " " + std::to_string(nd.child_count) + " " +
           std::to_string(nd.minimum_point_id) + " " + std::to_string(nd.coverage_size) + "\n";
    s += "C";
    for (const auto c : forest.child_ids) s += " " + std::to_string(c);
    s += "\n";
    for (const auto& b : forest.equal_level_batches)
      s += "B " + std::to_string(b.level_index) + " " + std::to_string(b.selected_edge_offset) + " " +
           std::to_string(b.selected_edge_count) + " " + std::to_string(b.merge_node_offset) + " " +
           std::to_string(b.merge_node_count) + " " + std::to_string(b.pre_batch_component_count) + " " +
           std::to_string(b.post_batch_component_count) + "\n";
    s += "R " + std::to_string(forest.root_node_id) + "\n";
    *needed = put_text(s, out, cap);
    return 0;
  } catch (const std::exception& e) {
    return report(e, err, errlen, 1);
  }
}

}  // extern "C"
