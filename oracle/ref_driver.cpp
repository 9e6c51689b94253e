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

// The budgeted protocol of the CPU baseline: canonical cloud + LBVH, then
// build_exact_pair_support_stream (include/morsehgp3d/hierarchy/pair_support_stream.hpp:415)
// with maximum_work_unit_count = work_units (the other limits unlimited).  stats[0] status
// (0 complete, 1 budget exhausted), [1] work units used, [2] resolved pairs, [3] total
// pairs, [4] events, [5] relevant extra-shell diagnostics; seconds[0] cloud + LBVH,
// seconds[1] the stream.
int ref_pairs_budget(const double* xyz, uint64_t n, uint64_t K, uint64_t work_units, uint64_t* stats,
                     double* seconds, char* err, uint64_t errlen) {
  try {
    using namespace morsehgp3d;
    const auto pts = points_from(xyz, n);
    const auto t0 = std::chrono::steady_clock::now();
    const CanonicalPointCloud cloud = CanonicalPointCloud::rejecting_duplicates(pts);
    const MortonLbvhIndex index = MortonLbvhIndex::build(cloud);
    const auto t1 = std::chrono::steady_clock::now();
    auto budget = unlimited_pair_budget();
    budget.maximum_work_unit_count = work_units;
    const auto res = hierarchy::build_exact_pair_support_stream(index, cloud, K, budget);
    const auto t2 = std::chrono::steady_clock::now();
    seconds[0] = std::chrono::duration<double>(t1 - t0).count();
    seconds[1] = std::chrono::duration<double>(t2 - t1).count();
    stats[0] = res.status == hierarchy::ExactPairSupportStreamStatus::complete ? 0 : 1;
    stats[1] = res.audit.work_unit_count;
    stats[2] = res.audit.resolved_pair_count;
    stats[3] = res.audit.total_pair_count;
    stats[4] = res.events.size();
    stats[5] = res.relevant_extra_shell_diagnostics.size();
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

#include "morsehgp3d/hierarchy/direct_morse_event_journal.hpp"
#include "morsehgp3d/hierarchy/direct_morse_forest_journal.hpp"
#include "morsehgp3d/hierarchy/direct_saddle_arm_seed_journal.hpp"
#include "morsehgp3d/hierarchy/direct_support_terminal.hpp"

namespace {

std::string level_text(const morsehgp3d::exact::ExactLevel& l) {
  return l.numerator_string() + " " + l.denominator_string();
}

std::string opt_text(const std::optional<std::size_t>& v) { return v ? std::to_string(*v) : std::string("-"); }
std::string opt_text(const std::optional<std::uint64_t>& v, int) { return v ? std::to_string(*v) : std::string("-"); }

template <class Key>
std::string key_text(const Key& k) {
  std::string t = std::to_string(k.point_count);
  for (std::size_t i = 0; i < k.point_count; ++i) t += " " + std::to_string(k.point_ids[i]);
  return t;
}

}  // namespace

extern "C" {

// The reference's direct hierarchy chain run to completion:
//   build_exact_pair_support_stream + build_exact_higher_support_stream
//   -> build_exact_direct_support_terminal_facade (direct_support_terminal.hpp:196)
//   -> build_exact_direct_morse_event_journal (direct_morse_event_journal.hpp:165)
//   -> build_exact_direct_saddle_arm_seed_journal (direct_saddle_arm_seed_journal.hpp:169)
//   -> build_exact_direct_morse_forest_journal (direct_morse_forest_journal.hpp:388).
// Text lines (one record each, in the reference's own arena order):
//   F idx size ids.. | interior.. | rank exterior num den birth_order saddle_order   (facade events)
//   X count                                                                       (relevant extra-shell diagnostics)
//   J batch order num den role_off role_cnt births saddles                         (journal batches)
//   Q role batch projection role(0 birth, 1 saddle)                                (role records)
//   Y family event projection role batch order num den arm_off arm_cnt             (saddle families)
//   Z seed family removed                                                          (arm seeds)
//   N node order num den kind child_off child_cnt birth group                      (forest nodes)
//   C child..                                                                      (child arena)
//   B birth proj batch order handle one_node | key                                 (birth records)
//   A binding seed family carrier prior | key                                      (arm-root bindings)
//   S saddle family event batch arm_off arm_cnt carriers latent prior group         (saddle records)
//   G group batch s_off s_cnt frozen latent prior c_off c_cnt created result kind  (atomic groups)
//   T batch src order num den b_off b_cnt s_off s_cnt g_off g_cnt pre_c pre_r post_c post_r
//   R root order handle node                                                       (final roots)
//   D journal_decision seed_decision forest_decision
int ref_hierarchy(const double* xyz, uint64_t n, uint64_t K, char* out, uint64_t cap, uint64_t* needed,
                  double* seconds, char* err, uint64_t errlen) {
  try {
    using namespace morsehgp3d;
    using namespace morsehgp3d::hierarchy;
    const auto pts = points_from(xyz, n);
    const CanonicalPointCloud cloud = CanonicalPointCloud::rejecting_duplicates(pts);
    const MortonLbvhIndex index = MortonLbvhIndex::build(cloud);
    const std::size_t big = std::size_t{1} << 40;
    ExactDirectSupportTerminalBudget tb;
    tb.pair = unlimited_pair_budget();
    tb.higher.maximum_work_unit_count = big;
    tb.higher.maximum_frontier_entry_count = big;
    tb.higher.maximum_auxiliary_frontier_entry_count = big;
    tb.higher.maximum_emitted_record_count = big;
    tb.higher.maximum_emitted_point_id_reference_count = big;
    tb.higher.maximum_prune_receipt_count = big;
    tb.higher.maximum_global_closed_ball_query_count = big;
    tb.higher.maximum_point_classification_count = big;
    const auto t0 = std::chrono::steady_clock::now();
    const auto pair = build_exact_pair_support_stream(index, cloud, K, tb.pair);
    const auto higher = build_exact_higher_support_stream(index, cloud, K, tb.higher);
    const auto t1 = std::chrono::steady_clock::now();
    const auto facade = build_exact_direct_support_terminal_facade(index, cloud, K, tb, pair, higher);
    const auto journal = build_exact_direct_morse_event_journal(cloud, facade);
    const ExactDirectSaddleArmSeedBudget sb{big, big, big, big};
    const auto seeds = build_exact_direct_saddle_arm_seed_journal(cloud, facade, journal, sb);
    ExactDirectMorseForestBudget fb;
    const std::size_t mid = std::size_t{1} << 22;
    fb.maximum_source_role_scan_count = big;
    fb.maximum_source_batch_scan_count = big;
    fb.maximum_source_family_scan_count = big;
    fb.maximum_source_arm_seed_scan_count = big;
    fb.maximum_birth_record_count = big;
    fb.maximum_arm_root_binding_count = big;
    fb.maximum_saddle_record_count = big;
    fb.maximum_atomic_group_count = big;
    fb.maximum_child_reference_count = big;
    fb.maximum_batch_record_count = big;
    fb.maximum_node_count = big;
    fb.maximum_final_root_count = big;
    fb.maximum_batch_distinct_arm_count = mid;
    fb.maximum_logical_output_entry_count = big;
    fb.maximum_aggregate_closure_node_count = big;
    fb.maximum_aggregate_closure_step_call_count = big;
    // the locator sizes its probing table from the binding caps: keep them modest
    const std::size_t loc = std::size_t{1} << 16, slots = std::size_t{1} << 19;
    fb.locator_budget = {loc, loc, 16 * loc, loc, loc, loc, loc, loc, 16 * loc, slots, slots};
    const ExactDirectSparseFacetDescentStepBudget step{
        ExactDirectSparsePositiveFacetProbeBudget{mid, mid},
        spatial::ExactLbvhTopKBudget{mid, mid, mid, mid, mid, mid, mid},
        ExactDirectSparsePositiveFacetProbeBudget{mid, mid}};
    fb.closure_budget = {direct_sparse_facet_descent_closure_maximum_seed_count,
                         direct_sparse_facet_descent_closure_maximum_node_count,
                         direct_sparse_facet_descent_closure_maximum_step_call_count,
                         direct_sparse_facet_descent_closure_maximum_memo_slot_count, step};
    fb.quotient_budget = {mid, mid, mid, mid, mid};
    ExactDirectMorseForestConfig fc;
    fc.locator_config.external_authority_id = 0x10F0;
    const auto forest = build_exact_direct_morse_forest_journal(index, cloud, facade, journal, sb, seeds, fb, fc,
                                                                 spatial::LbvhTraversalOrder::near_first);
    const auto t2 = std::chrono::steady_clock::now();
    if (seconds) {
      seconds[0] = std::chrono::duration<double>(t1 - t0).count();
      seconds[1] = std::chrono::duration<double>(t2 - t1).count();
    }
    std::string s;
    for (const auto& e : facade.events) {
      s += "F " + std::to_string(e.event_index) + " " + std::to_string((int)e.support_size);
      for (int i = 0; i < e.support_size; ++i) s += " " + std::to_string(e.support_ids[i]);
      s += " |" + ids_text(e.interior_ids) + " | " + std::to_string(e.closed_rank) + " " +
           std::to_string(e.exterior_count) + " " + level_text(e.squared_level) + " " + opt_text(e.birth_order) + " " +
           opt_text(e.saddle_order) + "\n";
    }
    s += "X " + std::to_string(facade.relevant_extra_shell_diagnostics.size()) + "\n";
    for (const auto& b : journal.batches)
      s += "J " + std::to_string(b.batch_index) + " " + std::to_string(b.order) + " " + level_text(b.squared_level) +
           " " + std::to_string(b.role_record_offset) + " " + std::to_string(b.role_record_count) + " " +
           std::to_string(b.birth_role_count) + " " + std::to_string(b.saddle_role_count) + "\n";
    for (const auto& r : journal.role_records)
      s += "Q " + std::to_string(r.role_record_index) + " " + std::to_string(r.batch_index) + " " +
           std::to_string(r.event_projection_index) + " " + std::to_string((int)r.role) + "\n";
    for (const auto& f : seeds.families)
      s += "Y " + std::to_string(f.family_index) + " " + std::to_string(f.source_event_index) + " " +
           std::to_string(f.journal_event_projection_index) + " " + std::to_string(f.journal_role_record_index) + " " +
           std::to_string(f.journal_batch_index) + " " + std::to_string(f.order) + " " +
           level_text(f.critical_squared_level) + " " + std::to_string(f.arm_seed_offset) + " " +
           std::to_string(f.arm_seed_count) + "\n";
    for (const auto& a : seeds.arm_seeds)
      s += "Z " + std::to_string(a.arm_seed_index) + " " + std::to_string(a.family_index) + " " +
           std::to_string(a.removed_support_point_id) + "\n";
    for (const auto& nd : forest.nodes)
      s += "N " + std::to_string(nd.node_id) + " " + std::to_string(nd.order) + " " + level_text(nd.squared_level) +
           " " + std::to_string((int)nd.kind) + " " + std::to_string(nd.child_offset) + " " +
           std::to_string(nd.child_count) + " " + opt_text(nd.birth_record_index) + " " +
           opt_text(nd.atomic_group_index) + "\n";
    {
      std::string c = "C";
      for (auto id : forest.child_node_ids) c += " " + std::to_string(id);
      s += c + "\n";
    }
    for (const auto& b : forest.birth_records)
      s += "B " + std::to_string(b.birth_record_index) + " " + std::to_string(b.source_event_projection_index) + " " +
           std::to_string(b.source_journal_batch_index) + " " + std::to_string(b.order) + " " +
           std::to_string(b.component_handle) + " " + opt_text(b.order_one_birth_node_id, 0) + " | " +
           key_text(b.facet_key) + "\n";
    for (const auto& a : forest.arm_root_bindings)
      s += "A " + std::to_string(a.binding_index) + " " + std::to_string(a.source_arm_seed_index) + " " +
           std::to_string(a.source_family_index) + " " + std::to_string(a.frozen_carrier_component_handle) + " " +
           opt_text(a.prior_reduced_root_node_id, 0) + " | " + key_text(a.strict_arm_key) + "\n";
    for (const auto& r : forest.saddle_records)
      s += "S " + std::to_string(r.saddle_record_index) + " " + std::to_string(r.source_family_index) + " " +
           std::to_string(r.source_event_index) + " " + std::to_string(r.source_journal_batch_index) + " " +
           std::to_string(r.arm_binding_offset) + " " + std::to_string(r.arm_binding_count) + " " +
           std::to_string(r.distinct_frozen_carrier_count) + " " + std::to_string(r.distinct_latent_carrier_count) +
           " " + std::to_string(r.distinct_prior_reduced_root_count) + " " + std::to_string(r.atomic_group_index) +
           "\n";
    for (const auto& g : forest.atomic_groups)
      s += "G " + std::to_string(g.atomic_group_index) + " " + std::to_string(g.batch_index) + " " +
           std::to_string(g.saddle_record_offset) + " " + std::to_string(g.saddle_record_count) + " " +
           std::to_string(g.frozen_carrier_count) + " " + std::to_string(g.latent_carrier_count) + " " +
           std::to_string(g.prior_reduced_root_count) + " " + std::to_string(g.child_offset) + " " +
           std::to_string(g.child_count) + " " + opt_text(g.created_node_id, 0) + " " +
           std::to_string(g.resulting_root_node_id) + " " + std::to_string((int)g.kind) + "\n";
    for (const auto& b : forest.batches)
      s += "T " + std::to_string(b.batch_index) + " " + std::to_string(b.source_journal_batch_index) + " " +
           std::to_string(b.order) + " " + level_text(b.squared_level) + " " + std::to_string(b.birth_record_offset) +
           " " + std::to_string(b.birth_record_count) + " " + std::to_string(b.saddle_record_offset) + " " +
           std::to_string(b.saddle_record_count) + " " + std::to_string(b.atomic_group_offset) + " " +
           std::to_string(b.atomic_group_count) + " " + std::to_string(b.strict_pre_batch_carrier_count) + " " +
           std::to_string(b.strict_pre_batch_reduced_root_count) + " " +
           std::to_string(b.closed_post_batch_carrier_count) + " " +
           std::to_string(b.closed_post_batch_reduced_root_count) + "\n";
    for (const auto& r : forest.final_roots)
      s += "R " + std::to_string(r.final_root_index) + " " + std::to_string(r.order) + " " +
           std::to_string(r.component_handle) + " " + std::to_string(r.root_node_id) + "\n";
    s += "D " + std::to_string((int)journal.decision) + " " + std::to_string((int)seeds.decision) + " " +
         std::to_string((int)forest.decision) + "\n";
    *needed = put_text(s, out, cap);
    return 0;
  } catch (const std::exception& e) {
    return report(e, err, errlen, 1);
  }
}

}  // extern "C"
