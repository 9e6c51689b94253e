// Compact k=1 merge forest from the device EMST (host code of the library).
//
// Reference: hierarchy::build_compact_k1_forest
// (include/morsehgp3d/hierarchy/k1_forest.hpp:108, src/cpu/hierarchy/k1_forest.cpp:665-845):
//  * tree edges in (squared length, u, v) order, split into batches of equal
//    exact length; the batch level is squared length / 4;
//  * components are frozen before each batch; each connected group of >= 2
//    pre-batch components joined by the batch becomes ONE merge node (a
//    multifusion when it has >= 3 children, never a chain of binary merges);
//  * merge nodes of a batch are ordered by the least PointId of their group,
//    children by their least PointId; leaves are the PointIds 0..n-1 and merge
//    node ids continue from n.
//
// The sweep is sequential in the batch order by definition; it runs on the
// host over the device's sorted edges and exact lengths (one 40 B/edge copy),
// where a union-find with least-index roots costs ~10 ns per edge.
#include "ehgp_internal.cuh"

#include <algorithm>
#include <cstring>
#include <vector>

namespace {

struct LeastRootDsu {
  std::vector<uint32_t> p;
  uint64_t count;
  explicit LeastRootDsu(uint64_t n) : p(n), count(n) {
    for (uint64_t i = 0; i < n; ++i) p[i] = (uint32_t)i;
  }
  uint32_t find(uint32_t x) {
    while (p[x] != x) {
      p[x] = p[p[x]];
      x = p[x];
    }
    return x;
  }
  bool unite(uint32_t a, uint32_t b) {
    a = find(a);
    b = find(b);
    if (a == b) return false;
    if (a > b) std::swap(a, b);
    p[b] = a;
    --count;
    return true;
  }
};

}  // namespace

extern "C" {

int ehgp_k1_forest(ehgp_ctx* ctx, const ehgp_k1_forest_out* out) {
  if (!ctx || !out) return EHGP_ERR_INVALID_ARGUMENT;
  if (!ctx->emst_ready) return ehgp::abi_fail(ctx, EHGP_ERR_NOT_BUILT, "ehgp_k1_forest needs ehgp_emst first");
  std::lock_guard<std::mutex> lock(ctx->mutex);
  const uint64_t n = ctx->built_n, m = n - 1;
  std::vector<uint32_t> u(m), v(m);
  std::vector<uint64_t> D(4 * m);
  cudaError_t e = cudaSuccess;
  if (m) {
    e = cudaMemcpy(u.data(), ctx->gb.sorted_u, m * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(v.data(), ctx->gb.sorted_v, m * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(D.data(), ctx->gb.edge_D, 32 * m, cudaMemcpyDeviceToHost);
  }
  if (e != cudaSuccess) return ehgp::abi_cuda_fail(ctx, e, "k=1 forest copy");
  auto same_len = [&](uint64_t a, uint64_t b) { return std::memcmp(&D[4 * a], &D[4 * b], 32) == 0; };
  LeastRootDsu comp(n);
  std::vector<uint64_t> node_of(n), cover;
  for (uint64_t i = 0; i < n; ++i) node_of[i] = i;
  uint64_t levels = 0, nodes = 0, children = 0, batches = 0;
  std::vector<uint32_t> roots;
  std::vector<std::vector<uint32_t>> groups;
  for (uint64_t b = 0; b < m;) {
    uint64_t end = b + 1;
    while (end < m && same_len(b, end)) ++end;
    const uint64_t level = levels++;
    if (out->level_num) std::memcpy(out->level_num + 4 * level, &D[4 * b], 32);
    const uint64_t pre = comp.count, node_off = nodes;
    if (end == b + 1) {  // a batch of one edge: one binary merge node
      uint32_t r0 = comp.find(u[b]), r1 = comp.find(v[b]);
      if (r0 == r1) return ehgp::abi_fail(ctx, EHGP_ERR_CUDA, "an EMST edge closes a cycle");
      if (r0 > r1) std::swap(r0, r1);
      const uint64_t id = n + nodes, c0 = node_of[r0], c1 = node_of[r1];
      const uint64_t cov = (c0 < n ? 1 : cover[c0 - n]) + (c1 < n ? 1 : cover[c1 - n]);
      if (out->child_ids) {
        out->child_ids[children] = c0;
        out->child_ids[children + 1] = c1;
      }
      if (out->nodes) {
        uint64_t* rec = out->nodes + 6 * nodes;
        rec[0] = id; rec[1] = level; rec[2] = children; rec[3] = 2; rec[4] = r0; rec[5] = cov;
      }
      children += 2;
      cover.push_back(cov);
      ++nodes;
      comp.unite(r0, r1);
      node_of[r0] = id;
      if (out->batches) {
        uint64_t* rec = out->batches + 7 * batches;
        rec[0] = level; rec[1] = b; rec[2] = 1; rec[3] = node_off; rec[4] = 1; rec[5] = pre; rec[6] = comp.count;
      }
      ++batches;
      b = end;
      continue;
    }
    roots.clear();
    for (uint64_t i = b; i < end; ++i) {
      roots.push_back(comp.find(u[i]));
      roots.push_back(comp.find(v[i]));
    }
    std::sort(roots.begin(), roots.end());
    roots.erase(std::unique(roots.begin(), roots.end()), roots.end());
    LeastRootDsu local(roots.size());
    auto pos = [&](uint32_t r) { return (uint32_t)(std::lower_bound(roots.begin(), roots.end(), r) - roots.begin()); };
    for (uint64_t i = b; i < end; ++i)
      if (!local.unite(pos(comp.find(u[i])), pos(comp.find(v[i]))))
        return ehgp::abi_fail(ctx, EHGP_ERR_CUDA, "an equality batch of the EMST contains a cycle");
    groups.assign(roots.size(), {});
    for (uint32_t li = 0; li < roots.size(); ++li) groups[local.find(li)].push_back(roots[li]);
    std::vector<std::pair<uint32_t, uint64_t>> pending;  // (least root, node id)
    for (const auto& g : groups) {
      if (g.empty()) continue;
      const uint64_t id = n + nodes;
      uint64_t cov = 0;
      for (uint32_t r : g) {
        const uint64_t child = node_of[r];
        if (out->child_ids) out->child_ids[children++] = child;
        else ++children;
        cov += child < n ? 1 : cover[child - n];
      }
      if (out->nodes) {
        uint64_t* rec = out->nodes + 6 * nodes;
        rec[0] = id;
        rec[1] = level;
        rec[2] = children - g.size();
        rec[3] = g.size();
        rec[4] = g.front();
        rec[5] = cov;
      }
      cover.push_back(cov);
      pending.emplace_back(g.front(), id);
      ++nodes;
    }
    for (uint64_t i = b; i < end; ++i) comp.unite(u[i], v[i]);
    for (const auto& [r, id] : pending) node_of[comp.find(r)] = id;
    if (out->batches) {
      uint64_t* rec = out->batches + 7 * batches;
      rec[0] = level;
      rec[1] = b;
      rec[2] = end - b;
      rec[3] = node_off;
      rec[4] = nodes - node_off;
      rec[5] = pre;
      rec[6] = comp.count;
    }
    ++batches;
    b = end;
  }
  if (comp.count != 1) return ehgp::abi_fail(ctx, EHGP_ERR_CUDA, "the EMST did not yield one root");
  if (out->counts) {
    out->counts[0] = levels;
    out->counts[1] = nodes;
    out->counts[2] = children;
    out->counts[3] = batches;
  }
  if (out->root_node_id) *out->root_node_id = node_of[comp.find(0)];
  return EHGP_OK;
}

}  // extern "C"
