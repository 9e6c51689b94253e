// Internal declarations shared by the sm_100a translation units of the
// MorseHGP3D product path.  Nothing here crosses the C ABI (include/ehgp.h).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <string>
#include <vector>

#include "ehgp.h"

#ifndef __CUDACC__
#error "ehgp_internal.cuh is CUDA-only"
#endif

#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ != 1000)
#error "this library is built for sm_100a only"
#endif

namespace ehgp {

// ---- device error word ---------------------------------------------------
// Kernels never trap: they OR a flag into the context's error word and skip
// the offending access; the host reads the word once per call.
enum DeviceErrorBit : uint32_t {
  kErrNonFinite = 1u << 0,
  kErrDuplicate = 1u << 1,
  kErrNumericRange = 1u << 2,
  kErrInternal = 1u << 3,
  kErrTimeout = 1u << 4,
  kErrCapacity = 1u << 5,
};

constexpr uint32_t kInvalid32 = 0xffffffffu;
constexpr int kMortonBitsPerAxis = 21;
constexpr uint64_t kMortonGrid = uint64_t{1} << kMortonBitsPerAxis;

// ---- binary64 total order -------------------------------------------------
// Same map as exact::binary64_total_order_key (include/morsehgp3d/exact/binary64.hpp:23-29)
// applied to canonical words (-0 already replaced by +0).
__host__ __device__ __forceinline__ uint64_t order_key(uint64_t bits) {
  return (bits >> 63) ? ~bits : (bits ^ (uint64_t{1} << 63));
}

// ---- radix sort of u32 indices by an indirect 64-bit key -----------------
struct RadixScratch {
  uint32_t* counts = nullptr;   // [256 * max_tiles]
  uint32_t* state = nullptr;    // per pass: [cur_in, trivial] pairs, kMaxPasses + 1 entries
  uint32_t max_tiles = 0;
};
constexpr int kRadixThreads = 256;
constexpr int kRadixItems = 4;
constexpr int kRadixTile = kRadixThreads * kRadixItems;
constexpr int kRadixMaxPasses = 32;
// State words: per pass (input buffer, trivial flag), then 256 digit totals.
constexpr int kRadixStateWords = 2 * (kRadixMaxPasses + 1) + 256;

// Key source for one sorting stage: key(v) = order_key(words[v]) when
// `order` is set, else words[v].
struct IndirectKey {
  const uint64_t* words;
  int order;
};

// Sorts vals (length n, ping-pong buffers vals0/vals1) stably by the keys of
// `stages` applied least-significant stage first, 8 bits per pass.  Returns
// nothing on the host: the buffer holding the result is recorded in
// scratch.state at index `passes` (0 -> vals0, 1 -> vals1).  The number of
// passes issued is returned.
int radix_sort_indirect(cudaStream_t stream, uint32_t n, uint32_t* vals0, uint32_t* vals1,
                        const IndirectKey* stages, const int* stage_bits, int stage_count,
                        RadixScratch& scratch, uint64_t* launches);

// Stable LSD sort of (keys0[i], vals0[i]) pairs by the low `bits` bits of the 64-bit keys,
// the keys moving with the indices (keys1 is scratch of the same size); result selection
// as for radix_sort_indirect.
int radix_sort_kv(cudaStream_t stream, uint32_t n, uint32_t* vals0, uint32_t* vals1, uint64_t* keys0,
                  uint64_t* keys1, int bits, RadixScratch& scratch, uint64_t* launches);

__device__ __forceinline__ const uint32_t* radix_result(const uint32_t* state, int passes,
                                                        const uint32_t* vals0, const uint32_t* vals1) {
  return state[2 * passes] ? vals1 : vals0;
}

// ---- context -----------------------------------------------------------------
struct LbvhBuffers {
  // input staging
  double* xyz_in = nullptr;        // [3*max_n] interleaved input (binary64)
  float* xyz_in_f32 = nullptr;     // [3*max_n] interleaved input (binary32)
  uint64_t* cin = nullptr;         // [3*max_n] canonical words by input index, axis-major
  // canonical cloud (by PointId)
  double* px = nullptr;            // [max_n]
  double* py = nullptr;
  double* pz = nullptr;
  uint32_t* source_index = nullptr;// [max_n]
  // Morton stage
  uint64_t* code = nullptr;        // [max_n] code by PointId
  uint32_t* vals0 = nullptr;       // [max_n]
  uint32_t* vals1 = nullptr;       // [max_n]
  uint32_t* leaf_pid = nullptr;    // [max_n] PointId at sorted position
  uint64_t* leaf_code = nullptr;   // [max_n]
  uint32_t* group_of = nullptr;    // [max_n] scan of heads
  uint32_t* block_sums = nullptr;  // scan partials
  uint32_t* gstart = nullptr;      // [max_n + 1]
  uint64_t* gcode = nullptr;       // [max_n]
  // top (unique-code) radix tree
  uint32_t* top_left = nullptr;    // [max_n] encoded child (bit31 = group leaf)
  uint32_t* top_right = nullptr;
  uint32_t* top_parent_int = nullptr;   // [max_n] parent of internal node i (or invalid)
  uint32_t* top_parent_grp = nullptr;   // [max_n] parent of group g
  uint32_t* grp_root_idx = nullptr;     // [max_n] postorder index of group subtree root
  uint32_t* grp_depth = nullptr;        // [max_n]
  // nodes in strict postorder (2n-1)
  uint32_t* n_left = nullptr;
  uint32_t* n_right = nullptr;
  uint32_t* n_begin = nullptr;
  uint32_t* n_end = nullptr;
  uint32_t* n_parent = nullptr;
  uint32_t* n_lo = nullptr;         // [3][2n] lower witnesses
  uint32_t* n_hi = nullptr;         // [3][2n] upper witnesses
  uint32_t* n_flag = nullptr;       // [2n] bottom-up arrival counters
  // frame
  uint64_t* frame = nullptr;        // [12]: lower bits[3], upper bits[3], lower wit[3], upper wit[3]
  unsigned long long* frame_partial = nullptr;  // per-block partials
  uint32_t* frame_done = nullptr;
  // results/export
  uint32_t* stats = nullptr;        // [8]: m, max_depth, collision groups, max collision, ...
  void* export_buf = nullptr;       // snapshot export (reference layout)
  uint64_t export_bytes = 0;
};

// Traversal node: outward-rounded binary32 box + children (32 bytes, two
// 16-byte loads).  Leaves: left == kInvalid32, right = PointId.
struct __align__(16) TNode {
  float lo[3];
  uint32_t left;
  float hi[3];
  uint32_t right;
};

// Buffers of the geometric stages (k-NN, Boruvka EMST, k=1 forest).
struct GeomBuffers {
  TNode* tnodes = nullptr;          // [2n]
  uint32_t* leaf_node = nullptr;    // [n] postorder index of the leaf at sorted position i
  int* scale = nullptr;             // [4]: S, max high bit, valid, spare
  // k-NN
  uint32_t* knn_ids = nullptr;      // [n * 11]
  uint32_t* knn_meta = nullptr;     // [n * 2]: strict count, shell count
  uint64_t* knn_cut = nullptr;      // [n * 4]: cutoff numerator limbs
  // Boruvka
  uint32_t* labels = nullptr;       // [n] frozen component label by PointId
  uint32_t* nlabel = nullptr;       // [2n] uniform node label or kInvalid32 (mixed)
  uint32_t* nflag = nullptr;        // [2n]
  uint32_t* best_q = nullptr;       // [n]
  double* best_d = nullptr;         // [n]
  unsigned long long* comp_dbits = nullptr;  // [n]
  uint32_t* comp_best = nullptr;    // [n]
  uint32_t* uf = nullptr;           // [n]
  uint32_t* counters = nullptr;     // [8]: components, minima, accepted
  uint32_t* minima = nullptr;       // [4 * 2n]: per round log (label, source, u, v)
  uint32_t* edge_u = nullptr;       // [n] accepted edges
  uint32_t* edge_v = nullptr;       // [n]
  uint64_t* key_u = nullptr;        // [n] sort keys
  uint64_t* key_v = nullptr;
  uint64_t* key_d = nullptr;
  uint32_t* order0 = nullptr;       // [n]
  uint32_t* order1 = nullptr;       // [n]
  uint64_t* edge_D = nullptr;       // [n * 4] exact squared lengths, sorted order
  uint32_t* sorted_u = nullptr;     // [n]
  uint32_t* sorted_v = nullptr;     // [n]
};

// Buffers of the pair-support stage.
struct PairBuffers {
  uint32_t* W = nullptr;            // [n * 32] witness lists (32 nearest, FP64 order)
  double* R2 = nullptr;             // [n] squared witness radius
  void* raw = nullptr;              // [capacity] 64-byte records, unordered
  void* sorted = nullptr;           // [capacity] records in (u, v) order
  uint64_t* key = nullptr;          // [capacity]
  uint32_t* order0 = nullptr;
  uint32_t* order1 = nullptr;
  uint64_t* levelD = nullptr;       // [capacity * 4] squared lengths of sorted records
  uint32_t* counters = nullptr;
  unsigned long long* stats = nullptr;  // [8] work counters of the enumeration kernel
  uint32_t* radix_counts = nullptr;
  uint32_t capacity = 0;
  uint32_t count = 0;               // records of the last run
  uint32_t K = 0;
  bool witness_ready = false;       // W / R2 computed for the resident cloud
  bool resident = false;            // records of the resident cloud for K are in `sorted`
};

// Buffers of the triple/quad-support stage.
struct HigherBuffers {
  uint32_t* nb = nullptr;           // [n * 512] neighbour lists
  uint32_t* nbc = nullptr;          // [n]
  uint32_t* cand = nullptr;         // [n * 256] candidate sets
  uint32_t* candc = nullptr;        // [n]
  double* gather_r2 = nullptr;      // [n] squared gather radius
  double* rcap = nullptr;           // [n] largest direction bound (radius the list must cover / 2)
  uint8_t* todo = nullptr;          // [n]
  float* dirs = nullptr;            // [642 * 3]
  double delta = 0;                 // covering angle of dirs
  double cos_lim = 0;               // cos(delta) + margin
  uint16_t* cells = nullptr;        // [6 * 32 * 32 * 8] cube-map cell -> nearby directions
  float* rho = nullptr;             // [n * 642] per-cone radius bounds
  void* raw = nullptr;              // [capacity] 64-byte records
  void* sorted = nullptr;
  uint64_t* khi = nullptr;
  uint64_t* klo = nullptr;
  uint32_t* order0 = nullptr;
  uint32_t* order1 = nullptr;
  uint32_t* counters = nullptr;
  unsigned long long* stats = nullptr;
  uint32_t* radix_counts = nullptr;
  uint32_t capacity = 0;
  uint32_t count = 0;
  uint32_t K = 0;
  double kernel_ms = 0;
  uint64_t stats_host[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  // owners whose certified neighbourhood holds more than the per-point list capacity
  uint32_t* big_ids = nullptr;      // [big_cap] owners on the large-neighbourhood path
  uint64_t* big_off = nullptr;      // [big_cap + 1] their offsets in the arena
  uint32_t* big_cnt = nullptr;      // [big_cap] neighbour counts
  uint32_t* big_arena = nullptr;    // [arena_cap] their neighbour ids
  uint64_t big_cap = 0, arena_cap = 0;
  uint64_t big_owners = 0, big_entries = 0;  // of the last call
  uint32_t list_cap = 1024;         // list entries before an owner takes the large path (<= the list capacity)
  // owners certified with more candidates than the per-point set holds
  uint32_t* large_ids = nullptr;    // [large_cap] owners in the order of their sets in cand_arena
  uint64_t* large_off = nullptr;    // [large_cap + 1] prefix offsets in cand_arena
  uint32_t* large_cnt = nullptr;    // [large_cap] candidate counts (launch order)
  uint64_t* large_dst = nullptr;    // [large_cap] destination offsets (launch order)
  uint32_t* cand_arena = nullptr;   // [carena_cap]
  uint32_t* adm_scratch = nullptr;  // [adm_words] face masks of the huge sets, one per block
  uint64_t large_cap = 0, carena_cap = 0, adm_words = 0;
  float* cand_dist = nullptr;       // [cdist_cap] distances of the sets sorted in the arena
  uint64_t cdist_cap = 0;
  uint32_t n_large = 0, n_huge = 0, n_mega = 0;  // owners with <= 1024, 4096, 16384 candidates (last call)
  uint32_t* split_off = nullptr;    // [split_cap] pair-chunk prefix of the owners with <= 1024 candidates
  uint32_t* split_adm = nullptr;    // [split_adm_words] their face masks, 1024 * 32 words each
  uint64_t split_cap = 0, split_adm_words = 0;
  uint32_t split_chunks = 0, split_chunks_huge = 0;  // blocks of one split launch per tier (last call)
  uint64_t large_entries = 0;
};

struct Ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  uint64_t max_points = 0;
  uint64_t device_bytes = 0;
  bool poisoned = false;
  std::mutex mutex;
  std::string last_error;
  double last_ms = 0.0;
  uint64_t last_launches = 0;
  uint64_t regrowths = 0;          // record buffers grown and enumerations re-run
  uint64_t pair_runs = 0, higher_runs = 0;  // support enumerations run on this context
  uint32_t* d_err = nullptr;       // device error word
  uint32_t* h_status = nullptr;    // pinned: [err, stats...]
  RadixScratch radix;
  LbvhBuffers lb;
  uint32_t* lb_top_split = nullptr;     // [max_n] split group of top internal node
  uint32_t* lb_top_gmin = nullptr;      // [max_n] first group of top internal node
  uint32_t* lb_top_gmax = nullptr;      // [max_n] last group of top internal node
  std::vector<void*> allocations;
  uint64_t built_n = 0;            // points of the resident index (0 = none)
  GeomBuffers gb;
  bool geom_ready = false;         // traversal nodes + scale built for built_n
  int scale_S = 0;                 // host copy of the cloud scale
  bool scale_valid = false;
  PairBuffers pb;
  HigherBuffers hb;
  // timing of the dominant kernel of the last stage, and of a whole step
  cudaEvent_t evk0 = nullptr, evk1 = nullptr, evs0 = nullptr, evs1 = nullptr;
  double kernel_ms = 0.0;
  uint64_t kernel_stats[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  uint32_t emst_rounds = 0;
  uint32_t emst_minima = 0;        // total per-round minima logged
  bool emst_ready = false;
  struct HierState* hier = nullptr;  // direct hierarchy (ehgp_hier.cu)
};

// Allocation helper: records the bytes on ctx.
cudaError_t ctx_alloc(Ctx& ctx, void** ptr, size_t bytes);
// Frees one allocation of ctx_alloc (bytes as allocated).
void ctx_free(Ctx& ctx, void* ptr, size_t bytes);

// LBVH stage (ehgp_lbvh.cu)
// Launch constants of the build that also size its scratch, shared by the context
// allocation (lbvh_alloc) and the allocation-free layout (ehgp_noalloc.cu).
constexpr int kLbvhFrameBlocks = 128;   // blocks of the exact-frame reduction (partials per axis)
constexpr int kLbvhScanThreads = 1024;  // elements per block of the collision-group scan
__host__ __device__ constexpr uint64_t lbvh_scan_block_sums(uint64_t n) {
  return (n + kLbvhScanThreads - 1) / kLbvhScanThreads + 1;
}
cudaError_t lbvh_alloc(Ctx& ctx);
// Runs the full device build on ctx.lb.xyz_in (input_kind 0 = f64, 1 = f32).
// Returns the number of kernel launches issued.
uint64_t lbvh_enqueue(Ctx& ctx, uint32_t n, int input_kind);
// Copies the requested snapshot parts to the host (synchronises).
cudaError_t lbvh_export(Ctx& ctx, uint32_t n, const ehgp_lbvh_out* out);

// Geometric stages (ehgp_geom.cu)
cudaError_t geom_alloc(Ctx& ctx);
// Traversal nodes, leaf map and cloud scale for the resident LBVH.
uint64_t geom_prepare(Ctx& ctx, uint32_t n);

// Pair supports (ehgp_pairs.cu)
cudaError_t pairs_alloc(Ctx& ctx);
// (Re)allocates the pair record buffers for `capacity` records.
cudaError_t pairs_records_alloc(Ctx& ctx, uint64_t capacity);
int pairs_run(Ctx& ctx, uint32_t K, uint32_t* out_count);

// Triple/quad supports (ehgp_higher.cu)
cudaError_t higher_alloc(Ctx& ctx);
// (Re)allocates the triple/quad record buffers for `capacity` records.
cudaError_t higher_records_alloc(Ctx& ctx, uint64_t capacity);
// Record capacity to allocate when a stage counted `needed` records: a margin above the
// count, within the 32-bit record indices of the stages.
inline uint64_t grown_capacity(uint64_t needed) {
  const uint64_t c = needed + needed / 8 + 4096;
  return c < 0xffff0000ull ? c : 0xffff0000ull;
}
int higher_run(Ctx& ctx, uint32_t K, uint32_t* out_count);

// Direct Morse hierarchy (ehgp_hier.cu)
int hier_run(Ctx& ctx, uint32_t K);
void hier_free(Ctx& ctx);

}  // namespace ehgp

extern "C" {
struct ehgp_ctx : ehgp::Ctx {};
}

// Shared status helpers of the C ABI (ehgp_context.cu).
namespace ehgp {
int abi_fail(Ctx* ctx, int status, const char* msg);
int abi_cuda_fail(Ctx* ctx, cudaError_t e, const char* where);
int abi_device_status(Ctx* ctx, uint32_t err);
}  // namespace ehgp
