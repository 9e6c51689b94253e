/*
 * ehgp.h — C ABI of the B200 (sm_100a) MorseHGP3D product path.
 *
 * Plain C: fixed-width integers, plain pointers and sizes, integer status
 * codes.  No C++ exceptions and no torch types cross this boundary.
 *
 * Every entry point below replaces one interface of the reference
 * (Ludwig-H/E-HGP, directory morsehgp3d/); the citation is given beside it.
 * Record layouts that a reference caller reads byte-for-byte keep the
 * reference's layout and carry a static size check in the implementation.
 *
 * Threading: one context owns one CUDA stream and its device buffers; calls
 * on one context are serialised by the context.  All calls are synchronous:
 * when an entry point returns, its host outputs are complete.
 *
 * Errors: a status other than EHGP_OK is returned and a message is kept in
 * the context (ehgp_last_error).  A CUDA failure poisons the context (every
 * later call returns EHGP_ERR_POISONED), mirroring the reference's
 * poisoned-context rule (src/cuda/phase14_morton_lbvh_build_internal.hpp:99-132).
 */
#ifndef EHGP_H_
#define EHGP_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
typedef enum ehgp_status {
  EHGP_OK = 0,
  EHGP_ERR_INVALID_ARGUMENT = 1, /* null pointer, n = 0, non-finite coordinate  */
  EHGP_ERR_DUPLICATE_POINT = 2,  /* two input points are geometrically equal    */
  EHGP_ERR_CAPACITY = 3,         /* n above the context's max_points            */
  EHGP_ERR_OUT_OF_MEMORY = 4,    /* device allocation refused                   */
  EHGP_ERR_TIMEOUT = 5,          /* a bounded device wait ran out               */
  EHGP_ERR_DEGENERATE = 6,       /* relevant extra-shell diagnostic (journal refuses) */
  EHGP_ERR_NUMERIC_RANGE = 7,    /* a fixed-width exact evaluation would overflow */
  EHGP_ERR_CUDA = 8,             /* CUDA runtime error; context is poisoned     */
  EHGP_ERR_POISONED = 9,         /* an earlier CUDA error poisoned the context  */
  EHGP_ERR_NOT_BUILT = 10        /* stage needs an earlier stage's device state  */
} ehgp_status;

/* ---- limits and context -------------------------------------------------- */
typedef struct ehgp_limits {
  uint64_t max_points;   /* largest cloud one call accepts                    */
  double hbm_fraction;   /* admission ceiling as a fraction of HBM (0.8)      */
} ehgp_limits;

typedef struct ehgp_ctx ehgp_ctx;

/* Replaces gpu::MortonLbvhBuildContext::MortonLbvhBuildContext(max_n)
 * (include/morsehgp3d/gpu/morton_lbvh_build.hpp:185-189): creates a context on
 * `device` whose buffers hold clouds of up to limits->max_points points. */
int ehgp_ctx_create(int device, const ehgp_limits* limits, ehgp_ctx** out_ctx);
/* Replaces ~MortonLbvhBuildContext (morton_lbvh_build.hpp:190). */
int ehgp_ctx_destroy(ehgp_ctx* ctx);
/* Message of the last failed call on ctx (empty string when none). */
const char* ehgp_last_error(const ehgp_ctx* ctx);
/* Static name of a status code. */
const char* ehgp_status_string(int status);
/* Device bytes owned by the context (resident buffers). */
uint64_t ehgp_ctx_device_bytes(const ehgp_ctx* ctx);

/* Support records are produced count -> allocate -> emit, as the reference's
 * stream contract asks (no truncation; the budgeted streams of
 * include/morsehgp3d/hierarchy/pair_support_stream.hpp:421-470 resume instead of
 * dropping records): an enumeration counts every record and writes the ones that
 * fit; when the count is above the buffer, the buffer grows to it and the
 * enumeration runs once more.  ehgp_ctx_reserve sets the record capacity of the
 * pair (stage 0) or triple/quad (stage 1) buffers up front, so that a caller who
 * knows its clouds avoids the second pass (the resident records of that stage
 * are dropped); ehgp_ctx_regrowths counts the second passes so far.  No
 * counterpart in the reference. */
int ehgp_ctx_reserve(ehgp_ctx* ctx, uint32_t stage, uint64_t records);
uint64_t ehgp_ctx_regrowths(const ehgp_ctx* ctx);

/* [0] device bytes, [1] record-buffer regrowths, [2] pair enumerations and [3]
 * triple/quad enumerations run on this context so far.  No reference counterpart. */
int ehgp_ctx_counters(const ehgp_ctx* ctx, uint64_t* out, uint32_t count);

/* Checkpoint and resume of a request after its support stages, in place of the
 * reference's chunk -> checkpoint -> commit support streams
 * (include/morsehgp3d/hierarchy/pair_support_stream.hpp:421-470) and its planned
 * preemption manifest (docs/GPU_G4_ARCHITECTURE.md:239-252).  save writes the
 * resident cloud (binary64, PointId order), K and the pair and triple/quad records
 * for K (enumerating them first when they are not resident) to `path` with a
 * 64-byte header and an FNV-1a checksum; load checks the file, rebuilds the cloud
 * on ctx (the same PointIds) and makes the records resident, so a following
 * ehgp_hierarchy(ctx, K) resumes without enumerating the supports again.  A file
 * that fails its checks is refused with EHGP_ERR_INVALID_ARGUMENT and leaves the
 * context as it was. */
int ehgp_checkpoint_save(ehgp_ctx* ctx, uint32_t K, const char* path);
int ehgp_checkpoint_load(ehgp_ctx* ctx, const char* path, uint32_t* K);

/* Tuning knobs of later calls on ctx; results never depend on them (no
 * counterpart in the reference).
 *   EHGP_TUNE_HIGHER_LIST: neighbour-list entries (1..1024, default 1024) that a
 *     triple/quad owner may hold before its certificate moves to the
 *     large-neighbourhood path (arena lists of any length). */
enum { EHGP_TUNE_HIGHER_LIST = 1 };
int ehgp_tune(ehgp_ctx* ctx, uint32_t knob, uint64_t value);

/* ---- LBVH snapshot records (reference layout) ---------------------------- */
/* Same fields, order and sizes as spatial::MortonLbvhSnapshotLeaf,
 * MortonLbvhSnapshotNode and MortonLbvhSnapshotCounters
 * (include/morsehgp3d/spatial/lbvh.hpp:44-50, 62-78, 80-89): 16, 80, 40 bytes. */
typedef struct ehgp_lbvh_leaf {
  uint64_t morton_code;
  uint64_t point_id;
} ehgp_lbvh_leaf;

#define EHGP_INVALID_NODE_INDEX (~(uint64_t)0)

typedef struct ehgp_lbvh_node {
  uint64_t lower_point_ids[3];
  uint64_t upper_point_ids[3];
  uint64_t left_child;  /* EHGP_INVALID_NODE_INDEX for a leaf */
  uint64_t right_child; /* EHGP_INVALID_NODE_INDEX for a leaf */
  uint64_t leaf_begin;
  uint64_t leaf_end;
} ehgp_lbvh_node;

typedef struct ehgp_lbvh_counters {
  uint64_t point_count;
  uint64_t node_count;
  uint64_t maximum_depth;
  uint64_t morton_collision_group_count;
  uint64_t maximum_morton_collision_size;
} ehgp_lbvh_counters;

/* Host-side outputs of ehgp_lbvh_build.  Any pointer may be NULL to skip that
 * output; the device-resident index is built either way. */
typedef struct ehgp_lbvh_out {
  uint64_t* source_index;        /* [n]: input position of PointId p          */
  ehgp_lbvh_leaf* leaves;        /* [n]: (Morton code, PointId), sorted       */
  ehgp_lbvh_node* nodes;         /* [2n-1]: strict left/right postorder        */
  ehgp_lbvh_counters* counters;  /* [1]                                       */
  uint64_t* root_aabb_bits;      /* [6]: lower xyz, upper xyz binary64 words  */
  uint64_t* root_node_index;     /* [1]: always 2n-2                          */
} ehgp_lbvh_out;

/* Canonical point cloud + exact Morton LBVH, fused on the device.
 *
 * Replaces, as one call:
 *   spatial::CanonicalPointCloud::rejecting_duplicates
 *     (include/morsehgp3d/spatial/point_cloud.hpp:31, src/cpu/spatial/point_cloud.cpp:40-94),
 *   spatial::MortonLbvhIndex::build (src/cpu/spatial/lbvh.cpp:484-549), and
 *   gpu::MortonLbvhBuildContext::build (include/morsehgp3d/gpu/morton_lbvh_build.hpp:196)
 *     with its launcher seam build_phase14_morton_lbvh_snapshot_on_gpu
 *     (src/cuda/phase14_morton_lbvh_build_internal.hpp:150-156).
 *
 * xyz: host array of n points, interleaved x,y,z binary64 values.
 * PointIds are the ranks of the points in lexicographic binary64 total order
 * (-0 canonicalised to +0).  Results are bit-identical to the reference's
 * MortonLbvhSnapshot.  Errors: EHGP_ERR_INVALID_ARGUMENT (n = 0, non-finite
 * coordinate), EHGP_ERR_DUPLICATE_POINT, EHGP_ERR_CAPACITY. */
int ehgp_lbvh_build(ehgp_ctx* ctx, const double* xyz, uint64_t n, const ehgp_lbvh_out* out);

/* Same as ehgp_lbvh_build for binary32 input, widened exactly to binary64. */
int ehgp_lbvh_build_f32(ehgp_ctx* ctx, const float* xyz, uint64_t n, const ehgp_lbvh_out* out);

/* Same as ehgp_lbvh_build, with xyz already resident in device memory
 * (interleaved binary64, 3n values); no host->device copy of the points. */
int ehgp_lbvh_build_device(ehgp_ctx* ctx, const double* d_xyz, uint64_t n, const ehgp_lbvh_out* out);

/* ---- exact geometry of the resident cloud --------------------------------- */
/* Exact fixed-point scale of the resident cloud: every coordinate x is the
 * integer x * 2^S, and every squared distance below is an integer numerator
 * N with value N / 2^(2S).  *valid = 0 when some |x| * 2^S >= 2^124; the exact
 * stages then return EHGP_ERR_NUMERIC_RANGE. */
int ehgp_cloud_scale(ehgp_ctx* ctx, int32_t* scale_exponent, int32_t* valid);

typedef struct ehgp_knn_out {
  uint32_t* ids;        /* [n*k]: per PointId p, its top-k canonical choice in (squared distance, PointId) order */
  uint32_t* meta;       /* [n*2]: (points strictly below the cutoff, points exactly at the cutoff) */
  uint64_t* cutoff_num; /* [n*4]: k-th squared distance numerator, 64-bit limbs, little endian, scale 2^-2S */
} ehgp_knn_out;

/* Exact k nearest other points (k <= 11) of every point of the resident cloud.
 * Replaces spatial::lbvh_top_k(index, cloud, query = point p, k, exclusions = {p})
 * (include/morsehgp3d/spatial/lbvh.hpp:424-430) for all p at once: the cutoff is
 * the k-th smallest exact squared distance, `meta` gives the strict count and
 * the COMPLETE equality-shell size, `ids` the canonical choice (strict points,
 * then the least shell PointIds; TopKPartition, src/cpu/spatial/brute_force.cpp:319-384). */
int ehgp_knn(ehgp_ctx* ctx, uint32_t k, const ehgp_knn_out* out);

typedef struct ehgp_emst_out {
  uint32_t* u;                  /* [n-1]: u < v, ordered by (squared length, u, v) */
  uint32_t* v;                  /* [n-1] */
  uint64_t* squared_length_num; /* [(n-1)*4]: exact numerators at scale 2^-2S (merge level = 1/4 of it) */
  uint32_t* rounds;             /* [1]: Boruvka rounds */
  uint32_t* minima;             /* [minima_capacity*4]: (round, component label, source PointId, target PointId) */
  uint64_t minima_capacity;
  uint64_t* minima_count;       /* [1] */
} ehgp_emst_out;

/* Exact Euclidean minimum spanning tree by LBVH Boruvka with frozen
 * least-PointId labels and kappa = (squared length, u, v) minima.  Replaces
 * hierarchy::build_exact_lbvh_boruvka (include/morsehgp3d/hierarchy/boruvka.hpp:130)
 * and gpu::build_gpu_proposed_cpu_exact_k1_boruvka
 * (include/morsehgp3d/gpu/k1_boruvka.hpp:1004): decisions are exact on the
 * device, no CPU replay. */
int ehgp_emst(ehgp_ctx* ctx, const ehgp_emst_out* out);

typedef struct ehgp_k1_forest_out {
  uint64_t* level_num;    /* [(n-1)*4]: batch squared lengths (numerators, scale 2^-2S); level = length / 4 */
  uint64_t* nodes;        /* [(n-1)*6]: id, level_index, child_offset, child_count, minimum_point_id, coverage_size */
  uint64_t* child_ids;    /* [2(n-1)]: child arena (leaves are PointIds, merge nodes n, n+1, ...) */
  uint64_t* batches;      /* [(n-1)*7]: level_index, edge_offset, edge_count, node_offset, node_count, pre, post */
  uint64_t* counts;       /* [4]: levels, merge nodes, child references, batches */
  uint64_t* root_node_id; /* [1] */
} ehgp_k1_forest_out;

/* Compact k=1 merge forest of the last ehgp_emst result: equal-length batches
 * frozen before each batch, one (multi)fusion node per connected group.
 * Replaces hierarchy::build_compact_k1_forest(point_count, edges)
 * (include/morsehgp3d/hierarchy/k1_forest.hpp:108) with the same arenas. */
int ehgp_k1_forest(ehgp_ctx* ctx, const ehgp_k1_forest_out* out);

/* ---- pair critical-sphere supports ------------------------------------------ */
/* One relevant pair support (64 bytes).  The sphere is the diametral sphere of
 * (u, v): centre (u + v) / 2, squared level |u - v|^2 / 4.  shell_count == 2
 * is an ExactPairSupportEvent (closed rank interior_count + 2); a larger shell
 * is an ExactPairSupportExtraShellDiagnostic
 * (include/morsehgp3d/hierarchy/pair_support_stream.hpp:256-289). */
typedef struct ehgp_pair_record {
  uint32_t u, v;                /* support PointIds, u < v */
  uint32_t interior_count;      /* strict interior points (<= s_max - 2) */
  uint32_t shell_count;         /* complete exact shell, supports included */
  uint32_t extra_shell_witness; /* least extra shell PointId, or 0xffffffff */
  uint32_t interior_ids[9];     /* ascending; unused slots 0xffffffff */
  uint32_t reserved[2];
} ehgp_pair_record;

typedef struct ehgp_pairs_out {
  ehgp_pair_record* records; /* [capacity], (u, v) order */
  uint64_t* level_num;       /* [capacity*4]: |u-v|^2 numerators at scale 2^-2S (level = 1/4 of it) */
  uint64_t capacity;
  uint64_t* count;           /* [1] */
} ehgp_pairs_out;

/* Every relevant pair support of the resident cloud for maximum order K <= 10
 * (s_max = min(min(K, n) + 1, n)).  Replaces
 * hierarchy::build_exact_pair_support_stream(index, cloud, K, budget)
 * (include/morsehgp3d/hierarchy/pair_support_stream.hpp:415) run to completion,
 * and its GPU proposal seam propose_pair_support_phi_on_gpu
 * (src/cuda/phase9_pair_support_phi_internal.hpp:110-114): decisions are exact
 * on the device.  records == NULL only counts. */
int ehgp_pairs(ehgp_ctx* ctx, uint32_t K, const ehgp_pairs_out* out);

/* ---- triple and quad critical-sphere supports ------------------------------ */
/* One relevant minimal 3- or 4-point support (64 bytes): an
 * ExactHigherSupportEvent when shell_count == size, else an
 * ExactHigherSupportExtraShellDiagnostic
 * (include/morsehgp3d/hierarchy/higher_support_stream.hpp:283-316).  The sphere
 * is the circumsphere of the support (for a triangle, the one centred in its
 * plane); its exact centre and level follow from the support ids. */
typedef struct ehgp_higher_record {
  uint32_t size;                /* 3 or 4 */
  uint32_t ids[4];              /* ascending; unused slot 0 */
  uint32_t interior_count;      /* <= s_max - size */
  uint32_t shell_count;         /* complete exact shell, support included */
  uint32_t extra_shell_witness; /* least extra shell PointId, or 0xffffffff */
  uint32_t interior_ids[8];     /* ascending; unused slots 0xffffffff */
} ehgp_higher_record;

typedef struct ehgp_higher_out {
  ehgp_higher_record* records; /* [capacity], (size, ids) order */
  uint64_t capacity;
  uint64_t* count;             /* [1] */
} ehgp_higher_out;

/* Every relevant minimal triple and quad support of the resident cloud for
 * maximum order K <= 10.  Replaces hierarchy::build_exact_higher_support_stream
 * (include/morsehgp3d/hierarchy/higher_support_stream.hpp:544) run to
 * completion.  records == NULL only counts. */
int ehgp_higher(ehgp_ctx* ctx, uint32_t K, const ehgp_higher_out* out);

/* CUDA-event time of the last triple/quad enumeration kernels and their work
 * counters: [0] candidate supports tested, [1] closed-ball classifications,
 * [2] records, [3] candidate-set entries, [4] support candidates (ids above
 * the owner), [5] minimal supports, [6] minimal supports dropped by the cone
 * bounds, [7] faces admitted; [8] owners whose certified neighbourhood
 * exceeded the 1024-entry list and took the large-neighbourhood path (count ->
 * allocate -> write), [9] entries of their lists, [10]-[12] owners whose
 * candidate set exceeded 256 and was staged as a large (<= 1024), huge
 * (<= 4096) or mega (<= 16384) set, [13] entries of those sets.  count <= 14. */
int ehgp_higher_stats(const ehgp_ctx* ctx, double* kernel_ms, uint64_t* stats, uint32_t count);

/* One exact predicate on PointIds of the resident cloud, evaluated on the device by
 * the enumeration's own helpers (FP64 with the uniform error bounds, then the
 * fixed-width exact integers); out[0] the result, out[1] 1 when an FP64 filter
 * decided it.  Stands in for the reference's predicate replay tool
 * (morsehgp3d/src/tools/predicate_replay.cpp) on the predicates this path uses:
 *   EHGP_PRED_SUPPORT_SIDE   ids = support (1-4) then the query: -1 strictly
 *                            inside, 0 on, +1 outside its support sphere
 *                            (support_sphere_side; a triangle's circle is
 *                            centred in its plane);
 *   EHGP_PRED_SUPPORT_STATUS ids = support (1-4): 0 minimal, 1 boundary reduced,
 *                            2 exterior centre, 3 affinely dependent
 *                            (circumcenter_support_analysis, support_status);
 *   EHGP_PRED_LEVEL_CMP      ids = left size, left ids, right ids: sign of
 *                            level(left) - level(right) (compare_support_levels);
 *   EHGP_PRED_DISTANCE_CMP   ids = a, p, q: sign of |p - a|^2 - |q - a|^2
 *                            (compare_squared_distances).
 * EHGP_ERR_NUMERIC_RANGE when the cloud leaves the exact fixed-point range. */
enum { EHGP_PRED_SUPPORT_SIDE = 1, EHGP_PRED_SUPPORT_STATUS = 2, EHGP_PRED_LEVEL_CMP = 3, EHGP_PRED_DISTANCE_CMP = 4 };
int ehgp_predicate_eval(ehgp_ctx* ctx, uint32_t predicate, const uint32_t* ids, uint32_t count, int32_t* out);

/* Allocation-free LBVH build.  No counterpart in the reference: it exists for
 * callers that may not call cudaMalloc (a host framework that owns all device
 * memory through its own pool, or a latency-critical caller that cannot
 * accept cudaMalloc's device-wide synchronisation), and so cannot create a
 * context.  Same inputs, outputs and results as ehgp_lbvh_build, with host
 * `xyz` and host outputs, run on `stream` (a cudaStream_t; NULL = the legacy
 * default stream) of the current device.  All scratch lives in one fixed
 * __device__ array of ehgp_lbvh_noalloc_scratch_bytes() bytes that every GPU
 * loading this library holds until exit; n above
 * ehgp_lbvh_noalloc_max_points() (16384) returns EHGP_ERR_CAPACITY.  The
 * first call on a device looks the array up (cudaGetSymbolAddress).  Every
 * call synchronises `stream` and copies status words back, so it must never
 * be called on a stream that is being captured into a CUDA graph; such a
 * stream is refused with EHGP_ERR_INVALID_ARGUMENT.  Calls share the array:
 * calls whose GPU work overlaps race and must not be issued. */
int ehgp_lbvh_build_noalloc(const double* xyz, uint64_t n, const ehgp_lbvh_out* out, void* stream);
uint64_t ehgp_lbvh_noalloc_max_points(void);
uint64_t ehgp_lbvh_noalloc_scratch_bytes(void);

/* Device time (ms) of the last call's kernels, measured with CUDA events on
 * the context's stream, and the number of kernel launches it issued. */
int ehgp_last_timing(const ehgp_ctx* ctx, double* device_ms, uint64_t* kernel_launches);

/* Step timing on the context's stream: ehgp_step_begin records a CUDA event,
 * ehgp_step_end records a second one, waits for it and returns the elapsed
 * device-timeline milliseconds (host stages in between included). */
int ehgp_step_begin(ehgp_ctx* ctx);
int ehgp_step_end(ehgp_ctx* ctx, double* elapsed_ms);

/* CUDA-event time of the dominant kernel of the last pair stage (the pair
 * enumeration) and its work counters: [0] LBVH node visits, [1] witness-list
 * classifications, [2] exact ball queries, [3] ball-query node visits,
 * [4] emitted records. */
int ehgp_kernel_stats(const ehgp_ctx* ctx, double* kernel_ms, uint64_t* stats, uint32_t count);

/* ---- direct Morse hierarchy ------------------------------------------------
 * One call runs the reference's direct chain on the resident cloud (pair and
 * triple/quad supports first when they are not resident for K):
 *   terminal facade  build_exact_direct_support_terminal_facade
 *                    (morsehgp3d/include/morsehgp3d/hierarchy/direct_support_terminal.hpp:196)
 *   event journal    build_exact_direct_morse_event_journal (direct_morse_event_journal.hpp:165)
 *   arm seeds        build_exact_direct_saddle_arm_seed_journal (direct_saddle_arm_seed_journal.hpp:169)
 *   forest journal   build_exact_direct_morse_forest_journal (direct_morse_forest_journal.hpp:388),
 *                    with its strict-arm descent (direct_sparse_facet_descent_step.hpp:239,
 *                    direct_sparse_facet_descent_closure.hpp:477) and frozen-root quotient
 *                    (direct_frozen_root_quotient.hpp:176).
 * Records keep the reference's arena order and index meaning; optional ids
 * are UINT32_MAX when absent.  Exact levels are referenced by `level_event`,
 * the facade index of an event at that level (UINT32_MAX: level 0), and are
 * materialised by ehgp_event_level.  A relevant extra-shell diagnostic stops
 * the chain after the facade (decision EHGP_ERR_DEGENERATE), as the
 * reference's no_journal_relevant_extra_shell_diagnostics does. */
typedef struct ehgp_hier_counts {
  uint64_t events, diagnostics;                 /* facade */
  uint64_t journal_batches, role_records;       /* event journal */
  uint64_t families, arm_seeds;                 /* arm seeds */
  uint64_t birth_records, nodes, children, arm_bindings, saddle_records, atomic_groups, final_roots;
  uint32_t decision;                            /* EHGP_OK when the forest journal is complete */
  uint32_t k_eff;
  uint64_t vertical_assignments;                /* vertical maps, orders 2..k_eff */
} ehgp_hier_counts;

int ehgp_hierarchy(ehgp_ctx* ctx, uint32_t K, ehgp_hier_counts* counts);

/* Facade event (64 bytes), in facade order (exact level, closed rank,
 * interior ids, support ids). */
typedef struct ehgp_event_record {
  uint32_t support_size;
  uint32_t support_ids[4];
  uint32_t interior_count;
  uint32_t closed_rank;
  uint32_t interior_ids[9];
} ehgp_event_record;

typedef struct ehgp_journal_batch {  /* ExactDirectMorseH0Batch */
  uint32_t order, level_event;
  uint32_t role_offset, role_count, birth_roles, saddle_roles;
} ehgp_journal_batch;

typedef struct ehgp_role_record {    /* ExactDirectMorseH0RoleRecord */
  uint32_t batch, projection, role;  /* projection: PointId (< n) or n + event; role 0 birth, 1 saddle */
} ehgp_role_record;

typedef struct ehgp_family_record {  /* ExactDirectSaddleArmFamilyRecord */
  uint32_t event, projection, role_record, batch, order, arm_offset, arm_count;
} ehgp_family_record;

typedef struct ehgp_forest_node {    /* ExactDirectMorseForestNode */
  uint32_t order, level_event, kind; /* kind: 0 order-one birth, 1 reduced birth, 2 multifusion */
  uint32_t child_offset, child_count, birth_record, atomic_group;
} ehgp_forest_node;

typedef struct ehgp_forest_birth {   /* ExactDirectMorseForestBirthRecord */
  uint32_t projection, batch, order, handle, order_one_node;
} ehgp_forest_birth;

typedef struct ehgp_forest_binding { /* ExactDirectMorseForestArmRootBinding */
  uint32_t arm_seed, family, carrier, prior_root;
} ehgp_forest_binding;

typedef struct ehgp_forest_saddle {  /* ExactDirectMorseForestSaddleRecord */
  uint32_t family, event, batch, arm_offset, arm_count, carriers, latent, prior_roots, group;
} ehgp_forest_saddle;

typedef struct ehgp_forest_group {   /* ExactDirectMorseForestAtomicGroup; kind 0 birth, 1 continuation, 2 multifusion */
  uint32_t batch, saddle_offset, saddle_count, frozen, latent, prior_roots, child_offset, child_count, created_node,
      result_node, kind;
} ehgp_forest_group;

typedef struct ehgp_forest_batch {   /* ExactDirectMorseForestBatch */
  uint32_t order, level_event, birth_offset, birth_count, saddle_offset, saddle_count, group_offset, group_count,
      pre_carriers, pre_roots, post_carriers, post_roots;
} ehgp_forest_batch;

typedef struct ehgp_forest_root {    /* ExactDirectMorseForestFinalRoot */
  uint32_t order, handle, node;
} ehgp_forest_root;

/* Vertical map v_{k-1,a} of the tower (contract-v2 VerticalAssignment,
 * morsehgp3d/schemas/morsehgp3d-contract-v2.schema.json $defs.VerticalAssignment; the
 * reference's direct vertical journal, direct_morse_vertical_journal.hpp:287, takes these
 * images as external proposals): every reduced node of order k >= 2 maps, at its own level
 * on the closed cut, to the root of order k - 1 whose component contains it.  Ordered by
 * source node; source_order = k, target order k - 1. */
typedef struct ehgp_vertical_assignment {
  uint32_t source_node, target_node, source_order, level_event;
} ehgp_vertical_assignment;

/* Host copies of the last ehgp_hierarchy result; every pointer may be NULL
 * and must otherwise hold the count reported in ehgp_hier_counts. */
typedef struct ehgp_hier_out {
  ehgp_event_record* events;
  ehgp_journal_batch* journal_batches;
  ehgp_role_record* roles;
  ehgp_family_record* families;
  uint32_t* arm_removed;             /* [arm_seeds] removed support PointId; family via families[] */
  ehgp_forest_node* nodes;
  uint32_t* children;
  ehgp_forest_birth* births;
  ehgp_forest_binding* bindings;
  ehgp_forest_saddle* saddles;
  ehgp_forest_group* groups;
  ehgp_forest_batch* batches;
  ehgp_forest_root* roots;
  ehgp_vertical_assignment* vertical;
} ehgp_hier_out;

int ehgp_hier_copy(ehgp_ctx* ctx, const ehgp_hier_out* out);

/* Schedule of later ehgp_hierarchy calls on ctx; results never depend on it.  No
 * counterpart in the reference, whose forest journal is one sequential pass
 * (src/cpu/hierarchy/direct_morse_forest_journal.cpp:1042-2150): single-role batches
 * per chunk that the host pool rebuilds in parallel (0: 16384), strict arms per part
 * of the descent that an order's union-find core consumes while the device descends
 * the next (0: 4,194,304), and host threads (0: every hardware thread). */
int ehgp_hier_schedule(ehgp_ctx* ctx, uint32_t chunk_batches, uint32_t part_arms, uint32_t host_threads);

/* Timing of the last ehgp_hierarchy call: ms[0] device stages (CUDA events),
 * ms[1] the strict-arm descent kernels, ms[2] the host forest pass, ms[3] its
 * slowest order (orders run on parallel host threads), ms[4] the exact
 * ordering of the facade runs that FP64 level intervals leave open (on the device), ms[5..7] the host forest pass split
 * into the order passes, the record offsets and the vertical maps,
 * ms[8 + k - 1] the union-find core of order k (k <= 16,
 * zero above the last order);
 * stats[0] strict arms, [1] descent steps, [2] facade boundaries settled
 * exactly (2304-bit level comparisons on the device), [3] facade events, [4] arms that are not themselves a
 * birth facet, [5] descent rounds (longest chain), [6..12] slow-path counts of
 * the descent (exhaustive miniball enumerations, exact hull signs, exact
 * closed-ball sides, exact level conversions, exact band orders, exact cutoff
 * comparisons, strictness checks at an equal cutoff), [13] LBVH nodes visited by
 * the descent steps' ball queries, [14] descent-step launches; ms[24] the summed
 * CUDA-event time of the descent-step launches; ms holds 25 doubles and stats 15
 * words. */
int ehgp_hier_stats(const ehgp_ctx* ctx, double* ms, uint64_t* stats);

/* Exact level of facade event `event` as num / (den 2^(2 scale)), two's
 * complement little-endian 64-bit limbs, 36 each (num = |N|^2, den = 4 A^2 of
 * the circumsphere at the cloud scale; not reduced). */
int ehgp_event_level(ehgp_ctx* ctx, uint64_t event, uint64_t* num, uint64_t* den, int32_t* scale);

/* Supports of facade events of the last ehgp_hierarchy result, for `count`
 * event indices (e.g. the level_event of forest nodes): out[5i] the support
 * size, out[5i + 1..4] its PointIds (unused 0); UINT32_MAX (level 0) gives size
 * 0.  A level is the squared circumradius of its support (the circumsphere of a
 * triangle centred in its plane; half the segment for a pair), so the supports
 * keep exact levels once the context moves on to another cloud.  Stands in for
 * reading ExactDirectSupportEvent::support_ids through the facade
 * (morsehgp3d/include/morsehgp3d/hierarchy/direct_support_terminal.hpp:59-74). */
int ehgp_event_supports(ehgp_ctx* ctx, const uint32_t* events, uint64_t count, uint32_t* out);

/* ---- serving: many clouds on one GPU, continuous batching -----------------
 * The reference plans a request front end over its contexts
 * (morsehgp3d/docs/GPU_G4_ARCHITECTURE.md:269-294: fit / result accessors; its
 * memory plan at 80 % of the device, :117-136) and has no batching or serving
 * code.  A server runs `workers` requests at a time, each on a context of its
 * own (CUDA stream, device buffers, host thread); submitted clouds queue and are
 * admitted in order as soon as a worker is idle and the device-memory
 * reservations of the running requests, with this one, stay within
 * hbm_fraction of the device's memory.  Every request runs the whole chain
 * (canonical cloud + LBVH, EMST, pair and triple/quad supports, direct
 * hierarchy with vertical maps) with its state on the device, and its result is
 * copied to host memory the request owns when it completes; it equals the
 * result of the same cloud run alone.  Calls are thread-safe. */
typedef struct ehgp_server ehgp_server;
typedef uint64_t ehgp_request_id;

typedef struct ehgp_server_limits {
  uint32_t workers;      /* requests on the device at a time (1..64)              */
  uint64_t max_points;   /* largest cloud a request may hold                       */
  double hbm_fraction;   /* admission ceiling as a fraction of device memory (0.8) */
} ehgp_server_limits;

enum { EHGP_DTYPE_F64 = 0, EHGP_DTYPE_F32 = 1 };
typedef struct ehgp_cloud_desc {
  const void* xyz;   /* host, n interleaved x,y,z values of `dtype`; copied at submit */
  uint64_t n;
  uint32_t dtype;    /* EHGP_DTYPE_F64 or EHGP_DTYPE_F32 (widened exactly)           */
  uint32_t K;        /* K_max, 1..10                                                 */
} ehgp_cloud_desc;

enum { EHGP_REQ_QUEUED = 0, EHGP_REQ_RUNNING = 1, EHGP_REQ_DONE = 2, EHGP_REQ_FAILED = 3 };
typedef struct ehgp_request_stats {
  int32_t state, status;     /* EHGP_REQ_*; the chain's status once finished        */
  uint64_t points;
  uint32_t K, worker;
  double queued_ms;          /* submit to admission                                  */
  double service_ms;         /* admission to completion (result in host memory)      */
  double latency_ms;         /* submit to completion                                 */
  double device_ms;          /* device timeline of the chain on its stream           */
  ehgp_hier_counts counts;   /* sizes of the result arrays                           */
} ehgp_request_stats;

/* Host copies of a completed request's result; sizes from ehgp_request_stats.counts
 * (nodes, children, journal_batches, final_roots, vertical_assignments) and n - 1
 * EMST edges; any pointer may be NULL.  node_supports holds 5 words per node:
 * the support size and PointIds of the event at the node's level (size 0: level
 * 0); level_event fields index the request's own facade. */
typedef struct ehgp_served_out {
  ehgp_forest_node* nodes;
  uint32_t* children;
  ehgp_forest_batch* batches;
  ehgp_forest_root* roots;
  ehgp_vertical_assignment* vertical;
  uint32_t* node_supports;
  uint32_t* emst_u;
  uint32_t* emst_v;
} ehgp_served_out;

int ehgp_server_create(int device, const ehgp_server_limits* limits, ehgp_server** out);
int ehgp_server_destroy(ehgp_server* server);
/* Queues a cloud (asynchronous; the points are copied).  EHGP_ERR_CAPACITY above
 * max_points; EHGP_ERR_OUT_OF_MEMORY when the cloud alone exceeds the budget. */
int ehgp_cloud_submit(ehgp_server* server, const ehgp_cloud_desc* cloud, ehgp_request_id* id);
int ehgp_poll(ehgp_server* server, ehgp_request_id id, int32_t* state);
/* Waits until the request has finished or timeout_ns passed (EHGP_ERR_TIMEOUT). */
int ehgp_wait(ehgp_server* server, ehgp_request_id id, uint64_t timeout_ns, int32_t* status);
int ehgp_request_info(ehgp_server* server, ehgp_request_id id, ehgp_request_stats* info);
const char* ehgp_request_error(ehgp_server* server, ehgp_request_id id);
int ehgp_result_copy(ehgp_server* server, ehgp_request_id id, const ehgp_served_out* out);
/* Drops a finished request and its result. */
int ehgp_result_release(ehgp_server* server, ehgp_request_id id);
/* [0] memory budget, [1] bytes reserved by running requests, [2] device bytes held
 * by the workers' contexts, [3] admission estimate in bytes per point, [4] queued,
 * [5] running, [6] completed requests, [7] admissions deferred for memory. */
int ehgp_server_info(ehgp_server* server, uint64_t* info, uint32_t count);

#ifdef __cplusplus
}
#endif

#endif /* EHGP_H_ */
