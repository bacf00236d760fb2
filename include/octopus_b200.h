/*
 * octopus_b200.h -- C ABI of the B200 (sm_100a) fixed-radius octree
 * neighbor search.
 *
 * The entry points fill the backend hooks that Octopus.jl's CUDA extension
 * fills today (src/Octopus.jl:46-54): a Julia extension (or any FFI host)
 * binds these symbols with plain pointers and sizes.  Every pointer argument
 * named *coords*, *senders*, *receivers*, *rel_*, *d_rel_* or *grad* is a
 * device pointer on the context's device; sizes are element counts.
 *
 * Conventions (same as the reference, src/types.jl):
 *   - coordinates are (ndims, n) column-major: x1 y1 z1 x2 y2 z2 ...
 *   - dtype 0 = Float32, 1 = Float64
 *   - indices (senders, receivers, perm, node ids) are 1-based Int32
 *   - rel_displacement is (ndims, n_edges) column-major, rel_dist_norm (1, n_edges)
 *
 * Every function returns an oct_status; on failure oct_ctx_last_error()
 * describes it.  Calls on one context are not re-entrant.
 */
#ifndef OCTOPUS_B200_H
#define OCTOPUS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OCT_API __attribute__((visibility("default")))

/* Status codes.  The host binding maps them to the exception types the
 * reference raises (src/api.jl, test/api.jl, test/backend_errors_cpu.jl). */
typedef enum {
    OCT_OK = 0,
    OCT_ERR_ARGUMENT = 1,   /* ArgumentError */
    OCT_ERR_DIMENSION = 2,  /* DimensionMismatch */
    OCT_ERR_INEXACT = 3,    /* InexactError: floor(Int32, ...) in bin_point, src/morton.jl:84 */
    OCT_ERR_CUDA = 4,       /* CUDA runtime failure */
    OCT_ERR_OVERFLOW = 5,   /* internal capacity retry did not converge */
    OCT_ERR_CAPACITY = 6,   /* caller buffer smaller than required */
    OCT_ERR_TIMEOUT = 7,    /* a bounded device wait ran out */
    OCT_ERR_STATE = 8       /* ErrorException: call order / missing build */
} oct_status;

typedef struct oct_ctx oct_ctx;   /* one device + one stream */
typedef struct oct_tree oct_tree; /* one point set's search structure */

/* Device views of a built tree: the DeviceView contract of
 * ext/OctopusCUDAExt.jl:23-35 (node_first/last, node_children, bounds,
 * perm), valid until the next oct_tree_build on the same tree. */
typedef struct {
    int64_t n_points;
    int64_t n_nodes;
    int32_t ndims;
    int32_t dtype;
    double radius;
    const int32_t* node_first;    /* (n_nodes,) 1-based inclusive range into perm */
    const int32_t* node_last;     /* (n_nodes,) */
    const int32_t* node_children; /* (2^ndims, n_nodes) column-major, -1 = empty slot */
    const void* bounds_min;       /* (ndims, n_nodes) column-major */
    const void* bounds_max;       /* (ndims, n_nodes) column-major */
    const int32_t* perm;          /* (n_points,) 1-based Morton order */
    const uint64_t* morton;       /* (n_points,) per original point, or NULL unless keep_morton */
} oct_tree_view;

/* Library version (major * 10000 + minor * 100 + patch). */
OCT_API int oct_version(void);

/* Human-readable name of a status code. */
OCT_API const char* oct_status_string(int status);

/* Create a context on `device` using the legacy default stream.  Replaces the
 * implicit CUDA.jl device/stream state the reference's extension uses
 * (ext/OctopusCUDAExt.jl:6-17). */
OCT_API int oct_ctx_create(int device, oct_ctx** out);
OCT_API int oct_ctx_destroy(oct_ctx* ctx);

/* Order all later work after the caller's stream (a cudaStream_t). */
OCT_API int oct_ctx_set_stream(oct_ctx* ctx, void* stream);

/* Message of the last failure on this context ("" when none). */
OCT_API const char* oct_ctx_last_error(const oct_ctx* ctx);

/* Block until all work issued on the context's stream has finished; also
 * reports OCT_ERR_STATE if a kernel's bounds guard fired since the last
 * oct_edges_count. */
OCT_API int oct_synchronize(oct_ctx* ctx);

/* A tree for one point set (the Octree of src/types.jl:23-42). */
OCT_API int oct_tree_create(oct_ctx* ctx, int ndims, int dtype, oct_tree** out);
OCT_API int oct_tree_destroy(oct_tree* tree);

/* run! for one dirty point set: origin, Morton binning, stable key sort,
 * BFS topology and bounds.  Replaces _build_gpu_tree!
 * (ext/cuda_build.jl:227-288) called from _run_cuda!
 * (ext/OctopusCUDAExt.jl:214-248) and reproduces the CPU build
 * (src/api.jl:194-250) exactly.  `coords` is read during the call only.
 * keep_morton != 0 retains the per-point Morton codes (set_refit_mode!,
 * src/api.jl:43-47) and, from the second build of the same size and radius
 * on, reuses the previous sorted order: keys are re-encoded in that order,
 * the changed ones are sorted and merged in, and when none changed only the
 * bounds are recomputed.  The result is identical to a full rebuild (the
 * reference rebuilds fully on every run!, test/refit.jl:15-40).  Returns
 * OCT_ERR_INEXACT where the reference's floor(Int32, ...) throws
 * InexactError (non-finite or out-of-range cell). */
OCT_API int oct_tree_build(oct_ctx* ctx, oct_tree* tree, const void* coords, int64_t n,
                           double radius, int keep_morton);

/* How the last oct_tree_build ordered the points: *path = 0 full sort,
 * 1 changed keys merged into the previous order, 2 no key changed (bounds
 * only); *n_changed = keys changed since the previous build, or -1 when the
 * previous order was not reusable.  No counterpart in the reference. */
OCT_API int oct_tree_last_build(const oct_tree* tree, int* path, int64_t* n_changed);

/* Batched run! for many independent point sets ("clouds") in one pass; no
 * counterpart in the reference, which builds one TNS per radius
 * (src/api.jl:24-29): cloud c is the points [cloud_offsets[c],
 * cloud_offsets[c+1]) of `coords` (host array, n_clouds + 1 entries) with
 * search radius radii[c] (host array).  Each cloud gets exactly the tree a
 * TNS of that cloud alone builds; the clouds share one forest, one sort and
 * one set of launches.  Searched with oct_edges_count / oct_edges_fill
 * (query == target, exclude_self = 1): the COO concatenates the clouds in
 * order, each cloud's edges exactly as a standalone build_edges, with
 * 1-based indices local to the cloud. */
OCT_API int oct_tree_build_batch(oct_ctx* ctx, oct_tree* tree, const void* coords, int64_t n,
                                 const int64_t* cloud_offsets, const double* radii, int32_t n_clouds);

/* After oct_edges_count on a batched tree: edge_offsets (host, n_clouds + 1)
 * receives where each cloud's edges start in the concatenated COO. */
OCT_API int oct_batch_edge_offsets(oct_ctx* ctx, oct_tree* tree, int64_t* edge_offsets);

/* Number of nodes of the last build (synchronizes). */
OCT_API int oct_tree_n_nodes(oct_ctx* ctx, const oct_tree* tree, int64_t* n_nodes);

/* Materialize the reference-layout arrays of a built tree.  Replaces
 * _device_view (ext/OctopusCUDAExt.jl:37-56); the pointers are owned by the
 * tree. */
OCT_API int oct_tree_view_get(oct_ctx* ctx, oct_tree* tree, oct_tree_view* out);

/* Pass A of build_edges for the pair (query, target): count neighbors per
 * query point (self pair excluded when exclude_self != 0), scan, and
 * return the edge total.  Replaces _count_edges_kernel! + cumsum! + the
 * host read of n_edges (ext/OctopusCUDAExt.jl:262-288, 369-387). */
OCT_API int oct_edges_count(oct_ctx* ctx, const oct_tree* query, const oct_tree* target,
                            int exclude_self, int64_t* n_edges);

/* Traversal statistics of the count pass for the pair (a diagnostic; the
 * reference's phase timers, benchmarks/profile_phases.jl:29-46, have no
 * counterpart at this level).  Runs the count pass once more with counters
 * and writes up to n_stats totals: [0] query groups, [1] query points,
 * [2] internal-node expansion rounds, [3] child boxes tested, [4] leaf chunks
 * staged, [5] target points staged, [6] pair-loop steps (four targets each),
 * [7] query-target distance tests issued, [8] pairs within the radius,
 * [9] SM cycles of the traversing warps, [10] of which in leaf chunks,
 * [11] of which in the pair loop.  Synchronizes; an oct_edges_fill must be
 * preceded by a new oct_edges_count. */
OCT_API int oct_edges_traversal_stats(oct_ctx* ctx, const oct_tree* query, const oct_tree* target, int exclude_self,
                                      uint64_t* stats, int n_stats);

/* Pass B of build_edges: write the flat COO of the last oct_edges_count on
 * the same pair into caller-owned device buffers of at least `capacity`
 * edges: senders (target j), receivers (query i), rel_displacement =
 * (x_i - x_j) / r and rel_dist_norm = |x_i - x_j| / r, in the CPU path's
 * order.  Replaces _fill_edges_kernel_{3d,2d}! (ext/OctopusCUDAExt.jl:290-343,
 * 401-411). */
OCT_API int oct_edges_fill(oct_ctx* ctx, const oct_tree* query, const oct_tree* target,
                           int exclude_self, int32_t* senders, int32_t* receivers,
                           void* rel_displacement, void* rel_dist_norm, int64_t capacity);

/* The forward of build_edges_diff for a self pair (the primal of
 * ext/OctopusCUDAChainRulesCoreExt.jl:21-32): oct_edges_fill of the last
 * oct_edges_count on (tree, tree, exclude_self = 1), plus mirror[k] = the
 * 0-based COO index of edge k's mirror (for k = (i <- j), the edge (j <- i)),
 * for oct_edges_diff_backward_mirror.  Not for a batched tree; at most
 * 2^31 - 1 edges (OCT_ERR_OVERFLOW). */
OCT_API int oct_edges_fill_diff(oct_ctx* ctx, const oct_tree* tree, int32_t* senders, int32_t* receivers,
                                void* rel_displacement, void* rel_dist_norm, int32_t* mirror, int64_t capacity);

/* materialize_all_neighbors! for the pair of the last oct_edges_count:
 * CSR neighbor lists, offsets (n_query + 1 Int32, offsets[0] = 0, row i of
 * query point i+1 at flat[offsets[i] .. offsets[i+1]-1]) and flat (1-based
 * target indices, the self pair excluded when exclude_self != 0), each row
 * in the reference's traversal order -- the senders column of build_edges'
 * COO.  Replaces materialize_cpu! (src/cpu/query_cpu.jl:149-192); the
 * reference raises on a CUDA TNS (src/api.jl:350).  OCT_ERR_OVERFLOW when
 * the total does not fit the Int32 offsets. */
OCT_API int oct_csr_fill(oct_ctx* ctx, const oct_tree* query, const oct_tree* target, int exclude_self,
                         int32_t* offsets, int32_t* flat, int64_t capacity);

/* apply_zsort: permute a user array by the tree's Morton order.  `in` and
 * `out` are distinct device arrays of n rows of row_bytes bytes each (a
 * (F, n) column-major matrix has rows of F elements; a vector, of one).
 * direction 0: out[:, i] = in[:, perm[i]] (apply_zsort,
 * src/cpu/zsort_cpu.jl:11-32, ext/OctopusCUDAExt.jl:422-432);
 * direction 1: out[:, perm[i]] = in[:, i] (the pullback of its rrule,
 * ext/OctopusChainRulesCoreExt.jl:65-94).  n must equal the tree's point
 * count (OCT_ERR_DIMENSION), and the tree must be built (OCT_ERR_STATE,
 * prepare_zsort's error, src/api.jl:380-386). */
OCT_API int oct_zsort_apply(oct_ctx* ctx, const oct_tree* tree, const void* in, void* out, int64_t n,
                            int64_t row_bytes, int direction);

/* The zsort hook in the reference's own shape: _apply_zsort_cuda(perm,
 * user_array) (ext/OctopusCUDAExt.jl:422-432, called from apply_zsort,
 * src/api.jl:404-408) with `perm` any 1-based Int32 device vector of n
 * entries (tns.permutation[set_id]).  `in` and `out` are distinct device
 * arrays of n rows of row_bytes bytes (a (F, n) column-major matrix has rows
 * of F elements).  direction 0: out[:, i] = in[:, perm[i]] (the reference's
 * user_array[:, perm]); direction 1: out[:, perm[i]] = in[:, i] (the scatter
 * of its rrule's pullback, ext/OctopusChainRulesCoreExt.jl:83-94).  An entry
 * outside 1..n is not dereferenced: the call returns OCT_ERR_ARGUMENT (the
 * reference's BoundsError).  Waits for the permute (it reads that check
 * back). */
OCT_API int oct_permute_rows(oct_ctx* ctx, const int32_t* perm, int64_t n, const void* in, void* out,
                             int64_t row_bytes, int direction);

/* Neighbors of n_queries points (device coords, (ndims, n_queries)) in the
 * target tree, in the reference's traversal order and without the self
 * filter: the host for_each_neighbor / get_neighborlist accessors
 * (src/cpu/iterator_cpu.jl:245-263, src/api.jl:282-292).  Writes
 * out_counts[q] and up to cap_per_query 1-based indices per query at
 * out_indices[q * cap_per_query ...]. */
OCT_API int oct_neighbors(oct_ctx* ctx, const oct_tree* target, const void* query_coords,
                          int64_t n_queries, int32_t* out_counts, int32_t* out_indices,
                          int64_t cap_per_query);

/* Pullback of build_edges_diff for a self pair: grad_coords (ndims, n_points)
 * = sum over edges of (+c on the receiver, -c on the sender) with
 * c = d_rel_displacement / r + rel_displacement * d_rel_dist_norm /
 * (rel_dist_norm * r) (distance term skipped when rel_dist_norm <= 1e-8).
 * Either cotangent may be NULL (zero).  Deterministic (no float atomics).
 * Replaces _build_edges_diff_pullback_kernel!
 * (ext/OctopusCUDAChainRulesCoreExt.jl:56-99) and matches the CPU rrule
 * (ext/OctopusChainRulesCoreExt.jl:137-192). */
OCT_API int oct_edges_diff_backward(oct_ctx* ctx, int ndims, int dtype, int64_t n_points,
                                    int64_t n_edges, const int32_t* senders,
                                    const int32_t* receivers, const void* rel_displacement,
                                    const void* rel_dist_norm, const void* d_rel_displacement,
                                    const void* d_rel_dist_norm, double radius, void* grad_coords);

/* Adjoint of build_edges for a cross pair (query set != target set): the
 * cotangent term of edge k (receiver i <- sender j, as in
 * oct_edges_diff_backward) is added to grad_query[:, i] and subtracted
 * from grad_target[:, j].  The reference's rrule covers the self pair only
 * and names this extension (ext/OctopusChainRulesCoreExt.jl:134-135);
 * deterministic, no floating-point atomics. */
OCT_API int oct_edges_diff_backward_pair(oct_ctx* ctx, int ndims, int dtype, int64_t n_query, int64_t n_target,
                                         int64_t n_edges, const int32_t* senders, const int32_t* receivers,
                                         const void* rel_displacement, const void* rel_dist_norm,
                                         const void* d_rel_displacement, const void* d_rel_dist_norm, double radius,
                                         void* grad_query, void* grad_target);

/* The same pullback without the stored features: rel_displacement and
 * rel_dist_norm are recomputed from `coords` ((ndims, n_points), the
 * coordinates the edges were built from) with the forward's exact arithmetic,
 * so a caller short of memory need not keep them for the backward pass.
 * Requires the self-pair COO of one point set (every edge has its mirror). */
OCT_API int oct_edges_diff_backward_recompute(oct_ctx* ctx, int ndims, int dtype, int64_t n_points,
                                              int64_t n_edges, const int32_t* senders,
                                              const int32_t* receivers, const void* coords,
                                              const void* d_rel_displacement, const void* d_rel_dist_norm,
                                              double radius, void* grad_coords);

/* The self-pair pullback with a processing order: `order` (n_points entries,
 * 1-based, a permutation such as the tree's perm from oct_tree_arrays) sets
 * which points a warp handles together.  A spatial order keeps the mirror
 * edges that each warp reads in the on-chip cache; the gradient is the same
 * for every permutation (and NULL means 1..n).  Features are read from
 * rel_displacement / rel_dist_norm, or recomputed from `coords` when it is
 * non-NULL (then the features may be NULL).  Entries of `order` outside
 * 1..n_points, and edge indices outside 1..n_points, return
 * OCT_ERR_ARGUMENT.  Same adjoint as oct_edges_diff_backward
 * (ext/OctopusChainRulesCoreExt.jl:137-192). */
OCT_API int oct_edges_diff_backward_ordered(oct_ctx* ctx, int ndims, int dtype, int64_t n_points,
                                            int64_t n_edges, const int32_t* senders,
                                            const int32_t* receivers, const void* rel_displacement,
                                            const void* rel_dist_norm, const void* coords,
                                            const void* d_rel_displacement, const void* d_rel_dist_norm,
                                            double radius, void* grad_coords, const int32_t* order);

/* The self-pair pullback in one pass, with the mirror indices that
 * oct_edges_fill_diff wrote for this COO: the same gradient, bit for bit, as
 * oct_edges_diff_backward_ordered (same arguments, plus `mirror`), without
 * searching each edge's mirror.  A mirror index outside the COO, or a COO not
 * grouped by receiver, falls back to that entry point's path.  Replaces the
 * pullback of ext/OctopusCUDAChainRulesCoreExt.jl:118-167
 * (ext/OctopusChainRulesCoreExt.jl:137-192 on the CPU). */
OCT_API int oct_edges_diff_backward_mirror(oct_ctx* ctx, int ndims, int dtype, int64_t n_points, int64_t n_edges,
                                           const int32_t* senders, const int32_t* receivers, const int32_t* mirror,
                                           const void* rel_displacement, const void* rel_dist_norm,
                                           const void* coords, const void* d_rel_displacement,
                                           const void* d_rel_dist_norm, double radius, void* grad_coords,
                                           const int32_t* order);

/* Edge count that allocates no device memory.  No counterpart in the
 * reference: it serves callers that cannot let a library call cudaMalloc --
 * hosts whose device memory belongs to their own pool allocator (a
 * framework's caching allocator, a fixed memory budget), where a raw
 * cudaMalloc may fail or fragment the pool, and latency-critical loops that
 * cannot afford the implicit device synchronization of cudaMalloc/cudaFree.
 * Same result and the same argument rules as oct_edges_count for the pair
 * (a batched tree only against itself with exclude_self = 1), but the caller
 * passes counts[n_q] (int32, per query point) and offsets[n_q + 1] (int64
 * exclusive scan, offsets[n_q] = edge total) as device outputs; *n_edges
 * (optional, host) receives the total after a stream synchronize, so it must
 * be NULL while the stream is being captured (OCT_ERR_STATE otherwise).  The scan's scratch is
 * a fixed 64 KiB device array that every GPU loading this library holds until
 * exit, which limits the query set to 16,777,216 points (larger sets get
 * OCT_ERR_CAPACITY).  The first call on a device looks up that array's device
 * address (make this first call before any stream capture begins); that
 * address does not survive cudaDeviceReset in the same process.  All calls
 * share the array: calls whose GPU work overlaps (other streams, other host
 * threads, other contexts on the same device) race and must not be issued.
 * It does not prepare oct_edges_fill. */
OCT_API int oct_edges_count_noalloc(oct_ctx* ctx, const oct_tree* query, const oct_tree* target,
                                    int exclude_self, int32_t* counts, int64_t* offsets,
                                    int64_t* n_edges);

/* Options of a context, read by every later call on it.  No counterpart in
 * the reference, whose launch shapes and capacities are fixed in its CUDA
 * extension; its overflow test drives the build kernels with a smaller node
 * capacity than they need and a canary region past it
 * (test/edges_cuda.jl:147-265), which OCT_OPT_NODE_CAPACITY and
 * OCT_OPT_GUARD_CHECK do through this interface.
 *   OCT_OPT_WAIT_LIMIT     polling rounds of a bounded device wait (the key
 *                          sort's look-back) before it gives up; the build
 *                          then returns OCT_ERR_TIMEOUT (default 4,194,304)
 *   OCT_OPT_NODE_CAPACITY  node capacity of each build's first topology
 *                          attempt, 0 = the estimate from the point count
 *                          (default); a smaller one overflows and the build
 *                          retries with the exact count
 *   OCT_OPT_RECORD_CAP     hit records per query point of the next counts,
 *                          0 = sized from the previous count (default); query
 *                          groups that run out are written by a second walk
 *   OCT_OPT_GUARD_CHECK    1: a canary region follows the written part of the
 *                          sort buffers and node arrays, checked after each
 *                          topology attempt (OCT_ERR_STATE if overwritten)
 *   OCT_OPT_WITHHOLD_TILE  test aid: tile k (0-based) of the first pass of the
 *                          look-back key sort never publishes its counts, so
 *                          the waits after it run out (-1 = off, default)
 * Kernel shapes (no result depends on them; 0 = the tuning table's choice,
 * or the default when no table is loaded, see oct_ctx_load_tuning):
 *   OCT_OPT_MAX_SEG        leaves sharing one staged chunk of the traversal, 1..16 (16)
 *   OCT_OPT_MULTI_POP      internal nodes the traversal expands together, 1..4 (4)
 *   OCT_OPT_FILL_CHUNK     the fill's stores: 1 direct (default), or 32, 64 or 128 for
 *                          bulk copies of that many edges per chunk (a table row says 0
 *                          for direct)
 *   OCT_OPT_GROUP_CAP      query points per traversal group, 8..32 (32), set at the build
 *   OCT_OPT_SUB_BOXES      boxes a group's queries are split into (runs of 32/k lanes)
 *                          for the test that skips distant target points: 1, 2 or 4 (1)
 *   OCT_OPT_PREFETCH       the traversal prefetches into L1 what it reads next (the next
 *                          leaf chunk's points, the next node's children): 1 off, 2 on (off)
 * Read-only (oct_ctx_get_option):
 *   OCT_STAT_TUNING_ROW       tuning-table row the last count or build used (-1 = defaults)
 *   OCT_STAT_BUILD_ATTEMPTS   topology attempts of the last build (1 = none retried)
 *   OCT_STAT_RECORD_OVERFLOW  query groups of the last count whose records overflowed
 *   OCT_STAT_RECORD_CAP       hit records per query point the last count used (0 = none) */
enum {
    OCT_OPT_WAIT_LIMIT = 1,
    OCT_OPT_NODE_CAPACITY = 2,
    OCT_OPT_RECORD_CAP = 3,
    OCT_OPT_GUARD_CHECK = 4,
    OCT_OPT_WITHHOLD_TILE = 5,
    OCT_OPT_MAX_SEG = 6,
    OCT_OPT_MULTI_POP = 7,
    OCT_OPT_FILL_CHUNK = 8,
    OCT_OPT_GROUP_CAP = 9,
    OCT_OPT_SUB_BOXES = 10,
    OCT_OPT_PREFETCH = 11,
    OCT_STAT_TUNING_ROW = 99,
    OCT_STAT_BUILD_ATTEMPTS = 100,
    OCT_STAT_RECORD_OVERFLOW = 101,
    OCT_STAT_RECORD_CAP = 102
};
OCT_API int oct_ctx_set_option(oct_ctx* ctx, int option, int64_t value);
OCT_API int oct_ctx_get_option(const oct_ctx* ctx, int option, int64_t* value);

/* Load the kernel-shape table written by the autotuner
 * (octopus.jl_b200/tune.py; the package ships octopus.jl_b200/tuning.tsv):
 * one row per line, "ndims dtype nlog2 nbr_log2 max_seg multi_pop fill_chunk
 * group_cap [sub_boxes [prefetch]]", '#' comments.  Each count (and each build, for group_cap) then
 * uses the row of the same ndims and dtype nearest to its point count
 * (log2) and neighbors per point (log2 of 1 + the last count's average),
 * unless an option forces a shape.  NULL or "" unloads the table.  No
 * counterpart in the reference, whose launch shapes are fixed
 * (ext/OctopusCUDAExt.jl:374-376, ext/cuda_build.jl:240-241). */
OCT_API int oct_ctx_load_tuning(oct_ctx* ctx, const char* path);

/* The selection of oct_ctx_load_tuning without a context or a device: the
 * shapes {max_seg, multi_pop, fill_chunk, group_cap, sub_boxes, prefetch} (six
 * entries) the table at `path` ("" = no table) gives a set of n points with nbrs_per_point neighbors per point
 * (< 0: not known yet), and the row (-1 = defaults). */
OCT_API int oct_tuning_select(const char* path, int ndims, int dtype, int64_t n, double nbrs_per_point,
                              int32_t* shapes, int32_t* row);

/* Per-phase device timing with CUDA events on the context's stream (the
 * phase timers of benchmarks/profile_phases.jl:29-46, taken on the device).
 * While enabled, every library call records its phases; oct_profile_read
 * synchronizes, returns the summed milliseconds and record counts per phase
 * (indices 0..n_phases-1, named by oct_profile_phase_name) and clears them. */
OCT_API int oct_profile_enable(oct_ctx* ctx, int on);
OCT_API const char* oct_profile_phase_name(int phase);
OCT_API int oct_profile_read(oct_ctx* ctx, double* ms, int64_t* launches, int n_phases);

/* Number of kernels this context has launched since it was created. */
OCT_API int64_t oct_profile_kernel_launches(const oct_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif /* OCTOPUS_B200_H */
