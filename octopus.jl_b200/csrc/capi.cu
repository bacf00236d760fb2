// C ABI (include/octopus_b200.h): argument checks, object lifetime and error
// reporting around the build / edge / adjoint pipelines.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>

#include "../../include/octopus_b200.h"
#include "capi_types.h"
#include "internal.h"

namespace oct {

cudaError_t ensure(DevBuf& b, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (b.bytes >= bytes) return cudaSuccess;
    if (b.p) {
        cudaError_t e = cudaFree(b.p);
        if (e != cudaSuccess) return e;
        b.p = nullptr;
        b.bytes = 0;
    }
    const size_t want = bytes + bytes / 8;  // slack so slowly growing inputs do not reallocate every call
    cudaError_t e = cudaMalloc(&b.p, want);
    if (e != cudaSuccess) {
        b.p = nullptr;
        return e;
    }
    b.bytes = want;
    return cudaSuccess;
}

void release(DevBuf& b) {
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
}

cudaEvent_t Ctx::get_event() {
    if (!event_pool.empty()) {
        cudaEvent_t e = event_pool.back();
        event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

PhaseTimer::PhaseTimer(Ctx& c, int ph) : ctx(&c), phase(ph) {
    if (!c.profiling) return;
    start = c.get_event();
    cudaEventRecord(start, c.stream);
}

PhaseTimer::~PhaseTimer() {
    if (!start) return;
    cudaEvent_t stop = ctx->get_event();
    cudaEventRecord(stop, ctx->stream);
    ctx->prof.push_back({phase, start, stop});
}

bool parse_tuning(const char* path, std::vector<TuneRow>& rows, std::string& err) {
    rows.clear();
    FILE* f = std::fopen(path, "r");
    if (!f) {
        err = std::string("cannot open tuning table ") + path;
        return false;
    }
    char line[512];
    int lineno = 0;
    bool ok = true;
    while (std::fgets(line, sizeof line, f)) {
        ++lineno;
        if (char* h = std::strchr(line, '#')) *h = '\0';
        int v[10];
        v[8] = 1;
        v[9] = 0;
        char extra[2];
        const int got = std::sscanf(line, "%d %d %d %d %d %d %d %d %d %d %1s", &v[0], &v[1], &v[2], &v[3], &v[4],
                                    &v[5], &v[6], &v[7], &v[8], &v[9], extra);
        if (got <= 0) continue;  // blank or comment
        const bool valid = got >= 8 && got <= 10 && (v[0] == 2 || v[0] == 3) && (v[1] == 0 || v[1] == 1) &&
                           v[2] >= 0 && v[2] <= 40 && v[3] >= 0 && v[3] <= 40 && v[4] >= 1 && v[4] <= 16 &&
                           v[5] >= 1 && v[5] <= 4 && (v[6] == 0 || v[6] == 32 || v[6] == 64 || v[6] == 128) && v[7] >= 8 &&
                           v[7] <= 32 && (v[8] == 1 || v[8] == 2 || v[8] == 4) && (v[9] == 0 || v[9] == 1);
        if (!valid) {
            err = std::string("tuning table ") + path + ": bad row at line " + std::to_string(lineno);
            ok = false;
            break;
        }
        TuneRow r;
        r.ndims = v[0];
        r.dtype = v[1];
        r.nlog2 = v[2];
        r.nbr_log2 = v[3];
        r.tn.max_seg = v[4];
        r.tn.multi_pop = v[5];
        r.tn.fill_chunk = v[6];
        r.tn.group_cap = v[7];
        r.tn.sub_boxes = v[8];
        r.tn.prefetch = v[9];
        rows.push_back(r);
    }
    std::fclose(f);
    if (!ok) rows.clear();
    return ok;
}

int select_tuning(const std::vector<TuneRow>& rows, int ndims, int dtype, int64_t n, double nbrs, Tuning& out) {
    out = Tuning{};
    int nlog2 = 0;
    while (nlog2 < 62 && (int64_t(1) << (nlog2 + 1)) <= n) ++nlog2;
    // an unknown neighbor count (no count yet) keys as the mid bucket 4 (~15 per point)
    int blog2 = 4;
    if (nbrs >= 0.0) {
        blog2 = 0;
        while (blog2 < 40 && (double)(int64_t(1) << (blog2 + 1)) <= nbrs + 1.0) ++blog2;
    }
    int best = -1, best_d = 1 << 30;
    for (size_t i = 0; i < rows.size(); ++i) {
        const TuneRow& r = rows[i];
        if (r.ndims != ndims || r.dtype != dtype) continue;
        const int d = std::abs(r.nlog2 - nlog2) + 2 * std::abs(r.nbr_log2 - blog2);
        if (d < best_d) {
            best_d = d;
            best = (int)i;
        }
    }
    if (best >= 0) out = rows[(size_t)best].tn;
    return best;
}

Tuning Ctx::tuning_for(int ndims, int dtype, int64_t n, double nbrs) {
    Tuning tn;
    last_tune_row = select_tuning(tune_table, ndims, dtype, n, nbrs, tn);
    if (tune_force.max_seg) tn.max_seg = tune_force.max_seg;
    if (tune_force.multi_pop) tn.multi_pop = tune_force.multi_pop;
    if (tune_force.fill_chunk) tn.fill_chunk = tune_force.fill_chunk == 1 ? 0 : tune_force.fill_chunk;
    if (tune_force.group_cap) tn.group_cap = tune_force.group_cap;
    if (tune_force.sub_boxes) tn.sub_boxes = tune_force.sub_boxes;
    if (tune_force.prefetch) tn.prefetch = tune_force.prefetch - 1;
    return tn;
}

int set_error(Ctx& ctx, int status, const std::string& msg) {
    ctx.last_error = msg;
    return status;
}

int cuda_status(Ctx& ctx, cudaError_t e, const char* where) {
    if (e == cudaSuccess) return OK;
    ctx.last_error = std::string(where) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return ERR_CUDA;
}

}  // namespace oct

namespace {

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

void release_tree(oct::Tree& t) {
    using oct::release;
    for (auto* b : {&t.b_coff, &t.b_cparam, &t.b_croot, &t.b_cstart, &t.b_cbounds, &t.b_eoff})
        release(*b);
    for (auto* b : {&t.keys[0], &t.keys[1], &t.vals[0], &t.vals[1], &t.hist, &t.sort_tmp, &t.look, &t.spts, &t.spts_tmp, &t.tnode, &t.nrange,
                    &t.parent, &t.fchild, &t.arrive, &t.groups, &t.gstart, &t.chain, &t.lohi, &t.blockcnt, &t.blockoff, &t.scan_tmp, &t.partials, &t.hdr,
                    &t.morton, &t.v_first, &t.v_last, &t.v_children, &t.v_bmin, &t.v_bmax, &t.v_perm, &t.iperm,
                    &t.rflag, &t.rcnt, &t.roff, &t.mkeys, &t.mvals, &t.mkeys2, &t.mvals2})
        release(*b);
    if (t.hdr_host) cudaFreeHost(t.hdr_host);
    t.hdr_host = nullptr;
}

bool bad_dims(int ndims) { return ndims != 2 && ndims != 3; }
bool bad_dtype(int dtype) { return dtype != 0 && dtype != 1; }

}  // namespace

extern "C" {

OCT_API int oct_version(void) { return 1 * 10000 + 0 * 100 + 0; }

OCT_API const char* oct_status_string(int status) {
    switch (status) {
        case OCT_OK: return "ok";
        case OCT_ERR_ARGUMENT: return "ArgumentError";
        case OCT_ERR_DIMENSION: return "DimensionMismatch";
        case OCT_ERR_INEXACT: return "InexactError";
        case OCT_ERR_CUDA: return "CUDA error";
        case OCT_ERR_OVERFLOW: return "capacity overflow";
        case OCT_ERR_CAPACITY: return "buffer too small";
        case OCT_ERR_TIMEOUT: return "device wait timed out";
        case OCT_ERR_STATE: return "ErrorException";
        default: return "unknown status";
    }
}

OCT_API int oct_ctx_create(int device, oct_ctx** out) {
    if (!out) return OCT_ERR_ARGUMENT;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return OCT_ERR_CUDA;
    if (device < 0 || device >= ndev) return OCT_ERR_ARGUMENT;
    oct_ctx* c = new (std::nothrow) oct_ctx();
    if (!c) return OCT_ERR_CUDA;
    c->c.device = device;
    c->c.stream = nullptr;
    *out = c;
    return OCT_OK;
}

OCT_API int oct_ctx_destroy(oct_ctx* ctx) {
    if (!ctx) return OCT_OK;
    DeviceGuard g(ctx->c.device);
    cudaStreamSynchronize(ctx->c.stream);
    using oct::release;
    for (auto* b : {&ctx->c.counts, &ctx->c.offsets, &ctx->c.scan_tmp, &ctx->c.total, &ctx->c.dkeys[0],
                    &ctx->c.dkeys[1], &ctx->c.dvals[0], &ctx->c.dvals[1], &ctx->c.dhist, &ctx->c.dsort_tmp, &ctx->c.droff,
                    &ctx->c.dsoff, &ctx->c.dstatus, &ctx->c.dredge, &ctx->c.dterm, &ctx->c.dseg, &ctx->c.tstats, &ctx->c.recs, &ctx->c.rcount, &ctx->c.gflag})
        release(*b);
    if (ctx->c.total_host) cudaFreeHost(ctx->c.total_host);
    for (auto& r : ctx->c.prof) {
        cudaEventDestroy(r.start);
        cudaEventDestroy(r.stop);
    }
    for (auto e : ctx->c.event_pool) cudaEventDestroy(e);
    delete ctx;
    return OCT_OK;
}

OCT_API int oct_ctx_set_stream(oct_ctx* ctx, void* stream) {
    if (!ctx) return OCT_ERR_ARGUMENT;
    ctx->c.stream = (cudaStream_t)stream;
    return OCT_OK;
}

OCT_API const char* oct_ctx_last_error(const oct_ctx* ctx) { return ctx ? ctx->c.last_error.c_str() : ""; }

OCT_API int oct_synchronize(oct_ctx* ctx) {
    if (!ctx) return OCT_ERR_ARGUMENT;
    DeviceGuard g(ctx->c.device);
    int st = oct::cuda_status(ctx->c, cudaStreamSynchronize(ctx->c.stream), "synchronize");
    if (st != OCT_OK || !ctx->c.dstatus.p) return st;
    int word = 0;
    st = oct::cuda_status(ctx->c, cudaMemcpy(&word, ctx->c.dstatus.p, 4, cudaMemcpyDeviceToHost), "status read");
    if (st != OCT_OK) return st;
    if (word != 0)
        return oct::set_error(ctx->c, OCT_ERR_STATE, "edge fill found more neighbors than counted (internal error)");
    return OCT_OK;
}

OCT_API int oct_tree_create(oct_ctx* ctx, int ndims, int dtype, oct_tree** out) {
    if (!ctx || !out) return OCT_ERR_ARGUMENT;
    *out = nullptr;
    if (bad_dims(ndims)) return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "ndims must be 2 or 3");
    if (bad_dtype(dtype)) return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "dtype must be 0 (Float32) or 1 (Float64)");
    oct_tree* t = new (std::nothrow) oct_tree();
    if (!t) return OCT_ERR_CUDA;
    t->t.ndims = ndims;
    t->t.dtype = dtype;
    t->owner = ctx;
    *out = t;
    return OCT_OK;
}

OCT_API int oct_tree_destroy(oct_tree* tree) {
    if (!tree) return OCT_OK;
    {
        DeviceGuard g(tree->owner ? tree->owner->c.device : 0);
        if (tree->owner) cudaStreamSynchronize(tree->owner->c.stream);
        release_tree(tree->t);
    }
    delete tree;
    return OCT_OK;
}

OCT_API int oct_tree_build(oct_ctx* ctx, oct_tree* tree, const void* coords, int64_t n, double radius,
                           int keep_morton) {
    if (!ctx || !tree) return OCT_ERR_ARGUMENT;
    ctx->c.last_error.clear();
    if (!(radius > 0.0)) return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "search radius must be positive");
    if (n < 0 || n > 2147483647LL)
        return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "point count must be in [0, 2^31 - 1] (Int32 indices)");
    if (n > 0 && !coords) return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "coords is NULL");
    DeviceGuard g(ctx->c.device);
    tree->t.keep_morton = keep_morton != 0;
    return oct::build_tree(ctx->c, tree->t, coords, n, radius);
}

OCT_API int oct_tree_build_batch(oct_ctx* ctx, oct_tree* tree, const void* coords, int64_t n,
                                 const int64_t* cloud_offsets, const double* radii, int32_t n_clouds) {
    if (!ctx || !tree) return OCT_ERR_ARGUMENT;
    ctx->c.last_error.clear();
    if (n_clouds < 1 || !cloud_offsets || !radii)
        return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "batch: need n_clouds >= 1, cloud_offsets and radii");
    if (n < 0 || n > 2147483647LL)
        return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "point count must be in [0, 2^31 - 1] (Int32 indices)");
    if (cloud_offsets[0] != 0 || cloud_offsets[n_clouds] != n)
        return oct::set_error(ctx->c, OCT_ERR_DIMENSION, "batch: cloud_offsets must start at 0 and end at n");
    for (int32_t c = 0; c < n_clouds; ++c) {
        if (cloud_offsets[c + 1] < cloud_offsets[c])
            return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "batch: cloud_offsets must be non-decreasing");
        if (!(radii[c] > 0.0)) return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "search radius must be positive");
    }
    if (n > 0 && !coords) return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "coords is NULL");
    DeviceGuard g(ctx->c.device);
    return oct::build_tree_batch(ctx->c, tree->t, coords, n, cloud_offsets, radii, n_clouds);
}

OCT_API int oct_batch_edge_offsets(oct_ctx* ctx, oct_tree* tree, int64_t* edge_offsets) {
    if (!ctx || !tree || !edge_offsets) return OCT_ERR_ARGUMENT;
    ctx->c.last_error.clear();
    if (!tree->t.built || tree->t.n_clouds < 1)
        return oct::set_error(ctx->c, OCT_ERR_STATE, "batch edge offsets: the tree is not a built batch");
    DeviceGuard g(ctx->c.device);
    return oct::batch_edge_offsets(ctx->c, tree->t, edge_offsets);
}

OCT_API int oct_tree_last_build(const oct_tree* tree, int* path, int64_t* n_changed) {
    if (!tree || !path || !n_changed) return OCT_ERR_ARGUMENT;
    *path = tree->t.last_path;
    *n_changed = tree->t.last_moved;
    return OCT_OK;
}

OCT_API int oct_tree_n_nodes(oct_ctx* ctx, const oct_tree* tree, int64_t* n_nodes) {
    if (!ctx || !tree || !n_nodes) return OCT_ERR_ARGUMENT;
    *n_nodes = tree->t.built ? tree->t.n_nodes : 0;
    return OCT_OK;
}

OCT_API int oct_tree_view_get(oct_ctx* ctx, oct_tree* tree, oct_tree_view* out) {
    if (!ctx || !tree || !out) return OCT_ERR_ARGUMENT;
    std::memset(out, 0, sizeof(*out));
    oct::Tree& t = tree->t;
    out->ndims = t.ndims;
    out->dtype = t.dtype;
    out->radius = t.radius;
    if (!t.built) return oct::set_error(ctx->c, OCT_ERR_STATE, "tree has not been built (call run! first)");
    if (t.n_clouds > 0) return oct::set_error(ctx->c, OCT_ERR_STATE, "a batched tree has no single-tree view");
    DeviceGuard g(ctx->c.device);
    const int st = oct::materialize_view(ctx->c, t);
    if (st != OCT_OK) return st;
    out->n_points = t.n;
    out->n_nodes = t.n_nodes;
    out->node_first = t.v_first.as<int32_t>();
    out->node_last = t.v_last.as<int32_t>();
    out->node_children = t.v_children.as<int32_t>();
    out->bounds_min = t.v_bmin.p;
    out->bounds_max = t.v_bmax.p;
    out->perm = t.v_perm.as<int32_t>();
    out->morton = (t.keep_morton && t.n > 0) ? t.morton.as<uint64_t>() : nullptr;
    return OCT_OK;
}

static int check_pair(oct_ctx* ctx, const oct_tree* query, const oct_tree* target) {
    if (!query || !target) return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "query/target tree is NULL");
    if (query->t.ndims != target->t.ndims || query->t.dtype != target->t.dtype)
        return oct::set_error(ctx->c, OCT_ERR_DIMENSION, "query and target trees differ in ndims or dtype");
    if (!target->t.built || !query->t.built)
        return oct::set_error(ctx->c, OCT_ERR_STATE, "query and target trees must be built before build_edges");
    return OCT_OK;
}

}  // extern "C"

int oct_check_count_pair(oct_ctx* ctx, const oct_tree* query, const oct_tree* target, int exclude_self) {
    const int st = check_pair(ctx, query, target);
    if (st != OCT_OK) return st;
    if (exclude_self && query != target)
        return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "exclude_self requires the same tree as query and target");
    if ((query->t.n_clouds > 0 || target->t.n_clouds > 0) && (query != target || !exclude_self))
        return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "a batched tree is searched against itself, self pairs excluded");
    return OCT_OK;
}

extern "C" {

OCT_API int oct_edges_count(oct_ctx* ctx, const oct_tree* query, const oct_tree* target, int exclude_self,
                            int64_t* n_edges) {
    if (!ctx || !n_edges) return OCT_ERR_ARGUMENT;
    ctx->c.last_error.clear();
    *n_edges = 0;
    const int st = oct_check_count_pair(ctx, query, target, exclude_self);
    if (st != OCT_OK) return st;
    DeviceGuard g(ctx->c.device);
    return oct::edges_count(ctx->c, query->t, target->t, exclude_self != 0, n_edges);
}

OCT_API int oct_edges_traversal_stats(oct_ctx* ctx, const oct_tree* query, const oct_tree* target, int exclude_self,
                                      uint64_t* stats, int n_stats) {
    if (!ctx || !stats || n_stats < 0) return OCT_ERR_ARGUMENT;
    ctx->c.last_error.clear();
    const int st = oct_check_count_pair(ctx, query, target, exclude_self);
    if (st != OCT_OK) return st;
    DeviceGuard g(ctx->c.device);
    return oct::traversal_stats(ctx->c, query->t, target->t, exclude_self != 0, stats, n_stats);
}

OCT_API int oct_edges_fill(oct_ctx* ctx, const oct_tree* query, const oct_tree* target, int exclude_self,
                           int32_t* senders, int32_t* receivers, void* rel_displacement, void* rel_dist_norm,
                           int64_t capacity) {
    if (!ctx) return OCT_ERR_ARGUMENT;
    ctx->c.last_error.clear();
    int st = check_pair(ctx, query, target);
    if (st != OCT_OK) return st;
    if (capacity > 0 && (!senders || !receivers || !rel_displacement || !rel_dist_norm))
        return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "edge output buffer is NULL");
    DeviceGuard g(ctx->c.device);
    return oct::edges_fill(ctx->c, query->t, target->t, exclude_self != 0, senders, receivers, rel_displacement,
                           rel_dist_norm, capacity);
}

OCT_API int oct_edges_fill_diff(oct_ctx* ctx, const oct_tree* tree, int32_t* senders, int32_t* receivers,
                                void* rel_displacement, void* rel_dist_norm, int32_t* mirror, int64_t capacity) {
    if (!ctx) return OCT_ERR_ARGUMENT;
    ctx->c.last_error.clear();
    int st = check_pair(ctx, tree, tree);
    if (st != OCT_OK) return st;
    if (capacity > 0 && (!senders || !receivers || !rel_displacement || !rel_dist_norm || !mirror))
        return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "edge output buffer is NULL");
    DeviceGuard g(ctx->c.device);
    return oct::edges_fill_diff(ctx->c, tree->t, senders, receivers, rel_displacement, rel_dist_norm, mirror,
                                capacity);
}

OCT_API int oct_csr_fill(oct_ctx* ctx, const oct_tree* query, const oct_tree* target, int exclude_self,
                         int32_t* offsets, int32_t* flat, int64_t capacity) {
    if (!ctx) return OCT_ERR_ARGUMENT;
    ctx->c.last_error.clear();
    int st = check_pair(ctx, query, target);
    if (st != OCT_OK) return st;
    if (!offsets || (capacity > 0 && !flat))
        return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "neighbor list output buffer is NULL");
    DeviceGuard g(ctx->c.device);
    return oct::csr_fill(ctx->c, query->t, target->t, exclude_self != 0, offsets, flat, capacity);
}

OCT_API int oct_zsort_apply(oct_ctx* ctx, const oct_tree* tree, const void* in, void* out, int64_t n,
                            int64_t row_bytes, int direction) {
    if (!ctx || !tree) return OCT_ERR_ARGUMENT;
    ctx->c.last_error.clear();
    DeviceGuard g(ctx->c.device);
    return oct::zsort_apply(ctx->c, tree->t, in, out, n, row_bytes, direction);
}

OCT_API int oct_permute_rows(oct_ctx* ctx, const int32_t* perm, int64_t n, const void* in, void* out,
                             int64_t row_bytes, int direction) {
    if (!ctx) return OCT_ERR_ARGUMENT;
    ctx->c.last_error.clear();
    DeviceGuard g(ctx->c.device);
    return oct::permute_rows(ctx->c, perm, n, in, out, row_bytes, direction);
}

OCT_API int oct_neighbors(oct_ctx* ctx, const oct_tree* target, const void* query_coords, int64_t n_queries,
                          int32_t* out_counts, int32_t* out_indices, int64_t cap_per_query) {
    if (!ctx || !target) return OCT_ERR_ARGUMENT;
    ctx->c.last_error.clear();
    if (n_queries < 0 || cap_per_query < 0) return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "negative size");
    if (n_queries > 0 && (!query_coords || !out_counts || (cap_per_query > 0 && !out_indices)))
        return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "NULL buffer");
    if (!target->t.built) return oct::set_error(ctx->c, OCT_ERR_STATE, "target tree has not been built");
    if (target->t.n_clouds > 0) return oct::set_error(ctx->c, OCT_ERR_STATE, "neighbor queries need a single-set tree");
    DeviceGuard g(ctx->c.device);
    return oct::neighbors_of(ctx->c, target->t, query_coords, n_queries, out_counts, out_indices, cap_per_query);
}

OCT_API int oct_edges_diff_backward(oct_ctx* ctx, int ndims, int dtype, int64_t n_points, int64_t n_edges,
                                    const int32_t* senders, const int32_t* receivers, const void* rel_displacement,
                                    const void* rel_dist_norm, const void* d_rel_displacement,
                                    const void* d_rel_dist_norm, double radius, void* grad_coords) {
    if (!ctx) return OCT_ERR_ARGUMENT;
    ctx->c.last_error.clear();
    if (bad_dims(ndims) || bad_dtype(dtype)) return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "bad ndims/dtype");
    if (n_points < 0 || n_edges < 0 || n_edges > 2147483647LL || n_points > 2147483647LL)
        return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "sizes must fit Int32");
    if (!(radius > 0.0)) return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "radius must be positive");
    if (n_points > 0 && !grad_coords) return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "grad_coords is NULL");
    if (n_edges > 0 && (!senders || !receivers || !rel_displacement || !rel_dist_norm))
        return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "edge array is NULL");
    DeviceGuard g(ctx->c.device);
    return oct::diff_backward(ctx->c, ndims, dtype, n_points, n_edges, senders, receivers, rel_displacement,
                              rel_dist_norm, d_rel_displacement, d_rel_dist_norm, radius, grad_coords, nullptr,
                              nullptr);
}

OCT_API int oct_edges_diff_backward_pair(oct_ctx* ctx, int ndims, int dtype, int64_t n_query, int64_t n_target,
                                         int64_t n_edges, const int32_t* senders, const int32_t* receivers,
                                         const void* rel_displacement, const void* rel_dist_norm,
                                         const void* d_rel_displacement, const void* d_rel_dist_norm, double radius,
                                         void* grad_query, void* grad_target) {
    if (!ctx) return OCT_ERR_ARGUMENT;
    ctx->c.last_error.clear();
    if (bad_dims(ndims) || bad_dtype(dtype)) return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "bad ndims/dtype");
    if (n_query < 0 || n_target < 0 || n_edges < 0 || n_edges > 2147483647LL || n_query > 2147483647LL ||
        n_target > 2147483647LL)
        return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "sizes must fit Int32");
    if (!(radius > 0.0)) return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "radius must be positive");
    if ((n_query > 0 && !grad_query) || (n_target > 0 && !grad_target))
        return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "gradient output is NULL");
    if (n_edges > 0 && (!senders || !receivers || !rel_displacement || !rel_dist_norm))
        return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "edge array is NULL");
    DeviceGuard g(ctx->c.device);
    return oct::diff_backward_pair(ctx->c, ndims, dtype, n_query, n_target, n_edges, senders, receivers,
                                   rel_displacement, rel_dist_norm, d_rel_displacement, d_rel_dist_norm, radius,
                                   grad_query, grad_target);
}

OCT_API int oct_edges_diff_backward_recompute(oct_ctx* ctx, int ndims, int dtype, int64_t n_points,
                                              int64_t n_edges, const int32_t* senders, const int32_t* receivers,
                                              const void* coords, const void* d_rel_displacement,
                                              const void* d_rel_dist_norm, double radius, void* grad_coords) {
    if (!ctx) return OCT_ERR_ARGUMENT;
    ctx->c.last_error.clear();
    if (bad_dims(ndims) || bad_dtype(dtype)) return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "bad ndims/dtype");
    if (n_points < 0 || n_edges < 0 || n_edges > 2147483647LL || n_points > 2147483647LL)
        return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "sizes must fit Int32");
    if (!(radius > 0.0)) return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "radius must be positive");
    if (n_points > 0 && (!grad_coords || !coords))
        return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "coords/grad_coords is NULL");
    if (n_edges > 0 && (!senders || !receivers))
        return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "edge array is NULL");
    DeviceGuard g(ctx->c.device);
    return oct::diff_backward(ctx->c, ndims, dtype, n_points, n_edges, senders, receivers, nullptr, nullptr,
                              d_rel_displacement, d_rel_dist_norm, radius, grad_coords, coords, nullptr);
}

OCT_API int oct_edges_diff_backward_ordered(oct_ctx* ctx, int ndims, int dtype, int64_t n_points, int64_t n_edges,
                                            const int32_t* senders, const int32_t* receivers,
                                            const void* rel_displacement, const void* rel_dist_norm,
                                            const void* coords, const void* d_rel_displacement,
                                            const void* d_rel_dist_norm, double radius, void* grad_coords,
                                            const int32_t* order) {
    if (!ctx) return OCT_ERR_ARGUMENT;
    ctx->c.last_error.clear();
    if (bad_dims(ndims) || bad_dtype(dtype)) return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "bad ndims/dtype");
    if (n_points < 0 || n_edges < 0 || n_edges > 2147483647LL || n_points > 2147483647LL)
        return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "sizes must fit Int32");
    if (!(radius > 0.0)) return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "radius must be positive");
    if (n_points > 0 && !grad_coords) return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "grad_coords is NULL");
    if (n_edges > 0 && (!senders || !receivers))
        return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "edge array is NULL");
    if (n_points > 0 && !coords && n_edges > 0 && (!rel_displacement || !rel_dist_norm))
        return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "give either the features or coords");
    DeviceGuard g(ctx->c.device);
    return oct::diff_backward(ctx->c, ndims, dtype, n_points, n_edges, senders, receivers,
                              coords ? nullptr : rel_displacement, coords ? nullptr : rel_dist_norm,
                              d_rel_displacement, d_rel_dist_norm, radius, grad_coords, coords, order);
}

OCT_API int oct_ctx_set_option(oct_ctx* ctx, int option, int64_t value) {
    if (!ctx) return OCT_ERR_ARGUMENT;
    oct::Ctx& c = ctx->c;
    c.last_error.clear();
    switch (option) {
        case OCT_OPT_WAIT_LIMIT:
            if (value < 0) return oct::set_error(c, OCT_ERR_ARGUMENT, "wait limit must be >= 0");
            c.wait_limit = value;
            return OCT_OK;
        case OCT_OPT_NODE_CAPACITY:
            if (value < 0 || value > 2147483647LL)
                return oct::set_error(c, OCT_ERR_ARGUMENT, "node capacity must be in [0, 2^31 - 1]");
            c.node_cap_override = value;
            return OCT_OK;
        case OCT_OPT_RECORD_CAP:
            if (value < 0) return oct::set_error(c, OCT_ERR_ARGUMENT, "record count must be >= 0");
            c.rec_cap_override = value;
            return OCT_OK;
        case OCT_OPT_GUARD_CHECK:
            c.guard_check = value != 0;
            return OCT_OK;
        case OCT_OPT_WITHHOLD_TILE:
            if (value < -1 || value > 2147483647LL)
                return oct::set_error(c, OCT_ERR_ARGUMENT, "withheld tile must be -1 or a tile index");
            c.withhold_tile = (int32_t)value;
            return OCT_OK;
        case OCT_OPT_MAX_SEG:
            if (value < 0 || value > 16) return oct::set_error(c, OCT_ERR_ARGUMENT, "max_seg must be in [0, 16]");
            c.tune_force.max_seg = (int)value;
            return OCT_OK;
        case OCT_OPT_MULTI_POP:
            if (value < 0 || value > 4) return oct::set_error(c, OCT_ERR_ARGUMENT, "multi_pop must be in [0, 4]");
            c.tune_force.multi_pop = (int)value;
            return OCT_OK;
        case OCT_OPT_FILL_CHUNK:  // 0 = table, 1 = direct stores, else the bulk-copy chunk
            if (value != 0 && value != 1 && value != 32 && value != 64 && value != 128)
                return oct::set_error(c, OCT_ERR_ARGUMENT, "fill_chunk must be 0, 1, 32, 64 or 128");
            c.tune_force.fill_chunk = (int)value;
            return OCT_OK;
        case OCT_OPT_GROUP_CAP:
            if (value != 0 && (value < 8 || value > 32))
                return oct::set_error(c, OCT_ERR_ARGUMENT, "group_cap must be 0 or in [8, 32]");
            c.tune_force.group_cap = (int)value;
            return OCT_OK;
        case OCT_OPT_SUB_BOXES:
            if (value != 0 && value != 1 && value != 2 && value != 4)
                return oct::set_error(c, OCT_ERR_ARGUMENT, "sub_boxes must be 0, 1, 2 or 4");
            c.tune_force.sub_boxes = (int)value;
            return OCT_OK;
        case OCT_OPT_PREFETCH:  // 0 = table, 1 = off, 2 = on
            if (value < 0 || value > 2) return oct::set_error(c, OCT_ERR_ARGUMENT, "prefetch must be 0, 1 or 2");
            c.tune_force.prefetch = (int)value;
            return OCT_OK;
        default:
            return oct::set_error(c, OCT_ERR_ARGUMENT, "unknown or read-only option");
    }
}

OCT_API int oct_ctx_get_option(const oct_ctx* ctx, int option, int64_t* value) {
    if (!ctx || !value) return OCT_ERR_ARGUMENT;
    const oct::Ctx& c = ctx->c;
    switch (option) {
        case OCT_OPT_WAIT_LIMIT: *value = c.wait_limit; return OCT_OK;
        case OCT_OPT_NODE_CAPACITY: *value = c.node_cap_override; return OCT_OK;
        case OCT_OPT_RECORD_CAP: *value = c.rec_cap_override; return OCT_OK;
        case OCT_OPT_GUARD_CHECK: *value = c.guard_check ? 1 : 0; return OCT_OK;
        case OCT_OPT_WITHHOLD_TILE: *value = c.withhold_tile; return OCT_OK;
        case OCT_OPT_MAX_SEG: *value = c.tune_force.max_seg; return OCT_OK;
        case OCT_OPT_MULTI_POP: *value = c.tune_force.multi_pop; return OCT_OK;
        case OCT_OPT_FILL_CHUNK: *value = c.tune_force.fill_chunk; return OCT_OK;
        case OCT_OPT_GROUP_CAP: *value = c.tune_force.group_cap; return OCT_OK;
        case OCT_OPT_SUB_BOXES: *value = c.tune_force.sub_boxes; return OCT_OK;
        case OCT_OPT_PREFETCH: *value = c.tune_force.prefetch; return OCT_OK;
        case OCT_STAT_TUNING_ROW: *value = c.last_tune_row; return OCT_OK;
        case OCT_STAT_BUILD_ATTEMPTS: *value = c.last_attempts; return OCT_OK;
        case OCT_STAT_RECORD_OVERFLOW: *value = c.rec_overflow; return OCT_OK;
        case OCT_STAT_RECORD_CAP: *value = c.rec_cap; return OCT_OK;
        default: return OCT_ERR_ARGUMENT;
    }
}

OCT_API int oct_ctx_load_tuning(oct_ctx* ctx, const char* path) {
    if (!ctx) return OCT_ERR_ARGUMENT;
    ctx->c.last_error.clear();
    if (!path || !*path) {
        ctx->c.tune_table.clear();
        return OCT_OK;
    }
    std::vector<oct::TuneRow> rows;
    std::string err;
    if (!oct::parse_tuning(path, rows, err)) return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, err);
    ctx->c.tune_table.swap(rows);
    return OCT_OK;
}

OCT_API int oct_tuning_select(const char* path, int ndims, int dtype, int64_t n, double nbrs_per_point,
                              int32_t* shapes, int32_t* row) {
    if (!path || !shapes || !row) return OCT_ERR_ARGUMENT;
    std::vector<oct::TuneRow> rows;
    std::string err;
    if (*path && !oct::parse_tuning(path, rows, err)) return OCT_ERR_ARGUMENT;
    oct::Tuning tn;
    *row = oct::select_tuning(rows, ndims, dtype, n, nbrs_per_point, tn);
    shapes[0] = tn.max_seg;
    shapes[1] = tn.multi_pop;
    shapes[2] = tn.fill_chunk;
    shapes[3] = tn.group_cap;
    shapes[4] = tn.sub_boxes;
    shapes[5] = tn.prefetch;
    return OCT_OK;
}

OCT_API int oct_edges_diff_backward_mirror(oct_ctx* ctx, int ndims, int dtype, int64_t n_points, int64_t n_edges,
                                           const int32_t* senders, const int32_t* receivers, const int32_t* mirror,
                                           const void* rel_displacement, const void* rel_dist_norm,
                                           const void* coords, const void* d_rel_displacement,
                                           const void* d_rel_dist_norm, double radius, void* grad_coords,
                                           const int32_t* order) {
    if (!ctx) return OCT_ERR_ARGUMENT;
    ctx->c.last_error.clear();
    if (bad_dims(ndims) || bad_dtype(dtype)) return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "bad ndims/dtype");
    if (n_points < 0 || n_edges < 0 || n_edges > 2147483647LL || n_points > 2147483647LL)
        return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "sizes must fit Int32");
    if (!(radius > 0.0)) return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "radius must be positive");
    if (n_points > 0 && !grad_coords) return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "grad_coords is NULL");
    if (n_edges > 0 && (!senders || !receivers || !mirror))
        return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "edge array is NULL");
    if (n_points > 0 && !coords && n_edges > 0 && (!rel_displacement || !rel_dist_norm))
        return oct::set_error(ctx->c, OCT_ERR_ARGUMENT, "give either the features or coords");
    DeviceGuard g(ctx->c.device);
    return oct::diff_backward_mirror(ctx->c, ndims, dtype, n_points, n_edges, senders, receivers, mirror,
                                     coords ? nullptr : rel_displacement, coords ? nullptr : rel_dist_norm, coords,
                                     d_rel_displacement, d_rel_dist_norm, radius, grad_coords, order);
}

static const char* kPhaseNames[oct::PH_NUM] = {"bounds", "encode", "sort", "gather", "topology",
                                               "refit", "count", "scan", "fill", "adjoint", "groups"};

OCT_API int oct_profile_enable(oct_ctx* ctx, int on) {
    if (!ctx) return OCT_ERR_ARGUMENT;
    ctx->c.profiling = on != 0;
    return OCT_OK;
}

OCT_API const char* oct_profile_phase_name(int phase) {
    return (phase >= 0 && phase < oct::PH_NUM) ? kPhaseNames[phase] : "";
}

OCT_API int64_t oct_profile_kernel_launches(const oct_ctx* ctx) { return ctx ? ctx->c.kernel_launches : 0; }

OCT_API int oct_profile_read(oct_ctx* ctx, double* ms, int64_t* launches, int n_phases) {
    if (!ctx) return OCT_ERR_ARGUMENT;
    DeviceGuard g(ctx->c.device);
    cudaError_t e = cudaStreamSynchronize(ctx->c.stream);
    if (e != cudaSuccess) return oct::cuda_status(ctx->c, e, "profile read");
    for (int i = 0; i < n_phases; ++i) {
        if (ms) ms[i] = 0.0;
        if (launches) launches[i] = 0;
    }
    for (auto& r : ctx->c.prof) {
        float t = 0.f;
        cudaEventElapsedTime(&t, r.start, r.stop);
        if (r.phase < n_phases) {
            if (ms) ms[r.phase] += t;
            if (launches) launches[r.phase] += 1;
        }
        ctx->c.event_pool.push_back(r.start);
        ctx->c.event_pool.push_back(r.stop);
    }
    ctx->c.prof.clear();
    return OCT_OK;
}

}  // extern "C"
