// Library-internal objects shared by the build, edge and C-ABI translation units.
#pragma once

#include <chrono>
#include <cstdint>
#include <string>
#include <vector>
#include <cuda_runtime.h>

#include "common.cuh"

namespace oct {

// Grow-only device allocation.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    template <class T> T* as() const { return static_cast<T*>(p); }
};

cudaError_t ensure(DevBuf& b, size_t bytes);
void release(DevBuf& b);

struct Ctx;

// Kernel shapes chosen per workload by the autotuner (octopus.jl_b200/tune.py).
// No result depends on them: they change how the work is cut, not what is
// computed.
struct Tuning {
    int max_seg = 16;     // leaves sharing one staged chunk of the traversal (1..16)
    int multi_pop = 4;    // internal nodes expanded together by the traversal (1..4)
    int fill_chunk = 0;   // the fill's stores: 0 direct, else bulk copies of chunks of 32, 64 or 128 edges
    int group_cap = 32;   // query points per traversal group, set at the build (8..32)
    int sub_boxes = 1;    // boxes a group's queries are split into for the target test (1, 2 or 4)
    int prefetch = 0;     // 1: the traversal prefetches the next chunk's points / children into L1
};

// One row of a tuning table: the shapes measured best for point sets of
// about 2^nlog2 points with about 2^nbr_log2 - 1 neighbors per point.
struct TuneRow {
    int ndims, dtype, nlog2, nbr_log2;
    Tuning tn;
};

// Parses a tuning table (one row per line: ndims dtype nlog2 nbr_log2 max_seg
// multi_pop fill_chunk group_cap [sub_boxes [prefetch]]; '#' starts a comment).  Returns false when
// the file cannot be read or a row is malformed.  A ninth value, sub_boxes,
// and a tenth, prefetch, are optional (1 and 0 when absent).
bool parse_tuning(const char* path, std::vector<TuneRow>& rows, std::string& err);
// The row nearest to (n, neighbors per point) among those of the same ndims
// and dtype (index into rows, -1 when none), and its shapes (defaults when none).
int select_tuning(const std::vector<TuneRow>& rows, int ndims, int dtype, int64_t n, double nbrs, Tuning& out);

// Phases timed by the optional CUDA-event profiler (oct_profile_*).
enum Phase : int {
    PH_BOUNDS = 0, PH_ENCODE, PH_SORT, PH_GATHER, PH_TOPOLOGY, PH_REFIT,
    PH_COUNT, PH_SCAN, PH_FILL, PH_ADJOINT, PH_GROUPS, PH_NUM
};

struct ProfRecord {
    int phase;
    cudaEvent_t start, stop;
};

// Records one phase between its constructor and destructor when profiling
// is on; otherwise does nothing.
struct PhaseTimer {
    Ctx* ctx;
    int phase;
    cudaEvent_t start = nullptr;
    PhaseTimer(Ctx& c, int ph);
    ~PhaseTimer();
};

// One point set's search structure (the reference's Octree + permutation +
// morton_codes, src/types.jl:23-42 and src/types.jl:153-154).
struct Tree {
    int ndims = 3;
    int dtype = 0;          // 0 = float32, 1 = float64
    int64_t n = 0;
    double radius = 0.0;
    int32_t leaf_size = kLeafSize;
    int32_t group_cap = 32;  // query points per traversal group of the last build
    bool built = false;
    bool keep_morton = false;
    uint64_t generation = 0;

    // Build results (host copies, valid after a successful build).
    int key_bytes = 4;
    int key_bits = 0;
    int sort_passes = 0;
    int64_t n_nodes = 0;
    int64_t capacity = 0;    // node capacity of the node arrays
    int n_mark_blocks = 0;
    double origin[3] = {0, 0, 0};

    // Device storage.
    DevBuf keys[2], vals[2];     // radix-sort ping-pong
    DevBuf hist;                 // radix digit histograms (+1 total slot)
    DevBuf sort_tmp;             // int64 tile sums of the histogram scan
    DevBuf look;                 // one-pass-per-digit sort: digit counts and tile look-back words
    DevBuf spts;                 // SPt<T,D>[n] in Morton order
    DevBuf spts_tmp;             // SPt<T,D>[n]: the key sort's intermediate passes
    DevBuf iperm;                // int32 [n]: sorted position of each original point
    // iperm holds the inverse of the current order (a full sort leaves it to
    // the first caller that needs it: ensure_iperm)
    mutable bool iperm_valid = false;
    const int32_t* perm_dev = nullptr;  // original index of each sorted position (null: identity)
    const void* skeys_dev = nullptr;    // sorted keys of the last build (key_bytes wide)
    DevBuf tnode;                // TNode<T,D>[capacity]
    DevBuf nrange;               // int2 {first,last} 0-based per node
    DevBuf parent;               // int32 per node (-1 for the root)
    DevBuf fchild;               // int32 per node: first child id from the id pass
    DevBuf arrive;               // int32 per node, refit arrival counters
    DevBuf lohi;                 // uint16 per position: first | last level starting here
    DevBuf blockcnt;             // int32 [(maxlev+1) * n_mark_blocks]
    DevBuf blockoff;             // int64 exclusive scan of blockcnt (+1)
    DevBuf scan_tmp;             // int64 tile sums for scans
    DevBuf partials;             // double per-block bounds partials
    DevBuf hdr;                  // OctHeader
    DevBuf morton;               // uint64 per original point (refit mode), filled with the views
    DevBuf groups;               // int2 {first position, count <= 32}: query groups
    DevBuf gstart;               // int32 per group: traversal start node (| 1 << 30: ascending flag), -1 = root
    int64_t n_groups = 0;
    int32_t dfs_start = 0;
    DevBuf chain;                // int32[64]: full-range chain node ids and flags

    // Refit mode across time steps: the previous build's sorted keys and
    // permutation (keys[sorted_buf], vals[sorted_buf]) seed the next build.
    int sorted_buf = -1;         // -1: no reusable order
    int64_t sorted_n = 0;
    double sorted_radius = 0.0;
    int sorted_key_bytes = 0;
    DevBuf rflag;                // uint8 per position: key changed
    DevBuf rcnt, roff;           // int32 per block / int64 scan (+1)
    DevBuf mkeys, mvals;         // changed keys, sorted in chunks
    DevBuf mkeys2, mvals2;       // changed keys, fully sorted
    int last_path = 0;           // 0 full sort, 1 merge of changed keys, 2 bounds only
    int64_t last_moved = -1;

    // Batched build (many clouds in one forest); n_clouds == 0 otherwise.
    int32_t n_clouds = 0;
    int32_t kbits = 0;
    // Neighbors per point of this tree's last count as a query set (-1 before
    // the first), which keys the tuning table.
    mutable double nbrs_hint = -1.0;
    DevBuf b_coff;               // int64 [n_clouds + 1]
    DevBuf b_cparam;             // double [n_clouds * kCloudParams]
    DevBuf b_croot, b_cstart;    // int32 [n_clouds]
    DevBuf b_cbounds;            // double [n_clouds * 8] per-cloud reduce
    DevBuf b_eoff;               // int64 [n_clouds + 1] per-cloud edge offsets
    Batch batch() const {
        Batch b;
        b.n_clouds = n_clouds;
        b.kbits = kbits;
        b.coff = b_coff.as<int64_t>();
        b.cparam = b_cparam.as<double>();
        b.croot = b_croot.as<int32_t>();
        b.cstart = b_cstart.as<int32_t>();
        return b;
    }
    int64_t group_capacity = 0;
    OctHeader* hdr_host = nullptr;  // pinned

    // Lazily materialized reference-layout views (DeviceView contract,
    // ext/OctopusCUDAExt.jl:23-35).
    bool view_valid = false;
    DevBuf v_first, v_last, v_children, v_bmin, v_bmax, v_perm;
};

struct Ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string last_error;
    // Edge-count state carried from oct_edges_count to oct_edges_fill.
    DevBuf counts;       // int32 per query point
    DevBuf offsets;      // int64 per query point + 1
    DevBuf scan_tmp;     // int64 tile sums
    DevBuf total;        // int64 device total, then the count of overflowed record groups
    DevBuf dstatus;      // int32 device error word set by kernels (bounds guards)
    int64_t* total_host = nullptr;  // pinned
    const Tree* plan_query = nullptr;
    const Tree* plan_target = nullptr;
    uint64_t plan_qgen = 0, plan_tgen = 0;
    int plan_exclude = -1;
    int64_t plan_edges = -1;
    // Hit records of the last count (edges.cu): rec_cap records per query
    // point (0 when the count did not record), rcount per query, gflag per
    // query group whose records overflowed (rec_overflow of them).
    DevBuf recs, rcount, gflag;
    int64_t rec_cap = 0;
    int64_t rec_cap_hint = 32;
    int64_t rec_edges_hint = 0;    // edge total of the last recording count
    int64_t rec_overflow = 0;
    // Adjoint scratch (diff.cu).
    DevBuf dkeys[2], dvals[2], dhist, dsort_tmp, droff, dsoff;
    DevBuf dredge;       // edges ordered by receiver (adjoint of a COO not grouped by receiver)
    DevBuf dterm;        // per-edge cotangent term of the searching self-pair adjoint (4 values)
    DevBuf dseg;         // per-point {first, end} edge of the self-pair adjoint
    DevBuf tstats;       // traversal statistics (oct_edges_traversal_stats)
    // Options (oct_ctx_set_option): the polling rounds of a bounded device
    // wait; a node capacity for each build's first topology attempt (0 =
    // estimate); hit records per query point (0 = automatic); canary regions
    // after the sort buffers and node arrays, checked after each topology
    // attempt; a look-back tile that never publishes (a test aid, -1 = off).
    int64_t wait_limit = 1 << 22;
    int64_t node_cap_override = 0;
    int64_t rec_cap_override = 0;
    bool guard_check = false;
    int32_t withhold_tile = -1;
    int32_t last_attempts = 0;    // topology attempts of the last build
    // Tuning: the table (oct_ctx_load_tuning), shapes forced by options
    // (0 = from the table), the shapes of the last count (used by its fill)
    // and the table row they came from (-1 = defaults).
    std::vector<TuneRow> tune_table;
    Tuning tune_force{0, 0, 0, 0, 0, 0};
    Tuning plan_tuning;
    int last_tune_row = -1;
    Tuning tuning_for(int ndims, int dtype, int64_t n, double nbrs);
    // Profiler.
    int64_t kernel_launches = 0;  // every kernel this context has launched
    bool profiling = false;
    std::vector<ProfRecord> prof;
    std::vector<cudaEvent_t> event_pool;
    cudaEvent_t get_event();
};

// Waits for the work queued on `s` by polling it: the library's host round
// trips (bounds, node count, edge count) sit between short kernels, where a
// blocking synchronize would add the host thread's wake-up latency each
// time.  After 200 ms of polling it blocks instead.
inline cudaError_t wait_stream(cudaStream_t s) {
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        const cudaError_t e = cudaStreamQuery(s);
        if (e != cudaErrorNotReady) return e;
        if (std::chrono::steady_clock::now() - t0 > std::chrono::milliseconds(200)) return cudaStreamSynchronize(s);
    }
}

// Build pipeline (build.cu).  Returns a Status.
int build_tree(Ctx& ctx, Tree& t, const void* coords, int64_t n, double radius);
int build_tree_batch(Ctx& ctx, Tree& t, const void* coords, int64_t n, const int64_t* coff_host,
                     const double* radii_host, int32_t n_clouds);
int batch_edge_offsets(Ctx& ctx, Tree& t, int64_t* out_host);
int materialize_view(Ctx& ctx, Tree& t);

// Edge pipeline (edges.cu).
int edges_count(Ctx& ctx, const Tree& q, const Tree& t, bool exclude_self, int64_t* n_edges);
int edges_fill(Ctx& ctx, const Tree& q, const Tree& t, bool exclude_self, int32_t* senders,
               int32_t* receivers, void* rel_disp, void* rel_dist, int64_t n_edges);
int edges_fill_diff(Ctx& ctx, const Tree& t, int32_t* senders, int32_t* receivers, void* rel_disp, void* rel_dist,
                    int32_t* mirror, int64_t n_edges);
// The inverse permutation of a built tree, computed on first use after a
// full sort (the build itself does not need it).
int ensure_iperm(Ctx& ctx, const Tree& t);
int edges_mirror_scan(Ctx& ctx, const int32_t* snd, const int32_t* rcv, int64_t m, int64_t n, const int64_t* off,
                      int32_t* mirror);
int traversal_stats(Ctx& ctx, const Tree& q, const Tree& t, bool exclude_self, uint64_t* out, int n_out);
int neighbors_of(Ctx& ctx, const Tree& t, const void* qcoords, int64_t nsel, int32_t* out_counts,
                 int32_t* out_idx, int64_t cap);
cudaError_t count_into(const Tree& q, const Tree& t, bool exclude_self, int32_t* counts, cudaStream_t s);
int csr_fill(Ctx& ctx, const Tree& q, const Tree& t, bool exclude_self, int32_t* offsets, int32_t* flat,
             int64_t capacity);

// Permutation of user arrays by a built tree (zsort.cu).
int zsort_apply(Ctx& ctx, const Tree& t, const void* in, void* out, int64_t n, int64_t row_bytes, int direction);
int permute_rows(Ctx& ctx, const int32_t* perm, int64_t n, const void* in, void* out, int64_t row_bytes,
                 int direction);

// Adjoint (diff.cu).
int diff_backward(Ctx& ctx, int ndims, int dtype, int64_t n_points, int64_t n_edges,
                  const int32_t* senders, const int32_t* receivers, const void* rel_disp,
                  const void* rel_dist, const void* d_disp, const void* d_dist, double radius,
                  void* grad, const void* coords, const int32_t* order);
int diff_backward_mirror(Ctx& ctx, int ndims, int dtype, int64_t n, int64_t m, const int32_t* snd,
                         const int32_t* rcv, const int32_t* mirror, const void* rel_disp, const void* rel_dist,
                         const void* coords, const void* d_disp, const void* d_dist, double radius, void* grad,
                         const int32_t* order);
int diff_backward_pair(Ctx& ctx, int ndims, int dtype, int64_t nq, int64_t nt, int64_t m, const int32_t* snd,
                       const int32_t* rcv, const void* rel_disp, const void* rel_dist, const void* d_disp,
                       const void* d_dist, double radius, void* grad_q, void* grad_t);

int set_error(Ctx& ctx, int status, const std::string& msg);
int cuda_status(Ctx& ctx, cudaError_t e, const char* where);

}  // namespace oct
