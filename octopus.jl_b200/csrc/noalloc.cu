// Edge count that allocates no device memory.
//
// Some callers cannot let a library call cudaMalloc: a host whose device
// memory is owned by its own pool allocator (a framework's caching allocator,
// a service with a fixed memory budget) where a raw cudaMalloc can fail on a
// full device or fragment the pool, and latency-critical time-stepping loops
// where the implicit device synchronization of cudaMalloc/cudaFree is not
// acceptable.  oct_edges_count_noalloc serves them: the caller passes the
// per-query counts and the offsets as outputs, and the only scratch -- the
// scan's per-tile sums and total -- lives in the fixed array below, which
// every GPU that loads this library holds until the process exits.
#include <cstdint>
#include <mutex>

#include "../../include/octopus_b200.h"
#include "capi_types.h"
#include "internal.h"
#include "scan.cuh"

namespace {

// Largest query set the fixed scratch can scan.
constexpr int64_t kNoAllocMaxQueries = 1LL << 24;  // 16,777,216
constexpr int64_t kNoAllocTiles = (kNoAllocMaxQueries + oct::kScanTile - 1) / oct::kScanTile;  // 8192

// Scan scratch: kNoAllocTiles per-tile sums followed by the total
// (8 B each: 64 KiB + 8 B per device).  Each call overwrites the entries it
// reads before reading them, so nothing has to start at zero.
static __device__ __align__(256) int64_t g_count_scratch[kNoAllocTiles + 1];

// Device address of g_count_scratch, looked up once per device.  In host
// code the symbol's name is only a stand-in for the device array, so kernels
// must be given this address instead.  The cached address belongs to the
// device's primary context: it does not survive cudaDeviceReset (nor a
// primary-context reset by another library in the process), after which this
// entry point must not be called again in the same process.
constexpr int kMaxDevices = 64;
int64_t* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mu;

cudaError_t scratch_address(int device, int64_t** out) {
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_count_scratch);  // the device is current here
        if (e != cudaSuccess) return e;
        g_scratch_addr[device] = static_cast<int64_t*>(p);
    }
    *out = g_scratch_addr[device];
    return cudaSuccess;
}

struct CurrentDevice {
    int prev = -1;
    explicit CurrentDevice(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~CurrentDevice() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

}  // namespace

extern "C" OCT_API int oct_edges_count_noalloc(oct_ctx* ctx, const oct_tree* query, const oct_tree* target,
                                               int exclude_self, int32_t* counts, int64_t* offsets,
                                               int64_t* n_edges) {
    if (!ctx) return OCT_ERR_ARGUMENT;
    oct::Ctx& c = ctx->c;
    c.last_error.clear();
    if (n_edges) *n_edges = 0;
    // The same rules as oct_edges_count, the batched-tree rule included.
    const int st = oct_check_count_pair(ctx, query, target, exclude_self);
    if (st != OCT_OK) return st;
    const oct::Tree& q = query->t;
    const oct::Tree& t = target->t;
    if (q.n > kNoAllocMaxQueries)
        return oct::set_error(c, OCT_ERR_CAPACITY,
                              "oct_edges_count_noalloc: the query set has more than 16,777,216 points, the "
                              "limit of its fixed scratch; use oct_edges_count");
    if (!offsets || (q.n > 0 && !counts))
        return oct::set_error(c, OCT_ERR_ARGUMENT, "counts/offsets output is NULL");
    CurrentDevice guard(c.device);
    cudaError_t e;
    if (n_edges) {
        // Reading the total back means a host copy and a stream synchronize,
        // neither of which a stream being captured allows.
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if ((e = cudaStreamIsCapturing(c.stream, &cs)) != cudaSuccess)
            return oct::cuda_status(c, e, "cudaStreamIsCapturing");
        if (cs != cudaStreamCaptureStatusNone)
            return oct::set_error(c, OCT_ERR_STATE,
                                  "oct_edges_count_noalloc: n_edges must be NULL while the stream is being captured "
                                  "(the total is offsets[n_query])");
    }
    int64_t* scratch = nullptr;
    e = scratch_address(c.device, &scratch);
    if (e != cudaSuccess) return oct::cuda_status(c, e, "cudaGetSymbolAddress(scan scratch)");
    if ((e = oct::count_into(q, t, exclude_self != 0, counts, c.stream)) != cudaSuccess)
        return oct::cuda_status(c, e, "edge count launch");
    oct::exclusive_scan_i32_i64(counts, offsets, q.n, scratch + kNoAllocTiles, scratch, c.stream);
    if ((e = cudaGetLastError()) != cudaSuccess) return oct::cuda_status(c, e, "edge count scan");
    if (n_edges) {
        int64_t total = 0;
        if ((e = cudaMemcpyAsync(&total, offsets + q.n, sizeof(int64_t), cudaMemcpyDeviceToHost, c.stream)) !=
                cudaSuccess ||
            (e = cudaStreamSynchronize(c.stream)) != cudaSuccess)
            return oct::cuda_status(c, e, "edge count total");
        *n_edges = total;
    }
    return OCT_OK;
}
