// Stable LSD radix sort of (key, int32 value) pairs on 8-bit digits.
#pragma once

#include <algorithm>

#include <cuda/atomic>

#include "common.cuh"
#include "scan.cuh"

namespace oct {

constexpr int kSortThreads = 256;
// Stable LSD radix sort on 8-bit digits: per-tile histogram, one scan of the
// digit-major histogram, then a stable scatter that ranks equal digits with
// warp match and per-warp shared-memory counters.
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;  // 2048 keys per tile

template <class K>
static __global__ void __launch_bounds__(kSortThreads) k_hist(const K* __restrict__ keys, int64_t n, int shift,
                                                   int32_t* __restrict__ hist, int ntiles) {
    __shared__ int32_t cnt[256];
    cnt[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kSortTile;
#pragma unroll
    for (int it = 0; it < kSortItems; ++it) {
        const int64_t i = base + it * kSortThreads + threadIdx.x;
        if (i < n) atomicAdd(&cnt[(unsigned)(keys[i] >> shift) & 255u], 1);
    }
    __syncthreads();
    hist[(int64_t)threadIdx.x * ntiles + blockIdx.x] = cnt[threadIdx.x];
}

// Stable scatter of one tile: each key's rank among the tile's keys of its
// digit (warp match within a warp, per-warp counters across warps), then the
// tile is staged in shared memory in digit order so that each digit's run is
// written to global memory by consecutive threads (whole sectors instead of
// one scattered store per key).
template <class K>
static __global__ void __launch_bounds__(kSortThreads) k_scatter(const K* __restrict__ kin, const int32_t* __restrict__ vin,
                                                      K* __restrict__ kout, int32_t* __restrict__ vout, int64_t n,
                                                      int shift, const int32_t* __restrict__ hoff, int ntiles) {
    __shared__ int32_t wc[kSortThreads / 32][256];
    __shared__ int32_t tstart[256];
    __shared__ int32_t scan_sm[kSortThreads / 32 + 1];
    __shared__ K skey[kSortTile];
    __shared__ int32_t sval[kSortTile];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < kSortThreads / 32; ++j) wc[j][threadIdx.x] = 0;
    __syncthreads();
    const int64_t tbase = (int64_t)blockIdx.x * kSortTile;
    const int64_t wbase = tbase + (int64_t)w * (32 * kSortItems);
    K key[kSortItems];
    int32_t val[kSortItems], rk[kSortItems];
    int dg[kSortItems];
#pragma unroll
    for (int it = 0; it < kSortItems; ++it) {
        const int64_t i = wbase + it * 32 + lane;
        const bool valid = i < n;
        key[it] = valid ? kin[i] : K(0);
        val[it] = valid ? (vin ? vin[i] : (int32_t)i) : 0;
        const int d = valid ? (int)((unsigned)(key[it] >> shift) & 255u) : 256;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int leader = __ffs(peers) - 1;
        const int before = __popc(peers & lanemask_lt());
        const int c0 = valid ? wc[w][d] : 0;
        __syncwarp();
        if (valid && lane == leader) wc[w][d] = c0 + __popc(peers);
        __syncwarp();
        rk[it] = c0 + before;
        dg[it] = d;
    }
    __syncthreads();
    // per digit (thread = digit): warp offsets within the tile's run, and the
    // run's start in the tile (exclusive scan over digits)
    int32_t run = 0;
#pragma unroll
    for (int j = 0; j < kSortThreads / 32; ++j) {
        const int32_t c = wc[j][threadIdx.x];
        wc[j][threadIdx.x] = run;
        run += c;
    }
    int32_t tile_total;
    tstart[threadIdx.x] = block_exclusive_scan<int32_t>(run, scan_sm, &tile_total);
    __syncthreads();
#pragma unroll
    for (int it = 0; it < kSortItems; ++it) {
        if (dg[it] < 256) {
            const int lp = tstart[dg[it]] + wc[w][dg[it]] + rk[it];
            skey[lp] = key[it];
            sval[lp] = val[it];
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < tile_total; i += kSortThreads) {
        const K k = skey[i];
        const int d = (int)((unsigned)(k >> shift) & 255u);
        const int64_t dst = (int64_t)hoff[(int64_t)d * ntiles + blockIdx.x] + (i - tstart[d]);
        kout[dst] = k;
        vout[dst] = sval[i];
    }
}


inline int sort_tiles(int64_t n) { return (int)((n + kSortTile - 1) / kSortTile); }
// Histogram buffer: 256 digit counts per tile plus the scan's total slot.
inline size_t sort_hist_bytes(int64_t n) { return (size_t)(256 * (int64_t)sort_tiles(n) + 1) * 4; }
// Scan scratch (int64 tile sums) for the histogram scan.
inline size_t sort_scan_bytes(int64_t n) { return (size_t)scan_tmp_elems(256 * (int64_t)sort_tiles(n)) * 8; }

// Sorts n pairs by the low `bits` bits of the key; 3 to 5 launches per 8-bit
// pass, added to *launches.  Input in (k[0], v[0])
// (v[0] may be null for the identity 0..n-1); returns the index (0 or 1) of
// the buffers holding the result.  With zero passes the result is the input
// and v[0] stays untouched (the caller treats a null value buffer as iota).
template <class K>
int radix_sort_pairs(K* k[2], int32_t* v[2], int32_t* hist, int64_t* scan_tmp, int64_t n, int bits,
                     bool vals_in, cudaStream_t s, int64_t* launches) {
    const int ntiles = sort_tiles(n);
    const int passes = (bits + 7) / 8;
    int src = 0;
    for (int p = 0; p < passes; ++p) {
        const int shift = 8 * p;
        k_hist<K><<<ntiles, kSortThreads, 0, s>>>(k[src], n, shift, hist, ntiles);
        *launches += 2 + exclusive_scan_i32_i32(hist, hist, (int64_t)256 * ntiles, scan_tmp, s);
        k_scatter<K><<<ntiles, kSortThreads, 0, s>>>(k[src], (p == 0 && !vals_in) ? nullptr : v[src], k[src ^ 1],
                                                     v[src ^ 1], n, shift, hist, ntiles);
        src ^= 1;
    }
    return src;
}

// ---------------------------------------------------------------------------
// One launch per digit (decoupled look-back).  k_digit_counts counts every
// pass's digits in one read of the keys; each pass's k_onesweep block then
// takes the next tile (tile ids handed out in the order blocks start, so a
// tile only waits on tiles whose blocks are already running), publishes its
// per-digit counts, and adds those of the tiles before it, walking back until
// a tile that has published its inclusive prefix.  The tile is staged in
// shared memory in digit order and written as contiguous digit runs.  Every
// wait is bounded: a wait that runs out sets DF_TIMEOUT in *status.
constexpr int kOnesweepMaxPasses = 8;
constexpr uint32_t kLookAggregate = 1u << 30;
constexpr uint32_t kLookPrefix = 2u << 30;
constexpr uint32_t kLookValue = (1u << 30) - 1;
// Default number of polling rounds a look-back wait makes before it gives up
// (a context option, OCT_OPT_WAIT_LIMIT, overrides it).
constexpr int64_t kLookSpinLimit = 1 << 22;
// Keys per sort this path takes.  Below ~6M keys its 1 + passes launches beat
// the 5 launches per pass of radix_sort_pairs (measured on B200, 3 passes:
// 0.032 vs 0.035 ms at 100k keys, 0.078 vs 0.083 ms at 1M, 0.179 vs 0.190 ms
// at 4M); above, the tiles' look-back walks cost more than the launches save
// (0.33 vs 0.32 ms at 8M, 0.65 vs 0.57 ms at 16M).  Counts and prefixes are
// 30-bit values, far above this bound.
constexpr int64_t kOnesweepMaxKeys = 6 * 1024 * 1024;

// Scratch words: for each of up to kOnesweepMaxPasses passes 256 digit counts
// and a tile counter, then per pass 256 look-back words per tile; all zero
// before the sort.
inline size_t onesweep_words(int64_t n, int passes) {
    return (size_t)kOnesweepMaxPasses * 257 + (size_t)passes * sort_tiles(n) * 256;
}

template <class K>
static __global__ void __launch_bounds__(kSortThreads) k_digit_counts(const K* __restrict__ keys, int64_t n,
                                                                       int passes, uint32_t* __restrict__ counts) {
    __shared__ uint32_t c[kOnesweepMaxPasses][256];
    for (int p = 0; p < passes; ++p) c[p][threadIdx.x] = 0;
    __syncthreads();
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const K k = keys[i];
        for (int p = 0; p < passes; ++p) atomicAdd(&c[p][(unsigned)(k >> (8 * p)) & 255u], 1u);
    }
    __syncthreads();
    for (int p = 0; p < passes; ++p)
        if (c[p][threadIdx.x]) atomicAdd(&counts[(size_t)p * 257 + threadIdx.x], c[p][threadIdx.x]);
}

template <class K>
static __global__ void __launch_bounds__(kSortThreads) k_onesweep(const K* __restrict__ kin,
                                                                   const int32_t* __restrict__ vin,
                                                                   K* __restrict__ kout, int32_t* __restrict__ vout,
                                                                   int64_t n, int pass, int ntiles,
                                                                   uint32_t* __restrict__ scratch,
                                                                   int* __restrict__ status, int64_t spin_limit,
                                                                   int withhold_tile) {
    __shared__ int32_t wc[kSortThreads / 32][256];
    __shared__ int32_t tstart[256];
    __shared__ int64_t gstart[256];
    __shared__ int32_t scan_sm[kSortThreads / 32 + 1];
    __shared__ K skey[kSortTile];
    __shared__ int32_t sval[kSortTile];
    __shared__ int tile_s;
    const int shift = 8 * pass;
    uint32_t* counts = scratch + (size_t)pass * 257;
    const size_t look_base = (size_t)kOnesweepMaxPasses * 257;  // after every pass's counts and counter
    uint32_t* look = scratch + look_base + (size_t)pass * ntiles * 256;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (threadIdx.x == 0) tile_s = (int)atomicAdd(&counts[256], 1u);
#pragma unroll
    for (int j = 0; j < kSortThreads / 32; ++j) wc[j][threadIdx.x] = 0;
    __syncthreads();
    const int t = tile_s;
    const int64_t wbase = (int64_t)t * kSortTile + (int64_t)w * (32 * kSortItems);
    K key[kSortItems];
    int32_t val[kSortItems], rk[kSortItems];
    int dg[kSortItems];
#pragma unroll
    for (int it = 0; it < kSortItems; ++it) {
        const int64_t i = wbase + it * 32 + lane;
        const bool valid = i < n;
        key[it] = valid ? kin[i] : K(0);
        val[it] = valid ? (vin ? vin[i] : (int32_t)i) : 0;
        const int d = valid ? (int)((unsigned)(key[it] >> shift) & 255u) : 256;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int leader = __ffs(peers) - 1;
        const int before = __popc(peers & lanemask_lt());
        const int c0 = valid ? wc[w][d] : 0;
        __syncwarp();
        if (valid && lane == leader) wc[w][d] = c0 + __popc(peers);
        __syncwarp();
        rk[it] = c0 + before;
        dg[it] = d;
    }
    __syncthreads();
    // thread = digit: warp offsets within the tile's run, the tile's count
    int32_t run = 0;
#pragma unroll
    for (int j = 0; j < kSortThreads / 32; ++j) {
        const int32_t c = wc[j][threadIdx.x];
        wc[j][threadIdx.x] = run;
        run += c;
    }
    const int d = threadIdx.x;
    cuda::atomic_ref<uint32_t, cuda::thread_scope_device> mine(look[(size_t)t * 256 + d]);
    // A withheld tile (a test aid: pass 0, tile `withhold_tile`) never
    // publishes, so the waits of the tiles after it run out.
    const bool publish = !(pass == 0 && t == withhold_tile);
    if (publish) mine.store((t == 0 ? kLookPrefix : kLookAggregate) | (uint32_t)run, cuda::memory_order_relaxed);
    uint32_t excl = 0;
    bool timed_out = false;
    if (t > 0) {
        // Four predecessors per round trip: their words are read together,
        // then added in order up to the first inclusive prefix; a word not
        // yet published stops the round and is read again.
        int j = t - 1;
        int64_t spins = 0;
        while (true) {
            uint32_t v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u)
                v[u] = j - u >= 0 ? cuda::atomic_ref<uint32_t, cuda::thread_scope_device>(look[(size_t)(j - u) * 256 + d])
                                        .load(cuda::memory_order_relaxed)
                                  : kLookPrefix;  // before tile 0: nothing more to add
            int u = 0;
            bool done = false;
            for (; u < 4; ++u) {
                if ((v[u] & ~kLookValue) == 0) break;
                excl += v[u] & kLookValue;
                if ((v[u] & ~kLookValue) == kLookPrefix) {
                    done = true;
                    break;
                }
            }
            if (done) break;
            j -= u;
            if (u < 4) {
                if (++spins > spin_limit) {
                    timed_out = true;
                    break;
                }
                __nanosleep(32);
            }
        }
        if (publish) mine.store(kLookPrefix | (excl + (uint32_t)run), cuda::memory_order_relaxed);
    }
    int32_t tile_total, all;
    tstart[d] = block_exclusive_scan<int32_t>(run, scan_sm, &tile_total);
    const int32_t base = block_exclusive_scan<int32_t>((int32_t)counts[d], scan_sm, &all);
    gstart[d] = (int64_t)base + excl;
    __syncthreads();
#pragma unroll
    for (int it = 0; it < kSortItems; ++it) {
        if (dg[it] < 256) {
            const int lp = tstart[dg[it]] + wc[w][dg[it]] + rk[it];
            skey[lp] = key[it];
            sval[lp] = val[it];
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < tile_total; i += kSortThreads) {
        const K k = skey[i];
        const int dd = (int)((unsigned)(k >> shift) & 255u);
        const int64_t dst = gstart[dd] + (i - tstart[dd]);
        if (dst >= 0 && dst < n) {  // always, unless a wait ran out and left a prefix short
            kout[dst] = k;
            vout[dst] = sval[i];
        } else {
            timed_out = true;
        }
    }
    if (timed_out) atomicOr(status, (int)DF_TIMEOUT);
}

// The same contract as radix_sort_pairs (stable, result in buffers
// (k[r], v[r]) with r returned), for n < kOnesweepMaxKeys; `scratch` holds
// onesweep_words(n, kOnesweepMaxPasses) words.  A look-back wait that ran out
// (after spin_limit polling rounds) leaves DF_TIMEOUT in *status and an
// unusable result, whose values may be stale; every store stays inside the
// n-entry outputs.  withhold_tile >= 0 is a test aid (see k_onesweep).
template <class K>
int onesweep_sort_pairs(K* k[2], int32_t* v[2], uint32_t* scratch, int64_t n, int bits, bool vals_in,
                        int* status, int sms, cudaStream_t s, int64_t* launches,
                        int64_t spin_limit = kLookSpinLimit, int withhold_tile = -1) {
    const int passes = (bits + 7) / 8;
    if (passes == 0) return 0;
    const int ntiles = sort_tiles(n);
    const size_t words = onesweep_words(n, passes);
    cudaMemsetAsync(scratch, 0, words * 4, s);
    const int hblocks = (int)std::min<int64_t>(ntiles, (int64_t)4 * std::max(sms, 1));
    k_digit_counts<K><<<hblocks, kSortThreads, 0, s>>>(k[0], n, passes, scratch);
    int src = 0;
    for (int p = 0; p < passes; ++p) {
        k_onesweep<K><<<ntiles, kSortThreads, 0, s>>>(k[src], (p == 0 && !vals_in) ? nullptr : v[src], k[src ^ 1],
                                                      v[src ^ 1], n, p, ntiles, scratch, status, spin_limit,
                                                      withhold_tile);
        src ^= 1;
    }
    *launches += 1 + passes;
    return src;
}

}  // namespace oct
