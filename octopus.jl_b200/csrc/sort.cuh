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
// Decoupled look-back state shared by the point-carrying sort (pointsort.cuh):
// each tile publishes its per-digit counts as an aggregate, then as an
// inclusive prefix once it has added those of the tiles before it.  Every
// wait is bounded: a wait that runs out sets DF_TIMEOUT in *status.
constexpr int kOnesweepMaxPasses = 8;
constexpr uint32_t kLookAggregate = 1u << 30;
constexpr uint32_t kLookPrefix = 2u << 30;
constexpr uint32_t kLookValue = (1u << 30) - 1;
// Default number of polling rounds a look-back wait makes before it gives up
// (a context option, OCT_OPT_WAIT_LIMIT, overrides it).
constexpr int64_t kLookSpinLimit = 1 << 22;

// Scratch words: for each of up to kOnesweepMaxPasses passes 256 digit counts
// and a tile counter, then per pass 256 look-back words per tile; all zero
// before the sort.
inline size_t onesweep_words(int64_t n, int passes) {
    return (size_t)kOnesweepMaxPasses * 257 + (size_t)passes * sort_tiles(n) * 256;
}

}  // namespace oct
