// Device-wide exclusive scan, reduce-then-scan in two launches (three above
// kInlineTiles tiles).  No kernel waits on another block, so there is nothing
// to spin on.
#include "scan.cuh"

namespace oct {

// Per-tile sums of kScanTile consecutive inputs.
template <class In>
__global__ void __launch_bounds__(kScanThreads) k_scan_tile_sums(const In* __restrict__ in, int64_t n,
                                                                 int64_t* __restrict__ tile_sums) {
    pdl_wait();
    pdl_trigger();
    __shared__ int64_t sm[kScanThreads / 32 + 1];
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
    int64_t s = 0;
#pragma unroll
    for (int it = 0; it < kScanItems; ++it) {
        const int64_t i = base + (int64_t)it * kScanThreads + threadIdx.x;
        if (i < n) s += in[i];
    }
    int64_t tot;
    block_exclusive_scan<int64_t>(s, sm, &tot);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = tot;
}

// Exclusive scan of the tile sums by one block, carrying across chunks.
__global__ void __launch_bounds__(1024) k_scan_tiles(int64_t* __restrict__ tile_sums, int64_t ntiles,
                                                     int64_t* __restrict__ d_total) {
    pdl_wait();
    pdl_trigger();
    __shared__ int64_t sm[1024 / 32 + 1];
    int64_t carry = 0;
    for (int64_t base = 0; base < ntiles; base += blockDim.x) {
        const int64_t i = base + threadIdx.x;
        const int64_t v = i < ntiles ? tile_sums[i] : 0;
        int64_t tot;
        const int64_t ex = block_exclusive_scan<int64_t>(v, sm, &tot);
        if (i < ntiles) tile_sums[i] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0 && d_total) *d_total = carry;
}

// Final pass: each tile scans its items in order (blocked per thread) and
// adds the tile offset.  SUMS: tile_off holds the tiles' sums (not yet
// scanned) and each block adds up those before its own (at most
// kInlineTiles of them, a few loads per thread), so no separate launch scans
// them; the last block also writes the total to *d_total.
template <class In, class Out, bool SUMS>
__global__ void __launch_bounds__(kScanThreads) k_scan_final(const In* in, int64_t n,
                                                             const int64_t* __restrict__ tile_off, Out* out,
                                                             int64_t* __restrict__ d_total) {
    pdl_wait();
    pdl_trigger();
    __shared__ int64_t sm[kScanThreads / 32 + 1];
    __shared__ In stage[kScanTile];
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
    int64_t toff;
    if (SUMS) {
        int64_t part = 0;
        for (int j = threadIdx.x; j < (int)blockIdx.x; j += kScanThreads) part += tile_off[j];
        int64_t before;
        block_exclusive_scan<int64_t>(part, sm, &before);
        toff = before;
    } else {
        toff = tile_off[blockIdx.x];
    }
    // Coalesced load into shared memory, then each thread owns kScanItems
    // consecutive elements.
#pragma unroll
    for (int it = 0; it < kScanItems; ++it) {
        const int j = it * kScanThreads + threadIdx.x;
        const int64_t i = base + j;
        stage[j] = i < n ? in[i] : 0;
    }
    __syncthreads();
    In v[kScanItems];
    int64_t s = 0;
#pragma unroll
    for (int it = 0; it < kScanItems; ++it) {
        v[it] = stage[threadIdx.x * kScanItems + it];
        s += v[it];
    }
    int64_t tot;
    int64_t run = block_exclusive_scan<int64_t>(s, sm, &tot) + toff;
#pragma unroll
    for (int it = 0; it < kScanItems; ++it) {
        const int64_t i = base + (int64_t)threadIdx.x * kScanItems + it;
        if (i < n) out[i] = (Out)run;
        run += v[it];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) {
        out[n] = (Out)(toff + tot);
        if (SUMS && d_total) *d_total = toff + tot;
    }
}

// Short inputs in one launch: each thread sums, then writes, its own run of
// consecutive elements (reading each element before writing it, so `in` and
// `out` may alias).
template <class In, class Out>
__global__ void __launch_bounds__(kSmallScanThreads) k_scan_small(const In* in, int64_t n, Out* out,
                                                                  int64_t* __restrict__ d_total) {
    pdl_wait();
    pdl_trigger();
    __shared__ int64_t sm[kSmallScanThreads / 32 + 1];
    const int64_t per = (n + kSmallScanThreads - 1) / kSmallScanThreads;
    const int64_t b = (int64_t)threadIdx.x * per;
    int64_t sum = 0;
    for (int64_t i = b; i < b + per && i < n; ++i) sum += in[i];
    int64_t tot;
    int64_t run = block_exclusive_scan<int64_t>(sum, sm, &tot);
    for (int64_t i = b; i < b + per && i < n; ++i) {
        const In x = in[i];
        out[i] = (Out)run;
        run += x;
    }
    if (threadIdx.x == 0) {
        out[n] = (Out)tot;
        if (d_total) *d_total = tot;
    }
}

// out[0..n] = exclusive scan of in[0..n-1]; out[n] = total (also *d_total).
// `in` and `out` may alias: each tile stages its inputs before writing.
template <class In, class Out>
int exclusive_scan(const In* in, Out* out, int64_t n, int64_t* d_total, int64_t* tile_tmp, cudaStream_t s) {
    if (n <= 0) {
        cudaMemsetAsync(out, 0, sizeof(Out), s);
        if (d_total) cudaMemsetAsync(d_total, 0, sizeof(int64_t), s);
        return 0;
    }
    if (n <= kSmallScan) {
        launch_pdl(k_scan_small<In, Out>, 1, kSmallScanThreads, 0, s, in, n, out, d_total);
        return 1;
    }
    const int ntiles = div_up(n, kScanTile);
    launch_pdl(k_scan_tile_sums<In>, ntiles, kScanThreads, 0, s, in, n, tile_tmp);
    if (ntiles <= kInlineTiles) {
        launch_pdl(k_scan_final<In, Out, true>, ntiles, kScanThreads, 0, s, in, n, tile_tmp, out, d_total);
        return 2;
    }
    launch_pdl(k_scan_tiles, 1, 1024, 0, s, tile_tmp, ntiles, d_total);
    launch_pdl(k_scan_final<In, Out, false>, ntiles, kScanThreads, 0, s, in, n, tile_tmp, out, nullptr);
    return 3;
}

int exclusive_scan_i32_i64(const int32_t* in, int64_t* out, int64_t n, int64_t* d_total, int64_t* tile_tmp,
                           cudaStream_t s) {
    return exclusive_scan<int32_t, int64_t>(in, out, n, d_total, tile_tmp, s);
}

int exclusive_scan_i32_i32(const int32_t* in, int32_t* out, int64_t n, int64_t* tile_tmp, cudaStream_t s) {
    return exclusive_scan<int32_t, int32_t>(in, out, n, nullptr, tile_tmp, s);
}

}  // namespace oct
