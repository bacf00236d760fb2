// Block- and device-wide exclusive scans (int32 counts -> int64 offsets).
#pragma once

#include "common.cuh"

namespace oct {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

// Inclusive warp scan.
template <class T> __device__ __forceinline__ T warp_inclusive_scan(T v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const T n = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += n;
    }
    return v;
}

// Exclusive block scan of one value per thread; returns the block total in
// *total.  `smem` holds blockDim.x / 32 + 1 elements.
template <class T> __device__ __forceinline__ T block_exclusive_scan(T v, T* smem, T* total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const T inc = warp_inclusive_scan(v);
    if (lane == 31) smem[w] = inc;
    __syncthreads();
    if (w == 0) {
        T s = lane < nw ? smem[lane] : T(0);
        const T si = warp_inclusive_scan(s);
        if (lane < nw) smem[lane] = si - s;
        if (lane == nw - 1) smem[nw] = si;  // block total, after the per-warp prefixes
    }
    __syncthreads();
    const T res = smem[w] + inc - v;
    *total = smem[nw];
    __syncthreads();
    return res;
}

// Both return the number of kernels launched (1 for n <= kSmallScan, 2 up to
// kInlineTiles tiles, else 3).
int exclusive_scan_i32_i64(const int32_t* in, int64_t* out, int64_t n, int64_t* d_total,
                           int64_t* tile_tmp, cudaStream_t s);
// In-place capable int32 scan; `out` holds n + 1 elements.
int exclusive_scan_i32_i32(const int32_t* in, int32_t* out, int64_t n, int64_t* tile_tmp, cudaStream_t s);
constexpr int kSmallScanThreads = 1024;
constexpr int64_t kSmallScan = 32 * kSmallScanThreads;  // one block scans up to this many
inline int64_t scan_tmp_elems(int64_t n) { return (n + kScanTile - 1) / kScanTile + 1; }
// Up to this many tiles (8M inputs) each final block adds up the sums of the
// tiles before it itself.
constexpr int kInlineTiles = 4096;

}  // namespace oct
