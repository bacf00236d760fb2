// Shared device/host helpers for the B200 octree neighbor-search library.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace oct {

// ---------------------------------------------------------------- status --
// Mirrors the exception classes the reference raises on this path
// (src/api.jl, src/morton.jl:84, ext/cuda_build.jl:156-163).
enum Status : int {
    OK = 0,
    ERR_ARGUMENT = 1,    // ArgumentError
    ERR_DIMENSION = 2,   // DimensionMismatch
    ERR_INEXACT = 3,     // InexactError from floor(Int32, (p - o) * inv_cs)
    ERR_CUDA = 4,        // a CUDA runtime call failed
    ERR_OVERFLOW = 5,    // internal capacity exceeded (the library retries)
    ERR_CAPACITY = 6,    // caller-supplied buffer too small
    ERR_TIMEOUT = 7,     // a bounded device wait ran out
    ERR_STATE = 8,       // ErrorException: wrong call order / missing build
};

// Device-side status word bits (OctHeader::status).
enum DevFlag : int {
    DF_NONFINITE = 1,    // a coordinate is NaN or +-Inf
    DF_NODE_OVERFLOW = 2,
    DF_RANGE = 4,        // binning out of Int32 range
    DF_TIMEOUT = 8,
    DF_KEY_WIDTH = 16,   // a re-encoded key does not fit the previous build's key width
};

constexpr int kWarp = 32;
constexpr int kLeafSize = 32;  // src/types.jl:177 (target_leaf_size)

template <int D> struct Dims;
template <> struct Dims<3> { static constexpr int bits = 21; static constexpr int nch = 8; };
template <> struct Dims<2> { static constexpr int bits = 31; static constexpr int nch = 4; };

// Worst-case DFS frontier: src/cpu/build_cpu.jl:39-43 (148 in 3D, 94 in 2D).
template <int D> __host__ __device__ constexpr int stack_depth() { return 1 + (Dims<D>::nch - 1) * Dims<D>::bits; }

// Sorted point record: coordinates in Morton order plus the point's original
// 0-based index, packed to a 16-byte multiple for vector loads.
template <class T, int D> struct alignas(16) SPt {
    T x[D];
    int32_t idx;
};

// Packed traversal node.  Internal: a = first child id (0-based, children are
// consecutive in BFS order), b = -(occupied-slot mask).  Leaf: a = first
// sorted position (0-based), b = point count (> 0).
template <class T, int D> struct alignas(16) TNode {
    T lo[D];
    T hi[D];
    int32_t a;
    int32_t b;
};

// Per-tree device header, copied to pinned host memory at the end of a build.
struct OctHeader {
    int32_t status;
    int32_t nan_flag;
    int64_t n_nodes;
    int64_t capacity;
    double gmin[3];
    double gmax[3];
    int32_t n_blocks_done;
    int32_t pad;
    int64_t n_groups;
    int32_t dfs_start;  // first node of the DFS below the root's single-child chain
    int32_t guard_bad;  // canary bytes found overwritten (guard-check mode)
    int64_t n_moved;    // refit mode: keys that changed since the previous build
};

// Packed pairs of floats with per-element IEEE round-to-nearest (sm_100+).
// Each operation alone is rounded exactly as the scalar __f*_rn operation.
// Chaining a packed add onto packed products is NOT: measured on B200 with
// CUDA 12.9, add.rn.f32x2(mul.rn.f32x2(..), mul.rn.f32x2(..)) disagreed with
// the separately rounded scalar sum in ~39% of random pairs (also with
// volatile asm and -Xptxas --fmad=false), while packed products summed with
// scalar __fadd_rn agreed in all 2M pairs tested.  Sums therefore stay scalar.
__device__ __forceinline__ unsigned long long sub2_rn(unsigned long long a, unsigned long long b) {
    unsigned long long d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ unsigned long long mul2_rn(unsigned long long a, unsigned long long b) {
    unsigned long long d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ unsigned long long pack2(float lo, float hi) {
    return ((unsigned long long)__float_as_uint(hi) << 32) | __float_as_uint(lo);
}
__device__ __forceinline__ float lo2(unsigned long long v) { return __uint_as_float((unsigned)v); }
__device__ __forceinline__ float hi2(unsigned long long v) { return __uint_as_float((unsigned)(v >> 32)); }

// A batch of independent point sets ("clouds") built as one forest.  Cloud c
// occupies positions [coff[c], coff[c+1]) both in input order and in sorted
// order, because the sort key is (c << kbits) | morton.  n_clouds == 0 means
// a single point set (every field unused).
constexpr int kCloudParams = 12;  // origin[3], inv_cs, r2, inv_r, bmin[3], bmax[3]
struct Batch {
    int32_t n_clouds = 0;
    int32_t kbits = 0;
    const int64_t* coff = nullptr;   // [n_clouds + 1]
    const double* cparam = nullptr;  // [n_clouds * kCloudParams], values exact in the element type
    int32_t* croot = nullptr;        // [n_clouds] root node id (-1 for an empty cloud)
    int32_t* cstart = nullptr;       // [n_clouds] first DFS node of each cloud's tree
};

// Cloud containing input (== sorted) position i: binary search of coff.
__device__ __forceinline__ int cloud_of_position(const Batch& b, int64_t i) {
    int lo = 0, hi = b.n_clouds - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (b.coff[mid] <= i) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// --------------------------------------------------- Julia float semantics --
// Base.min/max on IEEE floats for non-NaN operands: -0.0 orders below +0.0.
template <class T> __host__ __device__ __forceinline__ T jl_min(T x, T y) {
    return (y < x || (y == x && signbit(y) && !signbit(x))) ? y : x;
}
template <class T> __host__ __device__ __forceinline__ T jl_max(T x, T y) {
    return (y > x || (y == x && !signbit(y) && signbit(x))) ? y : x;
}

// Correctly rounded arithmetic without contraction (Julia never fuses).
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float sqrt_rn(float a) { return __fsqrt_rn(a); }
__device__ __forceinline__ double sqrt_rn(double a) { return __dsqrt_rn(a); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }

// Squared distance (x_t - x_q), summed left to right: ((dx*dx + dy*dy) + dz*dz),
// src/cpu/iterator_cpu.jl:96-97.
template <class T, int D>
__device__ __forceinline__ T dist2(const T* t, const T* q, T* diff) {
    T acc;
#pragma unroll
    for (int d = 0; d < D; ++d) {
        diff[d] = sub_rn(t[d], q[d]);
        const T s = mul_rn(diff[d], diff[d]);
        acc = (d == 0) ? s : add_rn(acc, s);
    }
    return acc;
}

// Box-to-box squared gap, conservative for the point test above: for a query
// point inside [qlo,qhi] and a target inside [lo,hi], each per-axis gap is <=
// |x_t - x_q| under monotone rounding, so the sum never exceeds dist2.
template <class T, int D>
__device__ __forceinline__ T box_gap2(const T* qlo, const T* qhi, const T* lo, const T* hi) {
    T acc;
#pragma unroll
    for (int d = 0; d < D; ++d) {
        T g = sub_rn(lo[d], qhi[d]);
        const T g2 = sub_rn(qlo[d], hi[d]);
        g = g > g2 ? g : g2;
        g = g > T(0) ? g : T(0);
        const T s = mul_rn(g, g);
        acc = (d == 0) ? s : add_rn(acc, s);
    }
    return acc;
}

// Morton interleave, src/morton.jl:13-23 and :50-58.
__host__ __device__ __forceinline__ uint64_t split_by_3(uint64_t x) {
    x &= 0x00000000001fffffULL;
    x = (x | (x << 32)) & 0x001f00000000ffffULL;
    x = (x | (x << 16)) & 0x001f0000ff0000ffULL;
    x = (x | (x << 8)) & 0x100f00f00f00f00fULL;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ULL;
    x = (x | (x << 2)) & 0x1249249249249249ULL;
    return x;
}
__host__ __device__ __forceinline__ uint64_t split_by_2(uint64_t x) {
    x &= 0x000000007fffffffULL;
    x = (x | (x << 16)) & 0x0000ffff0000ffffULL;
    x = (x | (x << 8)) & 0x00ff00ff00ff00ffULL;
    x = (x | (x << 4)) & 0x0f0f0f0f0f0f0f0fULL;
    x = (x | (x << 2)) & 0x3333333333333333ULL;
    x = (x | (x << 1)) & 0x5555555555555555ULL;
    return x;
}

// Inverses of split_by_3 / split_by_2: the cell index of one axis from a
// Morton code shifted so that the axis's bits are the lowest of each group.
__host__ __device__ __forceinline__ uint64_t compact_by_3(uint64_t x) {
    x &= 0x1249249249249249ULL;
    x = (x ^ (x >> 2)) & 0x10c30c30c30c30c3ULL;
    x = (x ^ (x >> 4)) & 0x100f00f00f00f00fULL;
    x = (x ^ (x >> 8)) & 0x001f0000ff0000ffULL;
    x = (x ^ (x >> 16)) & 0x001f00000000ffffULL;
    x = (x ^ (x >> 32)) & 0x00000000001fffffULL;
    return x;
}
__host__ __device__ __forceinline__ uint64_t compact_by_2(uint64_t x) {
    x &= 0x5555555555555555ULL;
    x = (x ^ (x >> 1)) & 0x3333333333333333ULL;
    x = (x ^ (x >> 2)) & 0x0f0f0f0f0f0f0f0fULL;
    x = (x ^ (x >> 4)) & 0x00ff00ff00ff00ffULL;
    x = (x ^ (x >> 8)) & 0x0000ffff0000ffffULL;
    x = (x ^ (x >> 16)) & 0x00000000ffffffffULL;
    return x;
}

// ------------------------------------------- programmatic dependent launch --
// A kernel launched with launch_pdl may be scheduled while the kernel before
// it in the stream is still running.  Its first statement is pdl_wait(),
// which returns once every earlier grid of the stream has completed and its
// memory is visible, so nothing it reads or writes overlaps the earlier
// kernel; pdl_trigger() then lets the next kernel be scheduled early in turn.
// What overlaps is the launch and block scheduling between the kernels.  In
// a launch without the attribute both are no-ops.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <class... P, class... A>
__host__ inline cudaError_t launch_pdl(void (*kern)(P...), int64_t grid, int block, size_t smem, cudaStream_t s,
                                       A&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, static_cast<A&&>(args)...);
}

// ---------------------------------------------------------- warp helpers --
__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

template <class T> __device__ __forceinline__ T warp_min(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = jl_min(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
template <class T> __device__ __forceinline__ T warp_max(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = jl_max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Integers: one redux.sync instead of a shuffle tree.
__device__ __forceinline__ int warp_min(int v) { return __reduce_min_sync(0xffffffffu, v); }
__device__ __forceinline__ int warp_max(int v) { return __reduce_max_sync(0xffffffffu, v); }

template <class T> __device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

inline int div_up(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

}  // namespace oct
