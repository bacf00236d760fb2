// Device-resident tree build: bounds reduce -> Morton encode -> stable LSD
// radix sort -> sorted point gather -> BFS topology -> bottom-up bounds.
//
// Replaces _build_gpu_tree! (ext/cuda_build.jl:227-288) and reproduces the
// CPU build exactly (src/cpu/bin_cpu.jl, src/sort.jl, src/cpu/build_cpu.jl,
// src/cpu/refit_cpu.jl): the same keys, the same stable order, the same
// leaves and BFS node numbering, and bit-identical bounds.
//
// Topology without per-level launches: a node at level L starts at sorted
// position k iff the level-L key prefix changes at k and the level-(L-1)
// group containing k holds more than 32 points (or k is the root).  A group
// holds more than 32 points iff some window of 33 consecutive positions
// around k shares its prefix, which one pass over the sorted keys detects.
// Each position therefore owns a contiguous range of levels [lo, hi], with
// hi the level of the leaf that contains it.  BFS ids are level-major,
// position-minor, so they come from one exclusive scan of per-block,
// per-level node counts; children of a node are consecutive ids.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include <cuda/atomic>

#include "internal.h"
#include "pointsort.cuh"
#include "scan.cuh"
#include "sort.cuh"

namespace oct {

constexpr int kThreads = 256;

// ------------------------------------------------------------ 1. bounds --
// Order key of an IEEE value: its bits with the magnitude bits flipped when
// the sign is set, so that signed integer order is the value order of every
// non-NaN value, -0.0 below +0.0 (Julia's min/max); the map is its own inverse.
template <class T> struct OrdKey;
template <> struct OrdKey<float> {
    using I = int32_t;
    static constexpr I kMag = 0x7fffffff, kExp = 0x7f800000;
    static constexpr I kMaxKey = 0x7fffffff, kMinKey = (I)0x80000000;
    __device__ static I bits(float x) { return __float_as_int(x); }
    __device__ static I key(I b) { return b ^ ((b >> 31) & kMag); }
    __device__ static float value(I k) { return __int_as_float(key(k)); }
};
template <> struct OrdKey<double> {
    using I = long long;
    static constexpr I kMag = 0x7fffffffffffffffLL, kExp = 0x7ff0000000000000LL;
    static constexpr I kMaxKey = 0x7fffffffffffffffLL, kMinKey = (I)0x8000000000000000ULL;
    __device__ static I bits(double x) { return __double_as_longlong(x); }
    __device__ static I key(I b) { return b ^ ((b >> 63) & kMag); }
    __device__ static double value(I k) { return __longlong_as_double(key(k)); }
};
__device__ __forceinline__ int32_t ord_warp_min(int32_t v) { return __reduce_min_sync(0xffffffffu, v); }
__device__ __forceinline__ int32_t ord_warp_max(int32_t v) { return __reduce_max_sync(0xffffffffu, v); }
__device__ __forceinline__ long long ord_warp_min(long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ long long ord_warp_max(long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Per-axis min/max (Julia min/max order) and a non-finite flag.  The last
// block to finish folds the per-block partials into the header.
template <class T, int D>
__global__ void __launch_bounds__(kThreads) k_bounds(const T* __restrict__ coords, int64_t n,
                                                     double* __restrict__ partials, OctHeader* hdr) {
    pdl_wait();
    pdl_trigger();
    __shared__ T smin[kThreads / 32][D], smax[kThreads / 32][D];
    __shared__ int snan;
    __shared__ bool is_last;
    if (threadIdx.x == 0) snan = 0;
    __syncthreads();
    // The fold runs on order keys (OrdKey): integer min/max give Julia's
    // min/max of finite values, and a magnitude at or above the exponent
    // mask marks a NaN or Inf (whose bounds then do not matter: the build
    // fails).
    using I = typename OrdKey<T>::I;
    I klo[D], khi[D], mag = 0;
#pragma unroll
    for (int d = 0; d < D; ++d) { klo[d] = OrdKey<T>::kMaxKey; khi[d] = OrdKey<T>::kMinKey; }
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x, nthr = (int64_t)gridDim.x * blockDim.x;
    auto take = [&](int d, T x) {
        const I b = OrdKey<T>::bits(x);
        const I k = OrdKey<T>::key(b);
        klo[d] = min(klo[d], k);
        khi[d] = max(khi[d], k);
        mag = max(mag, b & OrdKey<T>::kMag);
    };
    int64_t done = 0;  // points folded by the vector loop
    if constexpr (std::is_same<T, float>::value && D == 3) {
        if (((uintptr_t)coords & 15) == 0) {
            // Four points = 12 floats = three float4 (axes x y z x | y z x y | z x y z),
            // two groups of four points in flight per thread.
            const float4* v = reinterpret_cast<const float4*>(coords);
            const int64_t groups = n / 4;
            for (int64_t g = tid; g < groups; g += 2 * nthr) {
                const int64_t g2 = g + nthr;
                const float4 a = v[3 * g], b = v[3 * g + 1], c = v[3 * g + 2];
                float4 a2 = a, b2 = b, c2 = c;
                if (g2 < groups) {
                    a2 = v[3 * g2];
                    b2 = v[3 * g2 + 1];
                    c2 = v[3 * g2 + 2];
                }
                take(0, a.x); take(1, a.y); take(2, a.z); take(0, a.w);
                take(1, b.x); take(2, b.y); take(0, b.z); take(1, b.w);
                take(2, c.x); take(0, c.y); take(1, c.z); take(2, c.w);
                take(0, a2.x); take(1, a2.y); take(2, a2.z); take(0, a2.w);
                take(1, b2.x); take(2, b2.y); take(0, b2.z); take(1, b2.w);
                take(2, c2.x); take(0, c2.y); take(1, c2.z); take(2, c2.w);
            }
            done = groups * 4;
        }
    }
    for (int64_t i = done + tid; i < n; i += nthr) {
#pragma unroll
        for (int d = 0; d < D; ++d) take(d, coords[D * i + d]);
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    T lo[D], hi[D];
#pragma unroll
    for (int d = 0; d < D; ++d) {
        lo[d] = OrdKey<T>::value(ord_warp_min(klo[d]));
        hi[d] = OrdKey<T>::value(ord_warp_max(khi[d]));
    }
    const int bad = mag >= OrdKey<T>::kExp;
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(&snan, 1);
    if (lane == 0) {
#pragma unroll
        for (int d = 0; d < D; ++d) { smin[w][d] = lo[d]; smax[w][d] = hi[d]; }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w2 = 1; w2 < kThreads / 32; ++w2)
            for (int d = 0; d < D; ++d) {
                smin[0][d] = jl_min(smin[0][d], smin[w2][d]);
                smax[0][d] = jl_max(smax[0][d], smax[w2][d]);
            }
        double* p = partials + (size_t)blockIdx.x * 8;
        for (int d = 0; d < D; ++d) { p[d] = (double)smin[0][d]; p[3 + d] = (double)smax[0][d]; }
        p[6] = snan ? 1.0 : 0.0;
        __threadfence();
        const int ticket = atomicAdd(&hdr->n_blocks_done, 1);
        is_last = (ticket == (int)gridDim.x - 1);
    }
    __syncthreads();
    if (!is_last) return;
    // Last block: fold the per-block partials in parallel.
    __threadfence();
    T glo[D], ghi[D];
#pragma unroll
    for (int d = 0; d < D; ++d) { glo[d] = T(INFINITY); ghi[d] = T(-INFINITY); }
    int anynan = 0;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
        const double* p = partials + (size_t)b * 8;
#pragma unroll
        for (int d = 0; d < D; ++d) {
            glo[d] = jl_min(glo[d], (T)__ldcg(p + d));
            ghi[d] = jl_max(ghi[d], (T)__ldcg(p + 3 + d));
        }
        if (__ldcg(p + 6) != 0.0) anynan = 1;
    }
#pragma unroll
    for (int d = 0; d < D; ++d) {
        glo[d] = warp_min(glo[d]);
        ghi[d] = warp_max(ghi[d]);
    }
    anynan = __any_sync(0xffffffffu, anynan);
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int d = 0; d < D; ++d) { smin[w][d] = glo[d]; smax[w][d] = ghi[d]; }
        if (anynan) atomicOr(&snan, 2);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w2 = 1; w2 < kThreads / 32; ++w2)
            for (int d = 0; d < D; ++d) {
                smin[0][d] = jl_min(smin[0][d], smin[w2][d]);
                smax[0][d] = jl_max(smax[0][d], smax[w2][d]);
            }
        for (int d = 0; d < D; ++d) { hdr->gmin[d] = (double)smin[0][d]; hdr->gmax[d] = (double)smax[0][d]; }
        hdr->nan_flag = (snan & 2) ? 1 : 0;
        hdr->n_blocks_done = 0;
    }
}

// ------------------------------------------------------------ 2. encode --
// Morton key of one point's cell (src/cpu/bin_cpu.jl:12-31 with
// src/morton.jl:13-60): floor((x - origin) * inv_cs) per axis, clamped to the
// key's bits per axis, bit-interleaved with x in the lowest bit.
template <class T, int D>
__device__ __forceinline__ uint64_t cell_key(const T* __restrict__ x, const T* o, T inv_cs) {
    constexpr int64_t cmax = (1LL << Dims<D>::bits) - 1;
    uint64_t c[3] = {0, 0, 0};
#pragma unroll
    for (int d = 0; d < D; ++d) {
        const T v = mul_rn(sub_rn(x[d], o[d]), inv_cs);
        int64_t ci = (int64_t)floor(v);
        ci = ci < 0 ? 0 : (ci > cmax ? cmax : ci);
        c[d] = (uint64_t)ci;
    }
    return (D == 3) ? ((split_by_3(c[2]) << 2) | (split_by_3(c[1]) << 1) | split_by_3(c[0]))
                    : ((split_by_2(c[1]) << 1) | split_by_2(c[0]));
}

// bin_point + clamp + morton_encode (src/cpu/bin_cpu.jl:52-95).  The host has
// already proven every cell index fits Int32 (the max coordinate bins last).
template <class T, int D, class K>
__global__ void __launch_bounds__(kThreads) k_encode(const T* __restrict__ coords, int64_t n, T o0, T o1, T o2,
                                                     T inv_cs, K* __restrict__ keys,
                                                     Batch bt) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    T o[3] = {o0, o1, o2};
    int cloud = 0;
    if (bt.n_clouds) {
        // Each cloud has its own origin and cell size (one TNS per cloud).
        cloud = cloud_of_position(bt, i);
        const double* cp = bt.cparam + (size_t)cloud * kCloudParams;
        o[0] = (T)cp[0];
        o[1] = (T)cp[1];
        o[2] = (T)cp[2];
        inv_cs = (T)cp[3];
    }
    const uint64_t key = cell_key<T, D>(coords + D * i, o, inv_cs);
    keys[i] = bt.n_clouds ? (K)(((uint64_t)cloud << bt.kbits) | key) : (K)key;
}

// ------------------------------------------------------------ 4. gather --
// A permutation entry outside [0, n) can only come from a sort whose
// look-back wait ran out (DF_TIMEOUT is then set already): it is skipped, so
// neither the coordinate read nor the inverse-permutation store leaves its
// array.
template <class T, int D>
__global__ void __launch_bounds__(kThreads) k_gather(const T* __restrict__ coords, const int32_t* __restrict__ perm,
                                                     int64_t n, SPt<T, D>* __restrict__ spts,
                                                     int32_t* __restrict__ iperm, int* __restrict__ status) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int32_t j = perm ? perm[k] : (int32_t)k;
    if ((uint64_t)(uint32_t)j >= (uint64_t)n) {
        atomicOr(status, (int)DF_TIMEOUT);
        return;
    }
    SPt<T, D> p;
#pragma unroll
    for (int d = 0; d < D; ++d) p.x[d] = coords[(int64_t)D * j + d];
    p.idx = j;
    spts[k] = p;
    iperm[j] = (int32_t)k;
}

// ---------------------------------------------------------- 5. topology --
// Number of leading D-bit digits (of Dims<D>::bits) two keys share.
template <int D, class K> __device__ __forceinline__ int common_levels(K a, K b) {
    const uint64_t x = (uint64_t)(a ^ b);
    if (x == 0) return Dims<D>::bits;
    const int hb = 63 - __clzll((long long)x);
    return Dims<D>::bits - 1 - hb / D;
}

// Same, where keys of different clouds share no level (-1).
template <int D, class K> __device__ __forceinline__ int common_levels_b(K a, K b, const Batch& bt) {
    if (!bt.n_clouds) return common_levels<D, K>(a, b);
    if ((uint64_t)a >> bt.kbits != (uint64_t)b >> bt.kbits) return -1;
    const uint64_t m = (1ULL << bt.kbits) - 1;
    return common_levels<D, uint64_t>((uint64_t)a & m, (uint64_t)b & m);
}

// Digit (child slot) of a key at level L, from its Morton part.
template <int D, class K> __device__ __forceinline__ int slot_digit(K key, int shd, const Batch& bt) {
    uint64_t v = (uint64_t)key;
    if (bt.n_clouds) v &= (1ULL << bt.kbits) - 1;
    return (int)((v >> shd) & (uint64_t)(Dims<D>::nch - 1));
}

constexpr int kMarkTile = kThreads;  // positions per block in mark / emit

// lohi[k] = lo | hi << 8: the levels whose node starts at position k are
// lo..hi (empty when lo > hi); hi is the level of the leaf containing k
// (src/cpu/build_cpu.jl:146: leaf iff count <= 32 or level >= max_levels).
template <int D, class K>
__global__ void __launch_bounds__(kThreads) k_mark(const K* __restrict__ skeys, int64_t n,
                                                   uint16_t* __restrict__ lohi, int32_t* __restrict__ blockcnt,
                                                   int nblocks, Batch bt) {
    pdl_wait();
    pdl_trigger();
    constexpr int MAXLEV = Dims<D>::bits;
    constexpr int NLEV = MAXLEV + 1;
    __shared__ K sk[kMarkTile + 64];
    __shared__ int8_t sc[kMarkTile + 32];
    __shared__ int32_t wcnt[NLEV][kThreads / 32];
    const int64_t base = (int64_t)blockIdx.x * kMarkTile;
    for (int i = threadIdx.x; i < kMarkTile + 64; i += kThreads) {
        const int64_t p = base - 32 + i;
        sk[i] = (p >= 0 && p < n) ? skeys[p] : K(0);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kMarkTile + 32; i += kThreads) {
        const int64_t j = base - 32 + i;
        sc[i] = (j >= 0 && j + 32 <= n - 1) ? (int8_t)common_levels_b<D, K>(sk[i], sk[i + 32], bt) : (int8_t)-1;
    }
    __syncthreads();
    const int64_t k = base + threadIdx.x;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    // max of sc[x .. x + 32] for x = threadIdx.x: the suffix maximum of the
    // warp's first 32 entries from this lane on, with the prefix maximum of
    // the next 32 up to this lane
    int sa = sc[threadIdx.x], pb = sc[threadIdx.x + 32];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int a = __shfl_down_sync(0xffffffffu, sa, o);
        const int b = __shfl_up_sync(0xffffffffu, pb, o);
        if (lane + o < 32) sa = max(sa, a);
        if (lane >= o) pb = max(pb, b);
    }
    int lo = 1, hi = 0;
    if (k < n) {
        lo = (k == 0) ? 0 : common_levels_b<D, K>(sk[threadIdx.x + 31], sk[threadIdx.x + 32], bt) + 1;
        hi = min(max(sa, pb) + 1, MAXLEV);
        lohi[k] = (uint16_t)(lo | (hi << 8));
    }
    // per-level node counts of the warp, over the levels its positions span
    const int wlo = warp_min(lo <= hi ? lo : NLEV), whi = warp_max(lo <= hi ? hi : -1);
    if (lane < NLEV && (lane < wlo || lane > whi)) wcnt[lane][w] = 0;
    for (int L = wlo; L <= whi; ++L) {
        const unsigned b = __ballot_sync(0xffffffffu, lo <= L && L <= hi);
        if (lane == 0) wcnt[L][w] = __popc(b);
    }
    __syncthreads();
    if (threadIdx.x < NLEV) {
        int s = 0;
#pragma unroll
        for (int j = 0; j < kThreads / 32; ++j) s += wcnt[threadIdx.x][j];
        blockcnt[(int64_t)threadIdx.x * nblocks + blockIdx.x] = s;
    }
}

// Node (L, k) -> BFS id.  Writes nrange[id] = {k, L}, first_child[id] = the
// id of the first child (the node (L+1, k)) or -1 for a leaf, and
// node_end[id] = one past the node's last position; k_emit_nodes completes
// each node from these.
template <int D>
__global__ void __launch_bounds__(kThreads) k_emit_ids(int64_t n, const uint16_t* __restrict__ lohi,
                                                       const int64_t* __restrict__ blockoff, int nblocks,
                                                       int64_t capacity, int32_t* __restrict__ first_child,
                                                       int2* __restrict__ nrange, int32_t* __restrict__ node_end,
                                                       OctHeader* hdr, Batch bt) {
    pdl_wait();
    pdl_trigger();
    constexpr int NLEV = Dims<D>::bits + 1;
    __shared__ int32_t wpre[NLEV][kThreads / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t k = (int64_t)blockIdx.x * kMarkTile + threadIdx.x;
    int lo = 1, hi = 0;
    if (k < n) {
        const uint16_t v = lohi[k];
        lo = v & 0xff;
        hi = v >> 8;
    }
    const int wlo = warp_min(lo <= hi ? lo : NLEV), whi = warp_max(lo <= hi ? hi : -1);
    if (lane < NLEV && (lane < wlo || lane > whi)) wpre[lane][w] = 0;
    for (int L = wlo; L <= whi; ++L) {
        const unsigned b = __ballot_sync(0xffffffffu, lo <= L && L <= hi);
        if (lane == 0) wpre[L][w] = __popc(b);
    }
    __syncthreads();
    if (threadIdx.x < NLEV) {
        int run = 0;
#pragma unroll
        for (int j = 0; j < kThreads / 32; ++j) {
            const int c = wpre[threadIdx.x][j];
            wpre[threadIdx.x][j] = run;
            run += c;
        }
    }
    __syncthreads();
    if (hdr->n_nodes > capacity) {
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&hdr->status, (int)DF_NODE_OVERFLOW);
        return;
    }
    int32_t prev = -1;
    for (int L = whi; L >= wlo; --L) {
        const bool in = lo <= L && L <= hi;
        const unsigned b = __ballot_sync(0xffffffffu, in);
        if (in) {
            const int32_t id = (int32_t)(blockoff[(int64_t)L * nblocks + blockIdx.x] + wpre[L][w] +
                                         __popc(b & lanemask_lt()));
            nrange[id] = make_int2((int)k, L);
            first_child[id] = L < hi ? prev : -1;
            if (L == 0 && bt.n_clouds) bt.croot[cloud_of_position(bt, k)] = id;
            prev = id;
        }
    }
    // Node ends.  A level-L node ends where the level-L key prefix changes,
    // so the nodes holding position k that end at k + 1 are those of levels
    // lo(k + 1) .. hi(k) (every level at the end of the array).  The level-L
    // node holding k is the last one starting at or before k: its id is k's
    // inclusive rank among the level-L starts, minus one.
    int nlo = __shfl_down_sync(0xffffffffu, lo, 1);  // lo(k + 1)
    if (lane == 31 && k + 1 < n) nlo = lohi[k + 1] & 0xff;
    if (k + 1 >= n) nlo = 0;
    const bool ends = k < n && nlo <= hi;
    const int elo = warp_min(ends ? nlo : NLEV), ehi = warp_max(ends ? hi : -1);
    for (int L = elo; L <= ehi; ++L) {
        const unsigned b = __ballot_sync(0xffffffffu, lo <= L && L <= hi);
        if (ends && nlo <= L && L <= hi) {
            const int32_t id = (int32_t)(blockoff[(int64_t)L * nblocks + blockIdx.x] + wpre[L][w] +
                                         __popc(b & lanemask_lt()) + (int)((b >> lane) & 1u) - 1);
            node_end[id] = (int32_t)(k + 1);
        }
    }
}

// Completes node `id`: its last position (from the end k_emit_ids left in
// `arrive`, which is then reset for the refit), its occupied child slots and
// the children's parent links.
template <class T, int D, class K>
__global__ void __launch_bounds__(kThreads) k_emit_nodes(const K* __restrict__ skeys, int64_t n, int64_t capacity,
                                                         const int32_t* __restrict__ first_child_in,
                                                         TNode<T, D>* __restrict__ tnode, int2* __restrict__ nrange,
                                                         int32_t* __restrict__ parent, int32_t* __restrict__ arrive,
                                                         int32_t* __restrict__ chain, const int64_t* __restrict__ blockoff,
                                                         int nblocks, const OctHeader* hdr, Batch bt) {
    pdl_wait();
    pdl_trigger();
    constexpr int BITS = Dims<D>::bits;
    constexpr int NCH = Dims<D>::nch;
    const int64_t nn = hdr->n_nodes;
    const int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (nn > capacity || id >= nn) return;
    const int2 kl = nrange[id];
    const int64_t k = kl.x;
    const int L = kl.y;
    const int32_t first_child = first_child_in[id];
    // The point set holding k: [s0, s1) (a cloud, or everything).
    int cloud = 0;
    int64_t s0 = 0, s1 = n;
    if (bt.n_clouds) {
        cloud = cloud_of_position(bt, k);
        s0 = bt.coff[cloud];
        s1 = bt.coff[cloud + 1];
    }
    const int64_t e = arrive[id];  // the end written by k_emit_ids
    TNode<T, D> nd;
    if (first_child < 0) {
        nd.a = (int32_t)k;
        nd.b = (int32_t)(e - k);
    } else {
        // The children are the consecutive level-(L+1) ids from first_child
        // whose ranges start inside [k, e) (nrange[c].x, written by the id
        // pass, is their first position); each one's slot is its key's digit.
        const int shd = D * BITS - D * (L + 1);
        const int64_t lend = L + 2 <= BITS ? blockoff[(int64_t)(L + 2) * nblocks] : nn;  // first id past level L+1
        unsigned slots = 0u;
        for (int64_t c = first_child; c < lend && c < (int64_t)first_child + NCH; ++c) {
            const int64_t cs = nrange[c].x;
            if (cs >= e) break;
            slots |= 1u << slot_digit<D, K>(skeys[cs], shd, bt);
            parent[c] = (int32_t)id;
        }
        nd.a = first_child;
        nd.b = -(int32_t)slots;
    }
    if (k == s0 && e == s1) {
        // A node covering its whole point set has that set's bounds.
        if (bt.n_clouds) {
            const double* cp = bt.cparam + (size_t)cloud * kCloudParams;
#pragma unroll
            for (int d = 0; d < D; ++d) { nd.lo[d] = (T)cp[6 + d]; nd.hi[d] = (T)cp[9 + d]; }
        } else {
#pragma unroll
            for (int d = 0; d < D; ++d) { nd.lo[d] = (T)hdr->gmin[d]; nd.hi[d] = (T)hdr->gmax[d]; }
            // Full-range nodes form the root's chain: chain[L] = id, and
            // chain[32 + L] = 1 when the node's only child sits in slot 0.
            chain[L] = (int32_t)id;
            chain[32 + L] = (nd.b == -1) ? 1 : 0;
        }
    } else {
#pragma unroll
        for (int d = 0; d < D; ++d) { nd.lo[d] = T(0); nd.hi[d] = T(0); }
    }
    tnode[id] = nd;
    nrange[id] = make_int2((int)k, (int)(e - 1));
    arrive[id] = 0;
    if (L == 0) parent[id] = -1;  // a root (one per cloud in a batch)
}

// ------------------------------------------------------------- 6. refit --
// Leaves fold their points (src/cpu/refit_cpu.jl:39-48); the last child to
// arrive at a parent folds the children (src/cpu/refit_cpu.jl:50-60).  No
// thread waits: a thread that is not last simply stops.
template <class T, int D>
__global__ void __launch_bounds__(kThreads) k_refit(int64_t capacity, int64_t n, TNode<T, D>* tnode,
                                                    const int2* __restrict__ nrange, const int32_t* __restrict__ parent,
                                                    int32_t* arrive, const SPt<T, D>* __restrict__ spts,
                                                    const OctHeader* hdr, Batch bt) {
    pdl_wait();
    pdl_trigger();
    const int64_t nn = hdr->n_nodes;
    const int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (nn > capacity || id >= nn) return;
    const int32_t a = tnode[id].a, b = tnode[id].b;
    if (b <= 0) return;
    T lo[D], hi[D];
#pragma unroll
    for (int d = 0; d < D; ++d) { lo[d] = T(INFINITY); hi[d] = T(-INFINITY); }
    for (int32_t m = a; m < a + b; ++m) {
        const SPt<T, D> p = spts[m];
#pragma unroll
        for (int d = 0; d < D; ++d) { lo[d] = jl_min(lo[d], p.x[d]); hi[d] = jl_max(hi[d], p.x[d]); }
    }
#pragma unroll
    for (int d = 0; d < D; ++d) { tnode[id].lo[d] = lo[d]; tnode[id].hi[d] = hi[d]; }
    int32_t node = (int32_t)id;
    while (true) {
        const int32_t p = parent[node];
        if (p < 0) break;
        const int2 rg = nrange[p];
        int64_t s0 = 0, s1 = n;
        if (bt.n_clouds) {
            const int c = cloud_of_position(bt, rg.x);
            s0 = bt.coff[c];
            s1 = bt.coff[c + 1];
        }
        if (rg.x == s0 && (int64_t)rg.y == s1 - 1) break;  // bounds preset from the set's reduce
        const int32_t pa = tnode[p].a, pb = tnode[p].b;
        const int nc = __popc((unsigned)(-pb));
        // Release this node's bounds and, for the last arrival, acquire its
        // siblings' (one acquire-release read-modify-write, no full fences).
        const int old = cuda::atomic_ref<int32_t, cuda::thread_scope_device>(arrive[p]).fetch_add(
            1, cuda::memory_order_acq_rel);
        if (old != nc - 1) break;
#pragma unroll
        for (int d = 0; d < D; ++d) { lo[d] = T(INFINITY); hi[d] = T(-INFINITY); }
        for (int c = 0; c < nc; ++c) {
            const TNode<T, D>* cn = tnode + pa + c;
#pragma unroll
            for (int d = 0; d < D; ++d) {
                lo[d] = jl_min(lo[d], __ldcg(&cn->lo[d]));
                hi[d] = jl_max(hi[d], __ldcg(&cn->hi[d]));
            }
        }
#pragma unroll
        for (int d = 0; d < D; ++d) { tnode[p].lo[d] = lo[d]; tnode[p].hi[d] = hi[d]; }
        node = p;
    }
}

// ------------------------------------------------------- 7. query groups --
// A query group is a run of consecutive sibling leaves holding at most gmax
// (<= 32, a tuned shape) points in total (a leaf of more than gmax points is
// cut into chunks of gmax).  Siblings share a parent box, so a
// group's points are spatially compact; a window of 32 consecutive sorted
// positions can instead straddle a jump of the Morton curve and span the
// whole domain.  Each node counts the groups formed under it, a warp reserves
// room for its nodes' groups with one atomic on hdr->n_groups, and each node
// writes its groups there.  The groups' order does not matter: every result
// is per query point.
//
// Each group also gets the node its traversal may start from (gstart, when
// given): the deepest strict ancestor S of the group's parent P whose Morton
// cell contains every cell within kStartMargin cells of P's cell.  The cell
// size is the radius, so every point within the radius of a point of the group
// (one cell, plus one for the rounding of the two binnings) lies in S's cell,
// hence in S's subtree: a search from S meets every neighbor the search from
// the root meets, and in the same order, since a depth-first search restricted
// to a subtree visits it in the subtree's own order.  Bit 30 carries the
// ascending-order flag that S's stack entry has in the search from the root
// (some strict ancestor with its first child slot empty); -1 = start at the
// root.  The test reads keys and topology only, so it holds for as long as the
// keys do (the bounds-only refit keeps it).
constexpr int kStartMargin = 2;

template <int D, class K>
__device__ __forceinline__ uint64_t axis_cell(K key, int d) {
    return D == 3 ? compact_by_3((uint64_t)key >> d) : compact_by_2((uint64_t)key >> d);
}

template <class T, int D, class K>
__global__ void __launch_bounds__(kThreads) k_groups(const TNode<T, D>* __restrict__ tnode, int64_t capacity,
                                                     int2* __restrict__ groups, int64_t group_cap,
                                                     const int32_t* __restrict__ chain,
                                                     const int32_t* __restrict__ parent, OctHeader* hdr, int gmax,
                                                     const K* __restrict__ skeys, const int2* __restrict__ nrange,
                                                     int32_t* __restrict__ gstart) {
    pdl_wait();
    pdl_trigger();
    const int64_t nn = hdr->n_nodes;
    const int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (id == 0 && nn <= capacity) {
        // The DFS may start at the first chain node that is not an internal
        // node with a single child in slot 0: every node above it covers all
        // points (its box holds every query) and keeps descending order.
        int L = 0;
        while (L < 32 && chain[32 + L] == 1) ++L;
        hdr->dfs_start = chain[L];
    }
    if (nn > capacity || (int64_t)blockIdx.x * blockDim.x >= nn) return;  // block-uniform
    const bool live = id < nn;
    // pass 0 counts the node's groups, pass 1 writes them from `out`.
    int64_t out = 0;
    int32_t ng = 0;
    int32_t start = -1;  // the traversal start of this node's groups
    for (int pass = 0; pass < 2; ++pass) {
        ng = 0;
        if (pass && gstart && live && ng == 0) {
            const TNode<T, D> nd = tnode[id];
            if (nd.b <= 0) {
                // P = this node: its level (depth) and the ancestors' chain
                constexpr int BITS = Dims<D>::bits;
                int32_t anc[BITS + 2];
                int depth = 0;
                for (int32_t a = (int32_t)id; a >= 0 && depth < BITS + 2; a = parent[a]) anc[depth++] = a;
                const int lp = depth - 1;  // anc[0] = P at level lp, anc[lp] = root
                const K kp = skeys[nrange[id].x];
                constexpr int64_t cmax = (1LL << BITS) - 1;
                int la = -1;  // deepest level whose cell holds P's cell +- kStartMargin
                for (int L = lp - 1; L >= 1 && la < 0; --L) {
                    const int sh = BITS - L;
                    bool ok = true;
#pragma unroll
                    for (int d = 0; d < D; ++d) {
                        const int64_t c = (int64_t)axis_cell<D, K>(kp, d);
                        const int64_t plo = (c >> (BITS - lp)) << (BITS - lp);
                        const int64_t phi = plo + (1LL << (BITS - lp)) - 1;
                        const int64_t slo = (c >> sh) << sh, shi = slo + (1LL << sh) - 1;
                        int64_t nlo = plo - kStartMargin, nhi = phi + kStartMargin;
                        nlo = nlo < 0 ? 0 : nlo;
                        nhi = nhi > cmax ? cmax : nhi;
                        ok = ok && nlo >= slo && nhi <= shi;
                    }
                    if (ok) la = L;
                }
                if (la >= 1) {
                    const int32_t sid = anc[lp - la];
                    bool casc = false;  // a strict ancestor of S with its first slot empty
                    for (int j = lp - la + 1; j <= lp; ++j) casc = casc || !(((unsigned)(-tnode[anc[j]].b)) & 1u);
                    start = sid | (casc ? (1 << 30) : 0);
                }
            }
        }
        auto emit = [&](int32_t first, int32_t count) {
            if (pass && out + ng < group_cap) {
                groups[out + ng] = make_int2(first, count);
                if (gstart) gstart[out + ng] = start;
            }
            ++ng;
        };
        if (live) {
            const TNode<T, D> nd = tnode[id];
            if (nd.b > 0) {
                // Only a leaf root (one per cloud in a batch) forms groups of
                // its own; other leaves are grouped by their parent.
                if (parent[id] < 0)
                    for (int32_t c0 = 0; c0 < nd.b; c0 += gmax) emit(nd.a + c0, min(gmax, nd.b - c0));
            } else {
                const int nc = __popc((unsigned)(-nd.b));
                int32_t gfirst = 0, gcount = 0;
                for (int j = 0; j < nc; ++j) {
                    const TNode<T, D> c = tnode[nd.a + j];
                    if (c.b <= 0) {  // internal child: close the open group
                        if (gcount) emit(gfirst, gcount);
                        gcount = 0;
                    } else if (c.b > gmax) {
                        if (gcount) emit(gfirst, gcount);
                        gcount = 0;
                        for (int32_t c0 = 0; c0 < c.b; c0 += gmax) emit(c.a + c0, min(gmax, c.b - c0));
                    } else {
                        if (gcount + c.b > gmax) {
                            emit(gfirst, gcount);
                            gcount = 0;
                        }
                        if (gcount == 0) gfirst = c.a;
                        gcount += c.b;
                    }
                }
                if (gcount) emit(gfirst, gcount);
            }
        }
        if (pass == 0) {
            int incl = ng;
            const int lane = threadIdx.x & 31;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += v;
            }
            const int tot = __shfl_sync(0xffffffffu, incl, 31);
            unsigned long long base = 0;
            if (lane == 31 && tot) base = atomicAdd((unsigned long long*)&hdr->n_groups, (unsigned long long)tot);
            base = __shfl_sync(0xffffffffu, base, 31);
            out = (int64_t)base + incl - ng;
            if (tot == 0) return;  // warp-uniform
        }
    }
}

// --------------------------------------------------- 8. reference views --
template <class T, int D>
__global__ void k_view_nodes(const TNode<T, D>* __restrict__ tnode, const int2* __restrict__ nrange, int64_t nn,
                             int32_t* __restrict__ vf, int32_t* __restrict__ vl, int32_t* __restrict__ vc,
                             T* __restrict__ vmin, T* __restrict__ vmax) {
    constexpr int NCH = Dims<D>::nch;
    const int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= nn) return;
    const TNode<T, D> nd = tnode[id];
    const int2 rg = nrange[id];
    vf[id] = rg.x + 1;
    vl[id] = rg.y + 1;
    int j = 0;
    for (int c = 0; c < NCH; ++c) {
        int32_t v = -1;
        if (nd.b < 0 && (((unsigned)(-nd.b) >> c) & 1u)) v = nd.a + (j++) + 1;
        vc[id * NCH + c] = v;
    }
#pragma unroll
    for (int d = 0; d < D; ++d) { vmin[id * D + d] = nd.lo[d]; vmax[id * D + d] = nd.hi[d]; }
}

template <class T, int D>
__global__ void k_view_perm(const SPt<T, D>* __restrict__ spts, int64_t n, int32_t* __restrict__ vp) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) vp[k] = spts[k].idx + 1;
}

// The retained per-point Morton codes of refit mode (src/api.jl:234-238),
// scattered from the sorted keys on demand: morton[perm[k]] = key[k].
template <class T, int D, class K>
__global__ void k_view_morton(const SPt<T, D>* __restrict__ spts, const K* __restrict__ skeys, int64_t n,
                              uint64_t* __restrict__ morton) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) morton[spts[k].idx] = (uint64_t)skeys[k];
}

// --------------------------------------------------------- 9. batches ----
// Per-cloud min/max (Julia order) and non-finite flag, one block per cloud:
// out[c*8 + 0..2] = min, [3..5] = max, [6] = non-finite.
template <class T, int D>
__global__ void __launch_bounds__(kThreads) k_cloud_bounds(const T* __restrict__ coords, const int64_t* __restrict__ coff,
                                                           double* __restrict__ out) {
    __shared__ T smin[kThreads / 32][D], smax[kThreads / 32][D];
    __shared__ int snan;
    const int c = blockIdx.x;
    const int64_t s0 = coff[c], s1 = coff[c + 1];
    if (threadIdx.x == 0) snan = 0;
    __syncthreads();
    T lo[D], hi[D];
#pragma unroll
    for (int d = 0; d < D; ++d) { lo[d] = T(INFINITY); hi[d] = T(-INFINITY); }
    int bad = 0;
    for (int64_t i = s0 + threadIdx.x; i < s1; i += blockDim.x) {
#pragma unroll
        for (int d = 0; d < D; ++d) {
            const T x = coords[D * i + d];
            if (!isfinite(x)) bad = 1;
            lo[d] = jl_min(lo[d], x);
            hi[d] = jl_max(hi[d], x);
        }
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int d = 0; d < D; ++d) {
        lo[d] = warp_min(lo[d]);
        hi[d] = warp_max(hi[d]);
    }
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(&snan, 1);
    if (lane == 0) {
#pragma unroll
        for (int d = 0; d < D; ++d) { smin[w][d] = lo[d]; smax[w][d] = hi[d]; }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w2 = 1; w2 < kThreads / 32; ++w2)
            for (int d = 0; d < D; ++d) {
                smin[0][d] = jl_min(smin[0][d], smin[w2][d]);
                smax[0][d] = jl_max(smax[0][d], smax[w2][d]);
            }
        double* p = out + (size_t)c * 8;
        for (int d = 0; d < D; ++d) { p[d] = (double)smin[0][d]; p[3 + d] = (double)smax[0][d]; }
        p[6] = snan ? 1.0 : 0.0;
    }
}

// Each cloud's DFS starts below its root's single-child chain (children in
// slot 0 only), whose nodes all cover the whole cloud.
template <class T, int D>
__global__ void k_cloud_start(const TNode<T, D>* __restrict__ tnode, Batch bt, int64_t capacity,
                              const OctHeader* hdr) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= bt.n_clouds || hdr->n_nodes > capacity) return;
    int32_t node = bt.croot[c];
    if (node >= 0) {
        for (int it = 0; it < 64; ++it) {
            const TNode<T, D> nd = tnode[node];
            if (nd.b != -1) break;
            node = nd.a;
        }
    }
    bt.cstart[c] = node;
}

__global__ void k_gather_edge_offsets(const int64_t* __restrict__ offsets, const int64_t* __restrict__ coff,
                                      int n_clouds, int64_t* __restrict__ eoff) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c <= n_clouds) eoff[c] = offsets[coff[c]];
}

// ---------------------------------------------------- 10. time stepping --
// Refit mode keeps the previous build's sorted keys and permutation.  Points
// move little between steps, so most keys are unchanged: re-encoding every
// point at its previous sorted position leaves the unchanged keys U sorted by
// (key, index) in place.  The changed keys M are few; they are collected,
// sorted by (key, index) in shared-memory chunks and ranked across chunks,
// then merged with U: an unchanged key at position p lands at
// (p - changed keys before p) + (keys of M below it), and the keys of M that
// fall between two consecutive unchanged keys are placed by the first of
// the two.  The merged order is exactly the stable sort of the new keys
// (src/sort.jl:15-24), so the topology and everything after it equal a full
// rebuild.  When no key changed, order and topology are kept and only the
// bounds are recomputed.
constexpr int kChunk = 2048;
constexpr int64_t kMaxMerged = 65536;  // above this many changed keys a full sort is cheaper
inline int64_t merge_cap(int64_t n) { return std::min<int64_t>(kMaxMerged, std::max<int64_t>(kChunk, n / 8)); }
constexpr int64_t kSpeculate = -2;  // run_pipeline: merge with the count of changed keys still on the device
constexpr int kRetry = -1;          // run_pipeline: the speculative merge did not apply

template <class K>
__device__ __forceinline__ bool key_less(K ka, int32_t ia, K kb, int32_t ib) {
    return ka < kb || (ka == kb && ia < ib);
}

// Number of entries of the (key, index)-sorted array (k, v)[0, len) below (key, idx).
template <class K>
__device__ __forceinline__ int64_t count_below(const K* __restrict__ k, const int32_t* __restrict__ v, int64_t len,
                                               K key, int32_t idx) {
    int64_t a = 0, b = len;
    while (a < b) {
        const int64_t mid = (a + b) >> 1;
        if (key_less(k[mid], v[mid], key, idx)) a = mid + 1; else b = mid;
    }
    return a;
}

// Re-encodes point perm[p] at its previous sorted position p, flags a changed
// key, counts the changes per block and appends the changed (key, index)
// pairs to (mk, mv) in any order (slots past `cap` are counted, not
// written).  The origin comes from this build's bounds reduce, with the
// host's arithmetic (src/cpu/bin_cpu.jl:22).
template <class T, int D, class K>
__global__ void __launch_bounds__(kThreads) k_resort_mark(const T* __restrict__ coords, int64_t n,
                                                          const int32_t* __restrict__ perm,
                                                          const K* __restrict__ keys, T inv_cs, OctHeader* hdr,
                                                          uint8_t* __restrict__ changed, int32_t* __restrict__ blockcnt,
                                                          K* __restrict__ mk, int32_t* __restrict__ mv, int64_t cap) {
    pdl_wait();
    pdl_trigger();
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool c = false;
    K nk = 0;
    int32_t i = 0;
    if (p < n) {
        T o[3] = {T(0), T(0), T(0)};
#pragma unroll
        for (int d = 0; d < D; ++d) o[d] = sub_rn((T)hdr->gmin[d], T(1e-6));
        i = perm[p];
        const uint64_t key = cell_key<T, D>(coords + (int64_t)D * i, o, inv_cs);
        nk = (K)key;
        if ((uint64_t)nk != key) atomicOr(&hdr->status, (int)DF_KEY_WIDTH);
        c = nk != keys[p];
        changed[p] = (uint8_t)c;
    }
    const unsigned bal = __ballot_sync(0xffffffffu, c);
    if (bal) {
        const int lane = threadIdx.x & 31;
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd((unsigned long long*)&hdr->n_moved, (unsigned long long)__popc(bal));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (c) {
            const int64_t slot = (int64_t)base + __popc(bal & lanemask_lt());
            if (slot < cap) {
                mk[slot] = nk;
                mv[slot] = i;
            }
        }
    }
    const int cnt = __syncthreads_count(c);
    if (threadIdx.x == 0) blockcnt[blockIdx.x] = cnt;
}

// Sorts each chunk of up to kChunk changed keys by (key, index) in shared
// memory: a bitonic network of `width` entries (a power of two, the chunk
// size rounded up), width / 2 compare-exchanges per stage shared by the
// block's threads.  The count m is read on the device (*m_ptr); nothing is sorted
// when m exceeds cap.
template <class K>
__global__ void __launch_bounds__(kChunk / 2) k_moved_sort(const int64_t* __restrict__ m_ptr, int64_t cap,
                                                           K* __restrict__ mk, int32_t* __restrict__ mv) {
    pdl_wait();
    pdl_trigger();
    __shared__ K sk[kChunk];
    __shared__ int32_t sv[kChunk];
    const int64_t m = *m_ptr;
    if (m > cap || (int64_t)blockIdx.x * kChunk >= m) return;  // block-uniform
    int width = 64;
    while (width < m && width < kChunk) width <<= 1;
    const int64_t base = (int64_t)blockIdx.x * kChunk;
    for (int t = threadIdx.x; t < width; t += blockDim.x) {
        const int64_t j = base + t;
        if (j < m) {
            sk[t] = mk[j];
            sv[t] = mv[j];
        } else {
            sk[t] = ~K(0);
            sv[t] = INT32_MAX;  // above every real index: padding sorts last
        }
    }
    __syncthreads();
    for (int size = 2; size <= width; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int t = threadIdx.x; t < width / 2; t += blockDim.x) {
                const int i = 2 * t - (t & (stride - 1));
                const int j = i + stride;
                const bool up = (i & size) == 0;
                const K ki = sk[i], kj = sk[j];
                const int32_t vi = sv[i], vj = sv[j];
                if (key_less(kj, vj, ki, vi) == up) {
                    sk[i] = kj;
                    sk[j] = ki;
                    sv[i] = vj;
                    sv[j] = vi;
                }
            }
            __syncthreads();
        }
    }
    for (int t2 = threadIdx.x; t2 < width; t2 += blockDim.x) {
        const int64_t j = base + t2;
        if (j < m) {
            mk[j] = sk[t2];
            mv[j] = sv[t2];
        }
    }
}

// Global rank of each changed key: its rank in its own chunk plus the number
// of smaller keys in every other chunk.
template <class K>
__global__ void __launch_bounds__(kThreads) k_moved_rank(const int64_t* __restrict__ m_ptr, int64_t cap,
                                                         const K* __restrict__ ck, const int32_t* __restrict__ cv,
                                                         K* __restrict__ sk, int32_t* __restrict__ sv) {
    pdl_wait();
    pdl_trigger();
    const int64_t m = *m_ptr;
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (m > cap || m <= kChunk || j >= m) return;  // one chunk is already in order
    const K key = ck[j];
    const int32_t idx = cv[j];
    const int64_t own = j / kChunk;
    int64_t r = j - own * kChunk;
    const int64_t nchunks = (m + kChunk - 1) / kChunk;
    for (int64_t c = 0; c < nchunks; ++c) {
        if (c == own) continue;
        const int64_t b = c * kChunk;
        r += count_below(ck + b, cv + b, m - b < kChunk ? m - b : (int64_t)kChunk, key, idx);
    }
    sk[r] = key;
    sv[r] = idx;
}

template <class T, int D, class K>
__device__ __forceinline__ void put_sorted(int64_t pos, K key, int32_t idx, const T* __restrict__ coords,
                                           K* __restrict__ okeys, int32_t* __restrict__ operm,
                                           SPt<T, D>* __restrict__ spts, int32_t* __restrict__ iperm) {
    iperm[idx] = (int32_t)pos;
    okeys[pos] = key;
    operm[pos] = idx;
    SPt<T, D> sp;
#pragma unroll
    for (int d = 0; d < D; ++d) sp.x[d] = coords[(int64_t)D * idx + d];
    sp.idx = idx;
    spts[pos] = sp;
}

// Merges the unchanged keys (in place at their previous positions) with the
// sorted changed keys (mk, mv)[0, m) into (okeys, operm), and gathers the
// sorted points (the gather of section 4).  changed_before[b] counts the
// changed positions before block b.
template <class T, int D, class K>
__global__ void __launch_bounds__(kThreads) k_resort_merge(int64_t n, const int64_t* __restrict__ m_ptr, int64_t cap,
                                                           const K* __restrict__ keys,
                                                           const int32_t* __restrict__ perm,
                                                           const uint8_t* __restrict__ changed,
                                                           const int64_t* __restrict__ changed_before,
                                                           const K* __restrict__ mk1, const int32_t* __restrict__ mv1,
                                                           const K* __restrict__ mk2, const int32_t* __restrict__ mv2,
                                                           const T* __restrict__ coords, K* __restrict__ okeys,
                                                           int32_t* __restrict__ operm, SPt<T, D>* __restrict__ spts,
                                                           int32_t* __restrict__ iperm) {
    pdl_wait();
    pdl_trigger();
    __shared__ int wsum[kThreads / 32];
    __shared__ int64_t sbound[2];
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t m = *m_ptr;
    if (m > cap) {
        // Too many changed keys for a merge (the caller sorts afresh): keep
        // the previous order, so that what follows reads a valid permutation.
        if (p < n) put_sorted<T, D, K>(p, keys[p], perm[p], coords, okeys, operm, spts, iperm);
        return;
    }
    // Sorted changed keys: ranked across chunks when there are several.
    const K* __restrict__ mk = m > kChunk ? mk2 : mk1;
    const int32_t* __restrict__ mv = m > kChunk ? mv2 : mv1;
    if (m == n) {  // every key changed: the sorted changed keys are the result
        if (p < n) put_sorted<T, D, K>(p, mk[p], mv[p], coords, okeys, operm, spts, iperm);
        return;
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    // The previous (key, index) order is sorted, so the changed keys below any
    // entry of this block lie between those below its first entry and those
    // below the next block's first: two full searches per block, then each
    // thread searches only that span (usually a few entries).
    const int64_t b0 = (int64_t)blockIdx.x * blockDim.x;
    if (threadIdx.x < 2) {
        const int64_t q = b0 + (threadIdx.x ? (int64_t)blockDim.x : 0);
        sbound[threadIdx.x] = q < n ? count_below(mk, mv, m, keys[q], perm[q]) : m;
    }
    const bool in = p < n;
    const bool c = in && changed[p];
    const bool u = in && !c;
    const unsigned cbal = __ballot_sync(0xffffffffu, c);
    const unsigned ubal = __ballot_sync(0xffffffffu, u);
    if (lane == 0) wsum[w] = __popc(cbal);
    __syncthreads();
    const int64_t blo = sbound[0], bhi = sbound[1];
    int before = __popc(cbal & lanemask_lt());
    for (int j = 0; j < w; ++j) before += wsum[j];
    K key = 0;
    int32_t idx = 0;
    int64_t s = 0;
    if (u) {
        key = keys[p];
        idx = perm[p];
        s = blo + count_below(mk + blo, mv + blo, bhi - blo, key, idx);
    }
    // Changed keys below the next unchanged key: from the next unchanged lane
    // of this warp, or found past the warp's end.
    const unsigned later = ubal & ~((2u << lane) - 1u);
    const int src = later ? __ffs(later) - 1 : lane;
    int64_t sn = __shfl_sync(0xffffffffu, s, src);
    if (!u) return;
    if (!later) {
        int64_t q = p - lane + 32;
        while (q < n && changed[q]) ++q;
        if (q >= n)
            sn = m;
        else if (q < b0 + (int64_t)blockDim.x)
            sn = blo + count_below(mk + blo, mv + blo, bhi - blo, keys[q], perm[q]);
        else if (q == b0 + (int64_t)blockDim.x)
            sn = bhi;
        else
            sn = count_below(mk, mv, m, keys[q], perm[q]);
    }
    const int64_t ui = p - (changed_before[blockIdx.x] + before);  // rank among unchanged keys
    put_sorted<T, D, K>(ui + s, key, idx, coords, okeys, operm, spts, iperm);
    for (int64_t j = s; j < sn; ++j) put_sorted<T, D, K>(j + ui + 1, mk[j], mv[j], coords, okeys, operm, spts, iperm);
    if (ui == 0)
        for (int64_t j = 0; j < s; ++j) put_sorted<T, D, K>(j, mk[j], mv[j], coords, okeys, operm, spts, iperm);
}

// Bounds-only step (no key changed): the topology is kept; reset the refit
// arrival counters and preset the full-range nodes from this build's reduce.
template <class T, int D>
__global__ void __launch_bounds__(kThreads) k_refit_prepare(int64_t nn, int64_t n, TNode<T, D>* __restrict__ tnode,
                                                            const int2* __restrict__ nrange,
                                                            int32_t* __restrict__ arrive, OctHeader* hdr,
                                                            int64_t n_groups, int32_t dfs_start) {
    pdl_wait();
    pdl_trigger();
    const int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (id == 0) {
        hdr->n_nodes = nn;
        hdr->n_groups = n_groups;
        hdr->dfs_start = dfs_start;
    }
    if (id >= nn) return;
    arrive[id] = 0;
    const int2 rg = nrange[id];
    if (rg.x == 0 && (int64_t)rg.y == n - 1) {
#pragma unroll
        for (int d = 0; d < D; ++d) {
            tnode[id].lo[d] = (T)hdr->gmin[d];
            tnode[id].hi[d] = (T)hdr->gmax[d];
        }
    }
}

// ----------------------------------------------------------- 11. guards --
// Guard-check mode (OCT_OPT_GUARD_CHECK): a canary region follows the part of
// each sort buffer and node array that the build may write; after each
// topology attempt every canary byte is compared and the mismatches are
// counted into hdr->guard_bad.
constexpr size_t kGuardBytes = 16384;
constexpr unsigned char kGuardByte = 0xA5;

__global__ void k_guard_check(const unsigned char* __restrict__ p, int64_t len, int* __restrict__ bad) {
    int c = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x)
        c += p[i] != kGuardByte;
    c = warp_sum(c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(bad, c);
}

// ------------------------------------------------------------- host side --
namespace {

// In guard-check mode, `b` holds `bytes` plus a canary region after them.
cudaError_t ensure_g(const Ctx& ctx, DevBuf& b, size_t bytes) {
    return ensure(b, bytes + (ctx.guard_check ? kGuardBytes : 0));
}
cudaError_t guard_fill(const Ctx& ctx, const DevBuf& b, size_t bytes) {
    if (!ctx.guard_check) return cudaSuccess;
    return cudaMemsetAsync(static_cast<unsigned char*>(b.p) + bytes, kGuardByte, kGuardBytes, ctx.stream);
}
void guard_check(Ctx& ctx, const DevBuf& b, size_t bytes, OctHeader* hdr) {
    if (!ctx.guard_check) return;
    k_guard_check<<<8, 256, 0, ctx.stream>>>(static_cast<const unsigned char*>(b.p) + bytes, (int64_t)kGuardBytes,
                                            &hdr->guard_bad);
    ctx.kernel_launches += 1;
}

template <class T, int D, class K>
int run_pipeline(Ctx& ctx, Tree& t, const T* coords, int64_t n, T radius, int64_t moved = -1, int prev = -1) {
    const Batch bt = t.batch();
    cudaStream_t s = ctx.stream;
    cudaError_t err;
    constexpr int BITS = Dims<D>::bits;
    constexpr int NLEV = BITS + 1;
    const T inv_cs = T(1) / radius;  // src/cpu/bin_cpu.jl:60
    T o[3] = {T(0), T(0), T(0)};
    for (int d = 0; d < D; ++d) o[d] = (T)t.origin[d];

    if ((err = ensure(t.spts, (size_t)n * sizeof(SPt<T, D>))) || (err = ensure(t.iperm, (size_t)n * 4)))
        return cuda_status(ctx, err, "allocating points");
    OctHeader* hdr = t.hdr.as<OctHeader>();
    const K* skeys;
    const int32_t* perm;
    int sorted = -1;  // buffer holding this build's sorted keys and permutation
    if (moved == -1) {  // a full sort
        // Keys and points sorted together (stable: ties keep ascending
        // original index, src/sort.jl:15-24), the encode fused into the sort.
        const int passes = t.sort_passes;
        if ((err = ensure_g(ctx, t.keys[0], (size_t)n * sizeof(K))) ||
            (err = ensure_g(ctx, t.keys[1], (size_t)n * sizeof(K))) || (err = ensure_g(ctx, t.vals[0], (size_t)n * 4)) ||
            (err = ensure_g(ctx, t.spts, (size_t)n * sizeof(SPt<T, D>))) ||
            (err = ensure_g(ctx, t.spts_tmp, (size_t)n * sizeof(SPt<T, D>))) ||
            (err = ensure_g(ctx, t.iperm, (size_t)n * 4)) ||
            (err = ensure(t.vals[1], (size_t)n * 4)))  // the next refit-mode merge writes here
            return cuda_status(ctx, err, "allocating sort buffers");
        for (int b = 0; b < 2; ++b)
            if ((err = guard_fill(ctx, t.keys[b], (size_t)n * sizeof(K)))) return cuda_status(ctx, err, "sort guards");
        if ((err = guard_fill(ctx, t.vals[0], (size_t)n * 4)) ||
            (err = guard_fill(ctx, t.spts, (size_t)n * sizeof(SPt<T, D>))) ||
            (err = guard_fill(ctx, t.spts_tmp, (size_t)n * sizeof(SPt<T, D>))) ||
            (err = guard_fill(ctx, t.iperm, (size_t)n * 4)))
            return cuda_status(ctx, err, "sort guards");
        if (passes == 0) {
            // Every point in one cell: keys all equal, the input order stands.
            PhaseTimer pt_(ctx, PH_SORT);
            k_encode<T, D, K><<<div_up(n, kThreads), kThreads, 0, s>>>(coords, n, o[0], o[1], o[2], inv_cs,
                                                                        t.keys[0].as<K>(), bt);
            k_gather<T, D><<<div_up(n, kThreads), kThreads, 0, s>>>(coords, nullptr, n, t.spts.as<SPt<T, D>>(),
                                                                    t.iperm.as<int32_t>(), &hdr->status);
            ctx.kernel_launches += 2;
            t.iperm_valid = true;
            perm = nullptr;
        } else {
            if ((err = ensure(t.look, onesweep_words(n, passes) * 4)))
                return cuda_status(ctx, err, "allocating sort scratch");
            int sms = 0;
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx.device);
            EncodeParams<T> ep;
            ep.o[0] = o[0];
            ep.o[1] = o[1];
            ep.o[2] = o[2];
            ep.inv_cs = inv_cs;
            ep.bt = bt;
            PhaseTimer pt_(ctx, PH_SORT);
            // the inverse permutation is left to its first user (ensure_iperm)
            err = point_sort<T, D, K>(coords, ep, n, passes, t.keys[0].as<K>(), t.keys[1].as<K>(),
                                      t.spts.as<SPt<T, D>>(), t.spts_tmp.as<SPt<T, D>>(), t.vals[0].as<int32_t>(),
                                      nullptr, t.look.as<uint32_t>(), &hdr->status, sms, ctx.wait_limit,
                                      ctx.withhold_tile, s, &ctx.kernel_launches);
            if (err) return cuda_status(ctx, err, "key sort launch");
            t.iperm_valid = false;
            perm = t.vals[0].as<int32_t>();
            if (!bt.n_clouds) sorted = 0;
        }
        skeys = t.keys[0].as<K>();
        t.last_path = 0;
    } else {
        // Refit mode, keys already re-encoded in the previous order (section 10).
        K* kp = t.keys[prev].as<K>();
        int32_t* vp = t.vals[prev].as<int32_t>();
        skeys = kp;
        perm = vp;
        sorted = prev;
        if (moved == 0) {
            // Same keys, same order, same topology: new bounds only.
            {
                PhaseTimer pt_(ctx, PH_GATHER);
                k_gather<T, D><<<div_up(n, kThreads), kThreads, 0, s>>>(coords, vp, n, t.spts.as<SPt<T, D>>(),
                                                                    t.iperm.as<int32_t>(), &hdr->status);
                ctx.kernel_launches += 1;
                t.iperm_valid = true;
            }
            {
                PhaseTimer pt_(ctx, PH_REFIT);
                const int nb = div_up(t.n_nodes, kThreads);
                launch_pdl(k_refit_prepare<T, D>, nb, kThreads, 0, s, t.n_nodes, n, t.tnode.as<TNode<T, D>>(),
                    t.nrange.as<int2>(), t.arrive.as<int32_t>(), hdr, t.n_groups, t.dfs_start);
                launch_pdl(k_refit<T, D>, nb, kThreads, 0, s, t.capacity, n, t.tnode.as<TNode<T, D>>(),
                    t.nrange.as<int2>(), t.parent.as<int32_t>(), t.arrive.as<int32_t>(), t.spts.as<SPt<T, D>>(), hdr,
                    bt);
                ctx.kernel_launches += 2;
            }
            if ((err = cudaGetLastError())) return cuda_status(ctx, err, "bounds refit");
            t.last_path = 2;
            t.sorted_buf = sorted;
            t.perm_dev = vp;
            t.skeys_dev = skeys;
            t.key_bytes = (int)sizeof(K);
            return OK;
        }
        // The changed keys' count is read on the device; when it is not known
        // yet (a speculative build) the grids cover the merge capacity.
        const int nb = div_up(n, kThreads);
        const int64_t mcap = merge_cap(n);
        const int64_t mmax = moved == kSpeculate ? mcap : moved;
        const int64_t nchunks = div_up(mmax, kChunk);
        int width = 64;
        while (width < mmax && width < kChunk) width <<= 1;
        if ((err = ensure(t.mkeys2, (size_t)mmax * sizeof(K))) || (err = ensure(t.mvals2, (size_t)mmax * 4)))
            return cuda_status(ctx, err, "allocating changed keys");
        K* mk = t.mkeys.as<K>();
        int32_t* mv = t.mvals.as<int32_t>();
        K* ok = t.keys[1 - prev].as<K>();
        int32_t* ov = t.vals[1 - prev].as<int32_t>();
        {
            PhaseTimer pt_(ctx, PH_SORT);
            // Threads per chunk: width / 2 when the count is known, else 256.
            const int tpb = moved == kSpeculate ? 256 : std::max(32, width / 2);
            launch_pdl(k_moved_sort<K>, (unsigned)nchunks, tpb, 0, s, &hdr->n_moved, mcap, mk, mv);
            ctx.kernel_launches += 1;
            if (nchunks > 1) {
                launch_pdl(k_moved_rank<K>, div_up(mmax, kThreads), kThreads, 0, s, &hdr->n_moved, mcap, mk, mv,
                    t.mkeys2.as<K>(), t.mvals2.as<int32_t>());
                ctx.kernel_launches += 1;
            }
            launch_pdl(k_resort_merge<T, D, K>, nb, kThreads, 0, s, n, &hdr->n_moved, mcap, kp, vp,
                t.rflag.as<uint8_t>(), t.roff.as<int64_t>(), mk, mv, t.mkeys2.as<K>(), t.mvals2.as<int32_t>(), coords,
                ok, ov, t.spts.as<SPt<T, D>>(), t.iperm.as<int32_t>());
            ctx.kernel_launches += 1;
            t.iperm_valid = true;
        }
        skeys = ok;
        perm = ov;
        sorted = 1 - prev;
        t.last_path = 1;
    }

    // --- topology + refit (retried once with the exact node count on overflow)
    const int nblocks = div_up(n, kMarkTile);
    t.n_mark_blocks = nblocks;
    const int64_t nbc = (int64_t)NLEV * nblocks;
    if ((err = ensure(t.lohi, (size_t)n * 2)) || (err = ensure(t.blockcnt, (size_t)nbc * 4)) ||
        (err = ensure(t.blockoff, (size_t)(nbc + 1) * 8)) ||
        (err = ensure(t.scan_tmp, (size_t)scan_tmp_elems(nbc) * 8)))
        return cuda_status(ctx, err, "allocating topology scratch");
    int64_t est = (int64_t)Dims<D>::nch * ((n + 31) / 32) + 2 * NLEV + 64;
    if (ctx.node_cap_override > 0)
        t.capacity = ctx.node_cap_override;  // the first attempt's capacity, as set by the caller
    else if (t.capacity < est)
        t.capacity = est;
    // Query points per traversal group (a tuned shape; 32 by default).
    const int gmax = ctx.tuning_for(t.ndims, t.dtype, n, t.nbrs_hint).group_cap;
    t.group_cap = gmax;
    for (int attempt = 0; attempt < 3; ++attempt) {
        ctx.last_attempts = attempt + 1;
        const int64_t cap = t.capacity;
        const size_t gcap = (size_t)(cap + n / gmax + 2);
        if ((err = ensure_g(ctx, t.tnode, (size_t)cap * sizeof(TNode<T, D>))) ||
            (err = ensure_g(ctx, t.nrange, (size_t)cap * 8)) || (err = ensure_g(ctx, t.parent, (size_t)cap * 4)) ||
            (err = ensure_g(ctx, t.arrive, (size_t)cap * 4)) || (err = ensure_g(ctx, t.fchild, (size_t)cap * 4)) ||
            (err = ensure(t.scan_tmp, (size_t)scan_tmp_elems(nbc) * 8)) ||
            (err = ensure_g(ctx, t.groups, gcap * 8)) || (err = ensure(t.gstart, gcap * 4)) ||
            (err = ensure(t.chain, 64 * 4)))
            return cuda_status(ctx, err, "allocating node arrays");
        if ((err = cudaMemsetAsync(t.chain.p, 0xff, 64 * 4, s)) ||
            (err = cudaMemsetAsync(&hdr->n_groups, 0, sizeof(int64_t), s)))
            return cuda_status(ctx, err, "chain reset");
        if ((err = guard_fill(ctx, t.tnode, (size_t)cap * sizeof(TNode<T, D>))) ||
            (err = guard_fill(ctx, t.nrange, (size_t)cap * 8)) || (err = guard_fill(ctx, t.parent, (size_t)cap * 4)) ||
            (err = guard_fill(ctx, t.arrive, (size_t)cap * 4)) || (err = guard_fill(ctx, t.fchild, (size_t)cap * 4)) ||
            (err = guard_fill(ctx, t.groups, gcap * 8)))
            return cuda_status(ctx, err, "node array guards");
        if (bt.n_clouds && (err = cudaMemsetAsync(bt.croot, 0xff, (size_t)bt.n_clouds * 4, s)))
            return cuda_status(ctx, err, "cloud root reset");
        {
        PhaseTimer pt_(ctx, PH_TOPOLOGY);
        launch_pdl(k_mark<D, K>, nblocks, kThreads, 0, s, skeys, n, t.lohi.as<uint16_t>(), t.blockcnt.as<int32_t>(),
            nblocks, bt);
        ctx.kernel_launches += exclusive_scan_i32_i64(t.blockcnt.as<int32_t>(), t.blockoff.as<int64_t>(), nbc,
                                                      &hdr->n_nodes, t.scan_tmp.as<int64_t>(), s);
        launch_pdl(k_emit_ids<D>, nblocks, kThreads, 0, s, n, t.lohi.as<uint16_t>(), t.blockoff.as<int64_t>(), nblocks,
            cap, t.fchild.as<int32_t>(), t.nrange.as<int2>(), t.arrive.as<int32_t>(), hdr, bt);
        launch_pdl(k_emit_nodes<T, D, K>, div_up(cap, kThreads), kThreads, 0, s, skeys, n, cap, t.fchild.as<int32_t>(),
            t.tnode.as<TNode<T, D>>(), t.nrange.as<int2>(), t.parent.as<int32_t>(), t.arrive.as<int32_t>(),
            t.chain.as<int32_t>(), t.blockoff.as<int64_t>(), nblocks, hdr, bt);
        ctx.kernel_launches += 3;
        }
        {
        PhaseTimer pt_(ctx, PH_REFIT);
        launch_pdl(k_refit<T, D>, div_up(cap, kThreads), kThreads, 0, s, cap, n, t.tnode.as<TNode<T, D>>(),
            t.nrange.as<int2>(), t.parent.as<int32_t>(), t.arrive.as<int32_t>(), t.spts.as<SPt<T, D>>(), hdr, bt);
        ctx.kernel_launches += 1;
        }
        {
            PhaseTimer pt_(ctx, PH_GROUPS);
            launch_pdl(k_groups<T, D, K>, div_up(cap, kThreads), kThreads, 0, s, t.tnode.as<TNode<T, D>>(), cap,
                t.groups.as<int2>(), (int64_t)gcap, t.chain.as<int32_t>(), t.parent.as<int32_t>(), hdr, gmax, skeys,
                t.nrange.as<int2>(), bt.n_clouds ? nullptr : t.gstart.as<int32_t>());
            ctx.kernel_launches += 1;
            if (bt.n_clouds) {
                k_cloud_start<T, D><<<div_up(bt.n_clouds, 128), 128, 0, s>>>(t.tnode.as<TNode<T, D>>(), bt, cap, hdr);
                ctx.kernel_launches += 1;
            }
        }
        if (ctx.guard_check) {
            guard_check(ctx, t.tnode, (size_t)cap * sizeof(TNode<T, D>), hdr);
            guard_check(ctx, t.nrange, (size_t)cap * 8, hdr);
            guard_check(ctx, t.parent, (size_t)cap * 4, hdr);
            guard_check(ctx, t.arrive, (size_t)cap * 4, hdr);
            guard_check(ctx, t.fchild, (size_t)cap * 4, hdr);
            guard_check(ctx, t.groups, gcap * 8, hdr);
            if (moved == -1) {
                for (int b = 0; b < 2; ++b) guard_check(ctx, t.keys[b], (size_t)n * sizeof(K), hdr);
                guard_check(ctx, t.vals[0], (size_t)n * 4, hdr);
                guard_check(ctx, t.spts, (size_t)n * sizeof(SPt<T, D>), hdr);
                guard_check(ctx, t.spts_tmp, (size_t)n * sizeof(SPt<T, D>), hdr);
                guard_check(ctx, t.iperm, (size_t)n * 4, hdr);
            }
        }
        if ((err = cudaMemcpyAsync(t.hdr_host, hdr, sizeof(OctHeader), cudaMemcpyDeviceToHost, s)) ||
            (err = wait_stream(s)))
            return cuda_status(ctx, err, "tree build");
        if (t.hdr_host->guard_bad)
            return set_error(ctx, ERR_STATE, "tree build: a kernel wrote past the end of a sort buffer or node array");
        if (moved == kSpeculate &&
            (t.hdr_host->nan_flag || t.hdr_host->n_moved > merge_cap(n) || (t.hdr_host->status & DF_KEY_WIDTH)))
            return kRetry;  // the bounds say the merge did not apply: build again on the usual path
        if (t.hdr_host->status & DF_TIMEOUT)
            return set_error(ctx, ERR_TIMEOUT, "tree build: a radix-sort look-back wait ran out");
        if (t.hdr_host->status & DF_NODE_OVERFLOW) {
            t.capacity = t.hdr_host->n_nodes + t.hdr_host->n_nodes / 8 + 64;
            const int zero = 0;
            cudaMemcpyAsync(&hdr->status, &zero, sizeof(int), cudaMemcpyHostToDevice, s);
            continue;
        }
        t.n_nodes = t.hdr_host->n_nodes;
        t.n_groups = t.hdr_host->n_groups;
        t.dfs_start = t.hdr_host->dfs_start;
        t.sorted_buf = sorted;
        t.perm_dev = perm;
        t.skeys_dev = skeys;
        t.key_bytes = (int)sizeof(K);
        return OK;
    }
    return set_error(ctx, ERR_OVERFLOW, "tree build: node capacity retry did not converge");
}

// Refit mode: re-encodes every point at its previous sorted position and
// counts the changed keys into hdr->n_moved (read with the bounds).
template <class T, int D, class K>
int resort_mark(Ctx& ctx, Tree& t, const T* coords, int64_t n, T radius, int prev, int64_t cap) {
    cudaStream_t s = ctx.stream;
    cudaError_t err;
    const int nb = div_up(n, kThreads);
    if ((err = ensure(t.rflag, (size_t)n)) || (err = ensure(t.rcnt, (size_t)nb * 4)) ||
        (err = ensure(t.roff, (size_t)(nb + 1) * 8)) || (err = ensure(t.scan_tmp, (size_t)scan_tmp_elems(nb) * 8)) ||
        (err = ensure(t.mkeys, (size_t)cap * sizeof(K))) || (err = ensure(t.mvals, (size_t)cap * 4)))
        return cuda_status(ctx, err, "allocating refit-mode scratch");
    OctHeader* hdr = t.hdr.as<OctHeader>();
    PhaseTimer pt_(ctx, PH_ENCODE);
    launch_pdl(k_resort_mark<T, D, K>, nb, kThreads, 0, s, coords, n, t.vals[prev].as<int32_t>(), t.keys[prev].as<K>(),
        T(1) / radius, hdr, t.rflag.as<uint8_t>(), t.rcnt.as<int32_t>(), t.mkeys.as<K>(), t.mvals.as<int32_t>(), cap);
    ctx.kernel_launches += 1 + exclusive_scan_i32_i64(t.rcnt.as<int32_t>(), t.roff.as<int64_t>(), nb, nullptr,
                                                      t.scan_tmp.as<int64_t>(), s);
    return OK;
}

// Origin and key width on the host from the bounds in t.hdr_host, in T
// (src/cpu/bin_cpu.jl:22,35,60); InexactError where the reference's
// floor(Int32, ...) throws.
template <class T, int D>
int host_key_width(Ctx& ctx, Tree& t, T radius) {
    if (t.hdr_host->nan_flag)
        return set_error(ctx, ERR_INEXACT, "InexactError: floor(Int32, NaN/Inf) in bin_point (non-finite coordinate)");
    const T inv_cs = T(1) / radius;
    int64_t cmax_all = 0;
    for (int d = 0; d < D; ++d) {
        const T o = (T)t.hdr_host->gmin[d] - T(1e-6);
        t.origin[d] = (double)o;
        const T v = ((T)t.hdr_host->gmax[d] - o) * inv_cs;
        const T f = std::floor(v);
        if (!(f >= T(-2147483648.0) && f < T(2147483648.0)))
            return set_error(ctx, ERR_INEXACT, "InexactError: floor(Int32, (p - origin) / radius) exceeds Int32");
        int64_t c = (int64_t)f;
        const int64_t cm = (1LL << Dims<D>::bits) - 1;
        c = c < 0 ? 0 : (c > cm ? cm : c);
        cmax_all = std::max(cmax_all, c);
    }
    int nbits_axis = 0;
    while (nbits_axis < 63 && (cmax_all >> nbits_axis) != 0) ++nbits_axis;
    t.key_bits = D * nbits_axis;
    t.key_bytes = t.key_bits <= 32 ? 4 : 8;
    t.sort_passes = (t.key_bits + 7) / 8;
    return OK;
}

template <class T, int D>
int build_typed(Ctx& ctx, Tree& t, const T* coords, int64_t n, double radius_d) {
    cudaStream_t s = ctx.stream;
    cudaError_t err;
    const T radius = (T)radius_d;
    if ((err = ensure(t.hdr, sizeof(OctHeader)))) return cuda_status(ctx, err, "allocating header");
    if (!t.hdr_host) {
        if ((err = cudaMallocHost((void**)&t.hdr_host, sizeof(OctHeader)))) return cuda_status(ctx, err, "pinned header");
    }
    OctHeader* hdr = t.hdr.as<OctHeader>();
    if ((err = cudaMemsetAsync(hdr, 0, sizeof(OctHeader), s))) return cuda_status(ctx, err, "header reset");

    // --- 1. bounds (one host round trip, like ext/cuda_build.jl:235)
    const int nb = std::max(1, std::min(div_up(n, kThreads * 8), 4 * 148));
    if ((err = ensure(t.partials, (size_t)nb * 8 * 8))) return cuda_status(ctx, err, "allocating partials");
    {
        PhaseTimer pt_(ctx, PH_BOUNDS);
        launch_pdl(k_bounds<T, D>, nb, kThreads, 0, s, coords, n, t.partials.as<double>(), hdr);
        ctx.kernel_launches += 1;
    }
    // Refit mode with a reusable previous order: re-encode in that order now,
    // so the count of changed keys arrives with the bounds.
    const int prev = t.sorted_buf;
    t.sorted_buf = -1;
    const bool try_resort = t.keep_morton && prev >= 0 && t.sorted_n == n && t.sorted_radius == radius_d;
    // Merge at most this many changed keys; more are cheaper to sort afresh.
    const int64_t cap = merge_cap(n);
    if (try_resort) {
        const int st = t.sorted_key_bytes == 4 ? resort_mark<T, D, uint32_t>(ctx, t, coords, n, radius, prev, cap)
                                               : resort_mark<T, D, uint64_t>(ctx, t, coords, n, radius, prev, cap);
        if (st != OK) return st;
    }
    // Steady time stepping: the previous build merged its changed keys, so
    // merge again without waiting for the bounds.  The round trip at the end
    // of the topology brings the bounds, the count of changed keys and the
    // key-width flag; if the merge did not apply, build again below.
    if (try_resort && t.last_path == 1) {
        const int st = t.sorted_key_bytes == 4
                           ? run_pipeline<T, D, uint32_t>(ctx, t, coords, n, radius, kSpeculate, prev)
                           : run_pipeline<T, D, uint64_t>(ctx, t, coords, n, radius, kSpeculate, prev);
        if (st != kRetry) {
            if (st != OK) return st;
            const int kw = host_key_width<T, D>(ctx, t, radius);
            if (kw != OK) return kw;
            t.key_bytes = t.sorted_key_bytes;  // the width the keys were built with
            t.last_moved = t.hdr_host->n_moved;
            t.last_path = 1;
            t.sorted_n = n;
            t.sorted_radius = radius_d;
            return OK;
        }
        t.sorted_buf = -1;
    } else if ((err = cudaMemcpyAsync(t.hdr_host, hdr, sizeof(OctHeader), cudaMemcpyDeviceToHost, s)) ||
               (err = wait_stream(s))) {
        return cuda_status(ctx, err, "bounds reduce");
    }
    const int kw = host_key_width<T, D>(ctx, t, radius);
    if (kw != OK) return kw;
    // Merge the changed keys into the previous order unless they are too many
    // (or the key width changed).
    int64_t moved = -1;
    t.last_moved = try_resort ? t.hdr_host->n_moved : -1;
    if (try_resort && t.key_bytes == t.sorted_key_bytes && t.hdr_host->n_moved <= cap) moved = t.hdr_host->n_moved;
    const int st = t.key_bytes == 4 ? run_pipeline<T, D, uint32_t>(ctx, t, coords, n, radius, moved, prev)
                                    : run_pipeline<T, D, uint64_t>(ctx, t, coords, n, radius, moved, prev);
    if (st == OK && t.sorted_buf >= 0) {
        t.sorted_n = n;
        t.sorted_radius = radius_d;
        t.sorted_key_bytes = t.key_bytes;
    }
    return st;
}

template <class T, int D>
int build_batch_typed(Ctx& ctx, Tree& t, const T* coords, int64_t n, const int64_t* coff_host,
                      const double* radii_host, int32_t nc) {
    cudaStream_t s = ctx.stream;
    cudaError_t err;
    if ((err = ensure(t.hdr, sizeof(OctHeader))) || (err = ensure(t.b_coff, (size_t)(nc + 1) * 8)) ||
        (err = ensure(t.b_cparam, (size_t)nc * kCloudParams * 8)) || (err = ensure(t.b_croot, (size_t)nc * 4)) ||
        (err = ensure(t.b_cstart, (size_t)nc * 4)) || (err = ensure(t.b_cbounds, (size_t)nc * 8 * 8)) ||
        (err = ensure(t.b_eoff, (size_t)(nc + 1) * 8)))
        return cuda_status(ctx, err, "allocating batch arrays");
    if (!t.hdr_host) {
        if ((err = cudaMallocHost((void**)&t.hdr_host, sizeof(OctHeader)))) return cuda_status(ctx, err, "pinned header");
    }
    if ((err = cudaMemsetAsync(t.hdr.p, 0, sizeof(OctHeader), s)) ||
        (err = cudaMemcpyAsync(t.b_coff.p, coff_host, (size_t)(nc + 1) * 8, cudaMemcpyHostToDevice, s)))
        return cuda_status(ctx, err, "batch upload");
    {
        PhaseTimer pt_(ctx, PH_BOUNDS);
        k_cloud_bounds<T, D><<<nc, kThreads, 0, s>>>(coords, t.b_coff.as<int64_t>(), t.b_cbounds.as<double>());
        ctx.kernel_launches += 1;
    }
    std::vector<double> cb((size_t)nc * 8);
    if ((err = cudaMemcpyAsync(cb.data(), t.b_cbounds.p, cb.size() * 8, cudaMemcpyDeviceToHost, s)) ||
        (err = wait_stream(s)))
        return cuda_status(ctx, err, "cloud bounds");
    // Per cloud, in T, exactly what a TNS of that cloud alone computes
    // (src/cpu/bin_cpu.jl:22,35,60; src/cpu/edges_cpu.jl:184-185).
    std::vector<double> cp((size_t)nc * kCloudParams, 0.0);
    int64_t cmax_all = 0;
    for (int c = 0; c < nc; ++c) {
        if (coff_host[c + 1] == coff_host[c]) continue;
        const double* b = cb.data() + (size_t)c * 8;
        if (b[6] != 0.0)
            return set_error(ctx, ERR_INEXACT, "InexactError: floor(Int32, NaN/Inf) in bin_point (non-finite coordinate)");
        const T r = (T)radii_host[c];
        const T inv_cs = T(1) / r;
        double* p = cp.data() + (size_t)c * kCloudParams;
        for (int d = 0; d < D; ++d) {
            const T o = (T)b[d] - T(1e-6);
            p[d] = (double)o;
            const T f = std::floor(((T)b[3 + d] - o) * inv_cs);
            if (!(f >= T(-2147483648.0) && f < T(2147483648.0)))
                return set_error(ctx, ERR_INEXACT, "InexactError: floor(Int32, (p - origin) / radius) exceeds Int32");
            int64_t ci = (int64_t)f;
            const int64_t cm = (1LL << Dims<D>::bits) - 1;
            ci = ci < 0 ? 0 : (ci > cm ? cm : ci);
            cmax_all = std::max(cmax_all, ci);
            p[6 + d] = b[d];
            p[9 + d] = b[3 + d];
        }
        p[3] = (double)inv_cs;
        p[4] = (double)(r * r);
        p[5] = (double)(T(1) / r);
    }
    if ((err = cudaMemcpyAsync(t.b_cparam.p, cp.data(), cp.size() * 8, cudaMemcpyHostToDevice, s)))
        return cuda_status(ctx, err, "cloud parameters");
    int nbits_axis = 0;
    while (nbits_axis < 63 && (cmax_all >> nbits_axis) != 0) ++nbits_axis;
    int cbits = 0;
    while (cbits < 31 && ((int64_t)(nc - 1) >> cbits) != 0) ++cbits;
    t.kbits = D * nbits_axis;
    t.key_bits = t.kbits + cbits;
    if (t.key_bits > 64) return set_error(ctx, ERR_ARGUMENT, "batch: cloud id and Morton code exceed 64 key bits");
    t.key_bytes = t.key_bits <= 32 ? 4 : 8;
    t.sort_passes = (t.key_bits + 7) / 8;
    if (t.key_bytes == 4) return run_pipeline<T, D, uint32_t>(ctx, t, coords, n, T(0));
    return run_pipeline<T, D, uint64_t>(ctx, t, coords, n, T(0));
}

}  // namespace

int build_tree_batch(Ctx& ctx, Tree& t, const void* coords, int64_t n, const int64_t* coff_host,
                     const double* radii_host, int32_t n_clouds) {
    t.sorted_buf = -1;
    t.built = false;
    t.view_valid = false;
    t.n = n;
    t.radius = 0.0;
    t.keep_morton = false;
    ++t.generation;
    t.n_clouds = n_clouds;
    if (n == 0) {
        t.n_nodes = 0;
        t.n_groups = 0;
        t.built = true;
        return OK;
    }
    int st;
    if (t.dtype == 0)
        st = t.ndims == 3 ? build_batch_typed<float, 3>(ctx, t, (const float*)coords, n, coff_host, radii_host, n_clouds)
                          : build_batch_typed<float, 2>(ctx, t, (const float*)coords, n, coff_host, radii_host, n_clouds);
    else
        st = t.ndims == 3 ? build_batch_typed<double, 3>(ctx, t, (const double*)coords, n, coff_host, radii_host, n_clouds)
                          : build_batch_typed<double, 2>(ctx, t, (const double*)coords, n, coff_host, radii_host, n_clouds);
    if (st == OK) t.built = true;
    return st;
}

int batch_edge_offsets(Ctx& ctx, Tree& t, int64_t* out_host) {
    const int nc = t.n_clouds;
    cudaError_t err;
    if (ctx.plan_query != &t || ctx.plan_target != &t || ctx.plan_qgen != t.generation)
        return set_error(ctx, ERR_STATE, "batch edge offsets: no matching oct_edges_count for this tree");
    if (t.n == 0 || ctx.plan_edges <= 0) {
        for (int c = 0; c <= nc; ++c) out_host[c] = 0;
        return OK;
    }
    k_gather_edge_offsets<<<div_up(nc + 1, 128), 128, 0, ctx.stream>>>(ctx.offsets.as<int64_t>(), t.b_coff.as<int64_t>(),
                                                                        nc, t.b_eoff.as<int64_t>());
    ctx.kernel_launches += 1;
    if ((err = cudaMemcpyAsync(out_host, t.b_eoff.p, (size_t)(nc + 1) * 8, cudaMemcpyDeviceToHost, ctx.stream)) ||
        (err = wait_stream(ctx.stream)))
        return cuda_status(ctx, err, "batch edge offsets");
    return OK;
}

int build_tree(Ctx& ctx, Tree& t, const void* coords, int64_t n, double radius) {
    t.built = false;
    t.view_valid = false;
    t.n = n;
    t.radius = radius;
    t.n_clouds = 0;
    ++t.generation;
    if (n == 0) {
        t.n_nodes = 0;
        t.sorted_buf = -1;
        t.built = true;
        return OK;
    }
    int st;
    if (t.dtype == 0)
        st = t.ndims == 3 ? build_typed<float, 3>(ctx, t, (const float*)coords, n, radius)
                          : build_typed<float, 2>(ctx, t, (const float*)coords, n, radius);
    else
        st = t.ndims == 3 ? build_typed<double, 3>(ctx, t, (const double*)coords, n, radius)
                          : build_typed<double, 2>(ctx, t, (const double*)coords, n, radius);
    if (st == OK) t.built = true;
    return st;
}

int ensure_iperm(Ctx& ctx, const Tree& t) {
    if (t.iperm_valid || t.n == 0) return OK;
    if (!t.perm_dev) return set_error(ctx, ERR_STATE, "inverse permutation: the tree has no sorted order");
    OctHeader* hdr = t.hdr.as<OctHeader>();
    k_inverse_perm<<<(unsigned)div_up(t.n, kSortThreads), kSortThreads, 0, ctx.stream>>>(
        t.perm_dev, t.n, t.iperm.as<int32_t>(), &hdr->status);
    ctx.kernel_launches += 1;
    const cudaError_t err = cudaGetLastError();
    if (err) return cuda_status(ctx, err, "inverse permutation launch");
    t.iperm_valid = true;
    return OK;
}

namespace {
template <class T, int D>
int view_typed(Ctx& ctx, Tree& t) {
    cudaError_t err;
    const int64_t nn = std::max<int64_t>(t.n_nodes, 1), n = std::max<int64_t>(t.n, 1);
    constexpr int NCH = Dims<D>::nch;
    if ((err = ensure(t.v_first, nn * 4)) || (err = ensure(t.v_last, nn * 4)) || (err = ensure(t.v_children, nn * 4 * NCH)) ||
        (err = ensure(t.v_bmin, nn * sizeof(T) * D)) || (err = ensure(t.v_bmax, nn * sizeof(T) * D)) ||
        (err = ensure(t.v_perm, n * 4)))
        return cuda_status(ctx, err, "allocating views");
    if (t.n_nodes > 0)
        k_view_nodes<T, D><<<div_up(t.n_nodes, kThreads), kThreads, 0, ctx.stream>>>(
            t.tnode.as<TNode<T, D>>(), t.nrange.as<int2>(), t.n_nodes, t.v_first.as<int32_t>(), t.v_last.as<int32_t>(),
            t.v_children.as<int32_t>(), t.v_bmin.as<T>(), t.v_bmax.as<T>());
    if (t.n > 0)
        k_view_perm<T, D><<<div_up(t.n, kThreads), kThreads, 0, ctx.stream>>>(t.spts.as<SPt<T, D>>(), t.n,
                                                                               t.v_perm.as<int32_t>());
    if (t.keep_morton && t.n > 0 && !t.n_clouds) {
        if ((err = ensure(t.morton, (size_t)t.n * 8))) return cuda_status(ctx, err, "allocating morton codes");
        if (t.key_bytes == 4)
            k_view_morton<T, D, uint32_t><<<div_up(t.n, kThreads), kThreads, 0, ctx.stream>>>(
                t.spts.as<SPt<T, D>>(), (const uint32_t*)t.skeys_dev, t.n, t.morton.as<uint64_t>());
        else
            k_view_morton<T, D, uint64_t><<<div_up(t.n, kThreads), kThreads, 0, ctx.stream>>>(
                t.spts.as<SPt<T, D>>(), (const uint64_t*)t.skeys_dev, t.n, t.morton.as<uint64_t>());
    }
    if ((err = cudaStreamSynchronize(ctx.stream))) return cuda_status(ctx, err, "materializing views");
    t.view_valid = true;
    return OK;
}
}  // namespace

int materialize_view(Ctx& ctx, Tree& t) {
    if (t.view_valid) return OK;
    if (t.dtype == 0) return t.ndims == 3 ? view_typed<float, 3>(ctx, t) : view_typed<float, 2>(ctx, t);
    return t.ndims == 3 ? view_typed<double, 3>(ctx, t) : view_typed<double, 2>(ctx, t);
}

}  // namespace oct
