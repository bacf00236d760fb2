// Key sort of the build that carries the points along.
//
// The stable LSD radix sort of the Morton keys (ties keep ascending original
// index, src/sort.jl:15-24) with each point's record SPt {coordinates,
// original index} as the sorted value, so that the sorted points come out of
// the last pass instead of a gather at random original indices afterwards.
// The Morton encode (src/cpu/bin_cpu.jl:52-95) is fused in too:
//
//   k_point_counts  reads the coordinates once, encodes each key and counts
//                   every pass's 8-bit digits;
//   k_point_pass    one launch per digit: each block takes the next tile of
//                   2048 points (tile ids in the order blocks start), ranks
//                   its keys by digit (warp match, per-warp counters), adds the
//                   counts of the tiles before it by decoupled look-back
//                   (bounded waits), stages the tile in shared memory in digit
//                   order and writes each digit's run contiguously.  The first
//                   pass encodes from the coordinates; the last writes the
//                   sorted keys, the sorted points and the permutation;
//   k_inverse_perm  the inverse permutation (when asked for; the build
//                   leaves it to the first caller that needs it).
//
// Every wait is bounded (spin_limit polling rounds); one that runs out sets
// DF_TIMEOUT, and every store still stays inside its array.
#pragma once

#include <algorithm>

#include <cuda/atomic>

#include "common.cuh"
#include "sort.cuh"

namespace oct {

// Per-point encode parameters: one origin and cell size, or per cloud.
template <class T>
struct EncodeParams {
    T o[3];
    T inv_cs;
    Batch bt;
};

// Morton key of one point's cell (src/cpu/bin_cpu.jl:12-31,
// src/morton.jl:13-60): floor((x - origin) * inv_cs) per axis, clamped to the
// key's bits per axis, bit-interleaved with x in the lowest bit; in a batch,
// (cloud << kbits) | morton with the cloud's own origin and cell size.
template <class T, int D>
__device__ __forceinline__ uint64_t point_key(const T* __restrict__ x, int64_t i, const EncodeParams<T>& ep) {
    constexpr int64_t cmax = (1LL << Dims<D>::bits) - 1;
    T o[3] = {ep.o[0], ep.o[1], ep.o[2]};
    T inv_cs = ep.inv_cs;
    int cloud = 0;
    if (ep.bt.n_clouds) {
        cloud = cloud_of_position(ep.bt, i);
        const double* cp = ep.bt.cparam + (size_t)cloud * kCloudParams;
        o[0] = (T)cp[0];
        o[1] = (T)cp[1];
        o[2] = (T)cp[2];
        inv_cs = (T)cp[3];
    }
    uint64_t c[3] = {0, 0, 0};
#pragma unroll
    for (int d = 0; d < D; ++d) {
        const T v = mul_rn(sub_rn(x[d], o[d]), inv_cs);
        int64_t ci = (int64_t)floor(v);
        ci = ci < 0 ? 0 : (ci > cmax ? cmax : ci);
        c[d] = (uint64_t)ci;
    }
    const uint64_t m = (D == 3) ? ((split_by_3(c[2]) << 2) | (split_by_3(c[1]) << 1) | split_by_3(c[0]))
                                : ((split_by_2(c[1]) << 1) | split_by_2(c[0]));
    return ep.bt.n_clouds ? (((uint64_t)cloud << ep.bt.kbits) | m) : m;
}

template <class T, int D>
__device__ __forceinline__ SPt<T, D> load_point(const T* __restrict__ coords, int64_t i) {
    SPt<T, D> p;
#pragma unroll
    for (int d = 0; d < D; ++d) p.x[d] = coords[(int64_t)D * i + d];
    p.idx = (int32_t)i;
    return p;
}

// Every pass's digit counts in one read of the coordinates.
template <class T, int D, class K>
__global__ void __launch_bounds__(kSortThreads) k_point_counts(const T* __restrict__ coords, int64_t n, int passes,
                                                               EncodeParams<T> ep, uint32_t* __restrict__ counts) {
    pdl_wait();
    pdl_trigger();
    __shared__ uint32_t c[kOnesweepMaxPasses][256];
    for (int p = 0; p < passes; ++p) c[p][threadIdx.x] = 0;
    __syncthreads();
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        T x[D];
#pragma unroll
        for (int d = 0; d < D; ++d) x[d] = coords[(int64_t)D * i + d];
        const K k = (K)point_key<T, D>(x, i, ep);
        for (int p = 0; p < passes; ++p) atomicAdd(&c[p][(unsigned)(k >> (8 * p)) & 255u], 1u);
    }
    __syncthreads();
    for (int p = 0; p < passes; ++p)
        if (c[p][threadIdx.x]) atomicAdd(&counts[(size_t)p * 257 + threadIdx.x], c[p][threadIdx.x]);
}

// Shared memory of one k_point_pass block.
template <class T, int D, class K>
struct PointPassSmem {
    int32_t wc[kSortThreads / 32][256];
    int32_t tstart[256];
    int64_t gstart[256];
    int32_t scan_sm[kSortThreads / 32 + 1];
    int tile;
    K key[kSortTile];
    SPt<T, D> pt[kSortTile];
};

template <class T, int D, class K>
constexpr size_t point_pass_smem() { return sizeof(PointPassSmem<T, D, K>); }

// One pass on digit `pass`.  FIRST: the points come from `coords` (key
// encoded here, value = the point and its index); otherwise from (kin, pin).
// LAST: writes kout, pout (the sorted points) and perm[dst] = original index.
template <class T, int D, class K, bool FIRST, bool LAST>
__global__ void __launch_bounds__(kSortThreads) k_point_pass(
    const T* __restrict__ coords, EncodeParams<T> ep, const K* __restrict__ kin, const SPt<T, D>* __restrict__ pin,
    K* __restrict__ kout, SPt<T, D>* __restrict__ pout, int32_t* __restrict__ perm, int32_t* __restrict__ iperm,
    int64_t n, int pass, int ntiles, uint32_t* __restrict__ scratch, int* __restrict__ status, int64_t spin_limit,
    int withhold_tile) {
    pdl_wait();
    pdl_trigger();
    extern __shared__ __align__(16) unsigned char pp_smem[];
    PointPassSmem<T, D, K>& sm = *reinterpret_cast<PointPassSmem<T, D, K>*>(pp_smem);
    const int shift = 8 * pass;
    uint32_t* counts = scratch + (size_t)pass * 257;
    uint32_t* look = scratch + (size_t)kOnesweepMaxPasses * 257 + (size_t)pass * ntiles * 256;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (threadIdx.x == 0) sm.tile = (int)atomicAdd(&counts[256], 1u);
#pragma unroll
    for (int j = 0; j < kSortThreads / 32; ++j) sm.wc[j][threadIdx.x] = 0;
    __syncthreads();
    const int t = sm.tile;
    const int64_t wbase = (int64_t)t * kSortTile + (int64_t)w * (32 * kSortItems);
    K key[kSortItems];
    int32_t rk[kSortItems];
    int dg[kSortItems];
#pragma unroll
    for (int it = 0; it < kSortItems; ++it) {
        const int64_t i = wbase + it * 32 + lane;
        const bool valid = i < n;
        if (FIRST) {
            T x[D];
#pragma unroll
            for (int d = 0; d < D; ++d) x[d] = valid ? coords[(int64_t)D * i + d] : T(0);
            key[it] = valid ? (K)point_key<T, D>(x, i, ep) : K(0);
        } else {
            key[it] = valid ? kin[i] : K(0);
        }
        const int d = valid ? (int)((unsigned)(key[it] >> shift) & 255u) : 256;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int leader = __ffs(peers) - 1;
        const int before = __popc(peers & lanemask_lt());
        const int c0 = valid ? sm.wc[w][d] : 0;
        __syncwarp();
        if (valid && lane == leader) sm.wc[w][d] = c0 + __popc(peers);
        __syncwarp();
        rk[it] = c0 + before;
        dg[it] = d;
    }
    __syncthreads();
    // thread = digit: warp offsets within the tile's run, the tile's count
    int32_t run = 0;
#pragma unroll
    for (int j = 0; j < kSortThreads / 32; ++j) {
        const int32_t c = sm.wc[j][threadIdx.x];
        sm.wc[j][threadIdx.x] = run;
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
        // Four predecessors per round trip, added in order up to the first
        // inclusive prefix; a word not yet published stops the round.
        int j = t - 1;
        int64_t spins = 0;
        while (true) {
            uint32_t v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u)
                v[u] = j - u >= 0 ? cuda::atomic_ref<uint32_t, cuda::thread_scope_device>(look[(size_t)(j - u) * 256 + d])
                                        .load(cuda::memory_order_relaxed)
                                  : kLookPrefix;
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
    sm.tstart[d] = block_exclusive_scan<int32_t>(run, sm.scan_sm, &tile_total);
    const int32_t base = block_exclusive_scan<int32_t>((int32_t)counts[d], sm.scan_sm, &all);
    sm.gstart[d] = (int64_t)base + excl;
    __syncthreads();
    // Stage keys and points in digit order.  The points are loaded here (the
    // first pass builds them from the coordinates).
#pragma unroll
    for (int it = 0; it < kSortItems; ++it) {
        if (dg[it] < 256) {
            const int64_t i = wbase + it * 32 + lane;
            const int lp = sm.tstart[dg[it]] + sm.wc[w][dg[it]] + rk[it];
            sm.key[lp] = key[it];
            sm.pt[lp] = FIRST ? load_point<T, D>(coords, i) : pin[i];
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < tile_total; i += kSortThreads) {
        const K k = sm.key[i];
        const int dd = (int)((unsigned)(k >> shift) & 255u);
        const int64_t dst = sm.gstart[dd] + (i - sm.tstart[dd]);
        if (dst >= 0 && dst < n) {  // always, unless a wait ran out and left a prefix short
            const SPt<T, D> p = sm.pt[i];
            kout[dst] = k;
            pout[dst] = p;
            if (LAST) perm[dst] = p.idx;
        } else {
            timed_out = true;
        }
    }
    if (timed_out) atomicOr(status, (int)DF_TIMEOUT);
}

// iperm[perm[k]] = k: after the last pass, in a pass of its own, so that the
// random 4-byte stores land in a 4n-byte target that L2 holds while nothing
// else streams.  An entry outside [0, n) can only be stale after a look-back
// wait ran out (DF_TIMEOUT is then set already) and is skipped.
__global__ void __launch_bounds__(kSortThreads) k_inverse_perm(const int32_t* __restrict__ perm, int64_t n,
                                                               int32_t* __restrict__ iperm, int* __restrict__ status) {
    pdl_wait();
    pdl_trigger();
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int32_t j = perm[k];
    if ((uint64_t)(uint32_t)j < (uint64_t)n)
        iperm[j] = (int32_t)k;
    else
        atomicOr(status, (int)DF_TIMEOUT);
}

template <class T, int D, class K, bool FIRST, bool LAST>
cudaError_t launch_point_pass(const T* coords, const EncodeParams<T>& ep, const K* kin, const SPt<T, D>* pin, K* kout,
                              SPt<T, D>* pout, int32_t* perm, int32_t* iperm, int64_t n, int pass, int ntiles,
                              uint32_t* scratch, int* status, int64_t spin_limit, int withhold, cudaStream_t s) {
    constexpr size_t smem = point_pass_smem<T, D, K>();
    auto kern = k_point_pass<T, D, K, FIRST, LAST>;
    static bool attr_set = false;  // per instantiation
    if (!attr_set) {
        const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    launch_pdl(kern, ntiles, kSortThreads, smem, s, coords, ep, kin, pin, kout, pout, perm, iperm, n, pass, ntiles,
        scratch, status, spin_limit, withhold);
    return cudaGetLastError();
}

// Sorts the n points of `coords` by Morton key (passes 8-bit digits, 1..8):
// on return keys_out holds the sorted keys, spts the sorted points, perm the
// original index of each sorted position and iperm its inverse.  kt and ptmp
// are scratch of n keys / points (used when passes > 1); `scratch` holds
// onesweep_words(n, kOnesweepMaxPasses) words.  Launches 1 + passes kernels,
// plus k_inverse_perm when iperm is not null.
template <class T, int D, class K>
cudaError_t point_sort(const T* coords, const EncodeParams<T>& ep, int64_t n, int passes, K* keys_out, K* kt,
                       SPt<T, D>* spts, SPt<T, D>* ptmp, int32_t* perm, int32_t* iperm, uint32_t* scratch, int* status,
                       int sms, int64_t spin_limit, int withhold, cudaStream_t s, int64_t* launches) {
    const int ntiles = sort_tiles(n);
    cudaError_t e = cudaMemsetAsync(scratch, 0, onesweep_words(n, passes) * 4, s);
    if (e != cudaSuccess) return e;
    const int hblocks = (int)std::min<int64_t>(ntiles, (int64_t)4 * std::max(sms, 1));
    launch_pdl(k_point_counts<T, D, K>, hblocks, kSortThreads, 0, s, coords, n, passes, ep, scratch);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    *launches += 1 + passes;
    // Pass p writes the final buffers when passes - 1 - p is even, so the
    // last pass lands in (keys_out, spts).
    auto kb = [&](int p) { return ((passes - 1 - p) & 1) == 0 ? keys_out : kt; };
    auto pb = [&](int p) { return ((passes - 1 - p) & 1) == 0 ? spts : ptmp; };
    if (passes == 1) {
        if ((e = launch_point_pass<T, D, K, true, true>(coords, ep, nullptr, nullptr, keys_out, spts, perm, iperm, n, 0,
                                                        ntiles, scratch, status, spin_limit, withhold, s)))
            return e;
    } else {
        if ((e = launch_point_pass<T, D, K, true, false>(coords, ep, nullptr, nullptr, kb(0), pb(0), nullptr, nullptr,
                                                         n, 0, ntiles, scratch, status, spin_limit, withhold, s)))
            return e;
        for (int p = 1; p < passes - 1; ++p)
            if ((e = launch_point_pass<T, D, K, false, false>(coords, ep, kb(p - 1), pb(p - 1), kb(p), pb(p), nullptr,
                                                              nullptr, n, p, ntiles, scratch, status, spin_limit,
                                                              withhold, s)))
                return e;
        if ((e = launch_point_pass<T, D, K, false, true>(coords, ep, kb(passes - 2), pb(passes - 2), keys_out, spts,
                                                         perm, iperm, n, passes - 1, ntiles, scratch, status,
                                                         spin_limit, withhold, s)))
            return e;
    }
    if (iperm) {
        launch_pdl(k_inverse_perm, (unsigned)((n + kSortThreads - 1) / kSortThreads), kSortThreads, 0, s, perm, n,
            iperm, status);
        *launches += 1;
    }
    return cudaGetLastError();
}

}  // namespace oct
