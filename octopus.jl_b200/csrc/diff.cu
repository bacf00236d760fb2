// Adjoint of build_edges_diff (ext/OctopusChainRulesCoreExt.jl:137-192,
// ext/OctopusCUDAChainRulesCoreExt.jl:56-99), without floating-point atomics.
//
// Per edge k = (receiver i <- sender j) the cotangent contributes
//   c_k = d_disp[:,k] / r + rel_disp[:,k] * (d_dist[k] / (rel_dist[k] * r))
// (the second term only when rel_dist[k] > 1e-8), added to x_i and
// subtracted from x_j.  Edges grouped by receiver (the order build_edges
// writes) make the receiver sum a segmented reduction in edge order; the
// sender sum either reads each edge's mirror (self pairs) or the edges
// re-ordered by (sender, edge index) with the stable radix sort.  A COO that
// is not grouped is re-ordered by receiver the same way.  Every point sums
// its terms in a fixed order in double precision, so the result is
// bit-reproducible from run to run.

#include <algorithm>

#include "internal.h"
#include "sort.cuh"

namespace oct {

template <class T, int D>
__device__ __forceinline__ void edge_term(int64_t k, const T* __restrict__ rel_disp, const T* __restrict__ rel_dist,
                                          const T* __restrict__ d_disp, const T* __restrict__ d_dist, T r,
                                          double* out) {
#pragma unroll
    for (int d = 0; d < D; ++d) out[d] = 0.0;
    if (d_disp) {
#pragma unroll
        for (int d = 0; d < D; ++d) out[d] += (double)div_rn(d_disp[(int64_t)D * k + d], r);
    }
    if (d_dist) {
        const T dn = rel_dist[k];
        if (dn > T(1e-8)) {
            const T inv = div_rn(d_dist[k], mul_rn(dn, r));
#pragma unroll
            for (int d = 0; d < D; ++d) out[d] += (double)mul_rn(rel_disp[(int64_t)D * k + d], inv);
        }
    }
}

// off[i] = first edge whose (1-based) key is >= i + 1, for i in [0, n].
__global__ void k_segment_starts(const int32_t* __restrict__ keys1, int64_t m, int64_t n, int64_t* __restrict__ off) {
    pdl_wait();
    pdl_trigger();
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i > n) return;
    int64_t a = 0, b = m;
    while (a < b) {
        const int64_t mid = (a + b) >> 1;
        if ((int64_t)keys1[mid] >= i + 1) b = mid; else a = mid + 1;
    }
    off[i] = a;
}

__global__ void k_sender_keys(const int32_t* __restrict__ snd, int64_t m, uint32_t* __restrict__ keys) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < m) keys[k] = (uint32_t)(snd[k] - 1);
}

// off[j] = first sorted position whose 0-based sender key is >= j.
__global__ void k_sorted_starts(const uint32_t* __restrict__ skeys, int64_t m, int64_t n, int64_t* __restrict__ off) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j > n) return;
    int64_t a = 0, b = m;
    while (a < b) {
        const int64_t mid = (a + b) >> 1;
        if ((int64_t)skeys[mid] >= j) b = mid; else a = mid + 1;
    }
    off[j] = a;
}

// grad[i] = sum of the terms of i's receiver edges minus those of its sender
// edges, each list in edge order (through `rsorted_edge` / `sorted_edge`
// when the edges are not grouped that way).
template <class T, int D>
__global__ void k_grad(int64_t n, const int64_t* __restrict__ roff, const int32_t* __restrict__ rsorted_edge,
                       const int64_t* __restrict__ soff, const int32_t* __restrict__ sorted_edge,
                       const T* __restrict__ rel_disp,
                       const T* __restrict__ rel_dist, const T* __restrict__ d_disp, const T* __restrict__ d_dist, T r,
                       T* __restrict__ grad) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double acc[D];
#pragma unroll
    for (int d = 0; d < D; ++d) acc[d] = 0.0;
    double c[D];
    for (int64_t t = roff[i]; t < roff[i + 1]; ++t) {
        const int64_t k = rsorted_edge ? rsorted_edge[t] : t;
        edge_term<T, D>(k, rel_disp, rel_dist, d_disp, d_dist, r, c);
#pragma unroll
        for (int d = 0; d < D; ++d) acc[d] += c[d];
    }
    for (int64_t m = soff[i]; m < soff[i + 1]; ++m) {
        const int64_t k = sorted_edge ? sorted_edge[m] : m;
        edge_term<T, D>(k, rel_disp, rel_dist, d_disp, d_dist, r, c);
#pragma unroll
        for (int d = 0; d < D; ++d) acc[d] -= c[d];
    }
#pragma unroll
    for (int d = 0; d < D; ++d) grad[(int64_t)D * i + d] = (T)acc[d];
}

// One side of a cross pair's gradient: grad[i] = sign * sum of the terms of
// the edges listed for point i, in list order (edge order, or the
// sender-sorted order when `sorted_edge` is given).
template <class T, int D>
__global__ void k_grad_part(int64_t n, const int64_t* __restrict__ off, const int32_t* __restrict__ sorted_edge,
                            const T* __restrict__ rel_disp, const T* __restrict__ rel_dist,
                            const T* __restrict__ d_disp, const T* __restrict__ d_dist, T r, double sign,
                            T* __restrict__ grad) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double acc[D];
#pragma unroll
    for (int d = 0; d < D; ++d) acc[d] = 0.0;
    double c[D];
    for (int64_t m = off[i]; m < off[i + 1]; ++m) {
        const int64_t k = sorted_edge ? sorted_edge[m] : m;
        edge_term<T, D>(k, rel_disp, rel_dist, d_disp, d_dist, r, c);
#pragma unroll
        for (int d = 0; d < D; ++d) acc[d] += c[d];
    }
#pragma unroll
    for (int d = 0; d < D; ++d) grad[(int64_t)D * i + d] = (T)(sign * acc[d]);
}

// Self-pair adjoint without a sort, in one pass.
//
// The neighbor relation of a self pair is symmetric, so the edge k =
// (i <- j) of point i's segment has a mirror t = (j <- i) in j's segment, and
// point i's gradient is
//   sum over its segment of term(k) - term(t),
// term(e) = d_disp[:, e] / r + rel_disp[:, e] * (d_dist[e] / (rel_dist[e] * r))
// being the rrule's per-edge cotangent term (the second part only when
// rel_dist[e] > 1e-8; features recomputed from `coords` with the forward's
// arithmetic when RECOMPUTE), added in double precision in segment order for
// every point.  Four values per term so that a term is one aligned record.
template <class T>
struct alignas(4 * sizeof(T)) Term4 {
    T v[4];
};

// term[e] for every edge (one coalesced pass over the edge arrays, 16 B per
// edge for float), pass 1 of the searching adjoint.
template <class T, int D, bool RECOMPUTE>
__global__ void k_edge_terms(int64_t m, int64_t n, const int32_t* __restrict__ snd, const int32_t* __restrict__ rcv,
                             const T* __restrict__ rel_disp, const T* __restrict__ rel_dist,
                             const T* __restrict__ coords, const T* __restrict__ d_disp,
                             const T* __restrict__ d_dist, T r, T inv_r, Term4<T>* __restrict__ term) {
    pdl_wait();
    pdl_trigger();
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    T rd[D], rn = T(0);
    Term4<T> o;
#pragma unroll
    for (int d = 0; d < 4; ++d) o.v[d] = T(0);
    if (RECOMPUTE) {
        const int32_t i = rcv[k] - 1, j = snd[k] - 1;
        if (i < 0 || i >= n || j < 0 || j >= n) {  // flagged by k_adjoint_twins
            term[k] = o;
            return;
        }
        T diff[D];
        const T d2 = dist2<T, D>(coords + (int64_t)D * j, coords + (int64_t)D * i, diff);
#pragma unroll
        for (int d = 0; d < D; ++d) rd[d] = mul_rn(-diff[d], inv_r);
        rn = mul_rn(sqrt_rn(d2), inv_r);
    } else {
#pragma unroll
        for (int d = 0; d < D; ++d) rd[d] = rel_disp[(int64_t)D * k + d];
        rn = rel_dist[k];
    }
    if (d_disp) {
#pragma unroll
        for (int d = 0; d < D; ++d) o.v[d] = div_rn(d_disp[(int64_t)D * k + d], r);
    }
    if (d_dist && rn > T(1e-8)) {
        const T a = div_rn(d_dist[k], mul_rn(rn, r));
#pragma unroll
        for (int d = 0; d < D; ++d) o.v[d] = add_rn(o.v[d], mul_rn(rd[d], a));
    }
    term[k] = o;
}

// seg[i] = {first, end} of point i's edges, from off[i], off[i + 1].
__global__ void k_seg_pairs(const int64_t* __restrict__ off, int64_t n, int2* __restrict__ seg) {
    pdl_wait();
    pdl_trigger();
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) seg[i] = make_int2((int32_t)off[i], (int32_t)off[i + 1]);
}

// Status bits of the adjoint's checks (word 1 of the status buffer).
constexpr int kAdjMissingTwin = 1;  // an edge without its mirror: not a self-pair COO
constexpr int kAdjUngrouped = 2;    // receivers not in ascending order
constexpr int kAdjBadIndex = 4;     // a sender or receiver outside 1..n
constexpr int kAdjBadOrder = 8;     // an entry of the processing order outside 1..n

// Checks a COO: receivers (1..n_rcv) ascending, senders in 1..n_snd.
__global__ void k_check_coo(const int32_t* __restrict__ snd, const int32_t* __restrict__ rcv, int64_t m,
                            int64_t n_snd, int64_t n_rcv, int* __restrict__ status) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int bad = 0;
    if (k < m) {
        const int32_t a = rcv[k], j = snd[k];
        if (a < 1 || a > n_rcv || j < 1 || j > n_snd) bad |= kAdjBadIndex;
        if (k + 1 < m && rcv[k + 1] < a) bad |= kAdjUngrouped;
    }
    if (bad) atomicOr(status, bad);
}

// Layout of the self-pair adjoint: one group of kTwinLanes lanes per point,
// the points taken in the order `order` (the tree's Morton permutation,
// 1-based; null for 0..n-1).  With a spatial order the segments the warps in
// flight read belong to nearby points, so they stay in L2.  Lane s of a group
// takes the edges s, s + 8, s + 16, ... of its point's segment and adds their
// contributions in that order in double precision; the group's eight partial
// sums are then added in a fixed pairwise tree (xor shuffles; every lane ends
// with the same bits).  The shape of the sum depends on the segment alone, so
// the gradient is bit-reproducible whatever the order and the launch shape.
// Each edge also checks the COO (receiver of its segment, sender range, a
// mirror present); a failed check sets a status bit and the caller takes the
// sorted path.
constexpr int kTwinWarps = 4;
constexpr int kTwinLanes = 8;                    // lanes per point
constexpr int kTwinGroups = 32 / kTwinLanes;     // points per warp

// The point of this lane's group and its segment [k0, k0 + ne); p = -1 when
// the group has no point.  Flags a bad order entry or an ungrouped COO.
__device__ __forceinline__ void twin_point(int64_t n, int64_t m, const int32_t* __restrict__ order,
                                           const int2* __restrict__ seg, int64_t sl, int& p, int& k0, int& ne,
                                           int& bad) {
    p = -1;
    k0 = 0;
    ne = 0;
    if (sl >= n) return;
    const int64_t pp = order ? (int64_t)order[sl] - 1 : sl;
    if (pp < 0 || pp >= n) {
        bad |= kAdjBadOrder;
        return;
    }
    p = (int)pp;
    const int2 sg = seg[p];
    k0 = sg.x;
    ne = sg.y - sg.x;
    if (ne < 0 || (p == 0 && k0 != 0) || (p == n - 1 && sg.y != m)) {
        bad |= kAdjUngrouped;
        ne = 0;
    }
}

// Sum of the group's lanes in a fixed pairwise tree, in every lane.
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
    for (int o = kTwinLanes / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Index of the entry equal to `key` in snd[lo, hi) (one thread's scan of a
// segment, in aligned blocks of four entries: one 16-byte load per block when
// `vec`, the sender array being 16-byte aligned), -1 when absent.  Entries
// outside [lo, hi) in the first and last block are masked off.  (The adjoint
// kernel keeps its own form of the scan: measured faster there, slower here.)
__device__ __forceinline__ int32_t find_mirror(const int32_t* __restrict__ snd, int32_t m, bool vec, int32_t lo,
                                               int32_t hi, int32_t key) {
    // unsigned: indices below 2^31, so qa + 4 cannot wrap
    const uint32_t ulo = (uint32_t)lo, uhi = (uint32_t)hi, um = (uint32_t)m;
    for (uint32_t qa = ulo & ~3u; qa < uhi; qa += 4) {
        int32_t c[4];
        if (vec && qa + 4 <= um) {
            const int4 v = *reinterpret_cast<const int4*>(snd + qa);
            c[0] = v.x;
            c[1] = v.y;
            c[2] = v.z;
            c[3] = v.w;
        } else {
#pragma unroll
            for (int u = 0; u < 4; ++u) c[u] = qa + u < um ? snd[qa + u] : 0;
        }
        unsigned mm = (c[0] == key ? 1u : 0u) | (c[1] == key ? 2u : 0u) | (c[2] == key ? 4u : 0u) |
                      (c[3] == key ? 8u : 0u);
        if (qa < ulo) mm &= 0xfu << (ulo - qa);
        if (qa + 4 > uhi) mm &= 0xfu >> (qa + 4 - uhi);
        if (mm) return (int32_t)(qa + __ffs(mm) - 1);
    }
    return -1;
}

// Pass 2 of the searching adjoint: each edge's mirror found by scanning its
// sender's segment, term(k) - term(mirror) summed per point.  The term
// records stream in one coalesced pass (k_edge_terms) before this pass reads
// them.  `vec`: the sender array is 16-byte aligned, so the scan reads four
// entries per load.
template <class T>
__global__ void __launch_bounds__(kTwinWarps * 32) k_adjoint_twins(
    int64_t n, int64_t m, const int32_t* __restrict__ order, const int2* __restrict__ seg,
    const int32_t* __restrict__ snd, const int32_t* __restrict__ rcv, const Term4<T>* __restrict__ term, int ndims,
    bool vec, T* __restrict__ grad, int* __restrict__ status) {
    pdl_wait();
    pdl_trigger();
    const int lane = threadIdx.x & 31, sub = lane & (kTwinLanes - 1);
    const int64_t w0 = ((int64_t)blockIdx.x * kTwinWarps + (threadIdx.x >> 5)) * kTwinGroups;
    if (w0 >= n) return;  // warp-uniform
    int bad = 0, p, k0, ne;
    twin_point(n, m, order, seg, w0 + lane / kTwinLanes, p, k0, ne, bad);
    double acc[3] = {0.0, 0.0, 0.0};
    for (int e = sub; e < ne; e += kTwinLanes) {
        const int32_t k = k0 + e;
        const int32_t i1 = p + 1;
        const int32_t j1 = snd[k];
        if (rcv[k] != i1) bad |= kAdjUngrouped;
        const Term4<T> tk = term[k];
        if (j1 < 1 || j1 > n) {
            bad |= kAdjBadIndex;
            continue;
        }
        const int2 sj = seg[j1 - 1];
        int32_t tw = -1;
        if (vec) {
            // aligned blocks of four entries; the last block of the array is
            // read entry by entry
            for (int32_t qa = sj.x & ~3; qa < sj.y && tw < 0; qa += 4) {
                int32_t c[4];
                if ((int64_t)qa + 3 < m) {
                    const int4 v = *reinterpret_cast<const int4*>(snd + qa);
                    c[0] = v.x;
                    c[1] = v.y;
                    c[2] = v.z;
                    c[3] = v.w;
                } else {
#pragma unroll
                    for (int u = 0; u < 4; ++u) c[u] = (int64_t)qa + u < m ? snd[qa + u] : 0;
                }
#pragma unroll
                for (int u = 3; u >= 0; --u)
                    if (c[u] == i1 && (int64_t)qa + u >= sj.x && (int64_t)qa + u < sj.y) tw = qa + u;
            }
        } else {
            tw = find_mirror(snd, (int32_t)m, false, sj.x, sj.y, i1);
        }
        if (tw < 0) {
            bad |= kAdjMissingTwin;
            continue;
        }
        const Term4<T> tt = term[tw];
#pragma unroll
        for (int d = 0; d < 3; ++d) acc[d] += (double)tk.v[d] - (double)tt.v[d];
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) acc[d] = group_sum(acc[d]);
    if (p >= 0 && sub == 0) {
#pragma unroll
        for (int d = 0; d < 3; ++d)
            if (d < ndims) grad[(int64_t)ndims * p + d] = (T)acc[d];
    }
    if (bad) atomicOr(status, bad);
}

// One-pass self-pair adjoint from given mirror indices (written by the
// differentiable fill, oct_edges_fill_diff): the mirror t of edge k is read,
// not searched.  The mirror's features are exactly the edge's own with
// rel_displacement negated (x_j - x_i is the exact negation of x_i - x_j, and
// the squares and the distance are the same), so term(t) is formed from the
// mirror's cotangents and the edge's own features, bit for bit what the
// mirror's stored features give, and no per-edge term buffer is written.  A
// mirror index outside 0..m-1 sets kAdjMissingTwin.
template <class T, int D, bool RECOMPUTE>
__device__ __forceinline__ Term4<T> mirror_term(const T* rd, T rn, const T* __restrict__ d_disp,
                                                 const T* __restrict__ d_dist, int64_t e, T r, T sign) {
    Term4<T> o;
#pragma unroll
    for (int d = 0; d < 4; ++d) o.v[d] = T(0);
    if (d_disp) {
#pragma unroll
        for (int d = 0; d < D; ++d) o.v[d] = div_rn(d_disp[(int64_t)D * e + d], r);
    }
    if (d_dist && rn > T(1e-8)) {
        const T a = div_rn(d_dist[e], mul_rn(rn, r));
#pragma unroll
        for (int d = 0; d < D; ++d) o.v[d] = add_rn(o.v[d], mul_rn(sign * rd[d], a));
    }
    return o;
}

template <class T, int D, bool RECOMPUTE>
__global__ void __launch_bounds__(kTwinWarps * 32) k_adjoint_mirror(
    int64_t n, int64_t m, const int32_t* __restrict__ order, const int2* __restrict__ seg,
    const int32_t* __restrict__ snd, const int32_t* __restrict__ rcv, const int32_t* __restrict__ mirror,
    const T* __restrict__ rel_disp, const T* __restrict__ rel_dist, const T* __restrict__ coords,
    const T* __restrict__ d_disp, const T* __restrict__ d_dist, T r, T inv_r, T* __restrict__ grad,
    int* __restrict__ status) {
    pdl_wait();
    pdl_trigger();
    const int lane = threadIdx.x & 31, sub = lane & (kTwinLanes - 1);
    const int64_t w0 = ((int64_t)blockIdx.x * kTwinWarps + (threadIdx.x >> 5)) * kTwinGroups;
    if (w0 >= n) return;  // warp-uniform
    int bad = 0, p, k0, ne;
    twin_point(n, m, order, seg, w0 + lane / kTwinLanes, p, k0, ne, bad);
    double acc[3] = {0.0, 0.0, 0.0};
    for (int e = sub; e < ne; e += kTwinLanes) {
        const int32_t k = k0 + e;
        if (rcv[k] != p + 1) bad |= kAdjUngrouped;
        T rd[D], rn = T(0);
        if (RECOMPUTE) {
            const int32_t j = snd[k] - 1;
            if (j < 0 || j >= n) {
                bad |= kAdjBadIndex;
                continue;
            }
            T diff[D];
            const T d2 = dist2<T, D>(coords + (int64_t)D * j, coords + (int64_t)D * p, diff);
#pragma unroll
            for (int d = 0; d < D; ++d) rd[d] = mul_rn(-diff[d], inv_r);
            rn = mul_rn(sqrt_rn(d2), inv_r);
        } else {
#pragma unroll
            for (int d = 0; d < D; ++d) rd[d] = rel_disp[(int64_t)D * k + d];
            rn = rel_dist[k];
        }
        const int32_t t = mirror[k];
        if (!(t >= 0 && (int64_t)t < m)) {
            bad |= kAdjMissingTwin;
            continue;
        }
        const Term4<T> tk = mirror_term<T, D, RECOMPUTE>(rd, rn, d_disp, d_dist, k, r, T(1));
        const Term4<T> tt = mirror_term<T, D, RECOMPUTE>(rd, rn, d_disp, d_dist, t, r, T(-1));
#pragma unroll
        for (int d = 0; d < 3; ++d) acc[d] += (double)tk.v[d] - (double)tt.v[d];
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) acc[d] = group_sum(acc[d]);
    if (p >= 0 && sub == 0) {
#pragma unroll
        for (int d = 0; d < D; ++d) grad[(int64_t)D * p + d] = (T)acc[d];
    }
    if (bad) atomicOr(status, bad);
}

// Mirror index of every edge of a self-pair COO grouped by receiver, by
// scanning the sender's segment (off: int64 segment starts); -1 when absent.
__global__ void k_mirror_scan(const int32_t* __restrict__ snd, const int32_t* __restrict__ rcv, int64_t m, int64_t n,
                              const int64_t* __restrict__ off, int32_t* __restrict__ mirror) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    const int32_t i1 = rcv[k], j = snd[k] - 1;
    const bool vec = ((uintptr_t)snd & 15) == 0;
    mirror[k] = (j >= 0 && j < n) ? find_mirror(snd, (int32_t)m, vec, (int32_t)off[j], (int32_t)off[j + 1], i1) : -1;
}

namespace {

// Word 1 of the status buffer (word 0 belongs to the edge fill guard).
int* adjoint_status(Ctx& ctx) { return ctx.dstatus.as<int>() + 1; }

int read_status(Ctx& ctx, int* flags) {
    cudaError_t err;
    if ((err = cudaMemcpyAsync(flags, adjoint_status(ctx), 4, cudaMemcpyDeviceToHost, ctx.stream)) ||
        (err = wait_stream(ctx.stream)))
        return cuda_status(ctx, err, "adjoint status");
    return OK;
}

// Status bits of a COO (k_check_coo) for senders in 1..n_snd and receivers
// in 1..n_rcv.
int coo_flags(Ctx& ctx, const int32_t* snd, const int32_t* rcv, int64_t m, int64_t n_snd, int64_t n_rcv, int* flags) {
    cudaError_t err;
    if ((err = ensure(ctx.dstatus, 8)) || (err = cudaMemsetAsync(adjoint_status(ctx), 0, 4, ctx.stream)))
        return cuda_status(ctx, err, "adjoint status");
    k_check_coo<<<div_up(m, 256), 256, 0, ctx.stream>>>(snd, rcv, m, n_snd, n_rcv, adjoint_status(ctx));
    ctx.kernel_launches += 1;
    return read_status(ctx, flags);
}

// Stable order of the edges by a 1-based index (values in 1..nmax): the
// edges with index i + 1 are list[off[i] .. off[i + 1]), in edge order.
// The list is left in the sort's value buffers, or copied to `keep` when
// given (so that a second sort can reuse the buffers); *list is null when
// nmax is 1 (the edge order is the list).
int order_by_index(Ctx& ctx, const int32_t* idx, int64_t m, int64_t nmax, DevBuf& off, DevBuf* keep,
                   const int32_t** list) {
    cudaStream_t s = ctx.stream;
    cudaError_t err;
    if ((err = ensure(ctx.dkeys[0], m * 4)) || (err = ensure(ctx.dkeys[1], m * 4)) ||
        (err = ensure(ctx.dvals[0], m * 4)) || (err = ensure(ctx.dvals[1], m * 4)) ||
        (err = ensure(ctx.dhist, sort_hist_bytes(m))) || (err = ensure(ctx.dsort_tmp, sort_scan_bytes(m))) ||
        (err = ensure(off, (nmax + 1) * 8)) || (keep && (err = ensure(*keep, m * 4))))
        return cuda_status(ctx, err, "allocating adjoint scratch");
    const int tb = 256;
    k_sender_keys<<<div_up(m, tb), tb, 0, s>>>(idx, m, ctx.dkeys[0].as<uint32_t>());
    int bits = 0;
    while (bits < 32 && ((uint64_t)(nmax - 1) >> bits) != 0) ++bits;
    uint32_t* kb[2] = {ctx.dkeys[0].as<uint32_t>(), ctx.dkeys[1].as<uint32_t>()};
    int32_t* vb[2] = {ctx.dvals[0].as<int32_t>(), ctx.dvals[1].as<int32_t>()};
    const int src = radix_sort_pairs<uint32_t>(kb, vb, ctx.dhist.as<int32_t>(), ctx.dsort_tmp.as<int64_t>(), m, bits,
                                               false, s, &ctx.kernel_launches);
    k_sorted_starts<<<div_up(nmax + 1, tb), tb, 0, s>>>(kb[src], m, nmax, off.as<int64_t>());
    ctx.kernel_launches += 2;
    *list = nullptr;
    if (bits > 0) {
        if (keep) {
            if ((err = cudaMemcpyAsync(keep->p, vb[src], m * 4, cudaMemcpyDeviceToDevice, s)))
                return cuda_status(ctx, err, "adjoint order copy");
            *list = keep->as<int32_t>();
        } else {
            *list = vb[src];
        }
    }
    return cuda_status(ctx, cudaGetLastError(), "adjoint order");
}

int bad_coo(Ctx& ctx, int flags) {
    if (flags & kAdjBadOrder) return set_error(ctx, ERR_ARGUMENT, "build_edges_diff adjoint: order is not a permutation of 1..n");
    return set_error(ctx, ERR_ARGUMENT, "build_edges_diff adjoint: sender or receiver index out of range");
}

// Self-pair adjoint through the edges' mirrors; *flags = the status bits
// (0: grad written).
template <class T, int D>
int twins_typed(Ctx& ctx, int64_t n, int64_t m, const int32_t* snd, const int32_t* rcv, const void* rel_disp,
                const void* rel_dist, const void* coords, const void* d_disp, const void* d_dist, double radius,
                void* grad, const int32_t* order, int* flags) {
    cudaStream_t s = ctx.stream;
    cudaError_t err;
    const T r = (T)radius;
    const T inv_r = T(1) / r;
    if ((err = ensure(ctx.droff, (n + 1) * 8)) || (err = ensure(ctx.dstatus, 8)) ||
        (err = ensure(ctx.dseg, n * 8)) || (err = ensure(ctx.dterm, (size_t)m * sizeof(Term4<T>))))
        return cuda_status(ctx, err, "allocating adjoint scratch");
    const int tb = 256;
    PhaseTimer pt_(ctx, PH_ADJOINT);
    int* status = adjoint_status(ctx);
    if ((err = cudaMemsetAsync(status, 0, 4, s))) return cuda_status(ctx, err, "status reset");
    launch_pdl(k_segment_starts, div_up(n + 1, tb), tb, 0, s, rcv, m, n, ctx.droff.as<int64_t>());
    launch_pdl(k_seg_pairs, div_up(n, tb), tb, 0, s, ctx.droff.as<int64_t>(), n, ctx.dseg.as<int2>());
    Term4<T>* term = ctx.dterm.as<Term4<T>>();
    if (coords)
        launch_pdl(k_edge_terms<T, D, true>, div_up(m, tb), tb, 0, s, m, n, snd, rcv, nullptr, nullptr,
            (const T*)coords, (const T*)d_disp, (const T*)d_dist, r, inv_r, term);
    else
        launch_pdl(k_edge_terms<T, D, false>, div_up(m, tb), tb, 0, s, m, n, snd, rcv, (const T*)rel_disp,
            (const T*)rel_dist, nullptr, (const T*)d_disp, (const T*)d_dist, r, inv_r, term);
    const bool vec = ((uintptr_t)snd & 15) == 0;
    launch_pdl(k_adjoint_twins<T>, (unsigned)div_up(n, kTwinGroups * kTwinWarps), 32 * kTwinWarps, 0, s, n, m, order,
        ctx.dseg.as<int2>(), snd, rcv, term, D, vec, (T*)grad, status);
    ctx.kernel_launches += 4;
    if ((err = cudaGetLastError())) return cuda_status(ctx, err, "adjoint launch");
    return read_status(ctx, flags);
}

// Adjoint through sorted edge lists.  `flags` are the COO's status bits when
// known (-1: checked here).
template <class T, int D>
int backward_typed(Ctx& ctx, int64_t n, int64_t m, const int32_t* snd, const int32_t* rcv, const void* rel_disp,
                   const void* rel_dist, const void* d_disp, const void* d_dist, double radius, void* grad,
                   int flags) {
    cudaStream_t s = ctx.stream;
    cudaError_t err;
    const T r = (T)radius;
    if (m == 0 || (!d_disp && !d_dist)) {
        return cuda_status(ctx, cudaMemsetAsync(grad, 0, sizeof(T) * D * n, s), "zero gradient");
    }
    int st;
    if (flags < 0 && (st = coo_flags(ctx, snd, rcv, m, n, n, &flags)) != OK) return st;
    if (flags & kAdjBadIndex) return bad_coo(ctx, flags);
    PhaseTimer pt_(ctx, PH_ADJOINT);
    const int tb = 256;
    const int32_t* rlist = nullptr;
    if (flags & kAdjUngrouped) {
        if ((st = order_by_index(ctx, rcv, m, n, ctx.droff, &ctx.dredge, &rlist)) != OK) return st;
    } else {
        if ((err = ensure(ctx.droff, (n + 1) * 8))) return cuda_status(ctx, err, "allocating adjoint scratch");
        k_segment_starts<<<div_up(n + 1, tb), tb, 0, s>>>(rcv, m, n, ctx.droff.as<int64_t>());
        ctx.kernel_launches += 1;
    }
    const int32_t* slist = nullptr;
    if ((st = order_by_index(ctx, snd, m, n, ctx.dsoff, nullptr, &slist)) != OK) return st;
    k_grad<T, D><<<div_up(n, tb), tb, 0, s>>>(n, ctx.droff.as<int64_t>(), rlist, ctx.dsoff.as<int64_t>(), slist,
                                             (const T*)rel_disp, (const T*)rel_dist, (const T*)d_disp,
                                             (const T*)d_dist, r, (T*)grad);
    ctx.kernel_launches += 1;
    return cuda_status(ctx, cudaGetLastError(), "adjoint launch");
}

template <class T, int D>
int backward_pair_typed(Ctx& ctx, int64_t nq, int64_t nt, int64_t m, const int32_t* snd, const int32_t* rcv,
                        const void* rel_disp, const void* rel_dist, const void* d_disp, const void* d_dist,
                        double radius, void* grad_q, void* grad_t) {
    cudaStream_t s = ctx.stream;
    cudaError_t err;
    const T r = (T)radius;
    if (m == 0 || (!d_disp && !d_dist)) {
        if ((err = cudaMemsetAsync(grad_q, 0, sizeof(T) * D * nq, s)) ||
            (err = cudaMemsetAsync(grad_t, 0, sizeof(T) * D * nt, s)))
            return cuda_status(ctx, err, "zero gradient");
        return OK;
    }
    int flags = 0, st;
    if ((st = coo_flags(ctx, snd, rcv, m, nt, nq, &flags)) != OK) return st;
    if (flags & kAdjBadIndex) return bad_coo(ctx, flags);
    PhaseTimer pt_(ctx, PH_ADJOINT);
    const int tb = 256;
    const int32_t* rlist = nullptr;
    if (flags & kAdjUngrouped) {
        if ((st = order_by_index(ctx, rcv, m, nq, ctx.droff, &ctx.dredge, &rlist)) != OK) return st;
    } else {
        if ((err = ensure(ctx.droff, (nq + 1) * 8))) return cuda_status(ctx, err, "allocating adjoint scratch");
        k_segment_starts<<<div_up(nq + 1, tb), tb, 0, s>>>(rcv, m, nq, ctx.droff.as<int64_t>());
        ctx.kernel_launches += 1;
    }
    const int32_t* slist = nullptr;
    if ((st = order_by_index(ctx, snd, m, nt, ctx.dsoff, nullptr, &slist)) != OK) return st;
    k_grad_part<T, D><<<div_up(nq, tb), tb, 0, s>>>(nq, ctx.droff.as<int64_t>(), rlist, (const T*)rel_disp,
                                                    (const T*)rel_dist, (const T*)d_disp, (const T*)d_dist, r, 1.0,
                                                    (T*)grad_q);
    k_grad_part<T, D><<<div_up(nt, tb), tb, 0, s>>>(nt, ctx.dsoff.as<int64_t>(), slist, (const T*)rel_disp,
                                                    (const T*)rel_dist, (const T*)d_disp, (const T*)d_dist, r, -1.0,
                                                    (T*)grad_t);
    ctx.kernel_launches += 2;
    return cuda_status(ctx, cudaGetLastError(), "adjoint launch");
}

}  // namespace

int diff_backward_pair(Ctx& ctx, int ndims, int dtype, int64_t nq, int64_t nt, int64_t m, const int32_t* snd,
                       const int32_t* rcv, const void* rel_disp, const void* rel_dist, const void* d_disp,
                       const void* d_dist, double radius, void* grad_q, void* grad_t) {
    if (nq == 0 && nt == 0) return OK;
    if (nq == 0 || nt == 0) {
        // No edges can exist; the non-empty side's gradient is zero.
        const size_t es = dtype == 0 ? 4 : 8;
        cudaError_t err = cudaMemsetAsync(nq ? grad_q : grad_t, 0, es * ndims * (nq ? nq : nt), ctx.stream);
        return cuda_status(ctx, err, "zero gradient");
    }
    if (dtype == 0)
        return ndims == 3 ? backward_pair_typed<float, 3>(ctx, nq, nt, m, snd, rcv, rel_disp, rel_dist, d_disp, d_dist,
                                                          radius, grad_q, grad_t)
                          : backward_pair_typed<float, 2>(ctx, nq, nt, m, snd, rcv, rel_disp, rel_dist, d_disp, d_dist,
                                                          radius, grad_q, grad_t);
    return ndims == 3 ? backward_pair_typed<double, 3>(ctx, nq, nt, m, snd, rcv, rel_disp, rel_dist, d_disp, d_dist,
                                                       radius, grad_q, grad_t)
                      : backward_pair_typed<double, 2>(ctx, nq, nt, m, snd, rcv, rel_disp, rel_dist, d_disp, d_dist,
                                                       radius, grad_q, grad_t);
}

namespace {

template <class T, int D>
int mirror_typed(Ctx& ctx, int64_t n, int64_t m, const int32_t* snd, const int32_t* rcv, const int32_t* mirror,
                 const void* rel_disp, const void* rel_dist, const void* coords, const void* d_disp,
                 const void* d_dist, double radius, void* grad, const int32_t* order, int* flags) {
    cudaStream_t s = ctx.stream;
    cudaError_t err;
    const T r = (T)radius;
    const T inv_r = T(1) / r;
    if ((err = ensure(ctx.droff, (n + 1) * 8)) || (err = ensure(ctx.dstatus, 8)) || (err = ensure(ctx.dseg, n * 8)))
        return cuda_status(ctx, err, "allocating adjoint scratch");
    const int tb = 256;
    PhaseTimer pt_(ctx, PH_ADJOINT);
    int* status = adjoint_status(ctx);
    if ((err = cudaMemsetAsync(status, 0, 4, s))) return cuda_status(ctx, err, "status reset");
    launch_pdl(k_segment_starts, div_up(n + 1, tb), tb, 0, s, rcv, m, n, ctx.droff.as<int64_t>());
    launch_pdl(k_seg_pairs, div_up(n, tb), tb, 0, s, ctx.droff.as<int64_t>(), n, ctx.dseg.as<int2>());
    const unsigned blocks = (unsigned)div_up(n, kTwinGroups * kTwinWarps);
    const bool vec = ((uintptr_t)snd & 15) == 0;
    if (coords)
        launch_pdl(k_adjoint_mirror<T, D, true>, blocks, 32 * kTwinWarps, 0, s, n, m, order, ctx.dseg.as<int2>(), snd,
            rcv, mirror, nullptr, nullptr, (const T*)coords, (const T*)d_disp, (const T*)d_dist, r, inv_r, (T*)grad,
            status);
    else
        launch_pdl(k_adjoint_mirror<T, D, false>, blocks, 32 * kTwinWarps, 0, s, n, m, order, ctx.dseg.as<int2>(), snd,
            rcv, mirror, (const T*)rel_disp, (const T*)rel_dist, nullptr, (const T*)d_disp, (const T*)d_dist, r, inv_r,
            (T*)grad, status);
    ctx.kernel_launches += 3;
    if ((err = cudaGetLastError())) return cuda_status(ctx, err, "adjoint launch");
    return read_status(ctx, flags);
}

}  // namespace

int edges_mirror_scan(Ctx& ctx, const int32_t* snd, const int32_t* rcv, int64_t m, int64_t n, const int64_t* off,
                      int32_t* mirror) {
    if (m == 0) return OK;
    k_mirror_scan<<<div_up(m, 256), 256, 0, ctx.stream>>>(snd, rcv, m, n, off, mirror);
    ctx.kernel_launches += 1;
    return cuda_status(ctx, cudaGetLastError(), "mirror scan launch");
}

int diff_backward_mirror(Ctx& ctx, int ndims, int dtype, int64_t n, int64_t m, const int32_t* snd,
                         const int32_t* rcv, const int32_t* mirror, const void* rel_disp, const void* rel_dist,
                         const void* coords, const void* d_disp, const void* d_dist, double radius, void* grad,
                         const int32_t* order) {
    if (n == 0) return OK;
    if (m > 0 && (d_disp || d_dist)) {
        int flags = 0, st;
        if (dtype == 0)
            st = ndims == 3 ? mirror_typed<float, 3>(ctx, n, m, snd, rcv, mirror, rel_disp, rel_dist, coords, d_disp,
                                                     d_dist, radius, grad, order, &flags)
                            : mirror_typed<float, 2>(ctx, n, m, snd, rcv, mirror, rel_disp, rel_dist, coords, d_disp,
                                                     d_dist, radius, grad, order, &flags);
        else
            st = ndims == 3 ? mirror_typed<double, 3>(ctx, n, m, snd, rcv, mirror, rel_disp, rel_dist, coords, d_disp,
                                                      d_dist, radius, grad, order, &flags)
                            : mirror_typed<double, 2>(ctx, n, m, snd, rcv, mirror, rel_disp, rel_dist, coords, d_disp,
                                                      d_dist, radius, grad, order, &flags);
        if (st != OK || flags == 0) return st;
        if (flags & kAdjBadOrder) return bad_coo(ctx, flags);
        // A mirror index that does not fit, or a COO not grouped by receiver:
        // the general path checks and handles the COO from scratch.
    }
    return diff_backward(ctx, ndims, dtype, n, m, snd, rcv, rel_disp, rel_dist, d_disp, d_dist, radius, grad, coords,
                         order);
}

int diff_backward(Ctx& ctx, int ndims, int dtype, int64_t n, int64_t m, const int32_t* snd, const int32_t* rcv,
                  const void* rel_disp, const void* rel_dist, const void* d_disp, const void* d_dist, double radius,
                  void* grad, const void* coords, const int32_t* order) {
    if (n == 0) return OK;
    // The twin search scans a neighbor's whole segment per edge: worthwhile
    // for the sparse graphs of this path (tens of neighbors), while dense
    // graphs go through the sorted path.
    const bool twins = coords != nullptr || m <= 64 * n;
    int flags = -1;
    if (m > 0 && (d_disp || d_dist) && twins) {
        int st;
        if (dtype == 0)
            st = ndims == 3 ? twins_typed<float, 3>(ctx, n, m, snd, rcv, rel_disp, rel_dist, coords, d_disp, d_dist,
                                                    radius, grad, order, &flags)
                            : twins_typed<float, 2>(ctx, n, m, snd, rcv, rel_disp, rel_dist, coords, d_disp, d_dist,
                                                    radius, grad, order, &flags);
        else
            st = ndims == 3 ? twins_typed<double, 3>(ctx, n, m, snd, rcv, rel_disp, rel_dist, coords, d_disp, d_dist,
                                                     radius, grad, order, &flags)
                            : twins_typed<double, 2>(ctx, n, m, snd, rcv, rel_disp, rel_dist, coords, d_disp, d_dist,
                                                     radius, grad, order, &flags);
        if (st != OK || flags == 0) return st;
        if (flags & kAdjBadOrder) return bad_coo(ctx, flags);
        // Without the ungrouped bit every edge was visited, so the bits are
        // complete; otherwise the sorted path checks the whole COO again.
        if (flags & kAdjUngrouped) flags = -1;
        else if (flags & kAdjBadIndex) return bad_coo(ctx, flags);
        else flags &= ~kAdjMissingTwin;
        if (coords)
            return set_error(ctx, ERR_ARGUMENT,
                             "build_edges_diff adjoint: recomputing needs a self-pair COO grouped by receiver");
    }
    if (dtype == 0)
        return ndims == 3 ? backward_typed<float, 3>(ctx, n, m, snd, rcv, rel_disp, rel_dist, d_disp, d_dist, radius,
                                                     grad, flags)
                          : backward_typed<float, 2>(ctx, n, m, snd, rcv, rel_disp, rel_dist, d_disp, d_dist, radius,
                                                     grad, flags);
    return ndims == 3 ? backward_typed<double, 3>(ctx, n, m, snd, rcv, rel_disp, rel_dist, d_disp, d_dist, radius,
                                                  grad, flags)
                      : backward_typed<double, 2>(ctx, n, m, snd, rcv, rel_disp, rel_dist, d_disp, d_dist, radius,
                                                  grad, flags);
}

}  // namespace oct
