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

// Warp layout of the self-pair adjoint: one warp takes kTwinPoints points in
// the order `order` (the tree's Morton permutation, 1-based; null for
// 0..n-1) and their segments' edges one per lane.  With a spatial order the
// mirror edges read by the warps in flight lie in the segments of nearby
// points, so they stay in L2 while the segments of all points in flight fit: a
// few points per warp keep that working set small while the lanes still have
// an edge each.  The order changes only which warp handles a point, never a
// point's sum.  Each edge also checks the COO (receiver of its segment, sender
// range, a mirror present); a failed check sets a status bit and the caller
// takes the sorted path.
constexpr int kTwinWarps = 4;
constexpr int kTwinPoints = 4;  // points per warp (a power of two, at most 32)

// Pass 2 of the searching adjoint: each edge's mirror found by scanning its
// sender's segment, term(k) - term(mirror) summed per point.  Measured on
// B200 at 2M points, these two passes (1.19 ms) beat one pass that searches
// and reads the mirror's cotangents itself (1.63 ms): the term records
// stream in one coalesced pass before the searching pass reads them.
// One warp takes kTwinPoints points in the order `order` (the tree's Morton
// permutation, 1-based; null for 0..n-1) and their segments' edges one per
// lane.  With a spatial order the twins read by the warps in flight lie in
// the segments of nearby points, so they stay in L2 while the segments of
// all points in flight fit: a few points per warp keep that working set
// small while the lanes still have an edge each.  The order changes only
// which warp handles a point, never a point's sum.  Each edge also checks
// the COO (receiver of its segment, sender range, a twin present); a failed
// check sets a status bit and the caller takes the sorted path.  `vec`: the
// sender array is 16-byte aligned, so the twin scan reads four entries per
// load.

template <class T>
__global__ void __launch_bounds__(kTwinWarps * 32) k_adjoint_twins(
    int64_t n, int64_t m, const int32_t* __restrict__ order, const int2* __restrict__ seg,
    const int32_t* __restrict__ snd, const int32_t* __restrict__ rcv, const Term4<T>* __restrict__ term, int ndims,
    bool vec, T* __restrict__ grad, int* __restrict__ status) {
    __shared__ double snet[kTwinWarps][3][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t s0 = ((int64_t)blockIdx.x * kTwinWarps + w) * kTwinPoints;
    if (s0 >= n) return;  // warp-uniform
    const int64_t sl = s0 + lane;
    int p = -1, k0 = 0, ne = 0;
    int bad = 0;
    if (lane < kTwinPoints && sl < n) {
        const int64_t pp = order ? (int64_t)order[sl] - 1 : sl;
        if (pp < 0 || pp >= n) {
            bad |= kAdjBadOrder;
        } else {
            p = (int)pp;
            const int2 sg = seg[p];
            k0 = sg.x;
            ne = sg.y - sg.x;
            if (ne < 0 || (p == 0 && k0 != 0) || (p == n - 1 && sg.y != m)) {
                bad |= kAdjUngrouped;
                ne = 0;
            }
        }
    }
    int incl = ne;  // edge counts fit int32 (n_edges < 2^31)
#pragma unroll
    for (int o = 1; o < kTwinPoints; o <<= 1) {
        const int a = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += a;
    }
    const int excl = incl - ne;
    const int total = __shfl_sync(0xffffffffu, incl, kTwinPoints - 1);
    double acc[3] = {0.0, 0.0, 0.0};
    for (int f0 = 0; f0 < total; f0 += 32) {
        const int f = f0 + lane;
        // owner of flat edge f: the first lane whose inclusive end exceeds f
        int o = 0;
#pragma unroll
        for (int st = kTwinPoints / 2; st; st >>= 1) {
            const int v = __shfl_sync(0xffffffffu, incl, o + st - 1);
            if (v <= f) o += st;
        }
        const int ko = __shfl_sync(0xffffffffu, k0, o);
        const int eo = __shfl_sync(0xffffffffu, excl, o);
        const int po = __shfl_sync(0xffffffffu, p, o);
        double net[3] = {0.0, 0.0, 0.0};
        if (f < total) {
            const int32_t k = ko + (f - eo);
            const int32_t i1 = po + 1;
            const int32_t j1 = snd[k];
            if (rcv[k] != i1) bad |= kAdjUngrouped;
            const Term4<T> tk = term[k];
            if (j1 < 1 || j1 > n) {
                bad |= kAdjBadIndex;
            } else {
                const int2 sj = seg[j1 - 1];
                int32_t tw = -1;
                if (vec) {
                    // aligned blocks of four entries; the last block of the
                    // array is read entry by entry
                    for (int32_t qa = sj.x & ~3; qa < sj.y && tw < 0; qa += 4) {
                        int32_t c[4];
                        if ((int64_t)qa + 3 < m) {
                            const int4 v = *reinterpret_cast<const int4*>(snd + qa);
                            c[0] = v.x; c[1] = v.y; c[2] = v.z; c[3] = v.w;
                        } else {
#pragma unroll
                            for (int u = 0; u < 4; ++u) c[u] = (int64_t)qa + u < m ? snd[qa + u] : 0;
                        }
#pragma unroll
                        for (int u = 3; u >= 0; --u)
                            if (c[u] == i1 && (int64_t)qa + u >= sj.x && (int64_t)qa + u < sj.y) tw = qa + u;
                    }
                } else {
                    for (int32_t q = sj.x; q < sj.y && tw < 0; q += 4) {
                        int32_t c[4];
#pragma unroll
                        for (int u = 0; u < 4; ++u) c[u] = (int64_t)q + u < sj.y ? snd[q + u] : 0;
#pragma unroll
                        for (int u = 3; u >= 0; --u)
                            if (c[u] == i1 && (int64_t)q + u < sj.y) tw = q + u;
                    }
                }
                if (tw < 0) {
                    bad |= kAdjMissingTwin;
                } else {
                    const Term4<T> tt = term[tw];
#pragma unroll
                    for (int d = 0; d < 3; ++d) net[d] = (double)tk.v[d] - (double)tt.v[d];
                }
            }
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) snet[w][d][lane] = net[d];
        __syncwarp();
        // each lane adds the entries of its own segment, in edge order
        const int e1 = min(incl, f0 + 32);
        for (int e = max(excl, f0); e < e1; ++e) {
#pragma unroll
            for (int d = 0; d < 3; ++d) acc[d] += snet[w][d][e - f0];
        }
        __syncwarp();
    }
    if (p >= 0) {
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
    __shared__ double snet[kTwinWarps][3][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t s0 = ((int64_t)blockIdx.x * kTwinWarps + w) * kTwinPoints;
    if (s0 >= n) return;  // warp-uniform
    const int64_t sl = s0 + lane;
    int p = -1, k0 = 0, ne = 0;
    int bad = 0;
    if (lane < kTwinPoints && sl < n) {
        const int64_t pp = order ? (int64_t)order[sl] - 1 : sl;
        if (pp < 0 || pp >= n) {
            bad |= kAdjBadOrder;
        } else {
            p = (int)pp;
            const int2 sg = seg[p];
            k0 = sg.x;
            ne = sg.y - sg.x;
            if (ne < 0 || (p == 0 && k0 != 0) || (p == n - 1 && sg.y != m)) {
                bad |= kAdjUngrouped;
                ne = 0;
            }
        }
    }
    int incl = ne;
#pragma unroll
    for (int o = 1; o < kTwinPoints; o <<= 1) {
        const int a = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += a;
    }
    const int excl = incl - ne;
    const int total = __shfl_sync(0xffffffffu, incl, kTwinPoints - 1);
    double acc[3] = {0.0, 0.0, 0.0};
    for (int f0 = 0; f0 < total; f0 += 32) {
        const int f = f0 + lane;
        int o = 0;
#pragma unroll
        for (int st = kTwinPoints / 2; st; st >>= 1) {
            const int v = __shfl_sync(0xffffffffu, incl, o + st - 1);
            if (v <= f) o += st;
        }
        const int ko = __shfl_sync(0xffffffffu, k0, o);
        const int eo = __shfl_sync(0xffffffffu, excl, o);
        const int po = __shfl_sync(0xffffffffu, p, o);
        double net[3] = {0.0, 0.0, 0.0};
        if (f < total) {
            const int32_t k = ko + (f - eo);
            if (rcv[k] != po + 1) bad |= kAdjUngrouped;
            bool ok = true;
            int32_t j = -1;
            if (RECOMPUTE) {
                j = snd[k] - 1;
                if (j < 0 || j >= n) {
                    bad |= kAdjBadIndex;
                    ok = false;
                }
            }
            const int32_t t = mirror[k];
            T rd[D], rn = T(0);
            if (ok && !(t >= 0 && (int64_t)t < m)) {
                bad |= kAdjMissingTwin;
                ok = false;
            }
            if (RECOMPUTE) {
                if (j >= 0 && j < n) {
                    T diff[D];
                    const T d2 = dist2<T, D>(coords + (int64_t)D * j, coords + (int64_t)D * po, diff);
#pragma unroll
                    for (int d = 0; d < D; ++d) rd[d] = mul_rn(-diff[d], inv_r);
                    rn = mul_rn(sqrt_rn(d2), inv_r);
                }
            } else {
#pragma unroll
                for (int d = 0; d < D; ++d) rd[d] = rel_disp[(int64_t)D * k + d];
                rn = rel_dist[k];
            }
            if (ok) {
                const Term4<T> tk = mirror_term<T, D, RECOMPUTE>(rd, rn, d_disp, d_dist, k, r, T(1));
                const Term4<T> tt = mirror_term<T, D, RECOMPUTE>(rd, rn, d_disp, d_dist, t, r, T(-1));
#pragma unroll
                for (int d = 0; d < 3; ++d) net[d] = (double)tk.v[d] - (double)tt.v[d];
            }
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) snet[w][d][lane] = net[d];
        __syncwarp();
        const int e1 = min(incl, f0 + 32);
        for (int e = max(excl, f0); e < e1; ++e) {
#pragma unroll
            for (int d = 0; d < 3; ++d) acc[d] += snet[w][d][e - f0];
        }
        __syncwarp();
    }
    if (p >= 0) {
#pragma unroll
        for (int d = 0; d < D; ++d) grad[(int64_t)D * p + d] = (T)acc[d];
    }
    if (bad) atomicOr(status, bad);
}

// Mirror index of every edge of a self-pair COO grouped by receiver, by
// scanning the sender's segment (off: int64 segment starts) -- for the
// differentiable fill when the hit records were incomplete.  -1 when absent.
__global__ void k_mirror_scan(const int32_t* __restrict__ snd, const int32_t* __restrict__ rcv, int64_t m, int64_t n,
                              const int64_t* __restrict__ off, int32_t* __restrict__ mirror) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    const int32_t i1 = rcv[k], j = snd[k] - 1;
    int32_t t = -1;
    if (j >= 0 && j < n)
        for (int64_t q = off[j]; q < off[j + 1]; ++q)
            if (snd[q] == i1) {
                t = (int32_t)q;
                break;
            }
    mirror[k] = t;
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
    k_segment_starts<<<div_up(n + 1, tb), tb, 0, s>>>(rcv, m, n, ctx.droff.as<int64_t>());
    k_seg_pairs<<<div_up(n, tb), tb, 0, s>>>(ctx.droff.as<int64_t>(), n, ctx.dseg.as<int2>());
    Term4<T>* term = ctx.dterm.as<Term4<T>>();
    if (coords)
        k_edge_terms<T, D, true><<<div_up(m, tb), tb, 0, s>>>(m, n, snd, rcv, nullptr, nullptr, (const T*)coords,
                                                               (const T*)d_disp, (const T*)d_dist, r, inv_r, term);
    else
        k_edge_terms<T, D, false><<<div_up(m, tb), tb, 0, s>>>(m, n, snd, rcv, (const T*)rel_disp, (const T*)rel_dist,
                                                                nullptr, (const T*)d_disp, (const T*)d_dist, r, inv_r,
                                                                term);
    const bool vec = ((uintptr_t)snd & 15) == 0;
    k_adjoint_twins<T><<<(unsigned)div_up(n, kTwinPoints * kTwinWarps), 32 * kTwinWarps, 0, s>>>(
        n, m, order, ctx.dseg.as<int2>(), snd, rcv, term, D, vec, (T*)grad, status);
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
    k_segment_starts<<<div_up(n + 1, tb), tb, 0, s>>>(rcv, m, n, ctx.droff.as<int64_t>());
    k_seg_pairs<<<div_up(n, tb), tb, 0, s>>>(ctx.droff.as<int64_t>(), n, ctx.dseg.as<int2>());
    const unsigned blocks = (unsigned)div_up(n, kTwinPoints * kTwinWarps);
    const bool vec = ((uintptr_t)snd & 15) == 0;
    if (coords)
        k_adjoint_mirror<T, D, true><<<blocks, 32 * kTwinWarps, 0, s>>>(
            n, m, order, ctx.dseg.as<int2>(), snd, rcv, mirror, nullptr, nullptr, (const T*)coords, (const T*)d_disp,
            (const T*)d_dist, r, inv_r, (T*)grad, status);
    else
        k_adjoint_mirror<T, D, false><<<blocks, 32 * kTwinWarps, 0, s>>>(
            n, m, order, ctx.dseg.as<int2>(), snd, rcv, mirror, (const T*)rel_disp, (const T*)rel_dist, nullptr,
            (const T*)d_disp, (const T*)d_dist, r, inv_r, (T*)grad, status);
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
