// Adjoint of build_edges_diff (ext/OctopusChainRulesCoreExt.jl:137-192,
// ext/OctopusCUDAChainRulesCoreExt.jl:56-99), without floating-point atomics.
//
// Per edge k = (receiver i <- sender j) the cotangent contributes
//   c_k = d_disp[:,k] / r + rel_disp[:,k] * (d_dist[k] / (rel_dist[k] * r))
// (the second term only when rel_dist[k] > 1e-8), added to x_i and
// subtracted from x_j.  The edges are already grouped by receiver, so the
// receiver sum is a segmented reduction in edge order; the sender sum reads
// the edges re-ordered by (sender, edge index) with the stable radix sort.
// Every point sums its terms in a fixed order in double precision, so the
// result is bit-reproducible from run to run.

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

template <class T, int D>
__global__ void k_grad(int64_t n, const int64_t* __restrict__ roff, const int64_t* __restrict__ soff,
                       const int32_t* __restrict__ sorted_edge, const T* __restrict__ rel_disp,
                       const T* __restrict__ rel_dist, const T* __restrict__ d_disp, const T* __restrict__ d_dist, T r,
                       T* __restrict__ grad) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double acc[D];
#pragma unroll
    for (int d = 0; d < D; ++d) acc[d] = 0.0;
    double c[D];
    for (int64_t k = roff[i]; k < roff[i + 1]; ++k) {
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

// Self-pair adjoint without a sort.  The neighbor relation of a self pair is
// symmetric, so the edge k = (i <- j) of point i's segment has a twin
// t = (j <- i) in j's segment, found by scanning j's segment.  The twin's
// features are those of k mirrored exactly (rel_disp[t] = -rel_disp[k] and
// rel_dist[t] = rel_dist[k] bit for bit, from the forward's arithmetic), so
// only its cotangents are read.  Point i's gradient is
//   sum over its segment of term(k) - term(t),
// one value per edge here (v[k], in edge order), summed per segment by
// k_sum_segments.  A missing twin (the edges are not a self-pair COO) raises
// the flag and the caller takes the sorted path.
template <class T, int D, bool RECOMPUTE>
__global__ void k_edge_net(int64_t m, const int64_t* __restrict__ roff, const int32_t* __restrict__ snd,
                           const int32_t* __restrict__ rcv, const T* __restrict__ rel_disp,
                           const T* __restrict__ rel_dist, const T* __restrict__ coords,
                           const T* __restrict__ d_disp, const T* __restrict__ d_dist, T r, T inv_r,
                           double* __restrict__ v, int* __restrict__ missing) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    const int32_t i1 = rcv[k];
    const int32_t j = snd[k] - 1;
    const int64_t q1 = roff[j + 1];
    int64_t tw = -1;
    for (int64_t q = roff[j]; q < q1; ++q)
        if (snd[q] == i1) { tw = q; break; }
    if (tw < 0) {
        atomicOr(missing, 1);
        return;
    }
    // Features of edge k (receiver i = i1 - 1, sender j).
    T rd[D], rn;
    if (RECOMPUTE) {
        T diff[D];
        const T d2 = dist2<T, D>(coords + (int64_t)D * j, coords + (int64_t)D * (i1 - 1), diff);
#pragma unroll
        for (int d = 0; d < D; ++d) rd[d] = mul_rn(-diff[d], inv_r);
        rn = mul_rn(sqrt_rn(d2), inv_r);
    } else {
#pragma unroll
        for (int d = 0; d < D; ++d) rd[d] = rel_disp[(int64_t)D * k + d];
        rn = rel_dist[k];
    }
    double net[D];
#pragma unroll
    for (int d = 0; d < D; ++d) net[d] = 0.0;
    if (d_disp) {
#pragma unroll
        for (int d = 0; d < D; ++d)
            net[d] += (double)div_rn(d_disp[(int64_t)D * k + d], r) - (double)div_rn(d_disp[(int64_t)D * tw + d], r);
    }
    if (d_dist && rn > T(1e-8)) {
        const T a = div_rn(d_dist[k], mul_rn(rn, r));
        const T b = div_rn(d_dist[tw], mul_rn(rn, r));
        // term(t) uses rel_disp[t] = -rd, so it enters with the opposite sign.
#pragma unroll
        for (int d = 0; d < D; ++d) net[d] += (double)mul_rn(rd[d], a) + (double)mul_rn(rd[d], b);
    }
#pragma unroll
    for (int d = 0; d < D; ++d) v[(int64_t)D * k + d] = net[d];
}

// grad[i] = sum of v over point i's segment, in edge order.
template <class T, int D>
__global__ void k_sum_segments(int64_t n, const int64_t* __restrict__ roff, const double* __restrict__ v,
                               T* __restrict__ grad) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double acc[D];
#pragma unroll
    for (int d = 0; d < D; ++d) acc[d] = 0.0;
    const int64_t k1 = roff[i + 1];
    for (int64_t k = roff[i]; k < k1; ++k) {
#pragma unroll
        for (int d = 0; d < D; ++d) acc[d] += v[(int64_t)D * k + d];
    }
#pragma unroll
    for (int d = 0; d < D; ++d) grad[(int64_t)D * i + d] = (T)acc[d];
}

namespace {

template <class T, int D>
int twins_typed(Ctx& ctx, int64_t n, int64_t m, const int32_t* snd, const int32_t* rcv, const void* rel_disp,
                const void* rel_dist, const void* coords, const void* d_disp, const void* d_dist, double radius,
                void* grad, bool* ok) {
    cudaStream_t s = ctx.stream;
    cudaError_t err;
    const T r = (T)radius;
    const T inv_r = T(1) / r;
    if ((err = ensure(ctx.droff, (n + 1) * 8)) || (err = ensure(ctx.dstatus, 8)) ||
        (err = ensure(ctx.dnet, (size_t)m * D * 8)))
        return cuda_status(ctx, err, "allocating adjoint scratch");
    const int tb = 256;
    PhaseTimer pt_(ctx, PH_ADJOINT);
    // Word 1 of the status buffer (word 0 belongs to the edge fill guard).
    int* missing_flag = ctx.dstatus.as<int>() + 1;
    if ((err = cudaMemsetAsync(missing_flag, 0, 4, s))) return cuda_status(ctx, err, "status reset");
    double* v = ctx.dnet.as<double>();
    k_segment_starts<<<div_up(n + 1, tb), tb, 0, s>>>(rcv, m, n, ctx.droff.as<int64_t>());
    if (coords)
        k_edge_net<T, D, true><<<div_up(m, tb), tb, 0, s>>>(m, ctx.droff.as<int64_t>(), snd, rcv, nullptr, nullptr,
                                                             (const T*)coords, (const T*)d_disp, (const T*)d_dist, r,
                                                             inv_r, v, missing_flag);
    else
        k_edge_net<T, D, false><<<div_up(m, tb), tb, 0, s>>>(m, ctx.droff.as<int64_t>(), snd, rcv,
                                                              (const T*)rel_disp, (const T*)rel_dist, nullptr,
                                                              (const T*)d_disp, (const T*)d_dist, r, inv_r, v,
                                                              missing_flag);
    ctx.kernel_launches += 2;
    int missing = 0;
    if ((err = cudaMemcpyAsync(&missing, missing_flag, 4, cudaMemcpyDeviceToHost, s)) ||
        (err = wait_stream(s)))
        return cuda_status(ctx, err, "adjoint");
    *ok = missing == 0;
    if (!*ok) return OK;
    k_sum_segments<T, D><<<div_up(n, tb), tb, 0, s>>>(n, ctx.droff.as<int64_t>(), v, (T*)grad);
    ctx.kernel_launches += 1;
    return cuda_status(ctx, cudaGetLastError(), "adjoint launch");
}


template <class T, int D>
int backward_typed(Ctx& ctx, int64_t n, int64_t m, const int32_t* snd, const int32_t* rcv, const void* rel_disp,
                   const void* rel_dist, const void* d_disp, const void* d_dist, double radius, void* grad) {
    cudaStream_t s = ctx.stream;
    cudaError_t err;
    const T r = (T)radius;
    if (m == 0 || (!d_disp && !d_dist)) {
        return cuda_status(ctx, cudaMemsetAsync(grad, 0, sizeof(T) * D * n, s), "zero gradient");
    }
    if ((err = ensure(ctx.dkeys[0], m * 4)) || (err = ensure(ctx.dkeys[1], m * 4)) ||
        (err = ensure(ctx.dvals[0], m * 4)) || (err = ensure(ctx.dvals[1], m * 4)) ||
        (err = ensure(ctx.dhist, sort_hist_bytes(m))) || (err = ensure(ctx.dsort_tmp, sort_scan_bytes(m))) ||
        (err = ensure(ctx.droff, (n + 1) * 8)) ||
        (err = ensure(ctx.dsoff, (n + 1) * 8)))
        return cuda_status(ctx, err, "allocating adjoint scratch");
    const int tb = 256;
    PhaseTimer pt_(ctx, PH_ADJOINT);
    k_segment_starts<<<div_up(n + 1, tb), tb, 0, s>>>(rcv, m, n, ctx.droff.as<int64_t>());
    k_sender_keys<<<div_up(m, tb), tb, 0, s>>>(snd, m, ctx.dkeys[0].as<uint32_t>());
    int bits = 0;
    while (bits < 32 && ((uint64_t)(n - 1) >> bits) != 0) ++bits;
    uint32_t* kb[2] = {ctx.dkeys[0].as<uint32_t>(), ctx.dkeys[1].as<uint32_t>()};
    int32_t* vb[2] = {ctx.dvals[0].as<int32_t>(), ctx.dvals[1].as<int32_t>()};
    const int src = radix_sort_pairs<uint32_t>(kb, vb, ctx.dhist.as<int32_t>(), ctx.dsort_tmp.as<int64_t>(), m, bits,
                                               false, s, &ctx.kernel_launches);
    const int32_t* sorted_edge = bits > 0 ? vb[src] : nullptr;
    k_sorted_starts<<<div_up(n + 1, tb), tb, 0, s>>>(kb[src], m, n, ctx.dsoff.as<int64_t>());
    k_grad<T, D><<<div_up(n, tb), tb, 0, s>>>(n, ctx.droff.as<int64_t>(), ctx.dsoff.as<int64_t>(), sorted_edge,
                                             (const T*)rel_disp, (const T*)rel_dist, (const T*)d_disp,
                                             (const T*)d_dist, r, (T*)grad);
    ctx.kernel_launches += 4;
    return cuda_status(ctx, cudaGetLastError(), "adjoint launch");
}

}  // namespace

namespace {

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
    if ((err = ensure(ctx.dkeys[0], m * 4)) || (err = ensure(ctx.dkeys[1], m * 4)) ||
        (err = ensure(ctx.dvals[0], m * 4)) || (err = ensure(ctx.dvals[1], m * 4)) ||
        (err = ensure(ctx.dhist, sort_hist_bytes(m))) || (err = ensure(ctx.dsort_tmp, sort_scan_bytes(m))) ||
        (err = ensure(ctx.droff, (nq + 1) * 8)) || (err = ensure(ctx.dsoff, (nt + 1) * 8)))
        return cuda_status(ctx, err, "allocating adjoint scratch");
    const int tb = 256;
    PhaseTimer pt_(ctx, PH_ADJOINT);
    k_segment_starts<<<div_up(nq + 1, tb), tb, 0, s>>>(rcv, m, nq, ctx.droff.as<int64_t>());
    k_sender_keys<<<div_up(m, tb), tb, 0, s>>>(snd, m, ctx.dkeys[0].as<uint32_t>());
    int bits = 0;
    while (bits < 32 && ((uint64_t)(nt - 1) >> bits) != 0) ++bits;
    uint32_t* kb[2] = {ctx.dkeys[0].as<uint32_t>(), ctx.dkeys[1].as<uint32_t>()};
    int32_t* vb[2] = {ctx.dvals[0].as<int32_t>(), ctx.dvals[1].as<int32_t>()};
    const int src = radix_sort_pairs<uint32_t>(kb, vb, ctx.dhist.as<int32_t>(), ctx.dsort_tmp.as<int64_t>(), m, bits,
                                               false, s, &ctx.kernel_launches);
    const int32_t* sorted_edge = bits > 0 ? vb[src] : nullptr;
    k_sorted_starts<<<div_up(nt + 1, tb), tb, 0, s>>>(kb[src], m, nt, ctx.dsoff.as<int64_t>());
    k_grad_part<T, D><<<div_up(nq, tb), tb, 0, s>>>(nq, ctx.droff.as<int64_t>(), nullptr, (const T*)rel_disp,
                                                    (const T*)rel_dist, (const T*)d_disp, (const T*)d_dist, r, 1.0,
                                                    (T*)grad_q);
    k_grad_part<T, D><<<div_up(nt, tb), tb, 0, s>>>(nt, ctx.dsoff.as<int64_t>(), sorted_edge, (const T*)rel_disp,
                                                    (const T*)rel_dist, (const T*)d_disp, (const T*)d_dist, r, -1.0,
                                                    (T*)grad_t);
    ctx.kernel_launches += 5;
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

int diff_backward(Ctx& ctx, int ndims, int dtype, int64_t n, int64_t m, const int32_t* snd, const int32_t* rcv,
                  const void* rel_disp, const void* rel_dist, const void* d_disp, const void* d_dist, double radius,
                  void* grad, const void* coords) {
    if (n == 0) return OK;
    // The twin search scans a neighbor's whole segment per edge: worthwhile
    // for the sparse graphs of this path (tens of neighbors), while dense
    // graphs go through the sorted path.
    const bool twins = coords != nullptr || m <= 64 * n;
    if (m > 0 && (d_disp || d_dist) && twins) {
        bool ok = false;
        int st;
        if (dtype == 0)
            st = ndims == 3 ? twins_typed<float, 3>(ctx, n, m, snd, rcv, rel_disp, rel_dist, coords, d_disp, d_dist,
                                                    radius, grad, &ok)
                            : twins_typed<float, 2>(ctx, n, m, snd, rcv, rel_disp, rel_dist, coords, d_disp, d_dist,
                                                    radius, grad, &ok);
        else
            st = ndims == 3 ? twins_typed<double, 3>(ctx, n, m, snd, rcv, rel_disp, rel_dist, coords, d_disp, d_dist,
                                                     radius, grad, &ok)
                            : twins_typed<double, 2>(ctx, n, m, snd, rcv, rel_disp, rel_dist, coords, d_disp, d_dist,
                                                     radius, grad, &ok);
        if (st != OK || ok) return st;
        if (coords)
            return set_error(ctx, ERR_ARGUMENT, "build_edges_diff adjoint: recomputing needs a self-pair COO");
    }
    if (dtype == 0)
        return ndims == 3 ? backward_typed<float, 3>(ctx, n, m, snd, rcv, rel_disp, rel_dist, d_disp, d_dist, radius, grad)
                          : backward_typed<float, 2>(ctx, n, m, snd, rcv, rel_disp, rel_dist, d_disp, d_dist, radius, grad);
    return ndims == 3 ? backward_typed<double, 3>(ctx, n, m, snd, rcv, rel_disp, rel_dist, d_disp, d_dist, radius, grad)
                      : backward_typed<double, 2>(ctx, n, m, snd, rcv, rel_disp, rel_dist, d_disp, d_dist, radius, grad);
}

}  // namespace oct
