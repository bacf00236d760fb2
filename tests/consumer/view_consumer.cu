// A user kernel written against the exported tree view, the way Octopus.jl
// users write @cuda kernels against DeviceView with the inlined traversal
// macros (src/macros.jl:60-115 for 3D, :133-177 for 2D).  It includes only
// the public header and reads only the oct_tree_view arrays (1-based ids,
// -1 child sentinel, (2^D, n_nodes) children, (D, n_nodes) bounds, perm) and
// the caller's coordinates.  The traversal is the macro's: root id 1 pushed
// unconditionally, a node whose first child slot is -1 scanned as a leaf over
// perm[node_first .. node_last], otherwise children 1..2^D pushed in slot order
// when their box is within the radius, popped last in first out; no self
// filter.  Test code: it proves that the view supports such consumers.
#include <cstdint>
#include <cuda_runtime.h>

#include "octopus_b200.h"

namespace {

template <class T, int D>
__global__ void k_view_neighbors(oct_tree_view v, const T* __restrict__ cq, const T* __restrict__ ct, int64_t nq,
                                 T r_sq, int32_t* __restrict__ counts, int32_t* __restrict__ idx, int64_t cap) {
    constexpr int NCH = 1 << D;
    constexpr int STACK = 1 + (NCH - 1) * (D == 3 ? 21 : 31);  // STACK_DEPTH_3D / _2D
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nq) return;
    const T* bmin = static_cast<const T*>(v.bounds_min);
    const T* bmax = static_cast<const T*>(v.bounds_max);
    T p[D];
    for (int d = 0; d < D; ++d) p[d] = cq[(int64_t)D * i + d];
    int32_t stack[STACK];
    int sp = 0;
    int64_t c = 0;
    if (v.n_nodes > 0) stack[sp++] = 1;
    while (sp > 0) {
        const int32_t nid = stack[--sp];
        const int64_t n0 = nid - 1;
        if (v.node_children[NCH * n0] == -1) {
            for (int32_t k = v.node_first[n0]; k <= v.node_last[n0]; ++k) {
                const int32_t j = v.perm[k - 1];
                T d2 = T(0);
                for (int d = 0; d < D; ++d) {
                    const T dx = ct[(int64_t)D * (j - 1) + d] - p[d];  // compiled with -fmad=false
                    d2 = d == 0 ? dx * dx : d2 + dx * dx;
                }
                if (d2 <= r_sq) {
                    if (c < cap) idx[i * cap + c] = j;
                    ++c;
                }
            }
        } else {
            for (int s = 0; s < NCH; ++s) {
                const int32_t cid = v.node_children[NCH * n0 + s];
                if (cid == -1) continue;
                const int64_t c0 = cid - 1;
                T acc = T(0);
                for (int d = 0; d < D; ++d) {
                    T g = bmin[D * c0 + d] - p[d];
                    g = g > T(0) ? g : T(0);
                    const T g2 = p[d] - bmax[D * c0 + d];
                    g = g2 > g ? g2 : g;
                    acc = d == 0 ? g * g : acc + g * g;
                }
                if (acc <= r_sq && sp < STACK) stack[sp++] = cid;
            }
        }
    }
    counts[i] = (int32_t)c;
}

}  // namespace

// Neighbors of the nq query points `coords_q` ((D, nq) column-major, device)
// among the target points `coords_t` of the view's tree: counts[i] and up to
// cap 1-based indices per query at idx[i * cap ...], in traversal order.
extern "C" int view_consumer_neighbors(const oct_tree_view* v, const void* coords_q, const void* coords_t,
                                       int64_t nq, int32_t* counts, int32_t* idx, int64_t cap, void* stream) {
    if (!v || nq < 0) return 1;
    if (nq == 0) return 0;
    const unsigned blocks = (unsigned)((nq + 127) / 128);
    cudaStream_t s = (cudaStream_t)stream;
    const double r = v->radius;
    if (v->dtype == 0) {
        const float r_sq = (float)r * (float)r;
        if (v->ndims == 3)
            k_view_neighbors<float, 3><<<blocks, 128, 0, s>>>(*v, (const float*)coords_q, (const float*)coords_t, nq,
                                                                r_sq, counts, idx, cap);
        else
            k_view_neighbors<float, 2><<<blocks, 128, 0, s>>>(*v, (const float*)coords_q, (const float*)coords_t, nq,
                                                                r_sq, counts, idx, cap);
    } else {
        const double r_sq = r * r;
        if (v->ndims == 3)
            k_view_neighbors<double, 3><<<blocks, 128, 0, s>>>(*v, (const double*)coords_q, (const double*)coords_t, nq,
                                                                 r_sq, counts, idx, cap);
        else
            k_view_neighbors<double, 2><<<blocks, 128, 0, s>>>(*v, (const double*)coords_q, (const double*)coords_t, nq,
                                                                 r_sq, counts, idx, cap);
    }
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}
