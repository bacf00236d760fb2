// Z-order permutation of user arrays (apply_zsort) and its pullback.
//
// Replaces apply_zsort_cpu! (src/cpu/zsort_cpu.jl:11-32) and
// _apply_zsort_cuda (ext/OctopusCUDAExt.jl:422-432): out[:, i] = in[:, perm[i]]
// for a (F, N) column-major array (each point's F values contiguous) or a
// length-N vector, perm being the tree's Morton order.  The pullback of the
// reference's rrule (ext/OctopusChainRulesCoreExt.jl:65-94) scatters,
// grad[:, perm[i]] = dy[:, i]; it is run here as the equivalent gather
// grad[:, j] = dy[:, iperm[j]] so that the writes stay coalesced.  A point's
// row is moved in the widest word (16, 8, 4, 2 or 1 bytes) that divides the
// row and both base addresses.

#include "internal.h"

namespace oct {

namespace {

template <class W>
__global__ void k_permute_rows(const W* __restrict__ in, W* __restrict__ out, const int32_t* __restrict__ src,
                               int64_t n, int64_t words) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * words) return;
    const int64_t i = t / words;
    const int64_t w = t - i * words;
    const int64_t j = src ? (int64_t)src[i] : i;
    out[t] = in[j * words + w];
}

template <class W>
void launch(const void* in, void* out, const int32_t* src, int64_t n, int64_t row_bytes, cudaStream_t s) {
    const int64_t words = row_bytes / (int64_t)sizeof(W);
    k_permute_rows<W><<<(unsigned)div_up(n * words, 256), 256, 0, s>>>((const W*)in, (W*)out, src, n, words);
}

// A caller's 1-based permutation vector: direction 0 gathers,
// out[:, i] = in[:, perm[i]]; direction 1 scatters, out[:, perm[i]] =
// in[:, i].  An entry outside 1..n is never dereferenced: it sets *bad.
template <class W>
__global__ void k_permute_rows_by(const W* __restrict__ in, W* __restrict__ out, const int32_t* __restrict__ perm,
                                  int64_t n, int64_t words, int direction, int* __restrict__ bad) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * words) return;
    const int64_t i = t / words;
    const int64_t w = t - i * words;
    const int64_t j = (int64_t)perm[i] - 1;
    if (j < 0 || j >= n) {
        if (w == 0) atomicOr(bad, 1);
        return;
    }
    if (direction == 0)
        out[t] = in[j * words + w];
    else
        out[j * words + w] = in[t];
}

template <class W>
void launch_by(const void* in, void* out, const int32_t* perm, int64_t n, int64_t row_bytes, int direction, int* bad,
               cudaStream_t s) {
    const int64_t words = row_bytes / (int64_t)sizeof(W);
    k_permute_rows_by<W><<<(unsigned)div_up(n * words, 256), 256, 0, s>>>((const W*)in, (W*)out, perm, n, words,
                                                                        direction, bad);
}

}  // namespace

int permute_rows(Ctx& ctx, const int32_t* perm, int64_t n, const void* in, void* out, int64_t row_bytes,
                 int direction) {
    if (n < 0 || n > 2147483647LL || row_bytes <= 0 || direction < 0 || direction > 1)
        return set_error(ctx, ERR_ARGUMENT, "permute_rows: bad size, row size or direction");
    if (n == 0) return OK;
    if (!perm || !in || !out || in == out)
        return set_error(ctx, ERR_ARGUMENT, "permute_rows: perm, input and distinct output are required");
    cudaError_t err;
    if ((err = ensure(ctx.dstatus, 8))) return cuda_status(ctx, err, "permute_rows status");
    if (!ctx.total_host) {
        if ((err = cudaMallocHost((void**)&ctx.total_host, 16))) return cuda_status(ctx, err, "pinned status");
    }
    int* bad = ctx.dstatus.as<int>() + 1;  // word 0 is the edge fill's guard word
    if ((err = cudaMemsetAsync(bad, 0, 4, ctx.stream))) return cuda_status(ctx, err, "permute_rows status");
    const uintptr_t a = (uintptr_t)in | (uintptr_t)out | (uintptr_t)row_bytes;
    if (a % 16 == 0) launch_by<uint4>(in, out, perm, n, row_bytes, direction, bad, ctx.stream);
    else if (a % 8 == 0) launch_by<uint2>(in, out, perm, n, row_bytes, direction, bad, ctx.stream);
    else if (a % 4 == 0) launch_by<uint32_t>(in, out, perm, n, row_bytes, direction, bad, ctx.stream);
    else if (a % 2 == 0) launch_by<uint16_t>(in, out, perm, n, row_bytes, direction, bad, ctx.stream);
    else launch_by<uint8_t>(in, out, perm, n, row_bytes, direction, bad, ctx.stream);
    ctx.kernel_launches += 1;
    if ((err = cudaGetLastError())) return cuda_status(ctx, err, "permute_rows launch");
    int32_t* h = reinterpret_cast<int32_t*>(ctx.total_host);
    if ((err = cudaMemcpyAsync(h, bad, 4, cudaMemcpyDeviceToHost, ctx.stream)) || (err = wait_stream(ctx.stream)))
        return cuda_status(ctx, err, "permute_rows");
    if (h[0]) return set_error(ctx, ERR_ARGUMENT, "permute_rows: a permutation entry is outside 1..n (BoundsError)");
    return OK;
}

int zsort_apply(Ctx& ctx, const Tree& t, const void* in, void* out, int64_t n, int64_t row_bytes, int direction) {
    if (!t.built) return set_error(ctx, ERR_STATE, "prepare_zsort: call run! first so the permutation is available");
    if (t.n_clouds) return set_error(ctx, ERR_ARGUMENT, "apply_zsort: not defined for a batched tree");
    if (n != t.n)
        return set_error(ctx, ERR_DIMENSION, "apply_zsort: the array's last axis does not match the point set");
    if (row_bytes <= 0 || direction < 0 || direction > 1)
        return set_error(ctx, ERR_ARGUMENT, "apply_zsort: bad row size or direction");
    if (n == 0) return OK;
    if (!in || !out || in == out) return set_error(ctx, ERR_ARGUMENT, "apply_zsort: input and output must be distinct");
    // direction 0: gather by perm (sorted -> original); 1: gather by its inverse.
    if (direction == 1) {
        const int st = ensure_iperm(ctx, t);
        if (st != OK) return st;
    }
    const int32_t* src = direction == 0 ? t.perm_dev : t.iperm.as<int32_t>();
    const uintptr_t a = (uintptr_t)in | (uintptr_t)out | (uintptr_t)row_bytes;
    if (a % 16 == 0) launch<uint4>(in, out, src, n, row_bytes, ctx.stream);
    else if (a % 8 == 0) launch<uint2>(in, out, src, n, row_bytes, ctx.stream);
    else if (a % 4 == 0) launch<uint32_t>(in, out, src, n, row_bytes, ctx.stream);
    else if (a % 2 == 0) launch<uint16_t>(in, out, src, n, row_bytes, ctx.stream);
    else launch<uint8_t>(in, out, src, n, row_bytes, ctx.stream);
    ctx.kernel_launches += 1;
    return cuda_status(ctx, cudaGetLastError(), "apply_zsort launch");
}

}  // namespace oct
