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

}  // namespace

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
