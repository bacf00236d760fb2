// Fixed-radius traversal and flat-COO edge construction.
//
// Replaces _count_edges_kernel! / _fill_edges_kernel_{3d,2d}! /
// _build_edges_cuda! (ext/OctopusCUDAExt.jl:262-415) and reproduces the CPU
// path's output exactly (src/cpu/edges_cpu.jl:36-247):
//
//   * One warp serves one query group of the query set's tree: a run of
//     sibling leaves with at most 32 points (built with the tree), so the
//     group's box is compact.  The warp walks the target tree once, depth first, with
//     the box of its 32 queries: children are tested in slot order and
//     pushed in that order onto a shared-memory stack, so leaves pop in the
//     same order as the reference's per-query DFS
//     (src/cpu/iterator_cpu.jl:74-116).  The group box test is conservative
//     (box_gap2), so every leaf a single query would visit is visited, and
//     the exact per-pair test d2 = ((dx*dx + dy*dy) + dz*dz) <= r*r decides
//     membership.  Each query therefore emits its neighbors in the
//     reference's order: leaves in DFS order, points in ascending sorted
//     position inside a leaf.  An internal node whose first child slot is
//     empty counts as a leaf in the reference (src/cpu/iterator_cpu.jl:87),
//     so its subtree is walked in ascending slot order, which lists its
//     points in ascending position exactly as the reference's leaf loop.
//   * Leaf points are staged in shared memory and broadcast to the 32 lanes.
//   * counts -> int64 exclusive scan -> fill at the per-query cursor.

#include <algorithm>
#include <type_traits>

#include "internal.h"
#include "scan.cuh"

namespace oct {

constexpr int kEdgeWarps = 4;
constexpr int kEdgeThreads = kEdgeWarps * 32;
constexpr int kStage = 32;  // staged hits per lane, and points per leaf sub-chunk
constexpr int kMultiPop = 4;     // most internal nodes expanded together (the tuned multi_pop is <= this)
constexpr int kMultiLimit = 64;  // stack depth up to which they are
constexpr int kMaxSeg = 16;      // most leaves sharing one chunk (the tuned max_seg is <= this)

// The three passes of k_edges.
enum EdgePass {
    EP_COUNT = 0,   // per-query neighbor counts only
    EP_RECORD = 1,  // counts, plus each query's hit records (up to rec_cap of them)
    EP_FILL = 2,    // the COO at the scanned offsets by a second walk (groups whose records overflowed)
    EP_STATS = 3,   // the count pass with traversal statistics (a diagnostic, oct_edges_traversal_stats)
};

// Traversal statistics of EP_STATS, summed over the launch.
enum TraversalStat {
    TS_GROUPS = 0,     // query groups (warps)
    TS_QUERIES,        // query points
    TS_EXPANSIONS,     // internal-node expansion rounds
    TS_CHILDREN,       // child boxes tested
    TS_CHUNKS,         // leaf chunks staged
    TS_TARGETS,        // target points staged
    TS_STEPS,          // pair-loop steps executed (four targets each)
    TS_PAIR_TESTS,     // query-target distance tests issued (steps x 4 x queries of the group)
    TS_HITS,           // pairs within the radius (self pair excluded when asked)
    TS_CYCLES_TOTAL,   // SM cycles of the warps, summed
    TS_CYCLES_LEAF,    // ... of which in leaf chunks (staging and pair tests)
    TS_CYCLES_PAIRS,   // ... of which in the pair loop
    TS_NUM
};

// A hit record: the sorted position of a leaf's first point (of a leaf's
// 32-point part, for a larger leaf) and the bit mask of its points within the
// radius of one query.  A query's records, in order, list its neighbors in
// the reference's order.
constexpr int kMaxRecords = 65000;  // per query: the record count is stored in 16 bits
constexpr uint16_t kOverflowMark = 0xffff;  // record count of the queries of an overflowed group

// Edge k of the COO: sender = target point t, receiver = query qi at px
// (src/cpu/edges_cpu.jl:200-215: rel_displacement = (x_q - x_t) * inv(r),
// rel_dist_norm = sqrt(d2) * inv(r), 1-based indices).
template <class T, int D>
__device__ __forceinline__ void write_edge(int64_t k, const SPt<T, D>& t, const T* px, int32_t qi, int32_t base,
                                           T inv_r, int32_t* __restrict__ senders, int32_t* __restrict__ receivers,
                                           T* __restrict__ rdisp, T* __restrict__ rdist) {
    senders[k] = t.idx - base + 1;
    if (rdisp == nullptr) return;  // neighbor lists (CSR values) only
    T diff[D];
    const T d2 = dist2<T, D>(t.x, px, diff);
    receivers[k] = qi - base + 1;
#pragma unroll
    for (int d = 0; d < D; ++d) rdisp[(int64_t)D * k + d] = mul_rn(-diff[d], inv_r);
    rdist[k] = mul_rn(sqrt_rn(d2), inv_r);
}

// Starts moving the line holding p into L1 (no value is returned; p must lie
// inside an allocation).
__device__ __forceinline__ void prefetch_l1(const void* p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }

// The per-group traversal starts of a tree searched against itself (not a
// batch), else null (every group starts at the root).
__host__ __forceinline__ const int32_t* own_start(const Tree& q, const Tree& t) {
    return (&q == &t && !t.n_clouds) ? t.gstart.as<int32_t>() : nullptr;
}

// Radius and index base of the point set (cloud) holding sorted position p.
template <class T>
__device__ __forceinline__ void cloud_params(const Batch& bt, int64_t p, T& r2, T& inv_r, int32_t& start_node,
                                             int32_t& base) {
    if (bt.n_clouds) {
        const int c = cloud_of_position(bt, p);
        const double* cp = bt.cparam + (size_t)c * kCloudParams;
        r2 = (T)cp[4];
        inv_r = (T)cp[5];
        start_node = bt.cstart[c];
        base = (int32_t)bt.coff[c];
    }
}

// ocount: in the record pass, ocount[0] counts the groups whose records
// overflowed (those groups are walked again by the fill pass) and ocount[1]
// is the largest record count of a query; in the fill pass, ocount[0] is
// the bounds-guard word.  recs[qpos * rec_cap + r] = record r of the query at
// sorted position qpos, rcount[qpos] = its record count, gflag[g] = 1 when a
// query of group g had more than rec_cap records.
template <class T, int D, int PASS>
__global__ void __launch_bounds__(kEdgeThreads) k_edges(
    const SPt<T, D>* __restrict__ qpts, const int2* __restrict__ qgroups, int64_t n_groups,
    const TNode<T, D>* __restrict__ tnode, int32_t start_node,
    const SPt<T, D>* __restrict__ tpts, int64_t n_tnodes, T r2, T inv_r, int exclude_self,
    int32_t* __restrict__ counts, const int64_t* __restrict__ offsets, int32_t* __restrict__ senders,
    int32_t* __restrict__ receivers, T* __restrict__ rdisp, T* __restrict__ rdist, int* __restrict__ ocount,
    int2* __restrict__ recs, int64_t rec_cap, uint16_t* __restrict__ rcount, uint8_t* __restrict__ gflag, Batch bt,
    unsigned long long* __restrict__ stats, int max_seg, int multi_pop, int nbox, int prefetch,
    const int32_t* __restrict__ gstart) {
    pdl_wait();
    pdl_trigger();
    constexpr bool STAGE = PASS == EP_FILL;
    constexpr bool STATS = PASS == EP_STATS;
    long long st_t0 = 0, st_leaf = 0, st_pairs = 0;
    unsigned long long st_exp = 0, st_children = 0, st_chunks = 0, st_targets = 0, st_steps = 0;
    if constexpr (STATS) st_t0 = clock64();
    // The usual DFS bound, plus the room the multi-node expansions may take.
    constexpr int SD = stack_depth<D>() + kMultiLimit + 8;
    // Stack entries are the pushed node's (a, b) record; bit 31 of a marks
    // ascending-order subtrees (see below).
    __shared__ int2 stack[kEdgeWarps][SD];
    // The internal nodes expanded together: their stack entries and the
    // first lane of each one's children.
    __shared__ int2 snode[kEdgeWarps][kMultiPop];
    __shared__ int soff[kEdgeWarps][kMultiPop + 1];
    // The current leaf chunk, structure of arrays so pairs load as 8 bytes,
    // its leaf segments (first position, first slot; entry nseg holds the
    // point count), and per query lane the chunk slot of its own point
    // ((chunk number << 5) | slot).
    __shared__ __align__(16) T sx[kEdgeWarps][D][32];
    __shared__ int2 sseg[kEdgeWarps][kMaxSeg + 1];
    __shared__ int sself[kEdgeWarps][32];
    // The boxes of the group's nbox runs of 32 / nbox consecutive queries
    // (lo then hi per box): a target is tested only if it is within r of one.
    __shared__ T sbox[kEdgeWarps][4][2 * D];
    // Fill pass: each lane stages the sorted positions of its next hits; a
    // flush writes them as runs of consecutive edges of one query.
    __shared__ int32_t obuf[STAGE ? kEdgeWarps : 1][32][STAGE ? kStage + 1 : 1];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t g = (int64_t)blockIdx.x * kEdgeWarps + w;
    if (g >= n_groups) return;  // warp-uniform
    if (PASS == EP_FILL && recs != nullptr && gflag[g] == 0) return;  // expanded from its records
    const int2 grp = qgroups[g];
    const bool valid = lane < grp.y;
    const int64_t qpos = grp.x + (valid ? lane : 0);  // sorted position of this lane's query
    const SPt<T, D> q = qpts[qpos];
    // A batch searches each cloud in its own tree with its own radius and
    // reports cloud-local indices.
    int32_t base = 0;
    cloud_params<T>(bt, grp.x, r2, inv_r, start_node, base);
    // The group's box.  Plain min/max suffice here (the coordinates are finite,
    // and which zero a tie keeps does not move the box), unlike the build's
    // bounds, which follow Julia's min/max.
    T qlo[D], qhi[D];
#pragma unroll
    for (int d = 0; d < D; ++d) {
        T lo = q.x[d], hi = q.x[d];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        }
        qlo[d] = lo;
        qhi[d] = hi;
    }
    if (nbox > 1) {
        // sub-boxes over runs of 16 (nbox 2) or 8 (nbox 4) lanes; a lane
        // past the group's end holds the group's first point, inside the box
        const int width = 32 / nbox;
#pragma unroll
        for (int d = 0; d < D; ++d) {
            T lo = q.x[d], hi = q.x[d];
            for (int o = width >> 1; o > 0; o >>= 1) {
                lo = jl_min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
                hi = jl_max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
            }
            if ((lane & (width - 1)) == 0) {
                sbox[w][lane / width][d] = lo;
                sbox[w][lane / width][D + d] = hi;
            }
        }
        __syncwarp();
    }
    int64_t cnt = 0;
    int64_t cur = 0, cur_end = 0;
    if (PASS == EP_FILL && valid) {
        cur = offsets[q.idx];
        cur_end = offsets[q.idx + 1];
    }
    const bool self_pair = exclude_self != 0;
    int ocnt = 0;
    int nrec = 0;
    int chunk = 0;  // leaf chunks processed by this warp (warp-uniform)
    sself[w][lane] = -1;
    const int cap = (int)rec_cap;
    int2* myrec = PASS == EP_RECORD ? recs + qpos * rec_cap : nullptr;  // this query's records

    // One query per round: lane e writes the query's e-th staged edge, so a
    // round stores a run of consecutive edges of one segment.  Only the lanes
    // passing `need` are flushed, so each query leaves in long runs.
    auto flush = [&](bool need) {
        __syncwarp();
        unsigned busy = __ballot_sync(0xffffffffu, need && ocnt > 0);
        while (busy) {
            const int ql = __ffs(busy) - 1;
            busy &= busy - 1;
            const int nql = __shfl_sync(0xffffffffu, ocnt, ql);
            const long long cq = __shfl_sync(0xffffffffu, (long long)cur, ql);
            const long long ce = __shfl_sync(0xffffffffu, (long long)cur_end, ql);
            const int32_t qi = __shfl_sync(0xffffffffu, q.idx, ql);
            T px[D];
#pragma unroll
            for (int d = 0; d < D; ++d) px[d] = __shfl_sync(0xffffffffu, q.x[d], ql);
            if (lane < nql) {
                const int64_t k = cq + lane;
                if (k < ce)
                    write_edge<T, D>(k, tpts[obuf[w][ql][lane]], px, qi, base, inv_r, senders, receivers, rdisp,
                                     rdist);
                else
                    atomicOr(ocount, 1);  // never taken when count and fill agree
            }
        }
        if (need) {
            cur += ocnt;
            ocnt = 0;
        }
        __syncwarp();
    };

    int sp = 0;
    const int32_t gs = gstart ? gstart[g] : -1;
    if (gs >= 0) {
        // the group's own start node (k_groups): its subtree holds every
        // neighbor, and the group lies inside it
        const TNode<T, D> sn = tnode[gs & 0x3fffffff];
        if (lane == 0) stack[w][0] = make_int2(sn.a | ((gs >> 30) & 1 ? (int32_t)0x80000000 : 0), sn.b);
        sp = 1;
    } else if (n_tnodes > 0) {
        const TNode<T, D> root = tnode[start_node];
        if (box_gap2<T, D>(qlo, qhi, root.lo, root.hi) <= r2) {
            if (lane == 0) stack[w][0] = make_int2(root.a, root.b);
            sp = 1;
        }
    }
    __syncwarp();
    while (sp > 0) {
        const int2 ent = stack[w][--sp];
        const int32_t na = ent.x & 0x7fffffff;
        const int32_t nb = ent.y;
        if (nb > 0) {
            // Leaves: every (query, point) pair, points in ascending position
            // within a leaf, hits as a bit mask.  Leaves popped one after
            // another (the next stack entries, so the DFS order is kept)
            // share one chunk of at most kStage points as consecutive
            // segments; a leaf of more than kStage points is cut into chunks.
            for (int32_t c0 = 0; c0 < nb; c0 += kStage) {
                long long st_c0 = 0;
                if constexpr (STATS) st_c0 = clock64();
                __syncwarp();  // every lane is done with the previous chunk's segment table
                int total = min(kStage, nb - c0);
                int nseg = 1;
                if (lane == 0) sseg[w][0] = make_int2(na + c0, 0);
                if (nb <= kStage) {
                    while (sp > 0 && nseg < max_seg) {
                        const int2 nx = stack[w][sp - 1];
                        if (nx.y <= 0 || total + nx.y > kStage) break;
                        --sp;
                        if (lane == 0) sseg[w][nseg] = make_int2(nx.x & 0x7fffffff, total);
                        total += nx.y;
                        ++nseg;
                    }
                }
                if (lane == 0) sseg[w][nseg] = make_int2(0, total);
                const int mp = (total + 3) & ~3;  // padded to whole pairs of pairs with +inf points
                ++chunk;
                __syncwarp();
                // A target farther than r from the group's box can be no
                // query's neighbor (box_gap2 never exceeds a point distance):
                // the pair loop skips the steps whose targets all are.
                bool near = false;
                if (lane < total) {
                    int k = 0;
                    while (sseg[w][k + 1].y <= lane) ++k;
                    const int32_t pos = sseg[w][k].x + (lane - sseg[w][k].y);
                    const SPt<T, D> t = tpts[pos];
#pragma unroll
                    for (int d = 0; d < D; ++d) sx[w][d][lane] = t.x[d];
                    if (nbox == 1) {
                        near = box_gap2<T, D>(qlo, qhi, t.x, t.x) <= r2;
                    } else {
                        for (int b = 0; b < nbox && !near; ++b)
                            near = box_gap2<T, D>(&sbox[w][b][0], &sbox[w][b][D], t.x, t.x) <= r2;
                    }
                    if (self_pair) {  // query and target are the same tree: the group's own points
                        const int64_t sl = pos - grp.x;
                        if (sl >= 0 && sl < grp.y) sself[w][sl] = (chunk << 5) | lane;
                    }
                } else if (lane < mp) {
#pragma unroll
                    for (int d = 0; d < D; ++d) sx[w][d][lane] = T(INFINITY);
                }
                const unsigned keep = __ballot_sync(0xffffffffu, near);
                __syncwarp();
                if (prefetch && c0 + kStage >= nb) {
                    // The next chunk's points (the leaves now at the stack top)
                    // start their way into L1 while this chunk's pairs are tested.
                    int acc = 0, ppos = -1;
                    for (int j = sp - 1; j >= 0 && acc < 32; --j) {
                        const int2 nx = stack[w][j];
                        if (nx.y <= 0) break;
                        if (lane >= acc && lane < acc + nx.y) ppos = (nx.x & 0x7fffffff) + (lane - acc);
                        acc += nx.y;
                    }
                    if (ppos >= 0) prefetch_l1(tpts + ppos);
                }
                unsigned hm = 0;
                long long st_p0 = 0;
                if constexpr (STATS) {
                    st_p0 = clock64();
                    ++st_chunks;
                    st_targets += total;
                    st_steps += std::is_same<T, float>::value
                                    ? __popc((keep | keep >> 1 | keep >> 2 | keep >> 3) & 0x11111111u)
                                    : __popc(keep);
                }
                if constexpr (std::is_same<T, float>::value) {
                    unsigned long long P[D];
#pragma unroll
                    for (int d = 0; d < D; ++d) P[d] = pack2(q.x[d], q.x[d]);
                    // one bit per step of four targets with a target kept
                    const unsigned steps = (keep | keep >> 1 | keep >> 2 | keep >> 3) & 0x11111111u;
                    for (unsigned km = steps; km; km &= km - 1) {
                        const int j = __ffs(km) - 1;
                        // Four targets per step, two per packed operation:
                        // packed differences and squares, scalar sums
                        // ((dx*dx + dy*dy) + dz*dz) per element.  The sums stay
                        // scalar: packed add.rn.f32x2 sums after the packed
                        // squares changed results (8 of 1,547,624,876 edges of
                        // the 4M-point 2D set), as a fused multiply-add would.
                        float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
#pragma unroll
                        for (int d = 0; d < D; ++d) {
                            const unsigned long long* px = reinterpret_cast<const unsigned long long*>(&sx[w][d][j]);
                            const unsigned long long da = sub2_rn(px[0], P[d]);
                            const unsigned long long db = sub2_rn(px[1], P[d]);
                            const unsigned long long qa = mul2_rn(da, da);
                            const unsigned long long qb = mul2_rn(db, db);
                            s0 = (d == 0) ? lo2(qa) : __fadd_rn(s0, lo2(qa));
                            s1 = (d == 0) ? hi2(qa) : __fadd_rn(s1, hi2(qa));
                            s2 = (d == 0) ? lo2(qb) : __fadd_rn(s2, lo2(qb));
                            s3 = (d == 0) ? hi2(qb) : __fadd_rn(s3, hi2(qb));
                        }
                        hm |= ((s0 <= r2 ? 1u : 0u) | (s1 <= r2 ? 2u : 0u) | (s2 <= r2 ? 4u : 0u) |
                               (s3 <= r2 ? 8u : 0u)) << j;
                    }
                } else {
                    for (unsigned km = keep; km; km &= km - 1) {
                        const int j = __ffs(km) - 1;
                        T t[D], diff[D];
#pragma unroll
                        for (int d = 0; d < D; ++d) t[d] = sx[w][d][j];
                        hm |= (dist2<T, D>(t, q.x, diff) <= r2 ? 1u : 0u) << j;
                    }
                }
                if constexpr (STATS) st_pairs += clock64() - st_p0;
                if (!valid) hm = 0;
                if (self_pair) {
                    const int v = sself[w][lane];
                    if ((v >> 5) == chunk) hm &= ~(1u << (v & 31));
                }
                const int nh = __popc(hm);
                cnt += nh;
                if (PASS == EP_RECORD) {
                    // One record per leaf segment with hits, in pop order.
                    if (__any_sync(0xffffffffu, hm != 0)) {
                        for (int k = 0; k < nseg; ++k) {
                            const int2 sg = sseg[w][k];
                            const int len = sseg[w][k + 1].y - sg.y;
                            const unsigned sub = (hm >> sg.y) & (0xffffffffu >> (32 - len));
                            if (sub != 0u && nrec < cap) myrec[nrec] = make_int2(sg.x, (int32_t)sub);
                            nrec += sub != 0u;
                        }
                    }
                } else if (STAGE) {
                    if (__any_sync(0xffffffffu, ocnt + nh > kStage)) flush(ocnt + nh > kStage);
                    for (int k = 0; k < nseg; ++k) {
                        const int2 sg = sseg[w][k];
                        const int len = sseg[w][k + 1].y - sg.y;
                        unsigned sub = (hm >> sg.y) & (len >= 32 ? 0xffffffffu : ((1u << len) - 1u));
                        while (sub) {
                            const int j = __ffs(sub) - 1;
                            sub &= sub - 1;
                            obuf[w][lane][ocnt++] = sg.x + j;
                        }
                    }
                }
                if constexpr (STATS) st_leaf += clock64() - st_c0;
            }
        } else {
            // Internal nodes.  The popped node and up to kMultiPop - 1 further
            // internal entries at the stack top (the nodes the DFS expands
            // next) have their children box-tested together, one lane per
            // child; each node's passing children are pushed as a block, the
            // first node's on top, so the visiting order is unchanged.  Only
            // while the stack stays at most kMultiLimit deep: beyond it the
            // usual single expansions bound the depth.
            // The reference scans an internal node whose first child slot is
            // empty as one leaf, in ascending position order
            // (src/cpu/iterator_cpu.jl:87-101).  Below such a node the
            // children are therefore visited in ascending slot order.
            int nnodes = 1, totc = __popc((unsigned)(-nb));
            if (lane == 0) {
                snode[w][0] = ent;
                soff[w][0] = 0;
            }
            while (nnodes < multi_pop && sp > 0) {
                const int2 nx = stack[w][sp - 1];
                if (nx.y > 0) break;
                const int c = __popc((unsigned)(-nx.y));
                if (totc + c > 32 || sp - 1 + totc + c > kMultiLimit) break;
                --sp;
                if (lane == 0) {
                    snode[w][nnodes] = nx;
                    soff[w][nnodes] = totc;
                }
                totc += c;
                ++nnodes;
            }
            if (lane == 0) soff[w][nnodes] = totc;
            if constexpr (STATS) {
                ++st_exp;
                st_children += totc;
            }
            __syncwarp();
            int j = 0;
            if (lane < totc)
                while (soff[w][j + 1] <= lane) ++j;
            const int2 nd = snode[w][j];
            const unsigned slots = (unsigned)(-nd.y);
            const bool casc = nd.x < 0 || !(slots & 1u);
            const int o = soff[w][j], o2 = soff[w][j + 1];
            bool pass = false;
            int2 rec = make_int2(0, 0);
            if (lane < totc) {
                const TNode<T, D> c = tnode[(nd.x & 0x7fffffff) + (lane - o)];
                pass = box_gap2<T, D>(qlo, qhi, c.lo, c.hi) <= r2;
                rec = make_int2(c.a | (casc ? (int32_t)0x80000000 : 0), c.b);
            }
            const unsigned m = __ballot_sync(0xffffffffu, pass);
            if (pass) {
                const unsigned upto = o2 >= 32 ? 0xffffffffu : ((1u << o2) - 1u);  // lanes of nodes <= j
                const unsigned mine = m & upto & ~((1u << o) - 1u);
                const int deeper = __popc(m & ~upto);  // passing children of the later nodes, below
                const int np = __popc(mine);
                const int rk = __popc(mine & lanemask_lt());
                stack[w][sp + deeper + (casc ? np - 1 - rk : rk)] = rec;
            }
            sp += __popc(m);
            __syncwarp();
            if (prefetch && sp > 0) {
                // what the next pop reads: an internal node's children, or a leaf's points
                const int2 nx = stack[w][sp - 1];
                const int32_t a = nx.x & 0x7fffffff;
                if (nx.y <= 0) {
                    if (lane < __popc((unsigned)(-nx.y))) prefetch_l1(tnode + a + lane);
                } else if (lane < nx.y) {
                    prefetch_l1(tpts + a + lane);
                }
            }
        }
    }
    if (STAGE) flush(true);
    if (PASS != EP_FILL && valid) counts[q.idx] = (int32_t)cnt;
    if constexpr (STATS) {
        const unsigned long long hits = warp_sum((unsigned long long)cnt);
        const int nv = __popc(__ballot_sync(0xffffffffu, valid));
        if (lane == 0) {
            const unsigned long long v[TS_NUM] = {1ull, (unsigned long long)nv, st_exp, st_children, st_chunks,
                                                  st_targets, st_steps, 4ull * st_steps * (unsigned long long)nv, hits,
                                                  (unsigned long long)(clock64() - st_t0), (unsigned long long)st_leaf,
                                                  (unsigned long long)st_pairs};
#pragma unroll
            for (int k = 0; k < TS_NUM; ++k) atomicAdd(stats + k, v[k]);
        }
    }
    if (PASS == EP_RECORD) {
        const bool over = __any_sync(0xffffffffu, nrec > cap);
        if (valid) rcount[qpos] = over ? kOverflowMark : (uint16_t)nrec;
        int mx = nrec;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if (lane == 0) {
            gflag[g] = over ? 1 : 0;
            if (over) atomicAdd(ocount, 1);
            // The maximum settles after a few groups: most groups only read it.
            if (mx > __ldcg(ocount + 1)) atomicMax(ocount + 1, mx);
        }
    }
}

// Position (0..31) of the k-th set bit (k from 0) of m; k < popc(m).
__device__ __forceinline__ int kth_set_bit(unsigned m, int k) {
    int pos = 0;
    int c = __popc(m & 0xffffu);
    if (k >= c) { k -= c; m >>= 16; pos += 16; }
    c = __popc(m & 0xffu);
    if (k >= c) { k -= c; m >>= 8; pos += 8; }
    c = __popc(m & 0xfu);
    if (k >= c) { k -= c; m >>= 4; pos += 4; }
    c = __popc(m & 0x3u);
    if (k >= c) { k -= c; m >>= 2; pos += 2; }
    c = (int)(m & 1u);
    if (k >= c) pos += 1;
    return pos;
}

// Fill pass from the records with direct stores, in original index order
// (the default fill; k_expand below writes through bulk copies instead, a
// tuned alternative).  Warp v owns queries 32v .. 32v+31, one per lane; their
// records, query after query, form one flat list, and so do their edges, in
// the same order (a record's hits are consecutive edges of its query).  The
// warp loads the records 32 at a time (one per lane), scans their hit counts,
// lists each edge's (record lane, bit) in a per-warp shared-memory table (each
// record lane writes its hits at its edges' slots), and writes the batch's
// edges 32 at a time, one per lane:
//   * a record's query: the queries whose records reach into the 32-record
//     window set one bit each at their first record in the window (the one
//     running into the window at bit 0), so the query of record l is the
//     (popc of the bits up to l)-th of them (ballot, reduce-or, popc; no search);
//   * an edge's target is its record's leaf position plus the bit from the
//     table; its query's coordinates, index and radius come from the query's
//     lane by shuffles.
// Edge f of the flat list goes to COO slot kb[q] + f of its query q (slots
// relative to the warp's first slot).  Queries of an
// overflowed group (record count kOverflowMark) are left to the walking fill.
constexpr int kDirectWarps = 4;

template <class T, int D>
__global__ void __launch_bounds__(kDirectWarps * 32, sizeof(T) == 4 ? 10 : 1) k_expand_direct(
    int64_t nq, const int32_t* __restrict__ iperm, const SPt<T, D>* __restrict__ qpts,
    const SPt<T, D>* __restrict__ tpts, const int64_t* __restrict__ offsets, const int2* __restrict__ recs,
    int64_t rec_cap, const uint16_t* __restrict__ rcount, T inv_r, int32_t* __restrict__ senders,
    int32_t* __restrict__ receivers, T* __restrict__ rdisp, T* __restrict__ rdist, Batch bt) {
    pdl_wait();
    pdl_trigger();
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    // per warp: (record lane << 5 | bit) of each edge of the current record batch
    __shared__ uint16_t sedge[kDirectWarps][32 * 32];
    uint16_t* se = sedge[threadIdx.x >> 5];
    const int64_t i0 = ((int64_t)blockIdx.x * kDirectWarps + (threadIdx.x >> 5)) * 32;
    if (i0 >= nq) return;  // warp-uniform
    const int64_t i = i0 + lane;
    const bool valid = i < nq;
    const int64_t K0 = offsets[i0];  // the warp's first COO slot
    const int32_t qp = valid ? iperm[i] : 0;
    int nr = valid ? rcount[qp] : 0;
    int ne = 0;
    long long krel = 0;
    if (valid && nr != kOverflowMark) {
        const int64_t c0 = offsets[i];
        ne = (int)(offsets[i + 1] - c0);
        krel = c0 - K0;
    } else {
        nr = 0;
    }
    const SPt<T, D> q = qpts[qp];
    T r2 = T(0), ir = inv_r;
    int32_t start_node = 0, base = 0;
    cloud_params<T>(bt, qp, r2, ir, start_node, base);
    const int32_t qi = q.idx - base + 1;
    const bool feat = rdisp != nullptr;  // false: neighbor lists (CSR values) only
    const unsigned le = full >> (31 - lane);  // lanes up to this one
    // flat record and edge ranges of the queries
    int rinc = nr, einc = ne;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int a = __shfl_up_sync(full, rinc, o);
        const int b = __shfl_up_sync(full, einc, o);
        if (lane >= o) {
            rinc += a;
            einc += b;
        }
    }
    const int rexc = rinc - nr;
    const long long kb = krel - (einc - ne);  // slot of flat edge f of this query: kb + f
    const int R = __shfl_sync(full, rinc, 31);
    int32_t* snd_w = senders + K0;
    int32_t* rcv_w = receivers + K0;
    T* dist_w = rdist + K0;
    T* disp_w = feat ? rdisp + D * K0 : nullptr;
    int fdone = 0;  // flat edges of the earlier record batches
    for (int rb = 0; rb < R; rb += 32) {
        // record rho = rb + lane and its query
        // (queries without records set no bit, so the k-th bit belongs to the
        // k-th query lane that reaches into the window)
        const bool qin = nr > 0 && rexc < rb + 32 && rinc > rb;
        const unsigned qm = __ballot_sync(full, qin);
        const unsigned qs = __reduce_or_sync(full, qin ? 1u << max(rexc - rb, 0) : 0u);
        const int rq = kth_set_bit(qm, __popc(qs & le) - 1);  // query lane of this lane's record
        const int32_t rqp = __shfl_sync(full, qp, rq);
        const int rqx = __shfl_sync(full, rexc, rq);
        const int rho = rb + lane;
        int2 rec = make_int2(0, 0);
        if (rho < R) rec = recs[(int64_t)rqp * rec_cap + (rho - rqx)];
        const int c = __popc((unsigned)rec.y);
        int incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int a = __shfl_up_sync(full, incl, o);
            if (lane >= o) incl += a;
        }
        const int excl = incl - c;
        const int tot = __shfl_sync(full, incl, 31);
        // each record lane lists its hits at its edges' slots
        __syncwarp();  // the previous batch's table has been read
        {
            unsigned mb = (unsigned)rec.y;
            for (int k = excl; mb; ++k) {
                se[k] = (uint16_t)((lane << 5) | (__ffs(mb) - 1));
                mb &= mb - 1;
            }
        }
        __syncwarp();
        // two windows per round, both gathers in flight before either is written
        for (int w0 = 0; w0 < tot; w0 += 64) {
            int32_t tpos[2];
            long long slot[2];
            int eqw[2];
            bool ok[2];
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const int wu = w0 + 32 * u;
                const int e = wu + lane;
                const int sv = e < tot ? se[e] : 0;
                const int ri = sv >> 5;  // this lane's record
                const int rx = __shfl_sync(full, rec.x, ri);
                const int eq = __shfl_sync(full, rq, ri);  // this lane's query
                slot[u] = __shfl_sync(full, kb, eq) + (fdone + wu + lane);
                const int qend = __shfl_sync(full, einc, eq);  // flat end of the query's edges
                ok[u] = e < tot && fdone + e < qend;  // the second always holds when records and counts agree
                tpos[u] = ok[u] ? rx + (sv & 31) : 0;
                eqw[u] = eq;
            }
            SPt<T, D> t[2];
#pragma unroll
            for (int u = 0; u < 2; ++u)
                if (ok[u]) t[u] = tpts[tpos[u]];
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const int eq = eqw[u];
                const int32_t bq = __shfl_sync(full, base, eq);
                if (feat) {
                    const int32_t qiq = __shfl_sync(full, qi, eq);
                    const T iv = __shfl_sync(full, ir, eq);
                    T px[D];
#pragma unroll
                    for (int d = 0; d < D; ++d) px[d] = __shfl_sync(full, q.x[d], eq);
                    if (ok[u]) {
                        T diff[D];
                        const T d2 = dist2<T, D>(t[u].x, px, diff);
                        snd_w[slot[u]] = t[u].idx - bq + 1;
                        rcv_w[slot[u]] = qiq;
                        dist_w[slot[u]] = mul_rn(sqrt_rn(d2), iv);
#pragma unroll
                        for (int d = 0; d < D; ++d) disp_w[(long long)D * slot[u] + d] = mul_rn(-diff[d], iv);
                    }
                } else if (ok[u]) {
                    snd_w[slot[u]] = t[u].idx - bq + 1;
                }
            }
        }
        fdone += tot;
    }
}

// Fill pass from the records, in original index order.  Warp v writes the
// edges of queries 32v .. 32v+31, which own one contiguous range [K0, K1) of
// the COO, query after query, each query's edges in record order.  The warp
// takes the records of all its queries as one flat list, 32 per round (one per
// lane, the record's query found by a binary search of the queries' record
// counts), scans their hit counts, and then writes the round's hits with the
// lanes on consecutive hits, two per lane in flight: each lane finds its hit's
// record by a binary search of the scanned counts (shuffles), its point as the
// k-th set bit of the record's mask, and its query's coordinates, index and
// radius by shuffles from the query's lane.
//
// Output goes through a per-warp ring of NCH chunks of CHUNK edges in shared
// memory, one array per COO array, in the COO's own layout; a completed chunk
// is written to global memory by 1-D bulk copies (cp.async.bulk, issued by
// lane 0), so the stores leave the load/store pipe.  Ring slot s holds COO
// edge k with s = (k - base) mod RING, base = K0 rounded down to a multiple of
// 4: a bulk copy starts at an edge index that is a multiple of 4, which makes
// every source and destination address a multiple of 16 bytes (4-byte and
// 8-byte elements, D values per edge for rel_displacement) given 16-byte
// aligned output arrays, and every size a multiple of 16.  The at most three
// edges at each end of the warp's range that do not fill an aligned group of
// four are stored by lanes.  A warp with a query whose records overflowed
// (left to the walking fill), or with unaligned outputs, stores every edge
// from registers instead.
constexpr int kFillWarps = 4;

__device__ __forceinline__ void bulk_store(void* gdst, const void* ssrc, uint32_t bytes) {
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(ssrc);
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gdst), "r"(s), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void bulk_wait_read() {
    asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// Orders this thread's shared-memory writes before later bulk-copy reads.
__device__ __forceinline__ void fence_smem_to_bulk() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }


// Shared-memory bytes of one warp's ring of `ring` edges.
template <class T, int D, bool FEAT>
__host__ __device__ constexpr size_t fill_ring_bytes(int ring) {
    return FEAT ? (size_t)ring * (8 + (D + 1) * sizeof(T)) : (size_t)ring * 4;
}

template <class T, int D, bool FEAT, int CHUNK, int NCH>
__global__ void __launch_bounds__(kFillWarps * 32) k_expand(
    int64_t nq, const int32_t* __restrict__ iperm, const SPt<T, D>* __restrict__ qpts,
    const SPt<T, D>* __restrict__ tpts, const int64_t* __restrict__ offsets, const int2* __restrict__ recs,
    int64_t rec_cap, const uint16_t* __restrict__ rcount, T inv_r, int32_t* __restrict__ senders,
    int32_t* __restrict__ receivers, T* __restrict__ rdisp, T* __restrict__ rdist, Batch bt, int bulk_ok) {
    constexpr int RING = CHUNK * NCH;
    constexpr int U = 2;                                  // hits per lane in flight
    constexpr int SUB = 32 * U;                           // hits written per sub-round
    constexpr int SPAN = (SUB - 1 + CHUNK - 1) / CHUNK;   // chunk boundaries a sub-round may cross
    static_assert(CHUNK % 32 == 0 && (RING & (RING - 1)) == 0 && NCH - 1 - SPAN >= 0, "ring shape");
    constexpr unsigned FULL = 0xffffffffu;
    extern __shared__ __align__(128) unsigned char fill_smem[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t i0 = ((int64_t)blockIdx.x * kFillWarps + w) * 32;
    if (i0 >= nq) return;  // warp-uniform
    unsigned char* wsm = fill_smem + (size_t)w * fill_ring_bytes<T, D, FEAT>(RING);
    int32_t* r_snd = reinterpret_cast<int32_t*>(wsm);
    int32_t* r_rcv = r_snd + RING;
    T* r_dist = reinterpret_cast<T*>(r_rcv + RING);
    T* r_disp = r_dist + RING;

    // Lane j: query i0 + j.
    const int64_t i = i0 + lane;
    const bool valid = i < nq;
    const int nval = nq - i0 < 32 ? (int)(nq - i0) : 32;
    const int32_t qp = valid ? iperm[i] : 0;
    int nr = valid ? rcount[qp] : 0;
    const bool over = valid && nr == kOverflowMark;
    const long long k0 = valid ? offsets[i] : 0;
    const long long kn = valid ? offsets[i + 1] : 0;
    int ne = (int)(kn - k0);
    if (over) {  // written by the walking fill
        nr = 0;
        ne = 0;
    }
    const SPt<T, D> q = qpts[qp];
    T r2 = T(0), ir = inv_r;
    int32_t start_node = 0, base = 0;
    cloud_params<T>(bt, qp, r2, ir, start_node, base);
    const int32_t qi = q.idx - base + 1;
    // record and hit prefixes over the queries
    int rincl = nr, eincl = ne;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int a = __shfl_up_sync(FULL, rincl, o);
        const int b = __shfl_up_sync(FULL, eincl, o);
        if (lane >= o) {
            rincl += a;
            eincl += b;
        }
    }
    const int rexcl = rincl - nr;
    const int total_r = __shfl_sync(FULL, rincl, 31);
    // COO index of this query's flat hit 0 (flat hits count only the queries
    // written here): hit F of query j is COO edge kq_j + F
    const long long kq = k0 - (eincl - ne);
    const long long K0 = __shfl_sync(FULL, k0, 0);
    const long long K1 = __shfl_sync(FULL, kn, nval - 1);
    const bool bulk = bulk_ok && !__any_sync(FULL, over) && K1 - K0 >= 32;
    const long long kbase = K0 & ~3LL;  // ring slot 0 <-> COO edge kbase (mod RING)
    long long next_flush = 0;           // next ring chunk to write out (chunk c: [kbase + c*CHUNK, +CHUNK))
    long long cur_chunk = -1;           // highest chunk written so far

    // Writes out the chunks that end at or before `upto` (all that remain of
    // the range when `last`): the aligned part by bulk copies (one group per
    // chunk), the unaligned ends by lanes.
    auto flush = [&](long long upto, bool last) {
        while (true) {
            const long long cs = kbase + next_flush * CHUNK, ce = cs + CHUNK;
            if (cs >= K1 || (ce > upto && !last)) break;
            const long long lo = cs > K0 ? cs : K0, hi = ce < K1 ? ce : K1;
            long long a = (lo + 3) & ~3LL;
            if (a > hi) a = hi;
            const long long b = a + ((hi - a) & ~3LL);
            if (lane == 0) {
                if (b > a) {
                    const int sl = (int)((a - kbase) & (RING - 1));
                    const uint32_t m = (uint32_t)(b - a);
                    bulk_store(senders + a, r_snd + sl, 4u * m);
                    if (FEAT) {
                        bulk_store(receivers + a, r_rcv + sl, 4u * m);
                        bulk_store(rdist + a, r_dist + sl, (uint32_t)sizeof(T) * m);
                        bulk_store(rdisp + (long long)D * a, r_disp + D * sl, (uint32_t)(D * sizeof(T)) * m);
                    }
                }
                bulk_commit();  // one group per chunk, empty or not
            }
            // [lo, a) and [b, hi): at most three edges each
            const long long k = lane < 4 ? lo + lane : b + (lane - 4);
            if ((lane < 4 && k < a) || (lane >= 4 && lane < 8 && k < hi)) {
                const int sl = (int)((k - kbase) & (RING - 1));
                senders[k] = r_snd[sl];
                if (FEAT) {
                    receivers[k] = r_rcv[sl];
                    rdist[k] = r_dist[sl];
#pragma unroll
                    for (int d = 0; d < D; ++d) rdisp[(long long)D * k + d] = r_disp[D * sl + d];
                }
            }
            ++next_flush;
        }
    };

    int fbase = 0;  // flat hits of the earlier record rounds
    for (int r0 = 0; r0 < total_r; r0 += 32) {
        // record r0 + lane and its query: the last query whose first record is <= it
        const int rho = r0 + lane;
        int jr = 0;
#pragma unroll
        for (int st = 16; st > 0; st >>= 1) {
            const int v = __shfl_sync(FULL, rexcl, jr + st);
            if (v <= rho) jr += st;
        }
        const int32_t qpr = __shfl_sync(FULL, qp, jr);
        const int rx0 = __shfl_sync(FULL, rexcl, jr);
        int2 rec = make_int2(0, 0);
        if (rho < total_r) rec = recs[(int64_t)qpr * rec_cap + (rho - rx0)];
        const int p = __popc((unsigned)rec.y);
        int hincl = p;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int a = __shfl_up_sync(FULL, hincl, o);
            if (lane >= o) hincl += a;
        }
        const int hexcl = hincl - p;
        const int tot = __shfl_sync(FULL, hincl, 31);
        for (int e0 = 0; e0 < tot; e0 += SUB) {
            const int cnt = min(SUB, tot - e0);
            if (bulk) {
                // the sub-round writes COO edges [K0 + fbase + e0, + cnt): its
                // last chunk reuses the slots of that chunk minus NCH
                const long long c = (K0 + fbase + e0 + cnt - 1 - kbase) / CHUNK;
                if (c > cur_chunk) {
                    if (c >= NCH) {
                        if (lane == 0) bulk_wait_read<NCH - 1 - SPAN>();
                        __syncwarp();
                    }
                    cur_chunk = c;
                }
            }
            SPt<T, D> tp[U];
            int jq[U], tpos[U];
            long long kk[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int e = e0 + 32 * u + lane;
                int r = 0;
#pragma unroll
                for (int st = 16; st > 0; st >>= 1) {
                    const int v = __shfl_sync(FULL, hexcl, r + st);
                    if (v <= e) r += st;
                }
                const unsigned m = (unsigned)__shfl_sync(FULL, rec.y, r);
                const int rx = __shfl_sync(FULL, rec.x, r);
                const int er = __shfl_sync(FULL, hexcl, r);
                jq[u] = __shfl_sync(FULL, jr, r);
                kk[u] = __shfl_sync(FULL, kq, jq[u]) + fbase + e;
                tpos[u] = 0;
                if (e < tot) {
                    tpos[u] = rx + kth_set_bit(m, e - er);
                    tp[u] = tpts[tpos[u]];
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int e = e0 + 32 * u + lane;
                T px[D];
#pragma unroll
                for (int d = 0; d < D; ++d) px[d] = __shfl_sync(FULL, q.x[d], jq[u]);
                const T irq = __shfl_sync(FULL, ir, jq[u]);
                const int32_t bq = __shfl_sync(FULL, base, jq[u]);
                const int32_t qiq = __shfl_sync(FULL, qi, jq[u]);
                if (e >= tot) continue;
                const long long k = kk[u];
                const int32_t snd = tp[u].idx - bq + 1;
                T dv[D], dist = T(0);
                if (FEAT) {
                    T diff[D];
                    const T d2 = dist2<T, D>(tp[u].x, px, diff);
                    dist = mul_rn(sqrt_rn(d2), irq);
#pragma unroll
                    for (int d = 0; d < D; ++d) dv[d] = mul_rn(-diff[d], irq);
                }
                if (bulk) {
                    const int sl = (int)((k - kbase) & (RING - 1));
                    r_snd[sl] = snd;
                    if (FEAT) {
                        r_rcv[sl] = qiq;
                        r_dist[sl] = dist;
#pragma unroll
                        for (int d = 0; d < D; ++d) r_disp[D * sl + d] = dv[d];
                    }
                } else {
                    senders[k] = snd;
                    if (FEAT) {
                        receivers[k] = qiq;
                        rdist[k] = dist;
#pragma unroll
                        for (int d = 0; d < D; ++d) rdisp[(long long)D * k + d] = dv[d];
                    }
                }
            }
            if (bulk) {
                fence_smem_to_bulk();
                __syncwarp();
                flush(K0 + fbase + e0 + cnt, false);
            }
        }
        fbase += tot;
    }
    if (bulk) {
        __syncwarp();
        flush(K1, true);
        if (lane == 0) bulk_wait_all();
    }
}

// Per-thread reference-order DFS for a handful of query points (the
// get_neighborlist / for_each_neighbor accessors, src/api.jl:282-292 and
// src/cpu/iterator_cpu.jl:245-263).  No self filter.
template <class T, int D>
__global__ void k_neighbors_of(const T* __restrict__ qcoords, int64_t nsel, const TNode<T, D>* __restrict__ tnode,
                               const SPt<T, D>* __restrict__ tpts, int64_t n_tnodes, T r2,
                               int32_t* __restrict__ out_counts, int32_t* __restrict__ out_idx, int64_t cap) {
    constexpr int SD = stack_depth<D>();
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsel) return;
    T p[D];
#pragma unroll
    for (int d = 0; d < D; ++d) p[d] = qcoords[(int64_t)D * s + d];
    int32_t stack[SD];
    int sp = 0;
    int64_t c = 0;
    if (n_tnodes > 0) stack[sp++] = 0;
    while (sp > 0) {
        const int32_t ent = stack[--sp];
        const int32_t nid = ent & 0x7fffffff;
        const bool asc = ent < 0;
        const TNode<T, D> nd = tnode[nid];
        if (box_gap2<T, D>(p, p, nd.lo, nd.hi) > r2) continue;
        if (nd.b > 0) {
            for (int32_t k = nd.a; k < nd.a + nd.b; ++k) {
                const SPt<T, D> t = tpts[k];
                T diff[D];
                if (dist2<T, D>(t.x, p, diff) <= r2) {
                    if (c < cap) out_idx[s * cap + c] = t.idx + 1;
                    ++c;
                }
            }
        } else {
            const unsigned slots = (unsigned)(-nd.b);
            const bool casc = asc || !(slots & 1u);
            const int nc = __popc(slots);
            int pushed[Dims<D>::nch];
            int np = 0;
            for (int j = 0; j < nc; ++j) {
                const TNode<T, D> ch = tnode[nd.a + j];
                if (box_gap2<T, D>(p, p, ch.lo, ch.hi) <= r2) pushed[np++] = nd.a + j;
            }
            for (int j = 0; j < np; ++j)
                stack[sp++] = casc ? (pushed[np - 1 - j] | (int32_t)0x80000000) : pushed[j];
        }
    }
    out_counts[s] = (int32_t)c;
}

namespace {

// Hit records per query for the next count: 32 to start, then 1.25x the
// largest record count of the last count (at most kMaxRecords), within a
// budget of 4 GiB or 8 bytes per edge of the last count (a third of the
// COO's own size), whichever is larger, and at most 32 GiB.
constexpr int64_t kRecordBudget = 4LL << 30;
constexpr int64_t kRecordBudgetMax = 32LL << 30;

// A caller-set record count (OCT_OPT_RECORD_CAP) replaces the hint, within
// the same budget; records are used when there is room for 8 per query point
// (for a caller-set count, for 1).
int64_t record_cap(const Ctx& ctx, int64_t nq) {
    const int64_t budget = std::min(std::max(kRecordBudget, 8 * ctx.rec_edges_hint), kRecordBudgetMax);
    const int64_t fit = budget / (8 * std::max<int64_t>(nq, 1));
    const int64_t want = ctx.rec_cap_override > 0 ? std::min<int64_t>(ctx.rec_cap_override, kMaxRecords)
                                                  : ctx.rec_cap_hint;
    const int64_t cap = std::min<int64_t>(want, fit);
    return cap >= (ctx.rec_cap_override > 0 ? 1 : 8) ? cap : 0;
}

template <class T, int D>
int count_typed(Ctx& ctx, const Tree& q, const Tree& t, bool exclude_self, int64_t* n_edges) {
    cudaError_t err;
    cudaStream_t s = ctx.stream;
    const int64_t nq = q.n;
    if ((err = ensure(ctx.counts, (size_t)std::max<int64_t>(nq, 1) * 4)) ||
        (err = ensure(ctx.offsets, (size_t)(nq + 1) * 8)) ||
        (err = ensure(ctx.scan_tmp, (size_t)scan_tmp_elems(nq) * 8)) || (err = ensure(ctx.total, 16)) ||
        (err = ensure(ctx.dstatus, 8)))
        return cuda_status(ctx, err, "allocating edge scratch");
    if ((err = cudaMemsetAsync(ctx.dstatus.p, 0, 4, s)) || (err = cudaMemsetAsync(ctx.total.p, 0, 16, s)))
        return cuda_status(ctx, err, "status reset");
    if (!ctx.total_host) {
        if ((err = cudaMallocHost((void**)&ctx.total_host, 16))) return cuda_status(ctx, err, "pinned total");
    }
    const T r = (T)t.radius;
    const T r2 = r * r;  // src/cpu/edges_cpu.jl:184
    const Tuning tn = ctx.tuning_for(t.ndims, t.dtype, nq, q.nbrs_hint);
    ctx.plan_tuning = tn;
    ctx.rec_cap = 0;
    if (t.n_nodes == 0) {
        if ((err = cudaMemsetAsync(ctx.counts.p, 0, (size_t)nq * 4, s))) return cuda_status(ctx, err, "zero counts");
    } else {
        // Record each query's hits while counting, so that the fill pass
        // need not walk the tree again.
        const int64_t cap = record_cap(ctx, nq);
        if (cap > 0) {
            if ((err = ensure(ctx.recs, (size_t)nq * cap * 8)) || (err = ensure(ctx.rcount, (size_t)nq * 2)) ||
                (err = ensure(ctx.gflag, (size_t)std::max<int64_t>(q.n_groups, 1))))
                return cuda_status(ctx, err, "allocating hit records");
            ctx.rec_cap = cap;
        }
        PhaseTimer pt_(ctx, PH_COUNT);
        const int64_t ng = q.n_groups;
        if (ctx.rec_cap)
            launch_pdl(k_edges<T, D, EP_RECORD>, div_up(ng, kEdgeWarps), kEdgeThreads, 0, s, q.spts.as<SPt<T, D>>(),
                q.groups.as<int2>(), ng, t.tnode.as<TNode<T, D>>(), t.dfs_start, t.spts.as<SPt<T, D>>(), t.n_nodes, r2,
                T(0), exclude_self ? 1 : 0, ctx.counts.as<int32_t>(), nullptr, nullptr, nullptr, nullptr, nullptr,
                (int*)(ctx.total.as<int64_t>() + 1), ctx.recs.as<int2>(), ctx.rec_cap, ctx.rcount.as<uint16_t>(),
                ctx.gflag.as<uint8_t>(), t.batch(), nullptr, tn.max_seg, tn.multi_pop, tn.sub_boxes, tn.prefetch,
                own_start(q, t));
        else
            launch_pdl(k_edges<T, D, EP_COUNT>, div_up(ng, kEdgeWarps), kEdgeThreads, 0, s, q.spts.as<SPt<T, D>>(),
                q.groups.as<int2>(), ng, t.tnode.as<TNode<T, D>>(), t.dfs_start, t.spts.as<SPt<T, D>>(), t.n_nodes, r2,
                T(0), exclude_self ? 1 : 0, ctx.counts.as<int32_t>(), nullptr, nullptr, nullptr, nullptr, nullptr,
                nullptr, nullptr, 0, nullptr, nullptr, t.batch(), nullptr, tn.max_seg, tn.multi_pop, tn.sub_boxes,
                tn.prefetch, own_start(q, t));
        ctx.kernel_launches += 1;
    }
    {
        PhaseTimer pt_(ctx, PH_SCAN);
        ctx.kernel_launches += exclusive_scan_i32_i64(ctx.counts.as<int32_t>(), ctx.offsets.as<int64_t>(), nq,
                                                      ctx.total.as<int64_t>(), ctx.scan_tmp.as<int64_t>(), s);
    }
    if ((err = cudaMemcpyAsync(ctx.total_host, ctx.total.p, 16, cudaMemcpyDeviceToHost, s)) ||
        (err = wait_stream(s)))
        return cuda_status(ctx, err, "edge count");
    *n_edges = ctx.total_host[0];
    q.nbrs_hint = (double)*n_edges / (double)std::max<int64_t>(nq, 1);
    ctx.rec_overflow = 0;
    if (ctx.rec_cap) {
        // Size the next count's records for this one's largest query.
        const int32_t* w = reinterpret_cast<const int32_t*>(ctx.total_host + 1);
        ctx.rec_overflow = w[0];
        const int64_t need = ((int64_t)w[1] * 5 / 4 + 7) / 8 * 8;
        ctx.rec_cap_hint = std::min<int64_t>(std::max<int64_t>(need, 16), kMaxRecords);
        ctx.rec_edges_hint = *n_edges;
    }
    return OK;
}

// Ring of the fill: kFillRing chunks of CHUNK edges (32, 64 or 128: a tuned shape).
constexpr int kFillRing = 4;

template <class T, int D, bool FEAT, int CHUNK>
cudaError_t launch_expand_shape(Ctx& ctx, const Tree& q, const Tree& t, T inv_r, int32_t* senders, int32_t* receivers,
                                void* rel_disp, void* rel_dist, int bulk_ok) {
    constexpr size_t smem = kFillWarps * fill_ring_bytes<T, D, FEAT>(CHUNK * kFillRing);
    auto kern = k_expand<T, D, FEAT, CHUNK, kFillRing>;
    if (smem > 48 * 1024) {
        static bool attr_set = false;  // per instantiation
        if (!attr_set) {
            const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            attr_set = true;
        }
    }
    kern<<<div_up(q.n, 32 * kFillWarps), kFillWarps * 32, smem, ctx.stream>>>(
        q.n, q.iperm.as<int32_t>(), q.spts.as<SPt<T, D>>(), t.spts.as<SPt<T, D>>(), ctx.offsets.as<int64_t>(),
        ctx.recs.as<int2>(), ctx.rec_cap, ctx.rcount.as<uint16_t>(), inv_r, senders, receivers, (T*)rel_disp,
        (T*)rel_dist, t.batch(), bulk_ok);
    return cudaGetLastError();
}

// The fill of the last count's records with the tuned stores: direct
// (k_expand_direct) or bulk copies of 32-, 64- or 128-edge chunks (k_expand).
template <class T, int D, bool FEAT>
cudaError_t launch_expand(Ctx& ctx, const Tree& q, const Tree& t, T inv_r, int32_t* senders, int32_t* receivers,
                          void* rel_disp, void* rel_dist, int bulk_ok) {
    switch (ctx.plan_tuning.fill_chunk) {
        case 32:
            return launch_expand_shape<T, D, FEAT, 32>(ctx, q, t, inv_r, senders, receivers, rel_disp, rel_dist,
                                                       bulk_ok);
        case 64:
            return launch_expand_shape<T, D, FEAT, 64>(ctx, q, t, inv_r, senders, receivers, rel_disp, rel_dist,
                                                       bulk_ok);
        case 128:
            return launch_expand_shape<T, D, FEAT, 128>(ctx, q, t, inv_r, senders, receivers, rel_disp, rel_dist,
                                                        bulk_ok);
        default:  // direct stores
            launch_pdl(k_expand_direct<T, D>, div_up(q.n, 32 * kDirectWarps), kDirectWarps * 32, 0, ctx.stream, q.n,
                q.iperm.as<int32_t>(), q.spts.as<SPt<T, D>>(), t.spts.as<SPt<T, D>>(), ctx.offsets.as<int64_t>(),
                ctx.recs.as<int2>(), ctx.rec_cap, ctx.rcount.as<uint16_t>(), inv_r, senders, receivers, (T*)rel_disp,
                (T*)rel_dist, t.batch());
            return cudaGetLastError();
    }
}

template <class T, int D>
int fill_typed(Ctx& ctx, const Tree& q, const Tree& t, bool exclude_self, int32_t* senders, int32_t* receivers,
               void* rel_disp, void* rel_dist) {
    const T r = (T)t.radius;
    const T r2 = r * r;
    const T inv_r = T(1) / r;  // inv(r), src/cpu/edges_cpu.jl:185
    cudaStream_t s = ctx.stream;
    const Tuning& tn = ctx.plan_tuning;  // the shapes of the count this fill follows
    PhaseTimer pt_(ctx, PH_FILL);
    const int64_t ng = q.n_groups;
    if (ctx.rec_cap) {
        const int st = ensure_iperm(ctx, q);  // the fill visits the queries in original index order
        if (st != OK) return st;
        const bool feat = rel_disp != nullptr;
        auto aligned = [](const void* p) { return ((uintptr_t)p & 15u) == 0; };
        const int bulk_ok = aligned(senders) && (!feat || (aligned(receivers) && aligned(rel_disp) && aligned(rel_dist)));
        cudaError_t err = feat ? launch_expand<T, D, true>(ctx, q, t, inv_r, senders, receivers, rel_disp, rel_dist,
                                                           bulk_ok)
                               : launch_expand<T, D, false>(ctx, q, t, inv_r, senders, receivers, rel_disp, rel_dist,
                                                            bulk_ok);
        if (err != cudaSuccess) return cuda_status(ctx, err, "edge fill launch");
        ctx.kernel_launches += 1;
    }
    if (!ctx.rec_cap || ctx.rec_overflow) {
        // Groups without complete records walk the tree again.
        k_edges<T, D, EP_FILL><<<div_up(ng, kEdgeWarps), kEdgeThreads, 0, s>>>(
            q.spts.as<SPt<T, D>>(), q.groups.as<int2>(), ng, t.tnode.as<TNode<T, D>>(), t.dfs_start,
            t.spts.as<SPt<T, D>>(), t.n_nodes, r2, inv_r, exclude_self ? 1 : 0, nullptr, ctx.offsets.as<int64_t>(),
            senders, receivers, (T*)rel_disp, (T*)rel_dist, ctx.dstatus.as<int>(),
            ctx.rec_cap ? ctx.recs.as<int2>() : nullptr, ctx.rec_cap, nullptr, ctx.gflag.as<uint8_t>(), t.batch(),
            nullptr, tn.max_seg, tn.multi_pop, tn.sub_boxes, tn.prefetch, own_start(q, t));
        ctx.kernel_launches += 1;
    }
    return cuda_status(ctx, cudaGetLastError(), "edge fill launch");
}

template <class T, int D>
int neighbors_typed(Ctx& ctx, const Tree& t, const void* qcoords, int64_t nsel, int32_t* out_counts,
                    int32_t* out_idx, int64_t cap) {
    const T r = (T)t.radius;
    const T r2 = r * r;
    k_neighbors_of<T, D><<<div_up(nsel, 128), 128, 0, ctx.stream>>>(
        (const T*)qcoords, nsel, t.tnode.as<TNode<T, D>>(), t.spts.as<SPt<T, D>>(), t.n_nodes, r2, out_counts,
        out_idx, cap);
    ctx.kernel_launches += 1;
    return cuda_status(ctx, cudaGetLastError(), "neighbor query launch");
}

template <class T, int D>
cudaError_t count_into_typed(const Tree& q, const Tree& t, bool exclude_self, int32_t* counts, cudaStream_t s) {
    const T r = (T)t.radius;
    const T r2 = r * r;
    k_edges<T, D, EP_COUNT><<<div_up(q.n_groups, kEdgeWarps), kEdgeThreads, 0, s>>>(
        q.spts.as<SPt<T, D>>(), q.groups.as<int2>(), q.n_groups, t.tnode.as<TNode<T, D>>(), t.dfs_start,
        t.spts.as<SPt<T, D>>(), t.n_nodes, r2, T(0), exclude_self ? 1 : 0, counts, nullptr, nullptr, nullptr,
        nullptr, nullptr, nullptr, nullptr, 0, nullptr, nullptr, t.batch(), nullptr, kMaxSeg, kMultiPop, 1, 0, nullptr);
    return cudaGetLastError();
}

template <class T, int D>
int stats_typed(Ctx& ctx, const Tree& q, const Tree& t, bool exclude_self, unsigned long long* stats_dev) {
    const T r = (T)t.radius;
    const T r2 = r * r;
    const Tuning tn = ctx.tuning_for(t.ndims, t.dtype, q.n, q.nbrs_hint);
    k_edges<T, D, EP_STATS><<<div_up(q.n_groups, kEdgeWarps), kEdgeThreads, 0, ctx.stream>>>(
        q.spts.as<SPt<T, D>>(), q.groups.as<int2>(), q.n_groups, t.tnode.as<TNode<T, D>>(), t.dfs_start,
        t.spts.as<SPt<T, D>>(), t.n_nodes, r2, T(0), exclude_self ? 1 : 0, ctx.counts.as<int32_t>(), nullptr, nullptr,
        nullptr, nullptr, nullptr, nullptr, nullptr, 0, nullptr, nullptr, t.batch(), stats_dev, tn.max_seg,
        tn.multi_pop, tn.sub_boxes, tn.prefetch, own_start(q, t));
    ctx.kernel_launches += 1;
    return cuda_status(ctx, cudaGetLastError(), "traversal statistics launch");
}

}  // namespace

// Launches only the per-query count kernel into caller memory; allocates
// nothing (used by the allocation-free count entry point).
cudaError_t count_into(const Tree& q, const Tree& t, bool exclude_self, int32_t* counts, cudaStream_t s) {
    if (q.n == 0) return cudaSuccess;
    if (t.n_nodes == 0) return cudaMemsetAsync(counts, 0, (size_t)q.n * 4, s);
    if (t.dtype == 0)
        return t.ndims == 3 ? count_into_typed<float, 3>(q, t, exclude_self, counts, s)
                            : count_into_typed<float, 2>(q, t, exclude_self, counts, s);
    return t.ndims == 3 ? count_into_typed<double, 3>(q, t, exclude_self, counts, s)
                        : count_into_typed<double, 2>(q, t, exclude_self, counts, s);
}

int traversal_stats(Ctx& ctx, const Tree& q, const Tree& t, bool exclude_self, uint64_t* out, int n_out) {
    cudaError_t err;
    if ((err = ensure(ctx.counts, (size_t)std::max<int64_t>(q.n, 1) * 4)) || (err = ensure(ctx.tstats, TS_NUM * 8)))
        return cuda_status(ctx, err, "allocating statistics");
    if ((err = cudaMemsetAsync(ctx.tstats.p, 0, TS_NUM * 8, ctx.stream))) return cuda_status(ctx, err, "statistics");
    ctx.plan_query = nullptr;  // the counts buffer is reused: no fill may follow
    if (q.n > 0 && t.n_nodes > 0) {
        unsigned long long* sd = ctx.tstats.as<unsigned long long>();
        const int st = t.dtype == 0 ? (t.ndims == 3 ? stats_typed<float, 3>(ctx, q, t, exclude_self, sd)
                                                    : stats_typed<float, 2>(ctx, q, t, exclude_self, sd))
                                    : (t.ndims == 3 ? stats_typed<double, 3>(ctx, q, t, exclude_self, sd)
                                                    : stats_typed<double, 2>(ctx, q, t, exclude_self, sd));
        if (st != OK) return st;
    }
    uint64_t host[TS_NUM];
    if ((err = cudaMemcpyAsync(host, ctx.tstats.p, TS_NUM * 8, cudaMemcpyDeviceToHost, ctx.stream)) ||
        (err = cudaStreamSynchronize(ctx.stream)))
        return cuda_status(ctx, err, "statistics read");
    for (int k = 0; k < n_out && k < TS_NUM; ++k) out[k] = host[k];
    for (int k = TS_NUM; k < n_out; ++k) out[k] = 0;
    return OK;
}

int edges_count(Ctx& ctx, const Tree& q, const Tree& t, bool exclude_self, int64_t* n_edges) {
    ctx.plan_query = nullptr;
    int st = OK;
    if (q.n == 0) {
        *n_edges = 0;
    } else if (t.dtype == 0) {
        st = t.ndims == 3 ? count_typed<float, 3>(ctx, q, t, exclude_self, n_edges)
                          : count_typed<float, 2>(ctx, q, t, exclude_self, n_edges);
    } else {
        st = t.ndims == 3 ? count_typed<double, 3>(ctx, q, t, exclude_self, n_edges)
                          : count_typed<double, 2>(ctx, q, t, exclude_self, n_edges);
    }
    if (st != OK) return st;
    ctx.plan_query = &q;
    ctx.plan_target = &t;
    ctx.plan_qgen = q.generation;
    ctx.plan_tgen = t.generation;
    ctx.plan_exclude = exclude_self ? 1 : 0;
    ctx.plan_edges = *n_edges;
    return OK;
}

int edges_fill(Ctx& ctx, const Tree& q, const Tree& t, bool exclude_self, int32_t* senders, int32_t* receivers,
               void* rel_disp, void* rel_dist, int64_t n_edges) {
    if (ctx.plan_query != &q || ctx.plan_target != &t || ctx.plan_qgen != q.generation ||
        ctx.plan_tgen != t.generation || ctx.plan_exclude != (exclude_self ? 1 : 0))
        return set_error(ctx, ERR_STATE, "oct_edges_fill: no matching oct_edges_count for this pair and build");
    if (n_edges < ctx.plan_edges)
        return set_error(ctx, ERR_CAPACITY, "oct_edges_fill: output capacity is smaller than the edge count");
    if (ctx.plan_edges == 0 || q.n == 0 || t.n_nodes == 0) return OK;
    if (t.dtype == 0)
        return t.ndims == 3 ? fill_typed<float, 3>(ctx, q, t, exclude_self, senders, receivers, rel_disp, rel_dist)
                            : fill_typed<float, 2>(ctx, q, t, exclude_self, senders, receivers, rel_disp, rel_dist);
    return t.ndims == 3 ? fill_typed<double, 3>(ctx, q, t, exclude_self, senders, receivers, rel_disp, rel_dist)
                        : fill_typed<double, 2>(ctx, q, t, exclude_self, senders, receivers, rel_disp, rel_dist);
}

int edges_fill_diff(Ctx& ctx, const Tree& t, int32_t* senders, int32_t* receivers, void* rel_disp, void* rel_dist,
                    int32_t* mirror, int64_t n_edges) {
    if (ctx.plan_query != &t || ctx.plan_target != &t || ctx.plan_qgen != t.generation ||
        ctx.plan_tgen != t.generation || ctx.plan_exclude != 1)
        return set_error(ctx, ERR_STATE, "oct_edges_fill_diff: no matching self-pair oct_edges_count for this build");
    if (t.n_clouds) return set_error(ctx, ERR_ARGUMENT, "oct_edges_fill_diff: not defined for a batched tree");
    if (n_edges < ctx.plan_edges)
        return set_error(ctx, ERR_CAPACITY, "oct_edges_fill_diff: output capacity is smaller than the edge count");
    if (ctx.plan_edges > INT32_MAX)
        return set_error(ctx, ERR_OVERFLOW, "oct_edges_fill_diff: more than 2^31 - 1 edges overflow the Int32 mirrors");
    if (ctx.plan_edges == 0 || t.n == 0 || t.n_nodes == 0) return OK;
    // The COO first, then each edge's mirror by a scan of its sender's
    // segment.
    int st;
    if (t.dtype == 0)
        st = t.ndims == 3 ? fill_typed<float, 3>(ctx, t, t, true, senders, receivers, rel_disp, rel_dist)
                          : fill_typed<float, 2>(ctx, t, t, true, senders, receivers, rel_disp, rel_dist);
    else
        st = t.ndims == 3 ? fill_typed<double, 3>(ctx, t, t, true, senders, receivers, rel_disp, rel_dist)
                          : fill_typed<double, 2>(ctx, t, t, true, senders, receivers, rel_disp, rel_dist);
    if (st != OK) return st;
    return edges_mirror_scan(ctx, senders, receivers, ctx.plan_edges, t.n, ctx.offsets.as<int64_t>(), mirror);
}

namespace {
__global__ void k_offsets_i32(const int64_t* __restrict__ in, int64_t n, int32_t* __restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (int32_t)in[i];
}
}  // namespace

int csr_fill(Ctx& ctx, const Tree& q, const Tree& t, bool exclude_self, int32_t* offsets, int32_t* flat,
             int64_t capacity) {
    if (ctx.plan_query != &q || ctx.plan_target != &t || ctx.plan_qgen != q.generation ||
        ctx.plan_tgen != t.generation || ctx.plan_exclude != (exclude_self ? 1 : 0))
        return set_error(ctx, ERR_STATE, "oct_csr_fill: no matching oct_edges_count for this pair and build");
    if (ctx.plan_edges > INT32_MAX)
        return set_error(ctx, ERR_OVERFLOW, "oct_csr_fill: more than 2^31 - 1 neighbors overflow the Int32 offsets");
    if (capacity < ctx.plan_edges)
        return set_error(ctx, ERR_CAPACITY, "oct_csr_fill: flat capacity is smaller than the neighbor count");
    if (q.n == 0) return cuda_status(ctx, cudaMemsetAsync(offsets, 0, 4, ctx.stream), "csr offsets");
    k_offsets_i32<<<div_up(q.n + 1, 256), 256, 0, ctx.stream>>>(ctx.offsets.as<int64_t>(), q.n + 1, offsets);
    ctx.kernel_launches += 1;
    if (ctx.plan_edges == 0 || t.n_nodes == 0) return cuda_status(ctx, cudaGetLastError(), "csr offsets");
    if (t.dtype == 0)
        return t.ndims == 3 ? fill_typed<float, 3>(ctx, q, t, exclude_self, flat, nullptr, nullptr, nullptr)
                            : fill_typed<float, 2>(ctx, q, t, exclude_self, flat, nullptr, nullptr, nullptr);
    return t.ndims == 3 ? fill_typed<double, 3>(ctx, q, t, exclude_self, flat, nullptr, nullptr, nullptr)
                        : fill_typed<double, 2>(ctx, q, t, exclude_self, flat, nullptr, nullptr, nullptr);
}

int neighbors_of(Ctx& ctx, const Tree& t, const void* qcoords, int64_t nsel, int32_t* out_counts, int32_t* out_idx,
                 int64_t cap) {
    if (nsel == 0) return OK;
    if (t.n_nodes == 0) {
        return cuda_status(ctx, cudaMemsetAsync(out_counts, 0, (size_t)nsel * 4, ctx.stream), "neighbor query");
    }
    if (t.dtype == 0)
        return t.ndims == 3 ? neighbors_typed<float, 3>(ctx, t, qcoords, nsel, out_counts, out_idx, cap)
                            : neighbors_typed<float, 2>(ctx, t, qcoords, nsel, out_counts, out_idx, cap);
    return t.ndims == 3 ? neighbors_typed<double, 3>(ctx, t, qcoords, nsel, out_counts, out_idx, cap)
                        : neighbors_typed<double, 2>(ctx, t, qcoords, nsel, out_counts, out_idx, cap);
}

}  // namespace oct
