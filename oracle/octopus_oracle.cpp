// Octopus.jl CPU-path oracle -- TEST INFRASTRUCTURE ONLY.
//
// A plain C++17 restatement of the reference's CPU neighbor-search path, used
// by the test suite as the parity checker and by bench.py as the timed CPU
// baseline.  Nothing in the product (the CUDA library or its host mirror)
// links, loads or calls this file.
//
// Every function follows one reference function, cited as file:line inside
// the Octopus.jl project.  Floating-point operations are written in the same
// order as the Julia source and the file must be compiled with
// -ffp-contract=off -fno-fast-math so that no multiply-add is contracted
// (Julia does not contract either).
//
// Parity pin: the reference is Julia and cannot run in this environment, so
// the oracle is pinned against the known-answer tests the reference's own
// test files hold (test/morton.jl, test/edge_cases.jl, test/build.jl,
// src/api.jl doctest) and against brute force under the identical
// floating-point formula, which is exactly how the reference tests its CPU
// path (test/build.jl:13-28, test/edges_cpu.jl:14-39).
//
// Threading mirrors the reference's shape (src/cpu/bin_cpu.jl:61 binning is
// parallel; src/sort.jl, src/cpu/build_cpu.jl and src/cpu/refit_cpu.jl are
// serial; src/cpu/edges_cpu.jl:199,237 count/fill are parallel over
// n_query_chunks chunks; the scan between them is serial).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <type_traits>
#include <vector>
#include <omp.h>

namespace {

// ---------------------------------------------------------------- morton --
// src/morton.jl:13-23
inline uint64_t split_by_3(uint64_t x) {
    x &= 0x00000000001fffffULL;
    x = (x | (x << 32)) & 0x001f00000000ffffULL;
    x = (x | (x << 16)) & 0x001f0000ff0000ffULL;
    x = (x | (x << 8)) & 0x100f00f00f00f00fULL;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ULL;
    x = (x | (x << 2)) & 0x1249249249249249ULL;
    return x;
}
// src/morton.jl:25-33
inline uint64_t compact_by_3(uint64_t x) {
    x &= 0x1249249249249249ULL;
    x = (x | (x >> 2)) & 0x10c30c30c30c30c3ULL;
    x = (x | (x >> 4)) & 0x100f00f00f00f00fULL;
    x = (x | (x >> 8)) & 0x001f0000ff0000ffULL;
    x = (x | (x >> 16)) & 0x001f00000000ffffULL;
    x = (x | (x >> 32)) & 0x00000000001fffffULL;
    return x;
}
// src/morton.jl:50-58
inline uint64_t split_by_2(uint64_t x) {
    x &= 0x000000007fffffffULL;
    x = (x | (x << 16)) & 0x0000ffff0000ffffULL;
    x = (x | (x << 8)) & 0x00ff00ff00ff00ffULL;
    x = (x | (x << 4)) & 0x0f0f0f0f0f0f0f0fULL;
    x = (x | (x << 2)) & 0x3333333333333333ULL;
    x = (x | (x << 1)) & 0x5555555555555555ULL;
    return x;
}
// src/morton.jl:60-68
inline uint64_t compact_by_2(uint64_t x) {
    x &= 0x5555555555555555ULL;
    x = (x | (x >> 1)) & 0x3333333333333333ULL;
    x = (x | (x >> 2)) & 0x0f0f0f0f0f0f0f0fULL;
    x = (x | (x >> 4)) & 0x00ff00ff00ff00ffULL;
    x = (x | (x >> 8)) & 0x0000ffff0000ffffULL;
    x = (x | (x >> 16)) & 0x000000007fffffffULL;
    return x;
}
// src/morton.jl:35-40 (z<<2 | y<<1 | x)
inline uint64_t morton3(uint64_t ix, uint64_t iy, uint64_t iz) {
    return (split_by_3(iz) << 2) | (split_by_3(iy) << 1) | split_by_3(ix);
}
// src/morton.jl:70-74
inline uint64_t morton2(uint64_t ix, uint64_t iy) {
    return (split_by_2(iy) << 1) | split_by_2(ix);
}

// ------------------------------------------------- Julia float semantics --
// Base.min / Base.max for IEEE floats: NaN-propagating, -0.0 < +0.0.
template <class T> inline T jl_min(T x, T y) {
    if (std::isnan(x)) return x;
    if (std::isnan(y)) return y;
    if (y < x || (y == x && std::signbit(y) && !std::signbit(x))) return y;
    return x;
}
template <class T> inline T jl_max(T x, T y) {
    if (std::isnan(x)) return x;
    if (std::isnan(y)) return y;
    if (y > x || (y == x && !std::signbit(y) && std::signbit(x))) return y;
    return x;
}

// floor(Int32, v): src/morton.jl:84-86.  Julia throws InexactError when the
// floored value is NaN or outside Int32; that is reported as ok=false.
template <class T> inline int32_t floor_i32(T v, bool& ok) {
    T f = std::floor(v);
    if (!(f >= T(-2147483648.0) && f < T(2147483648.0))) { ok = false; return 0; }
    return (int32_t)f;
}

template <class T> inline int32_t clampi(int32_t v, int32_t lo, int32_t hi) {
    return v < lo ? lo : (v > hi ? hi : v);
}

// ------------------------------------------------------------- structures --
struct Tree {
    int ndims = 3;
    int64_t n = 0;
    int32_t n_nodes = 0;
    std::vector<int32_t> node_first, node_last;  // 1-based inclusive
    std::vector<int32_t> children;               // (NCH, n_nodes), 1-based ids, -1 = none
    std::vector<double> bmin_d, bmax_d;          // storage for T=double
    std::vector<float> bmin_f, bmax_f;           // storage for T=float
    std::vector<int32_t> perm;                   // 1-based
    std::vector<uint64_t> morton;                // per original point
    double origin[3] = {0, 0, 0};
    int dtype = 0;  // 0 = float32, 1 = float64
};

struct Edges {
    int64_t n_edges = 0;
    std::vector<int32_t> senders, receivers;
    std::vector<float> rdisp_f, rdist_f;
    std::vector<double> rdisp_d, rdist_d;
    std::vector<int64_t> offsets;  // n_q + 1, exclusive
};

// src/cpu/bin_cpu.jl:12-36 -- serial per-axis min, minus T(1e-6).
template <class T, int D>
void point_origin(const T* coords, int64_t n, T* o) {
    for (int d = 0; d < D; ++d) o[d] = coords[d];
    for (int64_t i = 1; i < n; ++i)
        for (int d = 0; d < D; ++d) o[d] = jl_min(o[d], coords[D * i + d]);
    for (int d = 0; d < D; ++d) o[d] = o[d] - T(1e-6);
}

// src/cpu/bin_cpu.jl:52-95 -- parallel (minbatch 4096) bin + encode.
template <class T, int D>
bool bin_encode(const T* coords, int64_t n, const T* o, T cell_size, uint64_t* keys, int nthreads) {
    const T inv_cs = T(1) / cell_size;
    const int32_t cmax = (D == 3) ? 0x1fffff : 0x7fffffff;
    int bad = 0;
#pragma omp parallel for schedule(static, 4096) num_threads(nthreads) reduction(| : bad)
    for (int64_t i = 0; i < n; ++i) {
        bool ok = true;
        int32_t c[3] = {0, 0, 0};
        for (int d = 0; d < D; ++d) {
            T v = (coords[D * i + d] - o[d]) * inv_cs;
            c[d] = clampi<T>(floor_i32(v, ok), 0, cmax);
        }
        if (!ok) { bad |= 1; keys[i] = 0; continue; }
        keys[i] = (D == 3) ? morton3((uint64_t)c[0], (uint64_t)c[1], (uint64_t)c[2])
                           : morton2((uint64_t)c[0], (uint64_t)c[1]);
    }
    return bad == 0;
}

// src/sort.jl:15-24 -- perm = 1:n stably sorted by key (Julia >= 1.9 QuickSort
// is stable, so ties keep ascending index).
void sort_by_key(std::vector<int32_t>& perm, const std::vector<uint64_t>& keys) {
    const int64_t n = (int64_t)keys.size();
    perm.resize(n);
    for (int64_t i = 0; i < n; ++i) perm[i] = (int32_t)(i + 1);
    std::stable_sort(perm.begin(), perm.end(),
                     [&](int32_t a, int32_t b) { return keys[a - 1] < keys[b - 1]; });
}

// src/cpu/build_cpu.jl:21-22, 46-49
template <int D> constexpr int bits_per_axis() { return D == 3 ? 21 : 31; }
template <int D> inline int level_shift(int L) { return D * bits_per_axis<D>() - D * (L + 1); }

// src/cpu/build_cpu.jl:100-194 -- serial BFS top-down build.
template <int D>
void build_topology(Tree& t, const std::vector<uint64_t>& keys, int32_t leaf_size) {
    constexpr int NCH = 1 << D;
    const int64_t n = (int64_t)t.perm.size();
    const int max_levels = bits_per_axis<D>();
    std::vector<int32_t> nf, nl, nlev, kids;
    nf.reserve(NCH * ((n + 31) / 32) + 16);
    nf.push_back(1); nl.push_back((int32_t)n); nlev.push_back(0);
    kids.assign(NCH, -1);
    int64_t next_open = 0;
    const uint64_t mask = (uint64_t)(NCH - 1);
    while (next_open < (int64_t)nf.size()) {
        const int64_t frontier_end = (int64_t)nf.size();
        for (int64_t nid = next_open; nid < frontier_end; ++nid) {
            const int32_t f = nf[nid], l = nl[nid], lvl = nlev[nid];
            const int32_t count = l - f + 1;
            if (count <= leaf_size || lvl >= max_levels) {
                for (int o = 0; o < NCH; ++o) kids[NCH * nid + o] = -1;
                continue;
            }
            // _partition_octants!  src/cpu/build_cpu.jl:55-82
            int32_t oc_first[NCH], oc_last[NCH];
            for (int o = 0; o < NCH; ++o) { oc_first[o] = -1; oc_last[o] = -2; }
            const int shift = level_shift<D>(lvl);
            int prev_o = -1;
            for (int32_t i = f; i <= l; ++i) {
                const int o = (int)((keys[t.perm[i - 1] - 1] >> shift) & mask);
                if (o != prev_o) {
                    if (prev_o != -1) oc_last[prev_o] = i - 1;
                    oc_first[o] = i;
                    prev_o = o;
                }
            }
            if (prev_o != -1) oc_last[prev_o] = l;
            for (int o = 0; o < NCH; ++o) {
                if (oc_first[o] == -1) {
                    kids[NCH * nid + o] = -1;
                } else {
                    const int32_t cid = (int32_t)nf.size() + 1;  // 1-based
                    nf.push_back(oc_first[o]);
                    nl.push_back(oc_last[o]);
                    nlev.push_back(lvl + 1);
                    kids.resize(NCH * nf.size(), -1);
                    kids[NCH * nid + o] = cid;
                }
            }
        }
        next_open = frontier_end;
    }
    t.n_nodes = (int32_t)nf.size();
    t.node_first.swap(nf);
    t.node_last.swap(nl);
    kids.resize((size_t)NCH * t.n_nodes);
    t.children.swap(kids);
}

// src/cpu/refit_cpu.jl:21-70 -- reverse-id bottom-up AABB fit.
template <class T, int D>
void refit_bounds(Tree& t, const T* coords, T* bmin, T* bmax) {
    constexpr int NCH = 1 << D;
    const T INF = std::numeric_limits<T>::infinity();
    for (int64_t nid = t.n_nodes - 1; nid >= 0; --nid) {
        if (t.children[NCH * nid] == -1) {
            const int32_t f = t.node_first[nid], l = t.node_last[nid];
            for (int d = 0; d < D; ++d) {
                T lo = INF, hi = -INF;
                for (int32_t k = f; k <= l; ++k) {
                    const T x = coords[D * (int64_t)(t.perm[k - 1] - 1) + d];
                    lo = jl_min(lo, x);
                    hi = jl_max(hi, x);
                }
                bmin[D * nid + d] = lo;
                bmax[D * nid + d] = hi;
            }
        } else {
            for (int d = 0; d < D; ++d) {
                T lo = INF, hi = -INF;
                for (int c = 0; c < NCH; ++c) {
                    const int32_t cid = t.children[NCH * nid + c];
                    if (cid == -1) continue;
                    lo = jl_min(lo, bmin[D * (int64_t)(cid - 1) + d]);
                    hi = jl_max(hi, bmax[D * (int64_t)(cid - 1) + d]);
                }
                bmin[D * nid + d] = lo;
                bmax[D * nid + d] = hi;
            }
        }
    }
}

template <class T> T* bmin_of(Tree& t);
template <> float* bmin_of<float>(Tree& t) { return t.bmin_f.data(); }
template <> double* bmin_of<double>(Tree& t) { return t.bmin_d.data(); }
template <class T> T* bmax_of(Tree& t);
template <> float* bmax_of<float>(Tree& t) { return t.bmax_f.data(); }
template <> double* bmax_of<double>(Tree& t) { return t.bmax_d.data(); }

template <class T> std::vector<T>& bminv(Tree& t);
template <> std::vector<float>& bminv<float>(Tree& t) { return t.bmin_f; }
template <> std::vector<double>& bminv<double>(Tree& t) { return t.bmin_d; }
template <class T> std::vector<T>& bmaxv(Tree& t);
template <> std::vector<float>& bmaxv<float>(Tree& t) { return t.bmax_f; }
template <> std::vector<double>& bmaxv<double>(Tree& t) { return t.bmax_d; }

// src/api.jl:194-250 (_run_cpu! for one dirty set).  Returns 0 or 1
// (1 = InexactError from floor(Int32, ...) in bin_cpu!).
template <class T, int D>
int run_build(Tree& t, const T* coords, int64_t n, T radius, int32_t leaf_size, int nthreads) {
    t.ndims = D;
    t.n = n;
    t.dtype = std::is_same<T, double>::value ? 1 : 0;
    if (n == 0) {
        t.n_nodes = 0;
        t.perm.clear(); t.morton.clear();
        t.node_first.clear(); t.node_last.clear(); t.children.clear();
        bminv<T>(t).clear(); bmaxv<T>(t).clear();
        return 0;
    }
    T o[3] = {0, 0, 0};
    point_origin<T, D>(coords, n, o);
    for (int d = 0; d < D; ++d) t.origin[d] = (double)o[d];
    t.morton.assign(n, 0);
    if (!bin_encode<T, D>(coords, n, o, radius, t.morton.data(), nthreads)) return 1;
    sort_by_key(t.perm, t.morton);
    build_topology<D>(t, t.morton, leaf_size);
    bminv<T>(t).assign((size_t)D * t.n_nodes, T(0));
    bmaxv<T>(t).assign((size_t)D * t.n_nodes, T(0));
    refit_bounds<T, D>(t, coords, bmin_of<T>(t), bmax_of<T>(t));
    return 0;
}

// src/cpu/iterator_cpu.jl:31-51
template <class T, int D>
inline T aabb_dist_sq(const T* p, const T* lo, const T* hi) {
    T acc = T(0);
    for (int d = 0; d < D; ++d) {
        T g = jl_max(lo[d] - p[d], T(0));
        g = jl_max(g, p[d] - hi[d]);
        const T g2 = g * g;
        acc = (d == 0) ? g2 : acc + g2;  // ((g1*g1 + g2*g2) + g3*g3)
    }
    return acc;
}

// src/cpu/iterator_cpu.jl:54-187 -- explicit-stack DFS.  Calls
// f(j_1based, diff[D], d2) for every target within r.
template <class T, int D, class F>
inline void traverse(const Tree& t, const T* bmin, const T* bmax, const T* coords_t,
                     const T* p, T r_sq, int32_t* stack, F&& f) {
    constexpr int NCH = 1 << D;
    if (t.n_nodes == 0) return;
    int sp = 0;
    stack[sp++] = 1;
    while (sp > 0) {
        const int32_t nid = stack[--sp];
        const int64_t n0 = nid - 1;
        const T dsq = aabb_dist_sq<T, D>(p, bmin + D * n0, bmax + D * n0);
        if (dsq > r_sq) continue;
        if (t.children[NCH * n0] == -1) {
            const int32_t f0 = t.node_first[n0], l0 = t.node_last[n0];
            for (int32_t k = f0; k <= l0; ++k) {
                const int32_t j = t.perm[k - 1];
                const T* q = coords_t + D * (int64_t)(j - 1);
                T diff[3];
                T d2 = T(0);
                for (int d = 0; d < D; ++d) {
                    diff[d] = q[d] - p[d];
                    const T s = diff[d] * diff[d];
                    d2 = (d == 0) ? s : d2 + s;
                }
                if (d2 <= r_sq) f(j, diff, d2);
            }
        } else {
            for (int c = 0; c < NCH; ++c) {
                const int32_t cid = t.children[NCH * n0 + c];
                if (cid != -1) {
                    const int64_t c0 = cid - 1;
                    const T cdsq = aabb_dist_sq<T, D>(p, bmin + D * c0, bmax + D * c0);
                    if (cdsq <= r_sq) stack[sp++] = cid;
                }
            }
        }
    }
}

// src/util.jl:38-50
inline void chunk_bounds(int64_t n, int64_t nchunks, int64_t c, int64_t& lo, int64_t& hi) {
    const int64_t base = n / nchunks, rem = n % nchunks;
    lo = (c - 1) * base + std::min(c - 1, rem) + 1;
    hi = lo + base - 1 + (c <= rem ? 1 : 0);
}
inline int64_t n_query_chunks(int64_t n, int64_t nstacks, int64_t nthreads) {
    const int64_t minwork = 1024;
    if (n <= minwork) return 1;
    const int64_t c = (n + minwork - 1) / minwork;
    return std::max<int64_t>(1, std::min(c, std::min(nstacks, nthreads)));
}

template <class T> std::vector<T>& rdispv(Edges& e);
template <> std::vector<float>& rdispv<float>(Edges& e) { return e.rdisp_f; }
template <> std::vector<double>& rdispv<double>(Edges& e) { return e.rdisp_d; }
template <class T> std::vector<T>& rdistv(Edges& e);
template <> std::vector<float>& rdistv<float>(Edges& e) { return e.rdist_f; }
template <> std::vector<double>& rdistv<double>(Edges& e) { return e.rdist_d; }

// src/cpu/edges_cpu.jl:172-247 (build_edges_cpu!) with the count and fill
// workers of :36-168.  The scan is carried in int64: the reference's Int32
// scan cannot represent 2^31 or more edges.
//
// q_first / q_last (1-based, inclusive) restrict the queries to a range: the
// result is then the slice of the full COO that those queries own (the COO
// lists each query's edges contiguously, in query order), with offsets
// relative to the slice's first edge.  The whole set is q_first = 1,
// q_last = n_q.
template <class T, int D>
void build_edges(Edges& e, Tree& t, const T* coords_q, int64_t n_q, const T* coords_t,
                 T r, bool exclude_self, int nthreads, int64_t q_first = 1, int64_t q_last = -1) {
    if (q_last < 0) q_last = n_q;
    const int64_t m_q = q_last - q_first + 1;  // queries in the range
    const T r_sq = r * r;
    const T inv_r = T(1) / r;
    const T* bmin = bmin_of<T>(t);
    const T* bmax = bmax_of<T>(t);
    const int depth = 1 + ((1 << D) - 1) * bits_per_axis<D>();
    // counts[i - q_first + 1] for query i of the range
    std::vector<int64_t> counts(m_q + 1, 0);
    const int64_t nchunks = n_query_chunks(m_q, nthreads, nthreads);
#pragma omp parallel for schedule(static, 1) num_threads(nthreads)
    for (int64_t c = 1; c <= nchunks; ++c) {
        int64_t lo, hi;
        chunk_bounds(m_q, nchunks, c, lo, hi);
        lo += q_first - 1;
        hi += q_first - 1;
        std::vector<int32_t> stack(depth + 8);
        for (int64_t i = lo; i <= hi; ++i) {
            const T* p = coords_q + D * (i - 1);
            int64_t cnt = 0;
            const int32_t i32 = (int32_t)i;
            traverse<T, D>(t, bmin, bmax, coords_t, p, r_sq, stack.data(),
                           [&](int32_t j, const T*, T) {
                               if (!exclude_self || j != i32) ++cnt;
                           });
            counts[i - q_first + 1] = cnt;
        }
    }
    for (int64_t i = 1; i <= m_q; ++i) counts[i] += counts[i - 1];
    e.n_edges = counts[m_q];
    e.offsets = counts;
    e.senders.assign(e.n_edges, 0);
    e.receivers.assign(e.n_edges, 0);
    rdispv<T>(e).assign((size_t)D * e.n_edges, T(0));
    rdistv<T>(e).assign((size_t)e.n_edges, T(0));
    int32_t* snd = e.senders.data();
    int32_t* rcv = e.receivers.data();
    T* rdisp = rdispv<T>(e).data();
    T* rdist = rdistv<T>(e).data();
#pragma omp parallel for schedule(static, 1) num_threads(nthreads)
    for (int64_t c = 1; c <= nchunks; ++c) {
        int64_t lo, hi;
        chunk_bounds(m_q, nchunks, c, lo, hi);
        lo += q_first - 1;
        hi += q_first - 1;
        std::vector<int32_t> stack(depth + 8);
        for (int64_t i = lo; i <= hi; ++i) {
            const T* p = coords_q + D * (i - 1);
            int64_t cur = counts[i - q_first];
            const int32_t i32 = (int32_t)i;
            traverse<T, D>(t, bmin, bmax, coords_t, p, r_sq, stack.data(),
                           [&](int32_t j, const T* diff, T d2) {
                               if (exclude_self && j == i32) return;
                               const int64_t k = cur++;
                               snd[k] = j;
                               rcv[k] = i32;
                               for (int d = 0; d < D; ++d) rdisp[D * k + d] = -diff[d] * inv_r;
                               rdist[k] = std::sqrt(d2) * inv_r;
                           });
        }
    }
}

// ext/OctopusChainRulesCoreExt.jl:150-189 -- serial pullback of
// build_edges_diff (self pair).  d_disp / d_dist may be null (zero tangent).
template <class T, int D>
void diff_backward(int64_t n_points, int64_t n_edges, const int32_t* snd, const int32_t* rcv,
                   const T* rel_disp, const T* rel_dist, const T* d_disp, const T* d_dist,
                   T r, T* grad) {
    std::memset(grad, 0, sizeof(T) * D * n_points);
    if (!d_disp && !d_dist) return;
    for (int64_t k = 0; k < n_edges; ++k) {
        const int64_t i = rcv[k] - 1, j = snd[k] - 1;
        if (d_disp) {
            for (int d = 0; d < D; ++d) {
                const T val = d_disp[D * k + d] / r;
                grad[D * i + d] += val;
                grad[D * j + d] -= val;
            }
        }
        if (d_dist) {
            const T d_norm = rel_dist[k];
            if (d_norm > T(1e-8)) {
                const T inv_dnr = d_dist[k] / (d_norm * r);
                for (int d = 0; d < D; ++d) {
                    const T g = rel_disp[D * k + d] * inv_dnr;
                    grad[D * i + d] += g;
                    grad[D * j + d] -= g;
                }
            }
        }
    }
}

// test/edges_cpu.jl:14-39 -- brute force under the same formula, in
// (receiver, sender) ascending order.
template <class T, int D>
int64_t brute_force(const T* cq, int64_t nq, const T* ct, int64_t nt, T r, bool exclude_self,
                    int32_t* snd, int32_t* rcv, int64_t cap) {
    const T r_sq = r * r;
    int64_t m = 0;
    for (int64_t i = 0; i < nq; ++i) {
        for (int64_t j = 0; j < nt; ++j) {
            if (exclude_self && i == j) continue;
            T d2 = T(0);
            for (int d = 0; d < D; ++d) {
                const T dx = cq[D * i + d] - ct[D * j + d];
                const T s = dx * dx;
                d2 = (d == 0) ? s : d2 + s;
            }
            if (d2 <= r_sq) {
                if (m < cap) { snd[m] = (int32_t)(j + 1); rcv[m] = (int32_t)(i + 1); }
                ++m;
            }
        }
    }
    return m;
}

}  // namespace

// =================================================================== C ABI
extern "C" {

uint64_t oracle_morton_encode3(uint32_t x, uint32_t y, uint32_t z) { return morton3(x, y, z); }
uint64_t oracle_morton_encode2(uint32_t x, uint32_t y) { return morton2(x, y); }
void oracle_morton_decode3(uint64_t c, uint32_t* out) {
    out[0] = (uint32_t)compact_by_3(c);
    out[1] = (uint32_t)compact_by_3(c >> 1);
    out[2] = (uint32_t)compact_by_3(c >> 2);
}
void oracle_morton_decode2(uint64_t c, uint32_t* out) {
    out[0] = (uint32_t)compact_by_2(c);
    out[1] = (uint32_t)compact_by_2(c >> 1);
}

// bin_point (src/morton.jl:83-95) in Float32; returns 0 or 1 (InexactError).
int oracle_bin_point_f32(int ndims, const float* p, const float* o, float inv_cs, int32_t* out) {
    bool ok = true;
    for (int d = 0; d < ndims; ++d) out[d] = floor_i32<float>((p[d] - o[d]) * inv_cs, ok);
    return ok ? 0 : 1;
}

// Build one point set's tree.  dtype 0 = Float32, 1 = Float64.  *status is 0,
// or 1 when floor(Int32, ...) would throw InexactError in the reference.
void* oracle_tree_build(const void* coords, int64_t n, int ndims, int dtype, double radius,
                        int32_t leaf_size, int nthreads, int* status) {
    Tree* t = new Tree();
    int st = 0;
    if (dtype == 0) {
        const float r = (float)radius;
        st = ndims == 3 ? run_build<float, 3>(*t, (const float*)coords, n, r, leaf_size, nthreads)
                        : run_build<float, 2>(*t, (const float*)coords, n, r, leaf_size, nthreads);
    } else {
        st = ndims == 3 ? run_build<double, 3>(*t, (const double*)coords, n, radius, leaf_size, nthreads)
                        : run_build<double, 2>(*t, (const double*)coords, n, radius, leaf_size, nthreads);
    }
    if (status) *status = st;
    return t;
}

int64_t oracle_tree_n_nodes(void* h) { return ((Tree*)h)->n_nodes; }

void oracle_tree_copy(void* h, int32_t* node_first, int32_t* node_last, int32_t* children,
                      void* bmin, void* bmax, int32_t* perm, uint64_t* morton, double* origin) {
    Tree* t = (Tree*)h;
    const int NCH = 1 << t->ndims;
    const size_t nn = (size_t)t->n_nodes;
    if (node_first) std::memcpy(node_first, t->node_first.data(), 4 * nn);
    if (node_last) std::memcpy(node_last, t->node_last.data(), 4 * nn);
    if (children) std::memcpy(children, t->children.data(), 4 * nn * NCH);
    const size_t es = t->dtype ? 8 : 4;
    if (bmin) std::memcpy(bmin, t->dtype ? (void*)t->bmin_d.data() : (void*)t->bmin_f.data(), es * nn * t->ndims);
    if (bmax) std::memcpy(bmax, t->dtype ? (void*)t->bmax_d.data() : (void*)t->bmax_f.data(), es * nn * t->ndims);
    if (perm) std::memcpy(perm, t->perm.data(), 4 * t->perm.size());
    if (morton) std::memcpy(morton, t->morton.data(), 8 * t->morton.size());
    if (origin) for (int d = 0; d < t->ndims; ++d) origin[d] = t->origin[d];
}

void oracle_tree_free(void* h) { delete (Tree*)h; }

// build_edges for the pair (query coords, target tree), restricted to the
// queries q_first..q_last (1-based, inclusive; q_last < 0: all of them).
void* oracle_edges_build_range(void* tree_t, const void* coords_q, int64_t n_q, const void* coords_t,
                               double radius, int exclude_self, int nthreads, int64_t q_first, int64_t q_last) {
    Tree* t = (Tree*)tree_t;
    Edges* e = new Edges();
    if (q_last < 0) q_last = n_q;
    if (t->dtype == 0) {
        const float r = (float)radius;
        if (t->ndims == 3)
            build_edges<float, 3>(*e, *t, (const float*)coords_q, n_q, (const float*)coords_t, r, exclude_self, nthreads,
                                  q_first, q_last);
        else
            build_edges<float, 2>(*e, *t, (const float*)coords_q, n_q, (const float*)coords_t, r, exclude_self, nthreads,
                                  q_first, q_last);
    } else {
        if (t->ndims == 3)
            build_edges<double, 3>(*e, *t, (const double*)coords_q, n_q, (const double*)coords_t, radius, exclude_self,
                                   nthreads, q_first, q_last);
        else
            build_edges<double, 2>(*e, *t, (const double*)coords_q, n_q, (const double*)coords_t, radius, exclude_self,
                                   nthreads, q_first, q_last);
    }
    return e;
}

void* oracle_edges_build(void* tree_t, const void* coords_q, int64_t n_q, const void* coords_t,
                         double radius, int exclude_self, int nthreads) {
    return oracle_edges_build_range(tree_t, coords_q, n_q, coords_t, radius, exclude_self, nthreads, 1, -1);
}

int64_t oracle_edges_n(void* h) { return ((Edges*)h)->n_edges; }

void oracle_edges_copy(void* h, int ndims, int dtype, int32_t* senders, int32_t* receivers,
                       void* rdisp, void* rdist, int64_t* offsets, int64_t n_q) {
    Edges* e = (Edges*)h;
    const size_t m = (size_t)e->n_edges;
    if (senders) std::memcpy(senders, e->senders.data(), 4 * m);
    if (receivers) std::memcpy(receivers, e->receivers.data(), 4 * m);
    if (dtype == 0) {
        if (rdisp) std::memcpy(rdisp, e->rdisp_f.data(), 4 * m * ndims);
        if (rdist) std::memcpy(rdist, e->rdist_f.data(), 4 * m);
    } else {
        if (rdisp) std::memcpy(rdisp, e->rdisp_d.data(), 8 * m * ndims);
        if (rdist) std::memcpy(rdist, e->rdist_d.data(), 8 * m);
    }
    if (offsets) std::memcpy(offsets, e->offsets.data(), 8 * (size_t)(n_q + 1));
}

void oracle_edges_free(void* h) { delete (Edges*)h; }

int64_t oracle_brute_force(const void* cq, int64_t nq, const void* ct, int64_t nt, int ndims,
                           int dtype, double radius, int exclude_self, int32_t* snd, int32_t* rcv,
                           int64_t cap) {
    if (dtype == 0) {
        const float r = (float)radius;
        return ndims == 3 ? brute_force<float, 3>((const float*)cq, nq, (const float*)ct, nt, r, exclude_self, snd, rcv, cap)
                          : brute_force<float, 2>((const float*)cq, nq, (const float*)ct, nt, r, exclude_self, snd, rcv, cap);
    }
    return ndims == 3 ? brute_force<double, 3>((const double*)cq, nq, (const double*)ct, nt, radius, exclude_self, snd, rcv, cap)
                      : brute_force<double, 2>((const double*)cq, nq, (const double*)ct, nt, radius, exclude_self, snd, rcv, cap);
}

void oracle_diff_backward(int ndims, int dtype, int64_t n_points, int64_t n_edges,
                          const int32_t* snd, const int32_t* rcv, const void* rel_disp,
                          const void* rel_dist, const void* d_disp, const void* d_dist,
                          double radius, void* grad) {
    if (dtype == 0) {
        const float r = (float)radius;
        if (ndims == 3)
            diff_backward<float, 3>(n_points, n_edges, snd, rcv, (const float*)rel_disp, (const float*)rel_dist,
                                    (const float*)d_disp, (const float*)d_dist, r, (float*)grad);
        else
            diff_backward<float, 2>(n_points, n_edges, snd, rcv, (const float*)rel_disp, (const float*)rel_dist,
                                    (const float*)d_disp, (const float*)d_dist, r, (float*)grad);
    } else {
        if (ndims == 3)
            diff_backward<double, 3>(n_points, n_edges, snd, rcv, (const double*)rel_disp, (const double*)rel_dist,
                                     (const double*)d_disp, (const double*)d_dist, radius, (double*)grad);
        else
            diff_backward<double, 2>(n_points, n_edges, snd, rcv, (const double*)rel_disp, (const double*)rel_dist,
                                     (const double*)d_disp, (const double*)d_dist, radius, (double*)grad);
    }
}

int oracle_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
