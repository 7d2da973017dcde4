// Linear quadtree (2D) / octree (3D) build from Morton keys.
//
// The reference's tree is d3-quadtree's insertion tree
// (crates/graph-core/src/layout/force/quadtree.rs:116-195, quadtree/build.rs:26-114):
// a root square snapped to floor(min) and doubled until it covers every point,
// split at exact midpoints, so every cell is a dyadic square of the root. A key
// that interleaves the points' dyadic coordinates in that root square
// (bit a of each D-bit group = "x_a >= midpoint", the reference's slot order,
// quadtree/bounds.rs:34-50) therefore sorts the points into the reference's own
// leaf preorder (quadtree/preorder.rs:56-114), and the cells that branch are
// exactly the reference's cells that hold two or more distinct keys.
//
// Build, all integer except the FP64 sums:
//   keys -> LSD radix sort -> unique keys (leaves) and the prefix of the points'
//   FP64 mass / mass-moment terms at every leaf start -> Karras binary radix
//   tree over the unique keys, each node marking the quad/oct cells among its
//   children (binary nodes whose level, common prefix / D, differs from their
//   parent's) -> preorder index of every cell from an exclusive scan of "cells
//   starting at leaf s" -> every cell written at once, its sums from its points
//   (a leaf) or as the difference of two prefixes, skip(cell) = P[last leaf + 1].
// A chain of single-child cells in the reference collapses to its deepest
// member here; the walk's far test is monotone in the cell width and the chain
// shares one mass and centre, so the collapsed cell opens and approximates
// exactly where the chain would.
#pragma once

#include "common.cuh"

namespace gr {

// Leaves per block of the cell-level scan (scan.cuh's SC_TILE); k_karras
// counts the level bits it sets per block of this many leaves.
constexpr uint32_t SC_TILE_LEAVES = 2048;

template <int D> struct Levels;
template <> struct Levels<2> { static constexpr int L = 32; };  // 64-bit keys
template <> struct Levels<3> { static constexpr int L = 21; };  // 63-bit keys

__device__ __forceinline__ uint64_t spread2(uint64_t x) {  // 32 bits -> even bits
    x &= 0xffffffffull;
    x = (x | (x << 16)) & 0x0000ffff0000ffffull;
    x = (x | (x << 8)) & 0x00ff00ff00ff00ffull;
    x = (x | (x << 4)) & 0x0f0f0f0f0f0f0f0full;
    x = (x | (x << 2)) & 0x3333333333333333ull;
    x = (x | (x << 1)) & 0x5555555555555555ull;
    return x;
}

__device__ __forceinline__ uint64_t spread3(uint64_t x) {  // 21 bits -> every third bit
    x &= 0x1fffffull;
    x = (x | (x << 32)) & 0x001f00000000ffffull;
    x = (x | (x << 16)) & 0x001f0000ff0000ffull;
    x = (x | (x << 8)) & 0x100f00f00f00f00full;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}

// The reference's root square (quadtree.rs:157-195, cover of the minimum then
// the maximum corner): corner floor(min), side the smallest power of two >= 1
// that holds the maximum. Returns the side; ok is false if it overflowed.
template <int D>
__device__ __forceinline__ double root_square(const double *mn, const double *mx, double *root0, bool &ok) {
    double z = 1.0;
    ok = true;
    for (int a = 0; a < D; a++) root0[a] = floor(mn[a]);
    for (bool grow = true; grow;) {
        grow = false;
        for (int a = 0; a < D; a++)
            if (mx[a] >= root0[a] + z) grow = true;
        if (grow) z *= 2.0;
        if (!isfinite(z)) {
            ok = false;
            break;
        }
    }
    return z;
}

// Left-aligned Morton key of one node in the root square: per axis
// q = floor((x - x0) * 2^L / side), exact in FP64 because the side is a power of
// two; bit a of each D-bit group is axis a (the reference's slot order).
template <int D>
__device__ __forceinline__ uint64_t morton_key(const float4 &p, const double *root0, double root_w) {
    constexpr int L = Levels<D>::L;
    const double scale = ldexp(1.0, L) / root_w;
    const double qmax = ldexp(1.0, L) - 1.0;
    const float c[3] = {p.x, p.y, p.z};
    uint64_t key = 0;
#pragma unroll
    for (int a = 0; a < D; a++) {
        double q = floor(((double)c[a] - root0[a]) * scale);
        q = fmin(fmax(q, 0.0), qmax);
        key |= (D == 2 ? spread2((uint64_t)q) : spread3((uint64_t)q)) << a;
    }
    return key << (64 - D * L);  // clz of a difference counts levels from the root
}

// ------------------------------------------------------------------ bounds --

constexpr int BND_THREADS = 256;

// Counters a later kernel of the tick accumulates into (nullable), zeroed by
// block 0 of the bounds pass so that no memset node precedes them.
struct ZeroWords {
    uint32_t *p[3] = {nullptr, nullptr, nullptr};
    uint32_t len[3] = {0, 0, 0};
    void add(uint32_t *q, uint32_t words) {
        for (int j = 0; j < 3; j++)
            if (!p[j]) {
                p[j] = q;
                len[j] = words;
                return;
            }
    }
    __device__ __forceinline__ void clear() const {
#pragma unroll
        for (int j = 0; j < 3; j++)
            for (uint32_t i = threadIdx.x; i < len[j]; i += blockDim.x) p[j][i] = 0u;
    }
};

// A block's extent and FP64 coordinate sums of this thread's positions (lo, hi,
// sum, accumulated over its strided nodes in order): warp shuffles for min / max,
// block_sum_d for the sums, one record of 3 D doubles per block in part.
template <int D>
__device__ __forceinline__ void bounds_block(const float *lo, const float *hi, const double *sum,
                                             double *__restrict__ part, double *s_red, float (*s_f)[32]) {
    const int lane = threadIdx.x % GR_WARP, w = threadIdx.x / GR_WARP;
#pragma unroll
    for (int a = 0; a < D; a++) {
        float l = lo[a], h = hi[a];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            l = fminf(l, __shfl_xor_sync(GR_FULL, l, o));
            h = fmaxf(h, __shfl_xor_sync(GR_FULL, h, o));
        }
        if (lane == 0) {
            s_f[a][w] = l;
            s_f[D + a][w] = h;
        }
    }
    double tot[D];
#pragma unroll
    for (int a = 0; a < D; a++) tot[a] = block_sum_d<BND_THREADS>(sum[a], s_red);
    if (threadIdx.x == 0) {
        double *q = part + (size_t)blockIdx.x * 3 * D;
        for (int a = 0; a < D; a++) {
            float l = INFINITY, h = -INFINITY;
            for (int k = 0; k < BND_THREADS / GR_WARP; k++) {
                l = fminf(l, s_f[a][k]);
                h = fmaxf(h, s_f[D + a][k]);
            }
            q[a] = l;
            q[D + a] = h;
            q[2 * D + a] = tot[a];
        }
    }
}

// The grid's last block: the block records folded in block order into the
// reference's root square (quadtree.rs:157-195 cover, both corners) and the
// mean gravity pulls toward (state.rs:208-218).
template <int D>
__device__ __forceinline__ void bounds_finish(const double *part, uint32_t n, DevState *st, double *s_red) {
    const int lane = threadIdx.x % GR_WARP, w = threadIdx.x / GR_WARP;
    double gl[D], gh[D], gs[D];
#pragma unroll
    for (int a = 0; a < D; a++) {
        gl[a] = INFINITY;
        gh[a] = -INFINITY;
        gs[a] = 0.0;
    }
    for (uint32_t b = threadIdx.x; b < gridDim.x; b += BND_THREADS) {
        const double *q = part + (size_t)b * 3 * D;
#pragma unroll
        for (int a = 0; a < D; a++) {
            gl[a] = fmin(gl[a], __ldcg(q + a));
            gh[a] = fmax(gh[a], __ldcg(q + D + a));
            gs[a] += __ldcg(q + 2 * D + a);
        }
    }
    // min / max are exact in any order: warp shuffles, then the warp results
    __shared__ double s_l[D][BND_THREADS / GR_WARP], s_h[D][BND_THREADS / GR_WARP];
#pragma unroll
    for (int a = 0; a < D; a++) {
        double l = gl[a], h = gh[a];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            l = fmin(l, __shfl_xor_sync(GR_FULL, l, o));
            h = fmax(h, __shfl_xor_sync(GR_FULL, h, o));
        }
        if (lane == 0) {
            s_l[a][w] = l;
            s_h[a][w] = h;
        }
    }
    double S[D];
#pragma unroll
    for (int a = 0; a < D; a++) S[a] = block_sum_d<BND_THREADS>(gs[a], s_red);
    if (threadIdx.x == 0) {
        double mn[D], mx[D];
        for (int a = 0; a < D; a++) {
            mn[a] = INFINITY;
            mx[a] = -INFINITY;
            for (int k = 0; k < BND_THREADS / GR_WARP; k++) {
                mn[a] = fmin(mn[a], s_l[a][k]);
                mx[a] = fmax(mx[a], s_h[a][k]);
            }
        }
        bool ok = true;
        const double z = root_square<D>(mn, mx, st->root0, ok);
        if (!ok) atomicOr(&st->error, (uint32_t)ERR_BOUNDS);
        st->root_w = z;
        for (int a = 0; a < D; a++) st->mean[a] = S[a] / (double)n;
        if (st->error) st->converged = 1;
    }
}

// Extent and FP64 coordinate sums of the positions into the root square and the
// mean. When the previous tick's update already computed them from these
// positions (bounds_stamp == iter_no + 1, bounds_block / bounds_finish over the
// same grid and the same per-thread order, so bit for bit the same), only the
// counters are zeroed. A grid of frc_blocks(n) blocks (the update's grid).
template <int D>
__global__ void __launch_bounds__(BND_THREADS)
k_bounds(const float4 *__restrict__ pos, uint32_t n, DevState *st, double *__restrict__ part, ZeroWords zw) {
    gr_pdl_enter();
    if (st->converged) return;
    if (blockIdx.x == 0) zw.clear();
    if (st->bounds_stamp == st->iter_no + 1u) return;
    __shared__ double s_red[32];
    __shared__ float s_f[2 * D][32];
    __shared__ bool s_last;
    float lo[D], hi[D];
    double sum[D];
#pragma unroll
    for (int a = 0; a < D; a++) {
        lo[a] = INFINITY;
        hi[a] = -INFINITY;
        sum[a] = 0.0;
    }
    bool bad = false;
    // this thread's points i0, i0 + stride, ... in order, BND_U loads in flight
    constexpr int BND_U = 4;
    const uint64_t stride = (uint64_t)gridDim.x * BND_THREADS;
    for (uint64_t i0 = blockIdx.x * BND_THREADS + threadIdx.x; i0 < n; i0 += stride * BND_U) {
        float4 pv[BND_U];
#pragma unroll
        for (int u = 0; u < BND_U; u++) {
            const uint64_t i = i0 + u * stride;
            pv[u] = i < n ? pos[i] : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int u = 0; u < BND_U; u++) {
            if (i0 + u * stride >= n) break;
            const float c[3] = {pv[u].x, pv[u].y, pv[u].z};
#pragma unroll
            for (int a = 0; a < D; a++) {
                if (!isfinite(c[a])) bad = true;
                lo[a] = fminf(lo[a], c[a]);
                hi[a] = fmaxf(hi[a], c[a]);
                sum[a] += (double)c[a];
            }
        }
    }
    if (__syncthreads_or(bad)) {
        if (threadIdx.x == 0) atomicOr(&st->error, (uint32_t)ERR_NONFINITE);
    }
    bounds_block<D>(lo, hi, sum, part, s_red, s_f);
    if (!last_block_done(&st->counters[0], &s_last)) return;
    bounds_finish<D>(part, n, st, s_red);
}

// Morton key of every node in the root square: per axis q = floor((x - x0) *
// 2^L / side), exact in FP64 because the side is a power of two.
template <int D>
__global__ void k_keys(const float4 *__restrict__ pos, uint32_t n, const DevState *st,
                       uint64_t *__restrict__ keys, uint32_t *__restrict__ vals) {
    gr_pdl_enter();
    if (st->converged) return;
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    keys[i] = morton_key<D>(pos[i], st->root0, st->root_w);
    vals[i] = i;
}

// Binary radix tree node arrays (Karras 2012, "Maximizing parallelism in the
// construction of BVHs, octrees, and k-d trees", HPG): internal node i covers
// unique leaves [first, last]; children are coded with LEAF_BIT when a leaf.
constexpr uint32_t LEAF_BIT = 0x80000000u;

struct BinTree {
    uint32_t *first, *last, *left, *right;
    int32_t *delta;       // common prefix length of the node's keys
    int32_t *int_parent;  // internal node -> parent (-1 at the root)
    int32_t *leaf_parent; // leaf -> parent (-1 when the tree is one leaf)
    uint32_t *visit;      // bottom-up arrival tickets
    uint32_t *cell_of;    // internal node -> its cell's preorder index, when it is a cell (nullable)
    int4 *rec;            // internal node -> {first, last, 0, delta} in one load (nullable)
    uint32_t *levels;     // unique leaf s -> bit l set when a cell of level l begins at s (nullable)
    uint8_t *cell_flag;   // internal node -> 1 when it is a cell (written with levels)
    uint32_t *marks;      // nullable: per SC_TILE-leaf block, the count of level bits set in it (zeroed before)
};

// What karras_node found for internal node i: its leaf range, split and
// common-prefix length.
struct KarrasNode {
    int32_t first, last, gamma, delta;
};

__device__ __forceinline__ int kdelta(const uint64_t *__restrict__ k, int32_t a, int32_t b, int32_t nu) {
    if (b < 0 || b >= nu) return -1;
    return __clzll(k[a] ^ k[b]);
}

// Internal node i of the binary radix tree over nu unique keys. The per-node
// arrays (first .. int_parent, visit) are written when t.left is set; the
// packed records when t.rec is set; leaf_parent always.
__device__ __forceinline__ KarrasNode karras_node(int32_t i, int32_t nu, const uint64_t *__restrict__ k, BinTree t) {
    const int dir = (kdelta(k, i, i + 1, nu) - kdelta(k, i, i - 1, nu)) > 0 ? 1 : -1;
    const int dmin = kdelta(k, i, i - dir, nu);
    int32_t lmax = 2;
    while (kdelta(k, i, i + lmax * dir, nu) > dmin) lmax <<= 1;
    int32_t l = 0;
    for (int32_t s = lmax >> 1; s >= 1; s >>= 1)
        if (kdelta(k, i, i + (l + s) * dir, nu) > dmin) l += s;
    const int32_t j = i + l * dir;
    const int dnode = kdelta(k, i, j, nu);
    int32_t s = 0;
    int32_t step = l;
    do {
        step = (step + 1) >> 1;
        if (kdelta(k, i, i + (s + step) * dir, nu) > dnode) s += step;
    } while (step > 1);
    const int32_t gamma = i + s * dir + (dir < 0 ? -1 : 0);
    const int32_t first = min(i, j), last = max(i, j);
    const bool arrays = t.left != nullptr;
    if (arrays) {
        t.first[i] = (uint32_t)first;
        t.last[i] = (uint32_t)last;
        t.delta[i] = dnode;
        t.visit[i] = 0;
    }
    if (t.rec) t.rec[i] = make_int4(first, last, 0, dnode);  // one 16-byte store
    if (first == gamma) {
        if (arrays) t.left[i] = (uint32_t)gamma | LEAF_BIT;
        t.leaf_parent[gamma] = i;
    } else {
        if (arrays) {
            t.left[i] = (uint32_t)gamma;
            t.int_parent[gamma] = i;
        }
    }
    if (last == gamma + 1) {
        if (arrays) t.right[i] = (uint32_t)(gamma + 1) | LEAF_BIT;
        t.leaf_parent[gamma + 1] = i;
    } else {
        if (arrays) {
            t.right[i] = (uint32_t)(gamma + 1);
            t.int_parent[gamma + 1] = i;
        }
    }
    if (i == 0 && arrays) t.int_parent[0] = -1;
    return KarrasNode{first, last, gamma, dnode};
}

// The cells among node i's internal children (and the root): a node is a cell
// when its level (common prefix / D) differs from its parent's. Each cell sets
// bit `level` of its first leaf's mask; the cells beginning at one leaf lie on
// one chain of ancestors and have distinct levels, so leaf s starts
// 1 + popc(levels[s]) cells and the level-l one is the popc(levels[s] & (2^l -
// 1))-th of them in preorder. A level is at most 31 (2D, 64-bit keys) or 20
// (3D, 63-bit keys).
// Adds 1 at marks[tgt] for every lane with `has`, with one atomic per warp when
// all those lanes name the same counter (the common case: a warp's nodes are
// 32 consecutive split positions). The whole warp calls it.
__device__ __forceinline__ void count_marks(bool has, uint32_t tgt, uint32_t *__restrict__ marks) {
    const uint32_t act = __ballot_sync(GR_FULL, has);
    if (act == 0u) return;
    const int leader = __ffs(act) - 1;
    const uint32_t t0 = __shfl_sync(GR_FULL, tgt, leader);
    if (__all_sync(GR_FULL, !has || tgt == t0)) {
        if ((int)(threadIdx.x % GR_WARP) == leader) atomicAdd(&marks[t0], (uint32_t)__popc(act));
    } else if (has) {
        atomicAdd(&marks[tgt], 1u);
    }
}

// With marks, each bit set also counts once in marks[leaf / mark_tile] (the
// block sums of the cell-level scan, so that scan needs no reduce pass). The
// whole warp calls it; lanes without a node (valid false) only vote.
template <int D>
__device__ __forceinline__ void mark_cells(bool valid, int32_t i, int32_t nu, const uint64_t *__restrict__ k,
                                           const KarrasNode &q, uint32_t *__restrict__ levels,
                                           uint8_t *__restrict__ cell_flag, uint32_t *__restrict__ marks,
                                           uint32_t mark_tile) {
    bool ml = false, mr = false;
    if (valid) {
        const int lv = q.delta / D;
        if (i == 0) {
            atomicOr(&levels[0], 1u << lv);
            if (marks) atomicAdd(&marks[0], 1u);
            cell_flag[0] = 1;
        }
        if (q.first != q.gamma) {  // left child [first, gamma], internal node gamma
            const int c = kdelta(k, q.first, q.gamma, nu) / D;
            ml = c != lv;
            if (ml) atomicOr(&levels[q.first], 1u << c);
            cell_flag[q.gamma] = ml ? 1 : 0;
        }
        if (q.last != q.gamma + 1) {  // right child [gamma + 1, last], internal node gamma + 1
            const int c = kdelta(k, q.gamma + 1, q.last, nu) / D;
            mr = c != lv;
            if (mr) atomicOr(&levels[q.gamma + 1], 1u << c);
            cell_flag[q.gamma + 1] = mr ? 1 : 0;
        }
    }
    if (marks) {
        count_marks(ml, valid ? (uint32_t)q.first / mark_tile : 0u, marks);
        count_marks(mr, valid ? (uint32_t)(q.gamma + 1) / mark_tile : 0u, marks);
    }
}

template <int D>
__global__ void k_karras(const DevState *st, const uint64_t *__restrict__ k, BinTree t) {
    gr_pdl_enter();
    if (st->converged) return;
    const int32_t nu = (int32_t)st->n_unique;
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0 && nu == 1) t.leaf_parent[0] = -1;
    const bool valid = i < nu - 1;
    if (__all_sync(GR_FULL, !valid)) return;  // whole warps only: mark_cells votes across the warp
    KarrasNode q{0, 0, 0, 0};
    if (valid) q = karras_node(i, nu, k, t);
    if (t.levels) mark_cells<D>(valid, i, nu, k, q, t.levels, t.cell_flag, t.marks, SC_TILE_LEAVES);
}

// ---- bodies without atomics: a prefix of the point terms (m, m x per axis;
// each an exact FP64 product of two FP32 values) over the sorted points, read
// at every leaf's first point, and every internal node's body as the
// difference of the prefixes at its range ends. Inside a tile of AG_TILE
// points the prefix is an FP64 scan (error ~1e-16 of the tile's sums); across
// tiles it is a double-double carry (exact to ~1e-32 of the whole sum), so a
// node's sums are as exact as a direct FP64 sum over its points. Every
// decomposition is fixed, so the result is the same every run.

struct DD {
    double hi, lo;
};

__device__ __forceinline__ DD dd_add(DD a, DD b) {  // Knuth's two-sum, renormalised
    const double s = a.hi + b.hi;
    const double bb = s - a.hi;
    double e = (a.hi - (s - bb)) + (b.hi - bb);
    e += a.lo + b.lo;
    const double hi = s + e;
    return DD{hi, e - (hi - s)};
}

struct BodyDD {
    DD m, c0, c1, c2;
};

template <int D>
__device__ __forceinline__ BodyDD bdd_add(const BodyDD &a, const BodyDD &b) {
    return BodyDD{dd_add(a.m, b.m), dd_add(a.c0, b.c0), dd_add(a.c1, b.c1),
                  D == 3 ? dd_add(a.c2, b.c2) : DD{0.0, 0.0}};
}

__device__ __forceinline__ BodyDD bdd_of(const Body &b) {
    return BodyDD{{b.m, 0.0}, {b.c0, 0.0}, {b.c1, 0.0}, {b.c2, 0.0}};
}

__device__ __forceinline__ double dd_diff(DD a, DD b) { return dd_add(a, DD{-b.hi, -b.lo}).hi; }

// 512 x 2: measured at 1M 2D nodes against 256 x 4 (2.4 us less) and 128 x 8 (20 us more)
constexpr int AG_T = 512, AG_I = 2, AG_TILE = AG_T * AG_I, AG_W = AG_T / GR_WARP;

// FP64 sums of the sorted points [a0, a1) of one leaf, in order; coinc = all
// points are the same point.
template <int D>
__device__ __forceinline__ Body leaf_sum(const float4 *__restrict__ sp, uint32_t a0, uint32_t a1, bool &coinc) {
    Body b{0.0, 0.0, 0.0, 0.0};
    const float4 f0 = sp[a0];
    coinc = true;
    for (uint32_t q = a0; q < a1; q++) {
        const float4 p = q == a0 ? f0 : sp[q];
        const double m = (double)p.w;
        b.m += m;
        b.c0 += m * (double)p.x;
        b.c1 += m * (double)p.y;
        if (D == 3) b.c2 += m * (double)p.z;
        coinc = coinc && p.x == f0.x && p.y == f0.y && (D == 2 || p.z == f0.z);
    }
    return b;
}

// Leaf bodies as an array (the adjoint reads them; the tick's own cell writer
// recomputes them with the same leaf_sum).
template <int D>
__global__ void k_leaf_body(const DevState *st, const float4 *__restrict__ sp, const uint32_t *__restrict__ leaf_start,
                            Body *__restrict__ leaf_body, uint8_t *__restrict__ leaf_coinc) {
    if (st->converged) return;
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= st->n_unique) return;
    bool coinc;
    body_store(&leaf_body[s], leaf_sum<D>(sp, leaf_start[s], leaf_start[s + 1], coinc));
    leaf_coinc[s] = coinc ? 1 : 0;
}

__device__ __forceinline__ DD dd_shfl_up(DD v, int o) {
    return DD{__shfl_up_sync(GR_FULL, v.hi, o), __shfl_up_sync(GR_FULL, v.lo, o)};
}

template <int D>
__device__ __forceinline__ BodyDD bdd_shfl_up(const BodyDD &v, int o) {
    return BodyDD{dd_shfl_up(v.m, o), dd_shfl_up(v.c0, o), dd_shfl_up(v.c1, o),
                  D == 3 ? dd_shfl_up(v.c2, o) : DD{0.0, 0.0}};
}

// a + b for a double-double a and a double b (two-sum, renormalised).
__device__ __forceinline__ DD dd_add_d(DD a, double b) {
    const double s = a.hi + b;
    const double bb = s - a.hi;
    double e = (a.hi - (s - bb)) + (b - bb);
    e += a.lo;
    const double hi = s + e;
    return DD{hi, e - (hi - s)};
}

template <int D>
__device__ __forceinline__ BodyDD bdd_add_body(const BodyDD &a, const Body &b) {
    return BodyDD{dd_add_d(a.m, b.m), dd_add_d(a.c0, b.c0), dd_add_d(a.c1, b.c1),
                  D == 3 ? dd_add_d(a.c2, b.c2) : DD{0.0, 0.0}};
}

// A point's exact FP64 terms: m and m * x per axis (a product of two FP32
// values is exact in FP64).
template <int D>
__device__ __forceinline__ Body point_body(const float4 &p) {
    const double m = (double)p.w;
    return Body{m, m * (double)p.x, m * (double)p.y, D == 3 ? m * (double)p.z : 0.0};
}

template <int D>
__device__ __forceinline__ Body body_sum(const Body &a, const Body &b) {
    return Body{a.m + b.m, a.c0 + b.c0, a.c1 + b.c1, D == 3 ? a.c2 + b.c2 : 0.0};
}

__device__ __forceinline__ double shfl_up_d(double v, int o) { return __shfl_up_sync(GR_FULL, v, o); }

// Exclusive block scan (AG_T threads) of one (FP64 Body, count) per thread in
// a fixed shape: Hillis-Steele warp scans, then a scan of the warp totals.
// Gives this thread's exclusive prefixes and the block totals (the same values
// for the same inputs, whichever kernel asks). s_w and s_c hold 2 AG_W entries.
template <int D>
__device__ __forceinline__ void block_scan_body(const Body &x, uint32_t c, Body &ex, uint32_t &exc, Body &total,
                                                uint32_t &tcnt, Body *s_w, uint32_t *s_c) {
    const int lane = threadIdx.x % GR_WARP, w = threadIdx.x / GR_WARP;
    Body inc = x;
    uint32_t ci = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const Body u{shfl_up_d(inc.m, o), shfl_up_d(inc.c0, o), shfl_up_d(inc.c1, o),
                     D == 3 ? shfl_up_d(inc.c2, o) : 0.0};
        const uint32_t cu = __shfl_up_sync(GR_FULL, ci, o);
        if (lane >= o) {
            inc = body_sum<D>(u, inc);
            ci += cu;
        }
    }
    if (lane == 31) {
        s_w[w] = inc;
        s_c[w] = ci;
    }
    __syncthreads();
    if (w == 0) {
        Body t = lane < AG_W ? s_w[lane] : Body{0.0, 0.0, 0.0, 0.0};
        uint32_t tc = lane < AG_W ? s_c[lane] : 0u;
#pragma unroll
        for (int o = 1; o < AG_W; o <<= 1) {
            const Body u{shfl_up_d(t.m, o), shfl_up_d(t.c0, o), shfl_up_d(t.c1, o), D == 3 ? shfl_up_d(t.c2, o) : 0.0};
            const uint32_t cu = __shfl_up_sync(GR_FULL, tc, o);
            if (lane >= o) {
                t = body_sum<D>(u, t);
                tc += cu;
            }
        }
        if (lane < AG_W) {
            s_w[AG_W + lane] = t;
            s_c[AG_W + lane] = tc;
        }
    }
    __syncthreads();
    const Body before = w > 0 ? s_w[AG_W + w - 1] : Body{0.0, 0.0, 0.0, 0.0};
    const uint32_t cbefore = w > 0 ? s_c[AG_W + w - 1] : 0u;
    total = s_w[2 * AG_W - 1];
    tcnt = s_c[2 * AG_W - 1];
    Body lanes_before{shfl_up_d(inc.m, 1), shfl_up_d(inc.c0, 1), shfl_up_d(inc.c1, 1),
                      D == 3 ? shfl_up_d(inc.c2, 1) : 0.0};  // inclusive scan of the lane before
    uint32_t clb = __shfl_up_sync(GR_FULL, ci, 1);
    if (lane == 0) {
        lanes_before = Body{0.0, 0.0, 0.0, 0.0};
        clb = 0;
    }
    __syncthreads();
    ex = body_sum<D>(before, lanes_before);
    exc = cbefore + clb;
}

// The stored prefix of leaf s: the FP64 in-tile part, D + 1 doubles (the mass,
// then the D mass moments; 24 B in 2D) stored at the leaf's first point, beside
// the double-double carry of the tile that holds that point (carry[nt] is the
// grand total, and point n, leaf nu's start, has in-tile part 0). The prefix is
// carry + in-tile part.
struct Prefix {
    const double *local;  // (n + 1) x (D + 1), at each leaf's first point (and 0 at point n)
    const BodyDD *carry;  // nt + 1
    const uint32_t *leaf_start;
    uint32_t nu, nt;
};

template <int D>
__device__ __forceinline__ void local_put(double *__restrict__ pre, uint32_t s, const Body &b) {
    double *q = pre + (size_t)s * (D + 1);
    q[0] = b.m;
    q[1] = b.c0;
    q[2] = b.c1;
    if (D == 3) q[3] = b.c2;
}

template <int D>
__device__ __forceinline__ BodyDD prefix_at(const Prefix &P, uint32_t s) {
    const uint32_t p = P.leaf_start[s];  // leaf_start[nu] = n
    const double *q = P.local + (size_t)p * (D + 1);
    const Body b{q[0], q[1], q[2], D == 3 ? q[3] : 0.0};
    const uint32_t tile = s >= P.nu ? P.nt : p / AG_TILE;
    return bdd_add_body<D>(P.carry[tile], b);
}

// This thread's AG_I consecutive sorted points p0 .. p0 + AG_I - 1 (< n): their
// keys, the "first of its key" bits (fl) and their FP64 terms summed in order.
template <int D>
__device__ __forceinline__ Body point_chunk(uint32_t n, uint32_t p0, const float4 *__restrict__ pts,
                                            const uint64_t *__restrict__ keys, uint64_t *k, uint32_t &fl) {
    const uint64_t kprev = (p0 > 0 && p0 <= n) ? keys[p0 - 1] : 0ull;
#pragma unroll
    for (int r = 0; r < AG_I; r++) k[r] = p0 + r < n ? keys[p0 + r] : 0ull;
    Body acc{0.0, 0.0, 0.0, 0.0};
    fl = 0;
#pragma unroll
    for (int r = 0; r < AG_I; r++) {
        const uint32_t p = p0 + r;
        if (p < n) {
            const bool f = p == 0 || k[r] != (r == 0 ? kprev : k[r - 1]);
            fl |= (f ? 1u : 0u) << r;
            acc = body_sum<D>(acc, point_body<D>(pts[r]));
        }
    }
    return acc;
}

// (1 of 2) Tile b of AG_TILE sorted points: the sorted point records sp[p] =
// pos[perm[p]], sorig[p] = perm[p]; the tile's FP64 term sums and its count of
// leaves (points that start a key), as block_scan_body totals them.
template <int D>
__global__ void __launch_bounds__(AG_T)
k_leaf_tiles(DevState *st, uint32_t n, const float4 *__restrict__ pos, const uint64_t *__restrict__ keys,
             const uint32_t *__restrict__ perm, float4 *__restrict__ sp, uint32_t *__restrict__ sorig,
             Body *__restrict__ tile_sum, uint32_t *__restrict__ tile_cnt, uint32_t *__restrict__ uid,
             double *__restrict__ pre) {
    gr_pdl_enter();
    if (st->converged) return;
    __shared__ Body s_w[2 * AG_W];
    __shared__ uint32_t s_c[2 * AG_W];
    const uint32_t b = blockIdx.x;
    const uint32_t p0 = b * AG_TILE + threadIdx.x * AG_I;
    uint32_t q[AG_I];
    float4 pt[AG_I];
#pragma unroll
    for (int r = 0; r < AG_I; r++) {
        q[r] = p0 + r < n ? perm[p0 + r] : 0u;
        if (q[r] >= n) {  // only after a sort pass gave up a wait (ERR_WAIT): keep the reads in bounds
            atomicOr(&st->error, (uint32_t)ERR_TREE);
            q[r] = 0;
        }
    }
#pragma unroll
    for (int r = 0; r < AG_I; r++) pt[r] = p0 + r < n ? pos[q[r]] : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int r = 0; r < AG_I; r++)
        if (p0 + r < n) {
            sp[p0 + r] = pt[r];
            sorig[p0 + r] = q[r];
        }
    uint64_t k[AG_I];
    uint32_t fl;
    const Body acc = point_chunk<D>(n, p0, pt, keys, k, fl);
    Body ex, total;
    uint32_t exc, tcnt;
    block_scan_body<D>(acc, (uint32_t)__popc(fl), ex, exc, total, tcnt, s_w, s_c);
    if (threadIdx.x == 0) {
        tile_sum[b] = total;
        tile_cnt[b] = tcnt;
    }
    // at each leaf's first point, the in-tile part of its prefix (indexed by the
    // point: it needs no carry); every point's in-tile leaf rank + 1 (0: its leaf
    // began in an earlier tile), bit 31 set at a leaf's first point
    uint32_t e = exc;
    Body run = ex;
#pragma unroll
    for (int r = 0; r < AG_I; r++) {
        const uint32_t p = p0 + r;
        if (p < n) {
            const bool f = (fl >> r) & 1u;
            if (f) {
                local_put<D>(pre, p, run);
                e++;
            }
            uid[p] = e | (f ? 0x80000000u : 0u);
            run = body_sum<D>(run, point_body<D>(pt[r]));
        }
    }
}

__device__ __forceinline__ DD dd_shfl_down(DD v, int o) {
    return DD{__shfl_down_sync(GR_FULL, v.hi, o), __shfl_down_sync(GR_FULL, v.lo, o)};
}

template <int D>
__device__ __forceinline__ BodyDD bdd_shfl_down(const BodyDD &v, int o) {
    return BodyDD{dd_shfl_down(v.m, o), dd_shfl_down(v.c0, o), dd_shfl_down(v.c1, o),
                  D == 3 ? dd_shfl_down(v.c2, o) : DD{0.0, 0.0}};
}

// Up to this many tiles each leaf-prefix block folds the tile sums before its
// own (at most 2,047 x 36 B of L2 reads a block); above it one block computes
// every carry (k_leaf_carry).
constexpr uint32_t LEAF_FOLD_MAX_TILES = 2048;

// The double-double sum of the tile sums before tile b and the count of the
// leaves they start, folded by the calling block (AG_T threads) in a fixed
// shape: thread t adds tiles t, t + AG_T, ... < b in turn, the lanes of a warp
// combine by a shuffle-down tree into lane 0, and one thread adds the warp
// totals in warp order. s_bw / s_bc hold AG_W + 1 entries.
template <int D>
__device__ __forceinline__ void tiles_before(uint32_t b, const Body *__restrict__ tile_sum,
                                             const uint32_t *__restrict__ tile_cnt, BodyDD &carry, uint32_t &count,
                                             BodyDD *s_bw, uint32_t *s_bc) {
    constexpr int U = 2;  // tile sums in flight per thread
    BodyDD acc{};
    uint32_t c = 0;
    for (uint32_t j0 = threadIdx.x; j0 < b; j0 += U * AG_T) {
        Body v[U];
        uint32_t k[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const uint32_t j = j0 + u * AG_T;
            v[u] = j < b ? tile_sum[j] : Body{0.0, 0.0, 0.0, 0.0};
            k[u] = j < b ? tile_cnt[j] : 0u;
        }
#pragma unroll
        for (int u = 0; u < U; u++)
            if (j0 + u * AG_T < b) {
                acc = bdd_add_body<D>(acc, v[u]);
                c += k[u];
            }
    }
    const int lane = threadIdx.x % GR_WARP, w = threadIdx.x / GR_WARP;
#pragma unroll
    for (int o = GR_WARP / 2; o >= 1; o >>= 1) {
        const BodyDD u = bdd_shfl_down<D>(acc, o);
        const uint32_t cu = __shfl_down_sync(GR_FULL, c, o);
        if (lane < o) {
            acc = bdd_add<D>(acc, u);
            c += cu;
        }
    }
    if (lane == 0) {
        s_bw[w] = acc;
        s_bc[w] = c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        BodyDD t = s_bw[0];
        uint32_t tc = s_bc[0];
        for (int q = 1; q < AG_W; q++) {
            t = bdd_add<D>(t, s_bw[q]);
            tc += s_bc[q];
        }
        s_bw[AG_W] = t;
        s_bc[AG_W] = tc;
    }
    __syncthreads();
    carry = s_bw[AG_W];
    count = s_bc[AG_W];
}

constexpr int CARRY_T = 1024;  // a multiple of 32, at most 1024

// One block, for graphs of more than LEAF_FOLD_MAX_TILES tiles (where each
// block's own fold of the tiles before it, tiles_before, would cost O(tiles^2)
// reads in all): the exclusive double-double prefix of the tile sums and
// the exclusive prefix of the tile leaf counts, in a fixed order (thread t
// folds tiles [t c, t c + c) in turn, then a fixed-shape scan over the
// threads). Writes n_unique, leaf_start[n_unique] = n, the grand total as
// carry[nt] and a zero in-tile part for leaf n_unique.
template <int D>
__global__ void __launch_bounds__(CARRY_T)
k_leaf_carry(DevState *st, uint32_t n, const Body *__restrict__ tile_sum, const uint32_t *__restrict__ tile_cnt,
             BodyDD *__restrict__ carry, uint32_t *__restrict__ ccarry, uint32_t *__restrict__ leaf_start,
             double *__restrict__ pre) {
    gr_pdl_enter();
    if (st->converged) return;
    constexpr int W = CARRY_T / GR_WARP;
    __shared__ BodyDD s_w[W];
    __shared__ uint32_t s_c[W];
    const uint32_t nt = (n + AG_TILE - 1) / AG_TILE;
    const uint32_t per = (nt + CARRY_T - 1) / CARRY_T;
    const uint32_t t0 = threadIdx.x * per, t1 = min(t0 + per, nt);
    BodyDD acc{};
    uint32_t cacc = 0;
    for (uint32_t j = t0; j < t1; j++) {
        acc = bdd_add_body<D>(acc, tile_sum[j]);
        cacc += tile_cnt[j];
    }
    const int lane = threadIdx.x % GR_WARP, w = threadIdx.x / GR_WARP;
    BodyDD inc = acc;
    uint32_t ci = cacc;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const BodyDD u = bdd_shfl_up<D>(inc, o);
        const uint32_t cu = __shfl_up_sync(GR_FULL, ci, o);
        if (lane >= o) {
            inc = bdd_add<D>(u, inc);
            ci += cu;
        }
    }
    if (lane == 31) {
        s_w[w] = inc;
        s_c[w] = ci;
    }
    __syncthreads();
    if (w == 0) {
        BodyDD t = lane < W ? s_w[lane] : BodyDD{};
        uint32_t tc = lane < W ? s_c[lane] : 0u;
#pragma unroll
        for (int o = 1; o < W; o <<= 1) {
            const BodyDD u = bdd_shfl_up<D>(t, o);
            const uint32_t cu = __shfl_up_sync(GR_FULL, tc, o);
            if (lane >= o) {
                t = bdd_add<D>(u, t);
                tc += cu;
            }
        }
        if (lane < W) {
            s_w[lane] = t;  // inclusive over warps 0 .. lane
            s_c[lane] = tc;
        }
    }
    __syncthreads();
    BodyDD lanes_before = bdd_shfl_up<D>(inc, 1);
    uint32_t clb = __shfl_up_sync(GR_FULL, ci, 1);
    if (lane == 0) {
        lanes_before = BodyDD{};
        clb = 0;
    }
    BodyDD run = bdd_add<D>(w > 0 ? s_w[w - 1] : BodyDD{}, lanes_before);
    uint32_t crun = (w > 0 ? s_c[w - 1] : 0u) + clb;
    for (uint32_t j = t0; j < t1; j++) {
        carry[j] = run;
        ccarry[j] = crun;
        run = bdd_add_body<D>(run, tile_sum[j]);
        crun += tile_cnt[j];
    }
    if (threadIdx.x == CARRY_T - 1) {  // the last thread's run is the grand total
        const uint32_t nu = min(crun, n);
        st->n_unique = nu;
        leaf_start[nu] = n;
        carry[nt] = run;
        local_put<D>(pre, n, Body{0.0, 0.0, 0.0, 0.0});  // the in-tile part at leaf_start[nu] = n
    }
}

// (2 of 2) Tile b again: the double-double carry of the tiles before it (its
// own fold of their sums, tiles_before, or with ccarry k_leaf_carry's, for
// more than LEAF_FOLD_MAX_TILES tiles); every point's leaf index uid[p] (its
// in-tile rank from k_leaf_tiles plus the leaves before the tile); at a leaf's
// first point leaf_start, ukey and an empty cell level mask. The last tile also
// writes n_unique, leaf_start[n_unique] = n, the grand total as carry[nt] and a
// zero in-tile part at point n.
template <int D>
__global__ void __launch_bounds__(AG_T)
k_leaf_prefix(DevState *st, uint32_t n, const uint64_t *__restrict__ keys, const Body *__restrict__ tile_sum,
              const uint32_t *__restrict__ tile_cnt, BodyDD *__restrict__ carry, const uint32_t *__restrict__ ccarry,
              uint32_t *__restrict__ uid, uint32_t *__restrict__ leaf_start, uint64_t *__restrict__ ukey,
              uint32_t *__restrict__ levels, double *__restrict__ pre) {
    gr_pdl_enter();
    if (st->converged) return;
    __shared__ BodyDD s_bw[AG_W + 1];
    __shared__ uint32_t s_bc[AG_W + 1];
    const uint32_t b = blockIdx.x;
    BodyDD cb;
    uint32_t cbefore;
    if (ccarry) {  // k_leaf_carry wrote the carries, the totals and n_unique
        cbefore = ccarry[b];
    } else {
        tiles_before<D>(b, tile_sum, tile_cnt, cb, cbefore, s_bw, s_bc);
    }
    if (!ccarry && threadIdx.x == 0) {
        carry[b] = cb;
        if (b + 1 == gridDim.x) {
            const uint32_t nu = min(cbefore + tile_cnt[b], n);
            st->n_unique = nu;
            leaf_start[nu] = n;
            carry[b + 1] = bdd_add_body<D>(cb, tile_sum[b]);
            local_put<D>(pre, n, Body{0.0, 0.0, 0.0, 0.0});
        }
    }
    const uint32_t p0 = b * AG_TILE + threadIdx.x * AG_I;
    uint32_t v[AG_I];
#pragma unroll
    for (int r = 0; r < AG_I; r++) v[r] = p0 + r < n ? uid[p0 + r] : 0u;
#pragma unroll
    for (int r = 0; r < AG_I; r++) {
        const uint32_t p = p0 + r;
        if (p < n) {
            const uint32_t e = cbefore + (v[r] & 0x7fffffffu) - 1u;  // the point's leaf
            uid[p] = e;
            if ((v[r] >> 31) && e < n) {  // e < n unless a sort pass gave up a wait
                leaf_start[e] = p;
                ukey[e] = keys[p];
                levels[e] = 0;
            }
        }
    }
}

// Internal node i covers leaves [first, last]: its sums are prefix[last + 1] -
// prefix[first].
__device__ __forceinline__ Body range_body(const BodyDD &a, const BodyDD &b) {
    return Body{dd_diff(b.m, a.m), dd_diff(b.c0, a.c0), dd_diff(b.c1, a.c1), dd_diff(b.c2, a.c2)};
}

// Every internal node's body as an array (the adjoint reads them; the tick's
// own cell writer takes range_body of the cells only).
template <int D>
__global__ void k_node_body(const DevState *st, BinTree t, Prefix pre, Body *__restrict__ int_body) {
    if (st->converged) return;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    pre.nu = st->n_unique;
    if (i + 1 >= pre.nu) return;
    body_store(&int_body[i], range_body(prefix_at<D>(pre, t.first[i]), prefix_at<D>(pre, t.last[i] + 1)));
}

template <int D>
__device__ __forceinline__ bool is_cell(const BinTree &t, int32_t node) {
    int32_t par = t.int_parent[node];
    return par < 0 || (t.delta[node] / D) != (t.delta[par] / D);
}

// Cell record, 2D: A = {cx, cy, mass, w^2}, B = {cx_lo, cy_lo, skip | -count, start}.
// 3D: A = {cx, cy, cz, mass}, B = {cx_lo, cy_lo, cz_lo, w^2}, C = {skip | -count, start, -, -}.
// The centre is an FP32 hi/lo pair of the FP64 centre of mass, so a node at
// 1e4 still resolves a nearby centre to ~1e-3 ulp instead of a whole FP32 ulp.
// In 2D the A and B records are two arrays (rec[k], rec_b[k]): the 32 lanes of a
// walk warp visit different but nearby cells, and one 32-byte sector of the A
// array holds two cells' A (measured: a per-cell 32-byte record made the 2D
// per-lane walk 13% slower). In 3D a cell's records lie together (rec[3k + 0] =
// A, + 1 = B, + 2 = C): one line per visit instead of three (the 3D walk 6%
// faster than with three arrays).
template <int D> struct CellF { static constexpr uint32_t F = D == 3 ? 3 : 1; };  // float4s per cell in rec

struct Cells {
    float4 *rec;     // 2D: A of cell k at rec[k]; 3D: cell k's A, B, C at rec[3k ..]
    float4 *rec_b;   // 2D: B of cell k at rec_b[k]; 3D: unused
    float4 *bounds;  // nullable: each cell's square {x0, y0, x1, y1} (2D), for range pruning
};

template <int D>
__device__ __forceinline__ float4 cell_a(const Cells &c, uint32_t k) {
    return __ldg(&c.rec[(size_t)k * CellF<D>::F]);
}
template <int D>
__device__ __forceinline__ float4 cell_b(const Cells &c, uint32_t k) {
    return D == 3 ? __ldg(&c.rec[(size_t)k * 3 + 1]) : __ldg(&c.rec_b[k]);
}
__device__ __forceinline__ int2 cell_c3(const Cells &c, uint32_t k) {  // 3D: {skip | -count, start}
    const float4 v = __ldg(&c.rec[(size_t)k * 3 + 2]);
    return make_int2(__float_as_int(v.x), __float_as_int(v.y));
}

// Float4 records a cells buffer holds for `cap` cells, and its two views.
__host__ __device__ inline size_t cells_float4s(uint32_t cap, int dim) { return (size_t)cap * (dim == 3 ? 3 : 2); }
__host__ __device__ inline Cells cells_view(float4 *buf, uint32_t cap, int dim) {
    Cells c;
    c.rec = buf;
    c.rec_b = dim == 3 ? nullptr : buf + cap;
    c.bounds = nullptr;
    return c;
}

// The square of the level-`level` cell holding point p: the root corner plus
// floor((p - corner) / w) sides, exact in FP64 (w is a power of two times the
// root side). Rounded to FP32 it still contains every point of the cell.
__device__ __forceinline__ void write_bounds(Cells c, uint32_t idx, const float4 &p, int level, const DevState *st) {
    const double w = ldexp(st->root_w, -level);
    const double bx = st->root0[0] + floor(((double)p.x - st->root0[0]) / w) * w;
    const double by = st->root0[1] + floor(((double)p.y - st->root0[1]) / w) * w;
    c.bounds[idx] = make_float4((float)bx, (float)by, (float)(bx + w), (float)(by + w));
}

template <int D>
__device__ __forceinline__ void write_cell(Cells c, uint32_t idx, const Body &b, int level, double root_w,
                                           int32_t skip_or_count, uint32_t start, const float4 *point = nullptr) {
    double inv = 1.0 / b.m;
    double cc[3] = {b.c0 * inv, b.c1 * inv, b.c2 * inv};
    if (point) {  // a one-point leaf's centre is the point itself, exactly
        cc[0] = point->x;
        cc[1] = point->y;
        cc[2] = point->z;
    }
    float hi[3], lo[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        hi[a] = (float)cc[a];
        lo[a] = (float)(cc[a] - (double)hi[a]);
    }
    double w = ldexp(root_w, -level);
    float w2 = (float)(w * w);
    float4 *r = c.rec + (size_t)idx * CellF<D>::F;
    if (D == 2) {
        r[0] = make_float4(hi[0], hi[1], (float)b.m, w2);
        c.rec_b[idx] = make_float4(lo[0], lo[1], __int_as_float(skip_or_count), __uint_as_float(start));
    } else {
        r[0] = make_float4(hi[0], hi[1], hi[2], (float)b.m);
        r[1] = make_float4(lo[0], lo[1], lo[2], w2);
        r[2] = make_float4(__int_as_float(skip_or_count), __uint_as_float(start), 0.f, 0.f);
    }
}

// Every cell at its preorder index, without walking chains: threads
// [0, n_slots) take unique leaf s = thread (its cell is the last of the
// 1 + popc(levels[s]) cells beginning at s), threads [n_slots, 2 n_slots) take
// internal node i = thread - n_slots when it is a cell (level l, first leaf f:
// index P[f] + popc(levels[f] & (2^l - 1))). A leaf's body comes from its
// points (leaf_sum), an internal cell's from the prefix at its range ends
// (range_body); skip(cell) = P[last leaf + 1]. A leaf of coincident points sits
// one level below its parent cell (where the reference chains them); a leaf of
// distinct points the key could not separate sits at the key's last level.
template <int D>
__global__ void k_assign_cells(const DevState *st, BinTree t, uint32_t n_slots, const float4 *__restrict__ sp,
                               const uint32_t *__restrict__ P, const uint32_t *__restrict__ levels,
                               const uint32_t *__restrict__ leaf_start, Prefix pre,
                               Cells cells, uint32_t *__restrict__ leaf_pre,
                               DevState *stw) {
    gr_pdl_enter();
    if (st->converged) return;
    constexpr int L = Levels<D>::L;
    const uint32_t nu = st->n_unique;
    const uint32_t ncells = st->n_cells;
    const double rw = st->root_w;
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < n_slots) {
        const uint32_t s = g;
        if (s >= nu) return;
        const uint32_t idx = P[s] + __popc(levels[s]);
        const uint32_t a0 = leaf_start[s], a1 = leaf_start[s + 1];
        if (idx >= ncells || a1 <= a0) {
            atomicOr(&stw->error, (uint32_t)ERR_TREE);
            return;
        }
        const float4 one = sp[a0];
        bool coinc;
        const Body body = leaf_sum<D>(sp, a0, a1, coinc);
        // the parent's record only for coincident points (one leaf alone is the root)
        const int level = nu == 1 ? 0 : coinc ? t.rec[t.leaf_parent[s]].w / D + 1 : L;
        write_cell<D>(cells, idx, body, level, rw, -(int32_t)(a1 - a0), a0, a1 - a0 == 1 ? &one : nullptr);
        if (D == 2 && cells.bounds) write_bounds(cells, idx, one, level, st);
        leaf_pre[s] = idx;
        return;
    }
    const uint32_t i = g - n_slots;
    if (i + 1 >= nu || !t.cell_flag[i]) return;
    const int4 R = t.rec[i];
    const int lv = R.w / D;
    const uint32_t f = (uint32_t)R.x, end = (uint32_t)R.y + 1;
    const uint32_t idx = P[f] + __popc(levels[f] & ((1u << lv) - 1u));
    const uint32_t skip = end == nu ? ncells : P[end];
    if (idx >= ncells || skip <= idx || skip > ncells) {
        atomicOr(&stw->error, (uint32_t)ERR_TREE);
        return;
    }
    const uint32_t a0 = leaf_start[f];
    pre.nu = nu;
    write_cell<D>(cells, idx, range_body(prefix_at<D>(pre, f), prefix_at<D>(pre, end)), lv, rw, (int32_t)skip, a0);
    if (D == 2 && cells.bounds) write_bounds(cells, idx, sp[a0], lv, st);
    if (t.cell_of) t.cell_of[i] = idx;
}

}  // namespace gr
