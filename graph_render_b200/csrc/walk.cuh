// Repulsion: warp-cooperative stackless preorder walk of the linear tree.
//
// Reference: crates/graph-core/src/layout/forceatlas2/state/barnes_hut.rs:115-184.
// Per node, in preorder: a cell that does not hold the node, with d2 > 0 and
// w^2 < theta^2 d2 (d to the cell's centre of mass, w its side), acts as one body
// of its mass and the walk skips its subtree; a leaf that is not far acts pair by
// pair (with the coincident-pair jiggle, state.rs:185-203); anything else opens.
//
// On the GPU a warp walks 32 consecutive Morton-sorted nodes together. The cell
// index k is warp-uniform; each lane keeps `resume`, the first cell index it
// takes part in again after it approximated a subtree (its skip). The warp
// descends (k + 1) when any participating lane opens the cell and jumps to
// skip otherwise; lanes never see a cell their own walk would not visit, so each
// node's interaction set is exactly the per-node walk's. Cell loads are
// warp-uniform broadcasts of float4 records; leaf points come from the sorted
// float4 node array.
#pragma once

#include "common.cuh"
#include "tree.cuh"

namespace gr {

constexpr int WALK_THREADS = 256;  // measured at 1M 2D nodes: 64 and 128 threads slower (by 3.5% / 1.6% of the walk)

struct WalkParams {
    uint32_t n;
    float kr;      // scaling_ratio
    float theta2;  // theta^2
    uint32_t seed;
};

// What one walk reads: the tree of this tick and the sorted nodes.
struct WalkView {
    Cells cells;
    const float4 *sp;
    const uint32_t *sorig, *uid, *leaf_pre;
    uint32_t n, ncells, iter, seed;
    float kr, th2;
    uint32_t *err;
};

// The whole warp calls this for the sorted nodes p = base + lane (lanes with
// p >= n take part in the votes only). Returns each lane's repulsion and its
// far / pair interaction counts.
template <int D, bool COUNT = true>
__device__ __forceinline__ void walk_group(const WalkView &V, uint32_t p, float &f0, float &f1, float &f2,
                                           uint32_t &nfar, uint32_t &npair) {
    const Cells cells = V.cells;
    const float4 *__restrict__ sp = V.sp;
    const uint32_t n = V.n, ncells = V.ncells, iter = V.iter;
    const bool valid = p < n;
    const float4 me = valid ? sp[p] : make_float4(0.f, 0.f, 0.f, 0.f);
    const uint32_t mylp = valid ? V.leaf_pre[V.uid[p]] : 0xffffffffu;
    const uint32_t oi = valid ? V.sorig[p] : 0u;
    uint32_t resume = valid ? 0u : 0xffffffffu;
    f0 = f1 = f2 = 0.f;
    nfar = npair = 0;
    const float th2 = V.th2, mk = me.w * V.kr;
    const uint32_t lane = threadIdx.x % GR_WARP;

    uint32_t k = 0;
    while (k < ncells) {
        const float4 A = cell_a<D>(cells, k);
        const float4 B = cell_b<D>(cells, k);
        int32_t sk;
        uint32_t start;
        float cx, cy, cz, cm, w2, lx, ly, lz;
        if (D == 2) {
            cx = A.x; cy = A.y; cz = 0.f; cm = A.z; w2 = A.w;
            lx = B.x; ly = B.y; lz = 0.f;
            sk = __float_as_int(B.z);
            start = __float_as_uint(B.w);
        } else {
            const int2 Cc = cell_c3(cells, k);
            cx = A.x; cy = A.y; cz = A.z; cm = A.w;
            lx = B.x; ly = B.y; lz = B.z; w2 = B.w;
            sk = Cc.x;
            start = (uint32_t)Cc.y;
        }
        const bool leaf = sk < 0;
        uint32_t skip = leaf ? k + 1 : (uint32_t)sk;
        if (skip <= k || skip > ncells) {  // malformed cell: record it, keep the walk finite
            if (lane == 0) atomicOr(V.err, (uint32_t)ERR_TREE);
            skip = k + 1;
        }
        const bool active = resume <= k;
        const bool holds = (k <= mylp) && (mylp < skip);
        const float dx = (me.x - cx) - lx;
        const float dy = (me.y - cy) - ly;
        const float dz = (D == 3) ? (me.z - cz) - lz : 0.f;
        const float d2 = (D == 3) ? dx * dx + dy * dy + dz * dz : dx * dx + dy * dy;
        const bool far = active && !holds && d2 > 0.f && w2 < th2 * d2;
        if (far) {
            const float f = __fdividef(mk * cm, d2);
            f0 += dx * f;
            f1 += dy * f;
            if (D == 3) f2 += dz * f;
            resume = skip;
            if (COUNT) nfar++;
        }
        const bool open = active && !far;
        if (sk == -1) {
            // One-point leaf: the exact pair (barnes_hut.rs:163-184) is the body
            // term above with the point as its own centre; only an exact
            // coincidence (d2 == 0) takes repel_delta's jiggle.
            if (open && !holds) {
                float ex = dx, ey = dy, ez = dz, e2 = d2;
                if (!(d2 > 0.f)) {
                    const uint32_t oj = __ldg(&V.sorig[start]);
                    const float sg = oi < oj ? 1.f : -1.f;
                    ex = sg * (float)jiggle(V.seed, iter, 0, oi, oj);
                    ey = sg * (float)jiggle(V.seed, iter, 1, oi, oj);
                    if (D == 3) ez = sg * (float)jiggle(V.seed, iter, 2, oi, oj);
                    e2 = (D == 3) ? ex * ex + ey * ey + ez * ez : ex * ex + ey * ey;
                }
                const float f = __fdividef(mk * cm, e2);
                f0 += ex * f;
                f1 += ey * f;
                if (D == 3) f2 += ez * f;
                if (COUNT) npair++;
            }
            k = k + 1;
        } else if (leaf) {
            if (__any_sync(GR_FULL, open)) {
                int32_t cnt = -sk;
                if (start >= n || (uint32_t)cnt > n - start) {
                    if (lane == 0) atomicOr(V.err, (uint32_t)ERR_TREE);
                    cnt = 0;
                }
                for (int32_t q = 0; q < cnt; q++) {
                    const uint32_t jp = start + (uint32_t)q;
                    const float4 o = __ldg(&sp[jp]);
                    if (open && jp != p) {
                        float ex = me.x - o.x, ey = me.y - o.y, ez = (D == 3) ? me.z - o.z : 0.f;
                        if (ex == 0.f && ey == 0.f && (D == 2 || ez == 0.f)) {
                            // repel_delta's jiggle, taken from the lower index
                            const uint32_t oj = __ldg(&V.sorig[jp]);
                            const float sg = oi < oj ? 1.f : -1.f;
                            ex = sg * (float)jiggle(V.seed, iter, 0, oi, oj);
                            ey = sg * (float)jiggle(V.seed, iter, 1, oi, oj);
                            if (D == 3) ez = sg * (float)jiggle(V.seed, iter, 2, oi, oj);
                        }
                        const float e2 = (D == 3) ? ex * ex + ey * ey + ez * ez : ex * ex + ey * ey;
                        const float f = __fdividef(mk * o.w, e2);
                        f0 += ex * f;
                        f1 += ey * f;
                        if (D == 3) f2 += ez * f;
                        if (COUNT) npair++;
                    }
                }
            }
            k = k + 1;
        } else {
            k = __any_sync(GR_FULL, open) ? k + 1 : skip;
        }
    }
}

// The same per-node walk with every lane on its own cell index (gathered cell
// loads, no warp vote): the warp runs as long as its longest path instead of
// the union of its 32 paths. Each lane meets its cells in the same preorder and
// adds the same terms in the same order as walk_group, so the forces are
// bit-identical; only the schedule differs.
// One node's per-lane walk, as state and one cell visit at a time.
struct LaneNode {
    float4 me;
    uint32_t p, mylp, oi, k;
    float mk, f0, f1, f2;
    uint32_t nfar, npair;
};

template <int D>
__device__ __forceinline__ void lane_init(const WalkView &V, uint32_t p, LaneNode &X) {
    const bool valid = p < V.n;
    X.p = p;
    X.me = valid ? V.sp[p] : make_float4(0.f, 0.f, 0.f, 0.f);
    X.mylp = valid ? V.leaf_pre[V.uid[p]] : 0u;
    X.oi = valid ? V.sorig[p] : 0u;
    X.mk = X.me.w * V.kr;
    X.f0 = X.f1 = X.f2 = 0.f;
    X.nfar = X.npair = 0;
    X.k = valid ? 0u : V.ncells;
}

// One cell's records as the walk reads them (C only in 3D).
struct CellRec {
    float4 A, B;
    int2 C;
};

template <int D>
__device__ __forceinline__ CellRec cell_rec(const Cells &cells, uint32_t k) {
    CellRec r;
    r.A = cell_a<D>(cells, k);
    r.B = cell_b<D>(cells, k);
    r.C = D == 3 ? cell_c3(cells, k) : make_int2(0, 0);
    return r;
}

// The visit of cell X.k (X.k < ncells) whose records are R: a body term, a
// leaf's pairs, or a descent; X.k moves on. COUNT: keep the far / pair
// interaction counts.
template <int D, bool COUNT = true>
__device__ __forceinline__ void lane_visit(const WalkView &V, LaneNode &X, const CellRec &R) {
    const float4 *__restrict__ sp = V.sp;
    const uint32_t n = V.n, iter = V.iter, k = X.k, oi = X.oi;
    const float4 me = X.me;
    const float th2 = V.th2, mk = X.mk;
    const float4 A = R.A;
    const float4 B = R.B;
    int32_t sk;
    uint32_t start;
    float cx, cy, cz, cm, w2, lx, ly, lz;
    if (D == 2) {
        cx = A.x; cy = A.y; cz = 0.f; cm = A.z; w2 = A.w;
        lx = B.x; ly = B.y; lz = 0.f;
        sk = __float_as_int(B.z);
        start = __float_as_uint(B.w);
    } else {
        const int2 Cc = R.C;
        cx = A.x; cy = A.y; cz = A.z; cm = A.w;
        lx = B.x; ly = B.y; lz = B.z; w2 = B.w;
        sk = Cc.x;
        start = (uint32_t)Cc.y;
    }
    const bool leaf = sk < 0;
    // a leaf (sk < 0) moves on to k + 1, a cell to its skip; every step moves
    // forward, whatever a cell holds (k < ncells <= 2^31)
    const uint32_t skip = (uint32_t)max(sk, (int32_t)k + 1);
    const bool holds = (k <= X.mylp) && (X.mylp < skip);
    const float dx = (me.x - cx) - lx;
    const float dy = (me.y - cy) - ly;
    const float dz = (D == 3) ? (me.z - cz) - lz : 0.f;
    const float d2 = (D == 3) ? dx * dx + dy * dy + dz * dz : dx * dx + dy * dy;
    const bool far = !holds && w2 < th2 * d2;  // w2 > 0, so this is false at d2 == 0
    // The common outcomes without a branch: a body term (far cell, or a
    // one-point leaf's pair) is added, anything else adds +-0 (an exact no-op:
    // the sums start at +0 and never hold -0); the walk moves to skip or k + 1.
    const bool body = far || (sk == -1 && !holds && d2 > 0.f);
    const float fb = __fdividef(mk * cm, d2);
    const float f = body ? fb : 0.f;
    X.f0 += dx * f;
    X.f1 += dy * f;
    if (D == 3) X.f2 += dz * f;
    if (COUNT) {
        X.nfar += far ? 1u : 0u;
        X.npair += (body && !far) ? 1u : 0u;
    }
    if (!leaf || body) {
        X.k = body ? skip : k + 1;
    } else if (!holds && sk == -1) {  // coincident one-point leaf: the jiggle
        const uint32_t oj = __ldg(&V.sorig[start]);
        const float sg = oi < oj ? 1.f : -1.f;
        const float ex = sg * (float)jiggle(V.seed, iter, 0, oi, oj);
        const float ey = sg * (float)jiggle(V.seed, iter, 1, oi, oj);
        const float ez = (D == 3) ? sg * (float)jiggle(V.seed, iter, 2, oi, oj) : 0.f;
        const float e2 = (D == 3) ? ex * ex + ey * ey + ez * ez : ex * ex + ey * ey;
        const float g = __fdividef(mk * cm, e2);
        X.f0 += ex * g;
        X.f1 += ey * g;
        if (D == 3) X.f2 += ez * g;
        if (COUNT) X.npair++;
        X.k = k + 1;
    } else {  // several points (or this node's own leaf): exact pairs
        int32_t cnt = -sk;
        if (start >= n || (uint32_t)cnt > n - start) {
            atomicOr(V.err, (uint32_t)ERR_TREE);
            cnt = 0;
        }
        for (int32_t q = 0; q < cnt; q++) {
            const uint32_t jp = start + (uint32_t)q;
            if (jp == X.p) continue;
            const float4 o = __ldg(&sp[jp]);
            float ex = me.x - o.x, ey = me.y - o.y, ez = (D == 3) ? me.z - o.z : 0.f;
            if (ex == 0.f && ey == 0.f && (D == 2 || ez == 0.f)) {
                const uint32_t oj = __ldg(&V.sorig[jp]);
                const float sg = oi < oj ? 1.f : -1.f;
                ex = sg * (float)jiggle(V.seed, iter, 0, oi, oj);
                ey = sg * (float)jiggle(V.seed, iter, 1, oi, oj);
                if (D == 3) ez = sg * (float)jiggle(V.seed, iter, 2, oi, oj);
            }
            const float e2 = (D == 3) ? ex * ex + ey * ey + ez * ez : ex * ex + ey * ey;
            const float g = __fdividef(mk * o.w, e2);
            X.f0 += ex * g;
            X.f1 += ey * g;
            if (D == 3) X.f2 += ez * g;
            if (COUNT) X.npair++;
        }
        X.k = k + 1;
    }
}

// The visit of cell X.k (X.k < ncells), its records loaded here.
template <int D, bool COUNT = true>
__device__ __forceinline__ void lane_step(const WalkView &V, LaneNode &X) {
    lane_visit<D, COUNT>(V, X, cell_rec<D>(V.cells, X.k));
}

template <int D, bool COUNT = true>
__device__ __forceinline__ void walk_lane(const WalkView &V, uint32_t p, float &f0, float &f1, float &f2,
                                          uint32_t &nfar, uint32_t &npair) {
    LaneNode X;
    lane_init<D>(V, p, X);
    while (X.k < V.ncells) lane_step<D, COUNT>(V, X);
    f0 = X.f0;
    f1 = X.f1;
    f2 = X.f2;
    nfar = X.nfar;
    npair = X.npair;
}

// One node of a two-node walk (walk_pair): its own state and its visit of
// cell k when k >= resume, with walk_lane's arithmetic.
struct PairNode {
    float4 me;
    uint32_t p, mylp, oi, resume;
    float mk, f0, f1, f2;
    uint32_t nfar, npair;
};

template <int D>
__device__ __forceinline__ void pair_init(const WalkView &V, uint32_t p, PairNode &X) {
    const bool valid = p < V.n;
    X.p = p;
    X.me = valid ? V.sp[p] : make_float4(0.f, 0.f, 0.f, 0.f);
    X.mylp = valid ? V.leaf_pre[V.uid[p]] : 0u;
    X.oi = valid ? V.sorig[p] : 0u;
    X.resume = valid ? 0u : 0xffffffffu;
    X.mk = X.me.w * V.kr;
    X.f0 = X.f1 = X.f2 = 0.f;
    X.nfar = X.npair = 0;
}

template <int D, bool COUNT = true>
__device__ __forceinline__ void pair_visit(const WalkView &V, PairNode &X, uint32_t k, float cx, float cy, float cz,
                                           float lx, float ly, float lz, float cm, float w2, int32_t sk,
                                           uint32_t start, uint32_t skip, bool leaf) {
    if (k < X.resume) return;  // inside a subtree this node approximated
    const bool holds = (k <= X.mylp) && (X.mylp < skip);
    const float dx = (X.me.x - cx) - lx;
    const float dy = (X.me.y - cy) - ly;
    const float dz = (D == 3) ? (X.me.z - cz) - lz : 0.f;
    const float d2 = (D == 3) ? dx * dx + dy * dy + dz * dz : dx * dx + dy * dy;
    const bool far = !holds && w2 < V.th2 * d2;
    const bool body = far || (sk == -1 && !holds && d2 > 0.f);
    const float fb = __fdividef(X.mk * cm, d2);
    const float f = body ? fb : 0.f;
    X.f0 += dx * f;
    X.f1 += dy * f;
    if (D == 3) X.f2 += dz * f;
    if (COUNT) {
        X.nfar += far ? 1u : 0u;
        X.npair += (body && !far) ? 1u : 0u;
    }
    X.resume = body ? skip : k + 1;
    if (!leaf || body) return;
    const float4 *__restrict__ sp = V.sp;
    const uint32_t n = V.n, iter = V.iter;
    if (!holds && sk == -1) {  // coincident one-point leaf: the jiggle
        const uint32_t oj = __ldg(&V.sorig[start]);
        const float sg = X.oi < oj ? 1.f : -1.f;
        const float ex = sg * (float)jiggle(V.seed, iter, 0, X.oi, oj);
        const float ey = sg * (float)jiggle(V.seed, iter, 1, X.oi, oj);
        const float ez = (D == 3) ? sg * (float)jiggle(V.seed, iter, 2, X.oi, oj) : 0.f;
        const float e2 = (D == 3) ? ex * ex + ey * ey + ez * ez : ex * ex + ey * ey;
        const float g = __fdividef(X.mk * cm, e2);
        X.f0 += ex * g;
        X.f1 += ey * g;
        if (D == 3) X.f2 += ez * g;
        if (COUNT) X.npair++;
        return;
    }
    int32_t cnt = -sk;  // several points (or this node's own leaf): exact pairs
    if (start >= n || (uint32_t)cnt > n - start) {
        atomicOr(V.err, (uint32_t)ERR_TREE);
        cnt = 0;
    }
    for (int32_t q = 0; q < cnt; q++) {
        const uint32_t jp = start + (uint32_t)q;
        if (jp == X.p) continue;
        const float4 o = __ldg(&sp[jp]);
        float ex = X.me.x - o.x, ey = X.me.y - o.y, ez = (D == 3) ? X.me.z - o.z : 0.f;
        if (ex == 0.f && ey == 0.f && (D == 2 || ez == 0.f)) {
            const uint32_t oj = __ldg(&V.sorig[jp]);
            const float sg = X.oi < oj ? 1.f : -1.f;
            ex = sg * (float)jiggle(V.seed, iter, 0, X.oi, oj);
            ey = sg * (float)jiggle(V.seed, iter, 1, X.oi, oj);
            if (D == 3) ez = sg * (float)jiggle(V.seed, iter, 2, X.oi, oj);
        }
        const float e2 = (D == 3) ? ex * ex + ey * ey + ez * ez : ex * ex + ey * ey;
        const float g = __fdividef(X.mk * o.w, e2);
        X.f0 += ex * g;
        X.f1 += ey * g;
        if (D == 3) X.f2 += ez * g;
        if (COUNT) X.npair++;
    }
}

// Two adjacent Morton-sorted nodes per thread over the union of their walks:
// one cell load and one loop step serve both, and each node acts only at the
// cells of its own walk (k >= its resume), in the same order, so its forces are
// walk_lane's bit for bit. Adjacent nodes' walks nearly coincide, so the union
// is little longer than either.
template <int D, bool COUNT = true>
__device__ __forceinline__ void walk_pair(const WalkView &V, PairNode &a, PairNode &b) {
    const Cells cells = V.cells;
    const uint32_t ncells = V.ncells;
    uint32_t k = min(a.resume, b.resume);
    while (k < ncells) {
        const float4 A = cell_a<D>(cells, k);
        const float4 B = cell_b<D>(cells, k);
        int32_t sk;
        uint32_t start;
        float cx, cy, cz, cm, w2, lx, ly, lz;
        if (D == 2) {
            cx = A.x; cy = A.y; cz = 0.f; cm = A.z; w2 = A.w;
            lx = B.x; ly = B.y; lz = 0.f;
            sk = __float_as_int(B.z);
            start = __float_as_uint(B.w);
        } else {
            const int2 Cc = cell_c3(cells, k);
            cx = A.x; cy = A.y; cz = A.z; cm = A.w;
            lx = B.x; ly = B.y; lz = B.z; w2 = B.w;
            sk = Cc.x;
            start = (uint32_t)Cc.y;
        }
        const bool leaf = sk < 0;
        // leaves move on to k + 1; every step moves forward, whatever a cell holds
        const uint32_t skip = (uint32_t)max(sk, (int32_t)k + 1);
        pair_visit<D, COUNT>(V, a, k, cx, cy, cz, lx, ly, lz, cm, w2, sk, start, skip, leaf);
        pair_visit<D, COUNT>(V, b, k, cx, cy, cz, lx, ly, lz, cm, w2, sk, start, skip, leaf);
        k = min(a.resume, b.resume);
    }
}

// Two independent per-lane walks per thread, stepped in turn: the lane's nodes
// p and p + 32 (a warp holds two groups of 32 consecutive sorted nodes, each
// group as coherent as walk_lane's warp), each with its own cell index. Both
// walks' cell records are requested before either is used, so every thread
// keeps two dependent chains of cell loads in flight where walk_lane keeps
// one. A walk that has finished re-reads its last cell (a cached load) and
// does nothing with it. Each node visits its own cells in its own order with
// lane_visit's arithmetic, so its forces are walk_lane's bit for bit.
template <int D, bool COUNT = true>
__device__ __forceinline__ void walk_two(const WalkView &V, LaneNode &a, LaneNode &b) {
    const uint32_t nc = V.ncells;
    const uint32_t last = nc - 1u;  // nc >= 1 whenever a node is valid
    while (a.k < nc || b.k < nc) {
        const CellRec ra = cell_rec<D>(V.cells, min(a.k, last));
        const CellRec rb = cell_rec<D>(V.cells, min(b.k, last));
        if (a.k < nc) lane_visit<D, COUNT>(V, a, ra);
        if (b.k < nc) lane_visit<D, COUNT>(V, b, rb);
    }
}

// Walk schedules: 0 = walk_group (a warp over the union of its 32 nodes),
// 1 = walk_lane (one node per lane), 2 = walk_pair (two adjacent nodes per
// lane), 3 = walk_two (two independent walks per lane, 32 nodes apart).
// COUNT: add the far / pair interaction counts to the state (a diagnostic; the
// forces are the same either way).
template <int D, int SCHED, bool COUNT>
__global__ void __launch_bounds__(WALK_THREADS)
k_walk_s(WalkParams P, const DevState *__restrict__ st, Cells cells, const float4 *__restrict__ sp,
         const uint32_t *__restrict__ sorig, const uint32_t *__restrict__ uid,
         const uint32_t *__restrict__ leaf_pre, float *__restrict__ rep, DevState *stw) {
    gr_pdl_enter();
    if (st->converged) return;
    const uint32_t g = blockIdx.x * WALK_THREADS + threadIdx.x;
    const uint32_t lane = threadIdx.x % GR_WARP;
    const uint32_t p = SCHED == 2 ? 2 * g : SCHED == 3 ? 2 * (g - lane) + lane : g;
    if (__all_sync(GR_FULL, p >= P.n)) return;
    WalkView V{cells, sp, sorig, uid, leaf_pre, P.n, st->n_cells, st->iter_no, P.seed, P.kr, P.theta2, &stw->error};
    uint32_t nfar, npair;
    if (SCHED == 3) {
        LaneNode a, b;
        lane_init<D>(V, p, a);
        lane_init<D>(V, p + GR_WARP, b);
        walk_two<D, COUNT>(V, a, b);
        const LaneNode *X[2] = {&a, &b};
#pragma unroll
        for (int j = 0; j < 2; j++)
            if (X[j]->p < P.n) {
                const uint32_t oi = X[j]->oi;
                rep[(size_t)oi * D + 0] = X[j]->f0;
                rep[(size_t)oi * D + 1] = X[j]->f1;
                if (D == 3) rep[(size_t)oi * D + 2] = X[j]->f2;
            }
        nfar = a.nfar + b.nfar;
        npair = a.npair + b.npair;
    } else if (SCHED == 2) {
        PairNode a, b;
        pair_init<D>(V, p, a);
        pair_init<D>(V, p + 1, b);
        walk_pair<D, COUNT>(V, a, b);
        const PairNode *X[2] = {&a, &b};
#pragma unroll
        for (int j = 0; j < 2; j++)
            if (X[j]->p < P.n) {
                const uint32_t oi = X[j]->oi;
                rep[(size_t)oi * D + 0] = X[j]->f0;
                rep[(size_t)oi * D + 1] = X[j]->f1;
                if (D == 3) rep[(size_t)oi * D + 2] = X[j]->f2;
            }
        nfar = a.nfar + b.nfar;
        npair = a.npair + b.npair;
    } else {
        float f0, f1, f2;
        if (SCHED == 1)
            walk_lane<D, COUNT>(V, p, f0, f1, f2, nfar, npair);
        else
            walk_group<D, COUNT>(V, p, f0, f1, f2, nfar, npair);
        if (p < P.n) {
            const uint32_t oi = sorig[p];
            rep[(size_t)oi * D + 0] = f0;
            rep[(size_t)oi * D + 1] = f1;
            if (D == 3) rep[(size_t)oi * D + 2] = f2;
        }
    }
    if (!COUNT) return;
    nfar = __reduce_add_sync(GR_FULL, nfar);
    npair = __reduce_add_sync(GR_FULL, npair);
    if ((threadIdx.x % GR_WARP) == 0) {
        atomicAdd(&stw->far_count, (unsigned long long)nfar);
        atomicAdd(&stw->pair_count, (unsigned long long)npair);
    }
}

}  // namespace gr
