// d3-force Barnes-Hut session tick (2D): link, many-body, center, collide,
// integrate, on the tree the FA2 tick builds (the same d3 insertion quadtree,
// chains collapsed; every node weighs 1, so a cell's mass is its point count and
// its centre the centroid).
//
// Reference: crates/graph-core/src/layout/force/barnes_hut/sim.rs:170-270 (tick
// order: alpha decay, link, charge, center, collide, integrate), link.rs (force,
// share: Jacobi over the tick's state, degree-weighted split), charge.rs
// (node_delta: `open >= l` descends or takes the leaf's points directly, else
// the cell acts as one body of its count; settle: distanceMax cut-off, jiggled
// zero axes, l clamped up to distanceMin), collide.rs (every point within 2 r
// of the projected position pushed apart by half the overlap), seed.rs (golden
// spiral). FP32 positions and velocities, FP64 alpha and mean.
//
// Two known differences from the reference's FP64 run, both confined to exact
// coincidences: a many-body jiggle (an axis exactly 0 to a cell's centre) is
// keyed on the cell's preorder index where the reference keys it on the arena
// index of its insertion tree; and the leaf of several unseparated points
// (distinct points the 32-level key cannot split) takes its centroid where the
// reference takes its chain head.
#pragma once

#include "common.cuh"
#include "forces.cuh"
#include "tree.cuh"

namespace gr {

struct D3State {
    double alpha;      // cooling schedule
    double alpha_target;
    uint32_t tick_no;  // ticks completed (the jiggle counter)
    uint32_t pad;
};

struct D3Params {
    uint32_t n, seed;
    float charge, th2, dmin2, dmax2;
    float link_distance, link_strength_scale;
    float reach, reach2, center_strength, velocity_decay;
    double alpha_decay;
};

constexpr int D3_T = 256;

// sim.rs:177: alpha += (alpha_target - alpha) * alpha_decay, each operation
// rounded on its own (no fused multiply-add), as the reference computes it.
__global__ void k_d3_alpha(D3State *s, double decay) {
    s->alpha = __dadd_rn(s->alpha, __dmul_rn(__dsub_rn(s->alpha_target, s->alpha), decay));
}

__global__ void k_d3_end(D3State *s) { s->tick_no++; }

// Projected records {x + vx, y + vy, 0, 1}: the link's state (link.rs
// displaced) and collide's tree input (collide.rs prepare).
__global__ void k_d3_project(uint32_t n, const float4 *__restrict__ p, const float2 *__restrict__ v,
                             float4 *__restrict__ pp) {
    const uint32_t i = blockIdx.x * D3_T + threadIdx.x;
    if (i >= n) return;
    const float4 a = p[i];
    const float2 b = v[i];
    pp[i] = make_float4(a.x + b.x, a.y + b.y, 0.f, 1.f);
}

// Node v's share of its simple edge to u (link.rs force + share).
__device__ __forceinline__ void d3_link_term(const D3Params &P, uint32_t v, uint32_t u, float s, float alpha,
                                             uint32_t tick, const float4 *__restrict__ pp,
                                             const uint32_t *__restrict__ rp, float &ax, float &ay) {
    const uint32_t lo = min(u, v), hi = max(u, v);
    const float4 a = pp[hi], b = pp[lo];
    float dx = a.x - b.x, dy = a.y - b.y;
    if (dx == 0.f) dx = (float)jiggle(P.seed, tick, 0, lo, hi);
    if (dy == 0.f) dy = (float)jiggle(P.seed, tick, 1, lo, hi);
    const float l = sqrtf(dx * dx + dy * dy);
    if (l == 0.f) return;
    const float dist = P.link_distance / fmaxf(0.4f, s);
    const float str = fminf(0.7f, P.link_strength_scale * s);
    const float dlo = (float)(rp[lo + 1] - rp[lo]), dhi = (float)(rp[hi + 1] - rp[hi]);
    const float bias = dlo / (dlo + dhi);
    const float factor = (l - dist) / l * alpha * str;
    if (v == hi) {
        ax -= dx * factor * bias;
        ay -= dy * factor * bias;
    } else {
        ax += dx * factor * (1.f - bias);
        ay += dy * factor * (1.f - bias);
    }
}

// Heavy rows: one warp per SEG-entry segment, summed by a fixed butterfly.
__global__ void __launch_bounds__(D3_T)
k_d3_link_seg(D3Params P, uint32_t nseg, const D3State *st, const float4 *__restrict__ pp,
              const uint32_t *__restrict__ rp, const uint32_t *__restrict__ col, const float *__restrict__ wt,
              const uint32_t *__restrict__ seg_row, const uint32_t *__restrict__ seg_first, float2 *__restrict__ seg_out) {
    const uint32_t sg = (blockIdx.x * D3_T + threadIdx.x) / GR_WARP, lane = threadIdx.x % GR_WARP;
    if (sg >= nseg) return;
    const uint32_t row = seg_row[sg];
    const uint32_t e0 = rp[row] + (sg - seg_first[row]) * SEG, e1 = min(e0 + SEG, rp[row + 1]);
    const float alpha = (float)st->alpha;
    float ax = 0.f, ay = 0.f;
    for (uint32_t e = e0 + lane; e < e1; e += GR_WARP) d3_link_term(P, row, col[e], wt[e], alpha, st->tick_no, pp, rp, ax, ay);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        ax += __shfl_xor_sync(GR_FULL, ax, o);
        ay += __shfl_xor_sync(GR_FULL, ay, o);
    }
    if (lane == 0) seg_out[sg] = make_float2(ax, ay);
}

// Every node's link delta (its row in CSR order; heavy rows from their
// segments in order) onto its own velocity. Reads only the projected records.
__global__ void __launch_bounds__(D3_T)
k_d3_link(D3Params P, const D3State *st, const float4 *__restrict__ pp, const uint32_t *__restrict__ rp,
          const uint32_t *__restrict__ col, const float *__restrict__ wt, const uint32_t *__restrict__ seg_first,
          const float2 *__restrict__ seg_out, float2 *__restrict__ v) {
    const uint32_t i = blockIdx.x * D3_T + threadIdx.x;
    if (i >= P.n) return;
    const float alpha = (float)st->alpha;
    const uint32_t e0 = rp[i], e1 = rp[i + 1];
    float ax = 0.f, ay = 0.f;
    if (seg_first == nullptr || e1 - e0 <= LIGHT_MAX) {
        for (uint32_t e = e0; e < e1; e++) d3_link_term(P, i, col[e], wt[e], alpha, st->tick_no, pp, rp, ax, ay);
    } else {
        const uint32_t s0 = seg_first[i], ns = (e1 - e0 + SEG - 1) / SEG;
        for (uint32_t s = s0; s < s0 + ns; s++) {
            ax += seg_out[s].x;
            ay += seg_out[s].y;
        }
    }
    float2 w = v[i];
    w.x += ax;
    w.y += ay;
    v[i] = w;
}

// charge.rs settle: false past distanceMax; a zero axis jiggled (passes 2, 3);
// l clamped up to distanceMin.
__device__ __forceinline__ bool d3_settle(const D3Params &P, uint32_t tick, uint32_t i, uint32_t key, float &dx,
                                          float &dy, float &l) {
    if (l >= P.dmax2) return false;
    if (dx == 0.f) {
        dx = (float)jiggle(P.seed, tick, 2, i, key);
        l += dx * dx;
    }
    if (dy == 0.f) {
        dy = (float)jiggle(P.seed, tick, 3, i, key);
        l += dy * dy;
    }
    if (l < P.dmin2) l = sqrtf(P.dmin2 * l);
    if (l == 0.f) l = fmaxf(P.dmin2, 1.17549435e-38f);
    return true;
}

// Many-body: per sorted node, the stackless preorder walk of charge.rs
// node_delta over the cells (A {cx, cy, count, w^2}, B {cx_lo, cy_lo, skip |
// -count, start}); the delta goes onto the node's own velocity. A cell the
// opening test resolves acts as one body of its count; a leaf it does not takes
// its points directly, every point at the leaf centre's offset (charge.rs
// direct), which is the same term with the count less this node when it lies in
// the leaf. So the common outcomes need no branch: the term is selected by
// predicate, the next cell by select; only an exactly zero axis (the jiggle)
// branches.
__global__ void __launch_bounds__(D3_T)
k_d3_charge(D3Params P, const D3State *st, const DevState *ts, Cells cells, const float4 *__restrict__ sp,
            const uint32_t *__restrict__ sorig, float2 *__restrict__ v) {
    const uint32_t p = blockIdx.x * D3_T + threadIdx.x;
    if (p >= P.n) return;
    const uint32_t ncells = ts->n_cells, tick = st->tick_no;
    const float ca = P.charge * (float)st->alpha;
    const float4 me = sp[p];
    const uint32_t oi = sorig[p];
    float ax = 0.f, ay = 0.f;
    uint32_t k = 0;
    while (k < ncells) {
        const float4 A = cell_a<2>(cells, k);
        const float4 B = cell_b<2>(cells, k);
        const int32_t sk = __float_as_int(B.z);
        const bool leaf = sk < 0;
        float dx = (A.x - me.x) + B.x, dy = (A.y - me.y) + B.y;
        float l = dx * dx + dy * dy;
        const bool open = A.w >= P.th2 * l;  // open >= l: w^2 / theta^2 >= l
        const bool in_range = l < P.dmax2;   // settle: nothing at or past distanceMax
        const uint32_t start = __float_as_uint(B.w), cnt = leaf ? (uint32_t)(-sk) : 0u;
        const bool self_in = leaf && p - start < cnt;  // this node is one of the leaf's points
        if (dx == 0.f || dy == 0.f) {  // the jiggle, keyed on the chain head (direct) or the cell (body)
            const uint32_t key = (open && leaf) ? __ldg(&sorig[start + cnt - 1]) : k;
            if (dx == 0.f) {
                dx = (float)jiggle(P.seed, tick, 2, oi, key);
                l += dx * dx;
            }
            if (dy == 0.f) {
                dy = (float)jiggle(P.seed, tick, 3, oi, key);
                l += dy * dy;
            }
        }
        l = l < P.dmin2 ? sqrtf(P.dmin2 * l) : l;
        l = l == 0.f ? fmaxf(P.dmin2, 1.17549435e-38f) : l;
        const bool descend = open && !leaf;
        const bool counted = !descend && in_range;
        const float m = (open && self_in) ? A.z - 1.f : A.z;
        const float f = counted ? m * ca / l : 0.f;
        ax += dx * f;
        ay += dy * f;
        k = (descend || leaf) ? k + 1 : max((uint32_t)sk, k + 1);
    }
    float2 w = v[oi];
    w.x += ax;
    w.y += ay;
    v[oi] = w;
}

// center.js: every position shifted by the mean (FP64, from the bounds pass
// over the same positions: the many-body tree's, or the mesh's) times the
// centering strength.
__global__ void k_d3_center(uint32_t n, float strength, const double *mean, float4 *__restrict__ p) {
    const uint32_t i = blockIdx.x * D3_T + threadIdx.x;
    if (i >= n) return;
    const float sx = (float)(mean[0] * (double)strength), sy = (float)(mean[1] * (double)strength);
    float4 a = p[i];
    a.x -= sx;
    a.y -= sy;
    p[i] = a;
}

// collide.js over the tree of projected positions: leaves take every other
// point within 2 r, internal cells whose square lies beyond reach are skipped
// (with a margin, so rounding never skips a point that counts).
__global__ void __launch_bounds__(D3_T)
k_d3_collide(D3Params P, const D3State *st, const DevState *ts, Cells cells, const float4 *__restrict__ sp,
             const uint32_t *__restrict__ sorig, float2 *__restrict__ v) {
    const uint32_t p = blockIdx.x * D3_T + threadIdx.x;
    if (p >= P.n) return;
    const uint32_t ncells = ts->n_cells, tick = st->tick_no;
    const float4 q = sp[p];
    const uint32_t oi = sorig[p];
    const float prune = P.reach * 1.0001f;
    float ax = 0.f, ay = 0.f;
    uint32_t k = 0;
    while (k < ncells) {
        const float4 B = cell_b<2>(cells, k);
        const int32_t sk = __float_as_int(B.z);
        if (sk < 0) {
            const uint32_t start = __float_as_uint(B.w), cnt = (uint32_t)(-sk);
            for (uint32_t j = start; j < start + cnt; j++) {
                if (j == p) continue;
                const float4 o = __ldg(&sp[j]);
                float dx = q.x - o.x, dy = q.y - o.y;
                float l = dx * dx + dy * dy;
                if (l >= P.reach2) continue;
                const uint32_t oj = __ldg(&sorig[j]);
                if (dx == 0.f) {
                    dx = (float)jiggle(P.seed, tick, 4, oi, oj);
                    l += dx * dx;
                }
                if (dy == 0.f) {
                    dy = (float)jiggle(P.seed, tick, 5, oi, oj);
                    l += dy * dy;
                }
                const float dist = sqrtf(l);
                const float push = (P.reach - dist) / dist * 0.5f;
                ax += dx * push;
                ay += dy * push;
            }
            k++;
        } else {
            const float4 b = __ldg(&cells.bounds[k]);
            const bool out = b.x > q.x + prune || b.z < q.x - prune || b.y > q.y + prune || b.w < q.y - prune;
            k = out ? max((uint32_t)sk, k + 1) : k + 1;
        }
    }
    float2 w = v[oi];
    w.x += ax;
    w.y += ay;
    v[oi] = w;
}

// simulation.js tick tail: v *= velocityDecay, x += v.
__global__ void k_d3_integrate(uint32_t n, float decay, float4 *__restrict__ p, float2 *__restrict__ v) {
    const uint32_t i = blockIdx.x * D3_T + threadIdx.x;
    if (i >= n) return;
    float2 w = v[i];
    w.x *= decay;
    w.y *= decay;
    float4 a = p[i];
    a.x += w.x;
    a.y += w.y;
    v[i] = w;
    p[i] = a;
}

}  // namespace gr
