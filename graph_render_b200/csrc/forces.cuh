// Attraction, gravity, the FP64 swing/traction reductions, the speed controller
// and the position update.
//
// Reference: crates/graph-core/src/layout/forceatlas2/state.rs:152-162 (attraction),
// 208-251 (gravity), state/schedule.rs:16-77 (swing/traction, estimate_factor,
// apply_update); the options graph-core leaves at their defaults follow networkx
// 3.6 `forceatlas2_layout` (networkx/drawing/layout.py:1806-1872): linlog,
// distributed_action (dissuade hubs), strong_gravity, weighted adjacency.
//
// Attraction is a CSR gather: node i sums w_ij * (p_j - p_i) over its own row in
// a fixed order, so there is no scatter and no float atomic, and the sum is the
// same every run. Every reduction folds per-block partials in block order in the
// grid's last block.
#pragma once

#include "common.cuh"
#include "tree.cuh"

namespace gr {

constexpr int FRC_THREADS = 256;
// k_forces and k_update stride over the nodes with at most FRC_MAX_BLOCKS
// blocks (4 per SM): fewer per-block partials and last-block tickets.
constexpr uint32_t FRC_MAX_BLOCKS = 4 * 148;  // measured: 8 and 16 per SM slower (3 and 8 us at 1M nodes)

__host__ __device__ inline uint32_t frc_blocks(uint32_t n) {
    const uint32_t b = (n + FRC_THREADS - 1) / FRC_THREADS;
    return b < 1 ? 1 : (b > FRC_MAX_BLOCKS ? FRC_MAX_BLOCKS : b);
}
// Rows longer than LIGHT_MAX are summed in SEG-entry segments, one warp each,
// so a hub of 30k neighbours costs ~120 warps instead of one thread's 30k steps.
// (64: on the 1M-node power-law tick 3 us faster than 32, 16 slower by 9 us.)
constexpr uint32_t LIGHT_MAX = 64;
constexpr uint32_t SEG = 256;

// One edge's pull on node p from neighbour q: w * (q - p), or with linlog
// w * log(1 + d) / d * (q - p) (networkx layout.py:1806-1813).
template <int D>
__device__ __forceinline__ void attr_term(const float4 &p, const float4 &q, float w, int lin_log, float &a0,
                                          float &a1, float &a2) {
    const float d0 = q.x - p.x, d1 = q.y - p.y, d2 = (D == 3) ? q.z - p.z : 0.f;
    float c = w;
    if (lin_log) {
        const float dist = sqrtf(d0 * d0 + d1 * d1 + d2 * d2);
        c *= dist > 0.f ? log1pf(dist) / dist : 0.f;
    }
    a0 += d0 * c;
    a1 += d1 * c;
    if (D == 3) a2 += d2 * c;
}

// Heavy rows: warp s sums entries [seg_begin(s), seg_begin(s) + SEG) of row
// seg_row[s] (lanes stride by 32, then a fixed butterfly), writing D floats.
// A null wt means every weight is 1.
template <int D>
__global__ void __launch_bounds__(FRC_THREADS)
k_attract_seg(uint32_t nseg, int lin_log, const DevState *st, const float4 *__restrict__ pos,
              const uint32_t *__restrict__ rp, const uint32_t *__restrict__ col, const float *__restrict__ wt,
              const uint32_t *__restrict__ seg_row, const uint32_t *__restrict__ seg_first,
              float *__restrict__ seg_out) {
    if (st->converged) return;
    const uint32_t s = (blockIdx.x * FRC_THREADS + threadIdx.x) / GR_WARP;
    const uint32_t lane = threadIdx.x % GR_WARP;
    if (s >= nseg) return;
    const uint32_t row = seg_row[s];
    const uint32_t e0 = rp[row] + (s - seg_first[row]) * SEG;
    const uint32_t e1 = min(e0 + SEG, rp[row + 1]);
    const float4 p = pos[row];
    float a0 = 0.f, a1 = 0.f, a2 = 0.f;
    for (uint32_t e = e0 + lane; e < e1; e += GR_WARP)
        attr_term<D>(p, pos[col[e]], wt ? wt[e] : 1.f, lin_log, a0, a1, a2);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a0 += __shfl_xor_sync(GR_FULL, a0, o);
        a1 += __shfl_xor_sync(GR_FULL, a1, o);
        if (D == 3) a2 += __shfl_xor_sync(GR_FULL, a2, o);
    }
    if (lane == 0) {
        seg_out[(size_t)s * D] = a0;
        seg_out[(size_t)s * D + 1] = a1;
        if (D == 3) seg_out[(size_t)s * D + 2] = a2;
    }
}

struct ForceParams {
    uint32_t n;
    float gravity;
    int lin_log, strong_gravity, dissuade_hubs;
    double jitter_tolerance;
};

// schedule.rs:33-60 estimate_factor (networkx's helper), FP64.
__device__ __forceinline__ void estimate_factor(DevState *st, double n, double jt) {
    const double swing = st->swing, traction = st->traction;
    const double opt_jitter = 0.05 * sqrt(n);
    const double min_jitter = sqrt(opt_jitter);
    const double min_se = 0.05;
    const double other = fmin(10.0, opt_jitter * traction / (n * n));
    double jitter = jt * fmax(min_jitter, other);
    double se = st->speed_efficiency, speed = st->speed;
    if (swing / traction > 2.0) {
        if (se > min_se) se *= 0.5;
        jitter = fmax(jitter, jt);
    }
    const double target = swing == 0.0 ? INFINITY : jitter * se * traction / swing;
    if (swing > jitter * traction) {
        if (se > min_se) se *= 0.7;
    } else if (speed < 1000.0) {
        se *= 1.3;
    }
    speed += fmin(target - speed, 0.5 * speed);
    st->speed = speed;
    st->speed_efficiency = se;
}

// Node i's force accumulator given its attraction (a*) and repulsion (r*):
// u = attraction (/ mass with dissuade hubs) + repulsion - gravity, gravity the
// unit vector first (state.rs:223-251) or strong (layout.py:1830-1832); writes u
// and returns the node's FP64 swing and traction terms (schedule.rs:16-30).
template <int D>
__device__ __forceinline__ void node_force(const ForceParams &P, const float4 &p, float a0, float a1, float a2,
                                           float r0, float r1, float r2, const double *mean, float *u, double &sw,
                                           double &tr) {
    if (P.dissuade_hubs) {
        a0 /= p.w;
        a1 /= p.w;
        a2 /= p.w;
    }
    float u0 = a0 + r0;
    float u1 = a1 + r1;
    float u2 = (D == 3) ? a2 + r2 : 0.f;
    const float c0 = (float)((double)p.x - mean[0]);
    const float c1 = (float)((double)p.y - mean[1]);
    const float c2 = (D == 3) ? (float)((double)p.z - mean[2]) : 0.f;
    const float g = P.gravity * p.w;
    if (P.strong_gravity) {
        u0 -= g * c0;
        u1 -= g * c1;
        u2 -= g * c2;
    } else {
        const float nrm = sqrtf(c0 * c0 + c1 * c1 + c2 * c2);
        if (nrm > 0.f) {
            u0 -= g * (c0 / nrm);
            u1 -= g * (c1 / nrm);
            u2 -= g * (c2 / nrm);
        }
    }
    u[0] = u0;
    u[1] = u1;
    if (D == 3) u[2] = u2;
    const double m = (double)p.w;
    const double b0 = (double)p.x - u0, b1 = (double)p.y - u1, b2 = (D == 3) ? (double)p.z - u2 : 0.0;
    const double g0 = (double)p.x + u0, g1 = (double)p.y + u1, g2 = (D == 3) ? (double)p.z + u2 : 0.0;
    sw = m * sqrt(b0 * b0 + b1 * b1 + b2 * b2);
    tr = 0.5 * m * sqrt(g0 * g0 + g1 * g1 + g2 * g2);
}

// schedule.rs:62-77 apply_update for one node: factor = speed / (1 + sqrt(speed
// * m * |u|)), p += u * factor; returns |step| summed over the axes (FP64).
template <int D>
__device__ __forceinline__ double node_update(float4 &p, const float *__restrict__ u, double speed, bool &bad) {
    const double u0 = u[0], u1 = u[1], u2 = (D == 3) ? u[2] : 0.0;
    const double nrm = sqrt(u0 * u0 + u1 * u1 + u2 * u2);
    const double factor = speed / (1.0 + sqrt(speed * (double)p.w * nrm));
    const float d0 = (float)(u0 * factor), d1 = (float)(u1 * factor), d2 = (float)(u2 * factor);
    p.x += d0;
    p.y += d1;
    if (D == 3) p.z += d2;
    bad = !(isfinite(p.x) && isfinite(p.y) && isfinite(p.z));
    return fabs((double)d0) + fabs((double)d1) + ((D == 3) ? fabs((double)d2) : 0.0);
}

// Attraction of node i over its own CSR row (rows of <= LIGHT_MAX entries), or
// its segment sums in segment order (longer rows, when seg_first is given).
// A null wt means every weight is 1 (the same terms, without the weight reads).
template <int D>
__device__ __forceinline__ void node_attraction(uint32_t i, const float4 &p, int lin_log,
                                                const float4 *__restrict__ pos, const uint32_t *__restrict__ rp,
                                                const uint32_t *__restrict__ col, const float *__restrict__ wt,
                                                const uint32_t *__restrict__ seg_first,
                                                const float *__restrict__ seg_out, float &a0, float &a1, float &a2) {
    a0 = a1 = a2 = 0.f;
    const uint32_t e0 = rp[i], e1 = rp[i + 1];
    if (seg_first == nullptr || e1 - e0 <= LIGHT_MAX) {
        for (uint32_t e = e0; e < e1; e++) attr_term<D>(p, pos[col[e]], wt ? wt[e] : 1.f, lin_log, a0, a1, a2);
    } else {  // the row's segment sums, in segment order
        const uint32_t s0 = seg_first[i], ns = (e1 - e0 + SEG - 1) / SEG;
        for (uint32_t s = s0; s < s0 + ns; s++) {
            a0 += seg_out[(size_t)s * D];
            a1 += seg_out[(size_t)s * D + 1];
            if (D == 3) a2 += seg_out[(size_t)s * D + 2];
        }
    }
}

// Every node's attraction (node_attraction) into att (n x D). It reads only the
// positions and the graph, so it can run beside the tree build and the walk.
template <int D>
__global__ void __launch_bounds__(FRC_THREADS)
k_attract(uint32_t n, int lin_log, const DevState *st, const float4 *__restrict__ pos,
          const uint32_t *__restrict__ rp, const uint32_t *__restrict__ col, const float *__restrict__ wt,
          const uint32_t *__restrict__ seg_first, const float *__restrict__ seg_out, float *__restrict__ att) {
    if (st->converged) return;
    const uint32_t i = blockIdx.x * FRC_THREADS + threadIdx.x;
    if (i >= n) return;
    float a0, a1, a2;
    node_attraction<D>(i, pos[i], lin_log, pos, rp, col, wt, seg_first, seg_out, a0, a1, a2);
    att[(size_t)i * D] = a0;
    att[(size_t)i * D + 1] = a1;
    if (D == 3) att[(size_t)i * D + 2] = a2;
}

// u_i for every node from its attraction (read from U, where k_attract put it;
// each thread reads and then overwrites only its own node's entries) and its
// repulsion; per-block FP64 swing and traction; the last block accumulates
// them into the state (cumulative, state.rs:141-143) and runs estimate_factor.
template <int D>
__global__ void __launch_bounds__(FRC_THREADS)
k_forces(ForceParams P, DevState *st, const float4 *__restrict__ pos, const float *__restrict__ rep, float *U,
         double *__restrict__ part, int speed_update) {
    gr_pdl_enter();
    if (st->converged) return;
    __shared__ double s_red[32];
    __shared__ bool s_last;
    double sw = 0.0, tr = 0.0;
    const double mean[3] = {st->mean[0], st->mean[1], st->mean[2]};
    for (uint32_t i = blockIdx.x * FRC_THREADS + threadIdx.x; i < P.n; i += gridDim.x * FRC_THREADS) {
        const float4 p = pos[i];
        float *u = U + (size_t)i * D;
        const float a0 = u[0], a1 = u[1], a2 = D == 3 ? u[2] : 0.f;
        double s1, t1;
        node_force<D>(P, p, a0, a1, a2, rep[(size_t)i * D + 0], rep[(size_t)i * D + 1],
                      D == 3 ? rep[(size_t)i * D + 2] : 0.f, mean, u, s1, t1);
        sw += s1;
        tr += t1;
    }
    if (!speed_update) return;
    sw = block_sum_d<FRC_THREADS>(sw, s_red);
    tr = block_sum_d<FRC_THREADS>(tr, s_red);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = sw;
        part[2 * blockIdx.x + 1] = tr;
    }
    if (!last_block_done(&st->counters[1], &s_last)) return;
    double a = strided_sum_cg<FRC_THREADS>(part, gridDim.x, 2, 0);
    double b = strided_sum_cg<FRC_THREADS>(part, gridDim.x, 2, 1);
    a = block_sum_d<FRC_THREADS>(a, s_red);
    b = block_sum_d<FRC_THREADS>(b, s_red);
    if (threadIdx.x == 0) {
        st->swing += a;
        st->traction += b;
        estimate_factor(st, (double)P.n, P.jitter_tolerance);
    }
}

// The update for every node; FP64 sum of |step| decides the 1e-10 early exit
// (state.rs:122-128). With bpart, the same pass also takes the new positions'
// extent and FP64 sums (bounds_block / bounds_finish over k_bounds' grid and
// per-thread order, so the same bits k_bounds would get) into the root square
// and mean of the next tick, and stamps them valid for it.
static_assert(FRC_THREADS == BND_THREADS, "k_update and k_bounds share one grid shape");
template <int D>
__global__ void __launch_bounds__(FRC_THREADS)
k_update(uint32_t n, DevState *st, float4 *__restrict__ pos, const float *__restrict__ U,
         double *__restrict__ part, double *__restrict__ bpart) {
    gr_pdl_enter();
    if (st->converged) return;
    __shared__ double s_red[32];
    __shared__ float s_f[2 * D][32];
    __shared__ bool s_last;
    double step = 0.0;
    bool bad = false;
    const double speed = st->speed;
    float lo[D], hi[D];
    double sum[D];
#pragma unroll
    for (int a = 0; a < D; a++) {
        lo[a] = INFINITY;
        hi[a] = -INFINITY;
        sum[a] = 0.0;
    }
    for (uint32_t i = blockIdx.x * FRC_THREADS + threadIdx.x; i < n; i += gridDim.x * FRC_THREADS) {
        float4 p = pos[i];
        bool b;
        step += node_update<D>(p, U + (size_t)i * D, speed, b);
        bad = bad || b;
        pos[i] = p;
        const float c[3] = {p.x, p.y, p.z};
#pragma unroll
        for (int a = 0; a < D; a++) {
            lo[a] = fminf(lo[a], c[a]);
            hi[a] = fmaxf(hi[a], c[a]);
            sum[a] += (double)c[a];
        }
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(&st->error, (uint32_t)ERR_NONFINITE);
    if (bpart) bounds_block<D>(lo, hi, sum, bpart, s_red, s_f);
    step = block_sum_d<FRC_THREADS>(step, s_red);
    if (threadIdx.x == 0) part[blockIdx.x] = step;
    if (!last_block_done(&st->counters[2], &s_last)) return;
    double a = strided_sum_cg<FRC_THREADS>(part, gridDim.x, 1, 0);
    a = block_sum_d<FRC_THREADS>(a, s_red);
    if (threadIdx.x == 0) {
        st->moved = a;
        st->iter_no += 1;
        if (a < 1e-10 || st->error) st->converged = 1;
    }
    if (bpart) {
        bounds_finish<D>(bpart, n, st, s_red);
        if (threadIdx.x == 0) st->bounds_stamp = st->iter_no + 1u;
    }
}

// Row-major n x D copy of the float4 positions (the per-tick buffer); with
// nonfinite, a non-finite coordinate sets it to 1.
template <int D>
__global__ void k_export(uint32_t n, const float4 *__restrict__ pos, float *__restrict__ out,
                         uint32_t *nonfinite = nullptr) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 p = pos[i];
    out[(size_t)i * D] = p.x;
    out[(size_t)i * D + 1] = p.y;
    if (D == 3) out[(size_t)i * D + 2] = p.z;
    if (nonfinite && !(isfinite(p.x) && isfinite(p.y) && (D == 2 || isfinite(p.z)))) *nonfinite = 1u;
}

template <int D>
__global__ void k_import(uint32_t n, float4 *__restrict__ pos, const float *__restrict__ in) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 p = pos[i];
    p.x = in[(size_t)i * D];
    p.y = in[(size_t)i * D + 1];
    p.z = (D == 3) ? in[(size_t)i * D + 2] : 0.f;
    pos[i] = p;
}

}  // namespace gr
