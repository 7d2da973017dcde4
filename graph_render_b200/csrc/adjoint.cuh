// Adjoint (vector-Jacobian product) of one FA2 tick, through the tree the tick
// built (its far / pair decisions held fixed; cell centres move with their
// points) and through the FP64 speed controller on its active branch.
//
// Notation for one tick: u = attraction + repulsion - gravity at p; sw, tr the
// FP64 swing / traction sums; (speed', se') = estimate_factor(SW + sw, TR + tr,
// speed, se); p' = p + f u, f = speed' / (1 + sqrt(speed' m |u|)). Given
// lam' = dL/dp' and the adjoints of the controller after the tick, the kernels
// below produce lam = dL/dp, the controller adjoints before the tick, and add
// dL/dc (attraction coefficient) per CSR entry. The same function restated in
// FP64 on the CPU (oracle, orc_fa2_adjoint) is what this is tested against.
#pragma once

#include "common.cuh"
#include "forces.cuh"
#include "tree.cuh"
#include "walk.cuh"

namespace gr {

struct AdjScalars {
    double LSW, LTR, Lsp, Lse;  // adjoints of the controller after the tick (from later ticks)
    double Lsw_cur, Ltr_cur;    // this tick's adjoints of sw, tr
    double vsum[3];             // sum of the gravity VJP terms
    uint32_t counters[4];
    uint32_t absmax;            // bit pattern of max |lam'| (a non-negative float orders as its bits)
    int shift;                  // this tick's rescale exponent
    long long exponent;         // lam' and the accumulated dL/dc are the true values times 2^-exponent
};

// estimate_factor's partial derivatives on its active branch: d[0..3] =
// d speed' / d(SW, TR, speed, se), d[4] = d se' / d se (schedule.rs:33-60).
__device__ inline void ef_diff(double n, double jt, double SW, double TR, double speed, double se, double *d) {
    const double opt = 0.05 * sqrt(n), minj = sqrt(opt);
    const double ratio = opt * TR / (n * n);
    const double other = ratio < 10.0 ? ratio : 10.0;
    double djit = 0.0, jitter;
    if (minj >= other) {
        jitter = jt * minj;
    } else {
        jitter = jt * other;
        if (ratio < 10.0) djit = jt * opt / (n * n);
    }
    double k1 = 1.0;
    if (SW / TR > 2.0) {
        if (se > 0.05) k1 = 0.5;
        if (jt > jitter) {
            jitter = jt;
            djit = 0.0;
        }
    }
    const double se1 = se * k1;
    double target = INFINITY, tSW = 0.0, tTR = 0.0, tse = 0.0;
    if (SW != 0.0) {
        target = jitter * se1 * TR / SW;
        tSW = -target / SW;
        tTR = jitter * se1 / SW + se1 * TR / SW * djit;
        tse = jitter * k1 * TR / SW;
    }
    double k2 = 1.0;
    if (SW > jitter * TR) {
        if (se1 > 0.05) k2 = 0.7;
    } else if (speed < 1000.0) {
        k2 = 1.3;
    }
    d[4] = k1 * k2;
    if (target - speed < 0.5 * speed) {
        d[0] = tSW;
        d[1] = tTR;
        d[2] = 0.0;
        d[3] = tse;
    } else {
        d[0] = d[1] = d[3] = 0.0;
        d[2] = 1.5;
    }
}

// d/d(delta) of k m M delta / |delta|^2, applied to v.
template <int D>
__device__ __forceinline__ void rep_jac(float coef, float dx, float dy, float dz, float vx, float vy, float vz,
                                        float &ox, float &oy, float &oz) {
    const float d2 = dx * dx + dy * dy + (D == 3 ? dz * dz : 0.f);
    const float dv = dx * vx + dy * vy + (D == 3 ? dz * vz : 0.f);
    const float a = coef / d2, b = 2.f * coef * dv / (d2 * d2);
    ox = a * vx - b * dx;
    oy = a * vy - b * dy;
    oz = (D == 3) ? a * vz - b * dz : 0.f;
}

// (1) The update: lam = lam', ub = f lam' + (lam'.u) grad_u f; the FP64 sum of
// (lam'.u) df/dspeed'; the last block runs the controller backward.
template <int D>
__global__ void __launch_bounds__(FRC_THREADS)
k_adj_update(uint32_t n, double jt, const DevState *st_after, const DevState *st_before, AdjScalars *A,
             const float4 *__restrict__ pos, const float *__restrict__ U, const float *__restrict__ lam1,
             float *__restrict__ lam, float *__restrict__ ub, double *__restrict__ part) {
    __shared__ double s_red[32];
    __shared__ bool s_last;
    const uint32_t i = blockIdx.x * FRC_THREADS + threadIdx.x;
    const double speed1 = st_after->speed;
    double acc = 0.0;
    if (i < n) {
        const float4 p = pos[i];
        double u[3] = {0, 0, 0}, l[3] = {0, 0, 0};
        for (int a = 0; a < D; a++) {
            u[a] = U[(size_t)i * D + a];
            l[a] = lam1[(size_t)i * D + a];
        }
        const double un = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]), m = p.w;
        const double q = sqrt(speed1 * m * un), f = speed1 / (1.0 + q);
        const double lu = l[0] * u[0] + l[1] * u[1] + l[2] * u[2];
        acc = lu * (q > 0.0 ? (1.0 + 0.5 * q) / ((1.0 + q) * (1.0 + q)) : 1.0);
        const double g = q > 0.0 ? -speed1 / ((1.0 + q) * (1.0 + q)) * speed1 * m / (2.0 * q * un) : 0.0;
        for (int a = 0; a < D; a++) {
            lam[(size_t)i * D + a] = (float)l[a];
            ub[(size_t)i * D + a] = (float)(f * l[a] + lu * g * u[a]);
        }
    }
    acc = block_sum_d<FRC_THREADS>(acc, s_red);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
    if (!last_block_done(&A->counters[0], &s_last)) return;
    double t = 0.0;
    t += strided_sum_cg<FRC_THREADS>(part, gridDim.x, 1, 0);
    t = block_sum_d<FRC_THREADS>(t, s_red);
    if (threadIdx.x == 0) {
        const double Lsp = A->Lsp + t;
        double d[5];
        ef_diff((double)n, jt, st_after->swing, st_after->traction, st_before->speed, st_before->speed_efficiency, d);
        const double LSW = A->LSW + Lsp * d[0], LTR = A->LTR + Lsp * d[1];
        const double Lse_prev = Lsp * d[3] + A->Lse * d[4];
        A->Lsp = Lsp * d[2];
        A->Lse = Lse_prev;
        A->LSW = LSW;
        A->LTR = LTR;
        A->Lsw_cur = LSW;
        A->Ltr_cur = LTR;
    }
}

// (2) Swing / traction (schedule.rs:16-30) and the gravity VJP terms v.
template <int D>
__global__ void __launch_bounds__(FRC_THREADS)
k_adj_node(uint32_t n, float gravity, int strong, const DevState *st, AdjScalars *A, const float4 *__restrict__ pos,
           const float *__restrict__ U, float *__restrict__ lam, float *__restrict__ ub, float *__restrict__ v,
           double *__restrict__ part) {
    __shared__ double s_red[32];
    __shared__ bool s_last;
    const uint32_t i = blockIdx.x * FRC_THREADS + threadIdx.x;
    double vs[3] = {0, 0, 0};
    if (i < n) {
        const float4 p = pos[i];
        const double pc[3] = {p.x, p.y, p.z};
        double b[3] = {0, 0, 0}, g[3] = {0, 0, 0}, uu[3] = {0, 0, 0};
        for (int a = 0; a < D; a++) {
            const double u = U[(size_t)i * D + a];
            b[a] = pc[a] - u;
            g[a] = pc[a] + u;
        }
        const double bn = sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]);
        const double gn = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
        const double m = p.w, Lsw = A->Lsw_cur, Ltr = A->Ltr_cur;
        for (int a = 0; a < D; a++) {
            const double tb = bn > 0.0 ? Lsw * m * b[a] / bn : 0.0;
            const double tg = gn > 0.0 ? Ltr * 0.5 * m * g[a] / gn : 0.0;
            lam[(size_t)i * D + a] += (float)(tb + tg);
            uu[a] = (double)ub[(size_t)i * D + a] - tb + tg;
            ub[(size_t)i * D + a] = (float)uu[a];
        }
        // gravity: g_i = -gm c/|c| (or -gm c), c = p - mean
        const double gm = (double)gravity * m;
        double c[3] = {0, 0, 0};
        for (int a = 0; a < D; a++) c[a] = pc[a] - st->mean[a];
        if (strong) {
            for (int a = 0; a < D; a++) vs[a] = -gm * uu[a];
        } else {
            const double cn2 = c[0] * c[0] + c[1] * c[1] + c[2] * c[2];
            if (cn2 > 0.0) {
                const double cn = sqrt(cn2), cu = c[0] * uu[0] + c[1] * uu[1] + c[2] * uu[2];
                for (int a = 0; a < D; a++) vs[a] = -gm * (uu[a] - c[a] * cu / cn2) / cn;
            }
        }
        for (int a = 0; a < D; a++) v[(size_t)i * D + a] = (float)vs[a];
    }
    double tot[3];
#pragma unroll
    for (int a = 0; a < 3; a++) tot[a] = (a < D) ? block_sum_d<FRC_THREADS>(vs[a], s_red) : 0.0;
    if (threadIdx.x == 0)
        for (int a = 0; a < D; a++) part[(size_t)blockIdx.x * 3 + a] = tot[a];
    if (!last_block_done(&A->counters[1], &s_last)) return;
    double S[3] = {0, 0, 0};
    for (int a = 0; a < D; a++) {
        double t = 0.0;
        t += strided_sum_cg<FRC_THREADS>(part, gridDim.x, 3, a);
        S[a] = block_sum_d<FRC_THREADS>(t, s_red);
    }
    if (threadIdx.x == 0)
        for (int a = 0; a < D; a++) A->vsum[a] = S[a];
}

// (3) The walk again, with the same decisions: for every far cell (and
// one-point leaf) lam_i += J ub_i and the cell's centre adjoint -= J ub_i (one
// FP64 atomic per warp and cell: the cell index is warp-uniform); for the pairs
// of a several-point leaf the other point gets -J ub_i directly.
template <int D>
__global__ void __launch_bounds__(WALK_THREADS)
k_adj_walk(WalkParams P, const DevState *__restrict__ st, Cells cells, const float4 *__restrict__ sp,
           const uint32_t *__restrict__ sorig, const uint32_t *__restrict__ uid,
           const uint32_t *__restrict__ leaf_pre, const float *__restrict__ ub, float *__restrict__ lam_rep,
           double *__restrict__ xbar, double *__restrict__ lam_pair) {
    const uint32_t n = P.n, ncells = st->n_cells;
    const uint32_t p = blockIdx.x * WALK_THREADS + threadIdx.x;
    if (__all_sync(GR_FULL, p >= n)) return;
    const bool valid = p < n;
    const float4 me = valid ? sp[p] : make_float4(0.f, 0.f, 0.f, 0.f);
    const uint32_t mylp = valid ? leaf_pre[uid[p]] : 0xffffffffu;
    const uint32_t oi = valid ? sorig[p] : 0u;
    float vx = 0.f, vy = 0.f, vz = 0.f;
    if (valid) {
        vx = ub[(size_t)oi * D];
        vy = ub[(size_t)oi * D + 1];
        if (D == 3) vz = ub[(size_t)oi * D + 2];
    }
    uint32_t resume = valid ? 0u : 0xffffffffu;
    float lx = 0.f, ly = 0.f, lz = 0.f;
    const float kr = P.kr, th2 = P.theta2;
    const uint32_t lane = threadIdx.x % GR_WARP;
    uint32_t k = 0;
    while (k < ncells) {
        const float4 A = cell_a<D>(cells, k);
        const float4 B = cell_b<D>(cells, k);
        int32_t sk;
        uint32_t start;
        float cx, cy, cz, cm, w2, ox, oy, oz;
        if (D == 2) {
            cx = A.x; cy = A.y; cz = 0.f; cm = A.z; w2 = A.w;
            ox = B.x; oy = B.y; oz = 0.f;
            sk = __float_as_int(B.z);
            start = __float_as_uint(B.w);
        } else {
            const int2 Cc = cell_c3(cells, k);
            cx = A.x; cy = A.y; cz = A.z; cm = A.w;
            ox = B.x; oy = B.y; oz = B.z; w2 = B.w;
            sk = Cc.x;
            start = (uint32_t)Cc.y;
        }
        const bool leaf = sk < 0;
        uint32_t skip = leaf ? k + 1 : (uint32_t)sk;
        if (skip <= k || skip > ncells) skip = k + 1;
        const bool active = resume <= k;
        const bool holds = (k <= mylp) && (mylp < skip);
        const float dx = (me.x - cx) - ox, dy = (me.y - cy) - oy, dz = (D == 3) ? (me.z - cz) - oz : 0.f;
        const float d2 = (D == 3) ? dx * dx + dy * dy + dz * dz : dx * dx + dy * dy;
        const bool far = active && !holds && d2 > 0.f && w2 < th2 * d2;
        const bool open = active && !far;
        // a one-point leaf's pair is its body term (the point is its own centre)
        const bool body = far || (sk == -1 && open && !holds && d2 > 0.f);
        float jx = 0.f, jy = 0.f, jz = 0.f;
        if (body) {
            rep_jac<D>(kr * me.w * cm, dx, dy, dz, vx, vy, vz, jx, jy, jz);
            lx += jx;
            ly += jy;
            lz += jz;
        }
        if (far) resume = skip;
        const uint32_t any_body = __ballot_sync(GR_FULL, body);
        if (any_body) {  // warp-aggregated centre adjoint of cell k
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                jx += __shfl_xor_sync(GR_FULL, jx, o);
                jy += __shfl_xor_sync(GR_FULL, jy, o);
                if (D == 3) jz += __shfl_xor_sync(GR_FULL, jz, o);
            }
            if (lane == 0) {
                atomicAdd(&xbar[(size_t)k * D], -(double)jx);
                atomicAdd(&xbar[(size_t)k * D + 1], -(double)jy);
                if (D == 3) atomicAdd(&xbar[(size_t)k * D + 2], -(double)jz);
            }
        }
        if (sk == -1) {
            k = k + 1;
        } else if (leaf) {
            if (__any_sync(GR_FULL, open)) {
                int32_t cnt = -sk;
                if (start >= n || (uint32_t)cnt > n - start) cnt = 0;
                for (int32_t q = 0; q < cnt; q++) {
                    const uint32_t jp = start + (uint32_t)q;
                    const float4 o = __ldg(&sp[jp]);
                    if (open && jp != p) {
                        const float ex = me.x - o.x, ey = me.y - o.y, ez = (D == 3) ? me.z - o.z : 0.f;
                        if (!(ex == 0.f && ey == 0.f && (D == 2 || ez == 0.f))) {  // a jiggled pair is constant
                            float ax, ay, az;
                            rep_jac<D>(kr * me.w * o.w, ex, ey, ez, vx, vy, vz, ax, ay, az);
                            lx += ax;
                            ly += ay;
                            lz += az;
                            atomicAdd(&lam_pair[(size_t)jp * D], -(double)ax);
                            atomicAdd(&lam_pair[(size_t)jp * D + 1], -(double)ay);
                            if (D == 3) atomicAdd(&lam_pair[(size_t)jp * D + 2], -(double)az);
                        }
                    }
                }
            }
            k = k + 1;
        } else {
            k = __any_sync(GR_FULL, open) ? k + 1 : skip;
        }
    }
    if (valid) {
        lam_rep[(size_t)oi * D] = lx;
        lam_rep[(size_t)oi * D + 1] = ly;
        if (D == 3) lam_rep[(size_t)oi * D + 2] = lz;
    }
}

// (4) A cell's centre is sum m_j p_j / M over its points: every point takes
// m_j * sum over the cells holding it of xbar / M (its leaf and the leaf's cell
// ancestors), plus its direct pair terms.
template <int D>
__global__ void k_adj_down(const DevState *st, BinTree t, const uint32_t *__restrict__ leaf_start,
                           const uint32_t *__restrict__ leaf_pre, const Body *__restrict__ leaf_body,
                           const Body *__restrict__ int_body, const float4 *__restrict__ sp,
                           const uint32_t *__restrict__ sorig, const double *__restrict__ xbar,
                           const double *__restrict__ lam_pair, float *__restrict__ lam_com) {
    const uint32_t nu = st->n_unique;
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nu) return;
    double acc[3] = {0, 0, 0};
    {
        const double M = leaf_body[s].m;
        const uint32_t c = leaf_pre[s];
        for (int a = 0; a < D; a++) acc[a] += xbar[(size_t)c * D + a] / M;
    }
    int32_t par = t.leaf_parent[s];
    for (int depth = 0; par >= 0 && depth <= 66; depth++) {
        if (is_cell<D>(t, par)) {
            const double M = int_body[par].m;
            const uint32_t c = t.cell_of[par];
            for (int a = 0; a < D; a++) acc[a] += xbar[(size_t)c * D + a] / M;
        }
        par = t.int_parent[par];
    }
    for (uint32_t q = leaf_start[s]; q < leaf_start[s + 1]; q++) {
        const uint32_t j = sorig[q];
        const double m = sp[q].w;
        for (int a = 0; a < D; a++) lam_com[(size_t)j * D + a] = (float)(m * acc[a] + lam_pair[(size_t)q * D + a]);
    }
}

// (5) Attraction (CSR gather, state.rs:152-162 and networkx's linlog /
// distributed_action), dL/dc per CSR entry, and the sum of every part into the
// next lam.
template <int D>
__global__ void __launch_bounds__(FRC_THREADS)
k_adj_final(uint32_t n, int lin_log, int dissuade, const AdjScalars *A, const float4 *__restrict__ pos,
            const uint32_t *__restrict__ rp, const uint32_t *__restrict__ col, const float *__restrict__ wt,
            const float *__restrict__ lam, const float *__restrict__ ub, const float *__restrict__ v,
            const float *__restrict__ lam_rep, const float *__restrict__ lam_com, double *__restrict__ gce,
            float *__restrict__ lam_out) {
    const uint32_t i = blockIdx.x * FRC_THREADS + threadIdx.x;
    if (i >= n) return;
    const float4 p = pos[i];
    const double pc[3] = {p.x, p.y, p.z};
    double ai[3] = {0, 0, 0}, acc[3] = {0, 0, 0};
    const double mi = dissuade ? (double)p.w : 1.0;
    for (int a = 0; a < D; a++) ai[a] = ub[(size_t)i * D + a] / mi;
    for (uint32_t e = rp[i]; e < rp[i + 1]; e++) {
        const uint32_t j = col[e];
        const float4 q = pos[j];
        const double qc[3] = {q.x, q.y, q.z};
        const double mj = dissuade ? (double)q.w : 1.0;
        double dl[3] = {0, 0, 0}, df[3] = {0, 0, 0};
        for (int a = 0; a < D; a++) {
            dl[a] = qc[a] - pc[a];
            df[a] = ub[(size_t)j * D + a] / mj - ai[a];
        }
        const double dist = sqrt(dl[0] * dl[0] + dl[1] * dl[1] + dl[2] * dl[2]);
        double phi = 1.0, dphi = 0.0;
        if (lin_log) {
            if (dist > 0.0) {
                phi = log1p(dist) / dist;
                dphi = (dist / (1.0 + dist) - log1p(dist)) / (dist * dist);
            } else {
                phi = 0.0;
            }
        }
        const double c = wt[e];
        const double ddot = dl[0] * df[0] + dl[1] * df[1] + dl[2] * df[2];
        double gi = 0.0;
        for (int a = 0; a < D; a++) {
            acc[a] += c * (phi * df[a] + (dist > 0.0 ? dphi * dl[a] * ddot / dist : 0.0));
            gi += phi * ai[a] * dl[a];
        }
        gce[e] += gi;
    }
    for (int a = 0; a < D; a++) {
        const size_t k = (size_t)i * D + a;
        lam_out[k] = (float)((double)lam[k] + ((double)v[k] - A->vsum[a] / (double)n) + (double)lam_rep[k] +
                             (double)lam_com[k] + acc[a]);
    }
}

// The adjoint of a run grows by orders of magnitude per tick (FA2's speed
// controller and repulsion make the map expansive: the FP64 oracle's
// dL/dp0 on a 2,000-node SBM has norm ~1e5 after 5 ticks and ~1e37 after
// 200), beyond FP32. Between ticks the carried adjoints (lam', the controller
// adjoints and the accumulated dL/dc) are multiplied by 2^-k so that max |lam'|
// lies in [0.5, 1). The VJP is linear in what it carries and a power-of-two
// scale is exact, so this changes no value's significand; the host multiplies
// the results by 2^exponent at the end.
__global__ void k_adj_absmax(uint32_t count, const float *__restrict__ lam, AdjScalars *A) {
    float m = 0.f;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf(lam[i]));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m > 0.f) atomicMax(&A->absmax, __float_as_uint(m));
}

__global__ void k_adj_shift(AdjScalars *A) {
    const float m = __uint_as_float(A->absmax);
    int k = 0;
    if (m > 0.f && isfinite(m)) frexpf(m, &k);  // m = f 2^k, f in [0.5, 1)
    A->shift = k;
    A->exponent += k;
    A->absmax = 0u;
    A->LSW = ldexp(A->LSW, -k);
    A->LTR = ldexp(A->LTR, -k);
    A->Lsp = ldexp(A->Lsp, -k);
    A->Lse = ldexp(A->Lse, -k);
}

__global__ void k_adj_rescale(uint32_t count, float *__restrict__ lam, uint64_t ne, double *__restrict__ gce,
                              const AdjScalars *A) {
    const int k = A->shift;
    if (k == 0) return;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride)
        lam[i] = ldexpf(lam[i], -k);
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += stride) gce[e] = ldexp(gce[e], -k);
}

// dL/dc per simple edge (its two CSR entries), times dc/dw, onto the raw edge
// that survived the simple-graph pass.
__global__ void k_adj_edges(uint32_t ne, const uint32_t *__restrict__ csr_simple, const double *__restrict__ gce,
                            double *__restrict__ gs) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    atomicAdd(&gs[csr_simple[e]], gce[e]);
}

__global__ void k_adj_raw(uint32_t ms, const double *__restrict__ gs, const uint32_t *__restrict__ sraw,
                          const float *__restrict__ dcdw, double *__restrict__ graw) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ms) return;
    graw[sraw[s]] = gs[s] * (double)dcdw[s];
}

}  // namespace gr
