// Particle-mesh many-body pass (2D) for the d3-force session: the positions'
// box placed on a side x side mesh, cloud-in-cell deposit of unit masses, FFT
// convolution with the law's vector Green's function (field = re, im), bilinear
// read, times charge * alpha onto each velocity.
//
// Reference: crates/graph-core/src/layout/force/particle_mesh/{mesh,frame,
// deposit,kernel,fft,charge}.rs. Frame placement (frame.rs place / fit: cell
// size 2^(step/4), the smallest step whose cells + reach fit the side) runs in
// FP64 in the last block of the bounds pass. The deposit is a gather: nodes are
// radix-sorted by their cell, and every mesh point sums the nodes of the four
// cells that touch it in a fixed order, so the density is the same every run.
// The FFT is radix-2 in shared memory along rows, with a tiled transpose between
// the two directions; spectra stay transposed, so the inverse's transpose
// restores the natural layout. FP32 mesh values, FP64 frame.
#pragma once

#include "common.cuh"

namespace gr {

constexpr int PM_T = 256;
constexpr int PM_MIN_SIDE = 128, PM_MAX_SIDE = 1024;  // mesh.rs side_for, fft.rs MAX_SIDE

struct PmState {
    double lo[2], hi[2];
    double mean[2];  // the positions' mean (center force)
    double h, ox, oy;
    int32_t step;
    uint32_t cells, reach, valid;
    uint32_t ticket;
};

// Extent (finite points) and FP64 coordinate sums; the last block folds the
// block partials in block order, places the frame and takes the mean.
__global__ void __launch_bounds__(PM_T)
k_pm_bounds(uint32_t n, const float4 *__restrict__ p, uint32_t side, double dmax, double dmax2,
            double *__restrict__ part, PmState *S) {
    __shared__ double s_red[PM_T / GR_WARP];
    __shared__ bool s_last;
    double lx = INFINITY, ly = INFINITY, hx = -INFINITY, hy = -INFINITY, sx = 0.0, sy = 0.0;
    for (uint32_t i = blockIdx.x * PM_T + threadIdx.x; i < n; i += gridDim.x * PM_T) {
        const float4 a = p[i];
        sx += (double)a.x;
        sy += (double)a.y;
        if (!isfinite(a.x) || !isfinite(a.y)) continue;
        lx = fmin(lx, (double)a.x);
        ly = fmin(ly, (double)a.y);
        hx = fmax(hx, (double)a.x);
        hy = fmax(hy, (double)a.y);
    }
    // min / max by warp butterflies then warp 0 (exact, so order-free)
    for (int o = 16; o > 0; o >>= 1) {
        lx = fmin(lx, __shfl_xor_sync(GR_FULL, lx, o));
        ly = fmin(ly, __shfl_xor_sync(GR_FULL, ly, o));
        hx = fmax(hx, __shfl_xor_sync(GR_FULL, hx, o));
        hy = fmax(hy, __shfl_xor_sync(GR_FULL, hy, o));
    }
    __shared__ double s_m[4][PM_T / GR_WARP];
    const int w = threadIdx.x / GR_WARP, l = threadIdx.x % GR_WARP;
    if (l == 0) {
        s_m[0][w] = lx;
        s_m[1][w] = ly;
        s_m[2][w] = hx;
        s_m[3][w] = hy;
    }
    sx = block_sum_d<PM_T>(sx, s_red);
    sy = block_sum_d<PM_T>(sy, s_red);
    if (threadIdx.x == 0) {
        for (int k = 1; k < PM_T / GR_WARP; k++) {
            s_m[0][0] = fmin(s_m[0][0], s_m[0][k]);
            s_m[1][0] = fmin(s_m[1][0], s_m[1][k]);
            s_m[2][0] = fmax(s_m[2][0], s_m[2][k]);
            s_m[3][0] = fmax(s_m[3][0], s_m[3][k]);
        }
        double *q = part + (size_t)blockIdx.x * 6;
        q[0] = s_m[0][0];
        q[1] = s_m[1][0];
        q[2] = s_m[2][0];
        q[3] = s_m[3][0];
        q[4] = sx;
        q[5] = sy;
    }
    if (!last_block_done(&S->ticket, &s_last)) return;
    // the last block folds the partials: thread t takes blocks t, t + PM_T, ... in
    // order, then the block combines the threads (min / max exact in any order, the
    // sums in block_sum_d's fixed shape)
    double L0 = INFINITY, L1 = INFINITY, H0 = -INFINITY, H1 = -INFINITY;
    for (uint32_t b = threadIdx.x; b < gridDim.x; b += PM_T) {
        const double *q = part + (size_t)b * 6;
        L0 = fmin(L0, __ldcg(q + 0));
        L1 = fmin(L1, __ldcg(q + 1));
        H0 = fmax(H0, __ldcg(q + 2));
        H1 = fmax(H1, __ldcg(q + 3));
    }
    double X = strided_sum_cg<PM_T>(part, gridDim.x, 6, 4);
    double Y = strided_sum_cg<PM_T>(part, gridDim.x, 6, 5);
    for (int o = 16; o > 0; o >>= 1) {
        L0 = fmin(L0, __shfl_xor_sync(GR_FULL, L0, o));
        L1 = fmin(L1, __shfl_xor_sync(GR_FULL, L1, o));
        H0 = fmax(H0, __shfl_xor_sync(GR_FULL, H0, o));
        H1 = fmax(H1, __shfl_xor_sync(GR_FULL, H1, o));
    }
    __syncthreads();  // s_m is reused
    if (l == 0) {
        s_m[0][w] = L0;
        s_m[1][w] = L1;
        s_m[2][w] = H0;
        s_m[3][w] = H1;
    }
    X = block_sum_d<PM_T>(X, s_red);
    Y = block_sum_d<PM_T>(Y, s_red);
    if (threadIdx.x != 0) return;
    for (int k = 1; k < PM_T / GR_WARP; k++) {
        L0 = fmin(L0, s_m[0][k]);
        L1 = fmin(L1, s_m[1][k]);
        H0 = fmax(H0, s_m[2][k]);
        H1 = fmax(H1, s_m[3][k]);
    }
    S->lo[0] = L0;
    S->lo[1] = L1;
    S->hi[0] = H0;
    S->hi[1] = H1;
    S->mean[0] = n ? X / (double)n : 0.0;
    S->mean[1] = n ? Y / (double)n : 0.0;
    S->valid = 0u;
    const double span = fmax(H0 - L0, H1 - L1);
    if (n < 2 || !(dmax2 > 0.0) || !(L0 <= H0) || !isfinite(span)) return;
    int step = (int)floor(4.0 * log2(span / (double)side));
    if (step < -32) step = -32;
    for (int guard = 0; guard < 8192; guard++, step++) {  // frame.rs place: the first step that fits
        const double h = exp2((double)step / 4.0);
        const double cells = floor(span / h) + 3.0;
        if (cells > (double)side) continue;
        const uint32_t c = (uint32_t)cells;
        const double rr = ceil(dmax / h);
        const uint32_t reach = rr > (double)(c - 1) ? c - 1 : (uint32_t)rr;
        if (c + reach > side) continue;
        S->step = step;
        S->h = h;
        S->cells = c;
        S->reach = reach;
        S->ox = floor(L0 / h) * h;
        S->oy = floor(L1 / h) * h;
        S->valid = 1u;
        return;
    }
}

// frame.rs scaled + split: the node's mesh cell and its fractions in it.
__device__ __forceinline__ void pm_split(const PmState &S, float px, float py, uint32_t &cx, uint32_t &cy, float &fx,
                                         float &fy) {
    const double u0 = ((double)px - S.ox) / S.h, u1 = ((double)py - S.oy) / S.h;
    const uint32_t top = S.cells - 2;
    const uint32_t c0 = u0 > 0.0 ? (uint32_t)fmin(u0, (double)top) : 0u;
    const uint32_t c1 = u1 > 0.0 ? (uint32_t)fmin(u1, (double)top) : 0u;
    cx = c0;
    cy = c1;
    fx = (float)fmin(fmax(u0 - (double)c0, 0.0), 1.0);
    fy = (float)fmin(fmax(u1 - (double)c1, 0.0), 1.0);
}

// Each node's cell key (row-major) and fractions, for the sort and the deposit.
__global__ void k_pm_stencil(uint32_t n, const float4 *__restrict__ p, const PmState *S, uint32_t side,
                             uint64_t *__restrict__ key, uint32_t *__restrict__ val, float2 *__restrict__ frac) {
    const uint32_t i = blockIdx.x * PM_T + threadIdx.x;
    if (i >= n || !S->valid) return;
    uint32_t cx, cy;
    float fx, fy;
    const float4 a = p[i];
    pm_split(*S, a.x, a.y, cx, cy, fx, fy);
    key[i] = (uint64_t)cy * side + cx;
    val[i] = i;
    frac[i] = make_float2(fx, fy);
}

// First and one-past-last sorted position of every occupied cell (the others
// were cleared to 0, 0).
__global__ void k_pm_mark(uint32_t n, const PmState *S, const uint64_t *__restrict__ key, uint32_t *__restrict__ cs,
                          uint32_t *__restrict__ ce) {
    const uint32_t q = blockIdx.x * PM_T + threadIdx.x;
    if (q >= n || !S->valid) return;
    const uint64_t k = key[q];
    if (q == 0 || key[q - 1] != k) cs[k] = q;
    if (q + 1 == n || key[q + 1] != k) ce[k] = q + 1;
}

// deposit.rs: mesh point (gx, gy) gathers the cloud-in-cell weights of the nodes
// in the four cells touching it, cell by cell in a fixed order, nodes in sorted
// order. Writes the whole mesh (zero where nothing lands).
__global__ void k_pm_deposit(uint32_t side, const PmState *S, const uint32_t *__restrict__ cs,
                             const uint32_t *__restrict__ ce, const uint32_t *__restrict__ val,
                             const float2 *__restrict__ frac, float2 *__restrict__ mesh) {
    const uint32_t g = blockIdx.x * PM_T + threadIdx.x;
    if (g >= side * side) return;
    float acc = 0.f;
    if (S->valid) {
        const int gx = (int)(g % side), gy = (int)(g / side), top = (int)S->cells - 2;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int sx = gx - 1 + (c & 1), sy = gy - 1 + (c >> 1);  // source cell
            if (sx < 0 || sy < 0 || sx > top || sy > top) continue;
            const bool xplus = (c & 1) == 0, yplus = (c >> 1) == 0;  // g is the source's +1 corner on that axis
            const uint32_t cell = (uint32_t)sy * side + (uint32_t)sx;
            for (uint32_t q = cs[cell]; q < ce[cell]; q++) {
                const float2 f = frac[val[q]];
                acc += (xplus ? f.x : 1.f - f.x) * (yplus ? f.y : 1.f - f.y);
            }
        }
    }
    mesh[g] = make_float2(acc, 0.f);
}

// kernel.rs sample + green: the law's vector Green's function at every mesh
// offset within reach (wrapped), scaled by 1 / side^2; zero elsewhere.
__global__ void k_pm_green(uint32_t side, const PmState *S, double dmin2, double dmax2, float2 *__restrict__ g) {
    const uint32_t q = blockIdx.x * PM_T + threadIdx.x;
    if (q >= side * side) return;
    float2 out = make_float2(0.f, 0.f);
    if (S->valid) {
        const int reach = (int)S->reach, c = (int)(q % side), r = (int)(q / side), sd = (int)side;
        // a wrapped index both offsets reach is written by the positive one (the later write)
        const int dx = c <= reach ? c : (c >= sd - reach ? c - sd : INT32_MIN);
        const int dy = r <= reach ? r : (r >= sd - reach ? r - sd : INT32_MIN);
        if (dx != INT32_MIN && dy != INT32_MIN) {
            const double rx = (double)dx * S->h, ry = (double)dy * S->h;
            double l = rx * rx + ry * ry;
            if (l != 0.0 && l < dmax2) {
                if (l < dmin2) l = sqrt(dmin2 * l);
                const double scale = 1.0 / ((double)side * (double)side);
                out = make_float2((float)(-rx / l * scale), (float)(-ry / l * scale));
            }
        }
    }
    g[q] = out;
}

// One radix-2 transform per row (one block per row), in shared memory:
// bit-reversed load, log2(side) butterfly stages, twiddles tw[k] = e^(-2 pi i k
// / side) (conjugated for the inverse); neither direction is scaled.
template <bool INV>
__global__ void k_pm_fft_rows(float2 *__restrict__ data, const float2 *__restrict__ tw, uint32_t side, uint32_t bits,
                              const PmState *S) {
    if (!S->valid) return;
    extern __shared__ float2 pm_row[];
    float2 *row = data + (size_t)blockIdx.x * side;
    for (uint32_t i = threadIdx.x; i < side; i += blockDim.x) pm_row[__brev(i) >> (32 - bits)] = row[i];
    __syncthreads();
    for (uint32_t m = 1; m < side; m <<= 1) {
        for (uint32_t b = threadIdx.x; b < side / 2; b += blockDim.x) {
            const uint32_t k = b % m, i0 = (b / m) * 2 * m + k, i1 = i0 + m;
            float2 w = tw[k * (side / (2 * m))];
            if (INV) w.y = -w.y;
            const float2 a = pm_row[i0], c = pm_row[i1];
            const float2 t = make_float2(c.x * w.x - c.y * w.y, c.x * w.y + c.y * w.x);
            pm_row[i0] = make_float2(a.x + t.x, a.y + t.y);
            pm_row[i1] = make_float2(a.x - t.x, a.y - t.y);
        }
        __syncthreads();
    }
    for (uint32_t i = threadIdx.x; i < side; i += blockDim.x) row[i] = pm_row[i];
}

// out = in^T, 32 x 32 tiles through shared memory.
__global__ void k_pm_transpose(const float2 *__restrict__ in, float2 *__restrict__ out, uint32_t side,
                               const PmState *S) {
    if (!S->valid) return;
    __shared__ float2 tile[32][33];
    const uint32_t bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (uint32_t j = threadIdx.y; j < 32; j += blockDim.y) tile[j][threadIdx.x] = in[(size_t)(by + j) * side + bx + threadIdx.x];
    __syncthreads();
    for (uint32_t j = threadIdx.y; j < 32; j += blockDim.y) out[(size_t)(bx + j) * side + by + threadIdx.x] = tile[threadIdx.x][j];
}

__global__ void k_pm_mul(uint32_t count, float2 *__restrict__ a, const float2 *__restrict__ b, const PmState *S) {
    const uint32_t q = blockIdx.x * PM_T + threadIdx.x;
    if (q >= count || !S->valid) return;
    const float2 x = a[q], y = b[q];
    a[q] = make_float2(x.x * y.x - x.y * y.y, x.x * y.y + x.y * y.x);
}

// mesh.rs read: the field bilinear at every node, times charge * alpha, onto
// its velocity.
__global__ void k_pm_read(uint32_t n, const float4 *__restrict__ p, const PmState *S, uint32_t side, float charge,
                          const double *alpha, const float2 *__restrict__ field, float2 *__restrict__ v) {
    const uint32_t i = blockIdx.x * PM_T + threadIdx.x;
    if (i >= n || !S->valid) return;
    uint32_t cx, cy;
    float fx, fy;
    const float4 a = p[i];
    pm_split(*S, a.x, a.y, cx, cy, fx, fy);
    const size_t at = (size_t)cy * side + cx;
    const float w[4] = {(1.f - fx) * (1.f - fy), fx * (1.f - fy), (1.f - fx) * fy, fx * fy};
    const size_t cell[4] = {at, at + 1, at + side, at + side + 1};
    float ex = 0.f, ey = 0.f;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const float2 e = field[cell[k]];
        ex += e.x * w[k];
        ey += e.y * w[k];
    }
    const float s = charge * (float)*alpha;
    float2 u = v[i];
    u.x += ex * s;
    u.y += ey * s;
    v[i] = u;
}

}  // namespace gr
