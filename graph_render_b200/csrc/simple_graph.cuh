// The simple graph every force layout shares (crates/graph-core/src/layout/force/mod.rs:60-131):
// self-loops dropped, each unordered pair kept once with the first raw edge's
// weight (ascending edge index), then a row CSR over both endpoints. Built on
// the device with the same radix sort as the tree: the sort is stable, so the
// first raw edge of a pair is the first of its run.
#pragma once

#include "common.cuh"

namespace gr {

constexpr uint64_t NO_EDGE = ~0ull;

__global__ void k_edge_keys(uint64_t m, const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst,
                            uint32_t n, uint64_t *__restrict__ keys, uint32_t *__restrict__ vals,
                            uint32_t *err) {
    uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m) return;
    uint32_t a = src[e], b = dst[e];
    uint64_t key = NO_EDGE;
    if (a >= n || b >= n)
        atomicOr(err, 1u);
    else if (a != b)
        key = ((uint64_t)min(a, b) << 32) | (uint64_t)max(a, b);
    keys[e] = key;
    vals[e] = (uint32_t)e;
}

__global__ void k_edge_flags(uint32_t m, const uint64_t *__restrict__ keys, uint32_t *__restrict__ flag) {
    uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= m) return;
    uint64_t k = keys[q];
    flag[q] = (k != NO_EDGE && (q == 0 || k != keys[q - 1])) ? 1u : 0u;
}

// One simple edge per flagged run head: its effective attraction weight
// w^influence, and two directed CSR entries (row << 32 | col).
__global__ void k_edge_emit(uint32_t m, const uint64_t *__restrict__ keys, const uint32_t *__restrict__ vals,
                            const uint32_t *__restrict__ flag, const uint32_t *__restrict__ excl,
                            const double *__restrict__ w, double influence, float *__restrict__ weff,
                            uint32_t *__restrict__ slo, uint32_t *__restrict__ shi,
                            uint64_t *__restrict__ dkeys, uint32_t *__restrict__ dvals, uint32_t *err,
                            uint32_t *__restrict__ sraw, float *__restrict__ dcdw) {
    uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= m || !flag[q]) return;
    uint32_t s = excl[q];
    uint64_t k = keys[q];
    uint32_t lo = (uint32_t)(k >> 32), hi = (uint32_t)k;
    double c = 1.0, dc = 0.0;
    if (w && influence != 0.0) {
        double x = w[vals[q]];
        if (!(isfinite(x) && x > 0.0)) atomicOr(err, 2u);
        c = influence == 1.0 ? x : pow(x, influence);
        dc = influence == 1.0 ? 1.0 : influence * c / x;  // d(w^influence)/dw
    }
    weff[s] = (float)c;
    sraw[s] = vals[q];  // the raw edge that survived (first of its pair)
    dcdw[s] = (float)dc;
    slo[s] = lo;
    shi[s] = hi;
    dkeys[2 * (uint64_t)s] = ((uint64_t)lo << 32) | hi;
    dvals[2 * (uint64_t)s] = s;
    dkeys[2 * (uint64_t)s + 1] = ((uint64_t)hi << 32) | lo;
    dvals[2 * (uint64_t)s + 1] = s;
}

// Row offsets (every row, empty ones included), columns and weights of the
// sorted directed entries.
__global__ void k_csr(uint32_t n, uint32_t ne, const uint64_t *__restrict__ dkeys,
                      const uint32_t *__restrict__ dvals, const float *__restrict__ weff,
                      uint32_t *__restrict__ rp, uint32_t *__restrict__ col, float *__restrict__ wt) {
    uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= ne) return;
    uint64_t k = dkeys[q];
    uint32_t row = (uint32_t)(k >> 32);
    col[q] = (uint32_t)k;
    wt[q] = weff[dvals[q]];
    int64_t prev = q == 0 ? -1 : (int64_t)(dkeys[q - 1] >> 32);
    for (int64_t r = prev + 1; r <= (int64_t)row; r++) rp[r] = q;
    if (q == ne - 1)
        for (uint32_t r = row + 1; r <= n; r++) rp[r] = ne;
}

// float4 node records: the start coordinates with mass = simple degree + 1
// (state.rs:86) in .w.
template <int D>
__global__ void k_init_nodes(uint32_t n, const float *__restrict__ xyz, const uint32_t *__restrict__ rp,
                             float4 *__restrict__ pos) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float m = (float)(rp[i + 1] - rp[i]) + 1.0f;
    pos[i] = make_float4(xyz[(size_t)i * D], xyz[(size_t)i * D + 1], D == 3 ? xyz[(size_t)i * D + 2] : 0.f, m);
}

}  // namespace gr
