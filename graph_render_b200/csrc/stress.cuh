// Kruskal stress-1 against hop distance, and the multi-source BFS it needs.
//
// Reference: crates/graph-cli/src/bench.rs:255-295 (`stress`): BFS from every
// max(n / SOURCES, 1)-th node, then over every reachable (source, target) pair
// with d = hops and e = |p_target - p_source| (the f32 difference per axis,
// widened to f64, then hypot): DE = sum d e, EE = sum e^2, DD = sum d^2 in FP64,
// stress = sqrt(max((DD - DE / EE * DE) / DD, 0)), or 1 when EE or DD is 0.
//
// The BFS runs 64 sources at a time as one level-synchronous pull: node v's
// 64-bit frontier word at level L is the OR of its neighbours' words at L - 1,
// minus the sources that reached v already; each new bit writes v's hop count
// for that source. Hop counts are integers, so the result is the reference's
// exactly. The sums are per-thread sequential over a fixed grid-stride, then
// block sums and one fold of the block partials in block order: the same value
// every run (the reference's own order differs, so they agree to FP64 rounding).
#pragma once

#include "common.cuh"

namespace gr {

constexpr int BFS_T = 256;
constexpr int STRESS_T = 256;
constexpr uint32_t HOP_NONE = 0xffffffffu;

// The batch's sources: bit b of node sources[k0 + b] in visited and frontier,
// hop 0 at that node.
__global__ void k_msbfs_seed(uint32_t n, uint32_t k0, uint32_t kb, const uint32_t *__restrict__ sources,
                             unsigned long long *visited, unsigned long long *frontier, uint32_t *__restrict__ hops) {
    const uint32_t b = threadIdx.x;
    if (b >= kb) return;
    const uint32_t v = sources[k0 + b];
    atomicOr(&visited[v], 1ull << b);
    atomicOr(&frontier[v], 1ull << b);
    hops[(size_t)(k0 + b) * n + v] = 0u;
}

// One level: node v takes the batch's sources that reached any neighbour at the
// previous level and not v yet. Reads frontier, writes next (ping-pong).
__global__ void __launch_bounds__(BFS_T)
k_msbfs_level(uint32_t n, const uint64_t *__restrict__ rp, const uint32_t *__restrict__ col, unsigned long long all,
              const unsigned long long *__restrict__ frontier, unsigned long long *__restrict__ visited,
              unsigned long long *__restrict__ next, uint32_t *__restrict__ hops, uint32_t k0, uint32_t level,
              uint32_t *changed) {
    const uint32_t v = blockIdx.x * BFS_T + threadIdx.x;
    if (v >= n) return;
    const unsigned long long vis = visited[v];
    unsigned long long acc = 0ull;
    if ((vis & all) != all) {
        const uint64_t e1 = rp[v + 1];
        for (uint64_t e = rp[v]; e < e1; e++) {
            acc |= frontier[col[e]];
            if (((acc | vis) & all) == all) break;  // nothing left to reach v
        }
        acc &= ~vis & all;
    }
    next[v] = acc;
    if (acc) {
        visited[v] = vis | acc;
        for (unsigned long long a = acc; a; a &= a - 1) hops[(size_t)(k0 + __ffsll((long long)a) - 1) * n + v] = level;
        *changed = 1u;
    }
}

// DE, EE, DD over every (source s, target v) pair of a k x n hop table; the last
// block folds the block partials in block order into out[0..3).
__global__ void __launch_bounds__(STRESS_T)
k_stress_sums(uint32_t n, uint32_t k, const uint32_t *__restrict__ sources, const uint32_t *__restrict__ hops,
              const float *__restrict__ x, const float *__restrict__ y, double *__restrict__ part, double *out,
              uint32_t *ticket) {
    __shared__ double s_red[STRESS_T / GR_WARP];
    __shared__ bool s_last;
    double de = 0.0, ee = 0.0, dd = 0.0;
    const uint64_t total = (uint64_t)k * n, stride = (uint64_t)gridDim.x * STRESS_T;
    for (uint64_t idx = (uint64_t)blockIdx.x * STRESS_T + threadIdx.x; idx < total; idx += stride) {
        const uint32_t s = (uint32_t)(idx / n), v = (uint32_t)(idx % n);
        const uint32_t from = sources[s], h = hops[idx];
        if (v == from || h == HOP_NONE) continue;
        const double dist = (double)h;
        const double dx = (double)(x[v] - x[from]), dy = (double)(y[v] - y[from]);
        const double e = hypot(dx, dy);
        de += dist * e;
        ee += e * e;
        dd += dist * dist;
    }
    de = block_sum_d<STRESS_T>(de, s_red);
    ee = block_sum_d<STRESS_T>(ee, s_red);
    dd = block_sum_d<STRESS_T>(dd, s_red);
    const uint32_t G = gridDim.x;
    if (threadIdx.x == 0) {
        part[blockIdx.x] = de;
        part[G + blockIdx.x] = ee;
        part[2 * G + blockIdx.x] = dd;
    }
    if (!last_block_done(ticket, &s_last)) return;
    if (threadIdx.x < 3) {
        double t = 0.0;
        for (uint32_t b = 0; b < G; b++) t += part[threadIdx.x * G + b];
        out[threadIdx.x] = t;
    }
}

}  // namespace gr
