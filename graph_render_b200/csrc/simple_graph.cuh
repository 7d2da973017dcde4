// The simple graph every force layout shares (crates/graph-core/src/layout/force/mod.rs:60-131):
// self-loops dropped, each unordered pair kept once with the first raw edge's
// weight (ascending edge index), then a row CSR over both endpoints. Built on
// the device with the same radix sort as the tree: the sort is stable, so the
// first raw edge of a pair is the first of its run.
#pragma once

#include "common.cuh"

namespace gr {

// An edge key packs its two node ids at the width of n: (a << bits) | b with
// bits = the bit length of n, so a key has 2 bits significant bits and the sort
// takes 2 bits / 8 digits (1M nodes: 40 bits, 5 digits, not 8). The largest
// 2-bits-bit value (no valid key reaches it, as a, b <= n - 1 < 2^bits - 1)
// marks a dropped edge and sorts last.
struct EdgeKey {
    int bits;
    __host__ __device__ uint64_t pack(uint32_t a, uint32_t b) const { return ((uint64_t)a << bits) | b; }
    __host__ __device__ uint32_t hi(uint64_t k) const { return (uint32_t)(k >> bits); }
    __host__ __device__ uint32_t lo(uint64_t k) const { return (uint32_t)(k & ((1ull << bits) - 1)); }
    __host__ __device__ uint64_t none() const { return bits >= 32 ? ~0ull : (1ull << (2 * bits)) - 1; }
};

inline EdgeKey edge_key_for(uint32_t n) {
    int b = 1;
    while (b < 32 && (n >> b) != 0u) b++;
    return EdgeKey{b};
}

__global__ void k_edge_keys(uint64_t m, const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst,
                            uint32_t n, EdgeKey ek, uint64_t *__restrict__ keys, uint32_t *__restrict__ vals,
                            uint32_t *err) {
    uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m) return;
    uint32_t a = src[e], b = dst[e];
    uint64_t key = ek.none();
    if (a >= n || b >= n)
        atomicOr(err, 1u);
    else if (a != b)
        key = ek.pack(min(a, b), max(a, b));
    keys[e] = key;
    vals[e] = (uint32_t)e;
}

__global__ void k_edge_flags(uint32_t m, EdgeKey ek, const uint64_t *__restrict__ keys, uint32_t *__restrict__ flag) {
    uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= m) return;
    uint64_t k = keys[q];
    flag[q] = (k != ek.none() && (q == 0 || k != keys[q - 1])) ? 1u : 0u;
}

// One simple edge per flagged run head: its effective attraction weight
// w^influence, and two directed CSR entries (row, col packed as an EdgeKey).
__global__ void k_edge_emit(uint32_t m, EdgeKey ek, const uint64_t *__restrict__ keys, const uint32_t *__restrict__ vals,
                            const uint32_t *__restrict__ flag, const uint32_t *__restrict__ excl,
                            const double *__restrict__ w, double influence, float *__restrict__ weff,
                            uint32_t *__restrict__ slo, uint32_t *__restrict__ shi,
                            uint64_t *__restrict__ dkeys, uint32_t *__restrict__ dvals, uint32_t *err,
                            uint32_t *__restrict__ sraw, float *__restrict__ dcdw) {
    uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= m || !flag[q]) return;
    uint32_t s = excl[q];
    uint64_t k = keys[q];
    uint32_t lo = ek.hi(k), hi = ek.lo(k);  // the smaller id is the key's high part
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
    dkeys[2 * (uint64_t)s] = ek.pack(lo, hi);
    dvals[2 * (uint64_t)s] = s;
    dkeys[2 * (uint64_t)s + 1] = ek.pack(hi, lo);
    dvals[2 * (uint64_t)s + 1] = s;
}

// Row offsets (every row, empty ones included), columns and weights of the
// sorted directed entries.
__global__ void k_csr(uint32_t n, uint32_t ne, EdgeKey ek, const uint64_t *__restrict__ dkeys,
                      const uint32_t *__restrict__ dvals, const float *__restrict__ weff,
                      uint32_t *__restrict__ rp, uint32_t *__restrict__ col, float *__restrict__ wt) {
    uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= ne) return;
    uint64_t k = dkeys[q];
    uint32_t row = ek.hi(k);
    col[q] = ek.lo(k);
    wt[q] = weff[dvals[q]];
    int64_t prev = q == 0 ? -1 : (int64_t)ek.hi(dkeys[q - 1]);
    for (int64_t r = prev + 1; r <= (int64_t)row; r++) rp[r] = q;
    if (q == ne - 1)
        for (uint32_t r = row + 1; r <= n; r++) rp[r] = ne;
}

// Draw k (from 0) of Mulberry32 seeded with `seed` as a float in [0, 1)
// (state.rs:272-283, synthetic.rs:37-50): the generator's state after k + 1
// steps is seed + (k + 1) * 0x6D2B79F5 (mod 2^32), so any draw is computed
// directly; u / 2^32 is exact in FP64 and then rounded to FP32 like the
// reference's f32 start.
__device__ __forceinline__ float mulberry32_draw(uint32_t seed, uint64_t k) {
    const uint32_t a = seed + (uint32_t)(k + 1u) * 0x6D2B79F5u;
    uint32_t t = (a ^ (a >> 15)) * (1u | a);
    t = (t + ((t ^ (t >> 7)) * (61u | t))) ^ t;
    return (float)((double)(t ^ (t >> 14)) * 0x1p-32);
}

// float4 node records: the start coordinates with mass = simple degree + 1
// (state.rs:86) in .w; a non-finite start coordinate sets bit 4 of *err. A
// null xyz means the seeded start: node i's axes are Mulberry32(seed) draws
// D i .. D i + D - 1.
template <int D>
__global__ void k_init_nodes(uint32_t n, const float *__restrict__ xyz, const uint32_t *__restrict__ rp,
                             float4 *__restrict__ pos, uint32_t *err, uint32_t seed = 0) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float m = (float)(rp[i + 1] - rp[i]) + 1.0f;
    if (!xyz) {
        const uint64_t k = (uint64_t)i * D;
        pos[i] = make_float4(mulberry32_draw(seed, k), mulberry32_draw(seed, k + 1),
                             D == 3 ? mulberry32_draw(seed, k + 2) : 0.f, m);
        return;
    }
    const float x = xyz[(size_t)i * D], y = xyz[(size_t)i * D + 1], z = D == 3 ? xyz[(size_t)i * D + 2] : 0.f;
    if (!(isfinite(x) && isfinite(y) && isfinite(z))) atomicOr(err, 4u);
    pos[i] = make_float4(x, y, z, m);
}

// The seeded start of a concatenation of graphs: node i of the concatenation
// belongs to graph g with off[g] <= i < off[g + 1] (off has graphs entries,
// ascending), and its axes are draws D (i - off[g]) .. + D - 1 of
// Mulberry32(seed[g]), each graph's own start.
template <int D>
__global__ void k_init_nodes_seeded(uint32_t n, const uint32_t *__restrict__ off, const uint32_t *__restrict__ seed,
                                    uint32_t graphs, const uint32_t *__restrict__ rp, float4 *__restrict__ pos) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || graphs == 0) return;
    uint32_t lo = 0, hi = graphs;  // the last g with off[g] <= i
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) / 2;
        if (off[mid] <= i) lo = mid;
        else hi = mid;
    }
    const uint64_t k = (uint64_t)(i - off[lo]) * D;
    const float m = (float)(rp[i + 1] - rp[i]) + 1.0f;
    pos[i] = make_float4(mulberry32_draw(seed[lo], k), mulberry32_draw(seed[lo], k + 1),
                         D == 3 ? mulberry32_draw(seed[lo], k + 2) : 0.f, m);
}

// Heavy rows (degree > light_max) take ceil(degree / seg) segments: the count
// per row, then (after an exclusive scan into first) each heavy row's segments.
__global__ void k_seg_count(uint32_t n, const uint32_t *__restrict__ rp, uint32_t light_max, uint32_t seg,
                            uint32_t *__restrict__ cnt) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t d = rp[i + 1] - rp[i];
    cnt[i] = d > light_max ? (d + seg - 1) / seg : 0u;
}

__global__ void k_seg_fill(uint32_t n, const uint32_t *__restrict__ rp, uint32_t light_max, uint32_t seg,
                           const uint32_t *__restrict__ first, uint32_t *__restrict__ seg_row) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t d = rp[i + 1] - rp[i];
    if (d <= light_max) return;
    const uint32_t c = (d + seg - 1) / seg, f = first[i];
    for (uint32_t k = 0; k < c; k++) seg_row[f + k] = i;
}

}  // namespace gr
