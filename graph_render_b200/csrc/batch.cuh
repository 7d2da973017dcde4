// Batched ForceAtlas2: thousands of independent graphs in one persistent launch.
//
// Each CTA takes graphs from a queue ordered largest first and runs every tick
// of its graph by itself: the same per-item functions as the one-graph engine
// (Morton key, Karras node with its cell marks, point-term prefix, cell writer,
// per-lane walk, node force, node update) over block-level sort / scan / reductions, with
// __syncthreads between phases instead of kernel boundaries. A graph's state
// (positions, CSR rows, FP64 speed controller) lives in global memory; the
// tree scratch lives in the CTA's slot, sized for the largest graph. No
// collective and no inter-CTA wait: graphs are independent.
#pragma once

#include "common.cuh"
#include "forces.cuh"
#include "tree.cuh"
#include "walk.cuh"

namespace gr {

struct BatchGraph {
    uint32_t off, n;          // global node range
    uint32_t heavy0, heavy1;  // range in the heavy-row list (rows > LIGHT_MAX entries)
    float kr, th2, gravity;
    uint32_t seed;
    int lin_log, strong_gravity, dissuade_hubs, pad;
    double jitter_tolerance;
};

struct BatchState {  // per graph; FP64 controller as in DevState
    double swing, traction, speed, speed_efficiency, moved;
    unsigned long long far_count, pair_count;
    uint32_t iter_no, converged, error, pad;
};

// Per-slot scratch, carved from one allocation in a fixed order.
struct SlotView {
    uint64_t *keys, *kalt, *ukey;
    uint32_t *vals, *valt, *sorig, *flag, *excl, *uid, *leaf_start, *levels, *P, *leaf_pre;
    float4 *sp;
    BinTree bt;
    BodyDD *pre;        // double-double prefix of the point terms at every leaf start (nu + 1)
    uint8_t *cell_flag;  // internal node -> 1 when it is a cell
    Cells cells;
    float *rep, *U, *att;
};

__host__ __device__ inline size_t slot_align(size_t x) { return (x + 255) & ~(size_t)255; }

template <typename T>
__host__ __device__ inline T *slot_take(unsigned char *base, size_t &off, size_t count) {
    off = slot_align(off);
    T *p = (T *)(base + off);
    off += (count ? count : 1) * sizeof(T);
    return p;
}

// Lays a slot out for graphs of up to nmax nodes; returns the bytes used.
__host__ __device__ inline size_t slot_carve(unsigned char *base, uint32_t nmax, int D, SlotView &v) {
    size_t off = 0;
    const size_t n = nmax;
    v.keys = slot_take<uint64_t>(base, off, n);
    v.kalt = slot_take<uint64_t>(base, off, n);
    v.ukey = slot_take<uint64_t>(base, off, n);
    v.vals = slot_take<uint32_t>(base, off, n);
    v.valt = slot_take<uint32_t>(base, off, n);
    v.sorig = slot_take<uint32_t>(base, off, n);
    v.flag = slot_take<uint32_t>(base, off, n);
    v.excl = slot_take<uint32_t>(base, off, n);
    v.uid = slot_take<uint32_t>(base, off, n);
    v.leaf_start = slot_take<uint32_t>(base, off, n + 1);
    v.levels = slot_take<uint32_t>(base, off, n);
    v.P = slot_take<uint32_t>(base, off, n + 1);
    v.leaf_pre = slot_take<uint32_t>(base, off, n);
    v.sp = slot_take<float4>(base, off, n);
    v.bt.first = slot_take<uint32_t>(base, off, n);
    v.bt.last = slot_take<uint32_t>(base, off, n);
    v.bt.left = slot_take<uint32_t>(base, off, n);
    v.bt.right = slot_take<uint32_t>(base, off, n);
    v.bt.delta = slot_take<int32_t>(base, off, n);
    v.bt.int_parent = slot_take<int32_t>(base, off, n);
    v.bt.leaf_parent = slot_take<int32_t>(base, off, n);
    v.bt.visit = slot_take<uint32_t>(base, off, n);
    v.bt.cell_of = nullptr;
    v.bt.rec = nullptr;
    v.bt.levels = nullptr;
    v.bt.cell_flag = nullptr;
    v.bt.marks = nullptr;
    v.pre = slot_take<BodyDD>(base, off, n + 1);
    v.cell_flag = slot_take<uint8_t>(base, off, n);
    v.cells = cells_view(slot_take<float4>(base, off, cells_float4s(2 * nmax, D)), 2 * nmax, D);
    v.rep = slot_take<float>(base, off, n * D);
    v.U = slot_take<float>(base, off, n * D);
    v.att = slot_take<float>(base, off, n * D);
    return slot_align(off);
}

// ------------------------------------------------------- block primitives --

// Exclusive scan of in[0..n) into out (block-wide, in order); returns the total.
template <int BT>
__device__ uint32_t block_scan_excl(const uint32_t *in, uint32_t *out, uint32_t n, uint32_t *s_warp) {
    const int t = threadIdx.x, lane = t % GR_WARP, w = t / GR_WARP;
    constexpr int W = BT / GR_WARP;
    uint32_t carry = 0;
    for (uint32_t base = 0; base < n; base += BT) {
        const uint32_t i = base + t;
        const uint32_t x = i < n ? in[i] : 0u;
        uint32_t s = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(GR_FULL, s, o);
            if (lane >= o) s += y;
        }
        if (lane == 31) s_warp[w] = s;
        __syncthreads();
        uint32_t wb = 0, tot = 0;
#pragma unroll
        for (int k = 0; k < W; k++) {
            const uint32_t z = s_warp[k];
            if (k < w) wb += z;
            tot += z;
        }
        if (i < n) out[i] = carry + wb + s - x;
        carry += tot;
        __syncthreads();
    }
    return carry;
}

// The double-double prefix of the sorted points' FP64 terms (m, m x per axis) at
// every leaf start: pre[e] for leaf e (flag[p] marks the first point of leaf
// excl[p]) and pre[nu] the total. Chunks of BT points, each an FP64 block scan
// in a fixed shape (warp scans, then the warp totals in warp order), carried
// across chunks in double-double: a cell's sums as the difference of two
// prefixes are as exact as a direct FP64 sum over its points.
template <int D, int BT>
__device__ void block_leaf_prefix(const float4 *sp, const uint32_t *flag, const uint32_t *excl, uint32_t n,
                                  uint32_t nu, BodyDD *pre, Body *s_bw, BodyDD *s_carry) {
    constexpr int W = BT / GR_WARP;
    const int t = threadIdx.x, lane = t % GR_WARP, w = t / GR_WARP;
    if (t == 0) *s_carry = BodyDD{};
    __syncthreads();
    for (uint32_t base = 0; base < n; base += BT) {
        const uint32_t p = base + t;
        const Body x = p < n ? point_body<D>(sp[p]) : Body{0.0, 0.0, 0.0, 0.0};
        Body inc = x;
#pragma unroll
        for (int o = 1; o < GR_WARP; o <<= 1) {
            const Body u{shfl_up_d(inc.m, o), shfl_up_d(inc.c0, o), shfl_up_d(inc.c1, o),
                         D == 3 ? shfl_up_d(inc.c2, o) : 0.0};
            if (lane >= o) inc = body_sum<D>(u, inc);
        }
        Body lanes_before{shfl_up_d(inc.m, 1), shfl_up_d(inc.c0, 1), shfl_up_d(inc.c1, 1),
                          D == 3 ? shfl_up_d(inc.c2, 1) : 0.0};
        if (lane == 0) lanes_before = Body{0.0, 0.0, 0.0, 0.0};
        if (lane == GR_WARP - 1) s_bw[w] = inc;
        __syncthreads();
        Body before{0.0, 0.0, 0.0, 0.0}, tot{0.0, 0.0, 0.0, 0.0};
        for (int k = 0; k < W; k++) {
            if (k < w) before = body_sum<D>(before, s_bw[k]);
            tot = body_sum<D>(tot, s_bw[k]);
        }
        if (p < n && flag[p]) pre[excl[p]] = bdd_add_body<D>(*s_carry, body_sum<D>(before, lanes_before));
        __syncthreads();
        if (t == 0) *s_carry = bdd_add_body<D>(*s_carry, tot);
        __syncthreads();
    }
    if (t == 0) pre[nu] = *s_carry;
    __syncthreads();
}

// Stable LSD radix sort of keys[0..n) with vals by the 8-bit digits
// first_digit .. first_digit + passes - 1 (passes even, so the result lands back
// in place; kalt/valt are the ping-pong partners). Warp w owns a contiguous chunk
// and ranks it in order with ballots/popc, so equal digits keep their input order.
template <int BT>
__device__ void block_sort(uint64_t *keys, uint32_t *vals, uint64_t *kalt, uint32_t *valt, uint32_t n,
                           uint32_t (*s_cnt)[256], uint32_t *s_tot, int first_digit = 0, int passes = 8) {
    const int t = threadIdx.x, lane = t % GR_WARP, w = t / GR_WARP;
    constexpr int W = BT / GR_WARP;
    const uint32_t chunk = ((n + W - 1) / W + 31) & ~31u;
    const uint32_t c0 = min(n, (uint32_t)w * chunk), c1 = min(n, c0 + chunk);
    const uint32_t lt = (1u << lane) - 1u;
    uint64_t *ka = keys, *kb = kalt;
    uint32_t *va = vals, *vb = valt;
    for (int pass = 0; pass < passes; pass++) {
        const int shift = 8 * (first_digit + pass);
        for (int d = lane; d < 256; d += GR_WARP) s_cnt[w][d] = 0;
        __syncwarp();
        for (uint32_t b = c0; b < c1; b += GR_WARP) {
            const uint32_t i = b + lane;
            const bool ok = i < c1;
            const uint32_t dgt = ok ? (uint32_t)(ka[i] >> shift) & 0xffu : 256u + lane;
            const uint32_t peers = warp_digit_peers(dgt, ok);
            if (ok && (peers & lt) == 0) s_cnt[w][dgt] += __popc(peers);
            __syncwarp();
        }
        __syncthreads();
        // per digit: total over warps, exclusive scan over digits, then warp offsets
        if (t < 256) {
            uint32_t tot = 0;
#pragma unroll
            for (int k = 0; k < W; k++) tot += s_cnt[k][t];
            s_tot[t] = tot;
        }
        __syncthreads();
        if (t < 32) {  // one warp scans the 256 totals: 8 per lane
            uint32_t v[8], sum = 0;
#pragma unroll
            for (int r = 0; r < 8; r++) {
                v[r] = s_tot[lane * 8 + r];
                sum += v[r];
            }
            uint32_t s = sum;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t y = __shfl_up_sync(GR_FULL, s, o);
                if (lane >= o) s += y;
            }
            uint32_t run = s - sum;
#pragma unroll
            for (int r = 0; r < 8; r++) {
                s_tot[lane * 8 + r] = run;
                run += v[r];
            }
        }
        __syncthreads();
        if (t < 256) {
            uint32_t run = s_tot[t];
#pragma unroll
            for (int k = 0; k < W; k++) {
                const uint32_t x = s_cnt[k][t];
                s_cnt[k][t] = run;
                run += x;
            }
        }
        __syncthreads();
        for (uint32_t b = c0; b < c1; b += GR_WARP) {
            const uint32_t i = b + lane;
            const bool ok = i < c1;
            const uint64_t key = ok ? ka[i] : 0ull;
            const uint32_t dgt = ok ? (uint32_t)(key >> shift) & 0xffu : 256u + lane;
            const uint32_t peers = warp_digit_peers(dgt, ok);
            const uint32_t base = ok ? s_cnt[w][dgt] : 0u;
            __syncwarp();
            if (ok) {
                const uint32_t pos = base + __popc(peers & lt);
                kb[pos] = key;
                vb[pos] = va[i];
                if ((peers & lt) == 0) s_cnt[w][dgt] = base + __popc(peers);
            }
            __syncwarp();
        }
        __syncthreads();
        uint64_t *tk = ka;
        ka = kb;
        kb = tk;
        uint32_t *tv = va;
        va = vb;
        vb = tv;
    }
}

// The same order as an 8-pass block_sort of the full keys, in fewer passes: a
// stable sort on the keys' top `top` digits (2 or 4 passes), then every run of
// equal sorted bits in full-key order, by one thread's in-place stable
// insertion sort (runs of up to 64) or, one after another, by the whole block's
// sort of the run's other digits (longer runs; their starts and lengths kept in
// runs[], at most n / 65 pairs). The one-graph engine's tick sort, at block
// level. block_sort_top(n) picks the passes: the top 16 bits up to 2^14 keys
// (runs stay short while n / 2^16 <= 1/4), else the high 32.
__host__ __device__ inline int block_sort_top(uint32_t n) { return n <= (1u << 14) ? 2 : 4; }

template <int BT>
__device__ void block_sort_keys(uint64_t *keys, uint32_t *vals, uint64_t *kalt, uint32_t *valt, uint32_t n,
                                uint32_t (*s_cnt)[256], uint32_t *s_tot, uint32_t *runs, uint32_t *s_nlong,
                                int top = 4) {
    const int shift = 64 - 8 * top;  // the sorted bits: key >> shift
    block_sort<BT>(keys, vals, kalt, valt, n, s_cnt, s_tot, 8 - top, top);
    if (threadIdx.x == 0) *s_nlong = 0;
    __syncthreads();
    for (uint32_t p = threadIdx.x; p < n; p += BT) {
        const uint64_t hi = keys[p] >> shift;
        if (p > 0 && (keys[p - 1] >> shift) == hi) continue;        // not the start of a run
        if (p + 1 >= n || (keys[p + 1] >> shift) != hi) continue;  // a run of one
        uint32_t r = 2;
        while (p + r < n && (keys[p + r] >> shift) == hi) r++;
        if (r <= 64) {
            for (uint32_t a = p + 1; a < p + r; a++) {
                const uint64_t k = keys[a];
                const uint32_t v = vals[a];
                uint32_t b = a;
                for (; b > p && keys[b - 1] > k; b--) {
                    keys[b] = keys[b - 1];
                    vals[b] = vals[b - 1];
                }
                keys[b] = k;
                vals[b] = v;
            }
        } else {
            const uint32_t q = atomicAdd(s_nlong, 1u);
            runs[2 * q] = p;
            runs[2 * q + 1] = r;
        }
    }
    __syncthreads();
    const uint32_t nlong = *s_nlong;
    for (uint32_t q = 0; q < nlong; q++) {
        const uint32_t p = runs[2 * q], r = runs[2 * q + 1];
        block_sort<BT>(keys + p, vals + p, kalt + p, valt + p, r, s_cnt, s_tot, 0, 8 - top);
    }
}

template <int BT>
__device__ __forceinline__ double block_sum_all(double v, double *s_red) {
    double r = block_sum_d<BT>(v, s_red);
    if (threadIdx.x == 0) s_red[32] = r;
    __syncthreads();
    r = s_red[32];
    __syncthreads();
    return r;
}

// ------------------------------------------------------------ the kernel --

struct BatchArgs {
    const BatchGraph *graphs;
    BatchState *state;
    const uint32_t *order;  // queue: graph ids, largest first
    uint32_t ngraphs;
    uint32_t *next;         // queue head
    float4 *pos;
    const uint32_t *rp, *col;
    const float *wt;
    const uint32_t *heavy;  // heavy rows (global ids), ascending
    unsigned char *slots;
    size_t slot_bytes;
    uint32_t nmax;
    uint32_t ticks;
};

// Resident CTAs per SM the register budget is set for (64 registers a thread at
// 4 x 256 and 1 x 1024): three of 512 threads (40 registers, a few spilled)
// measured 5-6% faster on the mixed batch than two at 64 registers; six of 256
// threads measured slower than four.
template <int BT>
struct BatchOcc {
    static constexpr int MIN_BLOCKS = BT == 512 ? 3 : BT == 256 ? 4 : 1;
};

template <int D, int BT>
__global__ void __launch_bounds__(BT, BatchOcc<BT>::MIN_BLOCKS) k_batch(BatchArgs A) {
    constexpr int W = BT / GR_WARP;
    __shared__ uint32_t s_cnt[W][256];
    __shared__ uint32_t s_tot[256];
    __shared__ uint32_t s_warp[32];
    __shared__ double s_red[33];
    __shared__ float s_fmin[D][W], s_fmax[D][W];
    __shared__ uint32_t s_graph;
    __shared__ double s_root0[3], s_root_w, s_mean[3];
    __shared__ BatchState s_st;
    __shared__ Body s_bw[32];
    __shared__ BodyDD s_carry;
    __shared__ uint32_t s_nlong;

    const int t = threadIdx.x, lane = t % GR_WARP, w = t / GR_WARP;
    SlotView S;
    slot_carve(A.slots + (size_t)blockIdx.x * A.slot_bytes, A.nmax, D, S);

    for (;;) {
        if (t == 0) {
            const uint32_t q = atomicAdd(A.next, 1u);
            s_graph = q < A.ngraphs ? A.order[q] : 0xffffffffu;
        }
        __syncthreads();
        const uint32_t g = s_graph;
        if (g == 0xffffffffu) return;
        const BatchGraph G = A.graphs[g];
        const uint32_t n = G.n;
        float4 *pos = A.pos + G.off;
        if (t == 0) s_st = A.state[g];
        __syncthreads();
        ForceParams FP;
        FP.n = n;
        FP.gravity = G.gravity;
        FP.lin_log = G.lin_log;
        FP.strong_gravity = G.strong_gravity;
        FP.dissuade_hubs = G.dissuade_hubs;
        FP.jitter_tolerance = G.jitter_tolerance;

        for (uint32_t tick = 0; tick < A.ticks && n > 0; tick++) {
            if (s_st.converged) break;
            // ---- extent, FP64 sums, root square, mean
            {
                float lo[D], hi[D];
                double sum[D];
#pragma unroll
                for (int a = 0; a < D; a++) {
                    lo[a] = INFINITY;
                    hi[a] = -INFINITY;
                    sum[a] = 0.0;
                }
                bool bad = false;
                for (uint32_t i = t; i < n; i += BT) {
                    const float4 p = pos[i];
                    const float c[3] = {p.x, p.y, p.z};
#pragma unroll
                    for (int a = 0; a < D; a++) {
                        if (!isfinite(c[a])) bad = true;
                        lo[a] = fminf(lo[a], c[a]);
                        hi[a] = fmaxf(hi[a], c[a]);
                        sum[a] += (double)c[a];
                    }
                }
                bad = __syncthreads_or(bad);
#pragma unroll
                for (int a = 0; a < D; a++) {
                    float l = lo[a], h = hi[a];
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) {
                        l = fminf(l, __shfl_xor_sync(GR_FULL, l, o));
                        h = fmaxf(h, __shfl_xor_sync(GR_FULL, h, o));
                    }
                    if (lane == 0) {
                        s_fmin[a][w] = l;
                        s_fmax[a][w] = h;
                    }
                }
                double tot[D];
#pragma unroll
                for (int a = 0; a < D; a++) tot[a] = block_sum_d<BT>(sum[a], s_red);
                if (t == 0) {
                    double mn[D], mx[D];
                    for (int a = 0; a < D; a++) {
                        mn[a] = INFINITY;
                        mx[a] = -INFINITY;
                        for (int k = 0; k < W; k++) {
                            mn[a] = fmin(mn[a], (double)s_fmin[a][k]);
                            mx[a] = fmax(mx[a], (double)s_fmax[a][k]);
                        }
                        s_mean[a] = tot[a] / (double)n;
                    }
                    bool ok = true;
                    s_root_w = root_square<D>(mn, mx, s_root0, ok);
                    if (!ok) s_st.error |= ERR_BOUNDS;
                    if (bad) s_st.error |= ERR_NONFINITE;
                    if (s_st.error) s_st.converged = 1;
                }
                __syncthreads();
                if (s_st.converged) break;
            }
            // ---- keys and sort
            for (uint32_t i = t; i < n; i += BT) {
                S.keys[i] = morton_key<D>(pos[i], s_root0, s_root_w);
                S.vals[i] = i;
            }
            __syncthreads();
            block_sort_keys<BT>(S.keys, S.vals, S.kalt, S.valt, n, s_cnt, s_tot, S.flag, &s_nlong,
                                block_sort_top(n));
            // ---- sorted nodes, unique keys
            for (uint32_t p = t; p < n; p += BT) {
                const uint32_t i = S.vals[p];
                S.sp[p] = pos[i];
                S.sorig[p] = i;
                S.flag[p] = (p == 0 || S.keys[p] != S.keys[p - 1]) ? 1u : 0u;
            }
            __syncthreads();
            const uint32_t nu = block_scan_excl<BT>(S.flag, S.excl, n, s_warp);
            for (uint32_t p = t; p < n; p += BT) {
                const uint32_t e = S.excl[p], f = S.flag[p];
                S.uid[p] = e + f - 1;
                if (f) {
                    S.leaf_start[e] = p;
                    S.ukey[e] = S.keys[p];
                    S.levels[e] = 0;
                }
                if (p == n - 1) S.leaf_start[e + f] = n;
            }
            __syncthreads();
            // ---- tree: the one-graph engine's construction at block level. The
            //      point-term prefix at every leaf start; Karras nodes, each marking
            //      the cells among its children (bit `level` at the cell's first
            //      leaf); leaf s starts 1 + popc(levels[s]) cells, so an exclusive
            //      scan gives every leaf's first cell; then every cell at once: a
            //      leaf's body from its points, an internal cell's as the
            //      difference of two prefixes.
            block_leaf_prefix<D, BT>(S.sp, S.flag, S.excl, n, nu, S.pre, s_bw, &s_carry);
            if (t == 0 && nu == 1) S.bt.leaf_parent[0] = -1;
            for (uint32_t i = t; i + 1 < nu; i += BT) {
                const KarrasNode q = karras_node((int32_t)i, (int32_t)nu, S.ukey, S.bt);
                mark_cells<D>(true, (int32_t)i, (int32_t)nu, S.ukey, q, S.levels, S.cell_flag, nullptr, 1u);
            }
            __syncthreads();
            for (uint32_t s = t; s < nu; s += BT) S.excl[s] = 1u + (uint32_t)__popc(S.levels[s]);
            __syncthreads();
            const uint32_t ncells = block_scan_excl<BT>(S.excl, S.P, nu, s_warp);
            {
                constexpr int L = Levels<D>::L;
                for (uint32_t s = t; s < nu; s += BT) {  // leaf cells
                    const uint32_t idx = S.P[s] + (uint32_t)__popc(S.levels[s]);
                    const uint32_t a0 = S.leaf_start[s], a1 = S.leaf_start[s + 1];
                    if (idx >= ncells || a1 <= a0) {
                        atomicOr(&s_st.error, (uint32_t)ERR_TREE);
                        continue;
                    }
                    const float4 one = S.sp[a0];
                    bool coinc;
                    const Body body = leaf_sum<D>(S.sp, a0, a1, coinc);
                    const int level = nu == 1 ? 0 : coinc ? S.bt.delta[S.bt.leaf_parent[s]] / D + 1 : L;
                    write_cell<D>(S.cells, idx, body, level, s_root_w, -(int32_t)(a1 - a0), a0,
                                  a1 - a0 == 1 ? &one : nullptr);
                    S.leaf_pre[s] = idx;
                }
                for (uint32_t i = t; i + 1 < nu; i += BT) {  // internal cells
                    if (!S.cell_flag[i]) continue;
                    const int lv = S.bt.delta[i] / D;
                    const uint32_t f = S.bt.first[i], end = S.bt.last[i] + 1;
                    const uint32_t idx = S.P[f] + (uint32_t)__popc(S.levels[f] & ((1u << lv) - 1u));
                    const uint32_t skip = end == nu ? ncells : S.P[end];
                    if (idx >= ncells || skip <= idx || skip > ncells) {
                        atomicOr(&s_st.error, (uint32_t)ERR_TREE);
                        continue;
                    }
                    write_cell<D>(S.cells, idx, range_body(S.pre[f], S.pre[end]), lv, s_root_w, (int32_t)skip,
                                  S.leaf_start[f]);
                }
            }
            __syncthreads();
            // ---- repulsion walk: warp w takes groups of 32 sorted nodes, one per lane
            //      (walk_lane: the same forces, bit for bit, as the warp-union walk)
            {
                WalkView V{S.cells, S.sp, S.sorig, S.uid, S.leaf_pre, n, ncells, s_st.iter_no, G.seed, G.kr, G.th2,
                           &s_st.error};
                uint32_t far_acc = 0, pair_acc = 0;
                for (uint32_t base = (uint32_t)w * GR_WARP; base < n; base += BT) {
                    float f0, f1, f2;
                    uint32_t nf, np_;
                    walk_lane<D>(V, base + lane, f0, f1, f2, nf, np_);
                    const uint32_t p = base + lane;
                    if (p < n) {
                        const uint32_t oi = S.sorig[p];
                        S.rep[(size_t)oi * D] = f0;
                        S.rep[(size_t)oi * D + 1] = f1;
                        if (D == 3) S.rep[(size_t)oi * D + 2] = f2;
                    }
                    far_acc += nf;
                    pair_acc += np_;
                }
                far_acc = __reduce_add_sync(GR_FULL, far_acc);
                pair_acc = __reduce_add_sync(GR_FULL, pair_acc);
                if (lane == 0 && (far_acc | pair_acc)) {
                    atomicAdd(&s_st.far_count, (unsigned long long)far_acc);
                    atomicAdd(&s_st.pair_count, (unsigned long long)pair_acc);
                }
            }
            // ---- heavy rows: one warp per row, fixed butterfly
            for (uint32_t h = G.heavy0 + w; h < G.heavy1; h += W) {
                const uint32_t row = A.heavy[h];
                const float4 p = A.pos[row];
                float a0 = 0.f, a1 = 0.f, a2 = 0.f;
                for (uint32_t e = A.rp[row] + lane; e < A.rp[row + 1]; e += GR_WARP)
                    attr_term<D>(p, A.pos[A.col[e]], A.wt[e], G.lin_log, a0, a1, a2);
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    a0 += __shfl_xor_sync(GR_FULL, a0, o);
                    a1 += __shfl_xor_sync(GR_FULL, a1, o);
                    if (D == 3) a2 += __shfl_xor_sync(GR_FULL, a2, o);
                }
                if (lane == 0) {
                    const uint32_t li = row - G.off;
                    S.att[(size_t)li * D] = a0;
                    S.att[(size_t)li * D + 1] = a1;
                    if (D == 3) S.att[(size_t)li * D + 2] = a2;
                }
            }
            __syncthreads();
            // ---- forces, FP64 swing / traction, speed
            {
                double sw_acc = 0.0, tr_acc = 0.0;
                for (uint32_t i = t; i < n; i += BT) {
                    const uint32_t gi = G.off + i;
                    const float4 p = A.pos[gi];
                    float a0 = 0.f, a1 = 0.f, a2 = 0.f;
                    const uint32_t e0 = A.rp[gi], e1 = A.rp[gi + 1];
                    if (e1 - e0 <= LIGHT_MAX) {
                        for (uint32_t e = e0; e < e1; e++) attr_term<D>(p, A.pos[A.col[e]], A.wt[e], G.lin_log, a0, a1, a2);
                    } else {
                        a0 = S.att[(size_t)i * D];
                        a1 = S.att[(size_t)i * D + 1];
                        if (D == 3) a2 = S.att[(size_t)i * D + 2];
                    }
                    double sw, tr;
                    node_force<D>(FP, p, a0, a1, a2, S.rep[(size_t)i * D], S.rep[(size_t)i * D + 1],
                                  D == 3 ? S.rep[(size_t)i * D + 2] : 0.f, s_mean, S.U + (size_t)i * D, sw, tr);
                    sw_acc += sw;
                    tr_acc += tr;
                }
                const double swt = block_sum_d<BT>(sw_acc, s_red);
                const double trt = block_sum_d<BT>(tr_acc, s_red);
                if (t == 0) {
                    DevState tmp;
                    tmp.swing = s_st.swing + swt;
                    tmp.traction = s_st.traction + trt;
                    tmp.speed = s_st.speed;
                    tmp.speed_efficiency = s_st.speed_efficiency;
                    estimate_factor(&tmp, (double)n, G.jitter_tolerance);
                    s_st.swing = tmp.swing;
                    s_st.traction = tmp.traction;
                    s_st.speed = tmp.speed;
                    s_st.speed_efficiency = tmp.speed_efficiency;
                }
                __syncthreads();
            }
            // ---- update
            {
                const double speed = s_st.speed;
                double step = 0.0;
                bool bad = false;
                for (uint32_t i = t; i < n; i += BT) {
                    float4 p = pos[i];
                    bool b = false;
                    step += node_update<D>(p, S.U + (size_t)i * D, speed, b);
                    bad = bad || b;
                    pos[i] = p;
                }
                bad = __syncthreads_or(bad);
                const double moved = block_sum_d<BT>(step, s_red);
                if (t == 0) {
                    s_st.moved = moved;
                    s_st.iter_no += 1;
                    if (bad) s_st.error |= ERR_NONFINITE;
                    if (moved < 1e-10 || s_st.error) s_st.converged = 1;
                }
                __syncthreads();
            }
        }
        if (t == 0) A.state[g] = s_st;
        __syncthreads();
    }
}

}  // namespace gr
