// ForceAtlas2 / Barnes-Hut engine for one graph on one B200, and its C ABI.
//
// One tick (crates/graph-core/src/layout/forceatlas2/state.rs:130-148):
//   bounds+mean -> Morton keys -> radix sort -> sorted nodes + unique keys ->
//   Karras tree -> FP64 cell sums -> cell preorder -> warp-cooperative walk
//   (repulsion) -> attraction + gravity + FP64 swing/traction + speed ->
//   update + FP64 step sum.
// Every launch is sized from n alone and reads the per-tick counts (leaves,
// cells, convergence) from device memory, so one tick is captured once into a
// CUDA graph and replayed.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "../../include/graph_cuda.h"
#include "common.cuh"
#include "forces.cuh"
#include "radix_sort.cuh"
#include "scan.cuh"
#include "simple_graph.cuh"
#include "tree.cuh"
#include "walk.cuh"
#include "batch.cuh"
#include "adjoint.cuh"
#include "stress.cuh"
#include "d3force.cuh"
#include "pm.cuh"

using namespace gr;

// ------------------------------------------------------------- errors ------

static thread_local int g_err = 0;
static thread_local int g_err_index = -1;
static thread_local char g_msg[256] = "";

static int set_err(int code, const char *msg, int index = -1) {
    g_err = code;
    g_err_index = index;
    snprintf(g_msg, sizeof g_msg, "%s", msg ? msg : "");
    return code;
}
static int ok() { return set_err(GR_OK, ""); }

#define CU(call)                                                                  \
    do {                                                                          \
        cudaError_t e_ = (call);                                                  \
        if (e_ != cudaSuccess) {                                                  \
            char b_[200];                                                         \
            snprintf(b_, sizeof b_, "%s: %s", #call, cudaGetErrorString(e_));     \
            return set_err(e_ == cudaErrorMemoryAllocation ? GR_ALLOC_FAILED      \
                                                           : GR_CUDA_ERROR, b_); \
        }                                                                         \
    } while (0)

// ------------------------------------------------------------- params ------

struct Spec {
    const char *name;
    int kind;
    double min, max, def, step;
    const char *doc;
};

// The first five are graph-core's Fa2Params schema (registry/tunable.rs:229-240);
// the rest are the options the engine adds, appended.
static const Spec kSpecs[] = {
    {"max_iter", GR_KIND_INT, 1.0, 10000.0, 100.0, 1.0, "iteration ceiling (networkx default 100)"},
    {"jitter_tolerance", GR_KIND_FLOAT, 0.0, 1e6, 1.0, 0.1, "jitter tolerance (networkx default 1.0)"},
    {"scaling_ratio", GR_KIND_FLOAT, 0.0, 1e6, 2.0, 0.1, "repulsion scale (networkx default 2.0)"},
    {"gravity", GR_KIND_FLOAT, 0.0, 1e6, 1.0, 0.1, "gravitational pull to the centroid (networkx default 1.0)"},
    {"seed", GR_KIND_INT, 0.0, 4294967295.0, 0.0, 1.0, "seeds the initial positions and the coincidence jiggle"},
    {"dim", GR_KIND_INT, 2.0, 3.0, 2.0, 1.0, "coordinates per node: 2, or 3 (octree)"},
    {"theta", GR_KIND_FLOAT, 0.0, 10.0, 0.8, 0.1, "Barnes-Hut opening angle; 0 sums every pair exactly"},
    {"lin_log", GR_KIND_BOOL, 0.0, 1.0, 0.0, 1.0, "logarithmic attraction (networkx linlog)"},
    {"strong_gravity", GR_KIND_BOOL, 0.0, 1.0, 0.0, 1.0, "gravity proportional to distance (networkx strong_gravity)"},
    {"dissuade_hubs", GR_KIND_BOOL, 0.0, 1.0, 0.0, 1.0, "attraction divided by mass (networkx distributed_action)"},
    {"edge_weight_influence", GR_KIND_FLOAT, 0.0, 10.0, 0.0, 0.1, "attraction weight = edge weight ^ influence; 0 = unit weights"},
};
static const uint32_t kNParams = sizeof(kSpecs) / sizeof(kSpecs[0]);
static const uint32_t kRefParams = 5;

enum { P_MAX_ITER, P_JT, P_SCALING, P_GRAVITY, P_SEED, P_DIM, P_THETA, P_LINLOG, P_STRONG, P_DISSUADE, P_INFLUENCE };

static int params_values(const uint8_t *bytes, size_t len, double *out) {
    for (uint32_t i = 0; i < kNParams; i++) out[i] = kSpecs[i].def;
    if (len == 0) return ok();
    if (!bytes || (len != (size_t)kNParams * 8 && len != (size_t)kRefParams * 8))
        return set_err(GR_PARAMS_MALFORMED, "params buffer is not 5 or 11 little-endian f64 values");
    uint32_t cnt = (uint32_t)(len / 8);
    for (uint32_t i = 0; i < cnt; i++) {
        double v;
        memcpy(&v, bytes + 8 * i, 8);
        const Spec &s = kSpecs[i];
        bool good = std::isfinite(v) && v >= s.min && v <= s.max;
        if (good && s.kind == GR_KIND_INT) good = std::floor(v) == v;
        if (good && s.kind == GR_KIND_BOOL) good = (v == 0.0 || v == 1.0);
        if (!good) {
            char b[160];
            snprintf(b, sizeof b, "parameter %s is out of range (refused, never clamped)", s.name);
            return set_err(GR_PARAM_OUT_OF_RANGE, b, (int)i);
        }
        out[i] = v;
    }
    return ok();
}

// ------------------------------------------------------------- engine ------

struct Adjoint;
static void adjoint_release(Adjoint *a);

struct gr_fa2 {
    int dim = 2;
    uint32_t n = 0;
    uint64_t m = 0;
    double prm[16];
    cudaStream_t stream = nullptr;
    bool own_stream = false;

    // graph
    uint32_t *rp = nullptr, *col = nullptr;
    float *wt = nullptr;
    uint32_t *csr_simple = nullptr;    // CSR entry -> simple edge
    uint32_t *simple_raw = nullptr;    // simple edge -> surviving raw edge
    float *simple_dcdw = nullptr;      // simple edge -> d(coefficient)/d(raw weight)
    uint64_t m_raw = 0;
    struct Adjoint *adj = nullptr;     // recorded run for the backward pass
    uint32_t nseg = 0;                 // heavy-row segments
    uint32_t *seg_row = nullptr;       // segment -> row
    uint32_t *seg_first = nullptr;     // row -> its first segment (heavy rows)
    float *seg_out = nullptr;          // segment sums, D per segment
    float4 *pos = nullptr;

    // per-tick buffers
    uint64_t *keys = nullptr, *ukey = nullptr;
    bool fast_sort = false;        // the tick sorts the keys' top digits and fixes the runs (keys_sort_fast)
    int sort_passes = 4;           // one-sweep passes of the tick's key sort (sort_passes_for)
    uint32_t *vals = nullptr, *sorig = nullptr, *uid = nullptr;
    uint32_t *leaf_start = nullptr, *levels = nullptr, *P = nullptr, *leaf_pre = nullptr;
    uint8_t *cell_flag = nullptr;  // internal node -> 1 when it is a cell
    float4 *sp = nullptr;
    BinTree bt{};
    Body *leaf_body = nullptr, *int_body = nullptr;
    double *pre_local = nullptr;         // (n + 1) x (D + 1): the in-tile part of every leaf's prefix
    Body *tile_sum = nullptr;            // per tile of AG_TILE sorted points: FP64 term sums
    BodyDD *tile_carry = nullptr;        // and their exclusive double-double prefix
    uint32_t *tile_cnt = nullptr;        // leaves starting in each tile, then (large graphs) their exclusive prefix
    uint8_t *leaf_coinc = nullptr;
    Cells cells{};
    float *rep = nullptr, *U = nullptr;
    double *part = nullptr;
    double *bpart = nullptr;  // the update's per-block bounds records (the next tick's bounds)
    DevState *st = nullptr;
    RadixSorter sorter;
    Scanner scanner;

    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint32_t graph_kernels = 0;
    int walk_schedule = 1;  // 0: warp-cooperative union walk, 1: per-lane walk, 2: two nodes per lane (create: 2 in 3D)
    bool count_interactions = true;  // the walk adds its far / pair interaction counts to the state
    // tick kernels launched as programmatic dependents of the kernel before them
    // (each waits in gr_pdl_enter); off when the environment sets GR_PDL=0, or
    // after a capture with them failed
    bool pdl = true;
    bool pdl_fell_back = false;  // a capture with programmatic launches failed
    // the same tick with event records at its phase boundaries (tick start,
    // tree built, walk done, tick end), for per-phase timing
    cudaGraph_t tgraph = nullptr;
    cudaGraphExec_t texec = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    bool timing_events = false;  // set while the timed graph is captured
    // the attraction branch of a captured tick: it forks after the tree build and
    // joins before the forces, beside the walk
    cudaStream_t aux = nullptr;
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    bool branch = false;  // set while a whole tick is captured
    // every edge weight is 1 (no weights given, or edge-weight influence 0): the
    // tick's attraction reads no weights (wt still holds them for the adjoint)
    bool unit_w = false;
    void *flush = nullptr;
    size_t flush_bytes = 0;
    uint32_t *stall_word = nullptr;  // zeroed and never written: the injected wait's flag

    std::vector<void *> allocs;

    // Device buffers come from the stream-ordered pool on the handle's stream
    // (keep_pool below keeps freed memory pooled), so creating and destroying a
    // handle costs no device-wide synchronisation per buffer.
    template <typename T>
    cudaError_t alloc(T **p, size_t count) {
        cudaError_t e = cudaMallocAsync((void **)p, (count ? count : 1) * sizeof(T), stream);
        if (e == cudaSuccess) allocs.push_back((void *)*p);
        return e;
    }
    void drop_graphs() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        if (texec) cudaGraphExecDestroy(texec);
        if (tgraph) cudaGraphDestroy(tgraph);
        texec = nullptr;
        tgraph = nullptr;
    }
    ~gr_fa2() {
        if (adj) adjoint_release(adj);
        drop_graphs();
        for (int i = 0; i < 4; i++)
            if (ev[i]) cudaEventDestroy(ev[i]);
        if (fork_ev) cudaEventDestroy(fork_ev);
        if (join_ev) cudaEventDestroy(join_ev);
        if (aux) cudaStreamDestroy(aux);
        if (flush) cudaFree(flush);
        for (void *p : allocs) cudaFreeAsync(p, stream);
        sorter.release();
        scanner.release();
        if (own_stream && stream) {
            cudaStreamSynchronize(stream);
            cudaStreamDestroy(stream);
        }
    }
    // k_bounds runs k_update's grid, so that the update can compute the same bounds
    uint32_t bnd_blocks() const { return frc_blocks(n); }
};

static cudaError_t alloc_tick_buffers(gr_fa2 *h) {
    const uint32_t n = h->n;
    const int D = h->dim;
    cudaError_t e;
#define A(p, c) if ((e = h->alloc(&(p), (c)))) return e
    A(h->keys, n);
    h->fast_sort = true;
    A(h->vals, n);
    A(h->ukey, n);
    A(h->sorig, n);
    A(h->uid, n);
    A(h->leaf_start, (size_t)n + 1);
    A(h->levels, n);
    A(h->cell_flag, n);
    A(h->P, (size_t)n + 1);
    A(h->leaf_pre, n);
    A(h->sp, n);
    A(h->bt.first, n);
    A(h->bt.last, n);
    A(h->bt.left, n);
    A(h->bt.right, n);
    A(h->bt.delta, n);
    A(h->bt.int_parent, n);
    A(h->bt.leaf_parent, n);
    A(h->bt.visit, n);
    A(h->bt.rec, n);
    A(h->leaf_body, n);
    A(h->int_body, n);
    A(h->leaf_coinc, n);
    A(h->pre_local, 4 * ((size_t)n + 1));
    A(h->tile_sum, div_up(n, AG_TILE) + 1);
    A(h->tile_carry, div_up(n, AG_TILE) + 1);
    A(h->tile_cnt, 2 * ((size_t)div_up(n, AG_TILE) + 1));
    {
        float4 *cb = nullptr;  // cells: 2n at most
        A(cb, cells_float4s(2 * n, D));
        h->cells = cells_view(cb, 2 * n, D);
    }
    A(h->rep, (size_t)n * D);
    A(h->U, (size_t)n * D);
    size_t np = std::max<size_t>((size_t)h->bnd_blocks() * 3 * D, 2 * (size_t)div_up(n, FRC_THREADS)) + 8;
    A(h->part, np);
    A(h->bpart, (size_t)frc_blocks(n) * 3 * D + 8);
#undef A
    if ((e = h->sorter.init(n, h->stream, true))) return e;
    if ((e = h->scanner.init(n, h->stream, true))) return e;
    return cudaSuccess;
}

enum Phase { PH_TREE = 1, PH_WALK = 2, PH_FINISH = 4, PH_ALL = 7 };

// After a stable sort on the key bits from `shift` up, every run of equal
// sorted bits put in full-key order in place, which makes the result identical
// to a stable sort of the whole key: a run of up to 64 keys by the thread at
// its first key (a stable insertion sort), a longer one by the whole block that
// holds its first key (a stable block radix sort of its low `low_passes`
// digits, an even count covering every digit the passes left out; scratch: the
// sorter's ping-pong pair at the run's own offsets, free after an even pass
// count). Runs are disjoint, so the result does not depend on which finishes
// first.
constexpr uint32_t FIX_T = 256, FIX_SHORT = 64;
__global__ void __launch_bounds__(FIX_T) k_fix_runs(uint64_t *__restrict__ keys, uint32_t *__restrict__ vals,
                                                    uint64_t *__restrict__ kalt, uint32_t *__restrict__ valt,
                                                    uint32_t n, int shift, int low_passes, const uint32_t *skip) {
    gr_pdl_enter();
    if (skip && *skip) return;
    __shared__ uint32_t s_cnt[FIX_T / GR_WARP][256];
    __shared__ uint32_t s_tot[256];
    __shared__ uint2 s_long[FIX_T];  // at most one run starts at each thread's key
    __shared__ uint32_t s_nlong;
    if (threadIdx.x == 0) s_nlong = 0;
    __syncthreads();
    const uint32_t i = blockIdx.x * FIX_T + threadIdx.x;
    if (i + 1 < n) {
        const uint64_t hi = keys[i] >> shift;
        // the first key of a run of two or more
        if ((keys[i + 1] >> shift) == hi && !(i > 0 && (keys[i - 1] >> shift) == hi)) {
            uint32_t len = 2;
            while (i + len < n && (keys[i + len] >> shift) == hi) len++;
            if (len > FIX_SHORT) {
                s_long[atomicAdd(&s_nlong, 1u)] = make_uint2(i, len);
            } else {
                for (uint32_t a = i + 1; a < i + len; a++) {
                    const uint64_t k = keys[a];
                    const uint32_t v = vals[a];
                    uint32_t b = a;
                    while (b > i && keys[b - 1] > k) {  // strictly greater: equal keys keep their order
                        keys[b] = keys[b - 1];
                        vals[b] = vals[b - 1];
                        b--;
                    }
                    keys[b] = k;
                    vals[b] = v;
                }
            }
        }
    }
    __syncthreads();
    const uint32_t nlong = s_nlong;
    for (uint32_t q = 0; q < nlong; q++) {
        const uint2 r = s_long[q];
        block_sort<FIX_T>(keys + r.x, vals + r.x, kalt + r.x, valt + r.x, r.y, s_cnt, s_tot, 0, low_passes);
    }
}

// Morton keys of every node (k_keys' work) fused with the one-sweep digit
// histograms of the keys' top PASSES digits (os_hist's work for digits
// 8 - PASSES .. 7) and the zeroing of those passes' look-back words. ghist
// (digit counts and tile counters) was zeroed by the bounds pass. Grid-stride
// over the nodes in order, 4 positions in flight per thread; counts are
// integers, so the histogram does not depend on the order the atomics land in.
template <int D, int PASSES>
__global__ void __launch_bounds__(OS_HIST_THREADS)
k_keys_hist(const float4 *__restrict__ pos, uint32_t n, const DevState *st, uint64_t *__restrict__ keys,
            uint32_t *__restrict__ vals, uint32_t *__restrict__ ghist, uint32_t *__restrict__ status,
            uint64_t status_words) {
    gr_pdl_enter();
    static_assert(OS_HIST_THREADS == RS_BINS, "one thread per digit");
    static_assert(PASSES >= 2 && PASSES <= 4, "the top two to four digits");
    constexpr int FIRST = 8 - PASSES, U = 4;
    if (st->converged) return;
    __shared__ uint32_t s_h[PASSES][RS_BINS];
    const int t = threadIdx.x;
#pragma unroll
    for (int p = 0; p < PASSES; p++) s_h[p][t] = 0;
    __syncthreads();
    const double r0[3] = {st->root0[0], st->root0[1], D == 3 ? st->root0[2] : 0.0};
    const double rw = st->root_w;
    const uint64_t stride = (uint64_t)gridDim.x * OS_HIST_THREADS;
    for (uint64_t i0 = (uint64_t)blockIdx.x * OS_HIST_THREADS + t; i0 < n; i0 += U * stride) {
        float4 pv[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const uint64_t i = i0 + u * stride;
            pv[u] = i < n ? pos[i] : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const uint64_t i = i0 + u * stride;
            if (i < n) {
                const uint64_t key = morton_key<D>(pv[u], r0, rw);
                keys[i] = key;
                vals[i] = (uint32_t)i;
#pragma unroll
                for (int p = 0; p < PASSES; p++) atomicAdd(&s_h[p][(uint32_t)(key >> (8 * (FIRST + p))) & 0xffu], 1u);
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int p = 0; p < PASSES; p++)
        if (s_h[p][t]) atomicAdd(&ghist[p * RS_BINS + t], s_h[p][t]);
    for (uint64_t i = (uint64_t)blockIdx.x * OS_HIST_THREADS + t; i < status_words; i += stride) status[i] = 0u;
}

// Small graphs: the keys and their whole sort in one CTA, in shared memory. A
// tick's sort otherwise takes four to six dependent kernels (keys with
// histograms, two to four one-sweep passes, the run fix-up), each a few
// microseconds of launch and drain at any size, which dominate a small graph's
// tick. Here the keys go to shared memory and block_sort_keys sorts them: two
// stable passes on the top 16 bits, then runs of equal sorted bits in full-key
// order (the batched kernel's sort), the same permutation as the stable 64-bit
// sort.
constexpr uint32_t SMALL_SORT_MAX = 3072;
constexpr int SMALL_SORT_T = 1024;
constexpr size_t SMALL_SORT_SMEM = (size_t)SMALL_SORT_MAX * (2 * sizeof(uint64_t) + 2 * sizeof(uint32_t)) +
                                   (size_t)(SMALL_SORT_T / GR_WARP) * 256 * 4 + 256 * 4 +
                                   2 * (SMALL_SORT_MAX / 65 + 1) * 4;

template <int D>
__global__ void __launch_bounds__(SMALL_SORT_T)
k_sort_small(const float4 *__restrict__ pos, uint32_t n, const DevState *st, uint64_t *__restrict__ keys_out,
             uint32_t *__restrict__ vals_out) {
    gr_pdl_enter();
    if (st->converged || n > SMALL_SORT_MAX) return;
    extern __shared__ __align__(16) unsigned char ss_sm[];
    uint64_t *k = (uint64_t *)ss_sm;
    uint64_t *ka = k + SMALL_SORT_MAX;
    uint32_t *v = (uint32_t *)(ka + SMALL_SORT_MAX);
    uint32_t *va = v + SMALL_SORT_MAX;
    uint32_t(*s_cnt)[256] = (uint32_t(*)[256])(va + SMALL_SORT_MAX);
    uint32_t *s_tot = (uint32_t *)(s_cnt + SMALL_SORT_T / GR_WARP);
    uint32_t *runs = s_tot + 256;  // (start, length) of the runs longer than 64
    __shared__ uint32_t s_nlong;
    const double r0[3] = {st->root0[0], st->root0[1], D == 3 ? st->root0[2] : 0.0};
    const double rw = st->root_w;
    for (uint32_t i = threadIdx.x; i < n; i += SMALL_SORT_T) {
        k[i] = morton_key<D>(pos[i], r0, rw);
        v[i] = i;
    }
    __syncthreads();
    block_sort_keys<SMALL_SORT_T>(k, v, ka, va, n, s_cnt, s_tot, runs, &s_nlong, block_sort_top(n));
    for (uint32_t i = threadIdx.x; i < n; i += SMALL_SORT_T) {
        keys_out[i] = k[i];
        vals_out[i] = v[i];
    }
}

// One-sweep passes of a tick's key sort for n nodes: the top 16 key bits up to
// 2^14 nodes, 24 up to 2^22, else the high 32. The fewer the passes, the more
// keys share their sorted bits and the longer the runs the fix-up puts in
// full-key order; while n / 2^(8 passes) stays at or below 1/4 (uniform points:
// a run of one in most cells; a cluster 30 times as dense: runs of about 8) a
// pass costs more than the longer runs.
static int sort_passes_for(uint32_t n) { return n <= (1u << 14) ? 2 : n <= (1u << 22) ? 3 : 4; }

// Keys, then a stable sort on the keys' top digits (h->sort_passes one-sweep
// passes), then every run of equal sorted bits put in full-key order
// (k_fix_runs). The order is exactly the full stable 64-bit sort's. With an odd
// pass count the keys are written to the sorter's scratch pair first, so the
// last pass lands in keys/vals. The bounds pass zeroed os_ghist. Up to
// SMALL_SORT_MAX nodes all of it is one kernel (k_sort_small).
template <int D>
static void keys_sort_fast(gr_fa2 *h, cudaStream_t s) {
    const uint32_t n = h->n;
    const uint32_t *conv = &h->st->converged;
    if (n <= SMALL_SORT_MAX) {
        cudaFuncSetAttribute(k_sort_small<D>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMALL_SORT_SMEM);
        gr_launch(h->pdl, k_sort_small<D>, 1, SMALL_SORT_T, SMALL_SORT_SMEM, s, h->pos, n, h->st, h->keys, h->vals);
        return;
    }
    int passes = 4;
    if (n < (1u << 30)) {
        passes = h->sort_passes;
        const uint32_t nt = div_up(n, os_tile_keys(n));
        const uint32_t hb = std::min<uint32_t>(div_up(n, OS_HIST_THREADS * 4), 4 * 148);
        const bool odd = passes & 1;
        uint64_t *k0 = odd ? h->sorter.k_alt : h->keys;
        uint32_t *v0 = odd ? h->sorter.v_alt : h->vals;
        uint32_t *gh = h->sorter.os_ghist, *ss = h->sorter.os_status;
        const uint64_t words = (uint64_t)passes * nt * RS_BINS;
        if (passes == 2)
            gr_launch(h->pdl, k_keys_hist<D, 2>, hb, OS_HIST_THREADS, 0, s, h->pos, n, h->st, k0, v0, gh, ss, words);
        else if (passes == 3)
            gr_launch(h->pdl, k_keys_hist<D, 3>, hb, OS_HIST_THREADS, 0, s, h->pos, n, h->st, k0, v0, gh, ss, words);
        else
            gr_launch(h->pdl, k_keys_hist<D, 4>, hb, OS_HIST_THREADS, 0, s, h->pos, n, h->st, k0, v0, gh, ss, words);
        h->sorter.onesweep_passes(h->keys, h->vals, n, 8 - passes, passes, s, &h->st->error, conv, h->pdl,
                                  &h->st->converged);
    } else {
        k_keys<D><<<div_up(n, 256), 256, 0, s>>>(h->pos, n, h->st, h->keys, h->vals);
        h->sorter.sort_digits(h->keys, h->vals, n, 4, 4, s, conv);
    }
    const int low = 8 - passes;  // the digits the passes left out, sorted within runs
    gr_launch(h->pdl, k_fix_runs, div_up(n, FIX_T), FIX_T, 0, s, h->keys, h->vals, h->sorter.k_alt,
              h->sorter.v_alt, n, 8 * low, low + (low & 1), conv);
}

static_assert(SC_TILE == (int)SC_TILE_LEAVES, "k_karras counts level bits per cell-level scan block");

// The repulsion walk in the handle's schedule, with or without its interaction counts.
template <int D, bool COUNT>
static void launch_walk(gr_fa2 *h, const WalkParams &wp, cudaStream_t s, bool pdl) {
    const uint32_t n = h->n;
    DevState *st = h->st;
    if (h->walk_schedule == 3)  // 64 nodes per warp: two groups of 32, one walk of each per lane
        gr_launch(pdl, k_walk_s<D, 3, COUNT>, div_up(n, 2 * WALK_THREADS), WALK_THREADS, 0, s, wp, st, h->cells,
                  h->sp, h->sorig, h->uid, h->leaf_pre, h->rep, st);
    else if (h->walk_schedule == 2)
        gr_launch(pdl, k_walk_s<D, 2, COUNT>, div_up(div_up(n, 2), WALK_THREADS), WALK_THREADS, 0, s, wp, st,
                  h->cells, h->sp, h->sorig, h->uid, h->leaf_pre, h->rep, st);
    else if (h->walk_schedule == 1)
        gr_launch(pdl, k_walk_s<D, 1, COUNT>, div_up(n, WALK_THREADS), WALK_THREADS, 0, s, wp, st, h->cells, h->sp,
                  h->sorig, h->uid, h->leaf_pre, h->rep, st);
    else
        gr_launch(pdl, k_walk_s<D, 0, COUNT>, div_up(n, WALK_THREADS), WALK_THREADS, 0, s, wp, st, h->cells, h->sp,
                  h->sorig, h->uid, h->leaf_pre, h->rep, st);
}

template <int D>
static void enqueue_tick(gr_fa2 *h, bool forces_only, int phases) {
    const uint32_t n = h->n;
    cudaStream_t s = h->stream;
    const uint32_t gn = div_up(n, 256);
    DevState *st = h->st;
    const uint32_t *conv = &st->converged;
    const int lin_log = (int)h->prm[P_LINLOG];
    // the attraction of every node into U (k_forces reads it there): the heavy
    // rows' segment sums, then every row
    auto attraction_seg = [&](cudaStream_t q) {
        if (h->nseg)
            k_attract_seg<D><<<div_up((uint64_t)h->nseg * GR_WARP, FRC_THREADS), FRC_THREADS, 0, q>>>(
                h->nseg, lin_log, st, h->pos, h->rp, h->col, h->unit_w ? nullptr : h->wt, h->seg_row,
                h->seg_first, h->seg_out);
    };
    auto attraction_rows = [&](cudaStream_t q) {
        k_attract<D><<<div_up(n, FRC_THREADS), FRC_THREADS, 0, q>>>(
            n, lin_log, st, h->pos, h->rp, h->col, h->unit_w ? nullptr : h->wt, h->nseg ? h->seg_first : nullptr,
            h->seg_out, h->U);
    };
    // In a captured whole tick the attraction runs on its own branch beside the
    // walk (which is bound by instruction issue, the attraction by memory
    // latency); beside the tree build it slowed the latency-bound tree kernels
    // by about as much as it saved.
    const bool branch = h->branch && phases == PH_ALL;
    if (h->timing_events) cudaEventRecordWithFlags(h->ev[0], s, cudaEventRecordExternal);
    if (phases & PH_TREE) {
        // counters later kernels of the tree build accumulate into: the fast
        // sort's digit counts and tile counters, the cell-level scan's marks
        ZeroWords zw;
        if (h->fast_sort) zw.add(h->sorter.os_ghist, RadixSorter::ghist_words());
        const bool fold_scan = h->scanner.folds(n);
        if (fold_scan) zw.add(h->scanner.bsum, div_up(n, SC_TILE));
        k_bounds<D><<<h->bnd_blocks(), BND_THREADS, 0, s>>>(h->pos, n, st, h->part, zw);
        const uint32_t ab = div_up(n, AG_TILE);
        if (h->fast_sort) {
            keys_sort_fast<D>(h, s);
        } else {
            k_keys<D><<<gn, 256, 0, s>>>(h->pos, n, st, h->keys, h->vals);
            h->sorter.sort(h->keys, h->vals, n, 64, s, conv);
        }
        gr_launch(h->pdl, k_leaf_tiles<D>, ab, AG_T, 0, s, st, n, h->pos, h->keys, h->vals, h->sp, h->sorig,
                  h->tile_sum, h->tile_cnt, h->uid, h->pre_local);
        const uint32_t *ccarry = nullptr;  // the carries come from one block above LEAF_FOLD_MAX_TILES tiles
        if (ab > LEAF_FOLD_MAX_TILES) {
            k_leaf_carry<D><<<1, CARRY_T, 0, s>>>(st, n, h->tile_sum, h->tile_cnt, h->tile_carry, h->tile_cnt + ab,
                                                  h->leaf_start, h->pre_local);
            ccarry = h->tile_cnt + ab;
        }
        gr_launch(h->pdl, k_leaf_prefix<D>, ab, AG_T, 0, s, st, n, h->keys, h->tile_sum, h->tile_cnt,
                  h->tile_carry, ccarry, h->uid, h->leaf_start, h->ukey, h->levels, h->pre_local);
        const Prefix pre{h->pre_local, h->tile_carry, h->leaf_start, 0u, ab};  // nu: read on the device
        const bool adjoint = h->bt.cell_of != nullptr;  // the adjoint reads leaf and node bodies as arrays
        BinTree bt = h->bt;  // the tick itself reads only the packed records and leaf_parent
        bt.levels = h->levels;
        bt.cell_flag = h->cell_flag;
        if (!adjoint) {
            bt.first = bt.last = bt.left = bt.right = bt.visit = nullptr;
            bt.delta = bt.int_parent = nullptr;
        }
        bt.marks = fold_scan ? h->scanner.bsum : nullptr;
        gr_launch(h->pdl, k_karras<D>, gn, 256, 0, s, st, h->ukey, bt);
        if (adjoint) k_leaf_body<D><<<gn, 256, 0, s>>>(st, h->sp, h->leaf_start, h->leaf_body, h->leaf_coinc);
        if (adjoint) k_node_body<D><<<gn, 256, 0, s>>>(st, h->bt, pre, h->int_body);
        if (fold_scan)
            h->scanner.scan_levels_marked(h->levels, h->P, n, &st->n_unique, &st->n_cells, s, conv, h->pdl);
        else
            h->scanner.scan_levels(h->levels, h->P, n, &st->n_unique, &st->n_cells, s, conv);
        // 128-thread blocks: measured faster than 256 and 512 (the 1M 3D tree by 3.5 us)
        const uint32_t cb = div_up(n, 128);
        gr_launch(h->pdl, k_assign_cells<D>, 2 * cb, 128, 0, s, st, bt, cb * 128, h->sp, h->P, h->levels,
                  h->leaf_start, pre, h->cells, h->leaf_pre, st);
    }
    if (h->timing_events) cudaEventRecordWithFlags(h->ev[1], s, cudaEventRecordExternal);
    if (branch) {
        cudaEventRecord(h->fork_ev, s);
        cudaStreamWaitEvent(h->aux, h->fork_ev, 0);
        attraction_seg(h->aux);
        attraction_rows(h->aux);
        cudaEventRecord(h->join_ev, h->aux);
    }
    if (phases & PH_WALK) {
        WalkParams wp;
        wp.n = n;
        wp.kr = (float)h->prm[P_SCALING];
        wp.theta2 = (float)(h->prm[P_THETA] * h->prm[P_THETA]);
        wp.seed = (uint32_t)h->prm[P_SEED];
        // in the timed graph an event record node stands before the walk: no
        // programmatic edge there
        const bool pdl = h->pdl && (phases & PH_TREE) && !h->timing_events;
        if (h->count_interactions)
            launch_walk<D, true>(h, wp, s, pdl);
        else
            launch_walk<D, false>(h, wp, s, pdl);
    }
    if (h->timing_events) cudaEventRecordWithFlags(h->ev[2], s, cudaEventRecordExternal);
    if (phases & PH_FINISH) {
        ForceParams fp;
        fp.n = n;
        fp.gravity = (float)h->prm[P_GRAVITY];
        fp.lin_log = lin_log;
        fp.strong_gravity = (int)h->prm[P_STRONG];
        fp.dissuade_hubs = (int)h->prm[P_DISSUADE];
        fp.jitter_tolerance = h->prm[P_JT];
        if (branch) {
            cudaStreamWaitEvent(s, h->join_ev, 0);
        } else {
            attraction_seg(s);
            attraction_rows(s);
        }
        k_forces<D><<<frc_blocks(n), FRC_THREADS, 0, s>>>(fp, st, h->pos, h->rep, h->U, h->part,
                                                                    forces_only ? 0 : 1);
        if (!forces_only)
            gr_launch(h->pdl, k_update<D>, frc_blocks(n), FRC_THREADS, 0, s, n, st, h->pos, h->U, h->part,
                      h->bpart);
    }
    if (h->timing_events) cudaEventRecordWithFlags(h->ev[3], s, cudaEventRecordExternal);
}

static void enqueue(gr_fa2 *h, bool forces_only, int phases = PH_ALL) {
    if (h->dim == 3)
        enqueue_tick<3>(h, forces_only, phases);
    else
        enqueue_tick<2>(h, forces_only, phases);
}

// One capture of a whole tick into *g, its node priorities set and the graph
// instantiated into *x (the error of the first step that failed).
static cudaError_t capture_once(gr_fa2 *h, bool timing, cudaGraph_t *g, cudaGraphExec_t *x) {
    cudaError_t e = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    h->branch = true;
    h->timing_events = timing;
    enqueue(h, false, PH_ALL);
    h->branch = false;
    h->timing_events = false;
    if ((e = cudaStreamEndCapture(h->stream, g)) != cudaSuccess) return e;
    // The attraction branch runs beside the walk and fills what the walk leaves
    // idle: its kernels run at the lowest priority, the tick's own path at the
    // highest, so a free SM slot goes to the walk's next block first.
    int least = 0, greatest = 0;
    if ((e = cudaDeviceGetStreamPriorityRange(&least, &greatest)) != cudaSuccess) return e;
    size_t nn = 0;
    if ((e = cudaGraphGetNodes(*g, nullptr, &nn)) != cudaSuccess) return e;
    std::vector<cudaGraphNode_t> nodes(nn);
    if ((e = cudaGraphGetNodes(*g, nodes.data(), &nn)) != cudaSuccess) return e;
    const void *side[4] = {(const void *)k_attract<2>, (const void *)k_attract<3>, (const void *)k_attract_seg<2>,
                           (const void *)k_attract_seg<3>};
    for (auto nd : nodes) {
        cudaGraphNodeType t;
        if ((e = cudaGraphNodeGetType(nd, &t)) != cudaSuccess) return e;
        if (t != cudaGraphNodeTypeKernel) continue;
        cudaKernelNodeParams kp;
        if ((e = cudaGraphKernelNodeGetParams(nd, &kp)) != cudaSuccess) return e;
        bool low = false;
        for (const void *f : side) low = low || kp.func == f;
        cudaLaunchAttributeValue v;
        memset(&v, 0, sizeof v);
        v.priority = low ? least : greatest;
        if ((e = cudaGraphKernelNodeSetAttribute(nd, cudaLaunchAttributePriority, &v)) != cudaSuccess) return e;
    }
    return cudaGraphInstantiate(x, *g, 0);
}

// Programmatic dependent launches for a new handle's ticks: on unless the
// environment sets GR_PDL=0.
static bool pdl_default() {
    const char *v = getenv("GR_PDL");
    return !(v && strcmp(v, "0") == 0);
}

// Captures one whole tick (with the attraction on its own branch), and with
// timing the event records at its phase boundaries. If the capture with
// programmatic dependent launches fails, the handle drops them and captures
// again with plain stream order.
static int capture(gr_fa2 *h, bool timing, cudaGraph_t *g, cudaGraphExec_t *x) {
    if (!h->aux) {
        CU(cudaStreamCreateWithFlags(&h->aux, cudaStreamNonBlocking));
        CU(cudaEventCreateWithFlags(&h->fork_ev, cudaEventDisableTiming));
        CU(cudaEventCreateWithFlags(&h->join_ev, cudaEventDisableTiming));
    }
    if (timing)
        for (int i = 0; i < 4; i++)
            if (!h->ev[i]) CU(cudaEventCreate(&h->ev[i]));
    for (;;) {
        *g = nullptr;
        *x = nullptr;
        cudaError_t e = capture_once(h, timing, g, x);
        if (e == cudaSuccess) return GR_OK;
        cudaGetLastError();  // a capture error is not sticky: clear it
        if (*x) cudaGraphExecDestroy(*x);
        if (*g) cudaGraphDestroy(*g);
        *g = nullptr;
        *x = nullptr;
        if (!h->pdl) return set_err(GR_CUDA_ERROR, cudaGetErrorString(e));
        h->pdl = false;
        h->pdl_fell_back = true;
    }
}

static int build_graph(gr_fa2 *h) {
    if (h->exec) return GR_OK;
    if (int c = capture(h, false, &h->graph, &h->exec)) return c;
    size_t nn = 0;
    CU(cudaGraphGetNodes(h->graph, nullptr, &nn));
    std::vector<cudaGraphNode_t> nodes(nn);
    CU(cudaGraphGetNodes(h->graph, nodes.data(), &nn));
    h->graph_kernels = 0;
    for (auto nd : nodes) {
        cudaGraphNodeType t;
        CU(cudaGraphNodeGetType(nd, &t));
        if (t == cudaGraphNodeTypeKernel) h->graph_kernels++;
    }
    return GR_OK;
}

static int build_timed_graph(gr_fa2 *h) {
    if (h->texec) return GR_OK;
    return capture(h, true, &h->tgraph, &h->texec);
}

static int read_state(gr_fa2 *h, DevState *out) {
    CU(cudaMemcpyAsync(out, h->st, sizeof(DevState), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    return GR_OK;
}

static int check_device(gr_fa2 *h, const DevState &s) {
    if (s.error & ERR_NONFINITE) return set_err(GR_LAYOUT_FAILED, "non-finite position (StageError::NonFinite)");
    if (s.error) {
        char b[96];
        snprintf(b, sizeof b, "device error bits 0x%x", s.error);
        return set_err(GR_DEVICE_FAULT, b);
    }
    return GR_OK;
}

// Heavy rows (degree > LIGHT_MAX) split into SEG-entry segments for the
// warp-per-segment attraction pass, counted, scanned and listed on the device.
static int build_segments(gr_fa2 *h) {
    const uint32_t n = h->n;
    if (n == 0 || h->m == 0) return GR_OK;
    cudaStream_t s = h->stream;
    cudaError_t e;
    uint32_t *cnt = nullptr, *total = nullptr;
    if ((e = h->alloc(&h->seg_first, n)) || (e = cudaMallocAsync((void **)&cnt, (size_t)n * 4, s)) ||
        (e = cudaMallocAsync((void **)&total, 4, s))) {
        if (cnt) cudaFreeAsync(cnt, s);
        return set_err(GR_ALLOC_FAILED, cudaGetErrorString(e));
    }
    Scanner sc;
    if ((e = sc.init(n, s, true))) {
        cudaFreeAsync(cnt, s);
        cudaFreeAsync(total, s);
        return set_err(GR_ALLOC_FAILED, cudaGetErrorString(e));
    }
    k_seg_count<<<div_up(n, 256), 256, 0, s>>>(n, h->rp, LIGHT_MAX, SEG, cnt);
    sc.scan(cnt, h->seg_first, n, nullptr, 0, total, nullptr, s);
    uint32_t nseg = 0;
    cudaMemcpyAsync(&nseg, total, 4, cudaMemcpyDeviceToHost, s);
    sc.release();
    cudaFreeAsync(cnt, s);
    cudaFreeAsync(total, s);
    CU(cudaStreamSynchronize(s));
    h->nseg = nseg;
    if (!nseg) return GR_OK;
    if ((e = h->alloc(&h->seg_row, nseg)) || (e = h->alloc(&h->seg_out, (size_t)nseg * h->dim)))
        return set_err(GR_ALLOC_FAILED, cudaGetErrorString(e));
    k_seg_fill<<<div_up(n, 256), 256, 0, s>>>(n, h->rp, LIGHT_MAX, SEG, h->seg_first, h->seg_row);
    CU(cudaGetLastError());
    return GR_OK;
}

// Once per device and process: the default stream-ordered pool keeps the memory
// it is given back instead of returning it to the device, so the next handle's
// buffers come from the pool. A process setting; nothing on the GPU outlives it.
static void keep_pool() {
    static std::mutex mu;
    static std::vector<int> done;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return;
    std::lock_guard<std::mutex> lock(mu);
    if (std::find(done.begin(), done.end(), dev) != done.end()) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    done.push_back(dev);
}

// Per-graph seeded starts of a concatenation of graphs (host arrays): graph g
// begins at node off[g] and draws from Mulberry32(seed[g]). Empty: one seed.
struct SeededStarts {
    uint32_t graphs = 0;
    const uint32_t *off = nullptr, *seed = nullptr;
};

static int create_impl(gr_fa2 **out, uint32_t n, uint64_t m, const uint32_t *src, const uint32_t *dst,
                       const double *weight, const uint8_t *params, size_t params_len, const float *pos0,
                       bool tick_buffers = true, SeededStarts starts = SeededStarts()) {
    if (!out) return set_err(GR_INVALID_ARGUMENT, "out is null");
    *out = nullptr;
    double prm[16];
    if (int c = params_values(params, params_len, prm)) return c;
    if (m && (!src || !dst)) return set_err(GR_INVALID_ARGUMENT, "edge arrays are null");
    if (m > 0x7fffffffull) return set_err(GR_INVALID_ARGUMENT, "more than 2^31 edges");
    const int D = (int)prm[P_DIM];
    // without pos0 the start is Mulberry32(seed), dim draws per node, drawn on
    // the device (k_init_nodes); a given one is checked there
    gr_fa2 *h = new (std::nothrow) gr_fa2();
    if (!h) return set_err(GR_ALLOC_FAILED, "host allocation failed");
    h->dim = D;
    h->n = n;
    // the autotuner's choice on both 1M-node graphs: per lane in 2D, two nodes per
    // lane over the union of their walks in 3D (0.43 against 0.46 ms)
    h->walk_schedule = D == 3 ? 2 : 1;
    h->sort_passes = sort_passes_for(n);
    memcpy(h->prm, prm, sizeof prm);
    int rc = GR_OK;
    do {
        if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
            rc = set_err(GR_CUDA_ERROR, "stream creation failed");
            break;
        }
        h->own_stream = true;
        h->pdl = pdl_default();
        keep_pool();
        cudaStream_t s = h->stream;
        cudaError_t e = cudaSuccess;
        // --- simple graph + CSR on the device
        uint32_t *d_src = nullptr, *d_dst = nullptr, *d_err = nullptr;
        double *d_w = nullptr;
        uint64_t *ek = nullptr, *dk = nullptr;
        uint32_t *ev = nullptr, *dv = nullptr, *eflag = nullptr, *eexcl = nullptr, *ms_d = nullptr;
        RadixSorter esort;
        Scanner escan;
        uint32_t ms = 0;
        // create's own buffers: the stream-ordered pool, freed on the stream
        auto tmp = [&](auto **p, size_t bytes) { return cudaMallocAsync((void **)p, bytes, s); };
        auto cleanup = [&]() {
            for (void *p : {(void *)d_src, (void *)d_dst, (void *)d_w, (void *)d_err, (void *)ek, (void *)ev,
                            (void *)dk, (void *)dv, (void *)eflag, (void *)eexcl, (void *)ms_d})
                if (p) cudaFreeAsync(p, s);
            esort.release();
            escan.release();
        };
        const uint64_t cap = std::max<uint64_t>(2 * m, 1);
        const EdgeKey ekf = edge_key_for(n);
        if ((e = tmp(&d_err, 2 * sizeof(uint32_t))) || (e = tmp(&ms_d, 2 * sizeof(uint32_t))) ||
            (e = tmp(&ek, cap * sizeof(uint64_t))) || (e = tmp(&ev, cap * sizeof(uint32_t))) ||
            (e = tmp(&dk, cap * sizeof(uint64_t))) || (e = tmp(&dv, cap * sizeof(uint32_t))) ||
            (e = tmp(&eflag, cap * sizeof(uint32_t))) || (e = tmp(&eexcl, cap * sizeof(uint32_t))) ||
            (e = esort.init((uint32_t)cap, s, true)) || (e = escan.init((uint32_t)cap, s, true))) {
            cleanup();
            rc = set_err(GR_ALLOC_FAILED, cudaGetErrorString(e));
            break;
        }
        cudaMemsetAsync(d_err, 0, 2 * sizeof(uint32_t), s);
        cudaMemsetAsync(ms_d, 0, 2 * sizeof(uint32_t), s);
        if (m) {
            if ((e = tmp(&d_src, m * 4)) || (e = tmp(&d_dst, m * 4)) || (weight && (e = tmp(&d_w, m * 8)))) {
                cleanup();
                rc = set_err(GR_ALLOC_FAILED, cudaGetErrorString(e));
                break;
            }
            cudaMemcpyAsync(d_src, src, m * 4, cudaMemcpyHostToDevice, s);
            cudaMemcpyAsync(d_dst, dst, m * 4, cudaMemcpyHostToDevice, s);
            if (weight) cudaMemcpyAsync(d_w, weight, m * 8, cudaMemcpyHostToDevice, s);
            k_edge_keys<<<div_up(m, 256), 256, 0, s>>>(m, d_src, d_dst, n, ekf, ek, ev, d_err);
            esort.sort_bits(ek, ev, (uint32_t)m, 2 * ekf.bits, s, d_err + 1);
            k_edge_flags<<<div_up(m, 256), 256, 0, s>>>((uint32_t)m, ekf, ek, eflag);
            escan.scan(eflag, eexcl, (uint32_t)m, nullptr, 0, ms_d, nullptr, s);
        }
        uint32_t hdr[2] = {0, 0};
        cudaMemcpyAsync(hdr, d_err, sizeof hdr, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(&ms, ms_d, 4, cudaMemcpyDeviceToHost, s);
        if ((e = cudaStreamSynchronize(s))) {
            cleanup();
            rc = set_err(GR_CUDA_ERROR, cudaGetErrorString(e));
            break;
        }
        if (hdr[0]) {
            cleanup();
            rc = set_err(GR_INVALID_ARGUMENT, "an edge names a node >= n");
            break;
        }
        if (hdr[1]) {
            cleanup();
            rc = set_err(GR_DEVICE_FAULT, "the edge sort gave up a bounded wait");
            break;
        }
        h->m = ms;
        h->unit_w = weight == nullptr || prm[P_INFLUENCE] == 0.0;
        uint32_t *slo = nullptr, *shi = nullptr;
        float *weff = nullptr;
        h->m_raw = m;
        if ((e = h->alloc(&h->rp, (size_t)n + 1)) || (e = h->alloc(&h->col, 2 * (size_t)ms)) ||
            (e = h->alloc(&h->wt, 2 * (size_t)ms)) || (e = h->alloc(&h->pos, n)) ||
            (e = h->alloc(&h->st, 1)) || (e = h->alloc(&slo, ms)) || (e = h->alloc(&shi, ms)) ||
            (e = h->alloc(&weff, ms)) || (e = h->alloc(&h->simple_raw, ms)) ||
            (e = h->alloc(&h->simple_dcdw, ms)) || (e = h->alloc(&h->csr_simple, 2 * (size_t)ms)) ||
            (tick_buffers && (e = alloc_tick_buffers(h)))) {
            cleanup();
            rc = set_err(GR_ALLOC_FAILED, cudaGetErrorString(e));
            break;
        }
        cudaMemsetAsync(h->rp, 0, ((size_t)n + 1) * 4, s);
        if (ms) {
            k_edge_emit<<<div_up(m, 256), 256, 0, s>>>((uint32_t)m, ekf, ek, ev, eflag, eexcl, d_w,
                                                          prm[P_INFLUENCE], weff, slo, shi, dk, dv, d_err,
                                                          h->simple_raw, h->simple_dcdw);
            esort.sort_bits(dk, dv, 2 * ms, 2 * ekf.bits, s, d_err + 1);
            k_csr<<<div_up(2 * (uint64_t)ms, 256), 256, 0, s>>>(n, 2 * ms, ekf, dk, dv, weff, h->rp, h->col,
                                                                 h->wt);
            cudaMemcpyAsync(h->csr_simple, dv, 2 * (size_t)ms * 4, cudaMemcpyDeviceToDevice, s);
        }
        float *d_xyz = nullptr;
        const size_t nxyz = (size_t)n * D;
        if (pos0 && (e = tmp(&d_xyz, std::max<size_t>(nxyz, 1) * 4))) {
            cleanup();
            rc = set_err(GR_ALLOC_FAILED, cudaGetErrorString(e));
            break;
        }
        uint32_t *d_goff = nullptr;  // per-graph seeded starts: offsets, then seeds
        if (n && !pos0 && starts.graphs) {
            if ((e = tmp(&d_goff, (size_t)starts.graphs * 8))) {
                cleanup();
                rc = set_err(GR_ALLOC_FAILED, cudaGetErrorString(e));
                break;
            }
            cudaMemcpyAsync(d_goff, starts.off, (size_t)starts.graphs * 4, cudaMemcpyHostToDevice, s);
            cudaMemcpyAsync(d_goff + starts.graphs, starts.seed, (size_t)starts.graphs * 4, cudaMemcpyHostToDevice,
                            s);
            if (D == 3)
                k_init_nodes_seeded<3><<<div_up(n, 256), 256, 0, s>>>(n, d_goff, d_goff + starts.graphs,
                                                                      starts.graphs, h->rp, h->pos);
            else
                k_init_nodes_seeded<2><<<div_up(n, 256), 256, 0, s>>>(n, d_goff, d_goff + starts.graphs,
                                                                      starts.graphs, h->rp, h->pos);
            cudaFreeAsync(d_goff, s);
        } else if (n) {
            if (pos0) cudaMemcpyAsync(d_xyz, pos0, nxyz * 4, cudaMemcpyHostToDevice, s);
            const uint32_t seed = (uint32_t)prm[P_SEED];
            if (D == 3)
                k_init_nodes<3><<<div_up(n, 256), 256, 0, s>>>(n, d_xyz, h->rp, h->pos, d_err, seed);
            else
                k_init_nodes<2><<<div_up(n, 256), 256, 0, s>>>(n, d_xyz, h->rp, h->pos, d_err, seed);
        }
        DevState init;
        memset(&init, 0, sizeof init);
        init.swing = init.traction = init.speed = init.speed_efficiency = 1.0;
        init.converged = n == 0 ? 1u : 0u;
        cudaMemcpyAsync(h->st, &init, sizeof init, cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(hdr, d_err, sizeof hdr, cudaMemcpyDeviceToHost, s);
        if (d_xyz) cudaFreeAsync(d_xyz, s);
        cleanup();
        e = cudaStreamSynchronize(s);
        if (e) {
            rc = set_err(GR_CUDA_ERROR, cudaGetErrorString(e));
            break;
        }
        if (hdr[0] & 4u) {
            rc = set_err(GR_INVALID_ARGUMENT, "non-finite start position");
            break;
        }
        if (hdr[0] & 2u) {
            rc = set_err(GR_INVALID_ARGUMENT, "edge weights must be finite and > 0 when edge_weight_influence != 0");
            break;
        }
        if (hdr[1]) {
            rc = set_err(GR_DEVICE_FAULT, "the edge sort gave up a bounded wait");
            break;
        }
        if (int c = build_segments(h)) {
            rc = c;
            break;
        }
    } while (0);
    if (rc != GR_OK) {
        delete h;
        return rc;
    }
    *out = h;
    return ok();
}

static int tick_impl(gr_fa2 *h, uint32_t ticks, float *dev_out, uint32_t *done) {
    if (!h) return set_err(GR_INVALID_HANDLE, "null handle");
    DevState s0;
    if (int c = read_state(h, &s0)) return c;
    if (h->n && ticks) {
        if (int c = build_graph(h)) return c;
        for (uint32_t t = 0; t < ticks; t++) {
            CU(cudaGraphLaunch(h->exec, h->stream));
            if (dev_out) {
                float *o = dev_out + (size_t)t * h->n * h->dim;
                if (h->dim == 3)
                    k_export<3><<<div_up(h->n, 256), 256, 0, h->stream>>>(h->n, h->pos, o);
                else
                    k_export<2><<<div_up(h->n, 256), 256, 0, h->stream>>>(h->n, h->pos, o);
            }
        }
    }
    DevState s1;
    if (int c = read_state(h, &s1)) return c;
    if (done) *done = s1.iter_no - s0.iter_no;
    if (int c = check_device(h, s1)) return c;
    return ok();
}

// ------------------------------------------------------------------ ABI -----

extern "C" {

uint32_t gr_abi_version(void) { return GR_ABI_VERSION; }
int gr_last_error(void) { return g_err; }
const char *gr_last_error_message(void) { return g_msg; }
int gr_last_error_index(void) { return g_err_index; }

static const char *kLayouts[] = {"layout.forceatlas2.barnes_hut.cuda", "layout.force.barnes_hut.cuda",
                                  "layout.force.particle_mesh.cuda"};

uint32_t gr_layout_count(void) { return 3; }
const char *gr_layout_id(uint32_t i) {
    if (i >= gr_layout_count()) {
        set_err(GR_INDEX_OUT_OF_RANGE, "layout index past the end");
        return nullptr;
    }
    ok();
    return kLayouts[i];
}

uint32_t gr_fa2_param_count(void) { return kNParams; }

int gr_fa2_param_spec(uint32_t i, const char **name, int *kind, double *min, double *max, double *def,
                      double *step, const char **doc) {
    if (i >= kNParams) return set_err(GR_INDEX_OUT_OF_RANGE, "parameter index past the end");
    const Spec &s = kSpecs[i];
    if (name) *name = s.name;
    if (kind) *kind = s.kind;
    if (min) *min = s.min;
    if (max) *max = s.max;
    if (def) *def = s.def;
    if (step) *step = s.step;
    if (doc) *doc = s.doc;
    return ok();
}

int gr_fa2_params_values(const uint8_t *params, size_t params_len, double *values_out) {
    double v[16];
    if (int c = params_values(params, params_len, v)) return c;
    if (values_out) memcpy(values_out, v, kNParams * sizeof(double));
    return ok();
}

int gr_fa2_create(gr_fa2 **out, uint32_t n, uint64_t m, const uint32_t *src, const uint32_t *dst,
                  const double *weight, const uint8_t *params, size_t params_len, const float *pos0) {
    return create_impl(out, n, m, src, dst, weight, params, params_len, pos0);
}

void gr_fa2_destroy(gr_fa2 *h) {
    if (!h) return;
    if (h->stream) cudaStreamSynchronize(h->stream);
    delete h;
}

int gr_fa2_tick(gr_fa2 *h, uint32_t ticks, uint32_t *done) { return tick_impl(h, ticks, nullptr, done); }

int gr_fa2_run(gr_fa2 *h, uint32_t *done) {
    if (!h) return set_err(GR_INVALID_HANDLE, "null handle");
    return tick_impl(h, (uint32_t)h->prm[P_MAX_ITER], nullptr, done);
}

int gr_fa2_tick_timed(gr_fa2 *h, uint32_t ticks, size_t l2_flush_bytes, float *ms_out, uint32_t *done) {
    if (!h) return set_err(GR_INVALID_HANDLE, "null handle");
    if (!ms_out) return set_err(GR_INVALID_ARGUMENT, "ms_out is null");
    DevState s0;
    if (int c = read_state(h, &s0)) return c;
    if (h->n && ticks) {
        if (int c = build_timed_graph(h)) return c;
        if (l2_flush_bytes && l2_flush_bytes != h->flush_bytes) {
            if (h->flush) cudaFree(h->flush);
            h->flush = nullptr;
            CU(cudaMalloc(&h->flush, l2_flush_bytes));
            h->flush_bytes = l2_flush_bytes;
        }
        for (uint32_t t = 0; t < ticks; t++) {
            if (l2_flush_bytes) CU(cudaMemsetAsync(h->flush, (int)(t & 0xff), l2_flush_bytes, h->stream));
            CU(cudaGraphLaunch(h->texec, h->stream));
            CU(cudaStreamSynchronize(h->stream));
            float a = 0.f, b = 0.f, c = 0.f, d = 0.f;
            CU(cudaEventElapsedTime(&a, h->ev[0], h->ev[1]));
            CU(cudaEventElapsedTime(&b, h->ev[1], h->ev[2]));
            CU(cudaEventElapsedTime(&c, h->ev[2], h->ev[3]));
            CU(cudaEventElapsedTime(&d, h->ev[0], h->ev[3]));
            ms_out[4 * t + 0] = a;
            ms_out[4 * t + 1] = b;
            ms_out[4 * t + 2] = c;
            ms_out[4 * t + 3] = d;
        }
    }
    DevState s1;
    if (int c = read_state(h, &s1)) return c;
    if (done) *done = s1.iter_no - s0.iter_no;
    if (int c = check_device(h, s1)) return c;
    return ok();
}

int gr_fa2_tick_record(gr_fa2 *h, uint32_t ticks, float *dev_out, uint32_t *done) {
    if (!dev_out) return set_err(GR_INVALID_ARGUMENT, "dev_out is null");
    return tick_impl(h, ticks, dev_out, done);
}

int gr_fa2_positions(gr_fa2 *h, float *out) {
    if (!h) return set_err(GR_INVALID_HANDLE, "null handle");
    if (!out) return set_err(GR_INVALID_ARGUMENT, "out is null");
    if (h->n == 0) return ok();
    // the copy flags a non-finite coordinate on the device (one word back, not a
    // host pass over every coordinate)
    const size_t count = (size_t)h->n * h->dim;
    float *d = nullptr;
    CU(cudaMallocAsync((void **)&d, count * 4 + 4, h->stream));
    uint32_t *flag = (uint32_t *)(d + count);
    cudaMemsetAsync(flag, 0, 4, h->stream);
    if (h->dim == 3)
        k_export<3><<<div_up(h->n, 256), 256, 0, h->stream>>>(h->n, h->pos, d, flag);
    else
        k_export<2><<<div_up(h->n, 256), 256, 0, h->stream>>>(h->n, h->pos, d, flag);
    uint32_t bad = 0;
    cudaMemcpyAsync(out, d, count * 4, cudaMemcpyDeviceToHost, h->stream);
    cudaMemcpyAsync(&bad, flag, 4, cudaMemcpyDeviceToHost, h->stream);
    cudaFreeAsync(d, h->stream);
    CU(cudaStreamSynchronize(h->stream));
    if (bad) return set_err(GR_LAYOUT_FAILED, "non-finite position (StageError::NonFinite)");
    return ok();
}

int gr_fa2_set_positions(gr_fa2 *h, const float *pos) {
    if (!h) return set_err(GR_INVALID_HANDLE, "null handle");
    if (!pos) return set_err(GR_INVALID_ARGUMENT, "pos is null");
    if (h->n == 0) return ok();
    for (size_t i = 0; i < (size_t)h->n * h->dim; i++)
        if (!std::isfinite(pos[i])) return set_err(GR_INVALID_ARGUMENT, "non-finite position");
    float *d = nullptr;
    CU(cudaMallocAsync((void **)&d, (size_t)h->n * h->dim * 4, h->stream));
    cudaMemcpyAsync(d, pos, (size_t)h->n * h->dim * 4, cudaMemcpyHostToDevice, h->stream);
    if (h->dim == 3)
        k_import<3><<<div_up(h->n, 256), 256, 0, h->stream>>>(h->n, h->pos, d);
    else
        k_import<2><<<div_up(h->n, 256), 256, 0, h->stream>>>(h->n, h->pos, d);
    cudaFreeAsync(d, h->stream);
    // the bounds the last update computed are not these positions'
    cudaMemsetAsync(&h->st->bounds_stamp, 0, sizeof(uint32_t), h->stream);
    CU(cudaStreamSynchronize(h->stream));
    return ok();
}

int gr_fa2_positions_device(gr_fa2 *h, const void **dev_nodes) {
    if (!h) return set_err(GR_INVALID_HANDLE, "null handle");
    if (!dev_nodes) return set_err(GR_INVALID_ARGUMENT, "dev_nodes is null");
    *dev_nodes = h->pos;
    return ok();
}

int gr_fa2_forces(gr_fa2 *h, float *out) {
    if (!h) return set_err(GR_INVALID_HANDLE, "null handle");
    if (!out) return set_err(GR_INVALID_ARGUMENT, "out is null");
    if (h->n == 0) return ok();
    DevState s0;
    if (int c = read_state(h, &s0)) return c;
    // a converged state still answers: evaluate on a copy that is not converged
    DevState s = s0;
    s.converged = 0;
    CU(cudaMemcpyAsync(h->st, &s, sizeof s, cudaMemcpyHostToDevice, h->stream));
    enqueue(h, true);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(out, h->U, (size_t)h->n * h->dim * 4, cudaMemcpyDeviceToHost, h->stream));
    DevState s1;
    if (int c = read_state(h, &s1)) return c;
    int rc = check_device(h, s1);
    // restore the speed controller and tick count; keep the interaction counters
    s0.far_count = s1.far_count;
    s0.pair_count = s1.pair_count;
    s0.n_cells = s1.n_cells;
    s0.n_unique = s1.n_unique;
    CU(cudaMemcpyAsync(h->st, &s0, sizeof s0, cudaMemcpyHostToDevice, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    if (rc) return rc;
    return ok();
}

int gr_fa2_get_info(gr_fa2 *h, gr_fa2_info *out) {
    if (!h) return set_err(GR_INVALID_HANDLE, "null handle");
    if (!out) return set_err(GR_INVALID_ARGUMENT, "out is null");
    DevState s;
    if (int c = read_state(h, &s)) return c;
    out->n = h->n;
    out->dim = (uint32_t)h->dim;
    out->m = h->m;
    out->iter_no = s.iter_no;
    out->converged = s.converged;
    out->n_cells = s.n_cells;
    out->n_leaves = s.n_unique;
    out->swing = s.swing;
    out->traction = s.traction;
    out->speed = s.speed;
    out->speed_efficiency = s.speed_efficiency;
    out->moved = s.moved;
    out->far_count = s.far_count;
    out->pair_count = s.pair_count;
    out->device_error = s.error;
    out->graph_kernels = h->graph_kernels;
    return ok();
}

int gr_fa2_set_walk_schedule(gr_fa2 *h, int schedule) {
    if (!h) return set_err(GR_INVALID_HANDLE, "null handle");
    if (schedule < 0 || schedule >= GR_WALK_SCHEDULES)
        return set_err(GR_INVALID_ARGUMENT, "walk schedule must be 0, 1, 2 or 3");
    if (schedule != h->walk_schedule) {
        h->walk_schedule = schedule;
        h->drop_graphs();
    }
    return ok();
}

int gr_fa2_launch_mode(gr_fa2 *h, int *programmatic) {
    if (!h) return set_err(GR_INVALID_HANDLE, "null handle");
    if (!programmatic) return set_err(GR_INVALID_ARGUMENT, "programmatic is null");
    *programmatic = h->pdl ? 1 : 0;
    return ok();
}

int gr_fa2_set_interaction_counting(gr_fa2 *h, int on) {
    if (!h) return set_err(GR_INVALID_HANDLE, "null handle");
    if (on != 0 && on != 1) return set_err(GR_INVALID_ARGUMENT, "on must be 0 or 1");
    if ((on == 1) != h->count_interactions) {
        h->count_interactions = on == 1;
        h->drop_graphs();
    }
    return ok();
}

int gr_fa2_set_wait_limit(gr_fa2 *h, uint32_t spins) {
    if (!h) return set_err(GR_INVALID_HANDLE, "null handle");
    const uint32_t limit = spins ? spins : OS_SPIN_LIMIT;
    if (limit != h->sorter.wait.limit) {
        h->sorter.wait.limit = limit;
        h->drop_graphs();
    }
    return ok();
}

int gr_fa2_inject_stalled_wait(gr_fa2 *h, int on) {
    if (!h) return set_err(GR_INVALID_HANDLE, "null handle");
    if (on != 0 && on != 1) return set_err(GR_INVALID_ARGUMENT, "on must be 0 or 1");
    if (on && !h->stall_word) {
        cudaError_t e = h->alloc(&h->stall_word, 1);
        if (e) return set_err(GR_ALLOC_FAILED, cudaGetErrorString(e));
        CU(cudaMemsetAsync(h->stall_word, 0, sizeof(uint32_t), h->stream));
        CU(cudaStreamSynchronize(h->stream));
    }
    const uint32_t *want = on ? h->stall_word : nullptr;
    if (want != h->sorter.wait.stall) {
        h->sorter.wait.stall = want;
        h->drop_graphs();
    }
    return ok();
}

int gr_fa2_tune(gr_fa2 *h, uint32_t sample_ticks, int *chosen, float *walk_ms_each) {
    if (!h) return set_err(GR_INVALID_HANDLE, "null handle");
    if (h->n == 0) return ok();
    if (sample_ticks == 0) sample_ticks = 1;
    // time each walk schedule over the same ticks from the same state, then restore it
    float4 *save_p = nullptr;
    DevState save_s;
    CU(cudaMalloc(&save_p, (size_t)h->n * sizeof(float4)));
    CU(cudaMemcpyAsync(save_p, h->pos, (size_t)h->n * sizeof(float4), cudaMemcpyDeviceToDevice, h->stream));
    if (int c = read_state(h, &save_s)) {
        cudaFree(save_p);
        return c;
    }
    std::vector<float> ms(4 * (size_t)sample_ticks);
    float best = 1e30f;
    int pick = h->walk_schedule, rc = GR_OK;
    for (int sch = 0; sch < GR_WALK_SCHEDULES && rc == GR_OK; sch++) {
        h->walk_schedule = sch;
        h->drop_graphs();
        uint32_t done = 0;
        rc = gr_fa2_tick_timed(h, sample_ticks, 0, ms.data(), &done);
        float w = 0.f;
        for (uint32_t t = 0; t < done; t++) w += ms[4 * t + 1];
        w /= std::max(done, 1u);
        if (walk_ms_each) walk_ms_each[sch] = w;
        if (rc == GR_OK && done && w < best) {
            best = w;
            pick = sch;
        }
        cudaMemcpyAsync(h->pos, save_p, (size_t)h->n * sizeof(float4), cudaMemcpyDeviceToDevice, h->stream);
        cudaMemcpyAsync(h->st, &save_s, sizeof save_s, cudaMemcpyHostToDevice, h->stream);
        cudaStreamSynchronize(h->stream);
    }
    cudaFree(save_p);
    h->walk_schedule = pick;
    h->drop_graphs();
    if (chosen) *chosen = pick;
    if (rc) return rc;
    return ok();
}

int gr_fa2_get_controller(gr_fa2 *h, gr_fa2_controller *out) {
    if (!h) return set_err(GR_INVALID_HANDLE, "null handle");
    if (!out) return set_err(GR_INVALID_ARGUMENT, "out is null");
    DevState s;
    if (int c = read_state(h, &s)) return c;
    out->swing = s.swing;
    out->traction = s.traction;
    out->speed = s.speed;
    out->speed_efficiency = s.speed_efficiency;
    out->iter_no = s.iter_no;
    out->converged = s.converged;
    return ok();
}

int gr_fa2_set_controller(gr_fa2 *h, const gr_fa2_controller *in) {
    if (!h) return set_err(GR_INVALID_HANDLE, "null handle");
    if (!in) return set_err(GR_INVALID_ARGUMENT, "in is null");
    if (!(std::isfinite(in->swing) && std::isfinite(in->traction) && std::isfinite(in->speed) &&
          std::isfinite(in->speed_efficiency)))
        return set_err(GR_INVALID_ARGUMENT, "non-finite controller state");
    DevState s;
    if (int c = read_state(h, &s)) return c;
    s.swing = in->swing;
    s.traction = in->traction;
    s.speed = in->speed;
    s.speed_efficiency = in->speed_efficiency;
    s.iter_no = in->iter_no;
    s.converged = (in->converged || h->n == 0) ? 1u : 0u;
    s.error = 0;
    CU(cudaMemcpyAsync(h->st, &s, sizeof s, cudaMemcpyHostToDevice, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    return ok();
}

int gr_fa2_set_stream(gr_fa2 *h, void *cuda_stream) {
    if (!h) return set_err(GR_INVALID_HANDLE, "null handle");
    if (h->stream) CU(cudaStreamSynchronize(h->stream));
    if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
    h->own_stream = false;
    h->stream = (cudaStream_t)cuda_stream;
    h->drop_graphs();
    return ok();
}

int gr_run(const char *layout_id, uint32_t n, uint64_t m, const uint32_t *src, const uint32_t *dst,
           const double *weight, const uint8_t *params, size_t params_len, float *out) {
    if (layout_id && strcmp(layout_id, kLayouts[1]) == 0) {
        // the d3-force row publishes no parameters (registry/layouts.rs LayoutParams::NONE)
        if (params_len) return set_err(GR_PARAMS_NOT_ACCEPTED, "layout.force.barnes_hut.cuda takes no parameters");
        return gr_force_run(n, m, src, dst, weight, out);
    }
    if (layout_id && strcmp(layout_id, kLayouts[2]) == 0) {
        if (params_len) return set_err(GR_PARAMS_NOT_ACCEPTED, "layout.force.particle_mesh.cuda takes no parameters");
        return gr_force_mesh_run(n, m, src, dst, weight, out);
    }
    if (!layout_id || strcmp(layout_id, kLayouts[0]) != 0)
        return set_err(GR_UNKNOWN_LAYOUT_ID, "unknown layout id");
    gr_fa2 *h = nullptr;
    if (int c = gr_fa2_create(&h, n, m, src, dst, weight, params, params_len, nullptr)) return c;
    int rc = gr_fa2_run(h, nullptr);
    if (rc == GR_OK) rc = gr_fa2_positions(h, out);
    int keep = g_err, keep_i = g_err_index;
    char msg[256];
    memcpy(msg, g_msg, sizeof msg);
    gr_fa2_destroy(h);
    g_err = keep;
    g_err_index = keep_i;
    memcpy(g_msg, msg, sizeof msg);
    return rc;
}

}  // extern "C"

// ------------------------------------------- allocation-free force pass ----
//
// gr_fa2_forces_static: one force evaluation (the same kernels as
// gr_fa2_forces) for callers that cannot allocate device memory at all — code
// running inside another runtime that owns every device allocation (its own
// stream-ordered or pooled allocator), or a plugin that is only handed device
// buffers by its host. Its scratch is the file-scope array below, sized for
// STATIC_MAX_N nodes; every GPU that loads this library holds that array until
// the process exits. The caller passes inputs and outputs in device memory;
// nothing here calls cudaMalloc, cudaFree or any allocating routine.

constexpr uint32_t STATIC_MAX_N = GR_FORCES_STATIC_MAX_N;
constexpr size_t STATIC_BYTES_PER_NODE = 400;
constexpr size_t STATIC_BYTES = STATIC_BYTES_PER_NODE * STATIC_MAX_N + (1u << 20);

static __device__ __align__(256) unsigned char g_static_scratch[STATIC_BYTES];

// Host-side device addresses of g_static_scratch, one per device, with the id
// of the context each was looked up in. In host code the symbol itself is only a
// stand-in, never a device address. A device reset (cudaDeviceReset) ends the
// context the address belongs to; the next call sees a new context id and looks
// the address up again.
static std::mutex g_static_mu;
static unsigned char *g_static_base[256];
static unsigned long long g_static_ctx[256];

// The id of the calling thread's current context (driver entry points found at
// run time, so the library links no driver library); false when there is none.
static bool current_context_id(unsigned long long *id) {
    typedef int (*CtxGetCurrent)(void **);
    typedef int (*CtxGetId)(void *, unsigned long long *);
    static CtxGetCurrent get_current = nullptr;
    static CtxGetId get_id = nullptr;
    static bool looked = false;
    if (!looked) {
        void *f = nullptr, *g = nullptr;
        cudaDriverEntryPointQueryResult q1, q2;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q1) == cudaSuccess &&
            cudaGetDriverEntryPoint("cuCtxGetId", &g, cudaEnableDefault, &q2) == cudaSuccess &&
            q1 == cudaDriverEntryPointSuccess && q2 == cudaDriverEntryPointSuccess) {
            get_current = (CtxGetCurrent)f;
            get_id = (CtxGetId)g;
        }
        cudaGetLastError();
        looked = true;
    }
    void *ctx = nullptr;
    if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx) return false;
    return get_id(ctx, id) == 0;
}

static int static_base(unsigned char **out) {
    int dev = 0;
    CU(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 256) return set_err(GR_INVALID_ARGUMENT, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_static_mu);
    unsigned long long id = 0;
    const bool known = current_context_id(&id);
    if (!g_static_base[dev] || !known || id != g_static_ctx[dev]) {
        void *p = nullptr;
        CU(cudaGetSymbolAddress(&p, g_static_scratch));  // makes the device's context current
        g_static_base[dev] = (unsigned char *)p;
        g_static_ctx[dev] = current_context_id(&id) ? id : 0ull;
    }
    *out = g_static_base[dev];
    return GR_OK;
}

// Bump layout of the per-call buffers inside the static array (256-byte aligned).
struct Carve {
    unsigned char *base;
    size_t off = 0;
    template <typename T>
    T *take(size_t count) {
        off = (off + 255) & ~(size_t)255;
        T *p = (T *)(base + off);
        off += (count ? count : 1) * sizeof(T);
        return p;
    }
};

__global__ void k_static_init(DevState *st, uint32_t tick) {
    DevState z;
    memset(&z, 0, sizeof z);
    z.swing = z.traction = z.speed = z.speed_efficiency = 1.0;
    z.iter_no = tick;
    *st = z;
}

template <int D>
static int forces_static(uint32_t n, const float4 *nodes, const uint32_t *rp, const uint32_t *col,
                         const float *wt, const double *prm, uint32_t tick, float *out, cudaStream_t s) {
    unsigned char *base = nullptr;
    if (int c = static_base(&base)) return c;
    Carve cv{base};
    gr_fa2 h;  // a view over static memory: owns nothing, allocates nothing
    h.dim = D;
    h.n = n;
    memcpy(h.prm, prm, sizeof h.prm);
    h.stream = s;
    h.own_stream = false;
    h.pdl = pdl_default();  // GR_PDL=0 in the environment: plain stream order
    h.st = cv.take<DevState>(1);  // first, at offset 0: gr_fa2_forces_static_status reads it there
    h.keys = cv.take<uint64_t>(n);
    h.vals = cv.take<uint32_t>(n);
    h.ukey = cv.take<uint64_t>(n);
    h.sorig = cv.take<uint32_t>(n);
    h.uid = cv.take<uint32_t>(n);
    h.leaf_start = cv.take<uint32_t>((size_t)n + 1);
    h.levels = cv.take<uint32_t>(n);
    h.cell_flag = cv.take<uint8_t>(n);
    h.P = cv.take<uint32_t>((size_t)n + 1);
    h.leaf_pre = cv.take<uint32_t>(n);
    h.sp = cv.take<float4>(n);
    h.bt.first = cv.take<uint32_t>(n);
    h.bt.last = cv.take<uint32_t>(n);
    h.bt.left = cv.take<uint32_t>(n);
    h.bt.right = cv.take<uint32_t>(n);
    h.bt.delta = cv.take<int32_t>(n);
    h.bt.int_parent = cv.take<int32_t>(n);
    h.bt.leaf_parent = cv.take<int32_t>(n);
    h.bt.visit = cv.take<uint32_t>(n);
    h.bt.rec = cv.take<int4>(n);
    h.leaf_body = cv.take<Body>(n);
    h.int_body = cv.take<Body>(n);
    h.leaf_coinc = cv.take<uint8_t>(n);
    h.pre_local = cv.take<double>(4 * ((size_t)n + 1));
    h.tile_sum = cv.take<Body>(div_up(n, AG_TILE) + 1);
    h.tile_carry = cv.take<BodyDD>(div_up(n, AG_TILE) + 1);
    h.tile_cnt = cv.take<uint32_t>(2 * ((size_t)div_up(n, AG_TILE) + 1));
    h.cells = cells_view(cv.take<float4>(cells_float4s(2 * n, D)), 2 * n, D);
    h.rep = cv.take<float>((size_t)n * D);
    h.part = cv.take<double>(std::max<size_t>((size_t)h.bnd_blocks() * 3 * D, 2 * (size_t)div_up(n, FRC_THREADS)) + 8);
    h.sorter.cap = n;
    h.sorter.ntiles = div_up(n, RS_TILE);
    h.sorter.k_alt = cv.take<uint64_t>(n);
    h.sorter.v_alt = cv.take<uint32_t>(n);
    h.sorter.hist = cv.take<uint32_t>((size_t)RS_BINS * h.sorter.ntiles);
    h.sorter.totals = cv.take<uint32_t>(8 * RS_BINS);
    h.scanner.cap = n;
    h.scanner.nb = div_up(n, SC_TILE);
    h.scanner.bsum = cv.take<uint32_t>(h.scanner.nb);
    if (cv.off > STATIC_BYTES) return set_err(GR_INVALID_ARGUMENT, "static scratch layout exceeds the array");
    h.rp = const_cast<uint32_t *>(rp);
    h.col = const_cast<uint32_t *>(col);
    h.wt = const_cast<float *>(wt);
    h.pos = const_cast<float4 *>(nodes);
    h.U = out;
    // seg_first stays null: every row takes the row loop.
    k_static_init<<<1, 1, 0, s>>>(h.st, tick);
    enqueue_tick<D>(&h, true, PH_ALL);
    cudaError_t e = cudaGetLastError();
    // the view must not release what it points at
    h.rp = nullptr;
    h.col = nullptr;
    h.wt = nullptr;
    h.pos = nullptr;
    h.U = nullptr;
    h.sorter = RadixSorter();
    h.scanner = Scanner();
    h.allocs.clear();
    if (e != cudaSuccess) return set_err(GR_CUDA_ERROR, cudaGetErrorString(e));
    return GR_OK;
}

extern "C" {

int gr_fa2_forces_static(uint32_t n, const void *nodes, const uint32_t *row_ptr, const uint32_t *col,
                         const float *weight, const uint8_t *params, size_t params_len, uint32_t tick,
                         float *out, void *stream) {
    double prm[16];
    if (int c = params_values(params, params_len, prm)) return c;
    if (n > STATIC_MAX_N) {
        char b[160];
        snprintf(b, sizeof b, "n = %u is beyond the static scratch's maximum of %u nodes", n, STATIC_MAX_N);
        return set_err(GR_INVALID_ARGUMENT, b);
    }
    if (n == 0) return ok();
    if (!nodes || !row_ptr || !col || !out || !weight) return set_err(GR_INVALID_ARGUMENT, "a device buffer is null");
    const cudaStream_t s = (cudaStream_t)stream;
    int rc = (int)prm[P_DIM] == 3 ? forces_static<3>(n, (const float4 *)nodes, row_ptr, col, weight, prm, tick, out, s)
                                  : forces_static<2>(n, (const float4 *)nodes, row_ptr, col, weight, prm, tick, out, s);
    if (rc) return rc;
    return ok();
}

int gr_fa2_forces_static_status(uint32_t *device_error) {
    unsigned char *base = nullptr;
    if (int c = static_base(&base)) return c;
    // forces_static carves its DevState first, at the array's offset 0
    DevState s;
    memset(&s, 0, sizeof s);
    CU(cudaMemcpy(&s.error, base + offsetof(DevState, error), sizeof s.error, cudaMemcpyDeviceToHost));
    if (device_error) *device_error = s.error;
    if (int c = check_device(nullptr, s)) return c;
    return ok();
}

}  // extern "C"

// ------------------------------------------------------------------ batch --
//
// Thousands of independent graphs in one persistent launch (batch.cuh). The
// concatenated graph (node ids offset per graph) goes through the one-graph
// create path for its simple-graph pass, CSR and start positions; the batch
// adds the per-graph table, the per-graph FP64 controller state, the work queue
// and one scratch slot per resident CTA.

struct gr_fa2_batch {
    gr_fa2 *g = nullptr;
    int dim = 2;
    uint32_t ngraphs = 0, nmax = 0, total_n = 0;
    std::vector<uint32_t> n_of, off_of;
    BatchGraph *d_graphs = nullptr;
    BatchState *d_state = nullptr;
    uint32_t *d_order = nullptr, *d_next = nullptr, *d_heavy = nullptr;
    unsigned char *d_slots = nullptr;
    size_t slot_bytes = 0;
    uint32_t max_slots = 0;
    int threads = 512;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint32_t graph_ticks = 0;
    int graph_threads = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    void drop_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
    }
    ~gr_fa2_batch() {
        drop_graph();
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        for (void *p : {(void *)d_graphs, (void *)d_state, (void *)d_order, (void *)d_next, (void *)d_heavy,
                        (void *)d_slots})
            if (p) cudaFree(p);
        if (g) {
            if (g->stream) cudaStreamSynchronize(g->stream);
            delete g;
        }
    }
};

template <int D, int BT>
static int batch_slots(uint32_t *slots) {
    int dev = 0, sms = 0, per = 0;
    CU(cudaGetDevice(&dev));
    CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_batch<D, BT>, BT, 0));
    *slots = (uint32_t)std::max(1, per) * (uint32_t)sms;
    return GR_OK;
}

static int batch_slots_for(int dim, int bt, uint32_t *slots) {
    if (dim == 3) {
        if (bt == 256) return batch_slots<3, 256>(slots);
        if (bt == 1024) return batch_slots<3, 1024>(slots);
        return batch_slots<3, 512>(slots);
    }
    if (bt == 256) return batch_slots<2, 256>(slots);
    if (bt == 1024) return batch_slots<2, 1024>(slots);
    return batch_slots<2, 512>(slots);
}

template <int D, int BT>
static void batch_launch(gr_fa2_batch *b, uint32_t ticks, uint32_t slots) {
    BatchArgs a;
    a.graphs = b->d_graphs;
    a.state = b->d_state;
    a.order = b->d_order;
    a.ngraphs = b->ngraphs;
    a.next = b->d_next;
    a.pos = b->g->pos;
    a.rp = b->g->rp;
    a.col = b->g->col;
    a.wt = b->g->wt;
    a.heavy = b->d_heavy;
    a.slots = b->d_slots;
    a.slot_bytes = b->slot_bytes;
    a.nmax = b->nmax;
    a.ticks = ticks;
    cudaMemsetAsync(b->d_next, 0, sizeof(uint32_t), b->g->stream);
    k_batch<D, BT><<<slots, BT, 0, b->g->stream>>>(a);
}

static int batch_enqueue(gr_fa2_batch *b, uint32_t ticks) {
    uint32_t slots = 0;
    if (int c = batch_slots_for(b->dim, b->threads, &slots)) return c;
    slots = std::min(slots, b->max_slots);
    if (b->dim == 3) {
        if (b->threads == 256) batch_launch<3, 256>(b, ticks, slots);
        else if (b->threads == 1024) batch_launch<3, 1024>(b, ticks, slots);
        else batch_launch<3, 512>(b, ticks, slots);
    } else {
        if (b->threads == 256) batch_launch<2, 256>(b, ticks, slots);
        else if (b->threads == 1024) batch_launch<2, 1024>(b, ticks, slots);
        else batch_launch<2, 512>(b, ticks, slots);
    }
    return GR_OK;
}

static int batch_run_impl(gr_fa2_batch *b, uint32_t ticks, float *ms) {
    cudaStream_t s = b->g->stream;
    if (!b->exec || b->graph_ticks != ticks || b->graph_threads != b->threads) {
        b->drop_graph();
        CU(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        int c = batch_enqueue(b, ticks);
        cudaError_t e = cudaStreamEndCapture(s, &b->graph);
        if (c) return c;
        if (e != cudaSuccess) return set_err(GR_CUDA_ERROR, cudaGetErrorString(e));
        CU(cudaGraphInstantiate(&b->exec, b->graph, 0));
        b->graph_ticks = ticks;
        b->graph_threads = b->threads;
    }
    if (!b->ev0) CU(cudaEventCreate(&b->ev0));
    if (!b->ev1) CU(cudaEventCreate(&b->ev1));
    CU(cudaEventRecord(b->ev0, s));
    CU(cudaGraphLaunch(b->exec, s));
    CU(cudaEventRecord(b->ev1, s));
    CU(cudaEventSynchronize(b->ev1));
    CU(cudaGetLastError());
    if (ms) CU(cudaEventElapsedTime(ms, b->ev0, b->ev1));
    return GR_OK;
}

extern "C" {

int gr_fa2_batch_create(gr_fa2_batch **out, uint32_t ngraphs, const uint32_t *node_counts,
                        const uint64_t *edge_counts, const uint32_t *src, const uint32_t *dst, const double *weight,
                        const double *params, uint32_t params_per_graph, const float *pos0) {
    if (!out) return set_err(GR_INVALID_ARGUMENT, "out is null");
    *out = nullptr;
    if (ngraphs == 0 || !node_counts || !edge_counts) return set_err(GR_INVALID_ARGUMENT, "no graphs");
    if (params_per_graph != 0 && params_per_graph != kRefParams && params_per_graph != kNParams)
        return set_err(GR_PARAMS_MALFORMED, "params_per_graph must be 0, 5 or 11");
    if (params_per_graph && !params) return set_err(GR_INVALID_ARGUMENT, "params is null");
    std::vector<double> prm((size_t)ngraphs * 16);
    int dim = -1;
    for (uint32_t g = 0; g < ngraphs; g++) {
        std::vector<uint8_t> b((size_t)params_per_graph * 8);
        if (params_per_graph) memcpy(b.data(), params + (size_t)g * params_per_graph, b.size());
        if (int c = params_values(b.data(), b.size(), &prm[(size_t)g * 16])) {
            char m[256];
            snprintf(m, sizeof m, "graph %u: %.200s", g, g_msg);
            int idx = g_err_index;
            return set_err(c, m, idx);
        }
        const int d = (int)prm[(size_t)g * 16 + P_DIM];
        if (dim >= 0 && d != dim) return set_err(GR_INVALID_ARGUMENT, "every graph of a batch has the same dim");
        dim = d;
    }
    uint64_t total_n = 0, total_m = 0;
    std::vector<uint32_t> off(ngraphs);
    uint32_t nmax = 1;
    for (uint32_t g = 0; g < ngraphs; g++) {
        off[g] = (uint32_t)total_n;
        total_n += node_counts[g];
        total_m += edge_counts[g];
        nmax = std::max(nmax, node_counts[g]);
    }
    if (total_n >= 0x7fffffffull || total_m > 0x7fffffffull)
        return set_err(GR_INVALID_ARGUMENT, "batch larger than 2^31 nodes or edges");
    if (total_m && (!src || !dst)) return set_err(GR_INVALID_ARGUMENT, "edge arrays are null");
    // global edge ids, effective weights (w ^ influence of the edge's graph)
    std::vector<uint32_t> gs(total_m), gd(total_m);
    std::vector<double> gw;
    bool any_influence = false;
    for (uint32_t g = 0; g < ngraphs; g++) any_influence |= prm[(size_t)g * 16 + P_INFLUENCE] != 0.0;
    if (weight && any_influence) gw.resize(total_m);
    uint64_t e = 0;
    for (uint32_t g = 0; g < ngraphs; g++) {
        const double infl = prm[(size_t)g * 16 + P_INFLUENCE];
        for (uint64_t k = 0; k < edge_counts[g]; k++, e++) {
            if (src[e] >= node_counts[g] || dst[e] >= node_counts[g])
                return set_err(GR_INVALID_ARGUMENT, "an edge names a node outside its graph");
            gs[e] = src[e] + off[g];
            gd[e] = dst[e] + off[g];
            if (!gw.empty()) {
                const double x = weight[e];
                if (infl != 0.0 && !(std::isfinite(x) && x > 0.0))
                    return set_err(GR_INVALID_ARGUMENT, "edge weights must be finite and > 0");
                gw[e] = infl == 0.0 ? 1.0 : (infl == 1.0 ? x : std::pow(x, infl));
            }
        }
    }
    // start positions: given, or Mulberry32(seed of the graph) per graph, drawn
    // on the device
    std::vector<uint32_t> seeds(ngraphs);
    for (uint32_t g = 0; g < ngraphs; g++) seeds[g] = (uint32_t)prm[(size_t)g * 16 + P_SEED];
    SeededStarts starts;
    if (!pos0) {
        starts.graphs = ngraphs;
        starts.off = off.data();
        starts.seed = seeds.data();
    }
    double base[11];
    for (uint32_t i = 0; i < kNParams; i++) base[i] = kSpecs[i].def;
    base[P_DIM] = dim;
    base[P_INFLUENCE] = gw.empty() ? 0.0 : 1.0;
    uint8_t bb[11 * 8];
    memcpy(bb, base, sizeof bb);
    gr_fa2 *G = nullptr;
    if (int c = create_impl(&G, (uint32_t)total_n, total_m, gs.data(), gd.data(), gw.empty() ? nullptr : gw.data(),
                            bb, sizeof bb, pos0, false, starts))
        return c;
    gr_fa2_batch *b = new (std::nothrow) gr_fa2_batch();
    if (!b) {
        gr_fa2_destroy(G);
        return set_err(GR_ALLOC_FAILED, "host allocation failed");
    }
    b->g = G;
    b->dim = dim;
    b->ngraphs = ngraphs;
    b->nmax = nmax;
    b->total_n = (uint32_t)total_n;
    b->n_of.assign(node_counts, node_counts + ngraphs);
    b->off_of = off;
    // heavy rows and the per-graph table
    std::vector<uint32_t> rp(total_n + 1);
    if (cudaMemcpy(rp.data(), G->rp, rp.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
        delete b;
        return set_err(GR_CUDA_ERROR, "reading the CSR offsets failed");
    }
    std::vector<uint32_t> heavy;
    std::vector<BatchGraph> tab(ngraphs);
    std::vector<BatchState> st(ngraphs);
    for (uint32_t g = 0; g < ngraphs; g++) {
        const double *v = &prm[(size_t)g * 16];
        BatchGraph &t = tab[g];
        memset(&t, 0, sizeof t);
        t.off = off[g];
        t.n = node_counts[g];
        t.heavy0 = (uint32_t)heavy.size();
        for (uint32_t i = off[g]; i < off[g] + node_counts[g]; i++)
            if (rp[i + 1] - rp[i] > LIGHT_MAX) heavy.push_back(i);
        t.heavy1 = (uint32_t)heavy.size();
        t.kr = (float)v[P_SCALING];
        t.th2 = (float)(v[P_THETA] * v[P_THETA]);
        t.gravity = (float)v[P_GRAVITY];
        t.seed = (uint32_t)v[P_SEED];
        t.lin_log = (int)v[P_LINLOG];
        t.strong_gravity = (int)v[P_STRONG];
        t.dissuade_hubs = (int)v[P_DISSUADE];
        t.jitter_tolerance = v[P_JT];
        memset(&st[g], 0, sizeof st[g]);
        st[g].swing = st[g].traction = st[g].speed = st[g].speed_efficiency = 1.0;
    }
    std::vector<uint32_t> order(ngraphs);
    for (uint32_t g = 0; g < ngraphs; g++) order[g] = g;
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t a, uint32_t c) { return node_counts[a] > node_counts[c]; });
    uint32_t slots = 0;
    for (int bt : {256, 512, 1024}) {
        uint32_t sl = 0;
        if (int c = batch_slots_for(dim, bt, &sl)) {
            delete b;
            return c;
        }
        slots = std::max(slots, sl);
    }
    slots = std::min(slots, ngraphs);
    SlotView sv;
    b->slot_bytes = slot_carve(nullptr, nmax, dim, sv);
    b->max_slots = slots;
    cudaError_t ce;
    if ((ce = cudaMalloc(&b->d_graphs, ngraphs * sizeof(BatchGraph))) ||
        (ce = cudaMalloc(&b->d_state, ngraphs * sizeof(BatchState))) ||
        (ce = cudaMalloc(&b->d_order, ngraphs * sizeof(uint32_t))) || (ce = cudaMalloc(&b->d_next, 4)) ||
        (ce = cudaMalloc(&b->d_heavy, std::max<size_t>(heavy.size(), 1) * 4)) ||
        (ce = cudaMalloc(&b->d_slots, b->slot_bytes * slots))) {
        delete b;
        return set_err(GR_ALLOC_FAILED, cudaGetErrorString(ce));
    }
    cudaMemcpy(b->d_graphs, tab.data(), ngraphs * sizeof(BatchGraph), cudaMemcpyHostToDevice);
    cudaMemcpy(b->d_state, st.data(), ngraphs * sizeof(BatchState), cudaMemcpyHostToDevice);
    cudaMemcpy(b->d_order, order.data(), ngraphs * 4, cudaMemcpyHostToDevice);
    if (!heavy.empty()) cudaMemcpy(b->d_heavy, heavy.data(), heavy.size() * 4, cudaMemcpyHostToDevice);
    if ((ce = cudaDeviceSynchronize())) {
        delete b;
        return set_err(GR_CUDA_ERROR, cudaGetErrorString(ce));
    }
    *out = b;
    return ok();
}

void gr_fa2_batch_destroy(gr_fa2_batch *b) { delete b; }

int gr_fa2_batch_set_threads(gr_fa2_batch *b, int threads) {
    if (!b) return set_err(GR_INVALID_HANDLE, "null batch");
    if (threads != 256 && threads != 512 && threads != 1024)
        return set_err(GR_INVALID_ARGUMENT, "threads per CTA must be 256, 512 or 1024");
    b->threads = threads;
    return ok();
}

int gr_fa2_batch_run(gr_fa2_batch *b, uint32_t ticks, float *ms) {
    if (!b) return set_err(GR_INVALID_HANDLE, "null batch");
    if (ticks == 0) return ok();
    if (int c = batch_run_impl(b, ticks, ms)) return c;
    return ok();
}

int gr_fa2_batch_tune(gr_fa2_batch *b, uint32_t sample_ticks, int *chosen, float *ms_each) {
    if (!b) return set_err(GR_INVALID_HANDLE, "null batch");
    if (sample_ticks == 0) sample_ticks = 1;
    // time each CTA size on a copy of the state, then put the state back
    const size_t pb = (size_t)b->total_n * sizeof(float4), sb = (size_t)b->ngraphs * sizeof(BatchState);
    void *save_p = nullptr, *save_s = nullptr;
    CU(cudaMalloc(&save_p, std::max<size_t>(pb, 16)));
    CU(cudaMalloc(&save_s, sb));
    CU(cudaMemcpy(save_p, b->g->pos, pb, cudaMemcpyDeviceToDevice));
    CU(cudaMemcpy(save_s, b->d_state, sb, cudaMemcpyDeviceToDevice));
    const int cands[3] = {256, 512, 1024};
    float best = 1e30f;
    int pick = b->threads, rc = GR_OK;
    for (int i = 0; i < 3 && rc == GR_OK; i++) {
        b->threads = cands[i];
        float ms = 0.f;
        rc = batch_run_impl(b, sample_ticks, &ms);
        if (ms_each) ms_each[i] = ms;
        if (rc == GR_OK && ms < best) {
            best = ms;
            pick = cands[i];
        }
        cudaMemcpy(b->g->pos, save_p, pb, cudaMemcpyDeviceToDevice);
        cudaMemcpy(b->d_state, save_s, sb, cudaMemcpyDeviceToDevice);
    }
    cudaFree(save_p);
    cudaFree(save_s);
    b->drop_graph();
    b->threads = pick;
    if (chosen) *chosen = pick;
    if (rc) return rc;
    CU(cudaDeviceSynchronize());
    return ok();
}

int gr_fa2_batch_positions(gr_fa2_batch *b, float *out) {
    if (!b) return set_err(GR_INVALID_HANDLE, "null batch");
    return gr_fa2_positions(b->g, out);
}

int gr_fa2_batch_stats(gr_fa2_batch *b, uint32_t *ticks_done, uint32_t *errors, uint64_t *interactions) {
    if (!b) return set_err(GR_INVALID_HANDLE, "null batch");
    std::vector<BatchState> st(b->ngraphs);
    CU(cudaMemcpy(st.data(), b->d_state, st.size() * sizeof(BatchState), cudaMemcpyDeviceToHost));
    for (uint32_t g = 0; g < b->ngraphs; g++) {
        if (ticks_done) ticks_done[g] = st[g].iter_no;
        if (errors) errors[g] = st[g].error;
        if (interactions) {
            interactions[2 * g] = st[g].far_count;
            interactions[2 * g + 1] = st[g].pair_count;
        }
    }
    return ok();
}

}  // extern "C"

// ---------------------------------------------------------------- adjoint --
//
// gr_fa2_adjoint_forward records a run (positions and controller every K
// ticks); gr_fa2_adjoint_backward replays each K-tick segment forward from its
// checkpoint, keeping every tick's state, then runs the adjoint kernels
// (adjoint.cuh) tick by tick in reverse. The replay uses the same kernels on the
// same inputs, so each tick's tree is the one the recorded run built.

struct Adjoint {
    uint32_t ticks = 0, every = 1, done = 0;
    float4 *ckpt = nullptr;  // (ticks / every + 1) x n node records
    DevState *ckst = nullptr;
    float4 *segp = nullptr;  // every x n
    DevState *segst = nullptr;
    float4 *final_pos = nullptr;
    DevState *final_st = nullptr;
    float *lam1 = nullptr, *lam = nullptr, *ub = nullptr, *v = nullptr, *lam_rep = nullptr, *lam_com = nullptr;
    double *lam_pair = nullptr, *xbar = nullptr, *gce = nullptr, *gs = nullptr, *graw = nullptr, *part = nullptr;
    AdjScalars *A = nullptr;
    DevState *before = nullptr;  // the state before the tick the captured adjoint tick differentiates
    std::vector<void *> allocs;
    template <typename T>
    cudaError_t alloc(T **p, size_t count) {
        cudaError_t e = cudaMalloc((void **)p, (count ? count : 1) * sizeof(T));
        if (e == cudaSuccess) allocs.push_back((void *)*p);
        return e;
    }
};

static void adjoint_release(Adjoint *a) {
    for (void *p : a->allocs) cudaFree(p);
    delete a;
}

template <int D>
static void adjoint_tick(gr_fa2 *h, Adjoint *a, const DevState *before) {
    const uint32_t n = h->n;
    cudaStream_t s = h->stream;
    DevState *st = h->st;
    // bring max |lam'| into [0.5, 1) by a power of two (k_adj_shift)
    const uint32_t rb = std::min<uint32_t>(div_up((uint64_t)n * D, 256), 4 * 148);
    k_adj_absmax<<<rb, 256, 0, s>>>(n * D, a->lam1, a->A);
    k_adj_shift<<<1, 1, 0, s>>>(a->A);
    k_adj_rescale<<<rb, 256, 0, s>>>(n * D, a->lam1, 2 * h->m, a->gce, a->A);
    // forward recompute up to the forces, with the controller update (no move)
    enqueue_tick<D>(h, false, PH_TREE | PH_WALK);
    ForceParams fp;
    fp.n = n;
    fp.gravity = (float)h->prm[P_GRAVITY];
    fp.lin_log = (int)h->prm[P_LINLOG];
    fp.strong_gravity = (int)h->prm[P_STRONG];
    fp.dissuade_hubs = (int)h->prm[P_DISSUADE];
    fp.jitter_tolerance = h->prm[P_JT];
    if (h->nseg)
        k_attract_seg<D><<<div_up((uint64_t)h->nseg * GR_WARP, FRC_THREADS), FRC_THREADS, 0, s>>>(
            h->nseg, fp.lin_log, st, h->pos, h->rp, h->col, h->wt, h->seg_row, h->seg_first, h->seg_out);
    k_attract<D><<<div_up(n, FRC_THREADS), FRC_THREADS, 0, s>>>(n, fp.lin_log, st, h->pos, h->rp, h->col, h->wt,
                                                                 h->nseg ? h->seg_first : nullptr, h->seg_out, h->U);
    k_forces<D><<<frc_blocks(n), FRC_THREADS, 0, s>>>(fp, st, h->pos, h->rep, h->U, h->part, 1);
    const uint32_t gb = div_up(n, FRC_THREADS);
    k_adj_update<D><<<gb, FRC_THREADS, 0, s>>>(n, h->prm[P_JT], st, before, a->A, h->pos, h->U, a->lam1, a->lam, a->ub,
                                                a->part);
    k_adj_node<D><<<gb, FRC_THREADS, 0, s>>>(n, (float)h->prm[P_GRAVITY], (int)h->prm[P_STRONG], st, a->A, h->pos,
                                              h->U, a->lam, a->ub, a->v, a->part);
    cudaMemsetAsync(a->xbar, 0, 2 * (size_t)n * D * sizeof(double), s);
    cudaMemsetAsync(a->lam_pair, 0, (size_t)n * D * sizeof(double), s);
    WalkParams wp;
    wp.n = n;
    wp.kr = (float)h->prm[P_SCALING];
    wp.theta2 = (float)(h->prm[P_THETA] * h->prm[P_THETA]);
    wp.seed = (uint32_t)h->prm[P_SEED];
    k_adj_walk<D><<<div_up(n, WALK_THREADS), WALK_THREADS, 0, s>>>(wp, st, h->cells, h->sp, h->sorig, h->uid,
                                                                    h->leaf_pre, a->ub, a->lam_rep, a->xbar,
                                                                    a->lam_pair);
    k_adj_down<D><<<div_up(n, 256), 256, 0, s>>>(st, h->bt, h->leaf_start, h->leaf_pre, h->leaf_body, h->int_body,
                                                  h->sp, h->sorig, a->xbar, a->lam_pair, a->lam_com);
    k_adj_final<D><<<gb, FRC_THREADS, 0, s>>>(n, fp.lin_log, fp.dissuade_hubs, a->A, h->pos, h->rp, h->col, h->wt,
                                               a->lam, a->ub, a->v, a->lam_rep, a->lam_com, a->gce, a->lam1);
}

// The adjoint tick captured once into a graph (its per-tick input, the state
// before the tick, read from a->before); retried in plain stream order if the
// capture with programmatic launches fails.
static int capture_adjoint(gr_fa2 *h, Adjoint *a, cudaGraph_t *g, cudaGraphExec_t *x) {
    for (;;) {
        *g = nullptr;
        *x = nullptr;
        cudaError_t e = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            if (h->dim == 3)
                adjoint_tick<3>(h, a, a->before);
            else
                adjoint_tick<2>(h, a, a->before);
            e = cudaStreamEndCapture(h->stream, g);
            if (e == cudaSuccess) e = cudaGraphInstantiate(x, *g, 0);
        }
        if (e == cudaSuccess) return GR_OK;
        cudaGetLastError();
        if (*x) cudaGraphExecDestroy(*x);
        if (*g) cudaGraphDestroy(*g);
        *g = nullptr;
        *x = nullptr;
        if (!h->pdl) return set_err(GR_CUDA_ERROR, cudaGetErrorString(e));
        h->pdl = false;
        h->pdl_fell_back = true;
    }
}

// Destroys a captured graph when the scope ends.
struct GraphGuard {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t x = nullptr;
    ~GraphGuard() {
        if (x) cudaGraphExecDestroy(x);
        if (g) cudaGraphDestroy(g);
    }
};

extern "C" {

int gr_fa2_adjoint_forward(gr_fa2 *h, uint32_t ticks, uint32_t every) {
    if (!h) return set_err(GR_INVALID_HANDLE, "null handle");
    if (every == 0) return set_err(GR_INVALID_ARGUMENT, "checkpoint interval must be >= 1");
    if (h->adj) {
        adjoint_release(h->adj);
        h->adj = nullptr;
    }
    const uint32_t n = h->n;
    const int D = h->dim;
    Adjoint *a = new (std::nothrow) Adjoint();
    if (!a) return set_err(GR_ALLOC_FAILED, "host allocation failed");
    a->ticks = ticks;
    a->every = every;
    const uint32_t nck = ticks / every + 1;
    const uint64_t ne = 2 * h->m;
    cudaError_t e;
    if ((e = a->alloc(&a->ckpt, (size_t)nck * n)) || (e = a->alloc(&a->ckst, nck)) ||
        (e = a->alloc(&a->segp, (size_t)every * n)) || (e = a->alloc(&a->segst, every)) ||
        (e = a->alloc(&a->final_pos, n)) || (e = a->alloc(&a->final_st, 1)) ||
        (e = a->alloc(&a->lam1, (size_t)n * D)) || (e = a->alloc(&a->lam, (size_t)n * D)) ||
        (e = a->alloc(&a->ub, (size_t)n * D)) || (e = a->alloc(&a->v, (size_t)n * D)) ||
        (e = a->alloc(&a->lam_rep, (size_t)n * D)) || (e = a->alloc(&a->lam_com, (size_t)n * D)) ||
        (e = a->alloc(&a->lam_pair, (size_t)n * D)) || (e = a->alloc(&a->xbar, 2 * (size_t)n * D)) ||
        (e = a->alloc(&a->gce, ne)) || (e = a->alloc(&a->gs, h->m)) || (e = a->alloc(&a->graw, h->m_raw)) ||
        (e = a->alloc(&a->part, 3 * (size_t)div_up(n, FRC_THREADS) + 8)) || (e = a->alloc(&a->A, 1)) ||
        (e = a->alloc(&a->before, 1))) {
        adjoint_release(a);
        return set_err(GR_ALLOC_FAILED, cudaGetErrorString(e));
    }
    if (!h->bt.cell_of) {
        if ((e = h->alloc(&h->bt.cell_of, n))) {
            adjoint_release(a);
            return set_err(GR_ALLOC_FAILED, cudaGetErrorString(e));
        }
        h->drop_graphs();  // the captured tick now also records each cell's node
    }
    h->adj = a;
    DevState s0;
    if (int c = read_state(h, &s0)) return c;
    if (n && ticks) {
        if (int c = build_graph(h)) return c;
        for (uint32_t t = 0; t < ticks; t++) {
            if (t % every == 0) {
                CU(cudaMemcpyAsync(a->ckpt + (size_t)(t / every) * n, h->pos, (size_t)n * sizeof(float4),
                                   cudaMemcpyDeviceToDevice, h->stream));
                CU(cudaMemcpyAsync(a->ckst + t / every, h->st, sizeof(DevState), cudaMemcpyDeviceToDevice, h->stream));
            }
            CU(cudaGraphLaunch(h->exec, h->stream));
        }
    }
    CU(cudaMemcpyAsync(a->final_pos, h->pos, (size_t)std::max(n, 1u) * sizeof(float4), cudaMemcpyDeviceToDevice,
                       h->stream));
    CU(cudaMemcpyAsync(a->final_st, h->st, sizeof(DevState), cudaMemcpyDeviceToDevice, h->stream));
    DevState s1;
    if (int c = read_state(h, &s1)) return c;
    a->done = s1.iter_no - s0.iter_no;
    if (int c = check_device(h, s1)) return c;
    return ok();
}

int gr_fa2_adjoint_backward(gr_fa2 *h, const float *dL_dpT, double *dL_dp0, double *dL_dw) {
    if (!h) return set_err(GR_INVALID_HANDLE, "null handle");
    Adjoint *a = h->adj;
    if (!a) return set_err(GR_INVALID_ARGUMENT, "no recorded run: call gr_fa2_adjoint_forward first");
    if (!dL_dpT || !dL_dp0) return set_err(GR_INVALID_ARGUMENT, "gradient buffers are null");
    const uint32_t n = h->n;
    const int D = h->dim;
    cudaStream_t s = h->stream;
    CU(cudaMemcpyAsync(a->lam1, dL_dpT, (size_t)n * D * 4, cudaMemcpyHostToDevice, s));
    CU(cudaMemsetAsync(a->A, 0, sizeof(AdjScalars), s));
    CU(cudaMemsetAsync(a->gce, 0, std::max<uint64_t>(2 * h->m, 1) * sizeof(double), s));
    GraphGuard adj;  // the adjoint tick, captured once per call
    if (n && a->done) {
        if (int c = build_graph(h)) return c;  // the replay runs the recorded run's own tick graph
        if (int c = capture_adjoint(h, a, &adj.g, &adj.x)) return c;
        const uint32_t nseg = (a->done + a->every - 1) / a->every;
        for (uint32_t g = nseg; g-- > 0;) {
            const uint32_t t0 = g * a->every, t1 = std::min(t0 + a->every, a->done);
            CU(cudaMemcpyAsync(h->pos, a->ckpt + (size_t)g * n, (size_t)n * sizeof(float4), cudaMemcpyDeviceToDevice, s));
            CU(cudaMemcpyAsync(h->st, a->ckst + g, sizeof(DevState), cudaMemcpyDeviceToDevice, s));
            for (uint32_t t = t0; t < t1; t++) {  // replay, keeping each tick's state
                CU(cudaMemcpyAsync(a->segp + (size_t)(t - t0) * n, h->pos, (size_t)n * sizeof(float4),
                                   cudaMemcpyDeviceToDevice, s));
                CU(cudaMemcpyAsync(a->segst + (t - t0), h->st, sizeof(DevState), cudaMemcpyDeviceToDevice, s));
                CU(cudaGraphLaunch(h->exec, s));
            }
            for (uint32_t t = t1; t-- > t0;) {
                CU(cudaMemcpyAsync(h->pos, a->segp + (size_t)(t - t0) * n, (size_t)n * sizeof(float4),
                                   cudaMemcpyDeviceToDevice, s));
                CU(cudaMemcpyAsync(h->st, a->segst + (t - t0), sizeof(DevState), cudaMemcpyDeviceToDevice, s));
                CU(cudaMemcpyAsync(a->before, a->segst + (t - t0), sizeof(DevState), cudaMemcpyDeviceToDevice, s));
                CU(cudaGraphLaunch(adj.x, s));
            }
        }
    }
    CU(cudaGetLastError());
    std::vector<float> lam0((size_t)n * D);
    AdjScalars Ah;
    if (n) CU(cudaMemcpyAsync(lam0.data(), a->lam1, (size_t)n * D * 4, cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(&Ah, a->A, sizeof(AdjScalars), cudaMemcpyDeviceToHost, s));
    if (dL_dw && h->m_raw) {
        CU(cudaMemsetAsync(a->gs, 0, std::max<uint64_t>(h->m, 1) * sizeof(double), s));
        CU(cudaMemsetAsync(a->graw, 0, h->m_raw * sizeof(double), s));
        if (h->m) {
            k_adj_edges<<<div_up(2 * h->m, 256), 256, 0, s>>>((uint32_t)(2 * h->m), h->csr_simple, a->gce, a->gs);
            k_adj_raw<<<div_up(h->m, 256), 256, 0, s>>>((uint32_t)h->m, a->gs, h->simple_raw, h->simple_dcdw, a->graw);
        }
        CU(cudaMemcpyAsync(dL_dw, a->graw, h->m_raw * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    // the handle goes back to the end of the recorded run
    CU(cudaMemcpyAsync(h->pos, a->final_pos, (size_t)std::max(n, 1u) * sizeof(float4), cudaMemcpyDeviceToDevice, s));
    CU(cudaMemcpyAsync(h->st, a->final_st, sizeof(DevState), cudaMemcpyDeviceToDevice, s));
    CU(cudaStreamSynchronize(s));
    // undo the running power-of-two scale (k_adj_shift); beyond FP64's range is non-finite
    const int ex = (int)std::max<long long>(-4096, std::min<long long>(4096, Ah.exponent));
    for (size_t i = 0; i < (size_t)n * D; i++) {
        dL_dp0[i] = std::ldexp((double)lam0[i], ex);
        if (!std::isfinite(dL_dp0[i])) return set_err(GR_LAYOUT_FAILED, "non-finite gradient");
    }
    if (dL_dw)
        for (uint64_t e = 0; e < h->m_raw; e++) {
            dL_dw[e] = std::ldexp(dL_dw[e], ex);
            if (!std::isfinite(dL_dw[e])) return set_err(GR_LAYOUT_FAILED, "non-finite gradient");
        }
    return ok();
}

}  // extern "C"

// ------------------------------------------------------------ stress / BFS --
//
// Multi-source BFS and Kruskal stress-1 on the device (stress.cuh). The
// adjacency of the raw edges (both directions, self-loops dropped) is counted
// and filled on the host, O(m), and copied once per call.

namespace {

struct DevBufs {  // device allocations released on every return path
    std::vector<void *> p;
    template <typename T>
    cudaError_t get(T **out, size_t count) {
        cudaError_t e = cudaMalloc((void **)out, (count ? count : 1) * sizeof(T));
        if (e == cudaSuccess) p.push_back((void *)*out);
        return e;
    }
    ~DevBufs() {
        for (void *q : p) cudaFree(q);
    }
};

struct StreamGuard {
    cudaStream_t s = nullptr;
    ~StreamGuard() {
        if (s) cudaStreamDestroy(s);
    }
};

constexpr uint64_t kMaxHopTableBytes = 16ull << 30;

// Hop counts from the k sources (device) to every node into hops (device, k x n,
// HOP_NONE when unreachable), 64 sources per level-synchronous pull.
int bfs_on_device(uint32_t n, uint64_t m, const uint32_t *src, const uint32_t *dst, uint32_t k,
                  const uint32_t *sources_dev, uint32_t *hops, cudaStream_t s, DevBufs &B) {
    std::vector<uint64_t> rp((size_t)n + 1, 0);
    for (uint64_t e = 0; e < m; e++) {
        if (src[e] >= n || dst[e] >= n) return set_err(GR_INDEX_OUT_OF_RANGE, "edge endpoint out of range", (int)e);
        if (src[e] == dst[e]) continue;
        rp[src[e] + 1]++;
        rp[dst[e] + 1]++;
    }
    for (uint32_t i = 0; i < n; i++) rp[i + 1] += rp[i];
    std::vector<uint32_t> col(std::max<uint64_t>(rp[n], 1));
    std::vector<uint64_t> fill(rp.begin(), rp.end() - 1);
    for (uint64_t e = 0; e < m; e++) {
        if (src[e] == dst[e]) continue;
        col[fill[src[e]]++] = dst[e];
        col[fill[dst[e]]++] = src[e];
    }
    uint64_t *d_rp;
    uint32_t *d_col, *d_changed;
    unsigned long long *vis, *fa, *fb;
    cudaError_t e;
    if ((e = B.get(&d_rp, (size_t)n + 1)) || (e = B.get(&d_col, col.size())) || (e = B.get(&d_changed, 1)) ||
        (e = B.get(&vis, n)) || (e = B.get(&fa, n)) || (e = B.get(&fb, n)))
        return set_err(GR_ALLOC_FAILED, cudaGetErrorString(e));
    CU(cudaMemcpyAsync(d_rp, rp.data(), rp.size() * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(d_col, col.data(), col.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    CU(cudaMemsetAsync(hops, 0xff, (size_t)k * n * sizeof(uint32_t), s));
    const uint32_t grid = div_up(n, BFS_T);
    for (uint32_t k0 = 0; k0 < k; k0 += 64) {
        const uint32_t kb = std::min<uint32_t>(64, k - k0);
        const unsigned long long all = kb == 64 ? ~0ull : ((1ull << kb) - 1ull);
        CU(cudaMemsetAsync(vis, 0, (size_t)n * 8, s));
        CU(cudaMemsetAsync(fa, 0, (size_t)n * 8, s));
        k_msbfs_seed<<<1, 64, 0, s>>>(n, k0, kb, sources_dev, vis, fa, hops);
        unsigned long long *cur = fa, *nxt = fb;
        for (uint32_t level = 1; level < n; level++) {  // a BFS is at most n - 1 levels deep
            uint32_t changed = 0;
            CU(cudaMemsetAsync(d_changed, 0, 4, s));
            k_msbfs_level<<<grid, BFS_T, 0, s>>>(n, d_rp, d_col, all, cur, vis, nxt, hops, k0, level, d_changed);
            CU(cudaMemcpyAsync(&changed, d_changed, 4, cudaMemcpyDeviceToHost, s));
            CU(cudaStreamSynchronize(s));
            if (!changed) break;
            std::swap(cur, nxt);
        }
    }
    CU(cudaGetLastError());
    return GR_OK;
}

}  // namespace

extern "C" {

int gr_bfs_hops(uint32_t n, uint64_t m, const uint32_t *source, const uint32_t *target, uint32_t k,
                const uint32_t *sources, uint32_t *hops_out) {
    if ((m && (!source || !target)) || (k && (!sources || !hops_out)))
        return set_err(GR_INVALID_ARGUMENT, "null buffer");
    if ((uint64_t)k * n * 4 > kMaxHopTableBytes) return set_err(GR_INVALID_ARGUMENT, "hop table above 16 GiB");
    for (uint32_t i = 0; i < k; i++)
        if (sources[i] >= n) return set_err(GR_INDEX_OUT_OF_RANGE, "source out of range", (int)i);
    if (k == 0 || n == 0) return ok();
    DevBufs B;
    StreamGuard g;
    CU(cudaStreamCreateWithFlags(&g.s, cudaStreamNonBlocking));
    uint32_t *d_src, *hops;
    cudaError_t e;
    if ((e = B.get(&d_src, k)) || (e = B.get(&hops, (size_t)k * n))) return set_err(GR_ALLOC_FAILED, cudaGetErrorString(e));
    CU(cudaMemcpyAsync(d_src, sources, (size_t)k * 4, cudaMemcpyHostToDevice, g.s));
    if (int c = bfs_on_device(n, m, source, target, k, d_src, hops, g.s, B)) return c;
    CU(cudaMemcpyAsync(hops_out, hops, (size_t)k * n * 4, cudaMemcpyDeviceToHost, g.s));
    CU(cudaStreamSynchronize(g.s));
    return ok();
}

}  // extern "C"

// Eight independent FMA chains per thread, so the FMA pipe, not a chain's
// latency, sets the rate. `sink` is written only if the sum is exactly -1,
// which these positive values never reach: it keeps the chains live.
__global__ void __launch_bounds__(256) k_fma_rate(uint32_t iters, float *sink) {
    float a[8];
#pragma unroll
    for (int j = 0; j < 8; j++) a[j] = 1.0f + 1e-7f * (float)(threadIdx.x + j);
    const float b = 0.9999999f, c = 1e-7f;
    for (uint32_t i = 0; i < iters; i++) {
#pragma unroll
        for (int j = 0; j < 8; j++) a[j] = fmaf(a[j], b, c);
    }
    float t = 0.f;
#pragma unroll
    for (int j = 0; j < 8; j++) t += a[j];
    if (t == -1.0f) sink[0] = t;
}

extern "C" {

int gr_measure_fp32_rate(uint32_t iters, double *tflops) {
    if (!tflops) return set_err(GR_INVALID_ARGUMENT, "tflops is null");
    if (iters == 0) return set_err(GR_INVALID_ARGUMENT, "iters must be > 0");
    int dev = 0, sms = 0;
    CU(cudaGetDevice(&dev));
    CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const uint32_t blocks = (uint32_t)sms * 8;  // 64 resident warps a SM
    float *sink = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaMalloc((void **)&sink, sizeof(float));
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    float ms = 0.f;
    if (e == cudaSuccess) {
        k_fma_rate<<<blocks, 256>>>(iters, sink);  // warm-up
        cudaEventRecord(e0);
        k_fma_rate<<<blocks, 256>>>(iters, sink);
        cudaEventRecord(e1);
        e = cudaEventSynchronize(e1);
    }
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (sink) cudaFree(sink);
    if (e != cudaSuccess) return set_err(GR_CUDA_ERROR, cudaGetErrorString(e));
    const double flops = (double)blocks * 256.0 * (double)iters * 8.0 * 2.0;  // an FMA counted as 2
    *tflops = flops / (ms * 1e-3) / 1e12;
    return ok();
}

int gr_stress(uint32_t n, uint64_t m, const uint32_t *source, const uint32_t *target, const float *x, const float *y,
              uint32_t sources, double *out) {
    if (!out || (m && (!source || !target)) || (n && (!x || !y))) return set_err(GR_INVALID_ARGUMENT, "null buffer");
    if (sources == 0) return set_err(GR_INVALID_ARGUMENT, "sources must be >= 1");
    *out = 1.0;
    if (n == 0) return ok();
    // the reference's sources: every max(n / sources, 1)-th node from 0 (bench.rs:266)
    const uint32_t step = std::max<uint32_t>(n / sources, 1u);
    std::vector<uint32_t> from;
    for (uint64_t v = 0; v < n; v += step) from.push_back((uint32_t)v);
    const uint32_t k = (uint32_t)from.size();
    if ((uint64_t)k * n * 4 > kMaxHopTableBytes) return set_err(GR_INVALID_ARGUMENT, "hop table above 16 GiB");
    DevBufs B;
    StreamGuard g;
    CU(cudaStreamCreateWithFlags(&g.s, cudaStreamNonBlocking));
    uint32_t *d_src, *hops, *ticket;
    float *dx, *dy;
    double *part, *d_out;
    const uint32_t G = 4 * 148;
    cudaError_t e;
    if ((e = B.get(&d_src, k)) || (e = B.get(&hops, (size_t)k * n)) || (e = B.get(&dx, n)) || (e = B.get(&dy, n)) ||
        (e = B.get(&part, 3 * (size_t)G)) || (e = B.get(&d_out, 3)) || (e = B.get(&ticket, 1)))
        return set_err(GR_ALLOC_FAILED, cudaGetErrorString(e));
    CU(cudaMemcpyAsync(d_src, from.data(), (size_t)k * 4, cudaMemcpyHostToDevice, g.s));
    CU(cudaMemcpyAsync(dx, x, (size_t)n * 4, cudaMemcpyHostToDevice, g.s));
    CU(cudaMemcpyAsync(dy, y, (size_t)n * 4, cudaMemcpyHostToDevice, g.s));
    CU(cudaMemsetAsync(ticket, 0, 4, g.s));
    if (int c = bfs_on_device(n, m, source, target, k, d_src, hops, g.s, B)) return c;
    k_stress_sums<<<G, STRESS_T, 0, g.s>>>(n, k, d_src, hops, dx, dy, part, d_out, ticket);
    double sums[3];
    CU(cudaMemcpyAsync(sums, d_out, sizeof sums, cudaMemcpyDeviceToHost, g.s));
    CU(cudaStreamSynchronize(g.s));
    const double de = sums[0], ee = sums[1], dd = sums[2];
    if (ee == 0.0 || dd == 0.0) return ok();
    *out = std::sqrt(std::max((dd - de / ee * de) / dd, 0.0));
    return ok();
}

}  // extern "C"

// ---------------------------------------------------- d3-force session ----
//
// A d3-force Barnes-Hut session (d3force.cuh) over an internal FA2 handle that
// holds the simple graph (CSR, edge strengths as weights, heavy-row segments),
// the stream and the tree buffers; every tick is one captured CUDA graph that
// builds the tree twice (positions for many-body, projected positions for
// collide).

struct gr_force_session {
    gr_fa2 *t = nullptr;
    uint32_t n = 0;
    gr_force_params prm{};
    D3Params P{};
    float4 *p4 = nullptr, *pp4 = nullptr, *bounds = nullptr;
    float2 *vel = nullptr, *seg_out = nullptr;
    D3State *ds = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint32_t graph_kernels = 0;
    // particle mesh (many-body on an FFT mesh instead of the tree)
    bool mesh = false;
    uint32_t side = 0, bits = 0, pm_blocks = 0;
    PmState *pm = nullptr;
    double *pm_part = nullptr;
    uint64_t *pm_key = nullptr;
    uint32_t *pm_val = nullptr, *pm_cs = nullptr, *pm_ce = nullptr;
    float2 *pm_frac = nullptr, *ga = nullptr, *gk = nullptr, *gt = nullptr, *tw = nullptr;
    RadixSorter pm_sorter;
    ~gr_force_session() {
        pm_sorter.release();
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (t) {
            if (t->stream) cudaStreamSynchronize(t->stream);
            delete t;  // also frees the session's buffers (allocated through t)
        }
    }
};

namespace {

int d3_validate(const gr_force_params &p) {
    const double v[] = {p.charge, p.theta, p.distance_min, p.distance_max, p.link_distance, p.link_strength_scale,
                        p.collide_radius, p.center_strength, p.velocity_decay, p.alpha_decay, p.alpha_min,
                        p.initial_alpha};
    for (size_t i = 0; i < sizeof v / sizeof v[0]; i++)
        if (!std::isfinite(v[i])) return set_err(GR_PARAM_OUT_OF_RANGE, "force parameter not finite", (int)i);
    if (p.theta < 0.0) return set_err(GR_PARAM_OUT_OF_RANGE, "theta must be >= 0", 1);
    if (p.distance_min < 0.0 || p.distance_max < 0.0)
        return set_err(GR_PARAM_OUT_OF_RANGE, "distances must be >= 0", 2);
    if (p.initial_alpha < 0.0 || p.initial_alpha > 1.0)
        return set_err(GR_PARAM_OUT_OF_RANGE, "initial alpha must be in [0, 1]", 11);
    return GR_OK;
}

// The mesh's many-body pass (pm.cuh): frame, stencils, cell sort, deposit,
// Green's function, forward FFTs (spectra transposed), product, inverse FFT
// (natural layout), bilinear read onto the velocities.
void pm_fft2(gr_force_session *S, float2 *a, float2 *scratch, bool inverse, cudaStream_t s) {
    const uint32_t side = S->side, th = std::min<uint32_t>(side / 2, 512);
    const size_t sm = (size_t)side * sizeof(float2);
    const dim3 tg(side / 32, side / 32), tb(32, 8);
    if (inverse) {
        k_pm_fft_rows<true><<<side, th, sm, s>>>(a, S->tw, side, S->bits, S->pm);
        k_pm_transpose<<<tg, tb, 0, s>>>(a, scratch, side, S->pm);
        k_pm_fft_rows<true><<<side, th, sm, s>>>(scratch, S->tw, side, S->bits, S->pm);
    } else {
        k_pm_fft_rows<false><<<side, th, sm, s>>>(a, S->tw, side, S->bits, S->pm);
        k_pm_transpose<<<tg, tb, 0, s>>>(a, scratch, side, S->pm);
        k_pm_fft_rows<false><<<side, th, sm, s>>>(scratch, S->tw, side, S->bits, S->pm);
    }
}

void pm_enqueue(gr_force_session *S) {
    cudaStream_t s = S->t->stream;
    const uint32_t n = S->n, side = S->side, g = div_up(n, PM_T);
    const uint32_t mg = div_up(side * side, PM_T);
    const double dmin2 = S->prm.distance_min * S->prm.distance_min;
    const double dmax2 = S->prm.distance_max * S->prm.distance_max;
    k_pm_bounds<<<S->pm_blocks, PM_T, 0, s>>>(n, S->p4, side, S->prm.distance_max, dmax2, S->pm_part, S->pm);
    k_pm_stencil<<<g, PM_T, 0, s>>>(n, S->p4, S->pm, side, S->pm_key, S->pm_val, S->pm_frac);
    // cell keys are row-major indices below side^2: 2 x bits significant bits, one-sweep
    // passes (a wait that gives up is reported through the tree handle's state)
    S->pm_sorter.sort_bits(S->pm_key, S->pm_val, n, 2 * (int)S->bits, s, &S->t->st->error);
    cudaMemsetAsync(S->pm_cs, 0, (size_t)side * side * 4, s);
    cudaMemsetAsync(S->pm_ce, 0, (size_t)side * side * 4, s);
    k_pm_mark<<<g, PM_T, 0, s>>>(n, S->pm, S->pm_key, S->pm_cs, S->pm_ce);
    k_pm_deposit<<<mg, PM_T, 0, s>>>(side, S->pm, S->pm_cs, S->pm_ce, S->pm_val, S->pm_frac, S->ga);
    k_pm_green<<<mg, PM_T, 0, s>>>(side, S->pm, dmin2, dmax2, S->gk);
    pm_fft2(S, S->gk, S->gt, false, s);  // kernel spectrum, transposed, in gt
    pm_fft2(S, S->ga, S->gk, false, s);  // density spectrum, transposed, in gk
    k_pm_mul<<<mg, PM_T, 0, s>>>(side * side, S->gk, S->gt, S->pm);
    pm_fft2(S, S->gk, S->ga, true, s);   // field, natural layout, in ga
    k_pm_read<<<g, PM_T, 0, s>>>(n, S->p4, S->pm, side, (float)S->prm.charge, &S->ds->alpha, S->ga, S->vel);
}

void d3_enqueue(gr_force_session *S) {
    gr_fa2 *t = S->t;
    cudaStream_t s = t->stream;
    const uint32_t n = S->n, g = div_up(n, D3_T);
    k_d3_alpha<<<1, 1, 0, s>>>(S->ds, S->prm.alpha_decay);
    k_d3_project<<<g, D3_T, 0, s>>>(n, S->p4, S->vel, S->pp4);
    if (t->nseg)
        k_d3_link_seg<<<div_up((uint64_t)t->nseg * GR_WARP, D3_T), D3_T, 0, s>>>(
            S->P, t->nseg, S->ds, S->pp4, t->rp, t->col, t->wt, t->seg_row, t->seg_first, S->seg_out);
    k_d3_link<<<g, D3_T, 0, s>>>(S->P, S->ds, S->pp4, t->rp, t->col, t->wt, t->nseg ? t->seg_first : nullptr,
                                 S->seg_out, S->vel);
    if (S->mesh) {  // many-body on the particle mesh
        pm_enqueue(S);
        k_d3_center<<<g, D3_T, 0, s>>>(n, (float)S->prm.center_strength, S->pm->mean, S->p4);
    } else {  // many-body: the tree of the positions
        t->pos = S->p4;
        enqueue_tick<2>(t, false, PH_TREE);
        k_d3_charge<<<g, D3_T, 0, s>>>(S->P, S->ds, t->st, t->cells, t->sp, t->sorig, S->vel);
        k_d3_center<<<g, D3_T, 0, s>>>(n, (float)S->prm.center_strength, t->st->mean, S->p4);
    }
    k_d3_project<<<g, D3_T, 0, s>>>(n, S->p4, S->vel, S->pp4);
    t->pos = S->pp4;  // collide: the tree of the projected positions, with cell squares
    t->cells.bounds = S->bounds;
    enqueue_tick<2>(t, false, PH_TREE);
    Cells cb = t->cells;
    t->cells.bounds = nullptr;
    t->pos = S->p4;
    k_d3_collide<<<g, D3_T, 0, s>>>(S->P, S->ds, t->st, cb, t->sp, t->sorig, S->vel);
    k_d3_integrate<<<g, D3_T, 0, s>>>(n, (float)S->prm.velocity_decay, S->p4, S->vel);
    k_d3_end<<<1, 1, 0, s>>>(S->ds);
}

int d3_build_graph(gr_force_session *S) {
    if (S->exec) return GR_OK;
    cudaStream_t s = S->t->stream;
    CU(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    d3_enqueue(S);
    cudaGraph_t g = nullptr;
    CU(cudaStreamEndCapture(s, &g));
    S->graph = g;
    size_t count = 0;
    CU(cudaGraphGetNodes(g, nullptr, &count));
    std::vector<cudaGraphNode_t> nodes(count);
    CU(cudaGraphGetNodes(g, nodes.data(), &count));
    S->graph_kernels = 0;
    for (auto nd : nodes) {
        cudaGraphNodeType ty;
        CU(cudaGraphNodeGetType(nd, &ty));
        if (ty == cudaGraphNodeTypeKernel) S->graph_kernels++;
    }
    CU(cudaGraphInstantiate(&S->exec, g, 0));
    return GR_OK;
}

}  // namespace

extern "C" {

void gr_force_default_params(gr_force_params *p) {
    if (!p) return;
    // crates/graph-core/src/layout/force/params.rs:60-75
    p->charge = -90.0;
    p->theta = 0.9;
    p->distance_min = 1.0;
    p->distance_max = 520.0;
    p->link_distance = 60.0;
    p->link_strength_scale = 0.15;
    p->collide_radius = 16.0;
    p->center_strength = 1.0;
    p->velocity_decay = 1.0 - 0.42;
    p->alpha_decay = 0.06;
    p->alpha_min = 0.001;
    p->initial_alpha = 1.0;
}

int gr_force_session_create(gr_force_session **out, uint32_t n, uint64_t m, const uint32_t *src, const uint32_t *dst,
                            const double *strength, const gr_force_params *params, const float *pos0) {
    if (!out) return set_err(GR_INVALID_ARGUMENT, "out is null");
    *out = nullptr;
    gr_force_params prm;
    gr_force_default_params(&prm);
    if (params) prm = *params;
    if (int c = d3_validate(prm)) return c;
    if (pos0)
        for (size_t i = 0; i < 2 * (size_t)n; i++)
            if (!std::isfinite(pos0[i])) return set_err(GR_INVALID_ARGUMENT, "non-finite start position");
    if (strength)
        for (uint64_t e = 0; e < m; e++)
            if (!std::isfinite(strength[e])) return set_err(GR_INVALID_ARGUMENT, "non-finite edge strength", (int)e);
    // the internal FA2 handle: 2D, edge strengths as the CSR weights (influence 1)
    double fv[11] = {100, 1.0, 2.0, 1.0, 0, 2, 0.8, 0, 0, 0, 1.0};
    uint8_t fb[sizeof fv];
    memcpy(fb, fv, sizeof fv);
    gr_fa2 *t = nullptr;
    if (int c = create_impl(&t, n, m, src, dst, strength, fb, sizeof fb, nullptr)) return c;
    gr_force_session *S = new (std::nothrow) gr_force_session();
    if (!S) {
        delete t;
        return set_err(GR_ALLOC_FAILED, "host allocation failed");
    }
    S->t = t;
    S->n = n;
    S->prm = prm;
    D3Params &P = S->P;
    P.n = n;
    P.seed = 0;  // session.rs:78 SEED
    P.charge = (float)prm.charge;
    P.th2 = (float)(prm.theta * prm.theta);
    P.dmin2 = (float)(prm.distance_min * prm.distance_min);
    P.dmax2 = (float)(prm.distance_max * prm.distance_max);
    P.link_distance = (float)prm.link_distance;
    P.link_strength_scale = (float)prm.link_strength_scale;
    const double diameter = 2.0 * prm.collide_radius;
    P.reach2 = (float)(diameter * diameter);
    P.reach = (float)std::sqrt(diameter * diameter);
    P.center_strength = (float)prm.center_strength;
    P.velocity_decay = (float)prm.velocity_decay;
    P.alpha_decay = prm.alpha_decay;
    cudaError_t e;
    if ((e = t->alloc(&S->p4, n)) || (e = t->alloc(&S->pp4, n)) || (e = t->alloc(&S->bounds, 2 * (size_t)n)) ||
        (e = t->alloc(&S->vel, n)) || (e = t->alloc(&S->seg_out, std::max<uint32_t>(t->nseg, 1))) ||
        (e = t->alloc(&S->ds, 1))) {
        delete S;
        return set_err(GR_ALLOC_FAILED, cudaGetErrorString(e));
    }
    // seed.rs golden_spiral: radius 12 sqrt(i + 1), angle i * golden angle, FP64 then narrowed
    std::vector<float4> host(n);
    for (uint32_t i = 0; i < n; i++) {
        double x, y;
        if (pos0) {
            x = pos0[2 * (size_t)i];
            y = pos0[2 * (size_t)i + 1];
        } else {
            const double radius = 12.0 * std::sqrt((double)i + 1.0), angle = (double)i * 2.399963229728653;
            x = std::cos(angle) * radius;
            y = std::sin(angle) * radius;
        }
        host[i] = make_float4((float)x, (float)y, 0.f, 1.f);
    }
    D3State d0{prm.initial_alpha, 0.0, 0u, 0u};
    cudaStream_t s = t->stream;
    if (n) {
        CU(cudaMemcpyAsync(S->p4, host.data(), (size_t)n * sizeof(float4), cudaMemcpyHostToDevice, s));
        CU(cudaMemsetAsync(S->vel, 0, (size_t)n * sizeof(float2), s));
    }
    CU(cudaMemcpyAsync(S->ds, &d0, sizeof d0, cudaMemcpyHostToDevice, s));
    CU(cudaStreamSynchronize(s));
    *out = S;
    return ok();
}

void gr_force_session_destroy(gr_force_session *S) { delete S; }

int gr_force_session_tick(gr_force_session *S, uint32_t ticks) {
    if (!S) return set_err(GR_INVALID_HANDLE, "null session");
    if (S->n == 0 || ticks == 0) return ok();
    if (int c = d3_build_graph(S)) return c;
    for (uint32_t k = 0; k < ticks; k++) CU(cudaGraphLaunch(S->exec, S->t->stream));
    DevState st;
    if (int c = read_state(S->t, &st)) return c;
    if (int c = check_device(S->t, st)) return c;
    return ok();
}

int gr_force_session_tick_timed(gr_force_session *S, uint32_t ticks, float *ms) {
    if (!S) return set_err(GR_INVALID_HANDLE, "null session");
    if (!ms) return set_err(GR_INVALID_ARGUMENT, "ms is null");
    *ms = 0.f;
    if (S->n == 0 || ticks == 0) return ok();
    if (int c = d3_build_graph(S)) return c;
    cudaStream_t s = S->t->stream;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CU(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return set_err(GR_CUDA_ERROR, "event creation failed");
    }
    cudaError_t e = cudaEventRecord(e0, s);
    for (uint32_t k = 0; k < ticks && e == cudaSuccess; k++) e = cudaGraphLaunch(S->exec, s);
    if (e == cudaSuccess) e = cudaEventRecord(e1, s);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) return set_err(GR_CUDA_ERROR, cudaGetErrorString(e));
    DevState st;
    if (int c = read_state(S->t, &st)) return c;
    if (int c = check_device(S->t, st)) return c;
    return ok();
}

int gr_force_session_positions(gr_force_session *S, float *out) {
    if (!S) return set_err(GR_INVALID_HANDLE, "null session");
    if (!out && S->n) return set_err(GR_INVALID_ARGUMENT, "out is null");
    std::vector<float4> host(S->n);
    if (S->n) CU(cudaMemcpyAsync(host.data(), S->p4, (size_t)S->n * sizeof(float4), cudaMemcpyDeviceToHost, S->t->stream));
    CU(cudaStreamSynchronize(S->t->stream));
    for (uint32_t i = 0; i < S->n; i++) {
        out[2 * (size_t)i] = host[i].x;
        out[2 * (size_t)i + 1] = host[i].y;
        if (!std::isfinite(host[i].x) || !std::isfinite(host[i].y))
            return set_err(GR_LAYOUT_FAILED, "non-finite position (StageError::NonFinite)");
    }
    return ok();
}

int gr_force_session_velocities(gr_force_session *S, float *out) {
    if (!S) return set_err(GR_INVALID_HANDLE, "null session");
    if (!out && S->n) return set_err(GR_INVALID_ARGUMENT, "out is null");
    if (S->n) CU(cudaMemcpyAsync(out, S->vel, (size_t)S->n * sizeof(float2), cudaMemcpyDeviceToHost, S->t->stream));
    CU(cudaStreamSynchronize(S->t->stream));
    return ok();
}

int gr_force_session_alpha(gr_force_session *S, double *alpha, uint32_t *ticks_done) {
    if (!S) return set_err(GR_INVALID_HANDLE, "null session");
    D3State d;
    CU(cudaMemcpyAsync(&d, S->ds, sizeof d, cudaMemcpyDeviceToHost, S->t->stream));
    CU(cudaStreamSynchronize(S->t->stream));
    if (alpha) *alpha = d.alpha;
    if (ticks_done) *ticks_done = d.tick_no;
    return ok();
}

int gr_force_session_reheat(gr_force_session *S, double alpha) {
    if (!S) return set_err(GR_INVALID_HANDLE, "null session");
    if (!std::isfinite(alpha) || alpha < 0.0 || alpha > 1.0)
        return set_err(GR_PARAM_OUT_OF_RANGE, "alpha must be a finite value in [0, 1]");
    CU(cudaMemcpyAsync(&S->ds->alpha, &alpha, sizeof alpha, cudaMemcpyHostToDevice, S->t->stream));
    CU(cudaStreamSynchronize(S->t->stream));
    return ok();
}

int gr_force_session_set_state(gr_force_session *S, const float *pos, const float *vel, double alpha,
                               uint32_t ticks_done) {
    if (!S) return set_err(GR_INVALID_HANDLE, "null session");
    if (!std::isfinite(alpha) || alpha < 0.0 || alpha > 1.0)
        return set_err(GR_PARAM_OUT_OF_RANGE, "alpha must be a finite value in [0, 1]");
    const size_t n = S->n;
    for (size_t i = 0; i < 2 * n; i++)
        if ((pos && !std::isfinite(pos[i])) || (vel && !std::isfinite(vel[i])))
            return set_err(GR_INVALID_ARGUMENT, "non-finite position or velocity", (int)(i / 2));
    cudaStream_t s = S->t->stream;
    std::vector<float4> host(n);
    if (pos && n) {
        for (size_t i = 0; i < n; i++) host[i] = make_float4(pos[2 * i], pos[2 * i + 1], 0.f, 1.f);
        CU(cudaMemcpyAsync(S->p4, host.data(), n * sizeof(float4), cudaMemcpyHostToDevice, s));
    }
    if (vel && n) CU(cudaMemcpyAsync(S->vel, vel, n * sizeof(float2), cudaMemcpyHostToDevice, s));
    D3State d;
    CU(cudaMemcpyAsync(&d, S->ds, sizeof d, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    d.alpha = alpha;
    d.tick_no = ticks_done;
    CU(cudaMemcpyAsync(S->ds, &d, sizeof d, cudaMemcpyHostToDevice, s));
    CU(cudaStreamSynchronize(s));
    return ok();
}

int gr_force_session_use_mesh(gr_force_session *S) {
    if (!S) return set_err(GR_INVALID_HANDLE, "null session");
    if (S->mesh) return ok();
    gr_fa2 *t = S->t;
    const uint32_t n = S->n;
    // mesh.rs side_for: next power of two of ceil(sqrt(n)), in [128, 1024]
    uint32_t root = (uint32_t)std::ceil(std::sqrt((double)n)), side = 1, bits = 0;
    while (side < root) {
        side <<= 1;
        bits++;
    }
    while (side < (uint32_t)PM_MIN_SIDE) {
        side <<= 1;
        bits++;
    }
    while (side > (uint32_t)PM_MAX_SIDE) {
        side >>= 1;
        bits--;
    }
    const size_t NN = (size_t)side * side;
    const uint32_t blocks = std::max<uint32_t>(1, std::min<uint32_t>(div_up(n, PM_T), 592));
    cudaError_t e;
    if ((e = t->alloc(&S->pm, 1)) || (e = t->alloc(&S->pm_part, 6 * (size_t)blocks)) ||
        (e = t->alloc(&S->pm_key, n)) || (e = t->alloc(&S->pm_val, n)) || (e = t->alloc(&S->pm_frac, n)) ||
        (e = t->alloc(&S->pm_cs, NN)) || (e = t->alloc(&S->pm_ce, NN)) || (e = t->alloc(&S->ga, NN)) ||
        (e = t->alloc(&S->gk, NN)) || (e = t->alloc(&S->gt, NN)) || (e = t->alloc(&S->tw, side / 2)) ||
        (e = S->pm_sorter.init(std::max<uint32_t>(n, 1), t->stream, true)))
        return set_err(GR_ALLOC_FAILED, cudaGetErrorString(e));
    // fft.rs Plan::new root: e^(-i TAU k / side), FP64 then narrowed
    std::vector<float2> tw(side / 2);
    for (uint32_t k = 0; k < side / 2; k++) {
        const double angle = -6.283185307179586 * (double)k / (double)side;
        tw[k] = make_float2((float)std::cos(angle), (float)std::sin(angle));
    }
    cudaStream_t s = t->stream;
    CU(cudaMemcpyAsync(S->tw, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice, s));
    CU(cudaMemsetAsync(S->pm, 0, sizeof(PmState), s));
    CU(cudaMemsetAsync(S->pm_key, 0, (size_t)std::max(n, 1u) * 8, s));
    CU(cudaMemsetAsync(S->pm_val, 0, (size_t)std::max(n, 1u) * 4, s));
    CU(cudaStreamSynchronize(s));
    S->side = side;
    S->bits = bits;
    S->pm_blocks = blocks;
    S->mesh = true;
    if (S->exec) cudaGraphExecDestroy(S->exec);
    if (S->graph) cudaGraphDestroy(S->graph);
    S->exec = nullptr;
    S->graph = nullptr;
    return ok();
}

int gr_force_mesh_run(uint32_t n, uint64_t m, const uint32_t *src, const uint32_t *dst, const double *strength,
                      float *out) {
    gr_force_session *S = nullptr;
    if (int c = gr_force_session_create(&S, n, m, src, dst, strength, nullptr, nullptr)) return c;
    int c = gr_force_session_use_mesh(S);
    if (c == GR_OK) c = gr_force_session_tick(S, GR_FORCE_TICKS);
    if (c == GR_OK) c = gr_force_session_positions(S, out);
    delete S;
    return c;
}

int gr_force_session_info(gr_force_session *S, uint32_t *graph_kernels, uint32_t *n_cells) {
    if (!S) return set_err(GR_INVALID_HANDLE, "null session");
    if (graph_kernels) *graph_kernels = S->graph_kernels;
    DevState st;
    if (int c = read_state(S->t, &st)) return c;
    if (n_cells) *n_cells = st.n_cells;
    return ok();
}

int gr_force_run(uint32_t n, uint64_t m, const uint32_t *src, const uint32_t *dst, const double *strength,
                 float *out) {
    gr_force_session *S = nullptr;
    if (int c = gr_force_session_create(&S, n, m, src, dst, strength, nullptr, nullptr)) return c;
    int c = gr_force_session_tick(S, GR_FORCE_TICKS);
    if (c == GR_OK) c = gr_force_session_positions(S, out);
    delete S;
    return c;
}

}  // extern "C"
