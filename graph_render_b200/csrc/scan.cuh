// Device-wide exclusive scan of uint32 counts (reduce, scan-of-block-sums,
// downsweep). The element count can live in device memory so the launches are
// sized for a host-side upper bound and stay graph-capturable while the real
// count changes from tick to tick.
#pragma once

#include "common.cuh"

namespace gr {

constexpr int SC_THREADS = 512;  // 512 x 4: the 1M-node tick's cell-level scan 2 us faster than 256 x 8
constexpr int SC_ITEMS = 4;
constexpr int SC_TILE = SC_THREADS * SC_ITEMS;

__device__ __forceinline__ uint32_t scan_count(uint32_t n_host, const uint32_t *n_dev, uint32_t add) {
    return n_dev ? *n_dev + add : n_host;
}

// The scanned value of an input word: the word itself, or with LV the count
// 1 + popc(word) of a cell level mask.
template <bool LV>
__device__ __forceinline__ uint32_t scan_item(uint32_t x) {
    return LV ? 1u + (uint32_t)__popc(x) : x;
}

template <bool LV>
__global__ void __launch_bounds__(SC_THREADS)
sc_reduce(const uint32_t *__restrict__ in, uint32_t n_host, const uint32_t *n_dev, uint32_t n_add,
          uint32_t *__restrict__ bsum, const uint32_t *skip) {
    if (skip && *skip) return;
    uint32_t n = scan_count(n_host, n_dev, n_add);
    __shared__ uint32_t s[SC_THREADS / GR_WARP];
    uint64_t base = (uint64_t)blockIdx.x * SC_TILE;
    uint32_t v = 0;
    if (base < n) {
#pragma unroll
        for (int r = 0; r < SC_ITEMS; r++) {
            uint64_t i = base + (uint64_t)r * SC_THREADS + threadIdx.x;
            if (i < n) v += scan_item<LV>(in[i]);
        }
    }
    v = __reduce_add_sync(GR_FULL, v);
    if (threadIdx.x % GR_WARP == 0) s[threadIdx.x / GR_WARP] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < SC_THREADS / GR_WARP; w++) t += s[w];
        bsum[blockIdx.x] = t;
    }
}

// Single block: exclusive scan of the block sums in place; the grand total goes
// to *total (and optionally to *total2).
__global__ void __launch_bounds__(1024)
sc_blocks(uint32_t *__restrict__ bsum, uint32_t nb, uint32_t *total, uint32_t *total2,
          const uint32_t *skip) {
    if (skip && *skip) return;
    __shared__ uint32_t s_w[32];
    const int t = threadIdx.x, lane = t % GR_WARP, w = t / GR_WARP;
    uint32_t running = 0;
    for (uint32_t off = 0; off < nb; off += 1024) {
        uint32_t i = off + t;
        uint32_t x = i < nb ? bsum[i] : 0u;
        uint32_t s = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(GR_FULL, s, o);
            if (lane >= o) s += y;
        }
        __syncthreads();
        if (lane == 31) s_w[w] = s;
        __syncthreads();
        uint32_t wb = 0, tot = 0;
        for (int k = 0; k < 32; k++) {
            uint32_t z = s_w[k];
            if (k < w) wb += z;
            tot += z;
        }
        if (i < nb) bsum[i] = running + wb + s - x;
        running += tot;
    }
    if (t == 0) {
        if (total) *total = running;
        if (total2) *total2 = running;
    }
}

template <bool LV>
__global__ void __launch_bounds__(SC_THREADS)
sc_down(const uint32_t *__restrict__ in, uint32_t *__restrict__ out, uint32_t n_host,
        const uint32_t *n_dev, uint32_t n_add, const uint32_t *__restrict__ bsum, const uint32_t *skip) {
    if (skip && *skip) return;
    uint32_t n = scan_count(n_host, n_dev, n_add);
    uint64_t base = (uint64_t)blockIdx.x * SC_TILE;
    if (base >= n) return;
    __shared__ uint32_t s_w[SC_THREADS / GR_WARP];
    const int t = threadIdx.x, lane = t % GR_WARP, w = t / GR_WARP;
    // blocked arrangement: thread t owns items [t*ITEMS, t*ITEMS+ITEMS)
    uint32_t x[SC_ITEMS];
    uint32_t sum = 0;
#pragma unroll
    for (int r = 0; r < SC_ITEMS; r++) {
        uint64_t i = base + (uint64_t)t * SC_ITEMS + r;
        x[r] = i < n ? scan_item<LV>(in[i]) : 0u;
        sum += x[r];
    }
    uint32_t s = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(GR_FULL, s, o);
        if (lane >= o) s += y;
    }
    if (lane == 31) s_w[w] = s;
    __syncthreads();
    uint32_t wb = 0;
    for (int k = 0; k < w; k++) wb += s_w[k];
    uint32_t run = bsum[blockIdx.x] + wb + s - sum;
#pragma unroll
    for (int r = 0; r < SC_ITEMS; r++) {
        uint64_t i = base + (uint64_t)t * SC_ITEMS + r;
        if (i < n) out[i] = run;
        run += x[r];
    }
}

// Up to this many blocks the cell-level scan runs as one pass (sc_levels_fold).
constexpr uint32_t SC_FOLD_MAX_BLOCKS = 2048;

// Exclusive scan of 1 + popc(levels[s]) over s < *n_dev in one pass, for at
// most SC_FOLD_MAX_BLOCKS blocks: marks[b], counted by the kernel that set the
// level bits, is the number of bits set in block b's leaves, so the sum of
// block b is its leaf count plus marks[b], and every block folds the sums of the
// blocks before its own (integers: the same value in any order). The block
// holding the last leaf writes the grand total.
__global__ void __launch_bounds__(SC_THREADS)
sc_levels_fold(const uint32_t *__restrict__ levels, uint32_t *__restrict__ out, const uint32_t *n_dev,
               const uint32_t *__restrict__ marks, uint32_t *total, const uint32_t *skip) {
    gr_pdl_enter();
    if (skip && *skip) return;
    const uint32_t n = *n_dev;
    const uint32_t b = blockIdx.x;
    const uint64_t base = (uint64_t)b * SC_TILE;
    if (base >= n) return;
    __shared__ uint32_t s_w[SC_THREADS / GR_WARP];
    __shared__ uint32_t s_pre;
    const int t = threadIdx.x, lane = t % GR_WARP, w = t / GR_WARP;
    uint32_t pm = 0;  // level bits set in the blocks before this one
    for (uint32_t j = t; j < b; j += SC_THREADS) pm += marks[j];
    pm = __reduce_add_sync(GR_FULL, pm);
    if (lane == 0) s_w[w] = pm;
    __syncthreads();
    if (t == 0) {
        uint32_t a = (uint32_t)base;  // one cell per leaf before this block
        for (int k = 0; k < SC_THREADS / GR_WARP; k++) a += s_w[k];
        s_pre = a;
    }
    __syncthreads();
    // blocked arrangement: thread t owns items [t*ITEMS, t*ITEMS+ITEMS)
    uint32_t x[SC_ITEMS];
    uint32_t sum = 0;
#pragma unroll
    for (int r = 0; r < SC_ITEMS; r++) {
        const uint64_t i = base + (uint64_t)t * SC_ITEMS + r;
        x[r] = i < n ? scan_item<true>(levels[i]) : 0u;
        sum += x[r];
    }
    uint32_t sc = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(GR_FULL, sc, o);
        if (lane >= o) sc += y;
    }
    if (lane == 31) s_w[w] = sc;
    __syncthreads();
    uint32_t wb = 0;
    for (int k = 0; k < w; k++) wb += s_w[k];
    uint32_t run = s_pre + wb + sc - sum;
#pragma unroll
    for (int r = 0; r < SC_ITEMS; r++) {
        const uint64_t i = base + (uint64_t)t * SC_ITEMS + r;
        if (i < n) out[i] = run;
        run += x[r];
    }
    if (t == SC_THREADS - 1 && (uint64_t)n <= base + SC_TILE) *total = run;
}

// Exclusive scan of in[0..n) into out[0..n) (in == out allowed); out[n] is not
// written, the total goes to *total. n = n_host, or *n_dev + n_add when n_dev
// is given (n_host is then the launch bound).
struct Scanner {
    uint32_t cap = 0, nb = 0;
    uint32_t *bsum = nullptr;
    cudaStream_t pool_stream = nullptr;  // with pooled: stream-ordered pool allocation on it
    bool pooled = false;
    cudaError_t init(uint32_t capacity, cudaStream_t s = nullptr, bool pool = false) {
        cap = capacity ? capacity : 1;
        nb = div_up(cap, SC_TILE);
        pool_stream = s;
        pooled = pool;
        const size_t bytes = (size_t)nb * sizeof(uint32_t);
        return pooled ? cudaMallocAsync((void **)&bsum, bytes, s) : cudaMalloc(&bsum, bytes);
    }
    void release() {
        if (bsum) {
            if (pooled)
                cudaFreeAsync(bsum, pool_stream);
            else
                cudaFree(bsum);
        }
        bsum = nullptr;
    }
    template <bool LV>
    void run(const uint32_t *in, uint32_t *out, uint32_t n_host, const uint32_t *n_dev, uint32_t n_add,
             uint32_t *total, uint32_t *total2, cudaStream_t s, const uint32_t *skip) {
        if (n_host == 0) return;
        uint32_t b = div_up(n_host, SC_TILE);
        sc_reduce<LV><<<b, SC_THREADS, 0, s>>>(in, n_host, n_dev, n_add, bsum, skip);
        sc_blocks<<<1, 1024, 0, s>>>(bsum, b, total, total2, skip);
        sc_down<LV><<<b, SC_THREADS, 0, s>>>(in, out, n_host, n_dev, n_add, bsum, skip);
    }
    void scan(const uint32_t *in, uint32_t *out, uint32_t n_host, const uint32_t *n_dev, uint32_t n_add,
              uint32_t *total, uint32_t *total2, cudaStream_t s, const uint32_t *skip = nullptr) {
        run<false>(in, out, n_host, n_dev, n_add, total, total2, s, skip);
    }
    // Exclusive scan of 1 + popc(levels[s]): the first cell index of every leaf.
    void scan_levels(const uint32_t *levels, uint32_t *out, uint32_t n_host, const uint32_t *n_dev,
                     uint32_t *total, cudaStream_t s, const uint32_t *skip = nullptr) {
        run<true>(levels, out, n_host, n_dev, 0, total, nullptr, s, skip);
    }
    // The same scan in one pass when the block sums were counted beforehand
    // into bsum (marks; zeroed before they were counted): up to
    // SC_FOLD_MAX_BLOCKS blocks, n_dev given.
    bool folds(uint32_t n_host) const { return div_up(n_host, SC_TILE) <= SC_FOLD_MAX_BLOCKS; }
    void scan_levels_marked(const uint32_t *levels, uint32_t *out, uint32_t n_host, const uint32_t *n_dev,
                            uint32_t *total, cudaStream_t s, const uint32_t *skip = nullptr, bool pdl = false) {
        if (n_host == 0) return;
        gr_launch(pdl, sc_levels_fold, div_up(n_host, SC_TILE), SC_THREADS, 0, s, levels, out, n_dev,
                  (const uint32_t *)bsum, total, skip);
    }
};

}  // namespace gr
