// Stable LSD radix sort of (uint64 key, uint32 value) pairs, 8-bit digits.
//
// Per digit: an upsweep (per-tile digit counts), a digit-parallel scan (one
// block per digit over the tiles, plus the exclusive prefix of the digit
// totals), and a downsweep that ranks each key inside its tile with warp
// match/popc and scatters it. Stability comes from ranking in input order:
// within a warp's contiguous chunk by round then lane, across warps by warp
// index. Integer work only, so the result is bit-exact against any stable
// CPU sort of the same keys.
#pragma once

#include "common.cuh"

namespace gr {

constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / GR_WARP;
constexpr int RS_ITEMS = 16;                      // keys per thread per tile
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;    // 4096 keys per tile
constexpr int RS_BINS = 256;
constexpr int RS_CHUNK = RS_ITEMS * GR_WARP;      // 512 keys per warp

__global__ void __launch_bounds__(RS_THREADS)
rs_upsweep(const uint64_t *__restrict__ keys, uint32_t n, int shift, uint32_t *__restrict__ hist,
           uint32_t *__restrict__ totals, uint32_t ntiles, const uint32_t *skip) {
    if (skip && *skip) return;
    __shared__ uint32_t s_hist[RS_BINS];
    s_hist[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * RS_TILE;
#pragma unroll
    for (int r = 0; r < RS_ITEMS; r++) {
        uint64_t i = base + (uint64_t)r * RS_THREADS + threadIdx.x;
        if (i < n) atomicAdd(&s_hist[(uint32_t)(keys[i] >> shift) & 0xffu], 1u);
    }
    __syncthreads();
    uint32_t c = s_hist[threadIdx.x];
    hist[(size_t)threadIdx.x * ntiles + blockIdx.x] = c;
    if (c) atomicAdd(&totals[threadIdx.x], c);
}

// One block per digit: exclusive scan of that digit's per-tile counts, offset by
// the number of keys with a smaller digit.
__global__ void __launch_bounds__(RS_THREADS)
rs_scan(uint32_t *__restrict__ hist, const uint32_t *__restrict__ totals, uint32_t ntiles,
        const uint32_t *skip) {
    if (skip && *skip) return;
    __shared__ uint32_t s_warp[RS_WARPS];
    __shared__ uint32_t s_base;
    const int d = blockIdx.x, t = threadIdx.x, lane = t % GR_WARP, w = t / GR_WARP;
    // base = sum of totals[0..d)
    uint32_t v = (t < d) ? totals[t] : 0u;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(GR_FULL, v, o);
    if (lane == 0) s_warp[w] = v;
    __syncthreads();
    if (t == 0) {
        uint32_t b = 0;
        for (int i = 0; i < RS_WARPS; i++) b += s_warp[i];
        s_base = b;
    }
    __syncthreads();
    uint32_t running = s_base;
    uint32_t *row = hist + (size_t)d * ntiles;
    for (uint32_t off = 0; off < ntiles; off += RS_THREADS) {
        uint32_t i = off + t;
        uint32_t x = (i < ntiles) ? row[i] : 0u;
        // inclusive warp scan
        uint32_t s = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(GR_FULL, s, o);
            if (lane >= o) s += y;
        }
        __syncthreads();
        if (lane == 31) s_warp[w] = s;
        __syncthreads();
        uint32_t wbase = 0;
        for (int k = 0; k < w; k++) wbase += s_warp[k];
        uint32_t total = 0;
        for (int k = 0; k < RS_WARPS; k++) total += s_warp[k];
        if (i < ntiles) row[i] = running + wbase + s - x;
        running += total;
    }
}

template <typename V>
__global__ void __launch_bounds__(RS_THREADS)
rs_downsweep(const uint64_t *__restrict__ kin, const V *__restrict__ vin, uint64_t *__restrict__ kout,
             V *__restrict__ vout, uint32_t n, int shift, const uint32_t *__restrict__ hist,
             uint32_t ntiles, const uint32_t *skip) {
    if (skip && *skip) return;
    __shared__ uint32_t s_cnt[RS_WARPS][RS_BINS];
    __shared__ uint32_t s_off[RS_BINS];
    const int t = threadIdx.x, lane = t % GR_WARP, w = t / GR_WARP;
    for (int i = t; i < RS_WARPS * RS_BINS; i += RS_THREADS) (&s_cnt[0][0])[i] = 0;
    s_off[t] = hist[(size_t)t * ntiles + blockIdx.x];
    __syncthreads();

    const uint64_t base = (uint64_t)blockIdx.x * RS_TILE + (uint64_t)w * RS_CHUNK;
    uint64_t key[RS_ITEMS];
    V val[RS_ITEMS];
    uint32_t rank[RS_ITEMS];
    const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
    for (int r = 0; r < RS_ITEMS; r++) {
        uint64_t i = base + (uint64_t)r * GR_WARP + lane;
        bool ok = i < n;
        key[r] = ok ? kin[i] : 0ull;
        val[r] = ok ? vin[i] : V(0);
        uint32_t dgt = ok ? ((uint32_t)(key[r] >> shift) & 0xffu) : (RS_BINS + lane);
        uint32_t peers = __match_any_sync(GR_FULL, dgt);
        uint32_t before = __popc(peers & lt);
        uint32_t c = ok ? s_cnt[w][dgt] : 0u;
        __syncwarp();
        if (ok && before == 0) s_cnt[w][dgt] = c + __popc(peers);
        __syncwarp();
        rank[r] = c + before;
    }
    __syncthreads();
    // exclusive prefix over warps, per digit
    {
        uint32_t run = 0;
#pragma unroll
        for (int k = 0; k < RS_WARPS; k++) {
            uint32_t x = s_cnt[k][t];
            s_cnt[k][t] = run;
            run += x;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RS_ITEMS; r++) {
        uint64_t i = base + (uint64_t)r * GR_WARP + lane;
        if (i < n) {
            uint32_t dgt = (uint32_t)(key[r] >> shift) & 0xffu;
            uint32_t pos = s_off[dgt] + s_cnt[w][dgt] + rank[r];
            kout[pos] = key[r];
            vout[pos] = val[r];
        }
    }
}

__global__ void rs_zero(uint32_t *__restrict__ totals) { totals[blockIdx.x * RS_BINS + threadIdx.x] = 0; }

// After a stable sort on the high 32 key bits: every run of equal high words
// is put in full-key order by a stable insertion sort in place, which makes the
// result identical to a stable sort of the whole key. A run longer than
// max_run is left alone and raises *too_long instead.
__global__ void rs_fix_runs(uint64_t *__restrict__ keys, uint32_t *__restrict__ vals, uint32_t n, uint32_t max_run,
                            uint32_t *long_count, uint2 *__restrict__ long_runs, const uint32_t *skip) {
    if (skip && *skip) return;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i + 1 >= n) return;
    const uint32_t hi = (uint32_t)(keys[i] >> 32);
    if ((uint32_t)(keys[i + 1] >> 32) != hi) return;  // not a run of two or more
    if (i > 0 && (uint32_t)(keys[i - 1] >> 32) == hi) return;  // not the run's first element
    uint32_t len = 2;
    while (i + len < n && (uint32_t)(keys[i + len] >> 32) == hi) len++;
    if (len > max_run) {  // one CTA sorts it (rs_fix_long_runs)
        const uint32_t q = atomicAdd(long_count, 1u);
        long_runs[q] = make_uint2(i, len);
        return;
    }
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

// The pieces the fix-up of long runs needs: the block-level stable sort.
template <int BT>
__device__ void block_sort(uint64_t *keys, uint32_t *vals, uint64_t *kalt, uint32_t *valt, uint32_t n,
                           uint32_t (*s_cnt)[256], uint32_t *s_tot);

// Device buffers for sorting up to `cap` pairs. keys/vals are sorted in place
// (the scratch pair is the ping-pong partner; an even pass count ends in the
// caller's buffers).
struct RadixSorter {
    uint32_t cap = 0, ntiles = 0;
    uint64_t *k_alt = nullptr;
    uint32_t *v_alt = nullptr;
    uint32_t *hist = nullptr;    // RS_BINS * ntiles
    uint32_t *totals = nullptr;  // 8 passes * RS_BINS

    cudaError_t init(uint32_t capacity) {
        cap = capacity ? capacity : 1;
        ntiles = div_up(cap, RS_TILE);
        cudaError_t e;
        if ((e = cudaMalloc(&k_alt, (size_t)cap * sizeof(uint64_t)))) return e;
        if ((e = cudaMalloc(&v_alt, (size_t)cap * sizeof(uint32_t)))) return e;
        if ((e = cudaMalloc(&hist, (size_t)RS_BINS * ntiles * sizeof(uint32_t)))) return e;
        if ((e = cudaMalloc(&totals, (size_t)8 * RS_BINS * sizeof(uint32_t)))) return e;
        return cudaSuccess;
    }
    void release() {
        if (k_alt) cudaFree(k_alt);
        if (v_alt) cudaFree(v_alt);
        if (hist) cudaFree(hist);
        if (totals) cudaFree(totals);
        k_alt = nullptr;
        v_alt = nullptr;
        hist = nullptr;
        totals = nullptr;
    }
    size_t bytes() const {
        return (size_t)cap * 12 + (size_t)RS_BINS * ntiles * 4 + 8 * RS_BINS * 4;
    }

    // Sorts keys[0..n) (low `bits` bits significant, a multiple of 16) with
    // their values, in place. Kernel launches only: graph-capturable.
    void sort(uint64_t *keys, uint32_t *vals, uint32_t n, int bits, cudaStream_t s,
              const uint32_t *skip = nullptr) {
        int passes = (bits + 7) / 8;
        passes += passes & 1;  // even, so the result lands back in keys/vals
        sort_digits(keys, vals, n, 0, passes, s, skip);
    }

    // The passes for digits first_digit .. first_digit + passes - 1 (an even
    // count, so the result lands back in keys/vals).
    void sort_digits(uint64_t *keys, uint32_t *vals, uint32_t n, int first_digit, int passes, cudaStream_t s,
                     const uint32_t *skip = nullptr) {
        if (n == 0) return;
        uint32_t nt = div_up(n, RS_TILE);
        rs_zero<<<8, RS_BINS, 0, s>>>(totals);  // a kernel, so the sort also fits graph bodies that take kernels only
        uint64_t *ka = keys, *kb = k_alt;
        uint32_t *va = vals, *vb = v_alt;
        for (int p = 0; p < passes; p++) {
            int shift = 8 * (first_digit + p);
            uint32_t *tot = totals + (size_t)p * RS_BINS;
            rs_upsweep<<<nt, RS_THREADS, 0, s>>>(ka, n, shift, hist, tot, nt, skip);
            rs_scan<<<RS_BINS, RS_THREADS, 0, s>>>(hist, tot, nt, skip);
            rs_downsweep<uint32_t><<<nt, RS_THREADS, 0, s>>>(ka, va, kb, vb, n, shift, hist, nt, skip);
            uint64_t *tk = ka;
            ka = kb;
            kb = tk;
            uint32_t *tv = va;
            va = vb;
            vb = tv;
        }
    }
};

}  // namespace gr
