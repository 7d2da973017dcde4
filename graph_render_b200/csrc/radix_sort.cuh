// Stable LSD radix sort of (uint64 key, uint32 value) pairs, 8-bit digits.
//
// Per digit: an upsweep (per-tile digit counts), a digit-parallel scan (one
// block per digit over the tiles, plus the exclusive prefix of the digit
// totals), and a downsweep that ranks each key inside its tile with warp
// ballots/popc and scatters it; or, for the tick's sort, the one-sweep passes
// further down. Stability comes from ranking in input order:
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

// Lanes whose 8-bit digit equals this lane's, from one ballot per digit bit
// (full issue rate, where match.any serialises); lanes with !ok match only
// lanes with !ok.
__device__ __forceinline__ uint32_t warp_digit_peers(uint32_t dgt, bool ok) {
    uint32_t peers = __ballot_sync(GR_FULL, ok);
    if (!ok) peers = ~peers;
#pragma unroll
    for (int bit = 0; bit < 8; bit++) {
        const uint32_t b = __ballot_sync(GR_FULL, (dgt >> bit) & 1u);
        peers &= ((dgt >> bit) & 1u) ? b : ~b;
    }
    return peers;
}

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
    for (int r = 0; r < RS_ITEMS; r++) {  // every load in flight before the first rank
        const uint64_t i = base + (uint64_t)r * GR_WARP + lane;
        key[r] = i < n ? kin[i] : 0ull;
        val[r] = i < n ? vin[i] : V(0);
    }
#pragma unroll
    for (int r = 0; r < RS_ITEMS; r++) {
        const bool ok = base + (uint64_t)r * GR_WARP + lane < n;
        uint32_t dgt = ok ? ((uint32_t)(key[r] >> shift) & 0xffu) : (RS_BINS + lane);
        uint32_t peers = warp_digit_peers(dgt, ok);
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

// ---- one-sweep passes (Adinets & Merrill 2022, "Onesweep: a faster least
// significant digit radix sort for GPUs"): one histogram kernel for every digit
// of the sort, then one kernel per digit. A block takes the next tile id from a
// counter, ranks its keys as rs_downsweep does, publishes its per-digit count,
// and finds the count of each digit in all earlier tiles by decoupled look-back
// over their published words ({flag, count} in one 32-bit word: flag A = this
// tile's count only, P = the inclusive prefix through this tile). Tile ids are
// handed out in start order, so a block only ever waits on blocks that are
// already running; each wait is still bounded and raises ERR_WAIT if it gives
// up. The keys are then ordered by digit in shared memory and written out with
// consecutive threads on consecutive addresses of each digit's run.

constexpr int OS_HIST_THREADS = 256;
constexpr int OS_MAX_PASSES = 8;
constexpr uint32_t OS_FLAG_A = 1u << 30, OS_FLAG_P = 2u << 30, OS_COUNT = (1u << 30) - 1u;
constexpr uint32_t OS_SPIN_LIMIT = 1u << 22;  // x 32 ns sleeps: ~0.1 s

// The bounds on a pass's look-back waits: `limit` sleeps before a wait gives up
// (ERR_WAIT in the pass's error word); `halt` (nullable) is set to 1 when one
// does, the word the caller's later kernels skip on; `stall` (nullable, fault
// injection for tests) makes tile 1 first wait for that word to become nonzero,
// which nothing does, so its wait gives up after `limit` sleeps.
struct OsWait {
    uint32_t limit = OS_SPIN_LIMIT;
    uint32_t *halt = nullptr;
    const uint32_t *stall = nullptr;
};

// The tile shape the engine uses: T threads x I keys, look-back window L
// (on B200 at 1M keys: 512 x 8 sorts 4 digits in 78 us, 256 x 8 in 105 us).
constexpr int OS_T = 512, OS_I = 8, OS_L = 8;
// From this many keys up the passes take tiles of OS_BIG_T x OS_BIG_I keys: fewer
// tiles to look back over, and at 1M keys 145 tiles of one block per SM, one wave
// on 148 SMs. In the 1M-node tick's 4 passes, against 512 x 8: 768 x 9 15 us less,
// 1024 x 8 and 768 x 10 7.5 us less, 1024 x 7 11 us less; 768 x 8, 1024 x 6 and
// 512 x 12 (163 tiles) 10-15 us more. Below it the smaller tiles keep more blocks
// busy (larger ones made small graphs' one-tile sorts slower).
constexpr int OS_BIG_T = 768, OS_BIG_I = 9;
constexpr uint32_t OS_BIG_MIN = 1u << 19;

// Keys per one-sweep tile for a sort of n keys.
__host__ __device__ inline uint32_t os_tile_keys(uint32_t n) {
    return n >= OS_BIG_MIN ? OS_BIG_T * OS_BIG_I : OS_T * OS_I;
}


// Digit histograms of `passes` digits from first_digit (ghist, zeroed by the
// caller, passes x 256), and the zeroing of every pass's look-back words.
__global__ void __launch_bounds__(OS_HIST_THREADS)
os_hist(const uint64_t *__restrict__ keys, uint32_t n, int first_digit, int passes, uint32_t *__restrict__ ghist,
        uint32_t *__restrict__ status, uint64_t status_words, const uint32_t *skip) {
    if (skip && *skip) return;
    __shared__ uint32_t s_h[OS_MAX_PASSES][RS_BINS];
    const int t = threadIdx.x;
    for (int p = 0; p < OS_MAX_PASSES; p++) s_h[p][t] = 0;
    __syncthreads();
    const uint64_t stride = (uint64_t)gridDim.x * OS_HIST_THREADS;
    for (uint64_t i0 = (uint64_t)blockIdx.x * OS_HIST_THREADS + t; i0 < n; i0 += 4 * stride) {
        uint64_t k[4];
#pragma unroll
        for (int u = 0; u < 4; u++) k[u] = i0 + u * stride < n ? keys[i0 + u * stride] : 0ull;
#pragma unroll
        for (int u = 0; u < 4; u++)
            if (i0 + u * stride < n)
                for (int p = 0; p < passes; p++)
                    atomicAdd(&s_h[p][(uint32_t)(k[u] >> (8 * (first_digit + p))) & 0xffu], 1u);
    }
    __syncthreads();
    for (int p = 0; p < passes; p++)
        if (s_h[p][t]) atomicAdd(&ghist[p * RS_BINS + t], s_h[p][t]);
    for (uint64_t i = (uint64_t)blockIdx.x * OS_HIST_THREADS + t; i < status_words; i += stride) status[i] = 0u;
}

// Exclusive scan of (a, b) over the block's first 256 threads (the digits;
// every thread of the block calls it, threads >= 256 with zeros).
template <int T>
__device__ __forceinline__ void os_scan2(uint32_t a, uint32_t b, uint32_t &ea, uint32_t &eb, uint2 *s_w) {
    const int t = threadIdx.x, lane = t % GR_WARP, w = t / GR_WARP;
    uint32_t sa = a, sb = b;
#pragma unroll
    for (int o = 1; o < GR_WARP; o <<= 1) {
        const uint32_t ya = __shfl_up_sync(GR_FULL, sa, o), yb = __shfl_up_sync(GR_FULL, sb, o);
        if (lane >= o) {
            sa += ya;
            sb += yb;
        }
    }
    if (lane == GR_WARP - 1) s_w[w] = make_uint2(sa, sb);
    __syncthreads();
    uint32_t ba = 0, bb = 0;
    for (int k = 0; k < w && k < RS_BINS / GR_WARP; k++) {
        ba += s_w[k].x;
        bb += s_w[k].y;
    }
    ea = ba + sa - a;
    eb = bb + sb - b;
}

// Dynamic shared memory of os_pass<V, T, I, L>.
template <typename V, int T, int I>
constexpr size_t os_smem() {
    return (size_t)T * I * (sizeof(uint64_t) + sizeof(V)) + (size_t)(T / GR_WARP) * RS_BINS * 4 + 2 * RS_BINS * 4 +
           (size_t)(T / GR_WARP) * sizeof(uint2) + 16;
}

template <typename V, int T, int I, int L>
__global__ void __launch_bounds__(T)
os_pass(const uint64_t *__restrict__ kin, const V *__restrict__ vin, uint64_t *__restrict__ kout, V *__restrict__ vout,
        uint32_t n, int shift, const uint32_t *__restrict__ ghist, uint32_t *status, uint32_t *counter, uint32_t *err,
        const uint32_t *skip, OsWait wt) {
    gr_pdl_enter();
    static_assert(T % RS_BINS == 0, "one thread per digit at least");
    constexpr int W = T / GR_WARP, TILE = T * I, CHUNK = I * GR_WARP;
    if (skip && *skip) return;
    extern __shared__ __align__(16) unsigned char os_sm[];
    uint64_t *s_k = (uint64_t *)os_sm;                                   // TILE keys in digit order
    V *s_v = (V *)(s_k + TILE);                                          // their values
    uint32_t(*s_cnt)[RS_BINS] = (uint32_t(*)[RS_BINS])(s_v + TILE);      // per warp, per digit
    uint32_t *s_base = (uint32_t *)(s_cnt + W);  // output index of this tile's first key of each digit
    uint32_t *s_loc = s_base + RS_BINS;          // tile-local index of the same key
    uint2 *s_w = (uint2 *)(s_loc + RS_BINS);
    uint32_t *s_tile = (uint32_t *)(s_w + W);
    const int t = threadIdx.x, lane = t % GR_WARP, w = t / GR_WARP;
    for (int i = t; i < W * RS_BINS; i += T) (&s_cnt[0][0])[i] = 0;
    if (t == 0) *s_tile = atomicAdd(counter, 1u);
    __syncthreads();
    const uint32_t tile = *s_tile;
    const uint64_t base = (uint64_t)tile * TILE + (uint64_t)w * CHUNK;
    uint64_t key[I];
    V val[I];
    uint32_t rank[I];
    const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
    for (int r = 0; r < I; r++) {  // every load in flight before the first rank
        const uint64_t i = base + (uint64_t)r * GR_WARP + lane;
        key[r] = i < n ? kin[i] : 0ull;
        val[r] = i < n ? vin[i] : V(0);
    }
#pragma unroll
    for (int r = 0; r < I; r++) {
        const bool ok = base + (uint64_t)r * GR_WARP + lane < n;
        const uint32_t dgt = ok ? ((uint32_t)(key[r] >> shift) & 0xffu) : (RS_BINS + lane);
        const uint32_t peers = warp_digit_peers(dgt, ok);
        const uint32_t before = __popc(peers & lt);
        const uint32_t c = ok ? s_cnt[w][dgt] : 0u;
        __syncwarp();
        if (ok && before == 0) s_cnt[w][dgt] = c + __popc(peers);
        __syncwarp();
        rank[r] = c + before;
    }
    __syncthreads();
    volatile uint32_t *vs = status;
    uint32_t cnt = 0;  // this tile's keys with digit t; s_cnt becomes the exclusive prefix over warps
    if (t < RS_BINS) {
#pragma unroll 8
        for (int k = 0; k < W; k++) {
            const uint32_t x = s_cnt[k][t];
            s_cnt[k][t] = cnt;
            cnt += x;
        }
        vs[(size_t)tile * RS_BINS + t] = (tile == 0 ? OS_FLAG_P : OS_FLAG_A) | cnt;
    }
    uint32_t loc, gpre;
    os_scan2<T>(cnt, t < RS_BINS ? ghist[t] : 0u, loc, gpre, s_w);
    if (t < RS_BINS) {
        uint32_t excl = 0;  // keys with digit t in tiles before this one
        if (tile > 0) {
            // L predecessors per step, loaded together, consumed in order up to the
            // first P (done) or the first tile that has published nothing (wait).
            int64_t j = (int64_t)tile - 1;
            uint32_t spins = 0;
            bool done = false, gave_up = false;
            if (wt.stall && tile == 1) {  // injected fault: a word that nothing sets
                while (*(volatile const uint32_t *)wt.stall == 0u) {
                    if (++spins > wt.limit) {
                        gave_up = done = true;
                        break;
                    }
                    __nanosleep(32);
                }
            }
            while (!done) {
                uint32_t v[L];
#pragma unroll
                for (int k = 0; k < L; k++)
                    v[k] = j - k >= 0 ? (uint32_t)vs[(size_t)(j - k) * RS_BINS + t] : (uint32_t)OS_FLAG_P;
                int used = 0;
                bool wait = false;
#pragma unroll
                for (int k = 0; k < L; k++) {
                    if (done || wait) continue;
                    if ((v[k] & ~OS_COUNT) == 0u) {
                        wait = true;
                        continue;
                    }
                    excl += v[k] & OS_COUNT;
                    used++;
                    done = (v[k] & OS_FLAG_P) != 0u;
                }
                j -= used;
                if (!done && wait) {
                    if (++spins > wt.limit) {
                        gave_up = true;
                        break;
                    }
                    __nanosleep(32);
                }
            }
            if (gave_up) {  // the counts are wrong: flag it and stop the caller's later kernels
                atomicOr(err, (uint32_t)ERR_WAIT);
                if (wt.halt) atomicExch(wt.halt, 1u);
            }
            vs[(size_t)tile * RS_BINS + t] = OS_FLAG_P | (excl + cnt);
        }
        s_loc[t] = loc;
        s_base[t] = gpre + excl;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < I; r++) {
        const uint64_t i = base + (uint64_t)r * GR_WARP + lane;
        if (i < n) {
            const uint32_t dgt = (uint32_t)(key[r] >> shift) & 0xffu;
            const uint32_t at = s_loc[dgt] + s_cnt[w][dgt] + rank[r];
            s_k[at] = key[r];
            s_v[at] = val[r];
        }
    }
    __syncthreads();
    const uint64_t t0 = (uint64_t)tile * TILE;
    const uint32_t tn = (uint32_t)min((uint64_t)TILE, n - t0);
    for (uint32_t i = t; i < tn; i += T) {
        const uint64_t k = s_k[i];
        const uint32_t dgt = (uint32_t)(k >> shift) & 0xffu;
        const uint32_t at = s_base[dgt] + (i - s_loc[dgt]);
        if (at < n) {  // always, unless a look-back wait gave up (ERR_WAIT)
            kout[at] = k;
            vout[at] = s_v[i];
        }
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
    uint32_t os_tiles = 0;
    uint32_t *os_ghist = nullptr;   // OS_MAX_PASSES * RS_BINS digit counts, then OS_MAX_PASSES tile counters
    uint32_t *os_status = nullptr;  // OS_MAX_PASSES * os_tiles * RS_BINS look-back words
    OsWait wait;                    // the one-sweep passes' wait bounds (halt is per call)

    // With a stream, the buffers come from the device's stream-ordered pool on it
    // and go back to it on release (no device-wide synchronisation).
    cudaStream_t pool_stream = nullptr;
    bool pooled = false;
    template <typename T>
    cudaError_t get(T **p, size_t bytes) {
        return pooled ? cudaMallocAsync((void **)p, bytes, pool_stream) : cudaMalloc((void **)p, bytes);
    }
    void put(void *p) {
        if (!p) return;
        if (pooled)
            cudaFreeAsync(p, pool_stream);
        else
            cudaFree(p);
    }

    cudaError_t init(uint32_t capacity, cudaStream_t s = nullptr, bool pool = false) {
        cap = capacity ? capacity : 1;
        ntiles = div_up(cap, RS_TILE);
        os_tiles = div_up(cap, OS_T * OS_I);
        pool_stream = s;
        pooled = pool;
        cudaError_t e;
        if ((e = get(&os_ghist, (size_t)OS_MAX_PASSES * (RS_BINS + 1) * sizeof(uint32_t)))) return e;
        if ((e = get(&os_status, (size_t)OS_MAX_PASSES * os_tiles * RS_BINS * sizeof(uint32_t)))) return e;
        if ((e = get(&k_alt, (size_t)cap * sizeof(uint64_t)))) return e;
        if ((e = get(&v_alt, (size_t)cap * sizeof(uint32_t)))) return e;
        if ((e = get(&hist, (size_t)RS_BINS * ntiles * sizeof(uint32_t)))) return e;
        if ((e = get(&totals, (size_t)8 * RS_BINS * sizeof(uint32_t)))) return e;
        return cudaSuccess;
    }
    void release() {
        put(k_alt);
        put(v_alt);
        put(hist);
        put(totals);
        put(os_ghist);
        put(os_status);
        os_ghist = nullptr;
        os_status = nullptr;
        k_alt = nullptr;
        v_alt = nullptr;
        hist = nullptr;
        totals = nullptr;
    }
    size_t bytes() const {
        return (size_t)cap * 12 + (size_t)RS_BINS * ntiles * 4 + 8 * RS_BINS * 4 +
               (size_t)OS_MAX_PASSES * (RS_BINS + 1) * 4 + (size_t)OS_MAX_PASSES * os_tiles * RS_BINS * 4;
    }

    // One-sweep passes for digits first_digit .. first_digit + passes - 1
    // (passes even, at most OS_MAX_PASSES; n < 2^30, the look-back word's count
    // field). Same result as sort_digits. A wait that gives up sets ERR_WAIT in *err.
    void sort_onesweep(uint64_t *keys, uint32_t *vals, uint32_t n, int first_digit, int passes, cudaStream_t s,
                       uint32_t *err, const uint32_t *skip = nullptr) {
        if (n == 0) return;
        const uint32_t nt = div_up(n, os_tile_keys(n));
        cudaMemsetAsync(os_ghist, 0, ghist_words() * sizeof(uint32_t), s);
        const uint64_t words = (uint64_t)passes * nt * RS_BINS;
        os_hist<<<std::min<uint32_t>(div_up(n, OS_HIST_THREADS * 4), 4 * 148), OS_HIST_THREADS, 0, s>>>(
            keys, n, first_digit, passes, os_ghist, os_status, words, skip);
        onesweep_passes(keys, vals, n, first_digit, passes, s, err, skip);
    }

    // Words of os_ghist (digit counts, then the passes' tile counters) that
    // must be zero before a histogram pass.
    static constexpr uint32_t ghist_words() { return (uint32_t)OS_MAX_PASSES * (RS_BINS + 1); }

    // The one-sweep passes alone, for a caller whose own kernel already filled
    // os_ghist (zeroed first) with the digit counts and zeroed the look-back
    // words (os_hist's work). The result lands in keys/vals: with an even pass
    // count the input is read from there, with an odd one from the scratch pair
    // (k_alt, v_alt), where the caller's kernel wrote it.
    // A wait that gives up sets ERR_WAIT in *err and, when halt is given, *halt = 1.
    void onesweep_passes(uint64_t *keys, uint32_t *vals, uint32_t n, int first_digit, int passes, cudaStream_t s,
                         uint32_t *err, const uint32_t *skip = nullptr, bool pdl = false, uint32_t *halt = nullptr) {
        if (n == 0) return;
        OsWait w = wait;
        w.halt = halt;
        if (n >= OS_BIG_MIN)
            passes_shaped<OS_BIG_T, OS_BIG_I>(keys, vals, n, first_digit, passes, s, err, skip, pdl, w);
        else
            passes_shaped<OS_T, OS_I>(keys, vals, n, first_digit, passes, s, err, skip, pdl, w);
    }

    template <int T, int I>
    void passes_shaped(uint64_t *keys, uint32_t *vals, uint32_t n, int first_digit, int passes, cudaStream_t s,
                       uint32_t *err, const uint32_t *skip, bool pdl, const OsWait &w) {
        static_assert(T * I >= OS_T * OS_I, "os_tiles counts tiles of the smallest shape");
        const uint32_t nt = div_up(n, T * I);
        constexpr size_t smem = os_smem<uint32_t, T, I>();
        if (smem > 48 * 1024)
            cudaFuncSetAttribute(os_pass<uint32_t, T, I, OS_L>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
        const bool odd = passes & 1;
        uint64_t *ka = odd ? k_alt : keys, *kb = odd ? keys : k_alt;
        uint32_t *va = odd ? v_alt : vals, *vb = odd ? vals : v_alt;
        for (int p = 0; p < passes; p++) {
            gr_launch(pdl, os_pass<uint32_t, T, I, OS_L>, nt, T, smem, s, ka, (const uint32_t *)va, kb, vb, n,
                      8 * (first_digit + p), (const uint32_t *)(os_ghist + p * RS_BINS),
                      os_status + (size_t)p * nt * RS_BINS, os_ghist + OS_MAX_PASSES * RS_BINS + p, err, skip, w);
            std::swap(ka, kb);
            std::swap(va, vb);
        }
    }

    // Sorts keys[0..n) (low `bits` bits significant) with their values, in
    // place: one-sweep passes when they fit (n < 2^30, at most OS_MAX_PASSES
    // digits), else the upsweep / scan / downsweep passes. A one-sweep wait that
    // gives up sets ERR_WAIT in *err.
    void sort_bits(uint64_t *keys, uint32_t *vals, uint32_t n, int bits, cudaStream_t s, uint32_t *err) {
        int passes = (bits + 7) / 8;
        passes += passes & 1;
        if (n < (1u << 30) && passes <= OS_MAX_PASSES)
            sort_onesweep(keys, vals, n, 0, passes, s, err);
        else
            sort(keys, vals, n, bits, s);
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
