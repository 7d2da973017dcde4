// Shared device helpers for the ForceAtlas2 / Barnes-Hut engine (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define GR_WARP 32
#define GR_FULL 0xffffffffu

namespace gr {

// Status codes. The numbering follows graph-wasm's `Code` enum
// (crates/graph-wasm/src/errors.rs:18-122) so a host that switches on the
// reference's codes reads the same refusal here; codes past 99 are this
// library's own (device and CUDA failures the wasm build cannot have).
enum Code : int {
    OK = 0,
    INVALID_HANDLE = 1,
    ALLOC_FAILED = 2,
    UNKNOWN_LAYOUT_ID = 5,
    LAYOUT_FAILED = 8,
    INDEX_OUT_OF_RANGE = 12,
    PARAM_OUT_OF_RANGE = 20,
    PARAMS_MALFORMED = 21,
    PARAMS_NOT_ACCEPTED = 22,
    INVALID_ARGUMENT = 100,
    CUDA_ERROR = 101,
    DEVICE_FAULT = 102,
};

// Device-resident per-graph scalars. The speed controller runs in FP64
// (schedule.rs:33-60); the rest are counters the host reads after a tick.
struct DevState {
    double swing, traction, speed, speed_efficiency;  // cumulative, state.rs:141-143
    double moved;                                     // last tick's summed |step|
    double mean[3];                                   // mean of positions this tick
    double root0[3];                                  // root square corner
    double root_w;                                    // root square side
    double pad0;
    unsigned long long far_count, pair_count;         // interactions since creation
    uint32_t iter_no;                                 // completed ticks
    uint32_t converged;                               // a tick moved < 1e-10
    uint32_t n_unique;                                // distinct Morton keys this tick
    uint32_t n_cells;                                 // tree cells this tick
    uint32_t error;                                   // device error bits
    uint32_t bounds_stamp;                            // iter_no + 1 when root0 / root_w / mean are the
                                                      // current positions' (the update wrote them); else 0
    uint32_t counters[7];                             // last-block-done tickets
};

enum DevError : uint32_t {
    ERR_NONFINITE = 1u,
    ERR_TREE = 2u,
    ERR_BOUNDS = 4u,
    ERR_WAIT = 8u,  // a bounded wait on another block gave up
};

struct Body {  // FP64 cell sums: mass and mass-weighted coordinate sums
    double m, c0, c1, c2;
};

__device__ __forceinline__ Body body_add(const Body &a, const Body &b) {
    Body r;
    r.m = a.m + b.m;
    r.c0 = a.c0 + b.c0;
    r.c1 = a.c1 + b.c1;
    r.c2 = a.c2 + b.c2;
    return r;
}

__device__ __forceinline__ void body_store(Body *p, const Body &b) {
    double2 *q = reinterpret_cast<double2 *>(p);
    q[0] = make_double2(b.m, b.c0);
    q[1] = make_double2(b.c1, b.c2);
}

// rng.rs:27-34: MurmurHash3 fmix64.
__host__ __device__ __forceinline__ uint64_t fmix64(uint64_t k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdULL;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ULL;
    k ^= k >> 33;
    return k;
}

// rng.rs:39-84: the counter-hash nudge for an exactly coincident pair, keyed on
// (seed, tick, pass = axis, min(i,j), max(i,j)); the same FP64 value the
// reference draws, narrowed to the engine's FP32.
__host__ __device__ __forceinline__ double jiggle(uint32_t seed, uint32_t tick, uint32_t pass,
                                                  uint32_t i, uint32_t j) {
    uint32_t lo = i <= j ? i : j, hi = i <= j ? j : i;
    uint64_t a = fmix64((uint64_t)seed ^ ((uint64_t)tick << 32));
    uint64_t b = fmix64(a ^ ((uint64_t)pass << 32) ^ (uint64_t)lo);
    uint64_t w = fmix64(b ^ ((uint64_t)hi << 32) ^ a) >> 11;
    if (w == (1ULL << 52)) w = (1ULL << 52) + 1;
    double u = (double)w * (1.0 / (double)(1ULL << 53));
    return (u - 0.5) * 1e-6;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(GR_FULL, v, o);
    return v;
}

// Deterministic block sum: warp butterflies, then warp 0 over the warp sums in
// warp order. Every thread of the block must call it; the result is valid in
// thread 0.
template <int THREADS>
__device__ __forceinline__ double block_sum_d(double v, double *smem) {
    v = warp_sum_d(v);
    const int w = threadIdx.x / GR_WARP, l = threadIdx.x % GR_WARP;
    if (l == 0) smem[w] = v;
    __syncthreads();
    double r = 0.0;
    if (w == 0) {
        r = (l < THREADS / GR_WARP) ? smem[l] : 0.0;
        r = warp_sum_d(r);
    }
    __syncthreads();
    return r;
}

// Sum of v[k * stride + off] over this thread's k = threadIdx.x, threadIdx.x +
// T, ... < count, added in k order; U loads are in flight at a time (the same
// sum as one load per step, without a round trip per step).
template <int T, int U = 8>
__device__ __forceinline__ double strided_sum_cg(const double *v, uint32_t count, uint32_t stride, uint32_t off) {
    double a = 0.0;
    for (uint32_t k0 = threadIdx.x; k0 < count; k0 += T * U) {
        double x[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const uint32_t k = k0 + u * T;
            x[u] = k < count ? __ldcg(&v[(size_t)k * stride + off]) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < U; u++)
            if (k0 + u * T < count) a += x[u];
    }
    return a;
}

// True in exactly one thread of the grid's last block to finish (threadfence
// reduction pattern); the ticket resets itself for the next launch.
__device__ __forceinline__ bool last_block_done(uint32_t *ticket, bool *smem_flag) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = atomicAdd(ticket, 1u);
        *smem_flag = (t == gridDim.x - 1);
        if (*smem_flag) *ticket = 0;
    }
    __syncthreads();
    if (*smem_flag) __threadfence();
    return *smem_flag;
}

// Programmatic dependent launch (sm_90 and later). A kernel launched with
// programmatic stream serialization (gr_launch with pdl) may be scheduled while
// the kernel before it in the stream drains. gr_pdl_enter first lets the next
// such kernel be scheduled once every block of this grid has started, then
// waits until the kernel before this one has completed and its writes are
// visible. Every kernel that calls it does so before any access to global
// memory, so it sees exactly what plain stream order would give it; in a kernel
// launched without the attribute both instructions return at once.
__device__ __forceinline__ void gr_pdl_enter() {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 900
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
#endif
}

// Launches kernel k on stream s; with pdl, as a programmatic dependent of the
// kernel before it in the stream (k must call gr_pdl_enter first).
template <typename... KArgs, typename... Args>
inline cudaError_t gr_launch(bool pdl, void (*k)(KArgs...), uint32_t grid, uint32_t block, size_t smem,
                             cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, k, args...);
}

__host__ __device__ __forceinline__ uint32_t div_up(uint64_t a, uint32_t b) {
    return (uint32_t)((a + b - 1) / b);
}

}  // namespace gr
