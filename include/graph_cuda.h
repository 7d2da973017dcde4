/*
 * graph_cuda.h — C ABI of the B200 (sm_100a) ForceAtlas2 / Barnes-Hut engine.
 *
 * The engine is a drop-in for graph-core's layout-registry row
 * `layout.forceatlas2.barnes_hut` (crates/graph-core/src/registry/layouts.rs:264-267),
 * reached in the reference through `Capability::run_params(&Topology, &[u8])`
 * (crates/graph-core/src/registry/params.rs:156-181) from `gm_run`
 * (crates/graph-wasm/src/exports/build.rs:69-101). It registers under its own id,
 * "layout.forceatlas2.barnes_hut.cuda", as the reference's own-id rule for a GPU
 * tier asks (docs/decisions/gpu-force-tier.md:34-38).
 *
 * Conventions (mirroring the reference's wasm ABI, docs/contract/wasm-abi.md):
 *   - Every call returns a status code; 0 is success. The numbering is graph-wasm's
 *     `Code` (crates/graph-wasm/src/errors.rs:18-122); gr_last_error() returns the
 *     last call's code and gr_last_error_message() a one-line reason.
 *   - Parameters travel as little-endian f64 values in schema order
 *     (crates/graph-contract/src/params.rs:154-170): an empty buffer means the
 *     defaults; a wrong length is refused (GR_PARAMS_MALFORMED); a non-finite,
 *     out-of-range, non-integral Int or non-0/1 Bool value is refused
 *     (GR_PARAM_OUT_OF_RANGE, index in gr_last_error_index()) and never clamped.
 *     The first five values are the reference's own FA2 schema
 *     (crates/graph-core/src/registry/tunable.rs:229-240); the rest are appended, so
 *     a reference-length (5-value) buffer keeps its meaning.
 *   - Buffers are copied in; the callee never frees a caller's buffer.
 *   - Positions are FP32, row-major n x dim, in topology node order
 *     (crates/graph-core/src/layout/mod.rs:54-66 Geometry columns, interleaved).
 */
#ifndef GRAPH_CUDA_H
#define GRAPH_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GR_ABI_VERSION 1

/* status codes (graph-wasm Code numbering; >= 100 are this library's own) */
#define GR_OK 0
#define GR_INVALID_HANDLE 1
#define GR_ALLOC_FAILED 2
#define GR_UNKNOWN_LAYOUT_ID 5
#define GR_LAYOUT_FAILED 8
#define GR_INDEX_OUT_OF_RANGE 12
#define GR_PARAM_OUT_OF_RANGE 20
#define GR_PARAMS_MALFORMED 21
#define GR_PARAMS_NOT_ACCEPTED 22
#define GR_INVALID_ARGUMENT 100
#define GR_CUDA_ERROR 101
#define GR_DEVICE_FAULT 102

/* parameter kinds (graph-contract ParamKind tags) */
#define GR_KIND_INT 0
#define GR_KIND_FLOAT 1
#define GR_KIND_BOOL 2

typedef struct gr_fa2 gr_fa2;

typedef struct gr_fa2_info {
    uint32_t n;              /* nodes */
    uint32_t dim;            /* 2 or 3 */
    uint64_t m;              /* simple edges */
    uint32_t iter_no;        /* ticks completed */
    uint32_t converged;      /* a tick moved the layout by < 1e-10 (state.rs:122-128) */
    uint32_t n_cells;        /* tree cells in the last tick */
    uint32_t n_leaves;       /* distinct keys (leaves) in the last tick */
    double swing, traction;  /* cumulative (state.rs:141-143) */
    double speed, speed_efficiency;
    double moved;            /* last tick's summed |step| */
    uint64_t far_count;      /* far-cell interactions since creation */
    uint64_t pair_count;     /* leaf pair interactions since creation */
    uint32_t device_error;   /* device error bits (1 non-finite, 2 tree, 4 bounds, 8 a bounded wait gave up) */
    uint32_t graph_kernels;  /* kernel launches in one captured tick (0 before the first tick) */
} gr_fa2_info;

/* ABI revision. */
uint32_t gr_abi_version(void);

/* Last call's status code, its one-line reason, and for GR_PARAM_OUT_OF_RANGE the
 * index of the refused value. Thread-local; reading them changes nothing. */
int gr_last_error(void);
const char *gr_last_error_message(void);
int gr_last_error_index(void);

/* Registry face (gm_layout_count / gm_layout_id, crates/graph-wasm/src/exports/build.rs:23-60). */
uint32_t gr_layout_count(void);
const char *gr_layout_id(uint32_t i);

/* Parameter schema (gm_layout_params; crates/graph-contract/src/params.rs:50-83 ParamSpec). */
uint32_t gr_fa2_param_count(void);
int gr_fa2_param_spec(uint32_t i, const char **name, int *kind, double *min, double *max,
                      double *def, double *step, const char **doc);
/* ParamsView::validate + values (crates/graph-contract/src/params.rs:147-170): writes
 * gr_fa2_param_count() values (defaults for the ones a short buffer leaves out). */
int gr_fa2_params_values(const uint8_t *params, size_t params_len, double *values_out);

/* Fa2State::new (crates/graph-core/src/layout/forceatlas2/state.rs:83-102) over a
 * topology's raw edges: self-loops dropped, parallel edges merged first-wins
 * (layout/force/mod.rs:101-120), mass = simple degree + 1. `weight` (nullable) is
 * the per-raw-edge weight the edge_weight_influence parameter raises; `pos0`
 * (nullable, n x dim) replaces the Mulberry32(seed) start (state.rs:272-283).
 * Device memory is allocated here and freed by gr_fa2_destroy. */
int gr_fa2_create(gr_fa2 **out, uint32_t n, uint64_t m, const uint32_t *src, const uint32_t *dst,
                  const double *weight, const uint8_t *params, size_t params_len, const float *pos0);
void gr_fa2_destroy(gr_fa2 *h);

/* Runs up to `ticks` ticks of Fa2State::iterate (state.rs:130-148), stopping early
 * once a tick moves the layout by < 1e-10 (state.rs:122-128). *done (nullable)
 * receives the ticks actually run. gr_fa2_run runs the max_iter parameter. */
int gr_fa2_tick(gr_fa2 *h, uint32_t ticks, uint32_t *done);
int gr_fa2_run(gr_fa2 *h, uint32_t *done);

/* Per-tick position buffer: runs up to `ticks` ticks and after each writes the
 * positions (row-major n x dim, FP32) to dev_out + t * n * dim, a DEVICE pointer. */
int gr_fa2_tick_record(gr_fa2 *h, uint32_t ticks, float *dev_out, uint32_t *done);

/* Measurement face: runs up to `ticks` ticks, each as three captured graphs
 * (tree build, repulsion walk, forces + update) bracketed by CUDA events on the
 * handle's stream, and writes 4 floats per tick to ms_out: tree, walk, finish and
 * whole-tick milliseconds. With l2_flush_bytes > 0 a buffer of that size is
 * overwritten before each tick, outside the events, so every tick starts with a
 * cold L2. No counterpart in the reference (which has no clock, stage.rs:4-8). */
int gr_fa2_tick_timed(gr_fa2 *h, uint32_t ticks, size_t l2_flush_bytes, float *ms_out, uint32_t *done);

/* Repulsion walk schedule: 0 = warp-cooperative (a warp visits the union of its 32
 * nodes' paths, one broadcast load per cell), 1 = per lane (each lane its own
 * path, gathered loads; the default in 2D), 2 = two adjacent nodes per lane over the
 * union of their two paths (the default in 3D), 3 = two independent per-lane walks per thread
 * (nodes 32 apart, stepped in turn, both cells' loads in flight together).
 * All give bit-identical forces.
 * gr_fa2_tune times sample_ticks ticks with each from the current state (restored
 * afterwards) and keeps the fastest; walk_ms_each (nullable, GR_WALK_SCHEDULES
 * floats) gets the mean walk time of each. */
#define GR_WALK_SCHEDULES 4
int gr_fa2_set_walk_schedule(gr_fa2 *h, int schedule);
/* Interaction counting (on = 1, the default): the walk adds every tick's far-cell
 * and exact-pair interaction counts to gr_fa2_info.far_count / pair_count. With
 * on = 0 the walk keeps no counts (fewer instructions per visited cell; the
 * forces are the same bit for bit) and the counters keep their values.
 * No counterpart in the reference (it counts nothing). */
int gr_fa2_set_interaction_counting(gr_fa2 *h, int on);
/* Launch mode of the tick's kernels: *programmatic = 1 when each is a programmatic
 * dependent launch (scheduled while the kernel before it drains, then waiting for
 * it before it reads anything; the default), 0 when they follow plain stream order
 * (GR_PDL=0 in the environment at create, or a capture with them failed).
 * No counterpart in the reference. */
int gr_fa2_launch_mode(gr_fa2 *h, int *programmatic);
int gr_fa2_tune(gr_fa2 *h, uint32_t sample_ticks, int *chosen, float *walk_ms_each);

/* Bounded waits and fault injection, for failure detection. No counterpart in the
 * reference (graph-core runs on one thread and never waits on another).
 * A tick's key sort is a one-sweep radix sort whose blocks wait for the digit
 * counts earlier blocks publish. Every such wait is bounded: after `spins`
 * sleeps of ~32 ns it gives up, sets device error bit 8 (ERR_WAIT), and the
 * tick's later kernels do nothing; the call returns GR_DEVICE_FAULT and the
 * handle stays halted (destroy it; other handles are unaffected).
 * gr_fa2_set_wait_limit sets `spins` for this handle's later ticks (0 restores
 * the default, 2^22). gr_fa2_inject_stalled_wait(h, 1) makes the second block
 * of every sort pass first wait for a device word that nothing ever sets, so
 * that wait runs out: the way a test drives the failure path without faulting
 * or hanging the GPU. (h, 0) removes the injection. */
int gr_fa2_set_wait_limit(gr_fa2 *h, uint32_t spins);
int gr_fa2_inject_stalled_wait(gr_fa2 *h, int on);

/* Current positions to a host buffer (n x dim), refusing non-finite ones as
 * `settle` does (crates/graph-core/src/layout/forceatlas2.rs:82-91). */
int gr_fa2_positions(gr_fa2 *h, float *out);
/* Replace the positions (host, n x dim). */
int gr_fa2_set_positions(gr_fa2 *h, const float *pos);
/* Device view of the node records: float4 {x, y, z, mass} per node, valid until the
 * next tick or destroy. */
int gr_fa2_positions_device(gr_fa2 *h, const void **dev_nodes);

/* One force evaluation at the current positions, without moving anything: the
 * tick's accumulator u = attraction + repulsion - gravity (state.rs:130-137),
 * n x dim to a host buffer. */
int gr_fa2_forces(gr_fa2 *h, float *out);

int gr_fa2_get_info(gr_fa2 *h, gr_fa2_info *out);

/* Checkpoint / resume: the FP64 speed controller (state.rs:151-171's swing,
 * traction, speed, speed_efficiency, iter_no). With gr_fa2_positions /
 * gr_fa2_set_positions it is the whole state a run carries from tick to tick. */
typedef struct gr_fa2_controller {
    double swing, traction, speed, speed_efficiency;
    uint32_t iter_no, converged;
} gr_fa2_controller;
int gr_fa2_get_controller(gr_fa2 *h, gr_fa2_controller *out);
int gr_fa2_set_controller(gr_fa2 *h, const gr_fa2_controller *in);

/* Adjoint (vector-Jacobian product) of a run, through each tick's tree (its far /
 * pair decisions held fixed; cell centres move with their points) and the speed
 * controller's active branch. No counterpart in the reference.
 * gr_fa2_adjoint_forward runs `ticks` ticks from the current state, recording
 * positions and controller every `checkpoint_every` ticks; gr_fa2_adjoint_backward
 * takes dL/d(final positions) (host, n x dim) and returns dL/d(start positions)
 * (host, n x dim, FP64) and, when dL_dw is not NULL, dL/d(raw edge weight) (host,
 * m; 0 for a self-loop or a repeated pair), replaying each segment from its
 * checkpoint. The carried adjoint is FP32 under a running power-of-two scale, so
 * gradients that outgrow FP32 over a long run (they grow by orders of magnitude
 * per tick) come back in FP64; GR_LAYOUT_FAILED if they outgrow FP64.
 * The handle is left at the end of the recorded run. */
int gr_fa2_adjoint_forward(gr_fa2 *h, uint32_t ticks, uint32_t checkpoint_every);
int gr_fa2_adjoint_backward(gr_fa2 *h, const float *dL_dpT, double *dL_dp0, double *dL_dw);

/* The FP32 FMA rate of the current device at its present clocks, in TFLOP/s (an
 * FMA counted as two operations): a kernel of 8 independent FMA chains per thread,
 * 64 resident warps per SM, `iters` steps each, timed with CUDA events after one
 * warm-up launch. The denominator of the repulsion walk's roofline. No
 * counterpart in the reference. */
int gr_measure_fp32_rate(uint32_t iters, double *tflops);

/* Multi-source BFS on the device: hop counts from k source nodes to every node
 * (host out, k x n, UINT32_MAX when unreachable) over the raw edges (source,
 * target), undirected, self-loops ignored. No counterpart in the reference, whose
 * stress runs one queue BFS per source on the host (graph-cli/src/bench.rs:264-277). */
int gr_bfs_hops(uint32_t n, uint64_t m, const uint32_t *source, const uint32_t *target, uint32_t k,
                const uint32_t *sources, uint32_t *hops_out);

/* Kruskal stress-1 of positions (x, y) against hop distance, the reference's
 * quality measure (graph-cli/src/bench.rs:255-295 `stress`, called with its
 * SOURCES = 16): BFS from every max(n / sources, 1)-th node, FP64 sums over every
 * reachable (source, target) pair, stress = sqrt(max((DD - DE/EE*DE) / DD, 0)), and
 * 1.0 for a collapsed layout or an edgeless graph. */
int gr_stress(uint32_t n, uint64_t m, const uint32_t *source, const uint32_t *target, const float *x, const float *y,
              uint32_t sources, double *out);

/* d3-force Barnes-Hut session (2D), the layout behind graph-core's
 * `layout.force.barnes_hut` (crates/graph-core/src/layout/force/barnes_hut.rs,
 * barnes_hut/sim.rs:170-270 tick) and the per-tick surface of the reference's live
 * session (crates/graph-core/src/layout/force/session.rs; graph-wasm
 * gm_force_session_*, docs/contract/wasm-abi.md): link, many-body over the
 * quadtree, center, collide, integrate, from the golden spiral (seed.rs) unless
 * pos0 (n x 2) is given. FP32 positions and velocities on the device.
 * gr_force_params mirrors params.rs ForceParams; gr_force_default_params fills its
 * defaults (params.rs:60-75), and a NULL params means those. strength (m, NULL:
 * 1) is each raw edge's strength; the first raw edge of a pair keeps it. */
typedef struct gr_force_session gr_force_session;
typedef struct gr_force_params {
    double charge, theta, distance_min, distance_max, link_distance, link_strength_scale, collide_radius,
        center_strength, velocity_decay, alpha_decay, alpha_min, initial_alpha;
} gr_force_params;
#define GR_FORCE_TICKS 112 /* params.rs TICKS: the frozen layout's tick count */
void gr_force_default_params(gr_force_params *out);
int gr_force_session_create(gr_force_session **out, uint32_t n, uint64_t m, const uint32_t *src, const uint32_t *dst,
                            const double *strength, const gr_force_params *params, const float *pos0);
void gr_force_session_destroy(gr_force_session *s);
int gr_force_session_tick(gr_force_session *s, uint32_t ticks);
/* The same ticks with their device time: *ms receives the milliseconds between
 * CUDA events recorded on the session's stream before the first tick and after
 * the last. No counterpart in the reference (which has no clock). */
int gr_force_session_tick_timed(gr_force_session *s, uint32_t ticks, float *ms);
int gr_force_session_positions(gr_force_session *s, float *out);
int gr_force_session_velocities(gr_force_session *s, float *out);
/* alpha after the ticks so far, and how many ticks have run. */
int gr_force_session_alpha(gr_force_session *s, double *alpha, uint32_t *ticks_done);
/* session.rs:247-251 reheat: alpha set outright, a finite value in [0, 1], never clamped. */
int gr_force_session_reheat(gr_force_session *s, double alpha);
/* Carries a state into the session (the reference session's columns handed over,
 * session/carry.rs): positions and velocities (n x 2 each; NULL keeps the session's
 * own), alpha (a finite value in [0, 1]) and the tick count the jiggle is keyed on. */
int gr_force_session_set_state(gr_force_session *s, const float *pos, const float *vel, double alpha,
                               uint32_t ticks_done);
/* ForceSession::with_particle_mesh (crates/graph-core/src/layout/force/
 * particle_mesh.rs): from the next tick on, the session's many-body pass runs on
 * a side x side FFT mesh (side the power of two of ceil(sqrt(n)) in [128, 1024])
 * instead of the tree; link, center, collide and the integration are unchanged. */
int gr_force_session_use_mesh(gr_force_session *s);
/* The frozen particle-mesh layout (ParticleMesh::run, particle_mesh.rs): a default
 * session on the mesh, GR_FORCE_TICKS ticks, positions (n x 2) into out. */
int gr_force_mesh_run(uint32_t n, uint64_t m, const uint32_t *src, const uint32_t *dst, const double *strength,
                      float *out);
/* Kernels in the captured tick graph, and the cell count of the last tree. */
int gr_force_session_info(gr_force_session *s, uint32_t *graph_kernels, uint32_t *n_cells);
/* The frozen layout (BarnesHut::run, barnes_hut.rs:134-140): default parameters,
 * GR_FORCE_TICKS ticks from the golden spiral, positions (n x 2) into out. */
int gr_force_run(uint32_t n, uint64_t m, const uint32_t *src, const uint32_t *dst, const double *strength,
                 float *out);

/* The stream every call of this handle enqueues on (default: the handle's own). */
int gr_fa2_set_stream(gr_fa2 *h, void *cuda_stream);

/* Allocation-free force evaluation. No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc: code that runs inside another GPU
 * runtime which owns every device allocation (its own pool or stream-ordered
 * allocator), or a plugin that is only handed device buffers by its host. It
 * computes what gr_fa2_forces computes (u = attraction + repulsion - gravity at
 * the given positions; the same tree build and walk) but takes every input and
 * output as device memory and keeps its scratch in a fixed array compiled into
 * this library, sized for GR_FORCES_STATIC_MAX_N nodes (about 14 MB, held on
 * every GPU that loads the library until the process exits). It calls no
 * cudaMalloc, cudaFree or other allocating routine.
 *
 *   nodes    device, n x float4 {x, y, z (0 in 2D), mass}; FA2's mass is degree + 1
 *   row_ptr  device, n + 1 CSR offsets over both endpoints of every simple edge
 *   col      device, neighbour per CSR entry (non-null even for an edgeless graph)
 *   weight   device, attraction weight per CSR entry, already raised to the
 *            edge_weight_influence power by the caller (1.0 for unit weights);
 *            non-null even for an edgeless graph
 *   params   host, the usual parameter buffer (dim, theta, scaling, gravity,
 *            lin_log, strong_gravity, dissuade_hubs are read; max_iter,
 *            jitter_tolerance and edge_weight_influence are not)
 *   tick     the tick number the coincident-pair jiggle is keyed on
 *   out      device, n x dim forces
 *   stream   the CUDA stream to enqueue on (NULL = legacy default stream)
 *
 * Enqueued asynchronously; the return value reports argument refusals only (n
 * beyond GR_FORCES_STATIC_MAX_N or a null device buffer is refused with
 * GR_INVALID_ARGUMENT). Device-side failures are read afterwards with
 * gr_fa2_forces_static_status: with a non-finite position the evaluation stops
 * early and leaves `out` as it was. The kernels are programmatic dependent
 * launches unless GR_PDL=0 is set in the environment. The first call on each
 * device looks up the array's device address (cudaGetSymbolAddress, with that
 * device current) and keeps it for that device's context (a new context, after
 * cudaDeviceReset, is looked up again): make that first call before any stream
 * capture. Every call shares the one array and it keeps the last call's
 * contents (each call initialises what it reads), so calls that overlap on the
 * GPU (different streams, or different host threads on the same device) race
 * and corrupt each other's results; serialise them on one stream. */
#define GR_FORCES_STATIC_MAX_N 32768
int gr_fa2_forces_static(uint32_t n, const void *nodes, const uint32_t *row_ptr, const uint32_t *col,
                         const float *weight, const uint8_t *params, size_t params_len, uint32_t tick,
                         float *out, void *stream);

/* The outcome of the last gr_fa2_forces_static evaluation on the current
 * device, read from the static array (a 4-byte device-to-host copy; nothing is
 * allocated). Call it once the stream that evaluation ran on has been
 * synchronised. *device_error (nullable) receives the device error bits (those
 * of gr_fa2_info's device_error; 0 before any evaluation). Returns GR_OK when
 * the bits are 0, GR_LAYOUT_FAILED when a position was non-finite, and
 * GR_DEVICE_FAULT for any other bit. */
int gr_fa2_forces_static_status(uint32_t *device_error);

/* Batched layouts: many independent graphs in one persistent launch (one CTA per
 * graph at a time, largest first; every tick of a graph inside its CTA). No
 * counterpart in the reference, which lays out one graph per call.
 *
 *   node_counts[g], edge_counts[g]   sizes of graph g
 *   src, dst                         concatenated raw edges, node ids local to their graph
 *   weight                           concatenated raw edge weights (nullable)
 *   params                           params_per_graph (0, 5 or 11) f64 values per graph,
 *                                    validated like a parameter buffer; every graph has
 *                                    the same dim
 *   pos0                             concatenated n x dim start positions (nullable:
 *                                    Mulberry32(seed of the graph) per graph) */
typedef struct gr_fa2_batch gr_fa2_batch;
int gr_fa2_batch_create(gr_fa2_batch **out, uint32_t graphs, const uint32_t *node_counts,
                        const uint64_t *edge_counts, const uint32_t *src, const uint32_t *dst,
                        const double *weight, const double *params, uint32_t params_per_graph,
                        const float *pos0);
void gr_fa2_batch_destroy(gr_fa2_batch *b);
/* CTA size of the persistent kernel: 256, 512 (default) or 1024 threads. */
int gr_fa2_batch_set_threads(gr_fa2_batch *b, int threads);
/* Autotuner: times sample_ticks ticks of the whole batch at each CTA size on a copy
 * of the state (restored afterwards) and keeps the fastest; ms_each (nullable, 3
 * floats) receives the times for 256, 512, 1024. */
int gr_fa2_batch_tune(gr_fa2_batch *b, uint32_t sample_ticks, int *chosen, float *ms_each);
/* Runs every graph up to `ticks` ticks (a converged graph stops) in one persistent
 * launch, captured once into a CUDA graph; *ms (nullable) receives its device time. */
int gr_fa2_batch_run(gr_fa2_batch *b, uint32_t ticks, float *ms);
/* Concatenated positions (sum of n x dim), graph order. */
int gr_fa2_batch_positions(gr_fa2_batch *b, float *out);
/* Per graph: ticks done, device error bits, far and pair interaction counts (2 per
 * graph); any pointer may be NULL. */
int gr_fa2_batch_stats(gr_fa2_batch *b, uint32_t *ticks_done, uint32_t *errors, uint64_t *interactions);

/* One-shot registry run, Capability::run_params (crates/graph-core/src/registry/params.rs:156-181):
 * create, run max_iter, write n x dim positions to a host buffer, destroy. */
int gr_run(const char *layout_id, uint32_t n, uint64_t m, const uint32_t *src, const uint32_t *dst,
           const double *weight, const uint8_t *params, size_t params_len, float *out);

#ifdef __cplusplus
}
#endif

#endif /* GRAPH_CUDA_H */
