"""GPU parity: the CUDA engine (through the C ABI) against the FP64 oracle.

Per-tick forces from identical positions must match within 1e-5 relative L2 on
the same tree (the oracle's insertion tree capped at the engine's Morton depth)
and the same theta. Integer structure (cell count, interaction counts) must
match the oracle's exactly or to the few borderline far tests FP32 can flip.
"""

import numpy as np
import pytest

from oracle import oracle as O
from graph_render_b200 import Fa2, synth
from tests.gpu_util import collapsed_cells, force_parity, oracle_state, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _check(n, src, dst, w, pos, prm, tol=TOL):
    rel, info, sc = force_parity(n, src, dst, w, pos, prm)
    assert info["device_error"] == 0
    assert rel < tol, rel
    return rel, info, sc


def test_sbm1500_forces_match_oracle():
    wl = synth.sbm_1500()
    rel, info, sc = _check(wl.n, wl.src, wl.dst, wl.weight, wl.pos0, wl.params)
    # the same tree: same cell count, and the same interactions up to FP32 borderline flips
    st = oracle_state(wl.n, wl.src, wl.dst, wl.weight, wl.pos0, wl.params)
    st.accumulate(7)
    assert info["n_cells"] == collapsed_cells(st)
    far_ref, pair_ref = st.scalars()["far"], st.scalars()["pair"]
    assert abs(info["far_count"] - far_ref) <= 1e-3 * far_ref + 2
    assert abs(info["pair_count"] - pair_ref) <= 1e-3 * pair_ref + 2


def test_sbm1500_forces_match_after_clustering():
    wl = synth.sbm_1500()
    with Fa2(wl.n, wl.src, wl.dst, params=wl.params, pos0=wl.pos0) as eng:
        eng.tick(60)
        pos = eng.positions()
    _check(wl.n, wl.src, wl.dst, None, pos, wl.params)


@pytest.mark.parametrize("gate_n", [2, 3, 5, 17, 64, 300, 601])
def test_gate_model_default_params(gate_n):
    s, d, _ = O.gate_edges(gate_n)
    pos = O.initial_positions(gate_n, 0, 2).astype(np.float32)
    _check(gate_n, s, d, None, pos, dict(theta=0.8))


def test_ba_linlog_dissuade_weighted():
    wl = synth.ba_100k(n=20_000)
    _check(wl.n, wl.src, wl.dst, wl.weight, wl.pos0, wl.params)


def test_powerlaw_3d_strong_gravity():
    wl = synth.powerlaw_1m(n=50_000, dim=3)
    _check(wl.n, wl.src, wl.dst, None, wl.pos0, wl.params)


def test_theta_zero_is_the_exact_sum():
    wl = synth.sbm_1500()
    prm = dict(wl.params, theta=0.0)
    rel, info, _ = force_parity(wl.n, wl.src, wl.dst, None, wl.pos0, prm, dense_oracle=True)
    assert rel < TOL
    assert info["far_count"] == 0 and info["pair_count"] == wl.n * (wl.n - 1)


def test_coincident_points_take_the_jiggle():
    rng = np.random.default_rng(4)
    n = 3000
    pos = np.round(rng.uniform(0, 40, (n, 2))).astype(np.float32)  # many exact duplicates
    s, d = synth.sbm([n], 0.002, 0.0, 9)
    _check(n, s, d, None, pos, dict(theta=1.2, seed=5))


def test_3d_coincident_and_theta0():
    rng = np.random.default_rng(6)
    n = 2000
    pos = np.round(rng.uniform(0, 12, (n, 3))).astype(np.float32)
    s, d = synth.ba(n, 2, 3)
    rel, info, _ = force_parity(n, s, d, None, pos, dict(dim=3, theta=0.0), dense_oracle=True)
    assert rel < TOL


def test_large_2d_powerlaw_forces():
    wl = synth.powerlaw_1m(n=1_000_000, dim=2)
    rel, info, sc = _check(wl.n, wl.src, wl.dst, None, wl.pos0, wl.params)
    assert abs(info["far_count"] - sc["far"]) <= 1e-3 * sc["far"]


def test_ba_100k_linlog_dissuade_weighted_full_size():
    # the 100k-node BA workload at its own size: lognormal weights, linlog,
    # dissuade hubs, theta 1.0
    wl = synth.ba_100k()
    rel, info, sc = _check(wl.n, wl.src, wl.dst, wl.weight, wl.pos0, wl.params)
    assert abs(info["far_count"] - sc["far"]) <= 1e-3 * sc["far"]


def test_powerlaw_1m_3d_strong_gravity_full_size():
    # the 1M-node octree workload at its own size: strong gravity, theta 1.2
    wl = synth.powerlaw_1m(n=1_000_000, dim=3)
    rel, info, sc = _check(wl.n, wl.src, wl.dst, None, wl.pos0, wl.params)
    assert abs(info["far_count"] - sc["far"]) <= 1e-3 * sc["far"]


def test_large_2d_forces_with_one_block_tile_carries():
    # past 2,048 tiles of 1,024 sorted points the leaf pass's tile carries come
    # from one block (k_leaf_carry) instead of each tile's own fold
    wl = synth.powerlaw_1m(n=2_200_000, dim=2)
    rel, info, sc = _check(wl.n, wl.src, wl.dst, None, wl.pos0, wl.params)
    assert abs(info["far_count"] - sc["far"]) <= 1e-3 * sc["far"]


def test_forces_past_the_one_pass_scan_limit():
    # past 2,048 scan blocks of 2,048 leaves (~4.2M distinct keys) the cell-level
    # scan runs as reduce / block-scan / downsweep, and the tile carries come from
    # one block: both fallbacks against the oracle
    wl = synth.powerlaw_1m(n=4_500_000, dim=2)
    rel, info, sc = _check(wl.n, wl.src, wl.dst, None, wl.pos0, wl.params)
    assert info["n_leaves"] > 2048 * 2048
    assert abs(info["far_count"] - sc["far"]) <= 1e-3 * sc["far"]


def test_run_is_deterministic():
    wl = synth.sbm_1500()
    outs = []
    for _ in range(2):
        with Fa2(wl.n, wl.src, wl.dst, params=wl.params, pos0=wl.pos0) as eng:
            eng.tick(100)
            outs.append(eng.positions())
    assert np.array_equal(outs[0], outs[1])
    assert np.isfinite(outs[0]).all()


def test_early_exit_when_nothing_moves():
    n = 50
    pos = synth.uniform(n, 2, 0, 10, 1)
    with Fa2(n, [], [], params=dict(gravity=0.0, scaling_ratio=0.0), pos0=pos) as eng:
        done = eng.tick(10)
        assert done == 1
        assert eng.info()["converged"] == 1
        assert np.array_equal(eng.positions(), pos)


def test_empty_and_single_node():
    with Fa2(0, [], []) as eng:
        assert eng.tick(5) == 0
        assert eng.positions().shape == (0, 2)
    with Fa2(1, [], []) as eng:
        eng.tick(100)
        assert np.isfinite(eng.positions()).all()


def test_trajectory_tracks_the_oracle_for_a_few_ticks():
    """Two ticks (the reference's gated budget): FP32 engine vs FP64 oracle."""
    wl = synth.sbm_1500()
    with Fa2(wl.n, wl.src, wl.dst, params=wl.params, pos0=wl.pos0) as eng:
        eng.tick(2)
        g = eng.positions().astype(np.float64)
    st = oracle_state(wl.n, wl.src, wl.dst, None, wl.pos0, wl.params)
    st.run(2)
    r = st.positions()
    ext = (r.max(0) - r.min(0)).max()
    assert np.abs(g - r).max() / ext < 1e-4


@pytest.mark.parametrize("case", ["sbm1500", "ba5k", "powerlaw5k_3d"])
def test_full_run_matches_the_oracle_on_energy_and_stress(case):
    """Whole runs diverge chaotically, so the finished layouts are compared on
    the FA2 energy (each term) and the sampled Kruskal stress, within 1%."""
    from graph_render_b200 import quality

    wl = {"sbm1500": synth.sbm_1500, "ba5k": lambda: synth.ba_100k(n=5000),
          "powerlaw5k_3d": lambda: synth.powerlaw_1m(n=5000, dim=3)}[case]()
    ticks = 100
    prm = dict(wl.params, max_iter=ticks)
    with Fa2(wl.n, wl.src, wl.dst, wl.weight, params=prm, pos0=wl.pos0) as eng:
        eng.run()
        g = eng.positions().astype(np.float64)
    st = oracle_state(wl.n, wl.src, wl.dst, wl.weight, wl.pos0, wl.params)
    st.run(ticks)
    r = st.positions()
    eg = quality.fa2_energy(g, wl.src, wl.dst, wl.weight, prm)
    er = quality.fa2_energy(r, wl.src, wl.dst, wl.weight, prm)
    for term in ("attraction", "repulsion", "gravity", "total"):
        assert abs(eg[term] - er[term]) <= 1e-2 * abs(er[term]), (term, eg[term], er[term])
    if g.shape[1] == 3:
        return  # the stress measure is the reference's 2D one
    sg = O.stress(g[:, 0], g[:, 1], wl.src, wl.dst, 16)
    sr = O.stress(r[:, 0], r[:, 1], wl.src, wl.dst, 16)
    assert abs(sg - sr) <= 1e-2 * sr, (sg, sr)


@pytest.mark.slow
@pytest.mark.parametrize("case", ["ba100k_500", "powerlaw1m_3d_300", "powerlaw1m_2d_100", "gate1m_defaults_100"])
def test_full_run_at_the_workloads_own_size(case):
    """Whole runs at the workloads' own sizes and tick counts: the 100k-node BA
    graph (linlog, dissuade hubs, lognormal weights, theta 1.0) for 500 ticks,
    the 1M-node 3D octree graph (strong gravity, theta 1.2) for 300 ticks, the
    bench's 1M-node 2D graph (theta 1.2) for 100 ticks, and the reference's own
    benchmark (its 1M-node gate model through the registry call with an empty
    parameter buffer: theta 0.8, 100 iterations, the Mulberry32(0) start the
    engine draws itself), against the oracle's FP64 runs on each energy term
    (repulsion estimated from 2^25 pairs, the same pairs for both layouts) and, in
    2D, the Kruskal stress from 16 BFS sources (the reference's measure,
    graph-cli/src/bench.rs:255-295), within 1%."""
    import time

    from graph_render_b200 import FA2_ID, Topology, find, quality

    if case == "ba100k_500":
        wl, ticks = synth.ba_100k(), 500
    elif case == "powerlaw1m_3d_300":
        wl, ticks = synth.powerlaw_1m(n=1_000_000, dim=3), 300
    elif case == "powerlaw1m_2d_100":
        wl, ticks = synth.powerlaw_1m(n=1_000_000, dim=2), 100
    else:
        wl, ticks = None, 100
    if wl is None:  # the drop-in call: no positions, default parameters
        n = 1_000_000
        src, dst, strength = synth.gate(n)
        geom = find(FA2_ID).run_params(Topology(n, src, dst, strength), b"")
        g = np.column_stack([np.asarray(geom.x, np.float64), np.asarray(geom.y, np.float64)])

        class W:
            pass

        wl = W()
        wl.n, wl.src, wl.dst, wl.weight = n, src, dst, None
        wl.pos0 = O.initial_positions(n, 0, 2).astype(np.float32)
        wl.params = dict(theta=0.8, dim=2, seed=0)
    else:
        prm = dict(wl.params, max_iter=ticks)
        with Fa2(wl.n, wl.src, wl.dst, wl.weight, params=prm, pos0=wl.pos0) as eng:
            assert eng.run() == ticks
            g = eng.positions().astype(np.float64)
    prm = dict(wl.params, max_iter=ticks)
    t0 = time.time()
    st = oracle_state(wl.n, wl.src, wl.dst, wl.weight, wl.pos0, wl.params)
    st.run(ticks)
    r = st.positions()
    t_oracle = time.time() - t0
    eg = quality.fa2_energy(g, wl.src, wl.dst, wl.weight, prm, pair_sample=1 << 25, seed=7)
    er = quality.fa2_energy(r, wl.src, wl.dst, wl.weight, prm, pair_sample=1 << 25, seed=7)
    gaps = {t: abs(eg[t] - er[t]) / abs(er[t]) for t in ("attraction", "repulsion", "gravity", "total")}
    if g.shape[1] == 2:
        sg = O.stress(g[:, 0], g[:, 1], wl.src, wl.dst, 16)
        sr = O.stress(r[:, 0], r[:, 1], wl.src, wl.dst, 16)
        gaps["stress"] = abs(sg - sr) / sr
    print(f"{case}: oracle {t_oracle:.1f} s; relative gaps " + ", ".join(f"{k} {v:.2e}" for k, v in gaps.items()))
    for k, v in gaps.items():
        assert v <= 1e-2, (k, v, gaps)


@pytest.mark.parametrize("dim", [2, 3])
def test_walk_schedules_give_bit_identical_forces_and_tuning_keeps_the_state(dim):
    wl = synth.powerlaw_1m(n=200_000, dim=dim)
    outs = []
    with Fa2(wl.n, wl.src, wl.dst, params=wl.params, pos0=wl.pos0) as eng:
        eng.tick(3)
        pos = eng.positions()
        for sch in (0, 1, 2, 3):
            eng.set_walk_schedule(sch)
            f0 = eng.info()["far_count"]
            outs.append((eng.forces(), eng.info()["far_count"] - f0))
        chosen, ms = eng.tune(2)
        assert chosen in (0, 1, 2, 3) and all(ms[i] > 0 for i in (0, 1, 2, 3))
        assert np.array_equal(eng.positions(), pos)
    for sch in (1, 2, 3):
        assert np.array_equal(outs[0][0], outs[sch][0])
        assert outs[0][1] == outs[sch][1]


@pytest.mark.parametrize("dim", [2, 3])
def test_walk_without_interaction_counts_gives_the_same_forces_and_run(dim):
    wl = synth.powerlaw_1m(n=100_000, dim=dim)
    with Fa2(wl.n, wl.src, wl.dst, params=wl.params, pos0=wl.pos0) as eng:
        eng.tick(2)
        ref = eng.forces()
        far = eng.info()["far_count"]
        assert far > 0
        eng.set_interaction_counting(False)
        for sch in (0, 1, 2, 3):
            eng.set_walk_schedule(sch)
            assert np.array_equal(eng.forces(), ref)
        eng.tick(2)
        assert eng.info()["far_count"] == far  # no counts while off
    ends = []
    for on in (True, False):
        with Fa2(wl.n, wl.src, wl.dst, params=wl.params, pos0=wl.pos0) as eng:
            eng.set_interaction_counting(on)
            eng.tick(5)
            ends.append(eng.positions())
    assert np.array_equal(ends[0], ends[1])


@pytest.mark.parametrize("dim", [2, 3])
def test_programmatic_launches_give_the_same_run(dim, monkeypatch):
    # each tick kernel waits for the one before it in gr_pdl_enter: the ticks are
    # those of plain stream order bit for bit (GR_PDL=0 is read at create)
    wl = synth.powerlaw_1m(n=200_000, dim=dim)
    ends = []
    for pdl in ("1", "0"):
        monkeypatch.setenv("GR_PDL", pdl)
        with Fa2(wl.n, wl.src, wl.dst, params=wl.params, pos0=wl.pos0) as eng:
            assert eng.programmatic_launches() == (pdl == "1")
            eng.tick(4)
            ends.append((eng.positions(), eng.forces(), eng.info()["far_count"]))
    assert np.array_equal(ends[0][0], ends[1][0])
    assert np.array_equal(ends[0][1], ends[1][1])
    assert ends[0][2] == ends[1][2]


@pytest.mark.parametrize("dim", [2, 3])
def test_update_bounds_equal_the_bounds_pass(dim):
    # a tick's update also computes the next tick's root square and mean; setting
    # the positions again makes the bounds pass recompute them: the runs agree bit
    # for bit
    wl = synth.powerlaw_1m(n=150_000, dim=dim)
    ends = []
    for reset in (False, True):
        with Fa2(wl.n, wl.src, wl.dst, params=wl.params, pos0=wl.pos0) as eng:
            eng.tick(3)
            if reset:
                eng.set_positions(eng.positions())
            eng.tick(3)
            ends.append((eng.positions(), eng.info()["moved"]))
    assert np.array_equal(ends[0][0], ends[1][0])
    assert ends[0][1] == ends[1][1]


def _full_sort_forces(n, src, dst, pos, prm):
    """Forces through gr_fa2_forces_static, which sorts the whole 64-bit key
    (8 passes) where a handle sorts the high word and fixes the runs."""
    import ctypes as C

    import torch

    from graph_render_b200 import _native as N, params_bytes
    from tests.test_zz_no_alloc import csr

    dim = int(prm.get("dim", 2))
    rp, col, wts, mass = csr(n, src, dst, None)
    nodes = np.zeros((n, 4), np.float32)
    nodes[:, :dim] = pos
    nodes[:, 3] = mass
    dev = torch.device("cuda", 0)
    col = col if len(col) else np.zeros(1, np.int32)
    t = [torch.from_numpy(a).to(dev) for a in (nodes, rp, col, np.ones(len(col), np.float32))]
    out = torch.zeros((n, dim), dtype=torch.float32, device=dev)
    pb = params_bytes(prm)
    N.check(N.lib().gr_fa2_forces_static(n, *[C.c_void_p(x.data_ptr()) for x in t], C.c_char_p(pb), len(pb), 0,
                                         C.c_void_p(out.data_ptr()),
                                         C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)))
    torch.cuda.synchronize(dev)
    return out.cpu().numpy()


def _uniform_graph(n, dim, seed, cluster=0, spread=0.0):
    """n points uniform in [0, 1000)^dim, the first `cluster` of them moved onto
    one point (spread 0) or into a cube of side `spread` around it, and 2n
    uniform random edges (degrees far below the 64 at which a handle splits a
    row's attraction into segments, which the allocation-free path does not)."""
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0, 1000, (n, dim)).astype(np.float32)
    if cluster:
        pos[:cluster] = pos[0]
        if spread:
            pos[1:cluster] += rng.uniform(0, spread, (cluster - 1, dim)).astype(np.float32)
    src = rng.integers(0, n, 2 * n).astype(np.uint32)
    dst = rng.integers(0, n, 2 * n).astype(np.uint32)
    return pos, src, dst


def _fast_equals_full(n, dim, pos, src, dst):
    prm = dict(dim=dim, theta=1.0, seed=3)
    with Fa2(n, src, dst, params=prm, pos0=pos) as eng:
        fast = eng.forces()
        assert eng.info()["device_error"] == 0
    full = _full_sort_forces(n, src, dst, pos, prm)
    assert np.array_equal(fast, full)


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("n", [4_096, 12_000, 32_768])
@pytest.mark.parametrize("cluster,spread", [(0, 0.0), (300, 0.0), (40, 1e-3), (3000, 1e-3)])
def test_one_sweep_sort_with_run_fixup_equals_the_full_sort(dim, n, cluster, spread):
    """Above 3,072 nodes a handle sorts the keys' top digits with one-sweep
    passes and then puts each run of equal sorted bits in full-key order in
    place: one thread's insertion sort up to 64 keys (the 40-point cluster), one
    CTA's block sort above (300 coincident points: equal keys, kept in index
    order; 3,000 distinct points in a cube of side 1e-3, which share the sorted
    bits). The order must be the full 64-bit stable sort's, which the
    allocation-free path computes with all 8 digits, so the forces are
    bit-identical."""
    pos, src, dst = _uniform_graph(n, dim, 11 + cluster + dim + n, cluster, spread)
    _fast_equals_full(n, dim, pos, src, dst)


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("n,cluster,spread", [(3072, 0, 0.0), (3072, 500, 0.0), (3072, 500, 1e-3), (1200, 70, 0.0),
                                              (2, 0, 0.0), (1, 0, 0.0)])
def test_small_graph_sort_equals_the_full_sort(dim, n, cluster, spread):
    """Up to 3,072 nodes a tick's keys and sort run as one CTA in shared memory
    (two passes on the top 16 bits, then runs of equal sorted bits, up to the 500-point clusters here
    by the block's own sort); the order must be the full 64-bit stable sort's
    (the allocation-free path sorts all 8 digits), so the forces are identical."""
    pos, src, dst = _uniform_graph(n, dim, n + cluster + dim, cluster, spread)
    _fast_equals_full(n, dim, pos, src, dst)


@pytest.mark.parametrize("dim", [2, 3])
def test_engine_result_flows_through_the_snapshot_encoder(dim):
    """run_params (the registry face) -> Geometry -> the snapshot's binary face ->
    decode: the f32 columns come back bit for bit, in the topology's order."""
    from graph_render_b200 import Topology, find, params_bytes
    from graph_render_b200 import snapshot as S

    n = 300
    src, dst, st = O.gate_edges(n)
    topo = Topology(n, src, dst, st)
    geom = find("layout.forceatlas2.barnes_hut.cuda").run_params(topo, params_bytes(dim=dim, max_iter=50))
    node_ids, edge_ids = S.gate_ids(n, len(src))
    snap = S.of_geometry(node_ids, edge_ids, topo, geom)
    b = snap.to_bytes()
    back = S.from_bytes(b)
    assert back.to_bytes() == b and back.dim == dim
    assert np.array_equal(back.x.view(np.uint32), np.asarray(geom.x, np.float32).view(np.uint32))
    assert np.array_equal(back.y.view(np.uint32), np.asarray(geom.y, np.float32).view(np.uint32))
    assert np.array_equal(back.source, src) and np.array_equal(back.target, dst)
    assert b[8:12] == (b"\x04\0\0\0" if dim == 3 else b"\x03\0\0\0")


def test_the_fp32_rate_is_measured():
    # the repulsion walk's roofline denominator: eight FMA chains a thread, timed
    # on the device; B200's nominal FP32 FMA rate is 74.4 TFLOP/s at 1,965 MHz
    import ctypes as C

    from graph_render_b200 import _native as N

    v = C.c_double()
    N.check(N.lib().gr_measure_fp32_rate(50_000, C.byref(v)))
    assert 20.0 < v.value < 100.0, v.value
    assert N.lib().gr_measure_fp32_rate(0, C.byref(v)) == N.GR_INVALID_ARGUMENT


@pytest.mark.parametrize("dim", [2, 3])
def test_recorded_run_builds_the_same_cells_as_a_plain_run(dim):
    """A run recorded for the adjoint builds its trees with the radix tree's
    full arrays and the leaf and node body kernels; a plain run keeps only the
    packed records. Clusters of coincident points make leaves whose level comes
    from their parent: both runs must give the same positions bit for bit."""
    n = 6000
    pos, src, dst = _uniform_graph(n, dim, 77 + dim, cluster=400)
    pos[1000:1100] = pos[1000]
    prm = dict(dim=dim, theta=1.0, seed=5)
    with Fa2(n, src, dst, params=prm, pos0=pos) as a, Fa2(n, src, dst, params=prm, pos0=pos) as b:
        a.adjoint_forward(6, every=3)
        b.tick(6)
        assert np.array_equal(a.positions(), b.positions())
