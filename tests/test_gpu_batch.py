"""The batched persistent kernel against the one-graph engine and the oracle.

Every graph of a batch is an independent FA2 run; the persistent kernel runs
the same per-item functions as the one-graph engine at block scope, so after a
tick each graph's positions match the one-graph engine's (the FP64 sums fold in
a different order, hence a tolerance) and the oracle's within the parity bar.
"""

import numpy as np
import pytest

from graph_render_b200 import Fa2, batch, synth
from tests.gpu_util import oracle_state

pytestmark = pytest.mark.gpu


def small_mix(count=48, seed=11, nmax=3000):
    return [batch.mixed_graph(seed, i, nmin=2, nmax=nmax) for i in range(count)]


def rel_extent(a, b):
    ext = max(float((b.max(0) - b.min(0)).max()), 1e-30)
    return float(np.abs(a - b).max() / ext)


@pytest.mark.parametrize("threads", [256, 512, 1024])
def test_batch_matches_the_one_graph_engine(threads):
    gs = small_mix()
    with batch.Batch(gs) as b:
        b.set_threads(threads)
        b.run(2)
        got = b.positions()
        st = b.stats()
    assert (st["errors"] == 0).all()
    assert (st["ticks"] == 2).all()
    for g, pos in zip(gs, got):
        with Fa2(g.n, g.src, g.dst, params=g.params, pos0=g.pos0) as eng:
            eng.tick(2)
            want = eng.positions()
        assert rel_extent(pos, want) < 1e-5, (g.kind, g.n)


@pytest.mark.parametrize("dim", [2, 3])
def test_coincident_clusters_take_the_long_run_sort(dim):
    # clusters of 70-400 coincident points: runs of equal high key words longer
    # than the in-place fix-up's 64, which the block sorts run by run
    gs = []
    rng = np.random.default_rng(7 + dim)
    for i, (n, cl) in enumerate([(900, 300), (1500, 70), (600, 400), (2000, 130)]):
        src = rng.integers(0, n, 3 * n).astype(np.uint32)
        dst = rng.integers(0, n, 3 * n).astype(np.uint32)
        pos = rng.uniform(0, 100, (n, dim)).astype(np.float32)
        pos[:cl] = pos[0]
        gs.append(batch.GraphSpec(n, src, dst, dict(dim=dim, theta=1.0, seed=i), None, pos, "clustered"))
    with batch.Batch(gs) as b:
        b.run(1)
        got = b.positions()
        st = b.stats()
    assert (st["errors"] == 0).all()
    for i, (g, pos) in enumerate(zip(gs, got)):
        with Fa2(g.n, g.src, g.dst, params=g.params, pos0=g.pos0) as eng:
            eng.tick(1)
            want = eng.positions()
            inf = eng.info()
        assert rel_extent(pos, want) < 1e-5, g.n
        assert (int(st["far"][i]), int(st["pair"][i])) == (inf["far_count"], inf["pair_count"]), g.n


def test_graphs_either_side_of_the_block_sort_limit_match_the_engine():
    # up to 2^14 nodes a graph's block sort takes two passes on the top 16 key
    # bits, above it four on the high 32 (block_sort_top); a clustered graph on
    # each side makes long runs of equal sorted bits
    gs = []
    rng = np.random.default_rng(21)
    for i, (n, cl) in enumerate([(16384, 0), (16385, 0), (16000, 500), (19000, 500)]):
        src = rng.integers(0, n, 3 * n).astype(np.uint32)
        dst = rng.integers(0, n, 3 * n).astype(np.uint32)
        pos = rng.uniform(0, 1000, (n, 2)).astype(np.float32)
        if cl:
            pos[:cl] = pos[0] + rng.uniform(0, 1e-3, (cl, 2)).astype(np.float32)
        gs.append(batch.GraphSpec(n, src, dst, dict(theta=1.0, seed=i), None, pos, "sized"))
    with batch.Batch(gs) as b:
        b.run(1)
        got = b.positions()
        st = b.stats()
    assert (st["errors"] == 0).all()
    for i, (g, pos) in enumerate(zip(gs, got)):
        with Fa2(g.n, g.src, g.dst, params=g.params, pos0=g.pos0) as eng:
            eng.tick(1)
            want = eng.positions()
            inf = eng.info()
        assert rel_extent(pos, want) < 1e-5, g.n
        assert (int(st["far"][i]), int(st["pair"][i])) == (inf["far_count"], inf["pair_count"]), g.n


def test_first_tick_interactions_equal_the_one_graph_engine():
    gs = small_mix(16, seed=3)
    with batch.Batch(gs) as b:
        b.run(1)
        st = b.stats()
    for i, g in enumerate(gs):
        with Fa2(g.n, g.src, g.dst, params=g.params, pos0=g.pos0) as eng:
            eng.tick(1)
            inf = eng.info()
        assert (int(st["far"][i]), int(st["pair"][i])) == (inf["far_count"], inf["pair_count"]), g.n


def test_batch_tracks_the_oracle():
    gs = small_mix(12, seed=5, nmax=1500)
    with batch.Batch(gs) as b:
        b.run(2)
        got = b.positions()
    for g, pos in zip(gs, got):
        st = oracle_state(g.n, g.src, g.dst, None, g.pos0, g.params)
        st.run(2)
        assert rel_extent(pos, st.positions()) < 1e-4, (g.kind, g.n)


def test_batch_is_deterministic_and_tuning_restores_the_state():
    gs = small_mix(32, seed=7)
    with batch.Batch(gs) as b:
        chosen, times = b.tune(2)
        assert chosen in (256, 512, 1024) and all(t > 0 for t in times.values())
        b.run(5)
        a = b.positions()
    with batch.Batch(gs) as b:
        b.set_threads(chosen)
        b.run(5)
        c = b.positions()
    for x, y in zip(a, c):
        assert np.array_equal(x, y)


def test_converged_graphs_stop_and_others_continue():
    still = batch.GraphSpec(20, np.zeros(0, np.uint32), np.zeros(0, np.uint32),
                            dict(gravity=0.0, scaling_ratio=0.0, dim=2), pos0=synth.uniform(20, 2, 0, 5, 1))
    moving = small_mix(3, seed=9)
    with batch.Batch([still] + moving) as b:
        b.run(10)
        st = b.stats()
        pos = b.positions()
    assert st["ticks"][0] == 1
    assert (st["ticks"][1:] == 10).all()
    assert np.array_equal(pos[0], still.pos0)


def test_batch_3d():
    gs = []
    for i in range(10):
        w = synth.powerlaw_1m(seed=30 + i, n=200 + 300 * i, dim=3)
        gs.append(batch.GraphSpec(w.n, w.src, w.dst, w.params, None, w.pos0, "powerlaw3d"))
    with batch.Batch(gs) as b:
        b.run(2)
        got = b.positions()
    for g, pos in zip(gs, got):
        with Fa2(g.n, g.src, g.dst, params=g.params, pos0=g.pos0) as eng:
            eng.tick(2)
            assert rel_extent(pos, eng.positions()) < 1e-5


def test_batch_full_runs_match_the_oracle_on_energy_and_stress():
    """Whole 100-tick runs of a dozen mixed graphs (SBM, BA, rewired grids of
    300-3,000 nodes) against the oracle's FP64 runs: each FA2 energy term and the
    sampled Kruskal stress within 1%."""
    from graph_render_b200 import quality
    from oracle import oracle as O

    gs = [g for g in small_mix(count=24, seed=5) if g.n >= 300][:12]
    assert len(gs) >= 6
    ticks = 100
    with batch.Batch(gs) as b:
        b.run(ticks)
        got = b.positions()
        st = b.stats()
    assert (st["errors"] == 0).all()
    for g, pos, done in zip(gs, got, st["ticks"]):
        o = oracle_state(g.n, g.src, g.dst, g.weight, g.pos0, g.params)
        assert o.run(ticks) == done, (g.kind, g.n)
        r = o.positions()
        prm = dict(g.params)
        eg = quality.fa2_energy(pos, g.src, g.dst, g.weight, prm)
        er = quality.fa2_energy(r, g.src, g.dst, g.weight, prm)
        for term in ("attraction", "repulsion", "gravity", "total"):
            assert abs(eg[term] - er[term]) <= 1e-2 * abs(er[term]) + 1e-9, (g.kind, g.n, term, eg[term], er[term])
        if g.params.get("dim", 2) == 2:
            sg = O.stress(pos[:, 0], pos[:, 1], g.src, g.dst, 16)
            sr = O.stress(r[:, 0], r[:, 1], g.src, g.dst, 16)
            assert abs(sg - sr) <= 1e-2 * sr, (g.kind, g.n, sg, sr)


@pytest.mark.parametrize("dim", [2, 3])
def test_graphs_without_positions_start_from_their_own_seeded_draws(dim):
    # no pos0 anywhere: each graph starts from Mulberry32(its own seed), drawn on
    # the device from its first node, bit for bit the one-graph engine's start
    from oracle import oracle as O

    rng = np.random.default_rng(40 + dim)
    gs = []
    for i, n in enumerate([1, 37, 2500, 700, 64]):
        src = rng.integers(0, max(n, 1), 2 * n).astype(np.uint32)
        dst = rng.integers(0, max(n, 1), 2 * n).astype(np.uint32)
        gs.append(batch.GraphSpec(n, src, dst, dict(dim=dim, seed=[3, 0, 5, 4294967295, 11][i]), None, None, "seeded"))
    with batch.Batch(gs) as b:
        got = b.positions()
    for g, pos in zip(gs, got):
        want = O.initial_positions(g.n, g.params["seed"], dim).astype(np.float32)
        assert pos.shape == (g.n, dim)
        assert np.array_equal(np.asarray(pos, np.float32).view(np.uint32), want.view(np.uint32)), g.n
