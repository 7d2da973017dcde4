"""The d3-force Barnes-Hut session on the GPU (gr_force_session_*) against the
FP64 oracle (orc_d3_*, itself bit-exact to the reference's golden digests).

A force simulation turns one rounding difference into a different picture over
many ticks (the reference's own gate for this layout is "different, but not
worse" by stress, registry/force.rs BARNES_HUT). So: the FP32 tick against the
FP64 tick from the same state, pass for pass (1 and 5 ticks, relative L2), and
the full 112-tick layout by its Kruskal stress."""

import numpy as np
import pytest

from graph_render_b200 import D3_ID, ForceSession, Topology, find, stress as S, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


def _gate(n):
    src, dst, st = O.gate_edges(n)
    return n, src, dst, st


def _sbm():
    wl = synth.sbm_1500()
    rng = np.random.default_rng(3)
    return wl.n, wl.src, wl.dst, rng.uniform(0.4, 0.8, len(wl.src))


def _cases():
    yield "gate601", _gate(601)
    yield "sbm1500", _sbm()


def _oracle(n, src, dst, st, pos0=None):
    lo, hi, w = O.simple_graph(n, src, dst, st)
    return O.D3(n, lo, hi, w, pos0=pos0)


@pytest.mark.parametrize("case", list(_cases()), ids=lambda c: c[0])
def test_first_tick_matches_the_oracle_from_the_golden_spiral(case):
    n, src, dst, st = case[1]
    with ForceSession(n, src, dst, st) as s:
        s.tick(1)
        gp, gv = s.positions(), s.velocities()
        assert s.ticks_done() == 1
    o = _oracle(n, src, dst, st)
    o.tick(1)
    assert rel(gp, o.positions()) < 1e-5
    assert rel(gv, o.velocities()) < 1e-4


@pytest.mark.parametrize("at", [3, 20, 60, 111])
@pytest.mark.parametrize("case", list(_cases()), ids=lambda c: c[0])
def test_one_tick_from_the_oracles_state_along_its_run(case, at):
    """The oracle's state after `at` ticks, rounded to FP32, handed to both; one
    tick each. Velocities (the tick's forces) to 1e-3 relative L2: late in the
    run a spring near its rest length cancels (l - distance) in FP32, which costs
    ~2e-4 on a settled graph; positions to 1e-5 of the drawing's extent."""
    n, src, dst, st = case[1]
    o = _oracle(n, src, dst, st)
    o.tick(at)
    p = o.positions().astype(np.float32)
    v = o.velocities().astype(np.float32)
    a = o.alpha()
    o.set_state(p.astype(np.float64), v.astype(np.float64), a, at)
    o.tick(1)
    with ForceSession(n, src, dst, st) as s:
        s.set_state(p, v, a, at)
        s.tick(1)
        gp, gv = s.positions(), s.velocities()
        assert s.alpha() == o.alpha()
    assert rel(gv, o.velocities()) < 1e-3
    ext = float(np.ptp(o.positions(), axis=0).max())
    assert np.abs(gp - o.positions()).max() / ext < 1e-5


def test_frozen_layout_is_not_worse_than_the_oracles_by_stress():
    for n, src, dst, st in (_gate(601), _sbm()):
        g = find(D3_ID).run_params(Topology(n, src, dst, st), b"")
        o = _oracle(n, src, dst, st)
        o.tick(O.D3_TICKS)
        po = o.positions()
        sg = S.kruskal_stress(g.x, g.y, src, dst)
        so = O.stress(po[:, 0].astype(np.float32), po[:, 1].astype(np.float32), src, dst)
        assert np.isfinite(g.x).all() and np.isfinite(g.y).all()
        assert sg <= so + 0.05, (n, sg, so)


@pytest.mark.parametrize("seed", range(8))
def test_the_gate_seeds_settle_where_the_oracle_does(seed):
    """2..9 nodes: small enough that the 112-tick run is not chaotic, so the FP32
    layout lands within a small fraction of the drawing's extent of the
    reference's (the oracle reproduces the reference's bytes here)."""
    n, src, dst, st = _gate(2 + seed)
    g = find(D3_ID).run_params(Topology(n, src, dst, st), b"")
    o = _oracle(n, src, dst, st)
    o.tick(O.D3_TICKS)
    po = o.positions()
    ext = max(float(np.ptp(po, axis=0).max()), 1.0)
    gp = np.stack([g.x, g.y], 1).astype(np.float64)
    assert np.abs(gp - po).max() / ext < 1e-3


def test_deterministic_and_the_alpha_schedule_is_the_references():
    n, src, dst, st = _sbm()
    outs = []
    for _ in range(2):
        with ForceSession(n, src, dst, st) as s:
            s.tick(20)
            outs.append(s.positions())
            a = 1.0
            for _ in range(20):
                a += (0.0 - a) * 0.06
            assert s.alpha() == a
            info = s.info()
            assert info["graph_kernels"] > 10 and info["n_cells"] >= n
    assert np.array_equal(outs[0], outs[1])


def test_reheat_is_refused_outside_zero_to_one_and_never_clamped():
    from graph_render_b200._native import EngineError

    n, src, dst, st = _gate(50)
    with ForceSession(n, src, dst, st) as s:
        s.tick(10)
        for bad in (1.5, -0.1, float("nan")):
            with pytest.raises(EngineError):
                s.reheat(bad)
        s.reheat(0.3)
        assert s.alpha() == 0.3
        s.tick(1)
        assert s.alpha() == 0.3 + (0.0 - 0.3) * 0.06


def test_coincident_and_collinear_starts_stay_finite_and_match_one_tick():
    """Many nodes on one point (many-body and collide jiggles) and on one line (a
    zero axis everywhere): the first tick against the oracle's."""
    n, src, dst, st = _gate(300)
    for pos in (np.zeros((n, 2)), np.stack([np.arange(n, dtype=np.float64) * 3.0, np.zeros(n)], 1)):
        pos = pos.copy()
        pos[150:] += [[40.0, 25.0]]
        with ForceSession(n, src, dst, st, pos0=pos) as s:
            s.tick(1)
            gp = s.positions()
            s.tick(30)
            assert np.isfinite(s.positions()).all()
        o = _oracle(n, src, dst, st, pos0=pos)
        o.tick(1)
        ext = float(np.ptp(o.positions(), axis=0).max())
        assert np.abs(gp - o.positions()).max() / ext < 1e-3


def test_empty_and_single_node():
    with ForceSession(0, [], []) as s:
        s.tick(3)
        assert s.positions().shape == (0, 2)
    with ForceSession(1, [], []) as s:
        s.tick(112)
        assert np.isfinite(s.positions()).all()


def test_timed_ticks_are_the_same_ticks():
    # gr_force_session_tick_timed runs the same captured ticks between two CUDA
    # events on the session's stream
    n, src, dst, st = _gate(2000)
    with ForceSession(n, src, dst, st) as a, ForceSession(n, src, dst, st) as b:
        a.tick(7)
        ms = b.tick_timed(7)
        assert ms > 0.0
        assert np.array_equal(a.positions(), b.positions())
        assert a.ticks_done() == b.ticks_done() == 7
