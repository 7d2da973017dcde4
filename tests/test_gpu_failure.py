"""Failure detection, driven from the host: nothing here faults or hangs a GPU.

- A bounded wait that runs out. The tick's key sort is a one-sweep radix sort
  whose blocks wait for counts that earlier blocks publish; every wait gives up
  after a limit. A test injects a wait on a device word that nothing sets
  (gr_fa2_inject_stalled_wait) with a short limit: the tick must return
  GR_DEVICE_FAULT with ERR_WAIT, its later kernels must do nothing, the handle
  must destroy cleanly, and a fresh handle must run as if nothing happened.
- Bad inputs refused with their codes: a non-finite start, an edge naming a
  node >= n (one graph and a batch), and a run that overflows FP32 and ends in
  the reference's NonFinite refusal (crates/graph-core/src/layout/forceatlas2.rs:86-88
  `settle`; the reference's own NaN tests are layout/force/quadtree/tests.rs:46-84).
"""

import numpy as np
import pytest

from graph_render_b200 import Fa2, StageError, Topology, batch, synth
from graph_render_b200 import _native as N

pytestmark = pytest.mark.gpu

ERR_NONFINITE, ERR_WAIT = 1, 8


def run_ticks(wl, ticks):
    with Fa2(wl.n, wl.src, wl.dst, wl.weight, params=wl.params, pos0=wl.pos0) as eng:
        eng.tick(ticks)
        return eng.positions()


# 20k nodes: five one-sweep tiles of 4,096 keys; 600k: tiles of 6,912 keys
@pytest.mark.parametrize("n", [20_000, 600_000])
def test_a_sort_wait_that_runs_out_halts_the_tick_and_reports_it(n):
    wl = synth.powerlaw_1m(n=n, dim=2)
    with Fa2(wl.n, wl.src, wl.dst, params=wl.params, pos0=wl.pos0) as eng:
        eng.tick(2)
        before = eng.positions()
        eng.set_wait_limit(2000)
        eng.inject_stalled_wait(True)
        with pytest.raises(N.EngineError) as ei:
            eng.tick(3)
        assert ei.value.code == N.GR_DEVICE_FAULT
        assert "0x8" in ei.value.message
        info = eng.info()
        assert info["device_error"] & ERR_WAIT
        assert info["iter_no"] == 2  # no update ran after the wait gave up
        assert info["converged"] == 1  # the handle stays halted
        with pytest.raises(N.EngineError) as ei2:  # and keeps answering with the fault
            eng.tick(1)
        assert ei2.value.code == N.GR_DEVICE_FAULT
    # every kernel returned: a fresh handle runs the same ticks as an untouched one
    assert np.array_equal(run_ticks(wl, 2), before)
    assert np.array_equal(run_ticks(wl, 5), run_ticks(wl, 5))


def test_the_wait_limit_alone_changes_nothing():
    wl = synth.powerlaw_1m(n=50_000, dim=2)
    want = run_ticks(wl, 3)
    with Fa2(wl.n, wl.src, wl.dst, params=wl.params, pos0=wl.pos0) as eng:
        eng.set_wait_limit(1 << 24)
        eng.inject_stalled_wait(True)
        eng.inject_stalled_wait(False)  # removed before any tick
        eng.tick(3)
        assert eng.info()["device_error"] == 0
        assert np.array_equal(eng.positions(), want)


def test_a_non_finite_start_is_refused():
    wl = synth.sbm_1500()
    for bad in (np.nan, np.inf, -np.inf):
        pos = wl.pos0.copy()
        pos[700, 1] = bad
        with pytest.raises(N.EngineError) as ei:
            Fa2(wl.n, wl.src, wl.dst, params=wl.params, pos0=pos)
        assert ei.value.code == N.GR_INVALID_ARGUMENT
        assert "non-finite" in ei.value.message


def test_an_edge_naming_a_missing_node_is_refused():
    wl = synth.sbm_1500()
    for end in ("src", "dst"):
        src, dst = wl.src.copy(), wl.dst.copy()
        (src if end == "src" else dst)[123] = wl.n
        with pytest.raises(N.EngineError) as ei:
            Fa2(wl.n, src, dst, params=wl.params, pos0=wl.pos0)
        assert ei.value.code == N.GR_INVALID_ARGUMENT
    # the registry face refuses the same topology with the same code
    from graph_render_b200 import FA2_ID, find

    src = wl.src.copy()
    src[0] = wl.n + 5
    with pytest.raises(N.EngineError) as ei:
        find(FA2_ID).run_params(Topology(wl.n, src, wl.dst, None), b"")
    assert ei.value.code == N.GR_INVALID_ARGUMENT


def test_a_batch_edge_outside_its_graph_is_refused():
    gs = [batch.mixed_graph(3, i, nmin=50, nmax=400) for i in range(4)]
    bad = gs[2]
    dst = bad.dst.copy()
    dst[0] = bad.n  # a valid node of the concatenation, but not of graph 2
    gs[2] = batch.GraphSpec(bad.n, bad.src, dst, bad.params, bad.weight, bad.pos0, bad.kind)
    with pytest.raises(N.EngineError) as ei:
        batch.Batch(gs)
    assert ei.value.code == N.GR_INVALID_ARGUMENT


def overflowing_star(dim=2):
    """A star whose leaves sit near FLT_MAX / 4 from its centre: the centre's
    attraction (the sum of its leaves' offsets) overflows FP32 on the first tick."""
    k = 12
    n = k + 1
    pos = np.zeros((n, dim), np.float32)
    pos[0, 0] = -8.0e37
    pos[1:, 0] = 8.0e37
    pos[1:, 1] = np.arange(k, dtype=np.float32) * 1.0e36
    src = np.zeros(k, np.uint32)
    dst = np.arange(1, n, dtype=np.uint32)
    return n, src, dst, pos


@pytest.mark.parametrize("dim", [2, 3])
def test_an_overflowing_run_ends_in_the_non_finite_refusal(dim):
    n, src, dst, pos = overflowing_star(dim)
    with Fa2(n, src, dst, params=dict(dim=dim, scaling_ratio=100.0), pos0=pos) as eng:
        with pytest.raises(N.EngineError) as ei:
            eng.tick(3)
        assert ei.value.code == N.GR_LAYOUT_FAILED
        assert eng.info()["device_error"] & ERR_NONFINITE
        with pytest.raises(N.EngineError) as ei:
            eng.positions()  # settle's refusal
        assert ei.value.code == N.GR_LAYOUT_FAILED
    # the registry face maps the code to StageError::NonFinite
    from graph_render_b200 import fa2 as F

    class Once(F.Fa2):
        def __init__(self, *a, **kw):
            kw["pos0"] = pos
            super().__init__(*a, **kw)

    orig = F.Fa2
    F.Fa2 = Once
    try:
        with pytest.raises(StageError) as se:
            F.run_values(Topology(n, src, dst, None), [3, 1.0, 100.0, 1.0, 0, dim, 0.8, 0, 0, 0, 0.0])
    finally:
        F.Fa2 = orig
    assert se.value.kind == "NonFinite"


def test_a_batch_graph_that_overflows_stops_alone():
    n, src, dst, pos = overflowing_star()
    gs = [batch.mixed_graph(5, i, nmin=50, nmax=600) for i in range(3)]
    gs.insert(1, batch.GraphSpec(n, src, dst, dict(scaling_ratio=100.0), None, pos, "overflow"))
    for g in gs:
        if g.pos0 is None:
            raise AssertionError("mixed graphs carry their start")
    with batch.Batch(gs) as b:
        b.run(5)
        st = b.stats()
    assert st["errors"][1] & ERR_NONFINITE
    assert st["ticks"][1] < 5
    others = [0, 2, 3]
    assert (st["errors"][others] == 0).all()
    assert (st["ticks"][others] == 5).all()
