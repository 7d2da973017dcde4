"""The GPU adjoint (gr_fa2_adjoint_forward / _backward) against the FP64 oracle.

The oracle's adjoint (oracle/fa2_oracle.c, orc_fa2_adjoint) is the exact VJP of
the tick in FP64 and is itself pinned to FP64 central differences
(tests/test_adjoint_oracle.py). Here the GPU's dL/d(start positions) and
dL/d(edge weights) for a fixed linear loss must match it within 1e-3 relative
L2 — all pairs exact (theta 0, the dense sum) on the 2,000-node instance of
the differentiated workload's generator, and through the same Barnes-Hut tree
(theta 1.2, the oracle capped at the engine's Morton depth).
"""

import numpy as np
import pytest

from oracle import oracle as O
from graph_render_b200 import Fa2, stress, synth
from tests.gpu_util import oracle_state

pytestmark = pytest.mark.gpu

TOL = 1e-3


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def instance(n=2000, theta=0.0):
    wl = synth.sbm_50k(n=n)
    rng = np.random.default_rng(5)
    w = rng.uniform(0.5, 1.5, wl.m)
    prm = dict(wl.params, theta=theta)
    return wl, w, prm


def gpu_grad(wl, w, prm, ticks, R, every=20):
    with Fa2(wl.n, wl.src, wl.dst, w, params=prm, pos0=wl.pos0) as eng:
        eng.adjoint_forward(ticks, every)
        return eng.adjoint_backward(R)


def oracle_grad(wl, w, prm, ticks, R, dense):
    st = oracle_state(wl.n, wl.src, wl.dst, w, wl.pos0, prm, dense=dense)
    lam0, gc = O.adjoint(st, ticks, np.asarray(R, np.float64))
    # simple edge -> raw edge (first of its pair), dc/dw = 1 at influence 1
    lo, hi, _ = O.simple_graph(wl.n, wl.src, wl.dst, w)
    graw = np.zeros(wl.m)
    key = {}
    for e, (a, b) in enumerate(zip(wl.src.tolist(), wl.dst.tolist())):
        if a != b:
            key.setdefault((min(a, b), max(a, b)), e)
    for s, (a, b) in enumerate(zip(lo.tolist(), hi.tolist())):
        graw[key[(a, b)]] = gc[s]
    return lam0, graw


@pytest.mark.parametrize("ticks", [1, 2])
def test_adjoint_matches_the_fp64_all_pairs_adjoint(ticks):
    wl, w, prm = instance(theta=0.0)
    R = np.random.default_rng(1).normal(size=(wl.n, 2))
    gp, gw = gpu_grad(wl, w, prm, ticks, R)
    op, ow = oracle_grad(wl, w, prm, ticks, R, dense=True)
    assert np.isfinite(gp).all() and np.isfinite(gw).all()
    assert rel(gp, op) < TOL, rel(gp, op)
    assert rel(gw, ow) < TOL, rel(gw, ow)


@pytest.mark.parametrize("theta,n", [(0.0, 2000), (1.2, 5000)])
def test_every_ticks_vjp_matches_the_oracle_along_a_200_tick_run(theta, n):
    """The chained gradient of a long run is ill-conditioned (a 1e-7 change of
    the start moves the exact FP64 gradient by 2% at 3 ticks and 4x at 8 on
    this instance), so FP32 and FP64 runs are compared tick by tick: at several
    depths of the GPU's own run, the VJP of one tick from the GPU's state
    (positions and FP64 controller) against the oracle's from the same state."""
    wl, w, prm = instance(n=n, theta=theta)
    R = np.random.default_rng(6).normal(size=(wl.n, 2))
    lo, hi, ws = O.simple_graph(wl.n, wl.src, wl.dst, w)
    with Fa2(wl.n, wl.src, wl.dst, w, params=prm, pos0=wl.pos0) as eng:
        done = 0
        for depth in (0, 5, 30, 120, 199):
            eng.tick(depth - done)
            pos = eng.positions()
            c = eng.controller()
            eng.adjoint_forward(1, 1)
            gp, gw = eng.adjoint_backward(R)
            done = depth + 1
            st = oracle_state(wl.n, wl.src, wl.dst, w, pos, prm, dense=(theta == 0.0))
            st.set_scalars(c["swing"], c["traction"], c["speed"], c["speed_efficiency"], c["iter_no"])
            op, ow = oracle_grad_from(st, wl, w, R)
            assert rel(gp, op) < TOL, (depth, rel(gp, op))
            assert rel(gw, ow) < TOL, (depth, rel(gw, ow))


def oracle_grad_from(st, wl, w, R):
    lam0, gc = O.adjoint(st, 1, np.asarray(R, np.float64))
    lo, hi, _ = O.simple_graph(wl.n, wl.src, wl.dst, w)
    key = {}
    for e, (a, b) in enumerate(zip(wl.src.tolist(), wl.dst.tolist())):
        if a != b:
            key.setdefault((min(a, b), max(a, b)), e)
    graw = np.zeros(wl.m)
    for s_, (a, b) in enumerate(zip(lo.tolist(), hi.tolist())):
        graw[key[(a, b)]] = gc[s_]
    return lam0, graw


@pytest.mark.parametrize("ticks", [1, 2])
def test_adjoint_through_the_same_tree(ticks):
    wl, w, prm = instance(n=5000, theta=1.2)
    R = np.random.default_rng(2).normal(size=(wl.n, 2))
    gp, gw = gpu_grad(wl, w, prm, ticks, R)
    op, ow = oracle_grad(wl, w, prm, ticks, R, dense=False)
    assert rel(gp, op) < TOL, rel(gp, op)
    assert rel(gw, ow) < TOL, rel(gw, ow)


def test_checkpoint_interval_does_not_change_the_gradient():
    wl, w, prm = instance(n=3000, theta=1.2)
    R = np.random.default_rng(3).normal(size=(wl.n, 2))
    a = gpu_grad(wl, w, prm, 30, R, every=30)
    b = gpu_grad(wl, w, prm, 30, R, every=7)
    assert rel(a[0], b[0]) < 1e-5 and rel(a[1], b[1]) < 1e-5


def test_stress_gradient_through_the_run_is_finite_and_the_state_is_kept():
    wl, w, prm = instance(n=4000, theta=1.2)
    a, b, h = stress.sample_pairs(wl.n, wl.src, wl.dst, 100_000, 5)
    with Fa2(wl.n, wl.src, wl.dst, w, params=prm, pos0=wl.pos0) as eng:
        eng.adjoint_forward(40, 20)
        pT = eng.positions()
        L, g = stress.stress(pT, a, b, h)
        gp, gw = eng.adjoint_backward(g)
        assert np.array_equal(eng.positions(), pT)  # the handle stays at the run's end
    assert np.isfinite(gp).all() and np.isfinite(gw).all()
    assert np.abs(gp).max() > 0 and np.abs(gw).max() > 0


def test_3d_adjoint_matches_the_oracle():
    wl = synth.powerlaw_1m(n=1500, dim=3)
    prm = dict(wl.params, theta=0.0, strong_gravity=0)
    R = np.random.default_rng(4).normal(size=(wl.n, 3))
    with Fa2(wl.n, wl.src, wl.dst, None, params=prm, pos0=wl.pos0) as eng:
        eng.adjoint_forward(3, 2)
        gp, _ = eng.adjoint_backward(R)
    st = oracle_state(wl.n, wl.src, wl.dst, None, wl.pos0, prm, dense=True)
    op, _ = O.adjoint(st, 3, R)
    assert rel(gp, op) < TOL


def test_long_run_adjoint_outgrows_fp32_and_stays_exactly_linear():
    """200 ticks with checkpoints every 20 (the differentiated workload's
    schedule) on the 2,000-node instance: the true dL/dp0 grows far beyond
    FP32 (the FP64 oracle's has norm ~1e37 here), so the engine carries the
    adjoint under a power-of-two scale. Scaling dL/dpT by 2^-40 must scale
    both gradients by exactly 2^-40."""
    wl, w, prm = instance(n=2000, theta=1.2)
    R = np.random.default_rng(2).normal(size=(wl.n, 2)).astype(np.float32)
    with Fa2(wl.n, wl.src, wl.dst, w, params=prm, pos0=wl.pos0) as eng:
        eng.adjoint_forward(200, 20)
        gp, gw = eng.adjoint_backward(R)
        gp2, gw2 = eng.adjoint_backward(np.ldexp(R, -40))
    assert np.isfinite(gp).all() and np.isfinite(gw).all()
    assert np.linalg.norm(gp) > 1e10
    assert np.array_equal(np.ldexp(gp, -40), gp2)
    assert np.array_equal(np.ldexp(gw, -40), gw2)


@pytest.mark.parametrize("theta,ticks", [(0.0, 1), (0.0, 2), (1.2, 2)])
def test_backward_seeded_with_the_stress_loss_matches_the_oracle(theta, ticks):
    """The differentiated workload's own seed: dL/dpT of the sampled stress
    (pairs and hops from the device BFS) at the GPU's final positions, carried
    back through the run on the GPU and by the FP64 oracle adjoint."""
    wl, w, prm = instance(n=2000, theta=theta)
    a, b, h = stress.sample_pairs(wl.n, wl.src, wl.dst, 200_000, 5, sources=200)
    with Fa2(wl.n, wl.src, wl.dst, w, params=prm, pos0=wl.pos0) as eng:
        eng.adjoint_forward(ticks, 1)
        pT = eng.positions()
        L, g = stress.stress(pT, a, b, h)
        gp, gw = eng.adjoint_backward(g)
    assert 0.0 < L < 1.0 and np.abs(g).max() > 0
    op, ow = oracle_grad(wl, w, prm, ticks, g, dense=(theta == 0.0))
    assert rel(gp, op) < TOL, rel(gp, op)
    assert rel(gw, ow) < TOL, rel(gw, ow)
