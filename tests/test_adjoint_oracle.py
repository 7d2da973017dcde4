"""The oracle's adjoint pinned to FP64 central differences (CPU).

orc_fa2_adjoint is the vector-Jacobian product of a run of ticks through the
trees the run built and the speed controller's active branch; here its
directional derivatives must equal central differences of the FP64 forward
run, for start positions and edge weights, with the dense sum and the tree,
and every option.
"""

import numpy as np
import pytest

from oracle import oracle as O
from graph_render_b200 import synth


def setup(n, seed=3, dim=2):
    s, d = synth.sbm([n // 2, n - n // 2], 8.0 / n, 1.0 / n, seed)
    lo, hi, _ = O.simple_graph(n, s, d)
    rng = np.random.default_rng(1)
    w = rng.uniform(0.5, 1.5, len(lo))
    pos = rng.uniform(0, 30, (n, dim))
    R = rng.normal(size=(n, dim))
    return lo, hi, w, pos, R, rng


def loss(n, lo, hi, w, pos, R, ticks, kw):
    st = O.State(n, lo, hi, w=w, pos0=pos, **kw)
    for _ in range(ticks):
        st.iterate()
    return float((st.positions() * R).sum())


@pytest.mark.parametrize("ticks,theta,opts", [
    (1, -1.0, {}), (3, -1.0, {}), (3, 0.8, {}), (5, 0.8, {}),
    (3, -1.0, {"lin_log": 1}), (3, 0.8, {"strong_gravity": 1, "dissuade_hubs": 1}),
    (3, -1.0, {"lin_log": 1, "dissuade_hubs": 1}), (2, 0.8, {"dim": 3}),
])
def test_adjoint_equals_central_differences(ticks, theta, opts):
    n = 60
    dim = opts.get("dim", 2)
    lo, hi, w, pos, R, rng = setup(n, dim=dim)
    kw = dict(theta=theta, edge_weight_influence=1.0, **opts)
    st = O.State(n, lo, hi, w=w, pos0=pos, **kw)
    lam0, gc = O.adjoint(st, ticks, R)
    v = rng.normal(size=pos.shape)
    vw = rng.normal(size=len(lo))
    h = 1e-6
    fdp = (loss(n, lo, hi, w, pos + h * v, R, ticks, kw) - loss(n, lo, hi, w, pos - h * v, R, ticks, kw)) / (2 * h)
    fdw = (loss(n, lo, hi, w + h * vw, pos, R, ticks, kw) - loss(n, lo, hi, w - h * vw, pos, R, ticks, kw)) / (2 * h)
    assert abs(fdp - (lam0 * v).sum()) <= 1e-5 * abs(fdp)
    assert abs(fdw - (gc * vw).sum()) <= 1e-5 * abs(fdw)


def test_adjoint_at_the_differentiated_workloads_step():
    """h = 1e-3 central differences, component by component (8 edge weights, 8
    start coordinates), on the 2,000-node instance of the SBM generator (all
    pairs, FP64), two ticks: within 1e-3."""
    wl = synth.sbm_50k(n=2000)
    lo, hi, _ = O.simple_graph(wl.n, wl.src, wl.dst)
    w = np.ones(len(lo))
    pos = wl.pos0.astype(np.float64)
    R = np.random.default_rng(9).normal(size=pos.shape)
    kw = dict(theta=-1.0, edge_weight_influence=1.0)
    st = O.State(wl.n, lo, hi, w=w, pos0=pos, **kw)
    lam0, gc = O.adjoint(st, 2, R)
    rng = np.random.default_rng(10)
    h = 1e-3
    f = lambda P, W: loss(wl.n, lo, hi, W, P, R, 2, kw)
    for e in rng.choice(len(lo), 8, replace=False):
        d = np.zeros(len(lo))
        d[e] = h
        fd = (f(pos, w + d) - f(pos, w - d)) / (2 * h)
        assert abs(fd - gc[e]) <= 1e-3 * abs(fd) + 1e-9, (e, fd, gc[e])
    for k in rng.choice(pos.size, 8, replace=False):
        d = np.zeros(pos.size)
        d[k] = h
        d = d.reshape(pos.shape)
        fd = (f(pos + d, w) - f(pos - d, w)) / (2 * h)
        assert abs(fd - lam0.reshape(-1)[k]) <= 1e-3 * abs(fd) + 1e-9, (k, fd)
