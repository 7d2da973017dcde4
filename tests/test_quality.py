"""The layout energy: its negative gradient is the oracle's dense FA2 force.

Central differences of `quality.fa2_energy` against the oracle's attraction +
repulsion (theta < 0: every pair exact). The gravity term's centre is the
layout's mean, which moves with every node, so its negative gradient is the
gravity force minus that force's mean over the nodes.
"""

import numpy as np
import pytest

from graph_render_b200 import quality
from tests.gpu_util import oracle_state


def _graph(n=40, m=90, seed=11):
    r = np.random.default_rng(seed)
    src = r.integers(0, n, m).astype(np.uint32)
    dst = r.integers(0, n, m).astype(np.uint32)
    src[:3], dst[:3] = [0, 5, 5], [0, 9, 9]  # a self-loop and a duplicate
    w = r.lognormal(0.0, 0.5, m)
    pos = r.uniform(-50.0, 50.0, (n, 2))
    return n, src, dst, w, pos


def _neg_grad(pos, src, dst, w, prm, h=1e-4):
    g = np.zeros_like(pos)
    for i in range(pos.shape[0]):
        for a in range(pos.shape[1]):
            q = pos.copy()
            q[i, a] += h
            ep = quality.fa2_energy(q, src, dst, w, prm)["total"]
            q[i, a] -= 2 * h
            em = quality.fa2_energy(q, src, dst, w, prm)["total"]
            g[i, a] = -(ep - em) / (2 * h)
    return g


@pytest.mark.parametrize("prm", [
    dict(gravity=0.0),
    dict(gravity=0.0, lin_log=1),
    dict(gravity=0.0, edge_weight_influence=1.0, scaling_ratio=3.5),
    dict(gravity=0.0, lin_log=1, edge_weight_influence=0.5),
])
def test_energy_gradient_is_attraction_plus_repulsion(prm):
    n, src, dst, w, pos = _graph()
    st = oracle_state(n, src, dst, w, pos.astype(np.float32), prm, dense=True)
    p = st.positions()
    f = st.accumulate(1 | 2)
    g = _neg_grad(p, src, dst, w, prm)
    assert np.abs(g - f).max() < 1e-5 * np.abs(f).max()


@pytest.mark.parametrize("strong", [0, 1])
def test_energy_gradient_of_gravity_about_the_moving_mean(strong):
    n, src, dst, w, pos = _graph(seed=12)
    prm = dict(gravity=2.5, strong_gravity=strong)
    st = oracle_state(n, src, dst, w, pos.astype(np.float32), prm, dense=True)
    p = st.positions()
    fg = st.accumulate(4)
    fa = st.accumulate(1 | 2)
    g = _neg_grad(p, src, dst, w, prm)
    want = fa + fg - fg.mean(0)
    assert np.abs(g - want).max() < 1e-5 * np.abs(want).max()


def test_simple_edges_drop_loops_and_keep_the_first_duplicate():
    lo, hi, w = quality.simple_edges(4, [0, 1, 2, 2, 3], [0, 2, 1, 1, 1], [9.0, 1.0, 2.0, 3.0, 4.0])
    assert lo.tolist() == [1, 1] and hi.tolist() == [2, 3] and w.tolist() == [1.0, 4.0]


def test_sampled_repulsion_estimates_the_pair_sum():
    # the estimator the full-size whole-run comparisons use (n too large for the
    # O(n^2) sum): 2^24 uniform pairs against every pair of a 5,000-node layout
    from graph_render_b200 import synth

    wl = synth.ba_100k(n=5000)
    p = wl.pos0.astype(np.float64)
    exact = quality.fa2_energy(p, wl.src, wl.dst, wl.weight, wl.params)["repulsion"]
    est = quality.fa2_energy(p, wl.src, wl.dst, wl.weight, wl.params, pair_sample=1 << 24, seed=3)["repulsion"]
    assert abs(est - exact) <= 1e-3 * abs(exact), (est, exact)
