"""The differentiated workload's loss and its gradient, on the CPU.

The loss is Kruskal stress-1 with the optimal scale over sampled node pairs
against hop distance, the reference's quality measure
(crates/graph-cli/src/bench.rs:255-295) restated over pairs drawn from a seed
(graph_render_b200/stress.py `stress`). Every backward pass starts from its
dL/d(final positions), so that gradient is checked here by central differences
(coordinate by coordinate and along random directions) within 1e-6 relative.
Hop counts come from the oracle's FIFO BFS, so nothing here needs a GPU.
"""

import numpy as np
import pytest

from oracle import oracle as O
from graph_render_b200 import stress, synth


def pairs_on_the_cpu(n, src, dst, pairs, seed, sources=200):
    """stress.sample_pairs' draw with the oracle's BFS for the hop counts."""
    per = max(1, pairs // sources)
    s = synth.randint(sources, n, seed).astype(np.uint32)
    t = synth.randint(sources * per, n, seed + 1).astype(np.uint32).reshape(sources, per)
    hops = O.bfs_hops(n, src, dst, s)
    h = np.take_along_axis(hops, t.astype(np.int64), axis=1).reshape(-1)
    a, b = np.repeat(s, per), t.reshape(-1)
    keep = (h != np.iinfo(np.uint32).max) & (a != b)
    return a[keep], b[keep], h[keep].astype(np.float64)


def instance(dim=2, n=2000, pairs=6000, seed=5):
    wl = synth.sbm_50k(n=n)
    a, b, h = pairs_on_the_cpu(wl.n, wl.src, wl.dst, pairs, seed)
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-500.0, 500.0, (wl.n, dim))
    return pos, a, b, h


def loss(pos, a, b, h):
    return stress.stress(pos, a, b, h)[0]


@pytest.mark.parametrize("dim", [2, 3])
def test_stress_gradient_matches_central_differences(dim):
    pos, a, b, h = instance(dim)
    L, g = stress.stress(pos, a, b, h)
    assert 0.0 < L < 1.0
    rng = np.random.default_rng(1)
    touched = np.unique(np.concatenate([a, b]))
    nodes = rng.choice(touched, 200, replace=False)
    step = 1e-2  # positions are O(500): truncation ~ step^2 * g / 500^2, rounding ~ 1e-16 * L / step
    fd, an = [], []
    for i in nodes:
        for ax in range(dim):
            p = pos.copy()
            p[i, ax] += step
            up = loss(p, a, b, h)
            p[i, ax] -= 2 * step
            dn = loss(p, a, b, h)
            fd.append((up - dn) / (2 * step))
            an.append(g[i, ax])
    fd, an = np.array(fd), np.array(an)
    assert np.linalg.norm(fd - an) <= 1e-6 * np.linalg.norm(an), np.linalg.norm(fd - an) / np.linalg.norm(an)
    # nodes in no sampled pair get no gradient
    idle = np.setdiff1d(np.arange(len(pos)), touched)
    assert np.all(g[idle] == 0.0)


@pytest.mark.parametrize("dim", [2, 3])
def test_stress_gradient_along_random_directions(dim):
    pos, a, b, h = instance(dim, seed=9)
    _, g = stress.stress(pos, a, b, h)
    rng = np.random.default_rng(2)
    for _ in range(8):
        v = rng.normal(size=pos.shape)
        v /= np.linalg.norm(v)
        step = 1e-1
        fd = (loss(pos + step * v, a, b, h) - loss(pos - step * v, a, b, h)) / (2 * step)
        an = float((g * v).sum())
        assert abs(fd - an) <= 1e-6 * abs(an) + 1e-15, (fd, an)


def test_stress_value_is_the_references_formula():
    # bench.rs:285-294: sqrt(max((DD - DE^2/EE)/DD, 0)) with e the Euclidean and
    # d the hop distance; an exact multiple of the hops gives 0, a collapsed
    # layout 1
    a = np.array([0, 0, 1], np.int64)
    b = np.array([1, 2, 2], np.int64)
    d = np.array([1.0, 2.0, 1.0])
    line = np.array([[0.0, 0.0], [3.0, 0.0], [6.0, 0.0]])
    assert stress.stress(line, a, b, d)[0] == 0.0
    assert stress.stress(np.zeros((3, 2)), a, b, d)[0] == 1.0
    bent = np.array([[0.0, 0.0], [1.0, 0.0], [1.0, 1.0]])
    e = np.array([1.0, np.sqrt(2.0), 1.0])
    DE, EE, DD = (d * e).sum(), (e * e).sum(), (d * d).sum()
    want = np.sqrt(max((DD - DE * DE / EE) / DD, 0.0))
    assert abs(stress.stress(bent, a, b, d)[0] - want) < 1e-15
