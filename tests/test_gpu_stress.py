"""The device's multi-source BFS and Kruskal stress-1 (gr_bfs_hops, gr_stress)
against the oracle's restatement of the reference's `stress`
(crates/graph-cli/src/bench.rs:255-295).

Hop counts are integers: equal exactly. The stress sums are FP64 in a different
order than the reference's: equal to 1e-12 relative. The reference's own unit
cases have sums exact in any order, so they are equal exactly."""

import numpy as np
import pytest

from graph_render_b200 import Fa2, stress as S, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _graphs():
    s, d, _ = O.gate_edges(601)
    yield "gate601", 601, s, d
    wl = synth.sbm_1500()
    yield "sbm1500", wl.n, wl.src, wl.dst
    a, b = synth.sbm([700, 500, 300], 0.01, 0.0, 3)  # three components
    yield "sbm-3-components", 1500, a, b
    wl = synth.powerlaw_1m(n=20_000, dim=2)
    yield "powerlaw20k", wl.n, wl.src, wl.dst


@pytest.mark.parametrize("case", list(_graphs()), ids=lambda c: c[0])
def test_bfs_hops_equal_the_oracle(case):
    _, n, s, d = case
    rng = np.random.default_rng(1)
    src = rng.integers(0, n, 130).astype(np.uint32)  # three batches of up to 64 sources
    src[:3] = [0, 0, n - 1]  # a repeated source
    assert np.array_equal(S.bfs_hops(n, s, d, src), O.bfs_hops(n, s, d, src))


@pytest.mark.parametrize("case", list(_graphs()), ids=lambda c: c[0])
def test_stress_equals_the_oracle_on_a_laid_out_graph(case):
    _, n, s, d = case
    with Fa2(n, s, d, params=dict(theta=1.0)) as eng:
        eng.tick(30)
        p = eng.positions()
    for sources in (16, 1, 100):
        g = S.kruskal_stress(p[:, 0], p[:, 1], s, d, sources)
        o = O.stress(p[:, 0], p[:, 1], s, d, sources)
        assert abs(g - o) <= 1e-12 * abs(o), (sources, g, o)


def test_stress_reference_unit_cases():
    assert S.kruskal_stress([0.0, 2.0, 4.0], [0.0] * 3, [0, 1], [1, 2]) == 0.0
    assert S.kruskal_stress([0.0, 1.0, 0.0], [0.0] * 3, [0, 1], [1, 2]) == (8.0 / 12.0) ** 0.5
    assert S.kruskal_stress([5.0] * 3, [5.0] * 3, [0, 1], [1, 2]) == 1.0
    assert S.kruskal_stress([0.0, 1.0], [0.0, 0.0], [], []) == 1.0
    assert S.kruskal_stress([0.0, 1.0, 100.0, 101.0], [0.0] * 4, [0, 2], [1, 3]) == 0.0


def test_refusals():
    from graph_render_b200._native import EngineError

    with pytest.raises(EngineError):
        S.bfs_hops(3, [0], [5], [0])  # endpoint out of range
    with pytest.raises(EngineError):
        S.bfs_hops(3, [0], [1], [3])  # source out of range
