"""The particle-mesh many-body oracle (orc_d3_use_mesh, orc_pm_field) against the
reference's own particle-mesh tests, restated
(crates/graph-core/src/layout/force/particle_mesh/tests.rs). The reference pins
no digest for this layout, so these properties are its pin (CPU)."""

import numpy as np
import pytest

from oracle import oracle as O


def direct(x, y, i, dmin2=1.0, dmax2=520.0 ** 2):
    """d3's law summed over every other node (tests.rs:27-42)."""
    e = np.zeros(2)
    for j in range(len(x)):
        if j == i:
            continue
        rx, ry = x[i] - x[j], y[i] - y[j]
        l = rx * rx + ry * ry
        if l >= dmax2:
            continue
        if l < dmin2:
            l = np.sqrt(dmin2 * l)
        e -= [rx / l, ry / l]
    return e


def placed(x, y):
    d = O.D3(len(x), [], [], [], pos0=np.stack([x, y], 1))
    d.use_mesh()
    return d


def test_the_mesh_field_follows_the_direct_sum_at_range():
    """tests.rs:44-69: rms relative error under 5% on a sheared 8 x 8 lattice."""
    x = np.array([(i % 8) * 70.0 + (i // 8) * 9.0 for i in range(64)])
    y = np.array([(i // 8) * 70.0 for i in range(64)])
    got = placed(x, y).mesh_field()
    want = np.array([direct(x, y, i) for i in range(64)])
    rel = np.sqrt(((got - want) ** 2).sum() / (want ** 2).sum())
    assert rel < 0.05, rel


def test_a_node_out_of_everyones_range_feels_no_force_from_itself():
    """tests.rs:71-83."""
    f = placed(np.array([0.0, 3000.0]), np.array([0.0, 17.5])).mesh_field()
    assert np.abs(f).max() < 1e-12


def _line(n):
    return np.arange(n - 1, dtype=np.uint32), np.arange(1, n, dtype=np.uint32), np.ones(n - 1)


def _run(n, lo, hi, st, mesh):
    d = O.D3(n, lo, hi, st)
    if mesh:
        d.use_mesh()
    d.tick(O.D3_TICKS)
    return d.positions()


def test_the_layout_is_finite_and_the_same_run_to_run():
    """tests.rs:85-96."""
    a = _run(120, *_line(120), True)
    b = _run(120, *_line(120), True)
    assert np.isfinite(a).all() and np.array_equal(a, b)


def test_a_chain_settles_to_barnes_huts_scale():
    """tests.rs:98-127: the mean link within 5% of Barnes-Hut's, no link collapsed."""
    pm = _run(60, *_line(60), True)
    bh = _run(60, *_line(60), False)
    link = lambda p: np.hypot(*np.diff(p, axis=0).T)  # noqa: E731
    assert abs(link(pm).mean() / link(bh).mean() - 1.0) < 0.05
    assert link(pm).min() > 1.0


@pytest.mark.parametrize("n", [0, 1])
def test_an_empty_and_a_single_node_graph_run(n):
    p = _run(n, [], [], [], True)
    assert p.shape == (n, 2) and np.isfinite(p).all()


def test_the_mesh_is_other_bytes_than_the_tree():
    """tests.rs:138-156's second half: the mesh tick is not the tree's."""
    assert not np.array_equal(_run(40, *_line(40), True), _run(40, *_line(40), False))
