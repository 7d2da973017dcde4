"""The particle-mesh many-body pass on the GPU (gr_force_session_use_mesh)
against the FP64 oracle (orc_d3_use_mesh), which passes the reference's own
particle-mesh tests, and against the direct law
(crates/graph-core/src/layout/force/particle_mesh/tests.rs)."""

import numpy as np
import pytest

from graph_render_b200 import PM_ID, ForceParams, ForceSession, Topology, find, stress as S, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


def gpu_field(x, y):
    """The mesh field at every node, from one tick with no edges, no collide,
    zero start velocity: v1 = decay * charge * alpha1 * field."""
    n = len(x)
    prm = ForceParams.defaults(collide_radius=0.0)
    with ForceSession(n, [], [], params=prm, pos0=np.stack([x, y], 1)) as s:
        s.use_mesh()
        s.tick(1)
        v = s.velocities().astype(np.float64)
        a = s.alpha()
    return v / (prm.velocity_decay * prm.charge * a)


def direct(x, y, i, dmin2=1.0, dmax2=520.0 ** 2):
    e = np.zeros(2)
    for j in range(len(x)):
        if j != i:
            rx, ry = x[i] - x[j], y[i] - y[j]
            l = rx * rx + ry * ry
            if l < dmax2:
                l = np.sqrt(dmin2 * l) if l < dmin2 else l
                e -= [rx / l, ry / l]
    return e


def test_the_mesh_field_follows_the_direct_sum_and_the_oracle():
    x = np.array([(i % 8) * 70.0 + (i // 8) * 9.0 for i in range(64)])
    y = np.array([(i // 8) * 70.0 for i in range(64)])
    got = gpu_field(x.astype(np.float32).astype(np.float64), y.astype(np.float32).astype(np.float64))
    want = np.array([direct(x, y, i) for i in range(64)])
    assert np.sqrt(((got - want) ** 2).sum() / (want ** 2).sum()) < 0.05
    o = O.D3(64, [], [], [], pos0=np.stack([x, y], 1))
    o.use_mesh()
    assert rel(got, o.mesh_field()) < 1e-4


def test_random_cloud_field_matches_the_oracle():
    rng = np.random.default_rng(5)
    n = 3000
    p = rng.uniform(0, 2500, (n, 2)).astype(np.float32).astype(np.float64)
    got = gpu_field(p[:, 0], p[:, 1])
    o = O.D3(n, [], [], [], pos0=p)
    o.use_mesh()
    assert rel(got, o.mesh_field()) < 1e-4


def test_a_node_out_of_everyones_range_feels_no_force_from_itself():
    f = gpu_field(np.array([0.0, 3000.0]), np.array([0.0, 17.5]))
    assert np.abs(f).max() < 1e-6


def _cases():
    n, (src, dst, st) = 601, O.gate_edges(601)
    yield "gate601", (n, src, dst, st)
    wl = synth.sbm_1500()
    yield "sbm1500", (wl.n, wl.src, wl.dst, np.random.default_rng(3).uniform(0.4, 0.8, len(wl.src)))


def _oracle(n, src, dst, st):
    lo, hi, w = O.simple_graph(n, src, dst, st)
    o = O.D3(n, lo, hi, w)
    o.use_mesh()
    return o


@pytest.mark.parametrize("at", [0, 20, 80])
@pytest.mark.parametrize("case", list(_cases()), ids=lambda c: c[0])
def test_one_tick_from_the_oracles_state(case, at):
    n, src, dst, st = case[1]
    o = _oracle(n, src, dst, st)
    o.tick(at)
    p = o.positions().astype(np.float32)
    v = o.velocities().astype(np.float32)
    a = o.alpha()
    o.set_state(p.astype(np.float64), v.astype(np.float64), a, at)
    o.tick(1)
    with ForceSession(n, src, dst, st) as s:
        s.use_mesh()
        s.set_state(p, v, a, at)
        s.tick(1)
        gp, gv = s.positions(), s.velocities()
    assert rel(gv, o.velocities()) < 1e-3
    ext = float(np.ptp(o.positions(), axis=0).max())
    assert np.abs(gp - o.positions()).max() / ext < 1e-5


def test_frozen_layout_is_not_worse_than_the_oracles_and_deterministic():
    for n, src, dst, st in (c[1] for c in _cases()):
        g = find(PM_ID).run_params(Topology(n, src, dst, st), b"")
        g2 = find(PM_ID).run_params(Topology(n, src, dst, st), b"")
        assert np.array_equal(g.x, g2.x) and np.array_equal(g.y, g2.y)
        o = _oracle(n, src, dst, st)
        o.tick(O.D3_TICKS)
        po = o.positions()
        sg = S.kruskal_stress(g.x, g.y, src, dst)
        so = O.stress(po[:, 0].astype(np.float32), po[:, 1].astype(np.float32), src, dst)
        assert np.isfinite(g.x).all() and sg <= so + 0.05, (n, sg, so)


@pytest.mark.parametrize("n", [0, 1, 2])
def test_empty_single_and_pair(n):
    with ForceSession(n, [0] if n == 2 else [], [1] if n == 2 else []) as s:
        s.use_mesh()
        s.tick(112)
        assert np.isfinite(s.positions()).all()
