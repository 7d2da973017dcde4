"""The oracle pinned: golden vectors, networkx, and the reference's own unit tests.

Everything here runs on the CPU. The oracle (oracle/fa2_oracle.c) is the FP64
restatement of graph-core's FA2 tick that the CUDA engine is checked against.
"""

import json
import os

import networkx as nx
import numpy as np
import pytest

from oracle import oracle as O
from tests.conftest import REFERENCE

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "fa2_nx_gate.jsonl")
REF_FIXTURE = os.path.join(REFERENCE, "crates/graph-cli/tests/fixtures/fa2-nx-reference.jsonl")
CEILING = 1e-7  # crates/graph-cli/src/oracle_python/fa2.rs:72-78


def gate_state(n, **kw):
    s, d, w = O.gate_edges(n)
    lo, hi, ws = O.simple_graph(n, s, d, w)
    return O.State(n, lo, hi, **kw), (lo, hi, ws)


def rel_gap(got, want):
    ext = (want.max(0) - want.min(0)).max()
    return float(np.abs(got - want).max() / max(ext, 1e-300))


def line(n):
    """forceatlas2/tests.rs:5-11: n{i-1} - n{i}."""
    src = np.arange(0, n - 1, dtype=np.uint32)
    dst = np.arange(1, n, dtype=np.uint32)
    return O.simple_graph(n, src, dst)


def bh_graph(n):
    """state/barnes_hut/tests.rs:103-114: node i linked to i/2 and (7i+3) % i."""
    src, dst = [], []
    for i in range(1, n):
        for j in (i // 2, (i * 7 + 3) % i):
            src.append(j)
            dst.append(i)
    return O.simple_graph(n, np.array(src, np.uint32), np.array(dst, np.uint32))


@pytest.mark.skipif(not os.path.exists(REF_FIXTURE), reason="reference tree not present")
def test_committed_golden_is_the_reference_fixture():
    """tests/golden/make_golden.py regenerates the reference's pinned networkx fixture."""
    a = [json.loads(x) for x in open(GOLDEN)]
    b = [json.loads(x) for x in open(REF_FIXTURE)]
    assert a == b


def test_oracle_matches_networkx_golden_vectors():
    """crates/graph-cli/tests/cli_fa2.rs:16-28: 64 gate seeds, 2 iterations, ceiling 1e-7."""
    worst = 0.0
    for line_ in open(GOLDEN):
        d = json.loads(line_)
        st, _ = gate_state(d["n"], seed=0, dim=2, theta=-1.0)
        st.run(d["max_iter"])
        worst = max(worst, rel_gap(st.positions(), np.column_stack([d["x"], d["y"]])))
    assert worst < CEILING, worst
    assert worst < 1e-12, worst  # the restatement is exact to rounding, well under the ceiling


def test_oracle_matches_the_3d_networkx_gate_fixture():
    """The 3D gate (docs/measurements/p12-t4b.md:67-80: networkx at dim 3, 2 iterations,
    ceiling 1e-7) over the committed fixture made by tests/golden/make_golden_3d.py."""
    worst = 0.0
    for line_ in open(os.path.join(HERE, "golden", "fa2_nx_gate_3d.jsonl")):
        d = json.loads(line_)
        st, _ = gate_state(d["n"], seed=0, dim=3, theta=-1.0)
        st.run(d["max_iter"])
        worst = max(worst, rel_gap(st.positions(), np.column_stack([d["x"], d["y"], d["z"]])))
    assert worst < 1e-12, worst


def nx_run(n, lo, hi, w, start, iters, **opts):
    g = nx.Graph()
    g.add_nodes_from(range(n))
    for a, b, c in zip(lo.tolist(), hi.tolist(), w.tolist()):
        g.add_edge(a, b, weight=c)
    pos = {i: start[i].copy() for i in range(n)}
    out = nx.forceatlas2_layout(g, pos=pos, max_iter=iters, **opts)
    return np.array([out[i] for i in range(n)])


@pytest.mark.parametrize("opts", [
    dict(linlog=True),
    dict(distributed_action=True),
    dict(strong_gravity=True),
    dict(weight="weight"),
    dict(linlog=True, distributed_action=True, weight="weight"),
    dict(dim=3),
    dict(dim=3, strong_gravity=True, linlog=True),
])
def test_oracle_options_match_networkx(opts):
    """The options graph-core does not implement, pinned to networkx 3.6 itself."""
    dim = opts.get("dim", 2)
    rng = np.random.default_rng(11)
    for n in (40, 150, 333):
        s, d, _ = O.gate_edges(n)
        lo, hi, _ = O.simple_graph(n, s, d)
        w = rng.lognormal(0.0, 0.5, len(lo))
        start = O.initial_positions(n, 0, dim)
        kw = dict(dim=dim, theta=-1.0, lin_log=int(opts.get("linlog", False)),
                  dissuade_hubs=int(opts.get("distributed_action", False)),
                  strong_gravity=int(opts.get("strong_gravity", False)),
                  edge_weight_influence=1.0 if "weight" in opts else 0.0)
        st = O.State(n, lo, hi, w=w, pos0=start, **kw)
        st.run(2)
        nx_opts = {k: v for k, v in opts.items() if k != "dim"}
        want = nx_run(n, lo, hi, w, start, 2, **nx_opts)
        assert rel_gap(st.positions(), want) < CEILING, (opts, n)


def errors(approx, exact):
    """barnes_hut/tests.rs:128-141: (per-node rms relative, whole-field relative)."""
    d2 = ((approx - exact) ** 2).sum(1)
    e2 = (exact ** 2).sum(1)
    return float(np.sqrt((d2 / e2).mean())), float(np.sqrt(d2.sum() / e2.sum()))


def settling(n, iterations):
    lo, hi, _ = bh_graph(n)
    st = O.State(n, lo, hi, max_iter=iterations, theta=-1.0)
    st.run(iterations)
    return st, lo, hi


def repulsion_on(st, lo, hi, theta):
    n = st.n
    probe = O.State(n, lo, hi, pos0=st.positions(), theta=theta)
    probe.set_scalars(**{k: v for k, v in st.scalars().items()
                         if k in ("swing", "traction", "speed", "speed_efficiency", "iter_no")})
    return probe.accumulate(2)


def test_closed_angle_sums_every_pair_exactly():
    """barnes_hut/tests.rs:154-164: theta = 0 tree == dense within 1e-12."""
    st, lo, hi = settling(400, 5)
    exact = repulsion_on(st, lo, hi, -1.0)
    tree = repulsion_on(st, lo, hi, 0.0)
    node, total = errors(tree, exact)
    assert node < 1e-12 and total < 1e-12, (node, total)


@pytest.mark.parametrize("n,iterations", [(1500, 0), (1500, 30), (1500, 100), (5000, 100)])
def test_far_cell_error_is_a_few_percent(n, iterations):
    """barnes_hut/tests.rs:166-182: theta 0.8, per-node rms < 2%, field < 5%."""
    st, lo, hi = settling(n, iterations)
    exact = repulsion_on(st, lo, hi, -1.0)
    tree = repulsion_on(st, lo, hi, 0.8)
    node, total = errors(tree, exact)
    assert node < 0.02 and total < 0.05, (node, total)


def test_tree_run_is_deterministic_and_finite():
    """barnes_hut/tests.rs:184-194."""
    lo, hi, _ = bh_graph(300)
    runs = []
    for _ in range(2):
        st = O.State(300, lo, hi, theta=0.8)
        st.run(100)
        runs.append(st.positions())
    assert np.array_equal(runs[0], runs[1])
    assert np.isfinite(runs[0]).all()


def test_gravity_multiplies_the_unit_vector():
    """state/tests.rs:26-62: u after one gravity pass is -g * (c / norm), bit for bit."""
    lo, hi, _ = line(20)
    st = O.State(20, lo, hi, theta=-1.0)
    u = st.accumulate(4)
    mean = st.mean()
    pos, mass = st.positions(), st.mass()
    same = differ = 0
    for i in range(20):
        c = pos[i] - mean
        norm = np.sqrt(c[0] * c[0] + c[1] * c[1])
        g = 1.0 * mass[i]
        for a in range(2):
            unit_first = -g * (c[a] / norm)
            offset_first = -g * c[a] / norm
            assert u[i, a] == unit_first
            if unit_first == offset_first:
                same += 1
            else:
                differ += 1
    assert differ > 0


def test_coincident_pair_is_nudged_by_the_counter_hash():
    """state/tests.rs:64-94."""
    lo, hi, _ = line(2)
    st = O.State(2, lo, hi, theta=-1.0)
    p = st.positions()
    p[1] = p[0]
    st.set_positions(p)
    d = st.repel_delta(0, 1)
    assert d[0] != 0.0 or d[1] != 0.0
    assert abs(d[0]) <= 5e-7 and abs(d[1]) <= 5e-7
    p[1, 0] = p[0, 0] + 1e-8
    p[1, 1] = p[0, 1] - 1e-8
    st.set_positions(p)
    want = np.array([p[0, 0] - p[1, 0], p[0, 1] - p[1, 1]])
    assert np.array_equal(st.repel_delta(0, 1), want)


def test_jiggle_is_symmetric_and_never_zero():
    """rng.rs:46-84: keyed on the unordered pair; the 0.5 word is moved off zero."""
    for t in range(50):
        a = O.jiggle(7, t, 0, 3, 9)
        assert a == O.jiggle(7, t, 0, 9, 3)
        assert a != 0.0 and abs(a) <= 5e-7


def test_empty_and_single_node():
    """forceatlas2/tests.rs:222-255."""
    st = O.State(0, np.zeros(0, np.uint32), np.zeros(0, np.uint32), theta=0.8)
    st.run(100)
    assert st.positions().shape == (0, 2)
    st = O.State(1, np.zeros(0, np.uint32), np.zeros(0, np.uint32), theta=0.8)
    st.run(100)
    assert np.isfinite(st.positions()).all()


def test_depth_cap_only_changes_unseparated_points():
    """A Morton-depth cap leaves the tree alone while points separate above it."""
    lo, hi, _ = bh_graph(800)
    rng = np.random.default_rng(3)
    pos = rng.uniform(-500, 500, (800, 2))
    a = O.State(800, lo, hi, pos0=pos, theta=0.8)
    b = O.State(800, lo, hi, pos0=pos, theta=0.8, depth_cap=32)
    assert np.array_equal(a.accumulate(7), b.accumulate(7))


def test_quadtree_cells_cover_their_points_and_subtrees_are_contiguous():
    """layout/force/quadtree/tests.rs: cover containment, subtree contiguity, chains."""
    rng = np.random.default_rng(5)
    n = 500
    pos = np.round(rng.uniform(0, 30, (n, 2)))  # many exact coincidences
    st = O.State(n, np.zeros(0, np.uint32), np.zeros(0, np.uint32), pos0=pos, theta=0.8)
    st.accumulate(2)
    t = st.tree()
    order = t["order"]
    assert sorted(order.tolist()) == list(range(n))
    K = len(t["skip"])
    for k in range(K):
        s, e, sk = t["start"][k], t["end"][k], t["skip"][k]
        assert k < sk <= K and s < e
        if sk != k + 1:  # children tile the parent's points
            c, q = k + 1, s
            while c < sk:
                assert t["start"][c] == q
                q = t["end"][c]
                c = t["skip"][c]
            assert q == e
        else:  # a leaf's points are one coincident chain
            pts = pos[order[s:e]]
            assert (pts == pts[0]).all()


def test_oracle_3d_tree_theta0_equals_dense():
    """The octree arm (no reference counterpart) at theta 0 is the dense sum."""
    lo, hi, _ = bh_graph(300)
    rng = np.random.default_rng(8)
    pos = rng.uniform(0, 100, (300, 3))
    a = O.State(300, lo, hi, pos0=pos, dim=3, theta=-1.0).accumulate(2)
    b = O.State(300, lo, hi, pos0=pos, dim=3, theta=0.0).accumulate(2)
    node, total = errors(b, a)
    assert node < 1e-12 and total < 1e-12


def test_oracle_stress_matches_the_references_unit_tests():
    """crates/graph-cli/src/bench/tests/plan.rs:70-90, restated."""
    assert O.stress([0.0, 2.0, 4.0], [0.0] * 3, [0, 1], [1, 2]) == 0.0  # isometric path
    assert O.stress([0.0, 1.0, 0.0], [0.0] * 3, [0, 1], [1, 2]) == (8.0 / 12.0) ** 0.5  # folded
    assert O.stress([5.0] * 3, [5.0] * 3, [0, 1], [1, 2]) == 1.0  # collapsed
    assert O.stress([0.0, 1.0], [0.0, 0.0], [], []) == 1.0  # edgeless
    assert O.stress([0.0, 1.0, 100.0, 101.0], [0.0] * 4, [0, 2], [1, 3]) == 0.0  # two components


def test_oracle_bfs_hops_on_a_path_with_a_loop_and_a_stray_node():
    h = O.bfs_hops(5, [0, 1, 2, 2], [1, 2, 3, 2], [0, 3])
    none = np.iinfo(np.uint32).max
    assert h[0].tolist() == [0, 1, 2, 3, none]
    assert h[1].tolist() == [3, 2, 1, 0, none]


@pytest.mark.parametrize("n", [2, 3, 17, 601, 20_000])
def test_product_gate_generator_draws_the_oracles_model(n):
    from graph_render_b200 import synth

    for a, b in zip(synth.gate(n), O.gate_edges(n)):
        assert np.array_equal(a, b)
