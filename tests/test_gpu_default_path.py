"""The drop-in default path: a graph-core caller's run, with no positions given.

graph-core's FA2 starts every run from Mulberry32(seed) uniform in [0, 1)^dim
(crates/graph-core/src/layout/forceatlas2/state.rs:272-283,
crates/graph-core/src/synthetic.rs:37-50) and takes no start positions. Its
gate is the networkx fixture for gate seeds 0..63 at 2 iterations
(crates/graph-cli/tests/cli_fa2.rs:16-28, fixture
crates/graph-cli/tests/fixtures/fa2-nx-reference.jsonl, committed here as
tests/golden/fa2_nx_gate.jsonl). These tests run that path through the
registry face and the C ABI with no pos0:

- the engine's own start equals f32(the oracle's Mulberry32 start), bit for bit;
- run_params at theta 0 (the exact sum) against the fixture, within 1e-5 of the
  extent (the engine computes in FP32 from an FP32 start; the fixture is FP64);
- an empty parameter buffer (the reference's defaults: theta 0.8, scaling 2,
  gravity 1, seed 0) on the 1,500-node SBM, forces within 1e-5 relative L2 of
  the oracle's at ticks 0 and 60, from the start the engine draws itself.
"""

import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from graph_render_b200 import FA2_ID, Fa2, Topology, find, params_bytes, synth
from tests.gpu_util import oracle_state, rel_l2

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "fa2_nx_gate.jsonl")


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("n,seed", [(1, 0), (2, 0), (65, 0), (1500, 0), (4097, 7), (100_000, 4294967295)])
def test_the_engines_own_start_is_the_references_mulberry32(n, seed, dim):
    s, d, _ = O.gate_edges(max(n, 2))
    keep = (s < n) & (d < n)
    with Fa2(n, s[keep], d[keep], params=dict(seed=seed, dim=dim)) as eng:
        got = eng.positions()
    want = O.initial_positions(n, seed, dim).astype(np.float32)
    assert got.dtype == np.float32 and got.shape == (n, dim)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("dim", [2, 3])
def test_run_params_without_positions_reproduces_the_networkx_fixture(dim):
    # 2D: the reference's own fixture; 3D: the same gate at dim 3 (its 1e-7 gate,
    # docs/measurements/p12-t4b.md:67-80), from tests/golden/make_golden_3d.py
    cap = find(FA2_ID)
    worst, worst_seed = 0.0, -1
    path = GOLDEN if dim == 2 else os.path.join(HERE, "golden", "fa2_nx_gate_3d.jsonl")
    lines = [json.loads(x) for x in open(path)]
    assert len(lines) == 64
    axes = ("x", "y", "z")[:dim]
    for d in lines:
        n = d["n"]
        src, dst, _ = O.gate_edges(n)
        geom = cap.run_params(Topology(n, src, dst, None),
                              params_bytes(max_iter=d["max_iter"], theta=0.0, dim=dim))
        got = np.column_stack([np.asarray(getattr(geom, a), np.float64) for a in axes])
        want = np.column_stack([d[a] for a in axes])
        ext = (want.max(0) - want.min(0)).max()
        gap = float(np.abs(got - want).max() / ext)
        if gap > worst:
            worst, worst_seed = gap, d["seed"]
    print(f"dim {dim}: worst gap {worst:.3e} of the extent (gate seed {worst_seed})")
    assert worst < 1e-5, (worst, worst_seed)


def test_reference_length_buffer_runs_the_default_start():
    # a 5-value buffer (the reference's own schema) keeps every appended
    # parameter at its default; the run starts from Mulberry32(seed)
    n = 300
    src, dst, _ = O.gate_edges(n)
    topo = Topology(n, src, dst, None)
    five = params_bytes([2, 1.0, 2.0, 1.0, 9])
    eleven = params_bytes(max_iter=2, seed=9)
    a = find(FA2_ID).run_params(topo, five)
    b = find(FA2_ID).run_params(topo, eleven)
    assert np.array_equal(np.asarray(a.x), np.asarray(b.x)) and np.array_equal(np.asarray(a.y), np.asarray(b.y))


@pytest.mark.parametrize("ticks", [0, 60])
def test_empty_params_on_the_sbm_match_the_oracle_from_the_engines_start(ticks):
    wl = synth.sbm_1500()
    with Fa2(wl.n, wl.src, wl.dst, params=b"") as eng:
        assert eng.values[6] == 0.8 and eng.values[4] == 0 and eng.dim == 2
        if ticks == 0:
            assert np.array_equal(eng.positions(), O.initial_positions(wl.n, 0, 2).astype(np.float32))
        eng.tick(ticks)
        pos = eng.positions()
        fg = eng.forces().astype(np.float64)
        assert eng.info()["device_error"] == 0
    st = oracle_state(wl.n, wl.src, wl.dst, None, pos, {})
    fr = st.accumulate(7)
    rel = rel_l2(fg, fr)
    print(f"ticks {ticks}: rel L2 {rel:.3e}")
    assert rel < 1e-5, rel
