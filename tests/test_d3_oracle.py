"""The d3-force Barnes-Hut oracle (oracle/fa2_oracle.c, orc_d3_*) pinned to the
reference's own golden digests, bit for bit (CPU).

- crates/graph-core/src/layout/force/session/tests/golden.rs FROZEN: for the gate
  model at seeds 0..64 (2 + seed nodes), sha256 of the frozen layout's f32 columns,
  all of x then all of y (tests/golden/d3_frozen_sha256.txt);
- harness/golden-2d-before.txt: sha256 of `graph-cli snapshot --layout
  layout.force.barnes_hut --seed S` for S = 0..7, through this repository's
  snapshot encoder (tests/golden/fa2_snapshot_sha256.txt).

The layout is 112 ticks of link, many-body over the insertion quadtree, center and
collide from the golden spiral, every value FP64, so one differing ulp anywhere
changes a digest.
"""

import hashlib
import os

import numpy as np
import pytest

from graph_render_b200 import snapshot as S
from oracle import oracle as O

HERE = os.path.join(os.path.dirname(__file__), "golden")


def _frozen():
    out = {}
    for line in open(os.path.join(HERE, "d3_frozen_sha256.txt")):
        if not line.startswith("#"):
            seed, digest = line.split()
            out[int(seed)] = digest
    return out


def _layout(seed):
    n = 2 + seed % 600
    src, dst, st = O.gate_edges(n)
    lo, hi, w = O.simple_graph(n, src, dst, st)
    d = O.D3(n, lo, hi, w)
    d.tick(O.D3_TICKS)
    return n, src, dst, d.positions()


def test_the_frozen_table_has_65_seeds():
    assert sorted(_frozen()) == list(range(65))


@pytest.mark.parametrize("seed", range(65))
def test_oracle_reproduces_the_frozen_column_digest(seed):
    _, _, _, p = _layout(seed)
    p = p.astype(np.float32)
    assert hashlib.sha256(p[:, 0].tobytes() + p[:, 1].tobytes()).hexdigest() == _frozen()[seed]


@pytest.mark.parametrize("seed", range(8))
def test_oracle_reproduces_the_snapshot_hash(seed):
    want = [ln.split()[2] for ln in open(os.path.join(HERE, "fa2_snapshot_sha256.txt"))
            if ln.startswith(f"layout.force.barnes_hut {seed} ")][0]
    n, src, dst, p = _layout(seed)
    node_ids, edge_ids = S.gate_ids(n, len(src))
    assert hashlib.sha256(S.of_layout(node_ids, edge_ids, src, dst, p).to_bytes()).hexdigest() == want


def test_alpha_follows_the_cooling_schedule():
    n = 20
    src, dst, st = O.gate_edges(n)
    lo, hi, w = O.simple_graph(n, src, dst, st)
    d = O.D3(n, lo, hi, w)
    a = 1.0
    for _ in range(5):
        d.tick(1)
        a += (0.0 - a) * 0.06
        assert d.alpha() == a
