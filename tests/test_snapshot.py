"""The snapshot encoder against the reference's byte contract, and the oracle's
dense FA2 against the reference's own golden snapshot hashes (CPU).

- the contract's pinned 84-byte example (docs/contract/binary-layout.md, "The
  pinned 84-byte example", from crates/graph-contract/src/binary/tests/pinned.rs:9-51)
  and its Curve variant, byte for byte;
- decode(encode(s)) == s for 2D/3D, every node and edge kind, notes;
- the refusals decode and construction share;
- the reference pins the sha256 of `graph-cli snapshot --layout layout.forceatlas2
  --seed S` for S = 0..7 (harness/golden-2d-before.txt:77-84): the gate model with
  2 + S nodes, the dense FA2 at its defaults (100 ticks), settled to f32. The
  oracle's FP64 run through this encoder must hash to exactly those bytes.
"""

import hashlib
import os

import numpy as np
import pytest

from graph_render_b200 import snapshot as S
from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "fa2_snapshot_sha256.txt")

PINNED = bytes.fromhex(
    "474d534e" "00000000" "03000000" "00000000" "01000000" "02000000" "01000000"
    "00000000" "01000000" "03000000" "61626300"
    "00000000" "01000000" "65000000"
    "00000000" "01000000"
    "0000803f" "000020c0" "00000000" "0000003f"
    "00000000")


def tiny(**kw):
    return S.Snapshot(["a", "bc"], ["e"], [0], [1], [1.0, -2.5], [0.0, 0.5], **kw)


def test_pinned_84_bytes():
    b = tiny().to_bytes()
    assert len(b) == 84
    assert b == PINNED


def test_pinned_curve_variant():
    b = tiny(edge_kind=S.CURVE, degree=2, edge_offsets=[0, 1], edge_points=[1.0, 0.5]).to_bytes()
    assert b[13] == 2
    assert b[:13] == PINNED[:13] and b[14:80] == PINNED[14:80]
    assert b[80:] == bytes.fromhex("02000000" "00000000" "01000000" "0000803f" "0000003f" "00000000")


def _same(a: S.Snapshot, b: S.Snapshot):
    assert a.to_bytes() == b.to_bytes()


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("node_kind", [S.POINT, S.CIRCLE, S.BOX])
@pytest.mark.parametrize("edge_kind", [S.LINE, S.POLYLINE, S.CURVE])
def test_round_trip(dim, node_kind, edge_kind):
    rng = np.random.default_rng(dim * 100 + node_kind * 10 + edge_kind)
    n, m = 7, 9
    ids = [f"n{i}-é" * (i % 3) + str(i) for i in range(n)]
    eids = [f"e{k}" for k in range(m)]
    sizes = tuple(rng.uniform(0, 3, n) for _ in S.NODE_COLUMNS[node_kind])
    kw = {}
    if edge_kind != S.LINE:
        per = rng.integers(0, 4, m)
        offs = np.concatenate([[0], np.cumsum(per)])
        kw = dict(edge_offsets=offs, edge_points=rng.normal(size=2 * int(offs[-1])),
                  degree=3 if edge_kind == S.CURVE else 0)
    s = S.Snapshot(ids, eids, rng.integers(0, n, m), rng.integers(0, n, m), rng.normal(size=n),
                   rng.normal(size=n), rng.normal(size=n) if dim == 3 else None, node_kind, sizes, edge_kind,
                   notes=[(1, 2), (1, 5), (3, S.SNAPSHOT_WIDE), (5, 0)], **kw)
    b = s.to_bytes()
    assert len(b) % 4 == 0
    assert b[14] == (1 if dim == 3 else 0)
    assert b[8:12] == (b"\x04\0\0\0" if dim == 3 else b"\x03\0\0\0")
    _same(S.from_bytes(b), s)


def test_refusals():
    b = tiny().to_bytes()
    with pytest.raises(S.SnapshotError):
        S.from_bytes(b[:-1])
    with pytest.raises(S.SnapshotError):
        S.from_bytes(b + b"\0\0\0\0")
    with pytest.raises(S.SnapshotError):
        S.from_bytes(b"GMSX" + b[4:])
    with pytest.raises(S.SnapshotError):
        S.from_bytes(b[:14] + b"\x02" + b[15:])  # dim 2 is reserved
    with pytest.raises(S.SnapshotError):
        S.from_bytes(b[:13] + b"\x03" + b[14:])  # edge tag 3 is reserved
    with pytest.raises(S.SnapshotError):
        tiny(notes=[(2, 0), (1, 0)])  # not ascending
    with pytest.raises(S.SnapshotError):
        tiny(notes=[(6, 0)])  # reserved code
    with pytest.raises(S.SnapshotError):
        S.Snapshot(["a", "a"], [], [], [], [0, 0], [0, 0])  # ids unique
    with pytest.raises(S.SnapshotError):
        S.Snapshot(["a"], [], [], [], [np.nan], [0])  # finite
    with pytest.raises(S.SnapshotError):
        S.Snapshot(["a"], ["e"], [0], [1], [0], [0])  # endpoint range


def _golden(layout):
    out = {}
    for line in open(GOLDEN):
        p = line.split()
        if len(p) == 3 and p[0] == layout:
            out[int(p[1])] = p[2]
    return out


@pytest.mark.parametrize("seed", range(8))
def test_oracle_dense_fa2_reproduces_the_reference_snapshot_hash(seed):
    """Bit-exact: the reference's f32 columns come from its FP64 state after 100
    ticks; one differing ulp anywhere changes the hash."""
    want = _golden("layout.forceatlas2")[seed]
    n = 2 + seed % 600
    src, dst, _ = O.gate_edges(n)
    lo, hi, _ = O.simple_graph(n, src, dst)
    st = O.State(n, lo, hi, dim=2, theta=-1.0)  # dense; defaults: start Mulberry32(0), 100 ticks
    st.run(100)
    node_ids, edge_ids = S.gate_ids(n, len(src))
    b = S.of_layout(node_ids, edge_ids, src, dst, st.positions()).to_bytes()
    assert hashlib.sha256(b).hexdigest() == want
