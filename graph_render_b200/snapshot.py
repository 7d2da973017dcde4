"""The snapshot's binary face: the bytes the reference's consumers read.

Restates graph-contract's snapshot encoding (docs/contract/binary-layout.md;
crates/graph-contract/src/binary.rs:170-197 to_bytes, binary/decode.rs:12-41
decode, snapshot.rs:132-167 header) and graph-core's `layout::snapshot`
(crates/graph-core/src/layout/mod.rs:198-232): the topology's ids and edge
endpoints in its own order, the layout's node columns, the edge geometry and the
notes. Columnar little-endian u32 / f32, every section a multiple of 4 bytes.

A layout's positions from the CUDA engine (`Fa2.positions()` or `run_values`)
become the same bytes a graph-core layout's Geometry would, so they flow through
the reference's snapshot consumers unchanged.
"""

from __future__ import annotations

import struct
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

MAGIC = b"GMSN"
HEADER_LEN = 28

# NodeGeometryKind / EdgeGeometryKind tags (geometry.rs:45-82)
POINT, CIRCLE, BOX = 0, 1, 2
LINE, POLYLINE, CURVE = 0, 1, 2
NODE_COLUMNS = {POINT: (), CIRCLE: ("r",), BOX: ("w", "h")}

# Note codes (notes.rs:99-108, 165-176); 6 is reserved and refused
NOTE_CODES = {1: "hierarchy.cycle_edge_dropped", 2: "hierarchy.extra_parent_dropped",
              3: "packing.approximate", 4: "dag.dummy_budget_exceeded", 5: "dag.edge_reversed"}
SNAPSHOT_WIDE = 0xFFFFFFFF


class SnapshotError(ValueError):
    """What Snapshot construction or decoding refuses (snapshot/error.rs)."""


def label_for(dim: int) -> Tuple[int, int]:
    """The format label follows the geometry: 0.3 for 2D, 0.4 for 3D (layout/mod.rs:213-218)."""
    return (0, 4) if dim == 3 else (0, 3)


def _padding(length: int) -> int:
    return (4 - length % 4) % 4


def _table(name: str, strs: Sequence[str]) -> bytes:
    """CSR string table: count + 1 u32 offsets, the UTF-8 bytes, zero padding to 4."""
    raw = [s.encode("utf-8") for s in strs]
    if len(set(raw)) != len(raw):
        raise SnapshotError(f"{name}: ids must be unique")
    offs = np.zeros(len(raw) + 1, "<u4")
    if raw:
        offs[1:] = np.cumsum([len(b) for b in raw])
    text = b"".join(raw)
    return offs.tobytes() + text + b"\0" * _padding(len(text))


@dataclass
class Snapshot:
    """One snapshot (SnapshotParts): valid by construction, like the reference's."""

    node_ids: List[str]
    edge_ids: List[str]
    source: np.ndarray
    target: np.ndarray
    x: np.ndarray
    y: np.ndarray
    z: Optional[np.ndarray] = None
    node_kind: int = POINT
    sizes: Tuple[np.ndarray, ...] = ()  # r (Circle) or w, h (Box)
    edge_kind: int = LINE
    degree: int = 0  # Curve only
    edge_offsets: Optional[np.ndarray] = None  # Polyline / Curve
    edge_points: Optional[np.ndarray] = None  # f32 x 2 per point
    notes: List[Tuple[int, int]] = field(default_factory=list)

    def __post_init__(self):
        n, m = len(self.node_ids), len(self.edge_ids)
        for name, ids in (("node.id", self.node_ids), ("edge.id", self.edge_ids)):
            if len(set(ids)) != len(ids):
                raise SnapshotError(f"{name}: ids must be unique")
        self.source = np.ascontiguousarray(self.source, np.uint32)
        self.target = np.ascontiguousarray(self.target, np.uint32)
        cols = [np.ascontiguousarray(c, np.float32) for c in (self.x, self.y)]
        self.x, self.y = cols
        if self.z is not None:
            self.z = np.ascontiguousarray(self.z, np.float32)
        self.sizes = tuple(np.ascontiguousarray(s, np.float32) for s in self.sizes)
        if len(self.source) != m or len(self.target) != m:
            raise SnapshotError("edge.source / edge.target: length must be the edge count")
        if m and (int(self.source.max()) >= n or int(self.target.max()) >= n):
            raise SnapshotError("edge endpoint out of range")
        names = ("node.x", "node.y") + (("node.z",) if self.z is not None else ())
        for name, c in zip(names, (self.x, self.y) + ((self.z,) if self.z is not None else ())):
            if len(c) != n:
                raise SnapshotError(f"{name}: length must be the node count")
            if not np.isfinite(c).all():
                raise SnapshotError(f"{name}: non-finite value")
        if self.node_kind not in NODE_COLUMNS:
            raise SnapshotError(f"unknown node geometry tag {self.node_kind}")
        if len(self.sizes) != len(NODE_COLUMNS[self.node_kind]):
            raise SnapshotError("size columns do not match the node kind")
        for name, c in zip(NODE_COLUMNS[self.node_kind], self.sizes):
            if len(c) != n or not np.isfinite(c).all() or (c < 0).any():
                raise SnapshotError(f"node.{name}: n finite values >= 0")
        if self.edge_kind not in (LINE, POLYLINE, CURVE):
            raise SnapshotError(f"edge geometry tag {self.edge_kind} is reserved or unknown")
        if self.edge_kind != LINE:
            self.edge_offsets = np.ascontiguousarray(self.edge_offsets, np.uint32)
            self.edge_points = np.ascontiguousarray(self.edge_points, np.float32).reshape(-1)
            o = self.edge_offsets
            if len(o) != m + 1 or o[0] != 0 or (np.diff(o.astype(np.int64)) < 0).any():
                raise SnapshotError("edge.offsets: m + 1 non-decreasing values from 0")
            if len(self.edge_points) != 2 * int(o[-1]) or not np.isfinite(self.edge_points).all():
                raise SnapshotError("edge.pts: 2 finite values per point")
            if self.edge_kind == CURVE and self.degree < 1:
                raise SnapshotError("edge.degree must be at least 1")
        prev = None
        for code, index in self.notes:
            if code not in NOTE_CODES:
                raise SnapshotError(f"note code {code} is reserved or unknown")
            if code == 3 and index != SNAPSHOT_WIDE:
                raise SnapshotError("packing.approximate is snapshot-wide")
            if code != 3 and index >= m:
                raise SnapshotError("note index must be an edge position")
            if prev is not None and (code, index) <= prev:
                raise SnapshotError("notes must be strictly ascending by (code, index)")
            prev = (code, index)

    @property
    def dim(self) -> int:
        return 3 if self.z is not None else 2

    def to_bytes(self) -> bytes:
        major, minor = label_for(self.dim)
        n, m = len(self.node_ids), len(self.edge_ids)
        out = [MAGIC, struct.pack("<II", major, minor),
               bytes([self.node_kind, self.edge_kind, 1 if self.dim == 3 else 0, 0]),
               struct.pack("<III", 1, n, m),
               _table("node.id", self.node_ids), _table("edge.id", self.edge_ids),
               self.source.astype("<u4").tobytes(), self.target.astype("<u4").tobytes(),
               self.x.astype("<f4").tobytes(), self.y.astype("<f4").tobytes()]
        if self.z is not None:
            out.append(self.z.astype("<f4").tobytes())
        out += [c.astype("<f4").tobytes() for c in self.sizes]
        if self.edge_kind == CURVE:
            out.append(struct.pack("<I", self.degree))
        if self.edge_kind != LINE:
            out += [self.edge_offsets.astype("<u4").tobytes(), self.edge_points.astype("<f4").tobytes()]
        codes = np.array([c for c, _ in self.notes], "<u4")
        idx = np.array([i for _, i in self.notes], "<u4")
        out += [struct.pack("<I", len(self.notes)), codes.tobytes(), idx.tobytes()]
        return b"".join(out)


class _Reader:
    def __init__(self, b: bytes):
        self.b, self.at = b, 0

    def take(self, k: int) -> bytes:
        if self.at + k > len(self.b):
            raise SnapshotError("truncated")
        v = self.b[self.at:self.at + k]
        self.at += k
        return v

    def u32s(self, k: int) -> np.ndarray:
        return np.frombuffer(self.take(4 * k), "<u4").astype(np.uint32)

    def f32s(self, k: int) -> np.ndarray:
        return np.frombuffer(self.take(4 * k), "<f4").astype(np.float32)

    def table(self, k: int) -> List[str]:
        offs = self.u32s(k + 1)
        text = self.take(int(offs[-1]))
        self.take(_padding(len(text)))
        return [text[offs[i]:offs[i + 1]].decode("utf-8") for i in range(k)]


def from_bytes(b: bytes) -> Snapshot:
    """Decodes the binary face; refuses what construction refuses, plus truncation
    and trailing bytes (binary/decode.rs:12-41)."""
    r = _Reader(b)
    if r.take(4) != MAGIC:
        raise SnapshotError("BadMagic")
    major, minor = struct.unpack("<II", r.take(8))
    if major > 0:
        raise SnapshotError(f"format major {major} is newer than this reader")
    node_kind, edge_kind, dim_byte, pad = r.take(4)
    if dim_byte > 1:
        raise SnapshotError("ReservedDim")
    if pad != 0:
        raise SnapshotError("header padding must be 0")
    stages, n, m = struct.unpack("<III", r.take(12))
    if stages != 1:
        raise SnapshotError("stage count must be 1")
    node_ids, edge_ids = r.table(n), r.table(m)
    source, target = r.u32s(m), r.u32s(m)
    x, y = r.f32s(n), r.f32s(n)
    z = r.f32s(n) if dim_byte == 1 else None
    if node_kind not in NODE_COLUMNS:
        raise SnapshotError(f"unknown node geometry tag {node_kind}")
    sizes = tuple(r.f32s(n) for _ in NODE_COLUMNS[node_kind])
    degree, offs, pts = 0, None, None
    if edge_kind == CURVE:
        (degree,) = struct.unpack("<I", r.take(4))
    if edge_kind in (POLYLINE, CURVE):
        offs = r.u32s(m + 1)
        pts = r.f32s(2 * int(offs[-1]))
    elif edge_kind != LINE:
        raise SnapshotError(f"edge geometry tag {edge_kind} is reserved or unknown")
    notes: List[Tuple[int, int]] = []
    if (major, minor) >= (0, 3):
        (k,) = struct.unpack("<I", r.take(4))
        codes, idx = r.u32s(k), r.u32s(k)
        notes = list(zip(codes.tolist(), idx.tolist()))
    if r.at != len(b):
        raise SnapshotError("trailing bytes")
    return Snapshot(node_ids, edge_ids, source, target, x, y, z, node_kind, sizes, edge_kind, degree, offs, pts,
                    notes)


def of_layout(node_ids: Sequence[str], edge_ids: Sequence[str], source, target, positions) -> Snapshot:
    """layout::snapshot for a point layout (Geometry::points, layout/mod.rs:116-122):
    the topology's ids and endpoints, the positions as f32 x, y (and z at dim 3),
    Line edges, no notes. positions: n x dim (the engine's output, node order)."""
    p = np.asarray(positions, np.float32)
    if p.ndim != 2 or p.shape[1] not in (2, 3):
        raise SnapshotError("positions must be n x 2 or n x 3")
    return Snapshot(list(node_ids), list(edge_ids), source, target, p[:, 0], p[:, 1],
                    p[:, 2] if p.shape[1] == 3 else None)


def of_geometry(node_ids: Sequence[str], edge_ids: Sequence[str], topology, geometry) -> Snapshot:
    """layout::snapshot(topology, geometry) for the registry mirror's types: a
    `registry.Topology` (edge endpoints in its order) and the `registry.Geometry`
    that `Capability.run_params` returns."""
    z = geometry.z if geometry.dim == 3 else None
    return Snapshot(list(node_ids), list(edge_ids), topology.source, topology.target, geometry.x, geometry.y, z)


def gate_ids(n: int, m: int) -> Tuple[List[str], List[str]]:
    """The gate model's node and edge ids (crates/graph-core/src/synthetic.rs:107-131):
    node i is "bench:db-{i % 8}:{i}", edge k is "bench-e-{k}"."""
    return [f"bench:db-{i % 8}:{i}" for i in range(n)], [f"bench-e-{k}" for k in range(m)]


__all__ = ["Snapshot", "SnapshotError", "from_bytes", "of_layout", "of_geometry", "gate_ids", "label_for", "POINT", "CIRCLE",
           "BOX", "LINE", "POLYLINE", "CURVE"]
