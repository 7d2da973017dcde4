"""Host mirror of graph-core's layout registry for the ForceAtlas2 entry.

Follows the reference's types and rules, with the engine behind them:

- ``ParamSpec`` / ``ParamsView.validate`` / ``values`` / ``encode``:
  crates/graph-contract/src/params.rs:50-205 (positional little-endian f64,
  empty buffer = defaults, wrong length refused, non-finite / out-of-range /
  non-integral Int / non-0-1 Bool refused by index, never clamped; the
  gm_layout_params wire body).
- ``Capability`` with ``run_params`` / ``params_values`` / ``run_values``:
  crates/graph-core/src/registry/capability.rs:40-50, registry/params.rs:140-181.
- ``LAYOUTS`` / ``find``: crates/graph-core/src/registry.rs:62-64.
- ``StageError``: crates/graph-core/src/stage.rs:35-52 (``Param{name, rule}``,
  ``NonFinite{column}``).
- ``Topology`` holds what the FA2 stage reads of graph-core's indexed topology:
  the node count and the raw edges (source, target, strength) in edge order.
- ``Geometry``: f32 point columns x, y (and z at dim 3), in node order
  (crates/graph-core/src/layout/mod.rs:54-66, 116-122).
"""

from __future__ import annotations

import ctypes as C
import struct
from dataclasses import dataclass, field
from typing import Callable, List, Optional, Sequence

import numpy as np

from . import _native as N

INT, FLOAT, BOOL = N.KIND_INT, N.KIND_FLOAT, N.KIND_BOOL


@dataclass(frozen=True)
class ParamSpec:
    name: str
    kind: int
    min: float
    max: float
    default: float
    step: float
    doc: str


class ParamsError(Exception):
    """graph-contract ParamsError: NotAccepted, Malformed or OutOfRange{index}."""

    def __init__(self, kind: str, index: Optional[int] = None):
        super().__init__(kind if index is None else f"{kind}[{index}]")
        self.kind = kind
        self.index = index


class StageError(Exception):
    """graph-core StageError: Param{name, rule} or NonFinite{column}."""

    def __init__(self, kind: str, name: str = "", rule: str = "", code: int = 0):
        super().__init__(f"{kind}: {name} {rule}".strip())
        self.kind = kind
        self.name = name
        self.rule = rule
        self.code = code


def _kind_holds(kind: int, v: float) -> bool:
    if kind == INT:
        return float(v).is_integer()
    if kind == BOOL:
        return v in (0.0, 1.0)
    return True


class ParamsView:
    """params.rs:95-205: a layout's published parameters and the buffer rules."""

    def __init__(self, specs: Sequence[ParamSpec], accepted_lengths: Sequence[int] = ()):
        self._specs = tuple(specs)
        # Buffer lengths (in values) accepted besides the full schema: the
        # engine also takes the reference's own 5-value FA2 buffer.
        self._lengths = tuple(sorted(set(accepted_lengths) | {len(self._specs)}))

    def specs(self):
        return self._specs

    def __len__(self):
        return len(self._specs)

    def is_empty(self) -> bool:
        return not self._specs

    def buffer_len(self) -> int:
        return 8 * len(self._specs)

    def defaults(self) -> List[float]:
        return [s.default for s in self._specs]

    def value(self, b: bytes, i: int) -> float:
        return struct.unpack_from("<d", b, 8 * i)[0]

    def validate(self, b: bytes) -> None:
        if self.is_empty() and len(b):
            raise ParamsError("NotAccepted")
        if len(b) % 8 or len(b) // 8 not in self._lengths:
            raise ParamsError("Malformed")
        for i in range(len(b) // 8):
            v = self.value(b, i)
            s = self._specs[i]
            if not np.isfinite(v) or v < s.min or v > s.max or not _kind_holds(s.kind, v):
                raise ParamsError("OutOfRange", i)

    def values(self, b: bytes) -> List[float]:
        self.validate(b)
        out = self.defaults()
        for i in range(len(b) // 8):
            out[i] = self.value(b, i)
        return out

    def encode(self) -> bytes:
        """The gm_layout_params wire body (docs/contract/wasm-abi.md, gm_layout_params)."""
        out = bytearray(struct.pack("<I", len(self._specs)))
        for s in self._specs:
            nb = s.name.encode()
            out += struct.pack("<I", len(nb)) + nb + struct.pack("<B", s.kind)
            out += struct.pack("<dddd", s.min, s.max, s.default, s.step)
            db = s.doc.encode()
            out += struct.pack("<I", len(db)) + db
        return bytes(out)


def encode_params(values: Sequence[float]) -> bytes:
    return struct.pack("<%dd" % len(values), *[float(v) for v in values])


@dataclass
class Topology:
    """The part of graph-core's Topology the FA2 stage reads."""

    node_count: int
    source: np.ndarray
    target: np.ndarray
    strength: Optional[np.ndarray] = None

    def __post_init__(self):
        self.source = np.ascontiguousarray(self.source, np.uint32)
        self.target = np.ascontiguousarray(self.target, np.uint32)
        if self.strength is not None:
            self.strength = np.ascontiguousarray(self.strength, np.float64)

    @property
    def edge_count(self) -> int:
        return int(len(self.source))


@dataclass
class Geometry:
    dim: int
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))

    @staticmethod
    def points(pos: np.ndarray) -> "Geometry":
        pos = np.asarray(pos, np.float32)
        d = pos.shape[1] if pos.ndim == 2 else 2
        z = pos[:, 2].copy() if d == 3 else np.zeros(0, np.float32)
        return Geometry(d, pos[:, 0].copy(), pos[:, 1].copy(), z)


@dataclass(frozen=True)
class Metadata:
    tier: int
    stage: str
    oracle: str
    complexity: str
    scale_ceiling: int
    degradation: str


@dataclass(frozen=True)
class Capability:
    id: str
    run: Callable[[Topology], Geometry]
    params: ParamsView
    meta: Metadata
    run_with: Callable[[Topology, List[float]], Geometry] = None

    def params_values(self, b: bytes) -> List[float]:
        """registry/params.rs:169-175: empty buffer = defaults, else validate."""
        if len(b) == 0:
            return self.params.defaults()
        return self.params.values(b)

    def run_values(self, topology: Topology, values: List[float]) -> Geometry:
        return self.run_with(topology, values)

    def run_params(self, topology: Topology, b: bytes) -> Geometry:
        """registry/params.rs:156-160: refusals become StageError::Param."""
        try:
            values = self.params_values(b)
        except ParamsError as why:
            if why.kind == "OutOfRange":
                name = self.params.specs()[why.index].name
                raise StageError("Param", name, "out of range, refused and never clamped",
                                 N.GR_PARAM_OUT_OF_RANGE) from None
            code = N.GR_PARAMS_MALFORMED if why.kind == "Malformed" else N.GR_PARAMS_NOT_ACCEPTED
            raise StageError("Param", "params", why.kind, code) from None
        return self.run_values(topology, values)


def _native_specs() -> List[ParamSpec]:
    L = N.lib()
    out = []
    for i in range(L.gr_fa2_param_count()):
        name, doc = C.c_char_p(), C.c_char_p()
        kind = C.c_int()
        mn, mx, df, st = C.c_double(), C.c_double(), C.c_double(), C.c_double()
        N.check(L.gr_fa2_param_spec(i, C.byref(name), C.byref(kind), C.byref(mn), C.byref(mx),
                                    C.byref(df), C.byref(st), C.byref(doc)))
        out.append(ParamSpec(name.value.decode(), kind.value, mn.value, mx.value, df.value, st.value,
                             doc.value.decode()))
    return out


FA2_ID = "layout.forceatlas2.barnes_hut.cuda"

FA2_META = Metadata(
    tier=1,
    stage="layout",
    oracle=("the FP64 CPU restatement of graph-core's forceatlas2 tick (oracle/), itself pinned to "
            "networkx 3.6 forceatlas2_layout; per-tick forces from identical positions within 1e-5 "
            "relative L2 on the same tree and theta"),
    complexity="O(n log n) per tick: Morton sort, linear tree, warp-cooperative walk; O(m) attraction",
    scale_ceiling=50_000_000,
    degradation="past device memory the create call refuses with GR_ALLOC_FAILED",
)

D3_ID = "layout.force.barnes_hut.cuda"

D3_META = Metadata(
    tier=1,
    stage="layout",
    oracle=("the FP64 CPU restatement of graph-core's layout.force.barnes_hut (oracle/, orc_d3_*), itself "
            "reproducing the reference's 65 frozen-layout digests and 8 snapshot hashes bit for bit; the "
            "FP32 GPU tick against it pass by pass, the layout's stress against it at the end"),
    complexity="O(n log n) per tick x 112 ticks: two Morton trees (positions, projected positions), "
               "link as a CSR gather",
    scale_ceiling=50_000_000,
    degradation="past device memory the create call refuses with GR_ALLOC_FAILED",
)

PM_ID = "layout.force.particle_mesh.cuda"

PM_META = Metadata(
    tier=1,
    stage="layout",
    oracle=("the FP64 CPU restatement of graph-core's layout.force.particle_mesh many-body pass (oracle/, "
            "orc_d3_use_mesh), passing the reference's own particle-mesh tests; the FP32 GPU mesh field and "
            "tick against it, the layout's stress at the end"),
    complexity="O(n + P^2 log P) per tick x 112 ticks (P the mesh side, <= 1024): deposit gather, two 2D FFTs, "
               "bilinear read; collide on the tree of projected positions",
    scale_ceiling=50_000_000,
    degradation="past device memory the create call refuses with GR_ALLOC_FAILED",
)

_LAYOUTS: Optional[List[Capability]] = None


def layouts() -> List[Capability]:
    """LAYOUTS (registry.rs:62-64), built on first use from the native schema."""
    global _LAYOUTS
    if _LAYOUTS is None:
        from . import fa2

        specs = _native_specs()
        view = ParamsView(specs, accepted_lengths=(5,))
        from . import d3force

        none = ParamsView([])  # registry/layouts.rs: LayoutParams::NONE
        _LAYOUTS = [Capability(FA2_ID, run=lambda t: fa2.run_values(t, view.defaults()), params=view,
                               meta=FA2_META, run_with=fa2.run_values),
                    Capability(D3_ID, run=lambda t: d3force.run_values(t, []), params=none, meta=D3_META,
                               run_with=d3force.run_values),
                    Capability(PM_ID, run=lambda t: d3force.run_values_mesh(t, []), params=none, meta=PM_META,
                               run_with=d3force.run_values_mesh)]
    return _LAYOUTS


def find(layout_id: str) -> Optional[Capability]:
    for cap in layouts():
        if cap.id == layout_id:
            return cap
    return None
