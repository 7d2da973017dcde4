"""ORACLE — test infrastructure only.

ctypes face of ``liboracle_fa2.so``: the FP64 CPU restatement of graph-core's
ForceAtlas2 tick (``crates/graph-core/src/layout/forceatlas2/state.rs``,
``state/schedule.rs``, ``state/barnes_hut.rs``, ``layout/force/quadtree*.rs``).
Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module; the product package never does.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle_fa2.so")
LIB_PATH = _LIB_PATH  # also carries the workload generators (csrc/synth.c), see Makefile
_lib = None


def build() -> str:
    """Compile the oracle library in place (``make -C oracle``)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


class Params(C.Structure):
    """``orc_params``: Fa2Params (state.rs:20-54) plus the networkx options."""

    _fields_ = [
        ("max_iter", C.c_int64),
        ("jitter_tolerance", C.c_double),
        ("scaling_ratio", C.c_double),
        ("gravity", C.c_double),
        ("seed", C.c_int64),
        ("dim", C.c_int64),
        ("theta", C.c_double),
        ("lin_log", C.c_int64),
        ("strong_gravity", C.c_int64),
        ("dissuade_hubs", C.c_int64),
        ("edge_weight_influence", C.c_double),
        ("depth_cap", C.c_int64),
        ("threads", C.c_int64),
    ]


def params(**kw) -> Params:
    """Reference defaults (state.rs:34-45): dense repulsion unless theta >= 0."""
    base = dict(max_iter=100, jitter_tolerance=1.0, scaling_ratio=2.0, gravity=1.0,
                seed=0, dim=2, theta=-1.0, lin_log=0, strong_gravity=0,
                dissuade_hubs=0, edge_weight_influence=0.0, depth_cap=0, threads=1)
    base.update(kw)
    return Params(**{k: base[k] for k, _ in Params._fields_})


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    L = C.CDLL(_LIB_PATH)
    P = C.c_void_p
    u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
    f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
    f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    L.orc_initial_positions.argtypes = [C.c_uint32, C.c_uint32, C.c_int, f64p]
    L.orc_jiggle.argtypes = [C.c_uint32] * 5
    L.orc_jiggle.restype = C.c_double
    L.orc_stress.argtypes = [C.c_uint32, C.c_int64, u32p, u32p, f32p, f32p, C.c_uint32]
    L.orc_stress.restype = C.c_double
    L.orc_bfs.argtypes = [C.c_uint32, C.c_int64, u32p, u32p, C.c_uint32, u32p, u32p]
    L.orc_d3_default_params.argtypes = [C.POINTER(D3Params)]
    L.orc_d3_new.argtypes = [C.c_uint32, C.c_uint32, u32p, u32p, f64p, C.POINTER(D3Params), P]
    L.orc_d3_new.restype = P
    L.orc_d3_free.argtypes = [P]
    L.orc_d3_tick.argtypes = [P, C.c_uint32]
    L.orc_d3_positions.argtypes = [P, f64p]
    L.orc_d3_velocities.argtypes = [P, f64p]
    L.orc_d3_alpha.argtypes = [P]
    L.orc_d3_alpha.restype = C.c_double
    L.orc_d3_set_state.argtypes = [P, f64p, f64p, C.c_double, C.c_uint32]
    L.orc_d3_use_mesh.argtypes = [P]
    L.orc_pm_field.argtypes = [P, f64p]
    L.orc_pm_field.restype = C.c_int
    L.orc_gate_edges.argtypes = [C.c_uint32, u32p, u32p, f64p, C.c_int64]
    L.orc_gate_edges.restype = C.c_int64
    L.orc_simple_graph.argtypes = [C.c_uint32, C.c_int64, u32p, u32p, P, u32p, u32p, f64p]
    L.orc_simple_graph.restype = C.c_int64
    L.orc_fa2_new.argtypes = [C.c_uint32, C.c_int64, u32p, u32p, P, C.POINTER(Params), P]
    L.orc_fa2_new.restype = P
    L.orc_fa2_free.argtypes = [P]
    L.orc_fa2_accumulate.argtypes = [P, C.c_int]
    L.orc_fa2_iterate.argtypes = [P]
    L.orc_fa2_iterate.restype = C.c_double
    L.orc_fa2_run.argtypes = [P, C.c_uint32]
    L.orc_fa2_run.restype = C.c_uint32
    for name in ("orc_fa2_get_positions", "orc_fa2_set_positions", "orc_fa2_get_forces",
                 "orc_fa2_get_mass", "orc_fa2_get_scalars", "orc_fa2_set_scalars",
                 "orc_fa2_mean"):
        getattr(L, name).argtypes = [P, f64p]
    L.orc_fa2_tree_cells.argtypes = [P]
    L.orc_fa2_tree_cells.restype = C.c_uint32
    L.orc_fa2_tree_dump.argtypes = [P, P, P, P, P, P, P, P]
    L.orc_fa2_repel_delta.argtypes = [P, C.c_uint32, C.c_uint32, f64p]
    _lib = L
    return L


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def initial_positions(n: int, seed: int, dim: int) -> np.ndarray:
    """state.rs:272-283: Mulberry32(seed), dim draws per node."""
    out = np.zeros((n, dim), np.float64)
    lib().orc_initial_positions(n, seed, dim, out.reshape(-1))
    return out


def jiggle(seed, tick, pass_, i, j) -> float:
    return lib().orc_jiggle(seed, tick, pass_, i, j)


def gate_edges(count: int):
    """synthetic.rs:92-170: the gate model's raw edges (source, target, strength)."""
    cap = 4 * count + 16
    src = np.zeros(cap, np.uint32)
    dst = np.zeros(cap, np.uint32)
    st = np.zeros(cap, np.float64)
    m = lib().orc_gate_edges(count, src, dst, st, cap)
    assert m <= cap
    return src[:m].copy(), dst[:m].copy(), st[:m].copy()


def _nonempty_u32(a):
    a = np.ascontiguousarray(a, np.uint32)
    return a if len(a) else np.zeros(1, np.uint32)


class D3Params(C.Structure):
    """crates/graph-core/src/layout/force/params.rs ForceParams (defaults at 60-75)."""
    _fields_ = [(k, C.c_double) for k in (
        "charge", "theta", "distance_min", "distance_max", "link_distance", "link_strength_scale",
        "collide_radius", "center_strength", "velocity_decay", "alpha_decay", "alpha_min", "initial_alpha")]


D3_TICKS = 112  # params.rs TICKS: the least k with 0.94^k < 0.001


def d3_params(**kw) -> D3Params:
    p = D3Params()
    lib().orc_d3_default_params(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, float(v))
    return p


class D3:
    """The frozen d3-force Barnes-Hut layout (barnes_hut.rs) over a simple graph
    (lo < hi, first-wins strength, simple_graph's edge order)."""

    def __init__(self, n, lo, hi, strength, pos0=None, **kw):
        self.n = int(n)
        self._lo = _nonempty_u32(lo)
        self._hi = _nonempty_u32(hi)
        st = np.ascontiguousarray(strength, np.float64)
        self._st = st if len(st) else np.zeros(1)
        self.p = d3_params(**kw)
        self._pos0 = None if pos0 is None else np.ascontiguousarray(pos0, np.float64).reshape(-1)
        self.h = lib().orc_d3_new(self.n, len(lo), self._lo, self._hi, self._st, C.byref(self.p), _ptr(self._pos0))

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_d3_free(self.h)
            self.h = None

    def tick(self, ticks: int = 1) -> None:
        lib().orc_d3_tick(self.h, ticks)

    def positions(self) -> np.ndarray:
        out = np.zeros(2 * max(self.n, 1))
        lib().orc_d3_positions(self.h, out)
        return out[:2 * self.n].reshape(self.n, 2)

    def velocities(self) -> np.ndarray:
        out = np.zeros(2 * max(self.n, 1))
        lib().orc_d3_velocities(self.h, out)
        return out[:2 * self.n].reshape(self.n, 2)

    def alpha(self) -> float:
        return lib().orc_d3_alpha(self.h)

    def use_mesh(self) -> None:
        """Many-body on the particle mesh (particle_mesh.rs) from here on."""
        lib().orc_d3_use_mesh(self.h)

    def mesh_field(self) -> np.ndarray:
        """The mesh's field (charge * alpha left out) at every node, n x 2."""
        out = np.zeros(2 * max(self.n, 1))
        lib().orc_pm_field(self.h, out)
        return out[:2 * self.n].reshape(self.n, 2)

    def set_state(self, pos, vel, alpha: float, tick_no: int) -> None:
        lib().orc_d3_set_state(self.h, np.ascontiguousarray(pos, np.float64).reshape(-1),
                               np.ascontiguousarray(vel, np.float64).reshape(-1), float(alpha), int(tick_no))


def stress(x, y, src, dst, sources: int = 16) -> float:
    """graph-cli/src/bench.rs:255-295: Kruskal stress-1 against hop distance from
    every max(n / sources, 1)-th node, in the reference's order."""
    x = np.ascontiguousarray(x, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    m = len(src)
    return lib().orc_stress(len(x), m, _nonempty_u32(src), _nonempty_u32(dst), x if len(x) else np.zeros(1, np.float32),
                            y if len(y) else np.zeros(1, np.float32), sources)


def bfs_hops(n, src, dst, sources) -> np.ndarray:
    """Hop counts (k x n uint32, UINT32_MAX when unreachable) by one FIFO BFS per source."""
    sources = np.ascontiguousarray(sources, np.uint32)
    out = np.zeros((len(sources), max(n, 1)), np.uint32)
    lib().orc_bfs(n, len(src), _nonempty_u32(src), _nonempty_u32(dst), len(sources), _nonempty_u32(sources),
                  out.reshape(-1))
    return out[:, :n]


def simple_graph(n, src, dst, w=None):
    """layout/force/mod.rs:101-120: (lo, hi, w) of the first raw edge per pair."""
    src = np.ascontiguousarray(src, np.uint32)
    dst = np.ascontiguousarray(dst, np.uint32)
    m = len(src)
    w64 = None if w is None else np.ascontiguousarray(w, np.float64)
    lo = np.zeros(max(m, 1), np.uint32)
    hi = np.zeros(max(m, 1), np.uint32)
    wo = np.zeros(max(m, 1), np.float64)
    k = lib().orc_simple_graph(n, m, src, dst, _ptr(w64), lo, hi, wo)
    return lo[:k].copy(), hi[:k].copy(), wo[:k].copy()


class State:
    """One Fa2State (state.rs:83-102) over simple edges."""

    def __init__(self, n, lo, hi, w=None, pos0=None, **kw):
        self.p = params(**kw)
        self.n = int(n)
        self.dim = int(self.p.dim)
        self._lo = np.ascontiguousarray(lo, np.uint32)
        self._hi = np.ascontiguousarray(hi, np.uint32)
        if len(self._lo) == 0:
            self._lo = np.zeros(1, np.uint32)
            self._hi = np.zeros(1, np.uint32)
            m = 0
        else:
            m = len(lo)
        self._w = None if w is None else np.ascontiguousarray(w, np.float64)
        self._pos0 = None if pos0 is None else np.ascontiguousarray(pos0, np.float64).reshape(-1)
        self.h = lib().orc_fa2_new(self.n, m, self._lo, self._hi, _ptr(self._w),
                                   C.byref(self.p), _ptr(self._pos0))

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_fa2_free(self.h)
            self.h = None

    def iterate(self) -> float:
        return lib().orc_fa2_iterate(self.h)

    def run(self, ticks: int) -> int:
        return lib().orc_fa2_run(self.h, ticks)

    def accumulate(self, terms: int = 7) -> np.ndarray:
        lib().orc_fa2_accumulate(self.h, terms)
        return self.forces()

    def positions(self) -> np.ndarray:
        out = np.zeros((self.n, self.dim), np.float64)
        lib().orc_fa2_get_positions(self.h, out.reshape(-1))
        return out

    def set_positions(self, pos) -> None:
        pos = np.ascontiguousarray(pos, np.float64).reshape(-1)
        lib().orc_fa2_set_positions(self.h, pos)

    def forces(self) -> np.ndarray:
        out = np.zeros((self.n, self.dim), np.float64)
        lib().orc_fa2_get_forces(self.h, out.reshape(-1))
        return out

    def mass(self) -> np.ndarray:
        out = np.zeros(self.n, np.float64)
        lib().orc_fa2_get_mass(self.h, out)
        return out

    def mean(self) -> np.ndarray:
        out = np.zeros(self.dim, np.float64)
        lib().orc_fa2_mean(self.h, out)
        return out

    def scalars(self) -> dict:
        out = np.zeros(7, np.float64)
        lib().orc_fa2_get_scalars(self.h, out)
        keys = ("swing", "traction", "speed", "speed_efficiency", "iter_no", "far", "pair")
        return dict(zip(keys, out.tolist()))

    def set_scalars(self, swing, traction, speed, speed_efficiency, iter_no) -> None:
        lib().orc_fa2_set_scalars(self.h, np.array(
            [swing, traction, speed, speed_efficiency, iter_no], np.float64))

    def repel_delta(self, i, j) -> np.ndarray:
        out = np.zeros(self.dim, np.float64)
        lib().orc_fa2_repel_delta(self.h, i, j, out)
        return out

    def tree(self) -> dict:
        k = lib().orc_fa2_tree_cells(self.h)
        width = np.zeros(max(k, 1), np.float64)
        skip = np.zeros(max(k, 1), np.uint32)
        start = np.zeros(max(k, 1), np.uint32)
        end = np.zeros(max(k, 1), np.uint32)
        mass = np.zeros(max(k, 1), np.float64)
        com = np.zeros(max(k, 1) * self.dim, np.float64)
        order = np.zeros(max(self.n, 1), np.uint32)
        lib().orc_fa2_tree_dump(self.h, _ptr(width), _ptr(skip), _ptr(start), _ptr(end),
                                _ptr(mass), _ptr(com), _ptr(order))
        return dict(width=width[:k], skip=skip[:k], start=start[:k], end=end[:k],
                    mass=mass[:k], com=com[:k * self.dim].reshape(-1, self.dim),
                    order=order[:self.n])


def _adjoint_lib():
    L = lib()
    if not getattr(L, "_adj", False):
        f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
        L.orc_fa2_adjoint.argtypes = [C.c_void_p, C.c_uint32, f64p, f64p, f64p]
        L.orc_fa2_get_coef.argtypes = [C.c_void_p, f64p]
        L.orc_fa2_set_coef.argtypes = [C.c_void_p, f64p]
        L._adj = True
    return L


def adjoint(state: "State", ticks: int, lam_T) -> tuple:
    """VJP of `ticks` ticks from the state's current positions: (dL/dp0, dL/dc per
    simple edge) for lam_T = dL/dp_T. The state ends at the final positions."""
    L = _adjoint_lib()
    lam_T = np.ascontiguousarray(lam_T, np.float64).reshape(-1)
    lam0 = np.zeros(state.n * state.dim, np.float64)
    gc = np.zeros(max(len(state._lo), 1), np.float64)
    L.orc_fa2_adjoint(state.h, ticks, lam_T, lam0, gc)
    return lam0.reshape(state.n, state.dim), gc[:len(state._lo)]


def coef(state: "State") -> np.ndarray:
    L = _adjoint_lib()
    out = np.zeros(max(len(state._lo), 1), np.float64)
    L.orc_fa2_get_coef(state.h, out)
    return out[:len(state._lo)]


def set_coef(state: "State", c) -> None:
    L = _adjoint_lib()
    c = np.ascontiguousarray(c, np.float64)
    if len(c) == 0:
        c = np.zeros(1)
    L.orc_fa2_set_coef(state.h, c)
