"""d3-force Barnes-Hut on the GPU, through the C ABI.

``ForceSession`` owns one session handle (``gr_force_session_create`` ..
``gr_force_session_destroy``): the per-tick surface of the reference's live
force session (crates/graph-core/src/layout/force/session.rs; graph-wasm's
gm_force_session_*): ``tick``, ``positions``, ``velocities``, ``alpha``,
``reheat``. ``run_values`` is the registry's ``Capability::run_values`` for
``layout.force.barnes_hut.cuda``: the frozen layout (barnes_hut.rs:134-140,
``BarnesHut::run``: default parameters, 112 ticks from the golden spiral).
"""

from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _native as N
from .registry import Geometry, StageError, Topology

TICKS = 112  # crates/graph-core/src/layout/force/params.rs TICKS


class ForceParams(C.Structure):
    """params.rs ForceParams, field for field (include/graph_cuda.h gr_force_params)."""
    _fields_ = [(k, C.c_double) for k in (
        "charge", "theta", "distance_min", "distance_max", "link_distance", "link_strength_scale",
        "collide_radius", "center_strength", "velocity_decay", "alpha_decay", "alpha_min", "initial_alpha")]

    @classmethod
    def defaults(cls, **kw) -> "ForceParams":
        p = cls()
        N.lib().gr_force_default_params(C.byref(p))
        for k, v in kw.items():
            setattr(p, k, float(v))
        return p


def _ptr(a: Optional[np.ndarray]):
    return None if a is None or a.size == 0 else a.ctypes.data_as(C.c_void_p)


class ForceSession:
    def __init__(self, n: int, src, dst, strength=None, params: Optional[ForceParams] = None, pos0=None, **kw):
        self._L = N.lib()
        self.n = int(n)
        src = np.ascontiguousarray(src, np.uint32)
        dst = np.ascontiguousarray(dst, np.uint32)
        st = None if strength is None else np.ascontiguousarray(strength, np.float64)
        p0 = None if pos0 is None else np.ascontiguousarray(pos0, np.float32).reshape(self.n, 2)
        prm = params if params is not None else ForceParams.defaults(**kw)
        h = C.c_void_p()
        N.check(self._L.gr_force_session_create(C.byref(h), self.n, len(src), _ptr(src), _ptr(dst), _ptr(st),
                                                C.byref(prm), _ptr(p0)))
        self.h = h

    def close(self) -> None:
        if getattr(self, "h", None):
            self._L.gr_force_session_destroy(self.h)
            self.h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def tick(self, ticks: int = 1) -> None:
        N.check(self._L.gr_force_session_tick(self.h, int(ticks)))

    def tick_timed(self, ticks: int = 1) -> float:
        """Runs `ticks` ticks; returns their device time in ms (CUDA events on the
        session's stream)."""
        ms = C.c_float()
        N.check(self._L.gr_force_session_tick_timed(self.h, int(ticks), C.byref(ms)))
        return ms.value

    def positions(self) -> np.ndarray:
        out = np.zeros((self.n, 2), np.float32)
        N.check(self._L.gr_force_session_positions(self.h, _ptr(out)))
        return out

    def velocities(self) -> np.ndarray:
        out = np.zeros((self.n, 2), np.float32)
        N.check(self._L.gr_force_session_velocities(self.h, _ptr(out)))
        return out

    def alpha(self) -> float:
        a, t = C.c_double(), C.c_uint32()
        N.check(self._L.gr_force_session_alpha(self.h, C.byref(a), C.byref(t)))
        return a.value

    def ticks_done(self) -> int:
        a, t = C.c_double(), C.c_uint32()
        N.check(self._L.gr_force_session_alpha(self.h, C.byref(a), C.byref(t)))
        return t.value

    def reheat(self, alpha: float) -> None:
        N.check(self._L.gr_force_session_reheat(self.h, float(alpha)))

    def use_mesh(self) -> None:
        """Many-body on the particle mesh from the next tick on (ForceSession::with_particle_mesh)."""
        N.check(self._L.gr_force_session_use_mesh(self.h))

    def set_state(self, positions=None, velocities=None, alpha: float = 1.0, ticks_done: int = 0) -> None:
        """Carries positions and velocities (n x 2; None keeps the session's), alpha
        and the tick count into the session."""
        p = None if positions is None else np.ascontiguousarray(positions, np.float32).reshape(self.n, 2)
        v = None if velocities is None else np.ascontiguousarray(velocities, np.float32).reshape(self.n, 2)
        N.check(self._L.gr_force_session_set_state(self.h, _ptr(p), _ptr(v), float(alpha), int(ticks_done)))

    def info(self) -> dict:
        k, c = C.c_uint32(), C.c_uint32()
        N.check(self._L.gr_force_session_info(self.h, C.byref(k), C.byref(c)))
        return {"graph_kernels": k.value, "n_cells": c.value}


def run_values(topology: Topology, values) -> Geometry:
    """The frozen layout for the registry row (no parameters): 112 ticks at the
    defaults; a non-finite position is StageError::NonFinite."""
    n = topology.node_count
    out = np.zeros((max(n, 1), 2), np.float32)
    src, dst = topology.source, topology.target
    rc = N.lib().gr_force_run(n, len(src), _ptr(src), _ptr(dst), _ptr(topology.strength), _ptr(out))
    if rc == N.GR_LAYOUT_FAILED:
        raise StageError("NonFinite", "node.x", "non-finite position", rc)
    N.check(rc)
    return Geometry.points(out[:n])


def run_values_mesh(topology: Topology, values) -> Geometry:
    """The frozen particle-mesh layout for the registry row (no parameters):
    ParticleMesh::run, 112 ticks at the defaults with many-body on the mesh."""
    n = topology.node_count
    out = np.zeros((max(n, 1), 2), np.float32)
    src, dst = topology.source, topology.target
    rc = N.lib().gr_force_mesh_run(n, len(src), _ptr(src), _ptr(dst), _ptr(topology.strength), _ptr(out))
    if rc == N.GR_LAYOUT_FAILED:
        raise StageError("NonFinite", "node.x", "non-finite position", rc)
    N.check(rc)
    return Geometry.points(out[:n])


def _main(argv=None) -> None:
    """python -m graph_render_b200.d3force --n N --ticks T: a session on the
    reference's benchmark model, T ticks after 3 warm-up ticks; prints ms per tick."""
    import argparse
    import json
    import time

    from . import synth

    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--ticks", type=int, default=5)
    ap.add_argument("--mesh", action="store_true", help="many-body on the particle mesh")
    a = ap.parse_args(argv)
    src, dst, st = synth.gate(a.n)
    with ForceSession(a.n, src, dst, st) as s:
        if a.mesh:
            s.use_mesh()
        s.tick(3)
        t0 = time.perf_counter()
        s.tick(a.ticks)
        ms = (time.perf_counter() - t0) * 1e3 / max(a.ticks, 1)
        print(json.dumps({"n": a.n, "ticks": a.ticks, "ms_per_tick": ms, **s.info()}))


if __name__ == "__main__":
    _main()
