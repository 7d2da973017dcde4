"""ForceAtlas2 / Barnes-Hut on the GPU, through the C ABI.

``Fa2`` owns one engine handle (``gr_fa2_create`` .. ``gr_fa2_destroy``) and
exposes the per-tick surface the reference lacks (``tick``, ``positions``,
``forces``, ``tick_record``); ``run_values`` is the registry's
``Capability::run_values`` for ``layout.forceatlas2.barnes_hut.cuda``
(crates/graph-core/src/layout/forceatlas2.rs:51-61 ``ForceAtlas2BarnesHut::run``
then ``settle``).
"""

from __future__ import annotations

import ctypes as C
from typing import Dict, Optional, Sequence, Union

import numpy as np

from . import _native as N
from .registry import Geometry, StageError, Topology, encode_params

PARAM_NAMES = ("max_iter", "jitter_tolerance", "scaling_ratio", "gravity", "seed", "dim", "theta",
               "lin_log", "strong_gravity", "dissuade_hubs", "edge_weight_influence")
DEFAULTS = dict(max_iter=100, jitter_tolerance=1.0, scaling_ratio=2.0, gravity=1.0, seed=0, dim=2,
                theta=0.8, lin_log=0, strong_gravity=0, dissuade_hubs=0, edge_weight_influence=0.0)

# walk schedules (include/graph_cuda.h GR_WALK_SCHEDULES): warp-union, per-lane, two nodes per lane over
# the union of their walks, two independent walks per lane
WALK_SCHEDULES = 4
WALK_SCHEDULE_NAMES = ("warp-union", "per-lane", "pair-per-lane", "two-per-lane")


def params_bytes(params: Union[None, bytes, Dict[str, float], Sequence[float]] = None, **kw) -> bytes:
    """A parameter buffer from a dict / keywords (unnamed ones at their defaults)."""
    if isinstance(params, (bytes, bytearray)):
        return bytes(params)
    vals = dict(DEFAULTS)
    if isinstance(params, dict):
        vals.update(params)
    elif params is not None:
        return encode_params(list(params))
    vals.update(kw)
    unknown = set(vals) - set(PARAM_NAMES)
    if unknown:
        raise KeyError(f"unknown parameters {sorted(unknown)}")
    return encode_params([vals[k] for k in PARAM_NAMES])


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Fa2:
    """One graph's layout state on the GPU."""

    def __init__(self, n: int, src, dst, weight=None, params=None, pos0=None, **kw):
        L = N.lib()
        self._L = L
        self.n = int(n)
        src = np.ascontiguousarray(src, np.uint32)
        dst = np.ascontiguousarray(dst, np.uint32)
        if len(src) != len(dst):
            raise ValueError("src and dst differ in length")
        w = None if weight is None else np.ascontiguousarray(weight, np.float64)
        pb = params_bytes(params, **kw)
        self.params_buffer = pb
        vals = (C.c_double * 11)()
        N.check(L.gr_fa2_params_values(C.c_char_p(pb) if pb else None, len(pb), vals))
        self.values = list(vals)
        self.dim = int(self.values[5])
        p0 = None
        if pos0 is not None:
            p0 = np.ascontiguousarray(pos0, np.float32).reshape(self.n, self.dim)
        h = C.c_void_p()
        self.m_raw = int(len(src))
        N.check(L.gr_fa2_create(C.byref(h), self.n, len(src), _ptr(src), _ptr(dst), _ptr(w),
                                C.c_char_p(pb) if pb else None, len(pb), _ptr(p0)))
        self.h = h

    def close(self) -> None:
        if getattr(self, "h", None):
            self._L.gr_fa2_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def tick(self, ticks: int = 1) -> int:
        done = C.c_uint32()
        N.check(self._L.gr_fa2_tick(self.h, int(ticks), C.byref(done)))
        return done.value

    def run(self) -> int:
        done = C.c_uint32()
        N.check(self._L.gr_fa2_run(self.h, C.byref(done)))
        return done.value

    def tick_record(self, ticks: int, dev_out_ptr: int) -> int:
        """Per-tick positions into a device buffer of ticks * n * dim float32."""
        done = C.c_uint32()
        N.check(self._L.gr_fa2_tick_record(self.h, int(ticks), C.c_void_p(dev_out_ptr), C.byref(done)))
        return done.value

    def tick_timed(self, ticks: int, l2_flush_bytes: int = 0) -> np.ndarray:
        """Per-tick device times (ms): columns tree, walk, finish, whole tick."""
        out = np.zeros((int(ticks), 4), np.float32)
        done = C.c_uint32()
        N.check(self._L.gr_fa2_tick_timed(self.h, int(ticks), int(l2_flush_bytes), _ptr(out), C.byref(done)))
        return out[:done.value]

    def adjoint_forward(self, ticks: int, every: int = 20) -> None:
        """Runs `ticks` ticks recording positions and controller every `every`
        ticks, for adjoint_backward."""
        N.check(self._L.gr_fa2_adjoint_forward(self.h, int(ticks), int(every)))

    def adjoint_backward(self, dL_dpT) -> tuple:
        """(dL/d start positions (n x dim), dL/d raw edge weight (m)) for
        dL_dpT = dL/d final positions of the recorded run."""
        g = np.ascontiguousarray(dL_dpT, np.float32).reshape(self.n, self.dim)
        dp0 = np.zeros((self.n, self.dim), np.float64)
        dw = np.zeros(max(self.m_raw, 1), np.float64)
        N.check(self._L.gr_fa2_adjoint_backward(self.h, _ptr(g), _ptr(dp0), _ptr(dw)))
        return dp0, dw[:self.m_raw]

    def positions(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        """The positions, row-major n x dim FP32. `out` (optional) is written in
        place: a C-contiguous float32 array of that shape, e.g. in pinned memory,
        which the device copies into directly."""
        if out is None:
            out = np.empty((self.n, self.dim), np.float32)
        elif out.dtype != np.float32 or out.shape != (self.n, self.dim) or not out.flags.c_contiguous:
            raise ValueError(f"out must be a C-contiguous float32 array of shape ({self.n}, {self.dim})")
        N.check(self._L.gr_fa2_positions(self.h, _ptr(out)))
        return out

    def set_positions(self, pos) -> None:
        pos = np.ascontiguousarray(pos, np.float32).reshape(self.n, self.dim)
        N.check(self._L.gr_fa2_set_positions(self.h, _ptr(pos)))

    def device_nodes(self) -> int:
        p = C.c_void_p()
        N.check(self._L.gr_fa2_positions_device(self.h, C.byref(p)))
        return int(p.value or 0)

    def forces(self) -> np.ndarray:
        out = np.zeros((self.n, self.dim), np.float32)
        N.check(self._L.gr_fa2_forces(self.h, _ptr(out)))
        return out

    def info(self) -> dict:
        inf = N.Info()
        N.check(self._L.gr_fa2_get_info(self.h, C.byref(inf)))
        return inf.as_dict()

    def set_walk_schedule(self, schedule: int) -> None:
        N.check(self._L.gr_fa2_set_walk_schedule(self.h, int(schedule)))

    def programmatic_launches(self) -> bool:
        """True when the tick's kernels are programmatic dependent launches."""
        v = C.c_int()
        N.check(self._L.gr_fa2_launch_mode(self.h, C.byref(v)))
        return bool(v.value)

    def set_interaction_counting(self, on: bool) -> None:
        """On (the default): the walk counts far / pair interactions into info();
        off: it keeps no counts (same forces, fewer instructions per cell)."""
        N.check(self._L.gr_fa2_set_interaction_counting(self.h, 1 if on else 0))

    def set_wait_limit(self, spins: int) -> None:
        """Sleeps (~32 ns each) a bounded wait of the tick's sort takes before it
        gives up (0: the default)."""
        N.check(self._L.gr_fa2_set_wait_limit(self.h, int(spins)))

    def inject_stalled_wait(self, on: bool = True) -> None:
        """Fault injection: a wait of every sort pass that nothing will end, so it
        runs out and the next tick fails with GR_DEVICE_FAULT (ERR_WAIT)."""
        N.check(self._L.gr_fa2_inject_stalled_wait(self.h, 1 if on else 0))

    def tune(self, sample_ticks: int = 3):
        """Autotunes the walk schedule; returns (chosen, {schedule: mean walk ms})."""
        chosen = C.c_int()
        ms = np.zeros(WALK_SCHEDULES, np.float32)
        N.check(self._L.gr_fa2_tune(self.h, int(sample_ticks), C.byref(chosen), _ptr(ms)))
        return chosen.value, {i: float(ms[i]) for i in range(WALK_SCHEDULES)}

    def controller(self) -> dict:
        c = N.Controller()
        N.check(self._L.gr_fa2_get_controller(self.h, C.byref(c)))
        return {k: getattr(c, k) for k, _ in c._fields_}

    def set_controller(self, swing, traction, speed, speed_efficiency, iter_no, converged=0) -> None:
        c = N.Controller(swing, traction, speed, speed_efficiency, iter_no, converged)
        N.check(self._L.gr_fa2_set_controller(self.h, C.byref(c)))

    def set_stream(self, stream_ptr: int) -> None:
        N.check(self._L.gr_fa2_set_stream(self.h, C.c_void_p(stream_ptr)))


def run_values(topology: Topology, values) -> Geometry:
    """Capability::run_values for layout.forceatlas2.barnes_hut.cuda: create,
    run max_iter ticks, settle (NonFinite refused), release."""
    pb = encode_params(values)
    try:
        with Fa2(topology.node_count, topology.source, topology.target, topology.strength, params=pb) as eng:
            eng.run()
            pos = eng.positions()
    except N.EngineError as e:
        if e.code == N.GR_LAYOUT_FAILED:
            raise StageError("NonFinite", "node.x", code=e.code) from None
        raise
    return Geometry.points(pos)


def layout(topology: Topology, params=None, **kw) -> Geometry:
    """One-shot run of the registered FA2 layout with a parameter buffer / dict."""
    from .registry import find, FA2_ID

    return find(FA2_ID).run_params(topology, params_bytes(params, **kw))
