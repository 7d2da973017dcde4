"""ctypes binding of ``libgraph_cuda.so`` (the C ABI in ``include/graph_cuda.h``).

The library is loaded from this package's directory only. There is no other
implementation of the engine: if the shared object is missing, every call
raises instead of falling back to anything else.
"""

from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgraph_cuda.so")

GR_OK = 0
GR_INVALID_HANDLE = 1
GR_ALLOC_FAILED = 2
GR_UNKNOWN_LAYOUT_ID = 5
GR_LAYOUT_FAILED = 8
GR_INDEX_OUT_OF_RANGE = 12
GR_PARAM_OUT_OF_RANGE = 20
GR_PARAMS_MALFORMED = 21
GR_PARAMS_NOT_ACCEPTED = 22
GR_INVALID_ARGUMENT = 100
GR_CUDA_ERROR = 101
GR_DEVICE_FAULT = 102

KIND_INT, KIND_FLOAT, KIND_BOOL = 0, 1, 2


class Info(C.Structure):
    _fields_ = [
        ("n", C.c_uint32),
        ("dim", C.c_uint32),
        ("m", C.c_uint64),
        ("iter_no", C.c_uint32),
        ("converged", C.c_uint32),
        ("n_cells", C.c_uint32),
        ("n_leaves", C.c_uint32),
        ("swing", C.c_double),
        ("traction", C.c_double),
        ("speed", C.c_double),
        ("speed_efficiency", C.c_double),
        ("moved", C.c_double),
        ("far_count", C.c_uint64),
        ("pair_count", C.c_uint64),
        ("device_error", C.c_uint32),
        ("graph_kernels", C.c_uint32),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Controller(C.Structure):
    _fields_ = [("swing", C.c_double), ("traction", C.c_double), ("speed", C.c_double),
                ("speed_efficiency", C.c_double), ("iter_no", C.c_uint32), ("converged", C.c_uint32)]


# Every symbol the header declares, with its ctypes signature.
P = C.c_void_p
u8p, u32p, f32p, f64p = C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p
SIGNATURES = {
    "gr_abi_version": ([], C.c_uint32),
    "gr_last_error": ([], C.c_int),
    "gr_last_error_message": ([], C.c_char_p),
    "gr_last_error_index": ([], C.c_int),
    "gr_layout_count": ([], C.c_uint32),
    "gr_layout_id": ([C.c_uint32], C.c_char_p),
    "gr_fa2_param_count": ([], C.c_uint32),
    "gr_fa2_param_spec": ([C.c_uint32, C.POINTER(C.c_char_p), C.POINTER(C.c_int), C.POINTER(C.c_double),
                           C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double),
                           C.POINTER(C.c_char_p)], C.c_int),
    "gr_fa2_params_values": ([u8p, C.c_size_t, f64p], C.c_int),
    "gr_fa2_create": ([C.POINTER(P), C.c_uint32, C.c_uint64, u32p, u32p, f64p, u8p, C.c_size_t, f32p], C.c_int),
    "gr_fa2_destroy": ([P], None),
    "gr_fa2_tick": ([P, C.c_uint32, C.POINTER(C.c_uint32)], C.c_int),
    "gr_fa2_run": ([P, C.POINTER(C.c_uint32)], C.c_int),
    "gr_fa2_tick_record": ([P, C.c_uint32, P, C.POINTER(C.c_uint32)], C.c_int),
    "gr_fa2_tick_timed": ([P, C.c_uint32, C.c_size_t, P, C.POINTER(C.c_uint32)], C.c_int),
    "gr_fa2_positions": ([P, f32p], C.c_int),
    "gr_fa2_set_positions": ([P, f32p], C.c_int),
    "gr_fa2_positions_device": ([P, C.POINTER(P)], C.c_int),
    "gr_fa2_forces": ([P, f32p], C.c_int),
    "gr_fa2_get_info": ([P, C.POINTER(Info)], C.c_int),
    "gr_fa2_set_stream": ([P, P], C.c_int),
    "gr_run": ([C.c_char_p, C.c_uint32, C.c_uint64, u32p, u32p, f64p, u8p, C.c_size_t, f32p], C.c_int),
    "gr_fa2_forces_static": ([C.c_uint32, P, P, P, P, u8p, C.c_size_t, C.c_uint32, P, P], C.c_int),
    "gr_fa2_forces_static_status": ([C.POINTER(C.c_uint32)], C.c_int),
    "gr_bfs_hops": ([C.c_uint32, C.c_uint64, P, P, C.c_uint32, P, P], C.c_int),
    "gr_measure_fp32_rate": ([C.c_uint32, C.POINTER(C.c_double)], C.c_int),
    "gr_force_default_params": ([P], None),
    "gr_force_session_create": ([P, C.c_uint32, C.c_uint64, P, P, P, P, P], C.c_int),
    "gr_force_session_destroy": ([P], None),
    "gr_force_session_tick": ([P, C.c_uint32], C.c_int),
    "gr_force_session_tick_timed": ([P, C.c_uint32, C.POINTER(C.c_float)], C.c_int),
    "gr_force_session_positions": ([P, P], C.c_int),
    "gr_force_session_velocities": ([P, P], C.c_int),
    "gr_force_session_alpha": ([P, C.POINTER(C.c_double), C.POINTER(C.c_uint32)], C.c_int),
    "gr_force_session_reheat": ([P, C.c_double], C.c_int),
    "gr_force_session_info": ([P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)], C.c_int),
    "gr_force_session_set_state": ([P, P, P, C.c_double, C.c_uint32], C.c_int),
    "gr_force_session_use_mesh": ([P], C.c_int),
    "gr_force_mesh_run": ([C.c_uint32, C.c_uint64, P, P, P, P], C.c_int),
    "gr_force_run": ([C.c_uint32, C.c_uint64, P, P, P, P], C.c_int),
    "gr_stress": ([C.c_uint32, C.c_uint64, P, P, P, P, C.c_uint32, C.POINTER(C.c_double)], C.c_int),
    "gr_fa2_batch_create": ([C.POINTER(P), C.c_uint32, P, P, P, P, P, P, C.c_uint32, P], C.c_int),
    "gr_fa2_batch_destroy": ([P], None),
    "gr_fa2_batch_set_threads": ([P, C.c_int], C.c_int),
    "gr_fa2_batch_run": ([P, C.c_uint32, C.POINTER(C.c_float)], C.c_int),
    "gr_fa2_batch_tune": ([P, C.c_uint32, C.POINTER(C.c_int), P], C.c_int),
    "gr_fa2_batch_positions": ([P, P], C.c_int),
    "gr_fa2_batch_stats": ([P, P, P, P], C.c_int),
    "gr_fa2_set_walk_schedule": ([P, C.c_int], C.c_int),
    "gr_fa2_set_interaction_counting": ([P, C.c_int], C.c_int),
    "gr_fa2_launch_mode": ([P, C.POINTER(C.c_int)], C.c_int),
    "gr_fa2_tune": ([P, C.c_uint32, C.POINTER(C.c_int), P], C.c_int),
    "gr_fa2_set_wait_limit": ([P, C.c_uint32], C.c_int),
    "gr_fa2_inject_stalled_wait": ([P, C.c_int], C.c_int),
    "gr_fa2_get_controller": ([P, P], C.c_int),
    "gr_fa2_set_controller": ([P, P], C.c_int),
    "gr_fa2_adjoint_forward": ([P, C.c_uint32, C.c_uint32], C.c_int),
    "gr_fa2_adjoint_backward": ([P, P, P, P], C.c_int),
}

_lib = None


class NativeMissing(RuntimeError):
    pass


def lib():
    """The loaded engine library; raises NativeMissing when it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise NativeMissing(
            f"{LIB_PATH} is missing: build it with `python -m graph_render_b200.build` "
            "(the engine has no non-CUDA path)")
    L = C.CDLL(LIB_PATH)
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


class EngineError(RuntimeError):
    """A refused or failed call: `code` is the graph-wasm-numbered status."""

    def __init__(self, code: int, message: str, index: int = -1):
        super().__init__(f"[{code}] {message}")
        self.code = code
        self.message = message
        self.index = index


def check(rc: int) -> None:
    if rc != GR_OK:
        L = lib()
        msg = L.gr_last_error_message()
        raise EngineError(rc, msg.decode() if msg else "", L.gr_last_error_index())
