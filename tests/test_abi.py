"""The C ABI and the registry mirror, on the CPU (no compute call needs a GPU here).

- the library loads and exports every function include/graph_cuda.h declares;
- the parameter schema and its refusal rules follow graph-contract's ParamsView
  (crates/graph-contract/src/params.rs:147-170) and graph-core's FA2 schema
  (crates/graph-core/src/registry/tunable.rs:229-240);
- the Python registry mirror gives the same answers as the C validator.
"""

import ctypes as C
import math
import os
import re
import struct

import numpy as np
import pytest
from hypothesis import given, settings, strategies as st

from graph_render_b200 import FA2_ID, ParamsError, StageError, Topology, _native as N, find, layouts
from graph_render_b200.registry import ParamsView, encode_params

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "graph_cuda.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gr_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert "gr_fa2_create" in names and "gr_run" in names and "gr_fa2_forces_static" in names
    lib = C.CDLL(N.LIB_PATH)
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(N.SIGNATURES), set(names) ^ set(N.SIGNATURES)


def test_static_library_is_built_beside_the_shared_one():
    assert os.path.exists(os.path.join(os.path.dirname(N.LIB_PATH), "libgraph_cuda.a"))


def test_abi_version_and_registry_face():
    L = N.lib()
    assert L.gr_abi_version() == 1
    assert L.gr_layout_count() == 3
    assert [L.gr_layout_id(i).decode() for i in range(3)] == [
        "layout.forceatlas2.barnes_hut.cuda", "layout.force.barnes_hut.cuda", "layout.force.particle_mesh.cuda"]
    assert L.gr_layout_id(0) == FA2_ID.encode()
    assert L.gr_layout_id(3) is None
    assert L.gr_last_error() == N.GR_INDEX_OUT_OF_RANGE
    assert [c.id for c in layouts()] == [FA2_ID, "layout.force.barnes_hut.cuda", "layout.force.particle_mesh.cuda"]
    assert find("layout.force.barnes_hut.cuda").params.is_empty()


def test_schema_starts_with_the_reference_fa2_schema():
    specs = find(FA2_ID).params.specs()
    ref = [("max_iter", 0, 1.0, 10_000.0, 100.0), ("jitter_tolerance", 1, 0.0, 1e6, 1.0),
           ("scaling_ratio", 1, 0.0, 1e6, 2.0), ("gravity", 1, 0.0, 1e6, 1.0),
           ("seed", 0, 0.0, 4_294_967_295.0, 0.0)]
    for s, (name, kind, mn, mx, df) in zip(specs, ref):
        assert (s.name, s.kind, s.min, s.max, s.default) == (name, kind, mn, mx, df)
    assert [s.name for s in specs[5:]] == ["dim", "theta", "lin_log", "strong_gravity", "dissuade_hubs",
                                           "edge_weight_influence"]
    assert specs[6].default == 0.8  # barnes_hut.rs:24 THETA2 = 0.8^2


def c_values(b: bytes):
    out = (C.c_double * 11)()
    rc = N.lib().gr_fa2_params_values(C.c_char_p(b) if b else None, len(b), out)
    return rc, N.lib().gr_last_error_index(), list(out)


def test_refusals_follow_params_view():
    view = find(FA2_ID).params
    d = view.defaults()
    assert c_values(b"") == (0, -1, d)
    assert c_values(encode_params(d[:5]))[0] == 0
    assert c_values(encode_params(d))[0] == 0
    for bad_len in (8, 16, 48, 8 * 12, 7):
        assert c_values(b"\0" * bad_len)[0] == N.GR_PARAMS_MALFORMED
    cases = [(0, 0.0), (0, 1.5), (0, 10_001.0), (1, -0.1), (1, math.nan), (2, math.inf), (4, -1.0),
             (4, 2.0 ** 32), (5, 4.0), (6, -1e-9), (7, 0.5), (8, 2.0), (10, 11.0)]
    for idx, v in cases:
        vals = list(d)
        vals[idx] = v
        rc, where, _ = c_values(encode_params(vals))
        assert (rc, where) == (N.GR_PARAM_OUT_OF_RANGE, idx), (idx, v)
        with pytest.raises(ParamsError) as e:
            view.validate(encode_params(vals))
        assert e.value.index == idx


@settings(max_examples=300, deadline=None)
@given(st.lists(st.floats(allow_nan=True, allow_infinity=True, width=64), min_size=0, max_size=12))
def test_python_mirror_agrees_with_the_c_validator(vals):
    b = encode_params(vals) if vals else b""
    rc, where, cv = c_values(b)
    view = find(FA2_ID).params
    try:
        pv = view.values(b) if b else view.defaults()
        assert rc == 0 and pv == cv
    except ParamsError as e:
        if e.kind == "Malformed":
            assert rc == N.GR_PARAMS_MALFORMED
        else:
            assert (rc, where) == (N.GR_PARAM_OUT_OF_RANGE, e.index)


def test_run_params_refuses_before_any_device_work():
    cap = find(FA2_ID)
    t = Topology(3, np.array([0, 1], np.uint32), np.array([1, 2], np.uint32))
    with pytest.raises(StageError) as e:
        cap.run_params(t, encode_params([0.5, 1, 2, 1, 0]))
    assert e.value.kind == "Param" and e.value.name == "max_iter"
    with pytest.raises(StageError) as e:
        cap.run_params(t, b"\0" * 24)
    assert e.value.code == N.GR_PARAMS_MALFORMED


def test_wire_schema_encoding():
    view = find(FA2_ID).params
    b = view.encode()
    (count,) = struct.unpack_from("<I", b, 0)
    assert count == 11
    at = 4
    for spec in view.specs():
        (ln,) = struct.unpack_from("<I", b, at)
        at += 4
        assert b[at:at + ln].decode() == spec.name
        at += ln
        assert b[at] == spec.kind
        at += 1
        assert struct.unpack_from("<dddd", b, at) == (spec.min, spec.max, spec.default, spec.step)
        at += 32
        (dl,) = struct.unpack_from("<I", b, at)
        at += 4 + dl
    assert at == len(b)


def test_empty_spec_view_refuses_any_buffer():
    v = ParamsView([])
    with pytest.raises(ParamsError) as e:
        v.validate(b"\0" * 8)
    assert e.value.kind == "NotAccepted"


def test_static_entry_point_refuses_oversize_without_touching_a_device():
    pb = encode_params(find(FA2_ID).params.defaults())
    rc = N.lib().gr_fa2_forces_static(1 << 20, None, None, None, None, C.c_char_p(pb), len(pb), 0, None, None)
    assert rc == N.GR_INVALID_ARGUMENT
    rc = N.lib().gr_fa2_forces_static(10, None, None, None, None, C.c_char_p(b"\0" * 8), 8, 0, None, None)
    assert rc == N.GR_PARAMS_MALFORMED


def test_d3_row_refuses_parameters_before_any_device_work():
    from graph_render_b200 import D3_ID, StageError, Topology

    with pytest.raises(StageError) as e:
        find(D3_ID).run_params(Topology(3, [0, 1], [1, 2]), b"\0" * 8)
    assert e.value.code == N.GR_PARAMS_NOT_ACCEPTED
