"""The allocation-free force entry point, gr_fa2_forces_static, on the GPU.

Some callers cannot allocate device memory: a plugin that only receives device
buffers from the runtime hosting it, or code enqueuing onto a stream that is
being captured into a CUDA graph. For them the library keeps the scratch of one
force evaluation in a fixed device array compiled into it. This test plays such
a caller: it owns its device buffers (torch allocates them, standing in for the
hosting runtime), calls the entry point through the C ABI twice in a row on two
different graphs, and checks each result against gr_fa2_forces on the same
graph and positions within the parity tolerance (1e-5 relative L2). It also
checks that a graph above the array's stated maximum is refused.

This file sorts last so a run that stops at the first failure has run every
other test before it.
"""

import ctypes as C

import numpy as np
import pytest

from graph_render_b200 import Fa2, _native as N, params_bytes, synth

pytestmark = pytest.mark.gpu

TOL = 1e-5


def csr(n, src, dst, w):
    """The engine's simple graph (first raw edge per pair wins) as a CSR sorted by
    (row, col), with mass = degree + 1."""
    src = np.asarray(src, np.uint64)
    dst = np.asarray(dst, np.uint64)
    keep = src != dst
    lo = np.minimum(src, dst)[keep]
    hi = np.maximum(src, dst)[keep]
    ww = (np.ones(len(src)) if w is None else np.asarray(w, np.float64))[keep]
    keys, first = np.unique((lo << np.uint64(32)) | hi, return_index=True)
    lo, hi, ww = lo[first], hi[first], ww[first]
    rows = np.concatenate([lo, hi]).astype(np.int64)
    cols = np.concatenate([hi, lo]).astype(np.int64)
    wts = np.concatenate([ww, ww])
    order = np.lexsort((cols, rows))
    rows, cols, wts = rows[order], cols[order], wts[order]
    rp = np.searchsorted(rows, np.arange(n + 1)).astype(np.int32)
    mass = (np.diff(rp) + 1).astype(np.float32)
    return rp, cols.astype(np.int32), wts, mass


def static_forces(n, src, dst, w, pos, prm):
    import torch

    dim = int(prm.get("dim", 2))
    rp, col, wts, mass = csr(n, src, dst, w)
    infl = float(prm.get("edge_weight_influence", 0.0))
    wq = np.ones_like(wts) if infl == 0.0 else wts ** infl
    nodes = np.zeros((n, 4), np.float32)
    nodes[:, :dim] = pos
    nodes[:, 3] = mass
    dev = torch.device("cuda", 0)
    d_nodes = torch.from_numpy(nodes).to(dev)
    d_rp = torch.from_numpy(rp).to(dev)
    d_col = torch.from_numpy(col if len(col) else np.zeros(1, np.int32)).to(dev)
    d_w = torch.from_numpy(wq.astype(np.float32) if len(wq) else np.ones(1, np.float32)).to(dev)
    d_out = torch.zeros((n, dim), dtype=torch.float32, device=dev)
    pb = params_bytes(prm)
    stream = torch.cuda.current_stream(dev)
    rc = N.lib().gr_fa2_forces_static(n, C.c_void_p(d_nodes.data_ptr()), C.c_void_p(d_rp.data_ptr()),
                                      C.c_void_p(d_col.data_ptr()), C.c_void_p(d_w.data_ptr()),
                                      C.c_char_p(pb), len(pb), 0, C.c_void_p(d_out.data_ptr()),
                                      C.c_void_p(stream.cuda_stream))
    N.check(rc)
    torch.cuda.synchronize(dev)
    return d_out.cpu().numpy().astype(np.float64)


def allocating_forces(n, src, dst, w, pos, prm):
    with Fa2(n, src, dst, w, params=dict(prm), pos0=pos) as eng:
        return eng.forces().astype(np.float64)


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_static_forces_match_the_allocating_entry_point_twice_in_a_row():
    wl = synth.sbm_1500()
    big = synth.powerlaw_1m(n=20_000, dim=3)  # hubs, octree, strong gravity
    cases = [(wl.n, wl.src, wl.dst, None, wl.pos0, wl.params),
             (big.n, big.src, big.dst, None, big.pos0, big.params)]
    for n, s, d, w, pos, prm in cases:
        got = static_forces(n, s, d, w, pos, prm)
        want = allocating_forces(n, s, d, w, pos, prm)
        assert np.isfinite(got).all()
        assert rel(got, want) < TOL, (n, rel(got, want))


def test_static_forces_refuse_a_graph_above_the_maximum():
    n = 32768 + 1
    pb = params_bytes({})
    rc = N.lib().gr_fa2_forces_static(n, None, None, None, None,
                                      C.c_char_p(pb), len(pb), 0, None, None)
    assert rc == N.GR_INVALID_ARGUMENT
    assert b"maximum" in N.lib().gr_last_error_message()
