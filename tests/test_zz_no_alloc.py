"""The allocation-free force entry point, gr_fa2_forces_static, on the GPU.

Some callers cannot allocate device memory: code running inside another GPU
runtime that owns every device allocation, or a plugin that only receives
device buffers from the program hosting it. For them the library keeps the
scratch of one force evaluation in a fixed device array compiled into it. This
test plays such a caller: it owns its device buffers (torch allocates them,
standing in for the hosting runtime), calls the entry point through the C ABI
several times in a row on graphs of different sizes and dimensions (the larger
graph first, so a dependence on what a larger earlier call left in the array
would show), checks that the device's free memory does not change across those
calls, and checks each result against gr_fa2_forces on the same graph and
positions within the parity tolerance (1e-5 relative L2). It also checks that
a graph above the array's stated maximum, and a null device buffer, are refused,
and that gr_fa2_forces_static_status reports a non-finite position of the last
evaluation (GR_LAYOUT_FAILED) and a clean one after it.

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


class StaticCall:
    """Device buffers for one graph, owned by the caller, and the call itself."""

    def __init__(self, n, src, dst, w, pos, prm):
        import torch

        self.n, self.prm = n, prm
        self.dim = int(prm.get("dim", 2))
        rp, col, wts, mass = csr(n, src, dst, w)
        infl = float(prm.get("edge_weight_influence", 0.0))
        wq = np.ones_like(wts) if infl == 0.0 else wts ** infl
        nodes = np.zeros((n, 4), np.float32)
        nodes[:, :self.dim] = pos
        nodes[:, 3] = mass
        self.dev = torch.device("cuda", 0)
        self.d_nodes = torch.from_numpy(nodes).to(self.dev)
        self.d_rp = torch.from_numpy(rp).to(self.dev)
        self.d_col = torch.from_numpy(col if len(col) else np.zeros(1, np.int32)).to(self.dev)
        self.d_w = torch.from_numpy(wq.astype(np.float32) if len(wq) else np.ones(1, np.float32)).to(self.dev)
        self.d_out = torch.zeros((n, self.dim), dtype=torch.float32, device=self.dev)
        self.pb = params_bytes(prm)

    def __call__(self):
        """Enqueues one evaluation on torch's current stream and waits for it."""
        import torch

        stream = torch.cuda.current_stream(self.dev)
        rc = N.lib().gr_fa2_forces_static(self.n, C.c_void_p(self.d_nodes.data_ptr()),
                                          C.c_void_p(self.d_rp.data_ptr()), C.c_void_p(self.d_col.data_ptr()),
                                          C.c_void_p(self.d_w.data_ptr()), C.c_char_p(self.pb), len(self.pb), 0,
                                          C.c_void_p(self.d_out.data_ptr()), C.c_void_p(stream.cuda_stream))
        N.check(rc)
        torch.cuda.synchronize(self.dev)
        return self.d_out.cpu().numpy().astype(np.float64)


def static_forces(n, src, dst, w, pos, prm):
    return StaticCall(n, src, dst, w, pos, prm)()


def allocating_forces(n, src, dst, w, pos, prm):
    with Fa2(n, src, dst, w, params=dict(prm), pos0=pos) as eng:
        return eng.forces().astype(np.float64)


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_static_forces_match_the_allocating_entry_point_twice_in_a_row():
    import torch

    wl = synth.sbm_1500()
    big = synth.powerlaw_1m(n=20_000, dim=3)  # hubs, octree, strong gravity
    cases = {"big": (big.n, big.src, big.dst, None, big.pos0, big.params),
             "small": (wl.n, wl.src, wl.dst, None, wl.pos0, wl.params)}
    calls = {k: StaticCall(*c) for k, c in cases.items()}
    # the first call of each kind loads its kernels (and the array with the
    # library's module); after that no call may change the free device memory
    for k in ("big", "small"):
        calls[k]()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    got = [(k, calls[k]()) for k in ("big", "small", "big", "small")]
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert np.array_equal(got[0][1], got[2][1]) and np.array_equal(got[1][1], got[3][1])
    for k, out in got[:2]:
        n, s, d, w, pos, prm = cases[k]
        want = allocating_forces(n, s, d, w, pos, prm)
        assert np.isfinite(out).all()
        assert rel(out, want) < TOL, (k, rel(out, want))


def test_static_forces_refuse_a_graph_above_the_maximum():
    n = 32768 + 1
    pb = params_bytes({})
    rc = N.lib().gr_fa2_forces_static(n, None, None, None, None,
                                      C.c_char_p(pb), len(pb), 0, None, None)
    assert rc == N.GR_INVALID_ARGUMENT
    assert b"maximum" in N.lib().gr_last_error_message()


def test_static_forces_refuse_a_null_device_buffer():
    import torch

    wl = synth.sbm_1500()
    call = StaticCall(wl.n, wl.src, wl.dst, None, wl.pos0, wl.params)
    args = [C.c_void_p(call.d_nodes.data_ptr()), C.c_void_p(call.d_rp.data_ptr()), C.c_void_p(call.d_col.data_ptr()),
            C.c_void_p(call.d_w.data_ptr())]
    for i in range(4):
        a = list(args)
        a[i] = None
        rc = N.lib().gr_fa2_forces_static(wl.n, *a, C.c_char_p(call.pb), len(call.pb), 0,
                                          C.c_void_p(call.d_out.data_ptr()), None)
        assert rc == N.GR_INVALID_ARGUMENT, i
    torch.cuda.synchronize()


def test_static_status_reports_a_non_finite_position_and_clears_on_the_next_call():
    import torch

    wl = synth.sbm_1500()
    call = StaticCall(wl.n, wl.src, wl.dst, None, wl.pos0, wl.params)
    want = call()
    bits = C.c_uint32(99)
    assert N.lib().gr_fa2_forces_static_status(C.byref(bits)) == N.GR_OK and bits.value == 0
    # a NaN coordinate: the bounds pass flags it and every later kernel returns
    # early, so the output buffer keeps what it held
    good = call.d_nodes[700, 1].item()
    call.d_nodes[700, 1] = float("nan")
    sentinel = torch.full_like(call.d_out, 7.0)
    call.d_out.copy_(sentinel)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream(call.dev)
    rc = N.lib().gr_fa2_forces_static(call.n, C.c_void_p(call.d_nodes.data_ptr()), C.c_void_p(call.d_rp.data_ptr()),
                                      C.c_void_p(call.d_col.data_ptr()), C.c_void_p(call.d_w.data_ptr()),
                                      C.c_char_p(call.pb), len(call.pb), 0, C.c_void_p(call.d_out.data_ptr()),
                                      C.c_void_p(stream.cuda_stream))
    assert rc == N.GR_OK  # enqueued: the failure is on the device
    torch.cuda.synchronize()
    rc = N.lib().gr_fa2_forces_static_status(C.byref(bits))
    assert rc == N.GR_LAYOUT_FAILED and bits.value & 1
    assert torch.equal(call.d_out, sentinel)
    # the next evaluation starts from a fresh state
    call.d_nodes[700, 1] = good
    assert np.array_equal(call(), want)
    assert N.lib().gr_fa2_forces_static_status(C.byref(bits)) == N.GR_OK and bits.value == 0
