"""Seeded synthetic workloads (host side): graphs, start positions, weights.

Thin ctypes face of ``libgraph_synth.so`` (``csrc/synth.c``) plus the workload
recipes the engine is measured on. No dataset is involved anywhere: every
graph is generated from its seed.
"""

from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgraph_synth.so")
_lib = None


def use_library(path: str) -> None:
    """Draw from another build of csrc/synth.c (the same generators and seeds),
    e.g. one linked into a CPU baseline's own library. Call before any draw."""
    global LIB_PATH, _lib
    if _lib is not None and path != LIB_PATH:
        raise RuntimeError("the generators are already loaded from " + LIB_PATH)
    LIB_PATH = path


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from .build import build_synth

            build_synth()
        L = C.CDLL(LIB_PATH)
        vp, i64, u64, u32, d = C.c_void_p, C.c_int64, C.c_uint64, C.c_uint32, C.c_double
        L.syn_sbm.argtypes = [u32, vp, d, d, u64, vp, vp, i64]
        L.syn_sbm.restype = i64
        L.syn_ba.argtypes = [u32, u32, u64, vp, vp, i64]
        L.syn_ba.restype = i64
        L.syn_config_powerlaw.argtypes = [u32, d, u32, d, u64, vp, vp, i64]
        L.syn_config_powerlaw.restype = i64
        L.syn_grid.argtypes = [u32, d, u64, vp, vp, i64]
        L.syn_grid.restype = i64
        L.syn_uniform.argtypes = [u32, u32, d, d, u64, vp]
        L.syn_lognormal.argtypes = [u64, d, d, u64, vp]
        L.syn_randint.argtypes = [u64, u32, u64, vp]
        L.syn_unit.argtypes = [u64, u64, vp]
        L.syn_gate.argtypes = [u32, vp, vp, vp, i64]
        L.syn_gate.restype = i64
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _edges(fn, guess: int, *args):
    cap = max(int(guess), 16)
    while True:
        src = np.zeros(cap, np.uint32)
        dst = np.zeros(cap, np.uint32)
        m = fn(*args, _p(src), _p(dst), cap)
        if m <= cap:
            return src[:m].copy(), dst[:m].copy()
        cap = int(m)


def sbm(sizes, p_in: float, p_out: float, seed: int):
    sizes = np.ascontiguousarray(sizes, np.uint32)
    n = int(sizes.sum())
    guess = 1.3 * (p_in * float((sizes.astype(np.float64) ** 2).sum()) / 2 + p_out * n * n / 2) + 64
    return _edges(lib().syn_sbm, guess, len(sizes), _p(sizes), p_in, p_out, seed)


def ba(n: int, m: int, seed: int):
    return _edges(lib().syn_ba, n * m + m + 16, n, m, seed)


def config_powerlaw(n: int, seed: int, alpha: float = 2.5, kmin: int = 2, xmin: float = 2.83):
    return _edges(lib().syn_config_powerlaw, n * 5 + 64, n, alpha, kmin, xmin, seed)


def grid(n: int, rewire: float, seed: int):
    return _edges(lib().syn_grid, 2 * n + 16, n, rewire, seed)


def uniform(n: int, dim: int, lo: float, hi: float, seed: int) -> np.ndarray:
    out = np.zeros((n, dim), np.float32)
    lib().syn_uniform(n, dim, lo, hi, seed, _p(out))
    return out


def lognormal(m: int, mu: float, sigma: float, seed: int) -> np.ndarray:
    out = np.zeros(m, np.float64)
    lib().syn_lognormal(m, mu, sigma, seed, _p(out))
    return out


def randint(count: int, n: int, seed: int) -> np.ndarray:
    out = np.zeros(count, np.uint32)
    lib().syn_randint(count, n, seed, _p(out))
    return out


def unit(count: int, seed: int) -> np.ndarray:
    out = np.zeros(count, np.float64)
    lib().syn_unit(count, seed, _p(out))
    return out


@dataclass
class Workload:
    name: str
    n: int
    src: np.ndarray
    dst: np.ndarray
    weight: Optional[np.ndarray]
    pos0: np.ndarray
    params: dict
    ticks: int

    @property
    def m(self) -> int:
        return int(len(self.src))


def sbm_1500(seed: int = 1) -> Workload:
    """SBM 1,500 nodes in 4 blocks (p_in 0.02, p_out 0.001), unit weights, start
    U[-1000, 1000]^2, scaling 2, gravity 1, theta 1.2, 100 ticks."""
    s, d = sbm([375] * 4, 0.02, 0.001, seed)
    pos = uniform(1500, 2, -1000.0, 1000.0, seed + 1000)
    return Workload("sbm1500-2d", 1500, s, d, None, pos,
                    dict(scaling_ratio=2.0, gravity=1.0, theta=1.2, dim=2, seed=seed, max_iter=100), 100)


def ba_100k(seed: int = 2, n: int = 100_000) -> Workload:
    """BA n=100k, m=3, lognormal(0, 0.5) weights, linlog + dissuade hubs,
    theta 1.0, start U[0, sqrt(n)*10]^2, 500 ticks."""
    s, d = ba(n, 3, seed)
    w = lognormal(len(s), 0.0, 0.5, seed + 7)
    side = math.sqrt(n) * 10.0
    pos = uniform(n, 2, 0.0, side, seed + 1000)
    return Workload(f"ba{n}-2d-linlog", n, s, d, w, pos,
                    dict(theta=1.0, lin_log=1, dissuade_hubs=1, edge_weight_influence=1.0, dim=2,
                         seed=seed, max_iter=500), 500)


def powerlaw_1m(seed: int = 3, n: int = 1_000_000, dim: int = 3) -> Workload:
    """Configuration model, power-law exponent 2.5, min degree 2, mean ~8
    (~4M edges), unit weights, start U[0, 1e4]^dim, theta 1.2; 3D with strong
    gravity (300 ticks), or the same graph laid out in 2D."""
    s, d = config_powerlaw(n, seed)
    pos = uniform(n, dim, 0.0, 1e4, seed + 1000)
    prm = dict(theta=1.2, dim=dim, seed=seed, max_iter=300 if dim == 3 else 100)
    if dim == 3:
        prm["strong_gravity"] = 1
    return Workload(f"powerlaw{n}-{dim}d", n, s, d, None, pos, prm, prm["max_iter"])


def sbm_50k(seed: int = 5, n: int = 50_000, blocks: int = 16) -> Workload:
    """SBM n nodes in `blocks` blocks (p_in 5e-3, p_out 5e-5 at 50k), weights 1, 200 ticks."""
    sizes = [n // blocks + (1 if b < n % blocks else 0) for b in range(blocks)]
    scale = 50_000 / n
    s, d = sbm(sizes, min(1.0, 5e-3 * scale), min(1.0, 5e-5 * scale), seed)
    pos = uniform(n, 2, 0.0, math.sqrt(n) * 10.0, seed + 1000)
    return Workload(f"sbm{n}-2d", n, s, d, np.ones(len(s)), pos,
                    dict(theta=1.2, dim=2, seed=seed, max_iter=200, edge_weight_influence=1.0), 200)


def gate(n: int):
    """The reference's benchmark model with n nodes (crates/graph-core/src/synthetic.rs:92-170):
    (source, target, strength) of its raw edges, in edge order."""
    cap = 2 * n + n // 20 + 16
    src = np.zeros(cap, np.uint32)
    dst = np.zeros(cap, np.uint32)
    st = np.zeros(cap, np.float64)
    m = lib().syn_gate(n, _p(src), _p(dst), _p(st), cap)
    assert m <= cap
    return src[:m].copy(), dst[:m].copy(), st[:m].copy()
