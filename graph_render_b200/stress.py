"""Sampled Kruskal stress-1 against hop distance, and its gradient.

The reference's quality measure (crates/graph-cli/src/bench.rs:256-295):
stress-1 with the optimal scale, sqrt((DD - DE^2/EE) / DD) over node pairs,
DE = sum d e, EE = sum e^2, DD = sum d^2, d the hop distance and e the
Euclidean distance. `kruskal_stress` is that measure (every target of the
evenly spaced BFS sources), on the device. For the differentiated workload the
pairs are sampled from a seed (`sample_pairs`, hop counts from the device BFS),
unreachable pairs are dropped, and `stress` also returns dL/dpositions.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from . import synth


def bfs_hops(n: int, src, dst, sources) -> np.ndarray:
    """Hop distances from each source to every node (uint32, MAX if unreachable),
    by the device's multi-source BFS (gr_bfs_hops)."""
    src = np.ascontiguousarray(src, np.uint32)
    dst = np.ascontiguousarray(dst, np.uint32)
    sources = np.ascontiguousarray(sources, np.uint32)
    out = np.zeros((len(sources), n), np.uint32)
    N.check(N.lib().gr_bfs_hops(n, len(src), _p(src), _p(dst), len(sources), _p(sources), _p(out)))
    return out


def kruskal_stress(x, y, src, dst, sources: int = 16) -> float:
    """The reference's quality measure (graph-cli/src/bench.rs:255-295 `stress`):
    Kruskal stress-1 of (x, y) against hop distance from every max(n / sources,
    1)-th node, on the device (gr_stress)."""
    x = np.ascontiguousarray(x, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    src = np.ascontiguousarray(src, np.uint32)
    dst = np.ascontiguousarray(dst, np.uint32)
    out = C.c_double()
    N.check(N.lib().gr_stress(len(x), len(src), _p(src), _p(dst), _p(x), _p(y), sources, C.byref(out)))
    return out.value


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p) if a.size else None


def sample_pairs(n: int, src, dst, pairs: int, seed: int, sources: int = 1000):
    """`pairs` node pairs: `sources` uniform source nodes (one BFS each), each
    with pairs/sources uniform targets. Returns (a, b, hops) for the reachable,
    distinct pairs."""
    sources = min(sources, n)
    per = max(1, pairs // sources)
    s = synth.randint(sources, n, seed).astype(np.uint32)
    t = synth.randint(sources * per, n, seed + 1).astype(np.uint32).reshape(sources, per)
    hops = bfs_hops(n, src, dst, s)
    h = np.take_along_axis(hops, t.astype(np.int64), axis=1)
    a = np.repeat(s, per)
    b = t.reshape(-1)
    h = h.reshape(-1)
    keep = (h != np.iinfo(np.uint32).max) & (a != b)
    return a[keep], b[keep], h[keep].astype(np.float64)


def stress(pos, a, b, hops):
    """(stress-1, dL/dpos) at positions pos (n x dim)."""
    p = np.asarray(pos, np.float64)
    diff = p[a] - p[b]
    e = np.sqrt((diff * diff).sum(1))
    d = hops
    DE, EE, DD = float((d * e).sum()), float((e * e).sum()), float((d * d).sum())
    if EE == 0.0 or DD == 0.0:
        return 1.0, np.zeros_like(p)
    S = max((DD - DE * DE / EE) / DD, 0.0)
    L = float(np.sqrt(S))
    if L == 0.0:
        return 0.0, np.zeros_like(p)
    dS_dDE = -2.0 * DE / (EE * DD)
    dS_dEE = DE * DE / (EE * EE * DD)
    dL_de = (dS_dDE * d + dS_dEE * 2.0 * e) / (2.0 * L)
    with np.errstate(invalid="ignore", divide="ignore"):
        unit = np.where(e[:, None] > 0, diff / e[:, None], 0.0)
    g = np.zeros_like(p)
    contrib = dL_de[:, None] * unit
    np.add.at(g, a, contrib)
    np.add.at(g, b, -contrib)
    return L, g
