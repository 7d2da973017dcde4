"""Batched ForceAtlas2: many independent graphs in one persistent launch.

``Batch`` wraps ``gr_fa2_batch_*`` (include/graph_cuda.h). ``mixed_batch``
draws the mixed workload (SBM / Barabasi-Albert / grid with rewiring, node
counts log-uniform, per-graph scaling and gravity), each graph from its own
seed so that a rank can generate only the graphs it owns; ``shard`` assigns
graphs to ranks by longest-processing-time first.
"""

from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import _native as N
from . import synth
from .fa2 import DEFAULTS, PARAM_NAMES


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


@dataclass
class GraphSpec:
    n: int
    src: np.ndarray
    dst: np.ndarray
    params: dict
    weight: Optional[np.ndarray] = None
    pos0: Optional[np.ndarray] = None
    kind: str = ""

    @property
    def m(self) -> int:
        return int(len(self.src))


def param_row(p: dict) -> List[float]:
    vals = dict(DEFAULTS)
    vals.update(p)
    return [float(vals[k]) for k in PARAM_NAMES]


class Batch:
    """A batch of graphs on one GPU (``gr_fa2_batch_create`` .. ``destroy``)."""

    def __init__(self, graphs: Sequence[GraphSpec]):
        L = N.lib()
        self._L = L
        self.graphs = list(graphs)
        G = len(self.graphs)
        self.dim = int(param_row(self.graphs[0].params)[5])
        self.n = np.array([g.n for g in self.graphs], np.uint32)
        self.m = np.array([g.m for g in self.graphs], np.uint64)
        self.off = np.concatenate([[0], np.cumsum(self.n.astype(np.int64))])
        src = np.ascontiguousarray(np.concatenate([g.src for g in self.graphs]) if G else [], np.uint32)
        dst = np.ascontiguousarray(np.concatenate([g.dst for g in self.graphs]) if G else [], np.uint32)
        has_w = any(g.weight is not None for g in self.graphs)
        w = None
        if has_w:
            w = np.ascontiguousarray(np.concatenate(
                [g.weight if g.weight is not None else np.ones(g.m) for g in self.graphs]), np.float64)
        prm = np.ascontiguousarray([param_row(g.params) for g in self.graphs], np.float64)
        pos = None
        if all(g.pos0 is not None for g in self.graphs):
            pos = np.ascontiguousarray(np.concatenate(
                [np.asarray(g.pos0, np.float32).reshape(g.n, self.dim) for g in self.graphs]), np.float32)
        self._keep = (src, dst, w, prm, pos)
        h = C.c_void_p()
        N.check(L.gr_fa2_batch_create(C.byref(h), G, _ptr(self.n), _ptr(self.m), _ptr(src), _ptr(dst), _ptr(w),
                                      _ptr(prm), len(PARAM_NAMES), _ptr(pos)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self._L.gr_fa2_batch_destroy(self.h)
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

    def set_threads(self, threads: int) -> None:
        N.check(self._L.gr_fa2_batch_set_threads(self.h, int(threads)))

    def tune(self, sample_ticks: int = 3):
        chosen = C.c_int()
        ms = np.zeros(3, np.float32)
        N.check(self._L.gr_fa2_batch_tune(self.h, int(sample_ticks), C.byref(chosen), _ptr(ms)))
        return chosen.value, dict(zip((256, 512, 1024), ms.tolist()))

    def run(self, ticks: int) -> float:
        """Runs every graph `ticks` ticks (or until it converges) in one launch;
        returns the launch's device time in ms."""
        ms = C.c_float()
        N.check(self._L.gr_fa2_batch_run(self.h, int(ticks), C.byref(ms)))
        return ms.value

    def positions(self) -> List[np.ndarray]:
        out = np.zeros((int(self.off[-1]), self.dim), np.float32)
        N.check(self._L.gr_fa2_batch_positions(self.h, _ptr(out)))
        return [out[self.off[i]:self.off[i + 1]] for i in range(len(self.graphs))]

    def stats(self) -> dict:
        G = len(self.graphs)
        ticks = np.zeros(G, np.uint32)
        err = np.zeros(G, np.uint32)
        inter = np.zeros(2 * G, np.uint64)
        N.check(self._L.gr_fa2_batch_stats(self.h, _ptr(ticks), _ptr(err), _ptr(inter)))
        return dict(ticks=ticks, errors=err, far=inter[0::2], pair=inter[1::2])


def _graph_rng(seed: int, i: int) -> np.random.Generator:
    return np.random.default_rng([int(seed), int(i)])


def mixed_graph(seed: int, i: int, nmin: int = 50, nmax: int = 20_000, ticks: int = 200) -> GraphSpec:
    """Graph i of the mixed batch: n log-uniform in [nmin, nmax], an SBM (2-8
    blocks), a BA (m 2-4) or a 2D grid with 5% rewiring, mean degree 4-10,
    scaling U[1, 10], gravity U[0.1, 5]."""
    r = _graph_rng(seed, i)
    n = int(round(math.exp(r.uniform(math.log(nmin), math.log(nmax)))))
    kind = ("sbm", "ba", "grid")[int(r.integers(0, 3))]
    gseed = int(r.integers(0, 2 ** 62))
    if kind == "sbm":
        blocks = int(r.integers(2, 9))
        kbar = float(r.uniform(4.0, 10.0))
        sizes = [n // blocks + (1 if b < n % blocks else 0) for b in range(blocks)]
        s = n / blocks
        ratio = 20.0  # p_in / p_out
        p_in = kbar / ((s - 1) + (n - s) / ratio) if n > 1 else 0.0
        src, dst = synth.sbm(sizes, min(1.0, p_in), min(1.0, p_in / ratio), gseed)
    elif kind == "ba":
        src, dst = synth.ba(n, int(r.integers(2, 5)), gseed)
    else:
        src, dst = synth.grid(n, 0.05, gseed)
    side = math.sqrt(n) * 10.0
    pos = synth.uniform(n, 2, 0.0, side, gseed + 1)
    prm = dict(scaling_ratio=float(r.uniform(1.0, 10.0)), gravity=float(r.uniform(0.1, 5.0)), theta=1.2, dim=2,
               seed=int(r.integers(0, 2 ** 31)), max_iter=ticks)
    return GraphSpec(n, src, dst, prm, None, pos, kind)


def shard(costs: Sequence[float], world: int) -> List[List[int]]:
    """Longest-processing-time assignment of items to `world` bins."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    bins: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        b = min(range(world), key=lambda k: (load[k], k))
        bins[b].append(i)
        load[b] += costs[i]
    return [sorted(x) for x in bins]


def graph_cost(seed: int, i: int, nmin: int = 50, nmax: int = 20_000) -> float:
    """The cost estimate `shard` uses (n log n), from the same draw as mixed_graph."""
    r = _graph_rng(seed, i)
    n = round(math.exp(r.uniform(math.log(nmin), math.log(nmax))))
    return n * math.log2(n + 1)
