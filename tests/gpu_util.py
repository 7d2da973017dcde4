"""Shared helpers for the GPU parity tests: run the engine and the oracle on
the same positions and compare."""

import os

import numpy as np

from oracle import oracle as O
from graph_render_b200 import Fa2

LEVELS = {2: 32, 3: 21}  # the engine's Morton depth per axis


def oracle_state(n, src, dst, w, pos, prm, theta=None, dense=False):
    lo, hi, ws = O.simple_graph(n, src, dst, w)
    dim = int(prm.get("dim", 2))
    th = prm.get("theta", 0.8) if theta is None else theta
    return O.State(
        n, lo, hi, w=ws, pos0=np.asarray(pos, np.float32).astype(np.float64),
        dim=dim, theta=-1.0 if dense else th,
        scaling_ratio=prm.get("scaling_ratio", 2.0), gravity=prm.get("gravity", 1.0),
        jitter_tolerance=prm.get("jitter_tolerance", 1.0), seed=prm.get("seed", 0),
        lin_log=prm.get("lin_log", 0), strong_gravity=prm.get("strong_gravity", 0),
        dissuade_hubs=prm.get("dissuade_hubs", 0),
        edge_weight_influence=prm.get("edge_weight_influence", 0.0),
        depth_cap=LEVELS[dim], threads=os.cpu_count() or 1)


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def force_parity(n, src, dst, w, pos, prm, dense_oracle=False):
    """(relative L2 of GPU forces vs oracle forces, engine info, oracle scalars)."""
    with Fa2(n, src, dst, w, params=dict(prm), pos0=pos) as eng:
        fg = eng.forces().astype(np.float64)
        info = eng.info()
    st = oracle_state(n, src, dst, w, pos, prm, dense=dense_oracle)
    fr = st.accumulate(7)
    return rel_l2(fg, fr), info, st.scalars()


def collapsed_cells(st) -> int:
    """Cells of the oracle's last tree once single-child chains are collapsed
    (the engine keeps only the deepest cell of a chain)."""
    t = st.tree()
    skip = t["skip"]
    k_total = 0
    for k in range(len(skip)):
        if skip[k] == k + 1:
            k_total += 1
            continue
        c, nch = k + 1, 0
        while c < skip[k]:
            nch += 1
            c = skip[c]
        if nch >= 2:
            k_total += 1
    return k_total
