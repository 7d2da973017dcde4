"""Layout quality of a finished ForceAtlas2 run: the energy of its force laws.

Full runs of the same graph diverge chaotically (one ulp at the start moves a
node by a quarter of the extent after 100 ticks), so two engines' final layouts
are compared on measures of the whole layout: this energy and the sampled
Kruskal stress (`stress.kruskal_stress`). The reference defines no FA2 energy;
this one is the potential whose negative gradient is each force the tick
applies (state.rs:152-251, networkx layout.py:1806-1832), with the gravity
centre held fixed at the layout's mean:

- attraction, per simple edge of weight c = w^influence: linear 1/2 c d^2
  (force c (q - p)); linlog c ((1 + d) ln(1 + d) - d) (force c ln(1 + d) / d
  (q - p)). With dissuade hubs the tick divides node i's attraction by its
  mass, which no single potential gives; the edge term is then weighted by
  (1/m_i + 1/m_j) / 2 (a convention, exact only when both masses are equal);
- repulsion, per node pair: -k_r m_i m_j ln d (force k_r m_i m_j / d^2 (p_i - p_j));
- gravity, per node, c_i = p_i - mean: g m_i |c_i| (force -g m_i c_i / |c_i|),
  or with strong gravity 1/2 g m_i |c_i|^2 (force -g m_i c_i).

Masses are degree + 1 over the simple graph (self-loops dropped, the first of
duplicate edges kept, state.rs:83-102). Computed in FP64 on the host over every
node pair (O(n^2), chunked): a measure for test and evaluation sizes, not a
step of the tick. For large graphs `pair_sample` estimates the repulsion term
from that many node pairs drawn uniformly from `seed` (the pair sum scaled by
n(n-1)/2 over the sample size); two layouts compared with the same sample and
seed are measured on the same pairs.
"""

from __future__ import annotations

import numpy as np

from .fa2 import DEFAULTS


def simple_edges(n: int, src, dst, weight=None):
    """(lo, hi, w) with lo < hi, self-loops dropped and the first of duplicate
    edges kept, in input order (layout/force/mod.rs:101-131)."""
    src = np.asarray(src, np.int64)
    dst = np.asarray(dst, np.int64)
    w = np.ones(len(src)) if weight is None else np.asarray(weight, np.float64)
    lo, hi = np.minimum(src, dst), np.maximum(src, dst)
    keep = lo != hi
    lo, hi, w = lo[keep], hi[keep], w[keep]
    _, first = np.unique(lo * int(n) + hi, return_index=True)
    first.sort()
    return lo[first], hi[first], w[first]


def sampled_repulsion(p, mass, kr: float, pairs: int, seed: int, chunk: int = 1 << 22) -> float:
    """-k_r sum m_i m_j ln d over all pairs i < j, estimated from `pairs` pairs
    (i, j), i != j, drawn uniformly from `seed`."""
    n = p.shape[0]
    rng = np.random.default_rng(seed)
    total, drawn = 0.0, 0
    while drawn < pairs:
        k = min(chunk, pairs - drawn)
        i = rng.integers(0, n, k)
        j = rng.integers(0, n - 1, k)
        j = j + (j >= i)  # uniform over j != i
        r = np.sqrt(((p[i] - p[j]) ** 2).sum(1))
        with np.errstate(divide="ignore"):
            total += float((mass[i] * mass[j] * np.log(r)).sum())
        drawn += k
    return -kr * total * (n * (n - 1) / 2.0) / pairs


def fa2_energy(pos, src, dst, weight=None, params=None, chunk: int = 2048, pair_sample=None,
               seed: int = 0) -> dict:
    """Energy terms of the layout `pos` (n x dim) under the FA2 parameters
    `params` (the engine's names and defaults): {"attraction", "repulsion",
    "gravity", "total"}. With `pair_sample` the repulsion term is estimated
    from that many uniformly drawn pairs (`sampled_repulsion`)."""
    prm = dict(DEFAULTS)
    prm.update(params or {})
    p = np.asarray(pos, np.float64)
    n = p.shape[0]
    lo, hi, w = simple_edges(n, src, dst, weight)
    mass = 1.0 + np.bincount(lo, minlength=n) + np.bincount(hi, minlength=n)
    c = w ** float(prm["edge_weight_influence"])
    d = np.sqrt(((p[hi] - p[lo]) ** 2).sum(1))
    if int(prm["lin_log"]):
        att = c * ((1.0 + d) * np.log1p(d) - d)
    else:
        att = 0.5 * c * d * d
    if int(prm["dissuade_hubs"]):
        att = att * 0.5 * (1.0 / mass[lo] + 1.0 / mass[hi])
    kr = float(prm["scaling_ratio"])
    rep = 0.0
    if pair_sample is not None and n > 1:
        rep = sampled_repulsion(p, mass, kr, int(pair_sample), seed)
    for a in (range(0, n, chunk) if pair_sample is None else ()):
        b = min(n, a + chunk)
        # pairs (i, j) with i in [a, b) and j > i
        dx = p[a:b, None, :] - p[None, a:, :]
        r = np.sqrt((dx * dx).sum(2))
        iu = np.arange(a, b)[:, None] < np.arange(a, n)[None, :]
        mm = mass[a:b, None] * mass[None, a:]
        with np.errstate(divide="ignore"):
            rep -= kr * float((mm * np.log(np.where(iu, r, 1.0)))[iu].sum())
    cc = p - p.mean(0)
    r = np.sqrt((cc * cc).sum(1))
    g = float(prm["gravity"])
    grav = 0.5 * g * (mass * r * r).sum() if int(prm["strong_gravity"]) else g * (mass * r).sum()
    out = {"attraction": float(att.sum()), "repulsion": rep, "gravity": float(grav)}
    out["total"] = out["attraction"] + out["repulsion"] + out["gravity"]
    return out
