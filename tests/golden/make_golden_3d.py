"""Writes tests/golden/fa2_nx_gate_3d.jsonl with networkx 3.6: the 3D gate fixture.

The reference gates its 3D FA2 arm (`layout.forceatlas2.3d`) against networkx's
forceatlas2_layout at dim 3 and 2 iterations, from its own start, with a 1e-7
ceiling (docs/measurements/p12-t4b.md:67-80; networkx takes the dimension from
the width of the start it is given). It commits no 3D fixture, so this script
makes one the same way tests/golden/make_golden.py remakes the 2D one: for gate
seeds 0..63 (n = seed + 2, crates/graph-core/src/stage/topology.rs:19-21), the
gate model's edges (crates/graph-core/src/synthetic.rs:92-170, restated in
oracle/fa2_oracle.c), the Mulberry32(0) start in [0, 1)^3 (three draws per node,
crates/graph-core/src/layout/forceatlas2/state.rs:272-283), networkx's own
forceatlas2_layout for 2 iterations.

Run from the repository root: python tests/golden/make_golden_3d.py
"""

import json
import os
import sys

import networkx as nx
import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402


def main(out_path=os.path.join(ROOT, "tests", "golden", "fa2_nx_gate_3d.jsonl")):
    lines = []
    for seed in range(64):
        n = seed + 2
        src, dst, _ = O.gate_edges(n)
        g = nx.Graph()
        g.add_nodes_from(range(n))
        g.add_edges_from(zip(src.tolist(), dst.tolist()))
        start = O.initial_positions(n, 0, 3)
        pos = {i: start[i].copy() for i in range(n)}
        out = nx.forceatlas2_layout(g, pos=pos, max_iter=2, dim=3)
        xyz = np.array([out[i] for i in range(n)])
        lines.append(json.dumps({"seed": seed, "n": n, "max_iter": 2, "x": xyz[:, 0].tolist(),
                                 "y": xyz[:, 1].tolist(), "z": xyz[:, 2].tolist()}))
    with open(out_path, "w") as f:
        f.write("\n".join(lines) + "\n")
    print(f"wrote {len(lines)} lines to {out_path} (networkx {nx.__version__})")


if __name__ == "__main__":
    main()
