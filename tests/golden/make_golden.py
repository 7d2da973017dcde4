"""Regenerates tests/golden/fa2_nx_gate.jsonl with networkx 3.6.

For gate seeds 0..63 (n = seed + 2, crates/graph-core/src/stage/topology.rs:19-21)
it builds the gate model's edges (crates/graph-core/src/synthetic.rs:92-170,
restated in oracle/fa2_oracle.c), starts from Mulberry32(0) positions
(crates/graph-core/src/layout/forceatlas2/state.rs:272-283) and runs networkx's
own forceatlas2_layout for 2 iterations, the reference's gated budget
(crates/graph-cli/tests/cli_fa2.rs:26). The output has the same keys as the
reference's crates/graph-cli/tests/fixtures/fa2-nx-reference.jsonl, which
tests/test_oracle.py compares it against when the reference tree is present.

Run from the repository root: python tests/golden/make_golden.py
"""

import json
import os
import sys

import networkx as nx
import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402


def main(out_path=os.path.join(ROOT, "tests", "golden", "fa2_nx_gate.jsonl")):
    lines = []
    for seed in range(64):
        n = seed + 2
        src, dst, _ = O.gate_edges(n)
        g = nx.Graph()
        g.add_nodes_from(range(n))
        g.add_edges_from(zip(src.tolist(), dst.tolist()))
        start = O.initial_positions(n, 0, 2)
        pos = {i: start[i].copy() for i in range(n)}
        out = nx.forceatlas2_layout(g, pos=pos, max_iter=2)
        xy = np.array([out[i] for i in range(n)])
        lines.append(json.dumps({"seed": seed, "n": n, "max_iter": 2,
                                 "x": xy[:, 0].tolist(), "y": xy[:, 1].tolist()}))
    with open(out_path, "w") as f:
        f.write("\n".join(lines) + "\n")
    print(f"wrote {len(lines)} lines to {out_path} (networkx {nx.__version__})")


if __name__ == "__main__":
    main()
