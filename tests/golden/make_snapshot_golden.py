"""Extracts tests/golden/fa2_snapshot_sha256.txt from the reference's 2D golden pin.

The reference pins, for every 2D layout and seeds 0..7, the sha256 of the
snapshot's binary face that `graph-cli snapshot --seed S --layout L --out-bin -`
writes (harness/golden-2d.sh, harness/golden-2d-before.txt). This keeps the
`layout.forceatlas2` lines (the dense FA2 arm over the gate model with n = 2 + seed
nodes, crates/graph-core/src/stage/topology.rs:19-35) and the
`layout.force.barnes_hut` lines, unchanged.

Run from the repository root with the reference tree present:
python tests/golden/make_snapshot_golden.py /path/to/reference
"""

import os
import sys

KEEP = ("layout.forceatlas2", "layout.force.barnes_hut")


def main(ref_root: str) -> None:
    src = os.path.join(ref_root, "harness", "golden-2d-before.txt")
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "fa2_snapshot_sha256.txt")
    lines = [ln.strip() for ln in open(src) if ln.split() and ln.split()[0] in KEEP]
    with open(out, "w") as f:
        f.write("# layout seed sha256 of the snapshot binary face (reference harness/golden-2d-before.txt)\n")
        f.write("\n".join(lines) + "\n")
    print(f"wrote {len(lines)} lines to {out}")


if __name__ == "__main__":
    if len(sys.argv) > 1:
        main(sys.argv[1])
    elif os.environ.get("GRAPH_RENDER_REFERENCE"):
        main(os.environ["GRAPH_RENDER_REFERENCE"])
    else:
        sys.exit(f"usage: python {sys.argv[0]} <reference checkout> (or set GRAPH_RENDER_REFERENCE)")
