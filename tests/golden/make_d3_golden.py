"""Extracts tests/golden/d3_frozen_sha256.txt from the reference's session tests.

crates/graph-core/src/layout/force/session/tests/golden.rs pins, for the gate
model at seeds 0..64 (2 + seed nodes), the sha256 of `layout.force.barnes_hut`'s
output columns as f32 little-endian, all of x then all of y, in node order. This
copies its FROZEN table, one "seed digest" line each.

Run from the repository root with the reference tree present:
python tests/golden/make_d3_golden.py /path/to/reference
"""

import os
import re
import sys


def main(ref_root: str) -> None:
    src = os.path.join(ref_root, "crates", "graph-core", "src", "layout", "force", "session", "tests", "golden.rs")
    text = open(src).read()
    table = text[text.index("FROZEN"):]
    rows = re.findall(r'"([0-9a-f]{64})",\s*// seed (\d+)', table)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "d3_frozen_sha256.txt")
    with open(out, "w") as f:
        f.write("# seed sha256(f32le x ++ f32le y) of layout.force.barnes_hut on the gate model "
                "(reference session/tests/golden.rs FROZEN)\n")
        for digest, seed in rows:
            f.write(f"{seed} {digest}\n")
    print(f"wrote {len(rows)} lines to {out}")


if __name__ == "__main__":
    if len(sys.argv) > 1:
        main(sys.argv[1])
    elif os.environ.get("GRAPH_RENDER_REFERENCE"):
        main(os.environ["GRAPH_RENDER_REFERENCE"])
    else:
        sys.exit(f"usage: python {sys.argv[0]} <reference checkout> (or set GRAPH_RENDER_REFERENCE)")
