"""bench.py's reference arm, on the CPU: it runs the oracle (the FP64 restatement
of graph-core's tick) on a small case of the workload and maps no library of the
product: the workload is drawn by the copy of the generators linked into the
oracle's own library."""

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBE = r"""
import json, os, sys
sys.argv = ["bench.py", "--impl", "reference", "--steps", "2", "--warmup", "1", "--n", "3000"]
sys.path.insert(0, os.getcwd())
import bench
bench.run_reference(bench.parse(), bench.Dist())
maps = sorted({l.split()[-1] for l in open("/proc/self/maps") if l.rstrip().endswith(".so") and os.getcwd() in l})
print("MAPS " + json.dumps(maps))
"""


def test_reference_arm_runs_the_oracle_and_maps_only_its_library():
    out = subprocess.run([sys.executable, "-c", PROBE], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = out.stdout.strip().splitlines()
    line = json.loads(next(x for x in lines if x.startswith("{")))
    assert line["impl"] == "reference" and line["value"] > 0 and line["steps"] == 2
    assert line["config"]["n"] == 3000 and line["cpu_baseline"]["kind"] == "port"
    assert line["vs_baseline"] is None
    maps = json.loads(next(x for x in lines if x.startswith("MAPS "))[5:])
    assert maps and all(m.startswith(os.path.join(ROOT, "oracle") + os.sep) for m in maps), maps
