"""The benchmark's CPU arm (``bench.py --impl reference``) on a short run: it
prints one JSON line on the GPU arm's metric and config, with a CPU baseline
of kind "port", zero host/device copies, and it loads the CPU oracle but
nothing of the GPU library (the arm runs the same way on a machine with a GPU)."""

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0", "--samples", "40000",
            "--cpu-seconds", "0.3"]
runpy.run_path("bench.py", run_name="__main__")
maps = open("/proc/self/maps").read()
print("MAPS", "libtodgpu" in maps, "libtodoracle" in maps)
"""


def test_reference_arm_line_and_libraries():
    out = subprocess.run([sys.executable, "-c", SCRIPT], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = out.stdout.strip().splitlines()
    line = json.loads(next(ln for ln in lines if ln.startswith("{")))
    maps = next(ln for ln in lines if ln.startswith("MAPS")).split()
    assert maps[1] == "False" and maps[2] == "True"  # no GPU library, the oracle
    assert line["impl"] == "reference" and line["unit"] == "samples/s" and line["higher_is_better"] is True
    assert line["value"] > 0 and line["cpu_baseline"]["kind"] == "port"
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    sys.path.insert(0, ROOT)
    import bench

    class A:
        mode = "bilinear"
        samples = 40000

    assert line["config"] == bench.bench_config(A, line["config"]["S"], 1)
    assert line["config"]["S"] == 1512
