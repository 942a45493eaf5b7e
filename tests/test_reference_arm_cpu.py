"""bench.py --impl reference: the reference's own CPU implementation of the
path (its CPU batching from oracle/_ref when built, else the oracle port, plus
the CPU restatement of its DAG code), timed on the host without the routing
library; its JSON line carries the same `config` as the GPU arm's for the same
workload."""
import json
import os
import subprocess
import sys

from helpers import ROOT

PROBE = """
import runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--workload", "small_64x64x5", "--steps", "2", "--warmup", "1",
            "--cpu-nets", "400"]
runpy.run_path("bench.py", run_name="__main__")
maps = open("/proc/self/maps").read()
print("LOADED", int("libgrb.so" in maps), int("libgrb_synth.so" in maps), int("liboracle.so" in maps))
"""


def test_reference_arm_runs_without_the_routing_library():
    res = subprocess.run([sys.executable, "-c", PROBE], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = res.stdout.strip().splitlines()
    line = json.loads(next(ln for ln in lines if ln.startswith("{")))
    loaded = next(ln for ln in lines if ln.startswith("LOADED")).split()[1:]
    assert loaded[0] == "0", "the reference arm loaded the routing library"
    assert loaded[1] == "1" and loaded[2] == "1"
    assert line["impl"] == "reference" and line["steps"] == 2 and line["warmup"] == 1
    assert line["value"] > 0 and line["unit"] == "nets/s" and line["higher_is_better"] is True
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["cpu_baseline"]["value"] == line["value"] and line["cpu_baseline"]["cores"] >= 1
    sys.path.insert(0, ROOT)
    import bench
    from grotor_b200.synth import WORKLOADS, Design
    d = Design(WORKLOADS["small_64x64x5"])
    assert line["config"] == bench.workload_config("small_64x64x5", d.grid, d.n_subnets, line["config"]["batches"])
    assert line["config"]["batches"] > 0
    if os.path.exists(os.path.join(ROOT, "oracle", "_ref", "ref_harness")):
        assert line["cpu_baseline"]["kind"] == "reference"
