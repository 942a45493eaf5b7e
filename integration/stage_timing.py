"""The reference router's default pipeline (stage one: L-shape; rip-up; stage
two: FLT) run end to end twice on the same CAP/NET -- the stock program
(oracle/_ref/grotor, the reference's own src/main.cu, CPU batching) and the
drop-in (integration/_build/grotor_grb: the same program with its routing hot
path on grotor_b200) -- with each program's own stage records, wall time,
.out agreement and the reference evaluator's scores.  Needs a GPU and both
programs built (oracle/ref.mk, integration/Makefile).

Records: BATCH_TIMING / DAG_TIMING per stage (the reference's stage metric is
batching ms + DAG ms), TOPOLOGY_TIMING (stage one: FLUTE and the nets'
topology; the stock program's also covers its host geometry and DFS),
GROTOR_COMPLETE (wall seconds of the whole program, reading and writing
included), OUTPUT_TIMING (the device .out writer: formatting, and the time
the pipeline waited for the file); from one more run, FLT_TRAFFIC (the FLT
stage's algorithmic bytes, grb_flt_traffic) and from it each executor's FLT
stage roofline.

Usage:  python integration/stage_timing.py [--workloads medium_320x320x10,large_800x800x10]
                                           [--executors persistent,plain] [--out FILE]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
REF_DIR = os.path.join(ROOT, "oracle", "_ref")
STOCK = os.path.join(REF_DIR, "grotor")
DRIVER = os.path.join(HERE, "_build", "grotor_grb")
EVALUATOR = os.path.join(REF_DIR, "evaluator")


def records(text: str) -> dict:
    """Stage records of one run: {'lshape': {...}, 'detour': {...}, ...}."""
    out = {"lshape": {}, "detour": {}}
    batch_stage = "lshape"
    for line in text.splitlines():
        tag, _, rest = line.partition(" ")
        if tag not in ("BATCH_TIMING", "DAG_TIMING", "TOPOLOGY_TIMING", "GROTOR_COMPLETE", "PIPELINE_TIMING",
                       "FLT_TRAFFIC", "OUTPUT_TIMING"):
            continue
        kv = dict(p.split("=", 1) for p in rest.split() if "=" in p)
        if tag == "OUTPUT_TIMING":
            out["output"] = {k: float(v) for k, v in kv.items() if k != "executor"}
        elif tag == "FLT_TRAFFIC":
            out["detour"]["algorithmic_bytes"] = {k: float(v) for k, v in kv.items()}
        elif tag == "GROTOR_COMPLETE":
            out["wall_s"] = float(kv["wall_seconds"])
        elif tag == "PIPELINE_TIMING":
            out["pipeline"] = {k: float(v) for k, v in kv.items()}
        elif tag == "BATCH_TIMING":
            # The stock program prints one record per batching call, stage one first.
            stage = kv.get("stage", batch_stage)
            out[stage]["batching_ms"] = float(kv["elapsed_ms"])
            out[stage]["nets"] = int(kv["nets"])
            out[stage]["batches"] = int(kv["batches"])
            batch_stage = "detour"
        elif tag == "DAG_TIMING" and kv.get("batch_index") == "-1":
            out[kv["stage"]]["dag_ms"] = float(kv["elapsed_ms"])
        elif tag == "TOPOLOGY_TIMING":
            out[kv["stage"] if kv["stage"] in out else "detour"]["topology_ms"] = float(kv["elapsed_ms"])
    for st in ("lshape", "detour"):
        r = out[st]
        if "batching_ms" in r and "dag_ms" in r:
            r["stage_ms"] = r["batching_ms"] + r["dag_ms"]
    return out


def flt_roofline(d: dict, algorithmic_bytes: dict) -> dict:
    """Roofline of the FLT stage (refresh + layer-change tables + DAG solve +
    commit; one launch in the persistent form): the model's bytes over the
    stage's device time."""
    peak, kind = measured_peak()
    ach = sum(algorithmic_bytes.values()) / (d["dag_ms"] / 1e3) / 1e9
    return {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
            "peak_source": f"{kind} hbm_gbs", "algorithmic_bytes": algorithmic_bytes}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def parse_out(path):
    nets, name, segs = [], None, None
    for line in open(path):
        line = line.rstrip("\n")
        if name is None:
            name = line
        elif line == "(":
            segs = []
        elif line == ")":
            nets.append((name, segs))
            name, segs = None, None
        else:
            segs.append(line)
    return nets


def scores(cap, net, out):
    res = subprocess.run([EVALUATOR, cap, net, out], capture_output=True, text=True)
    keep = ("overflow cost", "open nets", "incompleted nets", "wirelength cost", "via cost", "total cost")
    return [ln.strip() for ln in (res.stdout + res.stderr).splitlines()
            if any(k in ln for k in keep) and "time" not in ln.lower()]


def run(cmd):
    t = time.perf_counter()
    res = subprocess.run(cmd, capture_output=True, text=True, timeout=3600)
    if res.returncode:
        raise RuntimeError(f"{os.path.basename(cmd[0])} failed ({res.returncode}): {res.stderr[-2000:]}")
    return res.stdout, time.perf_counter() - t


def measure(workload, executors, log):
    from grotor_b200.synth import WORKLOADS, Design
    with tempfile.TemporaryDirectory() as w:
        cap, net = os.path.join(w, "d.cap"), os.path.join(w, "d.net")
        Design(WORKLOADS[workload]).write(cap, net)
        ref_out = os.path.join(w, "ref.out")
        text, t = run([STOCK, "-cap", cap, "-net", net, "-out", ref_out, "--lut-dir", REF_DIR, "--report-score", "0",
                       "--profile-stages", "1"])
        res = {"workload": workload, "reference": dict(records(text), process_s=t)}
        log(f"{workload}: stock reference in {t:.1f} s")
        ref_nets = parse_out(ref_out)
        ref_scores = scores(cap, net, ref_out)
        res["reference"]["scores"] = ref_scores
        for ex in executors:
            mine = os.path.join(w, f"{ex}.out")
            text, t = run([DRIVER, "-cap", cap, "-net", net, "-out", mine, "--lut-dir", REF_DIR, "--executor", ex])
            log(f"{workload}: drop-in ({ex}) in {t:.1f} s")
            got = parse_out(mine)
            same_order = [a for a, _ in ref_nets] == [b for b, _ in got]
            same_sets = same_order and all(sorted(a) == sorted(b) for (_, a), (_, b) in zip(ref_nets, got))
            sc = scores(cap, net, mine)
            r = dict(records(text), process_s=t, net_order_equal=same_order, segments_equal=same_sets,
                     scores_equal=sc == ref_scores)
            res[f"grotor_b200_{ex}"] = r
        # The byte model runs on the host after the stage: a separate run, so
        # that its time is in no timed record above.
        text, _ = run([DRIVER, "-cap", cap, "-net", net, "-out", os.devnull, "--lut-dir", REF_DIR, "--executor",
                       executors[0], "--report-traffic", "1"])
        model = records(text)["detour"].get("algorithmic_bytes")
        for ex in executors:
            d = res[f"grotor_b200_{ex}"]["detour"]
            if model and d.get("dag_ms"):
                d["roofline"] = flt_roofline(d, model)
        return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workloads", default="medium_320x320x10,large_800x800x10")
    ap.add_argument("--executors", default="persistent,plain")
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    for f in (STOCK, DRIVER, EVALUATOR):
        if not os.path.exists(f):
            sys.exit(f"{f} is not built (oracle/ref.mk, integration/Makefile)")

    def log(*a):
        print(*a, file=sys.stderr, flush=True)

    results = [measure(wl, args.executors.split(","), log) for wl in args.workloads.split(",")]
    text = json.dumps(results, indent=1)
    print(text)
    if args.out:
        with open(args.out, "w") as f:
            f.write(text)


if __name__ == "__main__":
    main()
