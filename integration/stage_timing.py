"""The reference router's pipelines run end to end twice on the same CAP/NET
-- the stock program (oracle/_ref: the reference's own src/main.cu built as
grotor, grotor_ggr and grotor_cugr2) and the drop-in (integration/_build: the
same program with its routing hot path on grotor_b200) -- with each program's
own stage records, wall time, .out agreement and the reference evaluator's
scores.  Needs a GPU and the programs built (oracle/ref.mk,
integration/Makefile).

Pipelines: "default" (stage one: L-shape; rip-up; stage two: FLT),
"ggr" (first-fit groups, bounding-box batches, Z-shape stage, the host
post-processing) and "cugr2" (L-shape, rip-up, FLT detour, the maze stage
with its score gate).

Records: BATCH_TIMING / DAG_TIMING per stage (the reference's stage metric is
batching ms + DAG ms), TOPOLOGY_TIMING (stage one: FLUTE and the nets'
topology; the stock program's also covers its host geometry and DFS),
MAZE_PHASE_TIMING / MAZE_SEARCH (the maze stage, host search included),
PIPELINE_TIMING (the stock program's phases) / DROPIN_TIMING (the drop-in's
phases, from program start),
GROTOR_COMPLETE (wall seconds of the whole program, reading and writing
included), OUTPUT_TIMING (the device .out writer: formatting, and the time
the pipeline waited for the file); from one more run of the default
pipeline, FLT_TRAFFIC (the FLT stage's algorithmic bytes, grb_flt_traffic)
and from it each executor's FLT stage roofline.

Usage:  python integration/stage_timing.py [--workloads medium_320x320x10,large_800x800x10]
                                           [--pipelines default,ggr,cugr2]
                                           [--executors persistent,plain] [--repeat R] [--out FILE]
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
EVALUATOR = os.path.join(REF_DIR, "evaluator")
# pipeline -> (stock program, drop-in driver, stages in the order their
# records appear when a program prints no ROUTING_STAGE_BEGIN)
PIPELINES = {
    "default": (os.path.join(REF_DIR, "grotor"), os.path.join(HERE, "_build", "grotor_grb"), ("lshape", "detour")),
    "ggr": (os.path.join(REF_DIR, "grotor_ggr"), os.path.join(HERE, "_build", "grotor_grb_ggr"), ("zshape",)),
    "cugr2": (os.path.join(REF_DIR, "grotor_cugr2"), os.path.join(HERE, "_build", "grotor_grb_cugr2"),
              ("lshape", "detour", "maze")),
}


def records(text: str, stages=("lshape", "detour")) -> dict:
    """Stage records of one run: {'lshape': {...}, 'detour': {...}, ...}.  A
    record is filed under the stage it names, else under the stage the last
    ROUTING_STAGE_BEGIN opened, else under the next stage of `stages` (the
    default program prints one BATCH_TIMING per batching call, stage one
    first)."""
    out = {st: {} for st in stages}
    pending = list(stages)
    current = None
    for line in text.splitlines():
        tag, _, rest = line.partition(" ")
        if tag not in ("BATCH_TIMING", "DAG_TIMING", "TOPOLOGY_TIMING", "GROTOR_COMPLETE", "PIPELINE_TIMING",
                       "FLT_TRAFFIC", "OUTPUT_TIMING", "DROPIN_TIMING", "ROUTING_STAGE_BEGIN", "MAZE_PHASE_TIMING",
                       "MAZE_SEARCH", "MAZE_QUALITY_GATE"):
            continue
        kv = dict(p.split("=", 1) for p in rest.split() if "=" in p)
        if tag == "ROUTING_STAGE_BEGIN":
            current = kv["stage"]
            out.setdefault(current, {})["stage_nets"] = int(kv["nets"])
        elif tag == "OUTPUT_TIMING":
            out["output"] = {k: float(v) for k, v in kv.items() if k != "executor"}
        elif tag == "FLT_TRAFFIC":
            out["detour"]["algorithmic_bytes"] = {k: float(v) for k, v in kv.items()}
        elif tag == "GROTOR_COMPLETE":
            out["wall_s"] = float(kv["wall_seconds"])
        elif tag in ("PIPELINE_TIMING", "DROPIN_TIMING"):
            out["pipeline"] = {k: float(v) for k, v in kv.items()}
        elif tag == "MAZE_PHASE_TIMING":
            out.setdefault("maze", {})["phase_ms"] = float(kv["elapsed_ms"])
        elif tag == "MAZE_SEARCH":
            out.setdefault("maze", {})["search_ms"] = float(kv["elapsed_ms"])
        elif tag == "MAZE_QUALITY_GATE":
            out.setdefault("maze", {})["accepted"] = int(kv["accepted"])
        elif tag == "BATCH_TIMING":
            stage = kv.get("stage") or current or (pending[0] if pending else "other")
            if stage in pending:
                pending.remove(stage)
            r = out.setdefault(stage, {})
            r["batching_ms"] = float(kv["elapsed_ms"])
            r["nets"] = int(kv["nets"])
            r["batches"] = int(kv["batches"])
        elif tag == "DAG_TIMING" and kv.get("batch_index") == "-1":
            out.setdefault(kv["stage"], {})["dag_ms"] = float(kv["elapsed_ms"])
        elif tag == "TOPOLOGY_TIMING":
            stage = kv["stage"] if kv["stage"] in out else ("detour" if "detour" in out else kv["stage"])
            out.setdefault(stage, {})["topology_ms"] = float(kv["elapsed_ms"])
    for r in out.values():
        if isinstance(r, dict) and "batching_ms" in r and "dag_ms" in r:
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


def median_run(runs):
    """The run with the median wall time, with every run's wall time."""
    runs = sorted(runs, key=lambda r: r.get("wall_s", r["process_s"]))
    pick = dict(runs[(len(runs) - 1) // 2])
    pick["wall_s_runs"] = [r.get("wall_s") for r in runs]
    return pick


def measure_pipeline(pipeline, cap, net, w, executors, log, repeat=1):
    """The stock program and the drop-in in each executor, `repeat` times in
    turn; each program's record is its median-wall run.  Outputs are compared
    on the first run."""
    stock, driver, stages = PIPELINES[pipeline]
    ref_out = os.path.join(w, f"{pipeline}_ref.out")
    runs = {"reference": []}
    runs.update({ex: [] for ex in executors})
    res = {"pipeline": pipeline}
    for rep in range(repeat):
        text, t = run([stock, "-cap", cap, "-net", net, "-out", ref_out, "--lut-dir", REF_DIR, "--report-score", "0",
                       "--profile-stages", "1"])
        runs["reference"].append(dict(records(text, stages), process_s=t))
        log(f"{pipeline}: stock reference in {t:.1f} s")
        if rep == 0:
            ref_nets = parse_out(ref_out)
            ref_bytes = open(ref_out, "rb").read()
            ref_scores = scores(cap, net, ref_out)
        for ex in executors:
            mine = os.path.join(w, f"{pipeline}_{ex}.out")
            text, t = run([driver, "-cap", cap, "-net", net, "-out", mine, "--lut-dir", REF_DIR, "--executor", ex])
            log(f"{pipeline}: drop-in ({ex}) in {t:.1f} s")
            r = dict(records(text, stages), process_s=t)
            if rep == 0:
                got = parse_out(mine)
                same_order = [a for a, _ in ref_nets] == [b for b, _ in got]
                same_sets = same_order and all(sorted(a) == sorted(b) for (_, a), (_, b) in zip(ref_nets, got))
                sc = scores(cap, net, mine)
                res[f"{ex}_equal"] = dict(net_order_equal=same_order, segments_equal=same_sets,
                                          bytes_equal=open(mine, "rb").read() == ref_bytes,
                                          scores_equal=sc == ref_scores)
            runs[ex].append(r)
    res["reference"] = dict(median_run(runs["reference"]), scores=ref_scores)
    for ex in executors:
        res[f"grotor_b200_{ex}"] = dict(median_run(runs[ex]), **res.pop(f"{ex}_equal"))
    if pipeline == "default":
        # The byte model runs on the host after the stage: a separate run, so
        # that its time is in no timed record above.
        text, _ = run([driver, "-cap", cap, "-net", net, "-out", os.devnull, "--lut-dir", REF_DIR, "--executor",
                       executors[0], "--report-traffic", "1"])
        model = records(text, stages)["detour"].get("algorithmic_bytes")
        for ex in executors:
            d = res[f"grotor_b200_{ex}"]["detour"]
            if model and d.get("dag_ms"):
                d["roofline"] = flt_roofline(d, model)
    return res


def measure(workload, pipelines, executors, log, repeat=1):
    from grotor_b200.synth import WORKLOADS, Design
    with tempfile.TemporaryDirectory() as w:
        cap, net = os.path.join(w, "d.cap"), os.path.join(w, "d.net")
        Design(WORKLOADS[workload]).write(cap, net)
        out = []
        for p in pipelines:
            r = measure_pipeline(p, cap, net, w, executors, lambda *a: log(f"{workload}:", *a), repeat)
            out.append(dict(workload=workload, **r))
        return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workloads", default="medium_320x320x10,large_800x800x10")
    ap.add_argument("--pipelines", default="default")
    ap.add_argument("--executors", default="persistent,plain")
    ap.add_argument("--repeat", type=int, default=1, help="runs of each program, in turn (median wall kept)")
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    pipelines = args.pipelines.split(",")
    for p in pipelines:
        for f in PIPELINES[p][:2] + (EVALUATOR,):
            if not os.path.exists(f):
                sys.exit(f"{f} is not built (oracle/ref.mk, integration/Makefile)")

    def log(*a):
        print(*a, file=sys.stderr, flush=True)

    results = [r for wl in args.workloads.split(",")
               for r in measure(wl, pipelines, args.executors.split(","), log, args.repeat)]
    text = json.dumps(results, indent=1)
    print(text)
    if args.out:
        with open(args.out, "w") as f:
            f.write(text)


if __name__ == "__main__":
    main()
