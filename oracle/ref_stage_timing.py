"""Times the reference router's own GPU L-shape stage against this library's,
on the same B200, the same topology and the same plan, and checks that the
routes are identical.  TEST INFRASTRUCTURE (runs the reference's code built
from its sources into oracle/_ref/ by oracle/ref.mk; needs a GPU).

Per workload (a seeded synthetic design written as CAP/NET files):
  1. ``ref_harness topo`` (CPU): the reference's subnets, FLUTE trees, HPWL
     order and CPU first-fit batches, dumped;
  2. ``ref_harness route`` (GPU): the reference's L-shape stage
     (Lshape_route, lshape.cuh:21-197) -- its BATCH_TIMING and DAG_TIMING
     records (router_state.hpp:238-265, generate_batches.hpp:14-26) and its
     routes, demand and statistics;
  3. this library on the dumped topology: GPU first-fit batching of the same
     order (persistent executor), then the stage on the reference's plan in the
     persistent and plain executors, timed with CUDA events on its stream; the
     batches, routes, demand and statistics are compared with the reference's.

Usage:  python oracle/ref_stage_timing.py [--workloads medium_320x320x10,large_800x800x10]
                                          [--out gpurun_out/ref_stage_timing.json] [--reps 3]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
HARNESS = os.path.join(HERE, "_ref", "ref_harness")
ROUTE_PER_PIN = 12  # router_state.hpp:31
EXT = {"i32": np.int32, "i64": np.int64, "f32": np.float32, "f64": np.float64}


def read_dir(d, keys=None):
    out = {}
    for f in os.listdir(d):
        base, _, e = f.rpartition(".")
        if e in EXT and (keys is None or base in keys):
            out[base] = np.fromfile(os.path.join(d, f), dtype=EXT[e])
    return out


def records(text, tag):
    """KEY=VALUE fields of every `tag` line the reference printed."""
    out = []
    for line in text.splitlines():
        if line.startswith(tag + " "):
            out.append(dict(kv.split("=", 1) for kv in line.split()[1:] if "=" in kv))
    return out


def run(cmd, **kw):
    t = time.perf_counter()
    res = subprocess.run(cmd, capture_output=True, text=True, **kw)
    if res.returncode:
        raise RuntimeError(f"{cmd[:2]} failed ({res.returncode}): {res.stderr[-2000:]}")
    return res.stdout, time.perf_counter() - t


def measure(workload, reps, log):
    import torch

    from grotor_b200 import GridArrays, NetArrays, Router
    from grotor_b200.synth import WORKLOADS, Design
    out = {"workload": workload}
    with tempfile.TemporaryDirectory() as w:
        cap, net = os.path.join(w, "d.cap"), os.path.join(w, "d.net")
        Design(WORKLOADS[workload]).write(cap, net)
        lut = os.path.dirname(HARNESS)
        _, t_topo = run([HARNESS, "topo", cap, net, w, lut])
        log(f"{workload}: reference topology and CPU batches in {t_topo:.1f} s")
        text, t_route = run([HARNESS, "route", cap, net, w, lut, os.devnull])
        log(f"{workload}: reference route run in {t_route:.1f} s")
        bt, dt = records(text, "BATCH_TIMING"), records(text, "DAG_TIMING")
        out["reference"] = {"batching_ms": float(bt[-1]["elapsed_ms"]), "batching_backend": bt[-1].get("backend"),
                            "dag_ms": float(dt[-1]["elapsed_ms"]), "nets": int(dt[-1]["nets"]),
                            "batches": int(dt[-1]["batches"]),
                            "timing_source": "BATCH_TIMING / DAG_TIMING records of its own run (host clock "
                                             "between device synchronisations)"}
        g = read_dir(w)
    L, X, Y, DIR = (int(v) for v in g["meta"])
    uw, uv = (float(v) for v in g["unit_costs"])
    grid = GridArrays(L, X, Y, DIR, uw, uv, g["short_costs"], g["x_edge_len"], g["y_edge_len"], g["capacity"])
    nets = NetArrays(g["node_off"], g["nodes"], g["parents"], g["pin_acc_num"].astype(np.int64) * ROUTE_PER_PIN,
                     g["point_off"], g["points"], g["hseg_off"], g["hsegs"], g["vseg_off"], g["vsegs"])
    r = Router(grid)
    r.upload_nets(nets)
    stream = torch.cuda.ExternalStream(r.stream_handle)

    def timed(fn):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        res = fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b), res

    bo, nb = r.generate_batches_rsmt(g["order"], 1000000, 1, "persistent")
    mine = {"batches_equal_reference": bool(nb == len(g["batch_off"]) - 1 and np.array_equal(bo, g["batch_of"]))}
    bms = [timed(lambda: r.generate_batches_rsmt(g["order"], 1000000, 1, "persistent"))[0] for _ in range(reps)]
    mine["batching_ms"] = float(np.median(bms))
    want_routes = g["ref_routes"][:-1]
    want_demand = (g["ref_demand"].astype(np.float64) * 2).astype(np.int32)
    for mode in ("persistent", "plain"):
        ms = []
        for k in range(reps + 1):
            r.reset()
            r.set_plan(g["ids"], g["batch_off"])
            r.set_stats(0.0, int(g["pin_vias"][0]))
            t, st = timed(lambda: r.lshape_route(mode))
            if k:
                ms.append(t)
        same = (np.array_equal(r.read_routes(), want_routes)
                and np.array_equal(r.read_tables()["demand_half"], want_demand)
                and st["wirelength"] == g["ref_stats"][0] and st["vias"] == int(g["ref_stats"][1]))
        mine[mode] = {"dag_ms": float(np.median(ms)), "routes_demand_stats_equal_reference": bool(same)}
    r.close()
    out["grotor_b200"] = mine
    ref = out["reference"]
    out["speedup"] = {
        "dag_persistent": ref["dag_ms"] / mine["persistent"]["dag_ms"],
        "dag_plain": ref["dag_ms"] / mine["plain"]["dag_ms"],
        "batching": ref["batching_ms"] / mine["batching_ms"],
        "stage": (ref["batching_ms"] + ref["dag_ms"]) / (mine["batching_ms"] + mine["persistent"]["dag_ms"]),
    }
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workloads", default="medium_320x320x10,large_800x800x10")
    ap.add_argument("--out", default=None)
    ap.add_argument("--reps", type=int, default=3)
    args = ap.parse_args()
    if not os.path.exists(HARNESS):
        sys.exit("oracle/_ref/ref_harness is not built (make -C oracle -f ref.mk REF=...)")

    def log(*a):
        print(*a, file=sys.stderr, flush=True)

    results = [measure(wl, args.reps, log) for wl in args.workloads.split(",")]
    text = json.dumps(results, indent=1)
    print(text)
    if args.out:
        with open(args.out, "w") as f:
            f.write(text)


if __name__ == "__main__":
    main()
