"""Generate the golden fixtures in this folder from the reference router itself.

Each fixture is a seeded synthetic design written as CAP/NET files and run
through ``oracle/_ref/ref_harness`` (the reference's own code, built from its
sources by ``oracle/ref.mk``):

* ``topo`` (CPU): subnets, FLUTE trees in the reference's DFS order, batching
  geometry, HPWL order and the reference CPU first-fit batches, grid tables;
* ``route`` and ``snap`` (GPU): routes, demand and statistics of the reference
  L-shape stage, cost tables after the stage, the .out file (SHA-256 and
  evaluator scores), and the cost tables before / routes after one batch;
* ``zshape`` (GPU, Z-shape fixtures, reference GGR build ``ref_harness_ggr``):
  the reference Z-shape pipeline -- order, first-fit groups, bbox batches,
  encoded trees and net boxes, routes, demand and statistics after the stage;
* ``flt`` (GPU, FLT fixtures): the reference default pipeline through its FLT
  stage -- demand and statistics before the stage, the rip-up set, the DAGs of
  the reference's host FLT builder, the FLT batching geometry and batches, and
  phase-two routes, demand and statistics after the stage.

Usage:  python tests/golden/make_golden.py --topo      (no GPU needed)
        python tests/golden/make_golden.py --route     (on a GPU box)
        python tests/golden/make_golden.py --flt       (on a GPU box)
        python tests/golden/make_golden.py --zshape    (on a GPU box)
The two passes update the same ``<name>.npz``.
"""
from __future__ import annotations

import argparse
import hashlib
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

REF = os.path.join(ROOT, "oracle", "_ref")
HARNESS = os.path.join(REF, "ref_harness")
EVALUATOR = os.path.join(REF, "evaluator")

# name -> (workload, overrides)
FIXTURES = {
    "ref_64x64x10_2k": ("small_64x64x5", dict(n_nets=2000, cap_layers=10, seed=11)),
    "ref_32x32x10_400": ("small_64x64x5", dict(n_nets=400, cap_layers=10, seed=12, X=32, Y=32)),
    # congested (capacity 1..4) so that the L-shape stage leaves overflow nets for FLT
    "ref_flt_48x48x10_1500": ("small_64x64x5", dict(n_nets=1500, cap_layers=10, seed=13, X=48, Y=48, cap_lo=1,
                                                    cap_hi=4)),
}
FLT_FIXTURES = {"ref_flt_48x48x10_1500"}
FIXTURES["ref_z_48x48x10_1500"] = FIXTURES["ref_flt_48x48x10_1500"]
FIXTURES["ref_z_40x56x10_800"] = ("small_64x64x5", dict(n_nets=800, cap_layers=10, seed=14, X=40, Y=56))
Z_FIXTURES = {"ref_z_48x48x10_1500", "ref_z_40x56x10_800"}
HARNESS_GGR = os.path.join(REF, "ref_harness_ggr")
TOPO_KEYS = ["meta", "short_costs", "unit_costs", "x_edge_len", "y_edge_len", "capacity", "pin_acc_num",
             "node_off", "nodes", "parents", "point_off", "points", "hseg_off", "hsegs", "vseg_off", "vsegs",
             "hpwl", "original", "pin_count", "order", "batch_of", "ids", "batch_off", "pin_vias",
             "rsmt_pos", "rsmt_adj_off", "rsmt_adj"]
EXT = {"i32": np.int32, "i64": np.int64, "f32": np.float32, "f64": np.float64}


def design_files(name: str, workdir: str):
    from dataclasses import replace

    from grotor_b200.synth import WORKLOADS, Design
    wl, over = FIXTURES[name]
    params = replace(WORKLOADS[wl], **over)
    d = Design(params)
    cap, net = os.path.join(workdir, "d.cap"), os.path.join(workdir, "d.net")
    d.write(cap, net)
    return cap, net


def read_dir(d: str, keys=None):
    out = {}
    for f in os.listdir(d):
        base, _, ext = f.rpartition(".")
        if ext in EXT and (keys is None or base in keys):
            out[base] = np.fromfile(os.path.join(d, f), dtype=EXT[ext])
    return out


def evaluate(cap, net, out):
    r = subprocess.run([EVALUATOR, cap, net, out], capture_output=True, text=True)
    return r.stdout + r.stderr


def parse_scores(text: str) -> dict:
    """Evaluator summary lines (wirelength, via and overflow costs, total)."""
    keys = {}
    for line in text.splitlines():
        low = line.lower()
        for k in ("wirelength cost", "via cost", "overflow cost", "total cost", "open nets", "incomplete"):
            if k in low and ":" in line:
                keys[k] = line.split(":", 1)[1].strip()
    return keys


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--topo", action="store_true")
    ap.add_argument("--route", action="store_true")
    ap.add_argument("--flt", action="store_true")
    ap.add_argument("--zshape", action="store_true")
    ap.add_argument("--only", default=None)
    ap.add_argument("--outdir", default=HERE, help="where to write the .npz files")
    ap.add_argument("--keep-out", action="store_true", help="also copy the reference .out into --outdir")
    args = ap.parse_args()
    for name in FIXTURES:
        if args.only and name != args.only:
            continue
        src = os.path.join(HERE, name + ".npz")
        path = os.path.join(args.outdir, name + ".npz")
        data = dict(np.load(src)) if os.path.exists(src) else {}
        with tempfile.TemporaryDirectory() as w:
            cap, net = design_files(name, w)
            if args.topo and name not in Z_FIXTURES:
                subprocess.run([HARNESS, "topo", cap, net, w, REF], check=True, stdout=subprocess.DEVNULL)
                data.update(read_dir(w, TOPO_KEYS))
            if args.zshape and name in Z_FIXTURES:
                subprocess.run([HARNESS_GGR, "zshape", cap, net, w, REF], check=True, stdout=subprocess.DEVNULL)
                got = read_dir(w)
                data.update({k: v for k, v in got.items()
                             if k.startswith("z_") or k in ("meta", "short_costs", "unit_costs", "x_edge_len",
                                                            "y_edge_len", "capacity", "pin_acc_num", "pin_vias")})
            if args.flt and name in FLT_FIXTURES:
                subprocess.run([HARNESS, "flt", cap, net, w, REF], check=True, stdout=subprocess.DEVNULL)
                got = read_dir(w)
                data.update({k: v for k, v in got.items() if k.startswith("flt_")})
            if args.route and name not in FLT_FIXTURES and name not in Z_FIXTURES:
                for k in TOPO_KEYS:  # the GPU passes read the committed plan
                    if k in data:
                        data[k].tofile(os.path.join(w, f"{k}.{_ext(data[k])}"))
                out = os.path.join(w, "ref.out")
                subprocess.run([HARNESS, "route", cap, net, w, REF, out], check=True, stdout=subprocess.DEVNULL)
                nb = len(data["batch_off"]) - 1
                subprocess.run([HARNESS, "snap", cap, net, w, REF, str(nb - 1)], check=True, stdout=subprocess.DEVNULL)
                got = read_dir(w)
                for k in ("ref_routes", "ref_demand", "ref_stats", "ref_wcost", "ref_vcost", "ref_presum",
                          "snap_wcost", "snap_vcost", "snap_presum", "snap_demand", "snap_routes", "snap_batch"):
                    data[k] = got[k]
                if name != "ref_32x32x10_400":  # tables only for the small grid
                    for k in ("ref_wcost", "ref_vcost", "ref_presum", "snap_wcost", "snap_vcost", "snap_presum",
                              "snap_demand"):
                        data.pop(k)
                blob = open(out, "rb").read()
                if args.keep_out:
                    with open(os.path.join(args.outdir, name + ".ref.out"), "wb") as f:
                        f.write(blob)
                data["ref_out_sha256"] = np.frombuffer(hashlib.sha256(blob).digest(), np.uint8)
                data["ref_out_bytes"] = np.array([len(blob)], np.int64)
                scores = evaluate(cap, net, out)
                data["ref_eval_text"] = np.frombuffer(scores.encode(), np.uint8)
        np.savez_compressed(path, **data)
        print(name, sorted(data))


def _ext(a):
    return {np.dtype(np.int32): "i32", np.dtype(np.int64): "i64", np.dtype(np.float32): "f32",
            np.dtype(np.float64): "f64"}[a.dtype]


if __name__ == "__main__":
    main()
