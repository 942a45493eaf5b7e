#!/usr/bin/env python
"""bench.py -- stage throughput of GRotor's routing hot path on B200.

One step is one L-shape routing stage over a whole synthetic design already
resident in HBM: exact first-fit batching on the GPU, then for every batch the
incremental cost / prefix refresh, the L-shape DP with layer assignment and the
demand commit -- in the persistent batched executor (one cooperative kernel per
part).  ``value`` = nets routed per second (batching + DAG, the reference's
stage-runtime definition, README.md:139).  The plain per-batch-launch form and
the CUDA-graph form run on the same GPU afterwards for the comparison the
metric names, and their routes are checked identical.

After the timed region, on rank 0 of a single-GPU run, the CPU leg runs the
reference's own CPU first-fit batching (built from its sources into
oracle/_ref/) on the whole order and the CPU restatement of its DAG code on the
whole plan (all host cores): their time is ``cpu_baseline``, and their results
are the checker of the GPU's -- ``parity`` records that the GPU's batches
equal the reference's and that every route word, the demand, the timestamps
and the statistics equal the restatement's (which evaluates the cost model's
exponential through the device's own values, grb_cost_exp, so its costs are
bit-identical).

``--impl reference`` times the reference's own CPU implementation of the path
on the host cores instead (the same two programs) on a bounded stride sample
of the same workload per step, plus one run of the reference's batching over
the whole order; it never loads the routing library (the workload generator is
a library of its own).

Multi-GPU: the path does not shard (batches depend on each other through
demand), so ``--gpus N`` runs N independent replicas (seed + rank); timing is
the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "stage runtime & nets/s on 1 B200: persistent batched vs plain, evaluator-exact"
WORKLOAD = "persistent_1600x1600x10"
BATCH_LIMIT = 1000000  # lshape.cuh:62,69
UNIT = "nets/s"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="grotor", choices=["grotor", "reference"])
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--no-compare", action="store_true", help="skip the plain / graph executor comparison")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--cpu-nets", type=int, default=0,
                    help="nets per step of --impl reference (a stride sample; 0: 30,000)")
    ap.add_argument("--no-tune", action="store_true", help="skip grb_autotune (default launch shapes)")
    ap.add_argument("--executor", default="persistent", choices=["persistent", "plain", "graph"],
                    help="executor of the timed step (the headline is the persistent one)")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the Z-shape and soft-min stage measurements (other workloads)")
    return ap.parse_args()


# --------------------------------------------------------------------------- helpers
class Clocks:
    """Samples SM clock, power and throttle reasons with nvidia-smi while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.dev), "-lms", "200"], stdout=open(self.path, "w"),
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(kernel: str, workload: str):
    """DRAM bytes per launch of `kernel` on `workload` from the committed ncu
    summaries (a line 'dram_bytes_per_launch <kernel> <workload> <bytes>'), else None."""
    d = os.path.join(ROOT, "profiles")
    if not os.path.isdir(d):
        return None
    for f in sorted(os.listdir(d)):
        if not f.endswith(".md"):
            continue
        for line in open(os.path.join(d, f)):
            parts = line.strip().strip("`").split()
            if len(parts) == 4 and parts[0] == "dram_bytes_per_launch" and parts[1] == kernel \
                    and parts[2] == workload:
                return float(parts[3])
    return None


def dist_init(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
        pg = dist
    return rank, world, local, pg


def max_over_ranks(pg, value: float, device: str = "cuda") -> float:
    """Slowest rank's time (every rank calls this with its own value)."""
    if pg is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def replica_params(workload: str, rank: int):
    """Rank r routes an independent replica of the workload (seed + 1000 r)."""
    from dataclasses import replace

    from grotor_b200.synth import WORKLOADS
    base = WORKLOADS[workload]
    return replace(base, seed=base.seed + 1000 * rank)


def barrier(pg):
    if pg is not None:
        import torch
        pg.barrier()
        torch.cuda.synchronize()


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def workload_config(name, grid, n_nets, n_batches):
    """The `config` of both arms' JSON lines (identical for the same workload)."""
    return {"workload": name, "grid": [grid.X, grid.Y, grid.L + 1], "nets": int(n_nets), "batches": int(n_batches),
            "batch_limit": BATCH_LIMIT,
            "l2": "inputs larger than L2 (cost/prefix/demand tables %.0f MB)" % (grid.cells * 32 / 1e6)}


def ref_batching(grid, order, geom):
    """The reference's own CPU first-fit batching (oracle/_ref/ref_harness,
    generate_batches_rsmt on one core) over `order`; returns (batch_of per
    order position, milliseconds it reports), or None when not built."""
    harness = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    if not os.path.exists(harness):
        return None
    with tempfile.TemporaryDirectory() as w:
        np.array([grid.L, grid.X, grid.Y, grid.DIR], np.int32).tofile(os.path.join(w, "meta.i32"))
        np.asarray(order, np.int32).tofile(os.path.join(w, "order.i32"))
        for name in ("point_off", "points", "hseg_off", "hsegs", "vseg_off", "vsegs"):
            np.asarray(getattr(geom, name), np.int32).tofile(os.path.join(w, f"{name}.i32"))
        res = subprocess.run([harness, "batch", w, str(BATCH_LIMIT), "1"], capture_output=True, text=True,
                             check=True)
        ms = float(res.stdout.split("elapsed_ms=")[1].split()[0])
        return np.fromfile(os.path.join(w, "ref_batch_of.i32"), np.int32), ms


def stride_sample(design, target):
    """Every k-th net of the stage order (sizes representative of the design)."""
    order = design.order
    k = max(1, len(order) // max(target, 1))
    return order[::k][:target]


def sub_nets(design, ids):
    """Topology and geometry of a subset of nets, re-indexed 0..m-1."""
    from grotor_b200.router import NetArrays
    n = design.nets

    def csr(off, data, width=1):
        counts = off[ids + 1] - off[ids]
        new_off = np.zeros(len(ids) + 1, np.int64)
        np.cumsum(counts, out=new_off[1:])
        idx = np.concatenate([np.arange(off[i], off[i + 1]) for i in ids]) if len(ids) else np.zeros(0, np.int64)
        if width == 1:
            return new_off.astype(np.int32), data[idx]
        return new_off.astype(np.int32), data.reshape(-1, width)[idx].reshape(-1)

    no, nodes = csr(n.node_off, n.nodes)
    _, parents = csr(n.node_off, n.parents)
    po, points = csr(n.point_off, n.points)
    ho, hsegs = csr(n.hseg_off, n.hsegs, 2)
    vo, vsegs = csr(n.vseg_off, n.vsegs, 2)
    cap = (n.route_off[ids + 1] - n.route_off[ids]).astype(np.int64)
    ro = np.zeros(len(ids) + 1, np.int64)
    np.cumsum(cap, out=ro[1:])
    return NetArrays(no, nodes, parents, ro, po, points, ho, hsegs, vo, vsegs)


def cpu_stage(design, n_sample, threads):
    """The reference's CPU batching (oracle/_ref, its own code) and the CPU
    restatement of its DAG code on a stride sample; returns (seconds, info)."""
    import oracle
    from grotor_b200.router import plan_from_batches
    g = design.grid
    ids = np.sort(stride_sample(design, n_sample))  # net ids of the sample
    # keep the stage order among the sample
    pos = np.empty(design.n_subnets, np.int64)
    pos[design.order] = np.arange(design.n_subnets)
    ids = ids[np.argsort(pos[ids], kind="stable")]
    sub = sub_nets(design, ids)
    order = np.arange(len(ids), dtype=np.int32)
    kind = "port"
    t0 = time.perf_counter()
    rb = ref_batching(g, order, sub)
    if rb is not None:
        bo, batch_ms = rb
        kind = "reference"
    else:
        tb = time.perf_counter()
        bo, _ = oracle.batches(g.X, g.Y, order, sub.point_off, sub.points, sub.hseg_off, sub.hsegs, sub.vseg_off,
                               sub.vsegs, BATCH_LIMIT, 1)
        batch_ms = (time.perf_counter() - tb) * 1e3
    nb = int(bo.max()) + 1 if len(bo) else 0
    pids, off = plan_from_batches(order, bo, nb)
    og = oracle.OrcGrid(g.L, g.X, g.Y, g.DIR, g.unit_wire, g.unit_via, g.short_costs, g.x_edge_len, g.y_edge_len,
                        g.capacity)
    td = time.perf_counter()
    r = oracle.lshape_stage(og, pids, off, sub.node_off, sub.nodes, sub.parents, sub.route_off, threads=threads)
    dag_ms = (time.perf_counter() - td) * 1e3
    assert r["status"] == 0
    wall = time.perf_counter() - t0
    sec = (batch_ms + dag_ms) / 1e3
    return sec, {"nets": int(len(ids)), "batches": nb, "batching_ms": batch_ms, "dag_ms": dag_ms, "kind": kind,
                 "wall_s": wall}


# --------------------------------------------------------------------------- own arm
def run_grotor(args):
    import torch

    from grotor_b200 import Router
    from grotor_b200.synth import Design

    rank, world, local, pg = dist_init(args.gpus)
    torch.cuda.set_device(local)
    params = replica_params(args.workload, rank)
    t = time.perf_counter()
    design = Design(params)
    log(f"[rank {rank}] design {args.workload}: {design.n_subnets} nets prepared in {time.perf_counter() - t:.1f}s")
    r = Router(design.grid, device=local)
    r.upload_nets(design.nets)
    stream = torch.cuda.ExternalStream(r.stream_handle, device=torch.device("cuda", local))
    order = design.order
    n_nets = design.n_subnets

    def step(mode):
        r.reset()
        r.generate_batches_rsmt(order, BATCH_LIMIT, 1, mode)
        return r.lshape_route(mode)

    tune = None
    if not args.no_tune:  # launch shapes by size bucket, chosen on this plan (untimed)
        r.generate_batches_rsmt(order, BATCH_LIMIT, 1, "persistent")
        tune = r.autotune()
    for _ in range(args.warmup):
        step(args.executor)
    barrier(pg)
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    l0 = r.kernel_launches
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    bt, dt = [], []
    e0.record(stream)
    for _ in range(args.steps):
        st = step(args.executor)
        bt.append(st["batching_ms"])
        dt.append(st["dag_ms"])
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(pg)
    clk = clocks.stop()
    launches = r.kernel_launches - l0
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(pg, ms)
    value = world * args.steps * n_nets / (ms_max / 1e3)
    ms_step = ms_max / args.steps
    routes_p = r.read_routes()
    tables_p = r.read_tables()
    ids, off = r.plan()
    stats_p = r.stats()

    # End to end through the public API with host buffers: H2D of the step's
    # topology and order from pinned memory, batching + stage, D2H of routes.
    nets = design.nets
    pinned = {}
    for name in ("node_off", "nodes", "parents", "route_off", "point_off", "points", "hseg_off", "hsegs",
                 "vseg_off", "vsegs"):
        a = np.asarray(getattr(nets, name))
        tt = torch.empty(a.shape, dtype=getattr(torch, str(a.dtype)), pin_memory=True)
        tt.numpy()[...] = a
        pinned[name] = tt
    from grotor_b200.router import NetArrays
    host_nets = NetArrays(*[pinned[k].numpy() for k in ("node_off", "nodes", "parents", "route_off", "point_off",
                                                        "points", "hseg_off", "hsegs", "vseg_off", "vsegs")])
    order_pin = torch.empty(len(order), dtype=torch.int32, pin_memory=True)
    order_pin.numpy()[...] = order
    h2d = sum(v.numel() * v.element_size() for v in pinned.values()) + order_pin.numel() * 4
    routes_pin = torch.empty(int(nets.route_off[-1]), dtype=torch.int32, pin_memory=True)
    d2h = int(nets.route_off[-1]) * 4 + len(order) * 4 + 16
    torch.cuda.synchronize()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(args.steps):
        r.upload_nets(host_nets)
        r.reset()
        r.generate_batches_rsmt(order_pin.numpy(), BATCH_LIMIT, 1, "plain" if args.executor != "persistent" else "persistent")
        r.lshape_route(args.executor)
        routes_e2e = r.read_routes(out=routes_pin.numpy())
    e3.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(pg, e2.elapsed_time(e3))
    e2e_value = world * args.steps * n_nets / (e2e_ms / 1e3)
    assert np.array_equal(routes_e2e, routes_p)

    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args.workload, design.grid, n_nets, stats_p["n_batches"]),
        "executor": args.executor, "parallelism": f"replicas{world}",
        "stage": {"batching_ms": float(np.mean(bt)), "dag_ms": float(np.mean(dt)),
                  "wirelength": stats_p["wirelength"], "vias": stats_p["vias"]},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(launches),
        "clocks": clk,
    }

    # Roofline of the two kernels of the persistent form.
    lib = r._lib
    out = np.zeros(4, np.float64)
    gs = design.grid.struct()
    P = lambda a: np.ascontiguousarray(a).ctypes.data_as(C.c_void_p)  # noqa: E731
    rc = lib.grb_stage_traffic(C.byref(gs), len(off) - 1, P(off), P(ids), P(nets.node_off), P(nets.nodes),
                               P(nets.parents), P(nets.route_off), P(routes_p), P(nets.point_off), P(nets.hseg_off),
                               P(nets.hsegs), P(nets.vseg_off), P(nets.vsegs), 1, P(out))
    assert rc == 0
    stage_bytes = out[0] + out[1] + out[2]
    batch_bytes = out[3]
    peak, peak_kind = measured_peak()
    stage_ms, batch_ms = float(np.mean(dt)), float(np.mean(bt))
    kernels = {
        "k_lshape_persistent": (stage_bytes, stage_ms),
        "k_batch_persistent": (batch_bytes, batch_ms),
    }
    dom = max(kernels, key=lambda k: kernels[k][1])
    roofs = {}
    for k, (byt, kms) in kernels.items():
        ach = byt / (kms / 1e3) / 1e9
        roofs[k] = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                    "traffic": profiled_traffic(k, args.workload), "algorithmic_bytes": byt, "ms": kms,
                    "peak_source": f"{peak_kind} hbm_gbs"}
    result["roofline"] = dict(roofs[dom], kernel=dom)
    result["roofline_all"] = roofs
    result["algorithmic_bytes"] = {"refresh": out[0], "dp": out[1], "commit": out[2], "batching": out[3]}

    if not args.no_compare:
        comp = {"persistent": {"ms": ms_step, "batching_ms": batch_ms, "dag_ms": stage_ms}}
        identical = True
        for mode in ("graph", "plain"):
            step(mode)  # warm (graph capture)
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            st = step(mode)
            b.record(stream)
            torch.cuda.synchronize()
            comp[mode] = {"ms": a.elapsed_time(b), "batching_ms": st["batching_ms"], "dag_ms": st["dag_ms"]}
            same = np.array_equal(r.read_routes(), routes_p) and np.array_equal(
                r.read_tables()["demand_half"], tables_p["demand_half"])
            identical &= bool(same)
        comp["speedup_persistent_vs_plain"] = comp["plain"]["ms"] / ms_step
        comp["speedup_persistent_vs_graph"] = comp["graph"]["ms"] / ms_step
        comp["routes_identical"] = identical
        result["executors"] = comp

    result["autotune"] = tune
    if rank == 0 and world == 1 and not args.no_cpu:
        # Untimed: the GPU's batch of every order position, for the checker.
        gpu_batch_of, _ = r.generate_batches_rsmt(order, BATCH_LIMIT, 1, args.executor)
        base, parity = cpu_leg(design, args.workload, gpu_batch_of, ids, off, routes_p, tables_p, stats_p)
        result["cpu_baseline"] = base
        result["parity"] = parity
    if rank == 0 and world == 1 and not args.no_extra:
        r.close()
        r = None
        result["zshape"] = zshape_measure(args)
        result["softmin"] = softmin_measure(args)
        result["pipeline"] = pipeline_measure(args)
        result["configs"] = configs_measure(args)
    if r is not None:
        r.close()
    if pg is not None:
        pg.destroy_process_group()
    if rank == 0:
        print(json.dumps(result), flush=True)


def cpu_leg(design, workload, gpu_batch_of, ids, off, routes, tables, stats):
    """The CPU baseline on the whole workload, which is also the checker of the
    GPU run: the reference's own CPU batching over the whole order (one core,
    its design), then the CPU restatement of its DAG code over the whole plan
    on every host core, with the device's values of the cost model's
    exponential.  Returns (cpu_baseline, parity)."""
    import oracle
    from grotor_b200 import _abi
    g, n = design.grid, design.nets
    cores = host_cores()
    t0 = time.perf_counter()
    rb = ref_batching(g, design.order, n)
    if rb is not None:
        ref_bo, batch_ms, kind = rb[0], rb[1], "reference"
    else:
        tb = time.perf_counter()
        ref_bo, _ = oracle.batches(g.X, g.Y, design.order, n.point_off, n.points, n.hseg_off, n.hsegs, n.vseg_off,
                                   n.vsegs, BATCH_LIMIT, 1)
        batch_ms, kind = (time.perf_counter() - tb) * 1e3, "port"
    og = oracle.OrcGrid(g.L, g.X, g.Y, g.DIR, g.unit_wire, g.unit_via, g.short_costs, g.x_edge_len, g.y_edge_len,
                        g.capacity)
    x = oracle.exp_args(og, int(tables["demand_half"].max()) + 8)
    y = np.empty_like(x)
    assert _abi.load().grb_cost_exp(0, x.ctypes.data_as(C.c_void_p), len(x), y.ctypes.data_as(C.c_void_p)) == 0
    oracle.set_exp_table(x, y)
    td = time.perf_counter()
    orc = oracle.lshape_stage(og, ids, off, n.node_off, n.nodes, n.parents, n.route_off, threads=cores)
    dag_ms = (time.perf_counter() - td) * 1e3
    misses = oracle.exp_table_misses()
    oracle.set_exp_table()
    log(f"cpu leg: batching {batch_ms:.0f} ms ({kind}), DAG {dag_ms:.0f} ms on {cores} cores, "
        f"{time.perf_counter() - t0:.0f} s in all")
    sec = (batch_ms + dag_ms) / 1e3
    base = {"value": n.n / sec, "unit": UNIT, "cores": cores, "kind": kind, "cpu_model": cpu_model(),
            "batching_ms": batch_ms, "dag_ms": dag_ms,
            "sample": (f"the whole workload ({n.n} nets, {int(ref_bo.max()) + 1} batches): the reference's CPU "
                       f"first-fit batching on 1 core (its own code, oracle/_ref) + the CPU restatement of its DAG "
                       f"code on {cores} threads")}
    checks = {
        "batches_equal_reference_cpu": bool(np.array_equal(ref_bo, gpu_batch_of)),
        "routes_equal_oracle": bool(np.array_equal(orc["routes"], routes)),
        "demand_equal_oracle": bool(np.array_equal(orc["demand_half"], tables["demand_half"])),
        "timestamps_equal_oracle": bool(np.array_equal(orc["timestamp"], tables["timestamp"])),
        "wirelength_equal_oracle": orc["wirelength"] == stats["wirelength"],
        "vias_equal_oracle": orc["vias"] == stats["vias"],
        "exp_table_misses": int(misses),
    }
    ok = all(v for k, v in checks.items() if k != "exp_table_misses") and misses == 0 and orc["status"] == 0
    parity = {"result": "identical" if ok else "DIFFERS", **checks,
              "how": ("GPU batches vs the reference's own CPU batching over the whole order; GPU stage vs the CPU "
                      "restatement on the same plan with the device's exponential values")}
    return base, parity


# --------------------------------------------------------------------------- other stages
def _stream(r):
    import torch
    return torch.cuda.ExternalStream(r.stream_handle, device=torch.device("cuda", torch.cuda.current_device()))


def zshape_measure(args, workload="large_800x800x10", steps=3, warmup=2):
    """Z-shape stage (the GGR pipeline, configuration 'large' 800x800x10 with
    900K nets) on the generator's trees: first-fit groups, bounding-box
    batches and the Z-shape stage per step, persistent and plain executors."""
    import torch

    from grotor_b200 import Router
    from grotor_b200.router import GrbError, NetArrays
    from grotor_b200.synth import WORKLOADS, Design
    d = Design(WORKLOADS[workload])
    z = d.zshape_trees()
    n = d.nets
    zn = np.diff(z["node_off"]).astype(np.int64)
    route_off = np.concatenate([[0], np.cumsum(1 + 64 * zn)]).astype(np.int64)
    r = Router(d.grid)
    r.upload_nets(NetArrays(n.node_off, n.nodes, n.parents, route_off, n.point_off, n.points, n.hseg_off, n.hsegs,
                            n.vseg_off, n.vsegs))
    r.upload_zshape(z)
    r.set_wire_cost_mode(True)
    stream = _stream(r)
    out = {"workload": workload, "nets": int(n.n), "batch_limit": 250}
    for mode in ("persistent", "plain"):
        times, dag, first = [], [], []
        for k in range(warmup + steps):
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            r.reset()
            r.generate_batches_rsmt(d.order, BATCH_LIMIT, 1, mode)
            fb = r.stats()["batching_ms"]
            nb = r.plan_bbox_batches(250)
            try:
                st = r.zshape_route(mode)
                status = "ok"
            except GrbError as e:  # the reference's "Z-shape DP failure": the stage still ran to the end
                st = r.stats()
                status = str(e)
            b.record(stream)
            torch.cuda.synchronize()
            if k >= warmup:
                times.append(a.elapsed_time(b))
                dag.append(st["dag_ms"])
                first.append(fb)
        out[mode] = {"ms_per_step": float(np.mean(times)), "nets_per_s": n.n / (np.mean(times) / 1e3),
                     "first_fit_ms": float(np.mean(first)), "dag_ms": float(np.mean(dag)), "batches": int(nb),
                     "wirelength": st["wirelength"], "vias": st["vias"], "status": status}
    out["speedup_persistent_vs_plain"] = out["plain"]["ms_per_step"] / out["persistent"]["ms_per_step"]
    # Roofline of the stage kernel: the model's bytes (grb_zshape_traffic:
    # refresh, DP reads of every net's box rows and columns, commit) over the
    # stage's device time, for each executor (same plan, same routes).
    ids, off = r.plan()
    routes = r.read_routes()
    traffic = np.zeros(3, np.float64)
    gs = d.grid.struct()
    Pp = lambda a: np.ascontiguousarray(a).ctypes.data_as(C.c_void_p)  # noqa: E731
    rc = r._lib.grb_zshape_traffic(C.byref(gs), len(off) - 1, Pp(off), Pp(ids), Pp(z["node_off"]), Pp(z["coord"]),
                                   Pp(z["child"]), Pp(route_off), Pp(routes), Pp(traffic))
    assert rc == 0
    peak, kind = measured_peak()
    out["algorithmic_bytes"] = {"refresh": traffic[0], "dp": traffic[1], "commit": traffic[2]}
    for mode in ("persistent", "plain"):
        ach = traffic.sum() / (out[mode]["dag_ms"] / 1e3) / 1e9
        out[mode]["roofline"] = {"kernel": "k_zshape_persistent" if mode == "persistent" else "per-batch launches",
                                 "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                                 "peak_source": f"{kind} hbm_gbs"}
    r.close()
    return out


def configs_measure(args, workloads=("small_64x64x5", "medium_320x320x10", "large_800x800x10"), reps=3):
    """The L-shape stage (batching + DAG) on the benchmark plan's other
    configurations -- 'small' (64x64x5, 5,000 nets), 'medium' (320x320x10,
    120K nets) and 'large' (800x800x10, 900K nets) -- in the persistent and
    plain executors: mean device time over `reps` steps after one warm-up,
    nets/s, and the routes of the two executors compared."""
    import torch

    from grotor_b200 import Router
    from grotor_b200.synth import WORKLOADS, Design
    out = {}
    for wl in workloads:
        d = Design(WORKLOADS[wl])
        r = Router(d.grid)
        r.upload_nets(d.nets)
        stream = _stream(r)
        res = {"nets": int(d.nets.n)}
        routes = {}
        for mode in ("persistent", "plain"):
            times, bt, dt = [], [], []
            for k in range(reps + 1):
                torch.cuda.synchronize()
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                r.reset()
                _, nb = r.generate_batches_rsmt(d.order, BATCH_LIMIT, 1, mode)
                st = r.lshape_route(mode)
                b.record(stream)
                torch.cuda.synchronize()
                if k:
                    times.append(a.elapsed_time(b))
                    bt.append(st["batching_ms"])
                    dt.append(st["dag_ms"])
            routes[mode] = r.read_routes()
            ms = float(np.mean(times))
            res[mode] = {"ms_per_step": ms, "nets_per_s": d.nets.n / (ms / 1e3), "batching_ms": float(np.mean(bt)),
                         "dag_ms": float(np.mean(dt)), "batches": int(nb)}
        res["speedup_persistent_vs_plain"] = res["plain"]["ms_per_step"] / res["persistent"]["ms_per_step"]
        res["routes_identical"] = bool(np.array_equal(routes["persistent"], routes["plain"]))
        r.close()
        out[wl] = res
    return out


def pipeline_measure(args, workload="medium_320x320x10"):
    """The default pipeline end to end through the drop-in driver
    (integration/_build/grotor_grb: the reference's program flow on this
    library, CAP/NET in, .out out) on the 'medium' design: stage one
    (L-shape) and stage two (rip-up + FLT, configuration 3's composite) with
    each stage's device time, nets/s and, for the FLT stage, its roofline from
    the byte model (a separate run with --report-traffic 1, untimed)."""
    driver = os.path.join(ROOT, "integration", "_build", "grotor_grb")
    lut = os.path.dirname(driver)  # FLUTE's tables beside the driver (integration/Makefile)
    if not os.path.exists(driver) or not os.path.exists(os.path.join(lut, "POWV9.dat")):
        return {"unavailable": "drop-in driver or FLUTE tables not built (integration/Makefile)"}
    from grotor_b200.synth import WORKLOADS, Design

    def records(text):
        out = {"lshape": {}, "detour": {}}
        for line in text.splitlines():
            tag, _, rest = line.partition(" ")
            kv = dict(p.split("=", 1) for p in rest.split() if "=" in p)
            if tag == "DAG_TIMING" and kv.get("batch_index") == "-1":
                out[kv["stage"]].update(dag_ms=float(kv["elapsed_ms"]), nets=int(kv["nets"]), batches=int(kv["batches"]))
            elif tag == "BATCH_TIMING":
                out[kv.get("stage", "lshape")]["batching_ms"] = float(kv["elapsed_ms"])
            elif tag == "TOPOLOGY_TIMING" and kv.get("stage") == "lshape":
                out["lshape"]["topology_ms"] = float(kv["elapsed_ms"])
            elif tag == "FLT_TRAFFIC":
                out["detour"]["algorithmic_bytes"] = sum(float(v) for v in kv.values())
            elif tag == "GROTOR_COMPLETE":
                out["wall_s"] = float(kv["wall_seconds"])
        for st in ("lshape", "detour"):
            d = out[st]
            if "dag_ms" in d and "batching_ms" in d:
                d["stage_ms"] = d["dag_ms"] + d["batching_ms"]
                d["nets_per_s"] = d["nets"] / (d["stage_ms"] / 1e3)
        return out

    res = {"workload": workload, "driver": "integration/_build/grotor_grb"}
    with tempfile.TemporaryDirectory() as w:
        cap, net = os.path.join(w, "d.cap"), os.path.join(w, "d.net")
        Design(WORKLOADS[workload]).write(cap, net)
        for ex in ("persistent", "plain"):
            run = subprocess.run([driver, "-cap", cap, "-net", net, "-out", os.path.join(w, ex + ".out"), "--lut-dir",
                                  lut, "--executor", ex], capture_output=True, text=True, timeout=900)
            if run.returncode:
                return {"unavailable": f"drop-in driver failed: {run.stderr[-300:]}"}
            res[ex] = records(run.stdout)
        res["outputs_identical"] = open(os.path.join(w, "persistent.out"), "rb").read() == \
            open(os.path.join(w, "plain.out"), "rb").read()
        run = subprocess.run([driver, "-cap", cap, "-net", net, "-out", os.devnull, "--lut-dir", lut, "--executor",
                              "persistent", "--report-traffic", "1"], capture_output=True, text=True, timeout=900)
    byt = records(run.stdout)["detour"].get("algorithmic_bytes") if run.returncode == 0 else None
    peak, kind = measured_peak()
    for ex in ("persistent", "plain"):
        d = res[ex]["detour"]
        if byt and d.get("dag_ms"):
            ach = byt / (d["dag_ms"] / 1e3) / 1e9
            d["roofline"] = {"kernel": "k_flt_persistent" if ex == "persistent" else "per-batch launches", "bound": "hbm",
                             "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                             "algorithmic_bytes": byt, "peak_source": f"{kind} hbm_gbs"}
    if res["plain"]["detour"].get("stage_ms") and res["persistent"]["detour"].get("stage_ms"):
        res["flt_speedup_persistent_vs_plain"] = res["plain"]["detour"]["stage_ms"] / res["persistent"]["detour"]["stage_ms"]
    return res


def softmin_measure(args, workload="softmin_320x320x10", taus=(1.0, 0.1, 0.01), reps=3):
    """Soft-min DAG forward and adjoint (configuration 'soft-min', 320x320x10,
    120K nets) in fp32, at the demand of the exact L-shape stage."""
    import torch

    from grotor_b200 import Router
    from grotor_b200.softmin import routing_cost
    from grotor_b200.synth import WORKLOADS, Design
    d = Design(WORKLOADS[workload])
    r = Router(d.grid)
    r.upload_nets(d.nets)
    r.generate_batches_rsmt(d.order, BATCH_LIMIT, 1, "persistent")
    r.lshape_route("persistent")
    g = d.grid
    out = {"workload": workload, "nets": int(d.n_subnets), "dtype": "f32"}
    # Byte model of one forward and one adjoint (T = 4 bytes, f32): cost tables
    # (capacity, unit wire cost and demand read, wire and via cost written),
    # track prefix (read + write), the DAG's read set (grb_dag_reads: distinct
    # prefix and via-cost entries per net, 8 B per tree node), net costs; the
    # adjoint repeats tables, prefix and reads, adds read-modify-write of the
    # adjoint entries, the suffix pass, the chain rule to capacity and unit
    # wire cost and the via-cost sum.
    reads = np.zeros(3, np.float64)
    gs = g.struct()
    Pp = lambda a: np.ascontiguousarray(a).ctypes.data_as(C.c_void_p)  # noqa: E731
    n = d.nets
    assert r._lib.grb_dag_reads(C.byref(gs), n.n, None, Pp(n.node_off), Pp(n.nodes), Pp(n.parents), Pp(reads)) == 0
    T, cells = 4.0, float(g.L * g.X * g.Y)
    tables, prefix = cells * (3 * T + 4 + 2 * T), cells * 2 * T
    dag = T * (reads[0] + reads[1]) + 8.0 * reads[2]
    fwd_bytes = tables + prefix + dag + T * n.n
    bwd_bytes = tables + prefix + 2 * cells * T + dag + 2 * T * (reads[0] + reads[1]) + cells * 2 * T + \
        cells * 6 * T + cells * T
    peak, kind = measured_peak()
    out["algorithmic_bytes"] = {"forward": fwd_bytes, "backward": bwd_bytes, "dag_prefix_entries": reads[0],
                                "dag_via_entries": reads[1], "tree_nodes": reads[2]}
    for tau in taus:
        cap = torch.tensor(np.asarray(g.capacity, np.float32), device="cuda").requires_grad_(True)
        uw = torch.full_like(cap, float(g.unit_wire)).requires_grad_(True)
        uv = torch.tensor(float(g.unit_via), device="cuda", requires_grad=True)
        fw, bw = [], []
        for k in range(reps + 1):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            F = routing_cost(r, cap, uw, uv, tau)
            t1 = time.perf_counter()
            F.backward()
            torch.cuda.synchronize()
            t2 = time.perf_counter()
            cap.grad = uw.grad = uv.grad = None
            if k:
                fw.append((t1 - t0) * 1e3)
                bw.append((t2 - t1) * 1e3)
        fa = fwd_bytes / (np.mean(fw) / 1e3) / 1e9
        ba = bwd_bytes / (np.mean(bw) / 1e3) / 1e9
        out[f"tau_{tau:g}"] = {
            "forward_ms": float(np.mean(fw)), "backward_ms": float(np.mean(bw)), "total_cost": float(F.item()),
            "roofline_forward": {"kernel": "k_soft_forward (+ tables, prefix)", "bound": "hbm", "achieved": fa,
                                 "peak": peak, "unit": "GB/s", "frac": fa / peak, "peak_source": f"{kind} hbm_gbs"},
            "roofline_backward": {"kernel": "k_soft_backward (+ tables, prefix, suffix, chain)", "bound": "hbm",
                                  "achieved": ba, "peak": peak, "unit": "GB/s", "frac": ba / peak,
                                  "peak_source": f"{kind} hbm_gbs"}}
    r.close()
    return out


# --------------------------------------------------------------------------- reference arm
def run_reference(args):
    """The reference's own CPU implementation of the path: its CPU first-fit
    batching (oracle/_ref, one core by design) and the CPU restatement of its
    DAG code (all host cores).  Per step a stride sample of the workload's nets
    (sized so the run ends within minutes); the reference's batching over the
    whole order is timed once besides.  Loads the workload generator and the
    restatement, never the routing library."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from grotor_b200.synth import WORKLOADS, Design
    design = Design(WORKLOADS[args.workload])
    threads = host_cores()
    target = args.cpu_nets or 30000
    rb = ref_batching(design.grid, design.order, design.nets)
    if rb is not None:
        full_bo, full_ms = rb
    else:
        import oracle
        g, n = design.grid, design.nets
        t = time.perf_counter()
        full_bo, _ = oracle.batches(g.X, g.Y, design.order, n.point_off, n.points, n.hseg_off, n.hsegs,
                                    n.vseg_off, n.vsegs, BATCH_LIMIT, 1)
        full_ms = (time.perf_counter() - t) * 1e3
    n_batches = int(full_bo.max()) + 1 if len(full_bo) else 0
    log(f"reference batching over the whole order: {full_ms:.0f} ms, {n_batches} batches")
    times, info = [], None
    for i in range(args.warmup + args.steps):
        sec, info = cpu_stage(design, target, threads)
        log(f"reference step {i}: {sec:.2f}s ({info})")
        if i >= args.warmup:
            times.append(sec)
    value = info["nets"] / float(np.mean(times))
    sample = (f"every {max(1, design.n_subnets // target)}-th net of {args.workload} in stage order "
              f"({info['nets']} nets, {info['batches']} batches): reference CPU batching (its own code, 1 core) "
              f"+ CPU restatement of its DAG code on {threads} threads; the sample has fewer batches than the "
              f"whole design, so its per-net batching is cheaper (whole order: {full_ms:.0f} ms for "
              f"{design.n_subnets} nets)")
    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(np.mean(times)) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args.workload, design.grid, design.n_subnets, n_batches),
        "parallelism": "host", "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": info["kind"],
                         "cpu_model": cpu_model(), "sample": sample},
        "full_order_batching_ms": full_ms,
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(result), flush=True)


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_grotor(args)


if __name__ == "__main__":
    main()
