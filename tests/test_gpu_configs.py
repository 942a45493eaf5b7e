"""The whole L-shape stage at the sizes of the benchmark configurations.

Against the CPU restatement.  For the seeded 'small' (64x64, 5 CAP layers,
5,000 nets), 'medium' (320x320x10, 120,000 nets) and 'large' (800x800x10,
900,000 nets) designs: GPU first-fit batching equals the oracle's batches
exactly; the stage then runs in all three executors (persistent, plain, CUDA
graph) and the oracle runs the same stage on the same plan with the device's
own values of the cost model's exponential (grb_cost_exp), so its cost tables
are bit-identical to the device's.  Every route word, the demand, the
timestamps and the wirelength / via statistics must be equal, and after a
final refresh the wire / via cost tables and the double prefix table must be
bit-identical to the oracle's.

Against the reference router itself.  For the 'medium' design written as
CAP/NET files, the reference's own code (oracle/_ref/ref_harness, built from its
sources) builds the topology (FLUTE trees, HPWL order, CPU first-fit batches)
and runs its GPU L-shape stage; on that topology and plan the B200 path must
reproduce the reference's route words, demand and statistics exactly, its GPU
batching must equal the reference's CPU batches, and the .out file written by
the reference's writer must be byte-identical with identical evaluator scores.
"""
import hashlib
import os
import subprocess

import numpy as np
import pytest

import oracle
from helpers import ROOT, device_exp_table, float_demand_to_half, golden_grid, golden_nets, orc_grid

pytestmark = pytest.mark.gpu

HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
EVALUATOR = os.path.join(ROOT, "oracle", "_ref", "evaluator")
LIMIT = 1000000  # lshape.cuh:62


def _equal(a, b, what):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, f"{what}: shape {a.shape} vs {b.shape}"
    bad = np.flatnonzero(a != b)
    assert len(bad) == 0, f"{what}: {len(bad)} of {a.size} differ, first at {bad[:5]}"


@pytest.mark.parametrize("workload", ["small_64x64x5", "medium_320x320x10", "large_800x800x10"])
def test_stage_equals_oracle(workload):
    from grotor_b200 import Router, plan_from_batches
    from grotor_b200.synth import WORKLOADS, Design
    d = Design(WORKLOADS[workload])
    g, n = d.grid, d.nets
    r = Router(g)
    r.upload_nets(n)
    bo, nb = r.generate_batches_rsmt(d.order, LIMIT, 1, "persistent")
    bo_ref, nb_ref = oracle.batches(g.X, g.Y, d.order, n.point_off, n.points, n.hseg_off, n.hsegs, n.vseg_off,
                                    n.vsegs, LIMIT, 1)
    assert nb == nb_ref
    _equal(bo, bo_ref, "batch of each order position")
    ids, off = r.plan()
    want_ids, want_off = plan_from_batches(d.order, bo_ref, nb_ref)
    _equal(ids, want_ids, "plan ids")
    _equal(off, want_off, "plan offsets")

    got = {}
    for mode in ("persistent", "plain", "graph"):
        r.reset()
        st = r.lshape_route(mode)
        got[mode] = (r.read_routes(), r.read_tables(), st)
    routes, t, st = got["persistent"]
    for mode in ("plain", "graph"):
        _equal(got[mode][0], routes, f"{mode} routes vs persistent")
        _equal(got[mode][1]["demand_half"], t["demand_half"], f"{mode} demand vs persistent")
        assert got[mode][2]["wirelength"] == st["wirelength"] and got[mode][2]["vias"] == st["vias"]

    og = orc_grid(g)
    with device_exp_table(og, max(64, int(t["demand_half"].max()) + 8)) as table:
        orc = oracle.lshape_stage(og, ids, off, n.node_off, n.nodes, n.parents, n.route_off)
        r.refresh_cost()
        final = r.read_tables()
        w, v = oracle.cost_full(og, final["demand_half"])
    assert table.misses == 0
    assert orc["status"] == 0
    _equal(routes, orc["routes"], "route words")
    _equal(t["demand_half"], orc["demand_half"], "demand")
    _equal(t["timestamp"], orc["timestamp"], "timestamps")
    assert st["stamp"] == orc["stamp"] == nb
    assert st["wirelength"] == orc["wirelength"]
    assert st["vias"] == orc["vias"]
    # Cost tables of the final demand: bit-identical with the device's exponential.
    _equal(final["wcost"].view(np.int32), w.view(np.int32), "wcost bits")
    _equal(final["vcost"].view(np.int32), v.view(np.int32), "vcost bits")
    _equal(final["presum"].view(np.int64), oracle.presum(og, final["wcost"]).view(np.int64), "presum bits")
    r.close()


def _harness(*args):
    subprocess.run([HARNESS, *args], check=True, stdout=subprocess.DEVNULL)


def _read_dir(d):
    ext = {"i32": np.int32, "i64": np.int64, "f32": np.float32, "f64": np.float64}
    out = {}
    for f in os.listdir(d):
        base, _, e = f.rpartition(".")
        if e in ext:
            out[base] = np.fromfile(os.path.join(d, f), dtype=ext[e])
    return out


def _scores(text):
    keep = ("overflow cost", "open nets", "incompleted nets", "wirelength cost", "via cost", "total cost", "FOR_STAT")
    lines = [ln.strip() for ln in text.splitlines() if any(k in ln for k in keep) and "time" not in ln.lower()]
    assert len(lines) >= 6, text
    return lines


def test_medium_stage_equals_reference_gpu_run(tmp_path):
    if not os.path.exists(HARNESS):
        pytest.skip("reference harness not built (oracle/ref.mk)")
    from grotor_b200 import Router
    from grotor_b200.synth import WORKLOADS, Design
    w = str(tmp_path)
    cap, net = os.path.join(w, "d.cap"), os.path.join(w, "d.net")
    Design(WORKLOADS["medium_320x320x10"]).write(cap, net)
    lut = os.path.dirname(HARNESS)
    _harness("topo", cap, net, w, lut)
    ref_out = os.path.join(w, "ref.out")
    _harness("route", cap, net, w, lut, ref_out)
    g = _read_dir(w)
    assert len(g["ids"]) > 100000

    # GPU batching on the reference's geometry and order = its CPU batches.
    grid, nets = golden_grid(g), golden_nets(g)
    r = Router(grid)
    r.upload_nets(nets)
    bo, nb = r.generate_batches_rsmt(g["order"], LIMIT, 1, "persistent")
    assert nb == len(g["batch_off"]) - 1
    _equal(bo, g["batch_of"], "batch of each order position vs reference CPU batching")
    ids, off = r.plan()
    _equal(ids, g["ids"], "plan vs reference")
    _equal(off, g["batch_off"], "plan offsets vs reference")

    for mode in ("persistent", "plain"):
        r.reset()
        r.set_stats(0.0, int(g["pin_vias"][0]))  # build_cuda_database seeds the via count
        st = r.lshape_route(mode)
        routes, t = r.read_routes(), r.read_tables()
        _equal(routes, g["ref_routes"][:-1], f"{mode} route words vs reference")
        _equal(t["demand_half"], float_demand_to_half(g["ref_demand"]), f"{mode} demand vs reference")
        assert st["wirelength"] == g["ref_stats"][0]
        assert st["vias"] == int(g["ref_stats"][1])
    r.close()

    # The .out through the reference's own writer, and its evaluator scores.
    rp = os.path.join(w, "routes.i32")
    np.concatenate([routes, np.zeros(1, np.int32)]).tofile(rp)
    mine = os.path.join(w, "mine.out")
    _harness("write", cap, net, w, lut, rp, mine)
    a, b = open(mine, "rb").read(), open(ref_out, "rb").read()
    assert hashlib.sha256(a).hexdigest() == hashlib.sha256(b).hexdigest()
    if os.path.exists(EVALUATOR):
        ev = [subprocess.run([EVALUATOR, cap, net, f], capture_output=True, text=True) for f in (mine, ref_out)]
        assert _scores(ev[0].stdout + ev[0].stderr) == _scores(ev[1].stdout + ev[1].stderr)
