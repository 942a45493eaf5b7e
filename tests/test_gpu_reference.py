"""The CUDA path against the reference router's own GPU run.

On the reference's topology, order and batches (fixtures from
tests/golden/make_golden.py) the B200 path must reproduce the reference's
route words, demand and statistics exactly; written through the reference's
own .out writer (oracle/_ref/ref_harness write) the file must be
byte-identical, and the reference evaluator must report identical scores.
"""
import hashlib
import os
import subprocess
import tempfile

import numpy as np
import pytest

from helpers import ROOT, float_demand_to_half, golden_grid, golden_nets, load_golden

pytestmark = pytest.mark.gpu

NAMES = ["ref_64x64x10_2k", "ref_32x32x10_400"]
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
EVALUATOR = os.path.join(ROOT, "oracle", "_ref", "evaluator")


def need(g, *keys):
    missing = [k for k in keys if k not in g]
    if missing:
        pytest.skip(f"fixture lacks reference GPU outputs {missing}")


def _route(g, mode):
    from grotor_b200 import Router
    r = Router(golden_grid(g))
    r.upload_nets(golden_nets(g))
    r.set_plan(g["ids"], g["batch_off"])
    r.set_stats(0.0, int(g["pin_vias"][0]))  # build_cuda_database seeds the via count
    st = r.lshape_route(mode)
    out = r.read_routes(), r.read_tables(), st
    r.close()
    return out


@pytest.mark.parametrize("mode", ["plain", "persistent"])
@pytest.mark.parametrize("name", NAMES)
def test_routes_equal_reference(name, mode):
    g = load_golden(name)
    need(g, "ref_routes", "ref_demand", "ref_stats")
    routes, t, st = _route(g, mode)
    np.testing.assert_array_equal(routes, g["ref_routes"][:-1])
    np.testing.assert_array_equal(t["demand_half"], float_demand_to_half(g["ref_demand"]))
    assert st["wirelength"] == g["ref_stats"][0]
    assert st["vias"] == int(g["ref_stats"][1])


def test_tables_equal_reference():
    """After the stage and one refresh, wcost/vcost agree with the reference's
    within 1e-6 relative (the same __expf, so in practice bit-equal) and the
    double prefix table is bit-identical."""
    from grotor_b200 import Router
    g = load_golden("ref_32x32x10_400")
    need(g, "ref_wcost", "ref_vcost", "ref_presum")
    r = Router(golden_grid(g))
    r.upload_nets(golden_nets(g))
    r.set_plan(g["ids"], g["batch_off"])
    r.lshape_route("persistent")
    r.refresh_cost()
    t = r.read_tables()
    r.close()
    np.testing.assert_allclose(t["wcost"], g["ref_wcost"], rtol=1e-6, atol=0)
    np.testing.assert_allclose(t["vcost"], g["ref_vcost"], rtol=1e-6, atol=0)
    np.testing.assert_array_equal(t["presum"].view(np.int64), g["ref_presum"].view(np.int64))


@pytest.mark.parametrize("name", NAMES)
def test_out_file_byte_identical_and_scores(name):
    g = load_golden(name)
    need(g, "ref_out_sha256", "ref_eval_text")
    if not os.path.exists(HARNESS):
        pytest.skip("reference harness not built (oracle/ref.mk)")
    from dataclasses import replace

    from grotor_b200.synth import WORKLOADS, Design
    from golden.make_golden import FIXTURES
    wl, over = FIXTURES[name]
    routes, _, _ = _route(g, "persistent")
    with tempfile.TemporaryDirectory() as w:
        d = Design(replace(WORKLOADS[wl], **over))
        cap, net = os.path.join(w, "d.cap"), os.path.join(w, "d.net")
        d.write(cap, net)
        words = np.concatenate([routes, np.zeros(1, np.int32)])
        rp = os.path.join(w, "routes.i32")
        words.tofile(rp)
        np.asarray(g["ids"], np.int32).tofile(os.path.join(w, "ids.i32"))  # publication order
        out = os.path.join(w, "mine.out")
        subprocess.run([HARNESS, "write", cap, net, w, os.path.dirname(HARNESS), rp, out], check=True,
                       stdout=subprocess.DEVNULL)
        blob = open(out, "rb").read()
        assert hashlib.sha256(blob).digest() == bytes(g["ref_out_sha256"])
        if os.path.exists(EVALUATOR):
            res = subprocess.run([EVALUATOR, cap, net, out], capture_output=True, text=True)
            assert _scores(res.stdout + res.stderr) == _scores(bytes(g["ref_eval_text"]).decode())


def _scores(text):
    """Evaluator report lines (costs, open / incomplete nets), timing excluded."""
    keep = ("overflow cost", "open nets", "incompleted nets", "wirelength cost", "via cost", "total cost", "FOR_STAT")
    lines = [ln.strip() for ln in text.splitlines() if any(k in ln for k in keep) and "time" not in ln.lower()]
    assert len(lines) >= 6, text
    return lines
