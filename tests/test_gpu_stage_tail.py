"""The stage tail: rip-up classification and congestion view of the final
demand, computed at the end of the L-shape stage (inside the persistent
kernel, no host round trip; separate launches after the last batch in the
plain and CUDA-graph forms).

On a congested seeded design, in every executor, the tail's results equal
the standalone entry points' (grb_ripup_classify, grb_congestion_view) on the
same final state and the oracle's restatement (congestion.cuh:8-112) of the
GPU's own demand and routes, bit for bit.  On the reference's FLT fixture the
tail reproduces the reference's own rip-up set and, where the fixture carries
it, the reference's congestion view.
"""
import numpy as np
import pytest

import oracle
from helpers import golden_grid, golden_nets, load_golden, orc_grid

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", ["persistent", "plain", "graph"])
def test_tail_equals_standalone_and_oracle(mode):
    from grotor_b200 import Router
    from grotor_b200.synth import WORKLOADS, Design
    d = Design(WORKLOADS["medium_320x320x10"].scaled(30000, seed=41, cap_lo=1, cap_hi=5))
    r = Router(d.grid)
    r.upload_nets(d.nets)
    r.generate_batches_rsmt(d.order, 1000000, 1, mode)
    for thr in (0, -1):
        r.set_stage_tail(ripup=True, view=True, threshold=thr)
        r.reset()
        r.lshape_route(mode)
        is_of, (cong, xs, ys) = r.stage_tail()
        np.testing.assert_array_equal(is_of, r.ripup(thr))
        c2, x2, y2 = r.congestion_view()
        np.testing.assert_array_equal(cong, c2)
        np.testing.assert_array_equal(xs.view(np.int32), x2.view(np.int32))
        np.testing.assert_array_equal(ys.view(np.int32), y2.view(np.int32))
        t = r.read_tables()
        og = orc_grid(d.grid)
        want = oracle.ripup_classify(og, t["demand_half"], thr, d.nets.route_off, r.read_routes())
        np.testing.assert_array_equal(is_of, want)
        oc, ox, oy = oracle.congestion_view(og, t["demand_half"])
        np.testing.assert_array_equal(cong, oc)
        np.testing.assert_array_equal(xs.view(np.int32), ox.view(np.int32))
        np.testing.assert_array_equal(ys.view(np.int32), oy.view(np.int32))
        assert is_of.sum() > 0 and cong.sum() > 0
    r.close()


def test_tail_equals_reference_fixture():
    from grotor_b200 import Router
    g = load_golden("ref_flt_48x48x10_1500")
    if "flt_of_nets" not in g:
        pytest.skip("fixture lacks the reference FLT run")
    r = Router(golden_grid(g))
    r.upload_nets(golden_nets(g))
    r.set_plan(g["ids"], g["batch_off"])
    r.set_stage_tail(ripup=True, view=True, threshold=0)
    r.lshape_route("persistent")
    is_of, (cong, xs, ys) = r.stage_tail()
    np.testing.assert_array_equal(np.flatnonzero(is_of), g["flt_of_nets"])
    if "flt_congestion" in g:
        np.testing.assert_array_equal(cong, g["flt_congestion"].astype(np.uint8))
        np.testing.assert_array_equal(xs.view(np.int32), g["flt_xsum"].view(np.int32))
        np.testing.assert_array_equal(ys.view(np.int32), g["flt_ysum"].view(np.int32))
    r.close()


def test_tail_off_and_errors():
    from grotor_b200 import GrbError, Router
    from grotor_b200._abi import GRB_EINVAL
    from grotor_b200.synth import WORKLOADS, Design
    d = Design(WORKLOADS["small_64x64x5"].scaled(500, seed=43))
    r = Router(d.grid)
    r.upload_nets(d.nets)
    r.generate_batches_rsmt(d.order)
    r.set_stage_tail(ripup=True, view=False)
    with pytest.raises(GrbError) as e:  # nothing computed yet
        r.stage_tail()
    assert e.value.code == GRB_EINVAL
    r.lshape_route("persistent")
    is_of, view = r.stage_tail()
    assert view is None and len(is_of) == d.n_subnets
    r.set_stage_tail(ripup=False, view=False)
    r.reset()
    r.lshape_route("persistent")  # no tail: the stage alone
    r.close()
