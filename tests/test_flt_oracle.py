"""The FLT-stage oracle against the reference router's own FLT run.

Fixture: tests/golden/ref_flt_*.npz (make_golden.py --flt).  On the
reference's topology and plan the CPU restatement replays the L-shape stage,
the rip-up classification, the FLT batching and the FLT stage
(flt.cuh:141-168 over the reference's own DAGs) and must reproduce the
reference's demand and statistics exactly and every net's route geometry
(unit wire edges and via stacks).  The restatement's cost tables use the
host's expf instead of CUDA's __expf (agreement within 1e-6 relative), so
where two candidates tie in real arithmetic -- one straight run split at
different DAG nodes -- float rounding may pick the other split; the segment
multisets themselves are compared exactly on the GPU (test_gpu_flt.py).
"""
import numpy as np
import pytest

import oracle
from helpers import (flt_by_net, float_demand_to_half, golden_grid, golden_nets, load_golden, orc_grid,
                     ref_routes2_of, route_geometry, segment_multiset)

NAMES = ["ref_flt_48x48x10_1500"]


def need_flt(g):
    if "flt_after_demand" not in g:
        pytest.skip("fixture lacks the reference FLT run")


def oracle_before_flt(g):
    import oracle
    grid = golden_grid(g)
    nets = golden_nets(g)
    og = orc_grid(grid)
    st = oracle.lshape_stage(og, g["ids"], g["batch_off"], nets.node_off, nets.nodes, nets.parents, nets.route_off)
    st["vias"] += int(g["pin_vias"][0])
    return og, nets, st


@pytest.mark.parametrize("name", NAMES)
def test_state_before_flt(name):
    g = load_golden(name)
    need_flt(g)
    _, _, st = oracle_before_flt(g)
    assert st["status"] == 0
    np.testing.assert_array_equal(st["demand_half"], float_demand_to_half(g["flt_before_demand"]))
    assert st["wirelength"] == g["flt_before_stats"][0]
    assert st["vias"] == int(g["flt_before_stats"][1])
    assert st["stamp"] == int(g["flt_before_stats"][2])


@pytest.mark.parametrize("name", NAMES)
def test_ripup_set_and_flt_batches(name):
    import oracle
    from grotor_b200.router import plan_from_batches
    g = load_golden(name)
    need_flt(g)
    og, nets, st = oracle_before_flt(g)
    is_of = oracle.ripup_classify(og, st["demand_half"], 0, nets.route_off, st["routes"])
    np.testing.assert_array_equal(np.flatnonzero(is_of), g["flt_of_nets"])
    _, geom, _ = flt_by_net(g)
    X, Y = int(g["meta"][1]), int(g["meta"][2])
    bo, nb = oracle.batches(X, Y, g["flt_nets"], *geom, 300000)
    ids, off = plan_from_batches(g["flt_nets"], bo, nb)
    np.testing.assert_array_equal(ids, g["flt_batch_ids"])
    np.testing.assert_array_equal(off, g["flt_batch_off"])


@pytest.mark.parametrize("name", NAMES)
def test_flt_stage_equals_reference(name):
    import oracle
    g = load_golden(name)
    need_flt(g)
    og, nets, st = oracle_before_flt(g)
    dags, _, route2_off = flt_by_net(g)
    out = oracle.flt_stage(og, dags, g["flt_batch_ids"], g["flt_batch_off"], nets.route_off, st["routes"],
                           route2_off, st["demand_half"], st["timestamp"], st["stamp"], True,
                           wirelength=st["wirelength"], vias=st["vias"])
    assert out["status"] == 0
    np.testing.assert_array_equal(out["demand_half"], float_demand_to_half(g["flt_after_demand"]))
    assert out["wirelength"] == g["flt_after_stats"][0]
    assert out["vias"] == int(g["flt_after_stats"][1])
    assert out["stamp"] == int(g["flt_after_stats"][2])
    X, Y = int(g["meta"][1]), int(g["meta"][2])
    same_segments = 0
    for net in g["flt_nets"]:
        ours, ref = out["routes2"][route2_off[net]:route2_off[net + 1]], ref_routes2_of(g, net)
        assert route_geometry(ours, X, Y) == route_geometry(ref, X, Y), f"net {net}"
        same_segments += segment_multiset(ours) == segment_multiset(ref)
    assert same_segments >= 0.95 * len(g["flt_nets"])


def test_congestion_view_equals_reference():
    """The oracle's congestion view (congestion.cuh:60-112) of the reference's
    demand after its L-shape stage equals the view the reference itself
    computed for its FLT topology builder, bit for bit: the per-cell flag and
    both row/column float prefixes (whose association the restatement
    follows)."""
    g = load_golden("ref_flt_48x48x10_1500")
    if "flt_congestion" not in g:
        pytest.skip("fixture lacks the reference congestion view")
    og = orc_grid(golden_grid(g))
    cong, xs, ys = oracle.congestion_view(og, float_demand_to_half(g["flt_before_demand"]))
    np.testing.assert_array_equal(cong, g["flt_congestion"].astype(np.uint8))
    np.testing.assert_array_equal(xs.view(np.int32), g["flt_xsum"].view(np.int32))
    np.testing.assert_array_equal(ys.view(np.int32), g["flt_ysum"].view(np.int32))
    assert cong.sum() > 0 and np.count_nonzero(xs) > 0
