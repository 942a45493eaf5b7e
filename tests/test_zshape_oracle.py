"""The Z-shape oracle against the reference router's own Z-shape run.

Fixtures: tests/golden/ref_z_*.npz (make_golden.py --zshape, the reference's
GGR build).  On the reference's first-fit groups, net boxes and encoded trees
the CPU restatement reproduces the reference's bounding-box batches
(zshape_topology.hpp:7-57) and, under the GGR integer wire costs, every route
word of the Z-shape stage (zshape.cuh:42-404, zshape_topology.hpp:249-290),
the demand and the statistics.  The Z-shape DP is integer arithmetic, so the
agreement is exact.
"""
import numpy as np
import pytest

from helpers import float_demand_to_half, golden_grid, load_golden

NAMES = ["ref_z_48x48x10_1500", "ref_z_40x56x10_800"]
ROUTE_PER_PIN_GGR = 256  # pipeline_ggr.hpp:9


def zgrid(g):
    import oracle
    gr = golden_grid(g)
    return oracle.OrcGrid(gr.L, gr.X, gr.Y, gr.DIR, gr.unit_wire, gr.unit_via, gr.short_costs, gr.x_edge_len,
                          gr.y_edge_len, gr.capacity, gr.of_cost_scale, integer_wire=True)


def bbox_plan(g):
    """First-fit groups refined by boxes, reversed (pipeline_ggr.hpp:51-55)."""
    import oracle
    X, Y = int(g["meta"][1]), int(g["meta"][2])
    go = g["z_group_off"]
    batches = []
    for k in range(len(go) - 1):
        batches += oracle.bbox_batches(X, Y, g["z_group_ids"][go[k]:go[k + 1]], g["z_bbox"])
    batches = batches[::-1]
    ids = np.concatenate([np.asarray(b, np.int32) for b in batches])
    return ids, np.cumsum([0] + [len(b) for b in batches]).astype(np.int32)


@pytest.mark.parametrize("name", NAMES)
def test_bbox_batches_equal_reference(name):
    g = load_golden(name)
    ids, off = bbox_plan(g)
    np.testing.assert_array_equal(ids, g["z_batch_ids"])
    np.testing.assert_array_equal(off, g["z_batch_off"])
    assert np.all(np.diff(off) <= 250)


@pytest.mark.parametrize("name", NAMES)
def test_zshape_stage_equals_reference(name):
    import oracle
    g = load_golden(name)
    route_off = g["pin_acc_num"].astype(np.int64) * ROUTE_PER_PIN_GGR
    trees = {"node_off": g["z_node_off"], "coord": g["z_coord"], "child": g["z_child"]}
    pin_vias = int(g["pin_vias"][0]) if "pin_vias" in g else None
    out = oracle.zshape_stage(zgrid(g), trees, g["z_batch_ids"], g["z_batch_off"], route_off,
                              vias=pin_vias or 0)
    assert out["status"] == int(g["z_stats"][3]) == 0
    np.testing.assert_array_equal(out["routes"], g["z_routes"][:-1])
    np.testing.assert_array_equal(out["demand_half"], float_demand_to_half(g["z_demand"]))
    assert out["wirelength"] == g["z_stats"][0]
    assert out["stamp"] == int(g["z_stats"][2])
    if pin_vias is not None:
        assert out["vias"] == int(g["z_stats"][1])
