"""The CUDA Z-shape stage and bounding-box batching against the reference's
own Z-shape run (its GGR build; fixtures tests/golden/ref_z_*.npz).

Given the reference's first-fit groups, the GPU refinement reproduces its
bounding-box batches; on those batches and its encoded trees, under the GGR
integer wire costs, the plain (thread-per-net commit), graph and persistent
executors reproduce every route word, the demand and the statistics exactly
(the Z-shape DP is integer arithmetic).
"""
import numpy as np
import pytest

from helpers import float_demand_to_half, golden_grid, load_golden

pytestmark = pytest.mark.gpu

NAMES = ["ref_z_48x48x10_1500", "ref_z_40x56x10_800"]
ROUTE_PER_PIN_GGR = 256  # pipeline_ggr.hpp:9


def zrouter(g):
    from grotor_b200 import Router
    from grotor_b200.router import NetArrays
    n = len(g["pin_acc_num"]) - 1
    z = np.zeros(n + 1, np.int32)
    e = np.zeros(0, np.int32)
    route_off = g["pin_acc_num"].astype(np.int64) * ROUTE_PER_PIN_GGR
    r = Router(golden_grid(g))
    r.upload_nets(NetArrays(z, e, e, route_off, z, e, z, e, z, e))
    r.upload_zshape({"node_off": g["z_node_off"], "coord": g["z_coord"], "child": g["z_child"]})
    r.set_wire_cost_mode(True)
    if "pin_vias" in g:
        r.set_stats(0.0, int(g["pin_vias"][0]))
    return r


def group_plan(g):
    """First-fit groups reversed into execution order (as grb_plan_batches leaves them)."""
    go = g["z_group_off"]
    groups = [g["z_group_ids"][go[k]:go[k + 1]] for k in range(len(go) - 1)][::-1]
    return np.concatenate(groups).astype(np.int32), np.cumsum([0] + [len(x) for x in groups]).astype(np.int32)


@pytest.mark.parametrize("name", NAMES)
def test_bbox_batches_on_gpu(name):
    g = load_golden(name)
    r = zrouter(g)
    for bbox in (None, g["z_bbox"]):
        r.set_plan(*group_plan(g))
        nb = r.plan_bbox_batches(250, bbox)
        ids, off = r.plan()
        assert nb == len(g["z_batch_off"]) - 1
        np.testing.assert_array_equal(ids, g["z_batch_ids"])
        np.testing.assert_array_equal(off, g["z_batch_off"])
    r.close()


@pytest.mark.parametrize("mode", ["plain", "graph", "persistent"])
@pytest.mark.parametrize("name", NAMES)
def test_zshape_stage_equals_reference(name, mode):
    g = load_golden(name)
    r = zrouter(g)
    r.set_plan(g["z_batch_ids"], g["z_batch_off"])
    st = r.zshape_route(mode)
    np.testing.assert_array_equal(r.read_routes(), g["z_routes"][:-1])
    np.testing.assert_array_equal(r.read_tables()["demand_half"], float_demand_to_half(g["z_demand"]))
    assert st["wirelength"] == g["z_stats"][0]
    assert st["stamp"] == int(g["z_stats"][2])
    if "pin_vias" in g:
        assert st["vias"] == int(g["z_stats"][1])
    r.close()


def test_zshape_synthetic_design_equals_oracle():
    """On a seeded 320x320x10 design (trees from the workload generator): GPU
    first-fit + bounding-box batches equal the oracle's refinement of the
    same groups, and the Z-shape stage's routes, demand and statistics equal
    the oracle's."""
    import oracle
    from grotor_b200 import Router
    from grotor_b200.router import NetArrays
    from grotor_b200.synth import WORKLOADS, Design
    from helpers import orc_grid
    d = Design(WORKLOADS["medium_320x320x10"].scaled(6000, seed=47))
    z = d.zshape_trees()
    n = d.nets
    zn = np.diff(z["node_off"]).astype(np.int64)
    route_off = np.concatenate([[0], np.cumsum(1 + 64 * zn)]).astype(np.int64)
    nets = NetArrays(n.node_off, n.nodes, n.parents, route_off, n.point_off, n.points, n.hseg_off, n.hsegs,
                     n.vseg_off, n.vsegs)
    r = Router(d.grid)
    r.upload_nets(nets)
    r.upload_zshape(z)
    r.set_wire_cost_mode(True)
    r.generate_batches_rsmt(d.order, 1000000)
    gids, goff = r.plan()
    # oracle refinement of the same groups (execution order: groups reversed)
    bbox = np.zeros((n.n, 4), np.int32)
    for i in range(n.n):
        c = z["coord"][z["node_off"][i]:z["node_off"][i + 1]] % (d.grid.X * d.grid.Y)
        xs, ys = c // d.grid.Y, c % d.grid.Y
        bbox[i] = (xs.min(), xs.max(), ys.min(), ys.max())
    groups = [gids[goff[k]:goff[k + 1]] for k in range(len(goff) - 1)][::-1]
    ref = []
    for grp in groups:
        ref += oracle.bbox_batches(d.grid.X, d.grid.Y, grp, bbox.reshape(-1))
    ref = ref[::-1]
    nb = r.plan_bbox_batches(250)
    ids, off = r.plan()
    assert nb == len(ref)
    np.testing.assert_array_equal(ids, np.concatenate([np.asarray(b, np.int32) for b in ref]))
    og = orc_grid(d.grid)
    og2 = oracle.OrcGrid(og.L, og.X, og.Y, og.DIR, og.unit_wire, og.unit_via, og.short_costs, og.x_edge_len,
                         og.y_edge_len, og.capacity, og.of_cost_scale, integer_wire=True)
    out = oracle.zshape_stage(og2, z, ids, off, route_off)
    assert out["status"] == 0
    for mode in ("persistent", "plain"):
        r.reset()
        st = r.zshape_route(mode)
        np.testing.assert_array_equal(r.read_routes(), out["routes"])
        np.testing.assert_array_equal(r.read_tables()["demand_half"], out["demand_half"])
        assert st["wirelength"] == out["wirelength"] and st["vias"] == out["vias"]
    r.close()
