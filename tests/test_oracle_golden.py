"""Pin the CPU restatement (oracle/) against outputs of the reference router.

The fixtures in tests/golden/ come from the reference's own code
(oracle/_ref/ref_harness, see make_golden.py): its CPU batches and FLUTE
topology (generated here), and -- produced on a GPU -- its L-shape routes,
demand, statistics and cost tables.  Tests needing the GPU-produced part skip
until those keys are present.
"""
import numpy as np
import pytest

import oracle
from helpers import float_demand_to_half, golden_grid, golden_nets, load_golden, orc_grid

NAMES = ["ref_64x64x10_2k", "ref_32x32x10_400"]


def need(g, *keys):
    missing = [k for k in keys if k not in g]
    if missing:
        pytest.skip(f"fixture lacks GPU-produced keys {missing}")


@pytest.mark.parametrize("name", NAMES)
def test_batching_equals_reference(name):
    g = load_golden(name)
    L, X, Y, DIR = g["meta"]
    bo, nb = oracle.batches(X, Y, g["order"], g["point_off"], g["points"], g["hseg_off"], g["hsegs"],
                            g["vseg_off"], g["vsegs"], 1000000, 1)
    assert nb == int(g["batch_of"].max()) + 1
    np.testing.assert_array_equal(bo, g["batch_of"])


@pytest.mark.parametrize("name", NAMES)
def test_batching_capacity_limit(name):
    """Small batch limits exercise the 'batch full' branch; every batch holds at
    most `limit` nets and the result equals a direct replay of the rule."""
    g = load_golden(name)
    L, X, Y, DIR = g["meta"]
    for limit in (1, 7, 64):
        bo, nb = oracle.batches(X, Y, g["order"], g["point_off"], g["points"], g["hseg_off"], g["hsegs"],
                                g["vseg_off"], g["vsegs"], limit, 1)
        assert np.bincount(bo).max() <= limit
        if limit == 1:
            np.testing.assert_array_equal(bo, np.arange(len(bo)))


def test_presum_order_equals_reference():
    g = load_golden("ref_32x32x10_400")
    need(g, "ref_wcost", "ref_presum")
    og = orc_grid(golden_grid(g))
    p = oracle.presum(og, g["ref_wcost"])
    np.testing.assert_array_equal(p.view(np.int64), g["ref_presum"].view(np.int64))


def test_cost_model_matches_reference():
    g = load_golden("ref_32x32x10_400")
    need(g, "ref_wcost", "ref_vcost", "ref_demand")
    og = orc_grid(golden_grid(g))
    w, v = oracle.cost_full(og, float_demand_to_half(g["ref_demand"]))
    np.testing.assert_allclose(w, g["ref_wcost"], rtol=1e-6, atol=0)
    np.testing.assert_allclose(v, g["ref_vcost"], rtol=1e-6, atol=0)


def test_dp_on_reference_tables_equals_reference_routes():
    """Given the reference's own cost tables before a batch, the oracle's DP
    reproduces the reference's routes for that batch word for word."""
    g = load_golden("ref_32x32x10_400")
    need(g, "snap_vcost", "snap_presum", "snap_routes", "snap_batch")
    grid, nets = golden_grid(g), golden_nets(g)
    og = orc_grid(grid)
    b = int(g["snap_batch"][0])
    ids = g["ids"][g["batch_off"][b]:g["batch_off"][b + 1]]
    routes = np.zeros(int(nets.route_off[-1]), np.int32)
    rc = oracle.lshape_batch(og, g["snap_vcost"], g["snap_presum"], ids, nets.node_off, nets.nodes, nets.parents,
                             nets.route_off, routes)
    assert rc == 0
    ref = g["snap_routes"]
    for i in ids:
        a, e = nets.route_off[i], nets.route_off[i + 1]
        n = routes[a]
        np.testing.assert_array_equal(routes[a:a + n], ref[a:a + n], err_msg=f"net {i}")


def test_snapshot_costs_match_oracle():
    g = load_golden("ref_32x32x10_400")
    need(g, "snap_wcost", "snap_vcost", "snap_presum", "snap_demand")
    og = orc_grid(golden_grid(g))
    w, v = oracle.cost_full(og, float_demand_to_half(g["snap_demand"]))
    np.testing.assert_allclose(w, g["snap_wcost"], rtol=1e-6, atol=0)
    np.testing.assert_allclose(v, g["snap_vcost"], rtol=1e-6, atol=0)
    p = oracle.presum(og, g["snap_wcost"])
    np.testing.assert_array_equal(p.view(np.int64), g["snap_presum"].view(np.int64))


@pytest.mark.parametrize("name", NAMES)
def test_commit_replay_equals_reference_demand(name):
    """Replaying the reference's routes through the oracle's commit, batch by
    batch, reproduces the reference's demand and statistics exactly."""
    g = load_golden(name)
    need(g, "ref_routes", "ref_demand", "ref_stats")
    grid, nets = golden_grid(g), golden_nets(g)
    og = orc_grid(grid)
    demand = np.zeros(grid.cells, np.int32)
    ts = np.zeros(grid.cells, np.int32)
    st = {"wirelength": 0.0, "vias": 0}
    routes = g["ref_routes"][:-1]
    off = g["batch_off"]
    for b in range(len(off) - 1):
        oracle.commit_batch(og, g["ids"][off[b]:off[b + 1]], nets.route_off, routes, b + 1, 1, demand, ts, st)
    np.testing.assert_array_equal(demand, float_demand_to_half(g["ref_demand"]))
    assert st["wirelength"] == g["ref_stats"][0]
    assert st["vias"] + int(g["pin_vias"][0]) == int(g["ref_stats"][1])


@pytest.mark.parametrize("name", NAMES)
def test_full_stage_routes_match_reference(name):
    """Whole stage on the CPU (host expf in place of __expf): the routes equal
    the reference's on every net whose decisions are not within an ulp tie;
    the two designs here have none."""
    g = load_golden(name)
    need(g, "ref_routes")
    grid, nets = golden_grid(g), golden_nets(g)
    r = oracle.lshape_stage(orc_grid(grid), g["ids"], g["batch_off"], nets.node_off, nets.nodes, nets.parents,
                            nets.route_off, threads=4)
    assert r["status"] == 0
    np.testing.assert_array_equal(r["routes"], g["ref_routes"][:-1])
