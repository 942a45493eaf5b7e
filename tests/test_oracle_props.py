"""Properties of the CPU restatement that hold independently of the reference."""
import numpy as np
import pytest

import oracle
from helpers import check_connected, net_routes, orc_grid


def _grid(L=5, X=40, Y=33, DIR=1, seed=0, cap=(0, 6)):
    from grotor_b200.router import GridArrays
    rng = np.random.default_rng(seed)
    return GridArrays(L, X, Y, DIR, 1.0, 2.0, rng.uniform(0.5, 2.0, L), rng.integers(1, 4, X - 1),
                      rng.integers(1, 4, Y - 1), rng.integers(cap[0], cap[1] + 1, (L, X, Y)).astype(np.float32))


@pytest.mark.parametrize("X,Y", [(2, 2), (3, 70), (64, 1), (129, 7), (1600, 3)])
def test_presum_single_pass_equals_logstep(X, Y):
    Y = max(Y, 2)
    g = orc_grid(_grid(L=3, X=X, Y=Y, seed=X * 31 + Y))
    w = np.random.default_rng(X + Y).uniform(0, 1e3, g.cells).astype(np.float32)
    a = oracle.presum(g, w)
    b = oracle.presum_logstep(g, w)
    np.testing.assert_array_equal(a.view(np.int64), b.view(np.int64))


def test_presum_is_exclusive_prefix():
    g = orc_grid(_grid(L=2, X=17, Y=9))
    w = np.ones(g.cells, np.float32)
    p = oracle.presum(g, w).reshape(g.L, g.X, g.Y)
    # layer 0 (DIR=1): along y; layer 1: along x
    np.testing.assert_array_equal(p[0, 3, :], np.arange(g.Y))
    np.testing.assert_array_equal(p[1, :, 5], np.arange(g.X))


def test_costs_monotone_in_demand():
    g = orc_grid(_grid(seed=3))
    d0 = np.zeros(g.cells, np.int32)
    w0, v0 = oracle.cost_full(g, d0)
    w1, v1 = oracle.cost_full(g, d0 + 4)
    assert np.all(w1 >= w0) and np.all(v1 >= v0)


@pytest.fixture(scope="module")
def small_design():
    from grotor_b200.synth import WORKLOADS, Design
    return Design(WORKLOADS["small_64x64x5"].scaled(1500))


def _stage(design, threads=2):
    from grotor_b200.router import plan_from_batches
    g = design.grid
    n = design.nets
    bo, nb = oracle.batches(g.X, g.Y, design.order, n.point_off, n.points, n.hseg_off, n.hsegs, n.vseg_off,
                            n.vsegs, 1000000, 1)
    ids, off = plan_from_batches(design.order, bo, nb)
    r = oracle.lshape_stage(orc_grid(g), ids, off, n.node_off, n.nodes, n.parents, n.route_off, threads=threads)
    return ids, off, r


def test_stage_routes_connected(small_design):
    d = small_design
    ids, off, r = _stage(d)
    assert r["status"] == 0
    g = d.grid
    check_connected(r["routes"], d.nets.route_off, d.nets.node_off, d.nets.nodes, g.X, g.Y, g.L, ids)


def test_stage_independent_of_thread_count(small_design):
    _, _, a = _stage(small_design, threads=1)
    _, _, b = _stage(small_design, threads=7)
    np.testing.assert_array_equal(a["routes"], b["routes"])
    np.testing.assert_array_equal(a["demand_half"], b["demand_half"])


def test_commit_then_ripup_restores_demand(small_design):
    """Committing a batch and ripping the same batch up with a later stamp
    (flt.cuh:143-150) returns demand to its previous value."""
    d = small_design
    ids, off, r = _stage(d)
    g = orc_grid(d.grid)
    demand = r["demand_half"].copy()
    ts = r["timestamp"].copy()
    st = {"wirelength": 0.0, "vias": 0}
    b = len(off) - 2
    sel = ids[off[b]:off[b + 1]]
    stamp = r["stamp"]
    oracle.commit_batch(g, sel, d.nets.route_off, r["routes"], stamp + 1, -1, demand, ts, st)
    oracle.commit_batch(g, sel, d.nets.route_off, r["routes"], stamp + 2, +1, demand, ts, st)
    np.testing.assert_array_equal(demand, r["demand_half"])
    assert st["wirelength"] == 0 and st["vias"] == 0


def test_wirelength_equals_route_length(small_design):
    d = small_design
    ids, off, r = _stage(d)
    g = d.grid
    XY = g.X * g.Y
    total = 0
    for i in ids:
        rr = net_routes(r["routes"], d.nets.route_off, i)
        for k in range(1, len(rr), 2):
            a, b = int(rr[k]), int(rr[k + 1])
            if a // XY == b // XY:
                total += abs(a % XY // g.Y - b % XY // g.Y) + abs(a % g.Y - b % g.Y)
    assert total == r["wirelength"]
