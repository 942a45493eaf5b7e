"""The three executors (plain launches, CUDA graph, persistent kernel) give
identical routes, demand and cost tables; the rip-up classification and the
congestion view equal the oracle's."""
import numpy as np
import pytest

import oracle
from helpers import check_connected, orc_grid

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def medium():
    from grotor_b200.synth import WORKLOADS, Design
    return Design(WORKLOADS["medium_320x320x10"].scaled(30000, seed=41))


def _run(design, mode, router=None):
    from grotor_b200 import Router
    r = router or Router(design.grid)
    if router is None:
        r.upload_nets(design.nets)
        r.generate_batches_rsmt(design.order, 1000000)
    else:
        r.reset()
    st = r.lshape_route(mode)
    return r, st, r.read_routes(), r.read_tables()


def test_modes_identical(medium):
    r, st_p, routes_p, t_p = _run(medium, "plain")
    _, st_g, routes_g, t_g = _run(medium, "graph", r)
    _, st_s, routes_s, t_s = _run(medium, "persistent", r)
    for routes, t, st in ((routes_g, t_g, st_g), (routes_s, t_s, st_s)):
        np.testing.assert_array_equal(routes, routes_p)
        np.testing.assert_array_equal(t["demand_half"], t_p["demand_half"])
        np.testing.assert_array_equal(t["timestamp"], t_p["timestamp"])
        assert st["wirelength"] == st_p["wirelength"] and st["vias"] == st_p["vias"]
    # After one more refresh every mode leaves identical cost tables.
    r.refresh_cost()
    t1 = r.read_tables()
    g = medium.grid
    og = orc_grid(g)
    w, v = oracle.cost_full(og, t1["demand_half"])
    np.testing.assert_allclose(t1["wcost"], w, rtol=1e-6, atol=0)
    np.testing.assert_allclose(t1["vcost"], v, rtol=1e-6, atol=0)
    np.testing.assert_array_equal(oracle.presum(og, t1["wcost"]).view(np.int64), t1["presum"].view(np.int64))
    ids, _ = r.plan()
    check_connected(routes_s, medium.nets.route_off, medium.nets.node_off, medium.nets.nodes, g.X, g.Y, g.L,
                    ids[:: max(1, len(ids) // 3000)])
    r.close()


def test_persistent_twice_and_commit_replay(medium):
    """Running the persistent stage twice from reset gives the same result, and
    replaying its routes through the oracle commit reproduces its demand."""
    r, st1, routes1, t1 = _run(medium, "persistent")
    _, st2, routes2, t2 = _run(medium, "persistent", r)
    np.testing.assert_array_equal(routes1, routes2)
    np.testing.assert_array_equal(t1["demand_half"], t2["demand_half"])
    ids, off = r.plan()
    g = medium.grid
    og = orc_grid(g)
    demand = np.zeros(g.cells, np.int32)
    ts = np.zeros(g.cells, np.int32)
    st = {"wirelength": 0.0, "vias": 0}
    for b in range(len(off) - 1):
        oracle.commit_batch(og, ids[off[b]:off[b + 1]], medium.nets.route_off, routes1, b + 1, 1, demand, ts, st)
    np.testing.assert_array_equal(demand, t1["demand_half"])
    assert st["wirelength"] == st1["wirelength"] and st["vias"] == st1["vias"]
    r.close()


def test_ripup_and_congestion_view(medium):
    r, st, routes, t = _run(medium, "persistent")
    g = medium.grid
    og = orc_grid(g)
    for thr in (0, 1, -2):
        got = r.ripup(thr)
        ref = oracle.ripup_classify(og, t["demand_half"], thr, medium.nets.route_off, routes)
        np.testing.assert_array_equal(got, ref)
    cong, xs, ys = r.congestion_view()
    c2, x2, y2 = oracle.congestion_view(og, t["demand_half"])
    np.testing.assert_array_equal(cong, c2)
    np.testing.assert_array_equal(xs.view(np.int32), x2.view(np.int32))
    np.testing.assert_array_equal(ys.view(np.int32), y2.view(np.int32))
    r.close()
