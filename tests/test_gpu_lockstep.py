"""CUDA path vs the CPU restatement, batch by batch, through the C ABI.

Per batch: refresh_cost on the GPU, then
  * wcost/vcost within 1e-6 relative of the oracle's (CUDA __expf vs host expf),
  * presum bit-identical to the oracle's prefix of the GPU's own wcost,
  * routes word-identical to the oracle's DP on the GPU's own tables,
  * demand, timestamps and statistics identical after the commit.
"""
import numpy as np
import pytest

import oracle
from helpers import check_connected, orc_grid

pytestmark = pytest.mark.gpu

RTOL = 1e-6  # cost values: CUDA __expf vs host expf

CASES = {
    "64x64x5_1500": ("small_64x64x5", 1500, {}),
    "64x64x10_1500": ("small_64x64x5", 1500, {"cap_layers": 10, "seed": 21}),
    "37x70x7_800": ("small_64x64x5", 800, {"X": 37, "Y": 70, "cap_layers": 7, "seed": 22, "cap_lo": 1, "cap_hi": 4}),
    "48x40x3_600_tight": ("small_64x64x5", 600, {"X": 48, "Y": 40, "cap_layers": 3, "seed": 23, "cap_lo": 0, "cap_hi": 2}),
}


def _design(case):
    from grotor_b200.synth import WORKLOADS, Design
    wl, n, kw = CASES[case]
    return Design(WORKLOADS[wl].scaled(n, **kw))


@pytest.mark.parametrize("case", list(CASES))
def test_lockstep_against_oracle(case):
    from grotor_b200 import Router, plan_from_batches
    d = _design(case)
    g, n = d.grid, d.nets
    og = orc_grid(g)
    bo, nb = oracle.batches(g.X, g.Y, d.order, n.point_off, n.points, n.hseg_off, n.hsegs, n.vseg_off, n.vsegs,
                            1000000, 1)
    ids, off = plan_from_batches(d.order, bo, nb)
    r = Router(g)
    r.upload_nets(n)
    r.set_plan(ids, off)
    demand = np.zeros(g.cells, np.int32)
    ts = np.zeros(g.cells, np.int32)
    routes = np.zeros(int(n.route_off[-1]), np.int32)
    st = {"wirelength": 0.0, "vias": 0}
    for b in range(nb):
        stamp = b + 1
        sel = ids[off[b]:off[b + 1]]
        r.refresh_cost()
        t = r.read_tables()
        w, v = oracle.cost_full(og, demand)
        np.testing.assert_allclose(t["wcost"], w, rtol=RTOL, atol=0, err_msg=f"wcost batch {b}")
        np.testing.assert_allclose(t["vcost"], v, rtol=RTOL, atol=0, err_msg=f"vcost batch {b}")
        p = oracle.presum(og, t["wcost"])
        np.testing.assert_array_equal(p.view(np.int64), t["presum"].view(np.int64), err_msg=f"presum batch {b}")
        r.route_batch(b, stamp)
        gpu_routes = r.read_routes()
        assert oracle.lshape_batch(og, t["vcost"], t["presum"], sel, n.node_off, n.nodes, n.parents, n.route_off,
                                   routes) == 0
        for i in sel:
            a = n.route_off[i]
            np.testing.assert_array_equal(gpu_routes[a:a + routes[a]], routes[a:a + routes[a]],
                                          err_msg=f"routes of net {i} in batch {b}")
        r.commit_batch_demand(b, stamp, 1)
        oracle.commit_batch(og, sel, n.route_off, routes, stamp, 1, demand, ts, st)
        t2 = r.read_tables()
        np.testing.assert_array_equal(t2["demand_half"], demand, err_msg=f"demand batch {b}")
        np.testing.assert_array_equal(t2["timestamp"], ts, err_msg=f"timestamps batch {b}")
    s = r.stats()
    assert s["wirelength"] == st["wirelength"] and s["vias"] == st["vias"]
    check_connected(routes, n.route_off, n.node_off, n.nodes, g.X, g.Y, g.L, ids)
    r.close()


def test_ripup_roundtrip_zero_demand():
    """Ripping every batch up again (K = -1, later stamps) returns demand,
    wirelength and via count to zero."""
    from grotor_b200 import Router
    d = _design("64x64x10_1500")
    r = Router(d.grid)
    r.upload_nets(d.nets)
    r.generate_batches_rsmt(d.order, 1000000)
    st = r.lshape_route("persistent")
    assert st["wirelength"] > 0
    nb = st["n_batches"]
    stamp = st["stamp"]
    for b in range(nb):
        stamp += 1
        r.commit_batch_demand(b, stamp, -1)
    t = r.read_tables()
    assert not t["demand_half"].any()
    s = r.stats()
    assert s["wirelength"] == 0 and s["vias"] == 0
    r.close()
