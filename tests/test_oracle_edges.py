"""Edge cases of the oracle.  First-fit batching, whatever the conflict rule:
an empty order, a single net, the batch-size limit, and the first-fit shape
of the result (a net opens at most one new batch, and never skips one).
Rip-up classification at threshold extremes, the congestion view of an
empty grid, and the execution plan built from a first-fit result."""
import numpy as np
import pytest

import oracle


@pytest.fixture(scope="module")
def design():
    from grotor_b200.synth import WORKLOADS, Design
    return Design(WORKLOADS["small_64x64x5"].scaled(400, seed=21))


def _batches(d, order, limit):
    n = d.nets
    return oracle.batches(d.grid.X, d.grid.Y, order, n.point_off, n.points, n.hseg_off, n.hsegs, n.vseg_off,
                          n.vsegs, limit, 1)


def test_empty_order(design):
    bo, nb = _batches(design, np.zeros(0, np.int32), 10)
    assert nb == 0 and len(bo) == 0


def test_single_net(design):
    bo, nb = _batches(design, design.order[:1], 10)
    assert nb == 1 and bo.tolist() == [0]


def test_limit_one_gives_one_batch_per_net(design):
    order = design.order[:200]
    bo, nb = _batches(design, order, 1)
    assert nb == len(order)
    np.testing.assert_array_equal(bo, np.arange(len(order)))


@pytest.mark.parametrize("limit", [3, 17, 1000000])
def test_first_fit_shape_and_limit(design, limit):
    bo, nb = _batches(design, design.order, limit)
    assert bo.min() == 0 and bo.max() == nb - 1
    opened = -1
    for b in bo:  # batch indices appear in first-fit order
        assert b <= opened + 1
        opened = max(opened, int(b))
    assert np.bincount(bo, minlength=nb).max() <= limit


def _routed(d):
    from grotor_b200.router import plan_from_batches
    from helpers import orc_grid
    n = d.nets
    bo, nb = _batches(d, d.order, 1000000)
    ids, off = plan_from_batches(d.order, bo, nb)
    r = oracle.lshape_stage(orc_grid(d.grid), ids, off, n.node_off, n.nodes, n.parents, n.route_off, threads=2)
    assert r["status"] == 0
    return orc_grid(d.grid), r


def _wire_length(d, routes, i):
    from helpers import net_routes
    g = d.grid
    XY = g.X * g.Y
    rr = net_routes(routes, d.nets.route_off, i)
    total = 0
    for k in range(1, len(rr), 2):
        a, b = int(rr[k]), int(rr[k + 1])
        if a // XY == b // XY:
            total += abs(a % XY // g.Y - b % XY // g.Y) + abs(a % g.Y - b % g.Y)
    return total


def test_ripup_threshold_extremes(design):
    """A net is ripped up when more than 10 unit edges of its wires carry
    overflow (congestion.cuh:114-136): with a threshold below every demand
    every edge counts, so exactly the nets longer than 10 edges are taken;
    with a threshold above every demand none is."""
    g, r = _routed(design)
    none = oracle.ripup_classify(g, r["demand_half"], 10**6, design.nets.route_off, r["routes"])
    assert not none.any()
    every = oracle.ripup_classify(g, r["demand_half"], -10**6, design.nets.route_off, r["routes"])
    want = np.array([_wire_length(design, r["routes"], i) > 10 for i in range(design.nets.n)], np.uint8)
    assert want.any() and not want.all()
    np.testing.assert_array_equal(every, want)


def test_congestion_view_without_demand(design):
    """No demand and non-negative capacities: no congested position and all
    running sums zero."""
    g, _ = _routed(design)
    cong, xs, ys = oracle.congestion_view(g, np.zeros(g.cells, np.int32))
    assert not cong.any()
    assert not xs.any() and not ys.any()


def test_plan_from_batches_reverses_and_keeps_order(design):
    """The execution plan runs the last first-fit batch first
    (lshape.cuh:70-77); inside a batch the nets keep their order."""
    from grotor_b200.router import plan_from_batches
    bo, nb = _batches(design, design.order, 37)
    ids, off = plan_from_batches(design.order, bo, nb)
    assert off[0] == 0 and off[-1] == len(design.order) and len(off) == nb + 1
    assert sorted(ids.tolist()) == sorted(design.order.tolist())
    for k in range(nb):
        want = [int(n) for n, b in zip(design.order, bo) if b == nb - 1 - k]
        assert ids[off[k]:off[k + 1]].tolist() == want
    e_ids, e_off = plan_from_batches(np.zeros(0, np.int32), np.zeros(0, np.int32), 0)
    assert len(e_ids) == 0 and e_off.tolist() == [0]
