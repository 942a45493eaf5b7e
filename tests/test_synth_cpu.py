"""Synthetic designs: seeded, and their topology is a valid stage input."""
import numpy as np
import pytest

from grotor_b200.synth import WORKLOADS, Design


@pytest.fixture(scope="module")
def design():
    return Design(WORKLOADS["medium_320x320x10"].scaled(3000, seed=5))


def test_deterministic():
    a = Design(WORKLOADS["small_64x64x5"].scaled(500, seed=9))
    b = Design(WORKLOADS["small_64x64x5"].scaled(500, seed=9))
    for k in ("node_off", "nodes", "parents", "points", "hsegs", "vsegs"):
        np.testing.assert_array_equal(getattr(a.nets, k), getattr(b.nets, k))
    np.testing.assert_array_equal(a.grid.capacity, b.grid.capacity)
    c = Design(WORKLOADS["small_64x64x5"].scaled(500, seed=10))
    assert not np.array_equal(a.grid.capacity, c.grid.capacity)


def test_trees_are_dfs_ordered(design):
    n = design.nets
    g = design.grid
    XY = g.X * g.Y
    for i in range(n.n):
        a, b = n.node_off[i], n.node_off[i + 1]
        par = n.parents[a:b]
        assert par[0] == -1
        assert np.all(par[1:] < np.arange(1, b - a)) and np.all(par[1:] >= 0)
        layers = n.nodes[a:b] // XY
        assert np.all(layers <= g.L)
        assert n.route_off[i + 1] - n.route_off[i] >= 1 + 8 * (b - a)


def test_subnets_at_most_12_pins_and_order(design):
    assert design.pin_count.max() <= 12
    assert np.all(np.diff(design.hpwl[design.order]) <= 0)
    assert sorted(design.order.tolist()) == list(range(design.n_subnets))


def test_geometry_contains_tree_nodes(design):
    n = design.nets
    g = design.grid
    XY = g.X * g.Y
    for i in range(0, n.n, 37):
        pts = set(n.points[n.point_off[i]:n.point_off[i + 1]].tolist())
        nodes = set((n.nodes[n.node_off[i]:n.node_off[i + 1]] % XY).tolist())
        assert nodes <= pts


def test_workload_distributions():
    d = Design(WORKLOADS["persistent_1600x1600x10"].scaled(20000, seed=7))
    assert d.grid.X == 1600 and d.grid.L == 9
    frac2 = np.mean(d.pin_count == 2)
    assert 0.45 < frac2 < 0.9
