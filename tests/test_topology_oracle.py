"""Topology construction on the CPU restatement (orc_build_topology).

Pinned to the reference: for every reference fixture, the trees the
reference's FLUTE step left in net::rsmt (dumped by oracle/_ref/ref_harness
topo) give exactly the reference's own depth-first arrays (Lshape_route,
lshape.cuh:85-98) and batching geometry (construct_rsmt, preprocess.hpp:
95-123).  Properties: trees given with relabelled nodes and shuffled adjacency
still flatten to a valid preorder (root first, parents before children) with
the same per-net geometry as sets; adjacency that is not a tree is refused.
"""
import numpy as np
import pytest

import oracle
from helpers import load_golden

KEYS = ("nodes", "parents", "point_off", "points", "hseg_off", "hsegs", "vseg_off", "vsegs")


@pytest.mark.parametrize("name", ["ref_32x32x10_400", "ref_64x64x10_2k", "ref_flt_48x48x10_1500"])
def test_trees_give_reference_topology(name):
    g = load_golden(name)
    L, X, Y, DIR = (int(v) for v in g["meta"])
    t = oracle.build_topology(X, Y, g["node_off"], g["rsmt_pos"], g["rsmt_adj_off"], g["rsmt_adj"])
    for k in KEYS:
        assert np.array_equal(t[k], g[k]), k


def _per_net_sorted(off, arr, w):
    a = np.asarray(arr).reshape(-1, w)
    net = np.repeat(np.arange(len(off) - 1), np.diff(off))
    return a[np.lexsort(tuple(a[:, k] for k in range(w - 1, -1, -1)) + (net,))]


def test_shuffled_trees_keep_geometry_and_preorder():
    from grotor_b200.synth import WORKLOADS, Design, steiner_trees
    d = Design(WORKLOADS["small_64x64x5"].scaled(3000))
    n = d.nets
    plain = steiner_trees(n)
    t = oracle.build_topology(d.grid.X, d.grid.Y, plain.node_off, plain.pos, plain.adj_off, plain.adj)
    assert np.array_equal(t["nodes"], n.nodes) and np.array_equal(t["parents"], n.parents)
    s = steiner_trees(n, shuffle_seed=7)
    u = oracle.build_topology(d.grid.X, d.grid.Y, s.node_off, s.pos, s.adj_off, s.adj)
    off = np.asarray(n.node_off)
    for i in range(n.n):
        par = u["parents"][off[i]:off[i + 1]]
        assert par[0] == -1 and np.all(par[1:] >= 0) and np.all(par[1:] < np.arange(1, len(par)))
        assert sorted(u["nodes"][off[i]:off[i + 1]]) == sorted(n.nodes[off[i]:off[i + 1]])
    assert np.array_equal(u["point_off"], t["point_off"])
    for k, w, o in (("points", 1, "point_off"), ("hsegs", 2, "hseg_off"), ("vsegs", 2, "vseg_off")):
        assert np.array_equal(_per_net_sorted(u[o], u[k], w), _per_net_sorted(t[o], t[k], w)), k


def test_non_trees_are_refused():
    node_off = np.array([0, 3], np.int32)
    pos = np.array([0, 5, 9], np.int32)
    # neighbour index outside the net
    with pytest.raises(ValueError):
        oracle.build_topology(4, 4, node_off, pos, np.array([0, 1, 2, 3], np.int32), np.array([1, 3, 0], np.int32))
    # node 2 never reached (0-1 joined twice)
    with pytest.raises(ValueError):
        oracle.build_topology(4, 4, node_off, pos, np.array([0, 2, 4, 4], np.int32),
                              np.array([1, 1, 0, 0], np.int32))
    # a valid path 0-1-2
    t = oracle.build_topology(4, 4, node_off, pos, np.array([0, 1, 3, 4], np.int32), np.array([1, 0, 2, 1], np.int32))
    assert list(t["parents"]) == [-1, 0, 1] and list(t["nodes"]) == [0, 5, 9]
