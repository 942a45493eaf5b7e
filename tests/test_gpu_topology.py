"""Topology construction on the GPU (grb_build_topology).

From the Steiner trees of the reference's FLUTE step (dumped by
oracle/_ref/ref_harness topo), the device builds exactly the reference's own
depth-first arrays and batching geometry.  On seeded designs with relabelled,
re-rooted trees and shuffled adjacency (120,000 nets) and on the 900,000-net
design, every array equals the CPU restatement's.  The L-shape stage on the
device-built nets gives the same batches, routes and demand as on the
host-built ones.  Adjacency that is not a tree is refused with GRB_EINVAL and
the context stays usable.
"""
import numpy as np
import pytest

import oracle
from helpers import golden_grid, load_golden

pytestmark = pytest.mark.gpu

KEYS = ("node_off", "nodes", "parents", "point_off", "points", "hseg_off", "hsegs", "vseg_off", "vsegs")


def _equal(a, b, what):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, f"{what}: shape {a.shape} vs {b.shape}"
    bad = np.flatnonzero(a != b)
    assert len(bad) == 0, f"{what}: {len(bad)} of {a.size} differ, first at {bad[:5]}"


@pytest.mark.parametrize("name", ["ref_32x32x10_400", "ref_64x64x10_2k", "ref_flt_48x48x10_1500"])
def test_build_equals_reference(name):
    from grotor_b200 import Router, TreeArrays
    g = load_golden(name)
    route_off = g["pin_acc_num"].astype(np.int64) * 12
    r = Router(golden_grid(g))
    r.build_topology(TreeArrays(g["node_off"], g["rsmt_pos"], g["rsmt_adj_off"], g["rsmt_adj"], route_off))
    got = r.read_topology()
    for k in KEYS:
        _equal(got[k], g[k], k)
    r.close()


@pytest.mark.parametrize("workload,seed", [("medium_320x320x10", 11), ("large_800x800x10", None)])
def test_build_equals_oracle(workload, seed):
    from grotor_b200 import Router
    from grotor_b200.synth import WORKLOADS, Design, steiner_trees
    d = Design(WORKLOADS[workload])
    t = steiner_trees(d.nets, shuffle_seed=seed)
    r = Router(d.grid)
    r.build_topology(t)
    got = r.read_topology()
    want = oracle.build_topology(d.grid.X, d.grid.Y, t.node_off, t.pos, t.adj_off, t.adj)
    for k in KEYS:
        _equal(got[k], want[k], k)
    r.close()


def test_stage_on_built_topology():
    from grotor_b200 import Router
    from grotor_b200.synth import WORKLOADS, Design, steiner_trees
    d = Design(WORKLOADS["medium_320x320x10"])
    res = []
    for built in (False, True):
        r = Router(d.grid)
        if built:
            r.build_topology(steiner_trees(d.nets))
        else:
            r.upload_nets(d.nets)
        bo, nb = r.generate_batches_rsmt(d.order, 1000000, 1, "persistent")
        st = r.lshape_route("persistent")
        res.append((bo, nb, r.read_routes(), r.read_tables()["demand_half"], st["wirelength"], st["vias"]))
        r.close()
    (a, b) = res
    assert a[1] == b[1]
    for k, what in enumerate(("batch_of", None, "routes", "demand")):
        if what:
            _equal(a[k], b[k], what)
    assert a[4] == b[4] and a[5] == b[5]


def test_non_trees_are_refused():
    from grotor_b200 import GrbError, Router, TreeArrays
    from grotor_b200.synth import WORKLOADS, Design, steiner_trees
    d = Design(WORKLOADS["small_64x64x5"].scaled(500))
    r = Router(d.grid)
    node_off = np.array([0, 3], np.int32)
    pos = np.array([0, 5, 9], np.int32)
    route_off = np.array([0, 36], np.int64)
    for adj_off, adj in (([0, 1, 2, 3], [1, 3, 0]), ([0, 2, 4, 4], [1, 1, 0, 0])):
        with pytest.raises(GrbError):
            r.build_topology(TreeArrays(node_off, pos, np.array(adj_off, np.int32), np.array(adj, np.int32),
                                        route_off))
    with pytest.raises(GrbError):  # a position beyond the Steiner layer
        r.build_topology(TreeArrays(node_off, np.array([0, 5, 64 * 64 * 7], np.int32),
                                    np.array([0, 1, 3, 4], np.int32), np.array([1, 0, 2, 1], np.int32), route_off))
    t = steiner_trees(d.nets)
    r.build_topology(t)
    got = r.read_topology()
    _equal(got["nodes"], d.nets.nodes, "nodes after a refused build")
    r.close()
