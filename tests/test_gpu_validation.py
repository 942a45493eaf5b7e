"""Input validation of grb_upload_nets.

The upload checks every element a stage kernel will dereference (tree nodes
inside the grid, parents before children, offsets non-decreasing and inside
the arrays, batching geometry inside the grid) on the device, and refuses a
bad upload with GRB_EINVAL naming the first offending item.  After a refused
upload no net id is accepted; a later valid upload routes exactly like a
fresh context.
"""
import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def design():
    from grotor_b200.synth import WORKLOADS, Design
    return Design(WORKLOADS["small_64x64x5"].scaled(400, seed=5))


def _bad(nets, **arrays):
    return dataclasses.replace(nets, **arrays)


def _cases(d):
    n = d.nets
    XY = d.grid.X * d.grid.Y
    out = []
    nodes = n.nodes.copy()
    nodes[n.node_off[7]] = (d.grid.L + 1) * XY  # one layer past the Steiner layer
    out.append(("node outside", _bad(n, nodes=nodes), "tree node outside the grid", 7))
    nodes = n.nodes.copy()
    nodes[n.node_off[3]] = -1
    out.append(("negative node", _bad(n, nodes=nodes), "tree node outside the grid", 3))
    par = n.parents.copy()
    i = next(i for i in range(n.n) if n.node_off[i + 1] - n.node_off[i] >= 3)
    par[n.node_off[i] + 1] = 2  # a parent that follows its child
    out.append(("parent order", _bad(n, parents=par), "parents must precede children", i))
    par = n.parents.copy()
    par[n.node_off[11]] = 0  # a root with a parent
    out.append(("root parent", _bad(n, parents=par), "parents must precede children", 11))
    ro = n.route_off.copy()
    ro[5], ro[6] = ro[6], ro[5]
    out.append(("route offsets", _bad(n, route_off=ro), "offsets must be non-decreasing", 5))
    pts = n.points.copy()
    pts[len(pts) // 2] = XY
    out.append(("point outside", _bad(n, points=pts), "batching geometry outside the grid", None))
    hs = n.hsegs.copy()
    hs[-1] = -3
    out.append(("segment outside", _bad(n, hsegs=hs), "batching geometry outside the grid", None))
    return out


def test_bad_uploads_are_refused(design):
    from grotor_b200 import GrbError, Router
    from grotor_b200._abi import GRB_EINVAL
    r = Router(design.grid)
    for name, nets, msg, item in _cases(design):
        with pytest.raises(GrbError) as e:
            r.upload_nets(nets)
        assert e.value.code == GRB_EINVAL, name
        assert msg in str(e.value), (name, str(e.value))
        if item is not None:
            assert f"(item {item})" in str(e.value), (name, str(e.value))
        with pytest.raises(GrbError):  # no net id is accepted after a refused upload
            r.generate_batches_rsmt(design.order)
    r.close()


def test_valid_upload_after_refusal_routes_like_fresh_context(design):
    from grotor_b200 import GrbError, Router
    fresh = Router(design.grid)
    fresh.upload_nets(design.nets)
    fresh.generate_batches_rsmt(design.order)
    fresh.lshape_route("plain")
    want_d, want_r = fresh.read_tables()["demand_half"], fresh.read_routes()
    fresh.close()

    r = Router(design.grid)
    r.upload_nets(design.nets)
    with pytest.raises(GrbError):
        r.upload_nets(_cases(design)[0][1])
    r.upload_nets(design.nets)
    r.generate_batches_rsmt(design.order)
    r.lshape_route("plain")
    np.testing.assert_array_equal(r.read_tables()["demand_half"], want_d)
    np.testing.assert_array_equal(r.read_routes(), want_r)
    r.close()
