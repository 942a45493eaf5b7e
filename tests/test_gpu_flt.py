"""The CUDA FLT stage against the reference router's own FLT run and the oracle.

On the reference's topology, plan, rip-up set, FLT DAGs and FLT batches
(tests/golden/ref_flt_*.npz) the B200 path replays the L-shape stage, then:
GPU rip-up classification equals the reference's set, GPU batching of the FLT
geometry equals the reference's FLT batches, and the FLT stage (plain, graph
and persistent executors) reproduces the reference's demand, statistics and
every net's phase-two segment multiset exactly (the reference appends
segments with atomics, so their order is not defined), and the oracle's
route words word for word except where the oracle's tolerance-level costs
split a straight run differently.
"""
import numpy as np
import pytest

from helpers import (flt_by_net, float_demand_to_half, golden_grid, golden_nets, load_golden, orc_grid,
                     ref_routes2_of, route_geometry, segment_multiset)

pytestmark = pytest.mark.gpu

NAMES = ["ref_flt_48x48x10_1500"]


def need_flt(g):
    if "flt_after_demand" not in g:
        pytest.skip("fixture lacks the reference FLT run")


def router_after_lshape(g):
    from grotor_b200 import Router
    r = Router(golden_grid(g))
    r.upload_nets(golden_nets(g))
    r.set_plan(g["ids"], g["batch_off"])
    r.set_stats(0.0, int(g["pin_vias"][0]))
    r.lshape_route("persistent")
    return r


@pytest.mark.parametrize("name", NAMES)
def test_ripup_and_flt_batches_on_gpu(name):
    g = load_golden(name)
    need_flt(g)
    r = router_after_lshape(g)
    np.testing.assert_array_equal(r.read_tables()["demand_half"], float_demand_to_half(g["flt_before_demand"]))
    np.testing.assert_array_equal(np.flatnonzero(r.ripup(0)), g["flt_of_nets"])
    _, geom, _ = flt_by_net(g)
    r.upload_geometry(*geom)
    for mode in ("plain", "persistent"):
        r.generate_batches_rsmt(g["flt_nets"], 300000, 1, mode)
        ids, off = r.plan()
        np.testing.assert_array_equal(ids, g["flt_batch_ids"])
        np.testing.assert_array_equal(off, g["flt_batch_off"])
    r.close()


@pytest.mark.parametrize("mode", ["plain", "graph", "persistent"])
@pytest.mark.parametrize("name", NAMES)
def test_flt_stage_equals_reference(name, mode):
    g = load_golden(name)
    need_flt(g)
    r = router_after_lshape(g)
    dags, _, route2_off = flt_by_net(g)
    r.upload_flt(dags, route2_off)
    r.set_plan(g["flt_batch_ids"], g["flt_batch_off"])
    st = r.flt_route(mode, remove_phase_one=True)
    t = r.read_tables()
    np.testing.assert_array_equal(t["demand_half"], float_demand_to_half(g["flt_after_demand"]))
    assert st["wirelength"] == g["flt_after_stats"][0]
    assert st["vias"] == int(g["flt_after_stats"][1])
    assert st["stamp"] == int(g["flt_after_stats"][2])
    routes2 = r.read_routes2()
    for net in g["flt_nets"]:
        ours = routes2[route2_off[net]:route2_off[net + 1]]
        assert segment_multiset(ours) == segment_multiset(ref_routes2_of(g, net)), f"net {net}"
    r.close()


@pytest.mark.parametrize("name", NAMES)
def test_flt_stage_equals_oracle(name):
    import oracle
    g = load_golden(name)
    need_flt(g)
    r = router_after_lshape(g)
    before = r.read_tables()
    stats0 = r.stats()
    dags, _, route2_off = flt_by_net(g)
    r.upload_flt(dags, route2_off)
    r.set_plan(g["flt_batch_ids"], g["flt_batch_off"])
    r.flt_route("persistent", remove_phase_one=True)
    routes2 = r.read_routes2()
    nets = golden_nets(g)
    out = oracle.flt_stage(orc_grid(golden_grid(g)), dags, g["flt_batch_ids"], g["flt_batch_off"], nets.route_off,
                           r.read_routes(), route2_off, before["demand_half"], before["timestamp"], stats0["stamp"],
                           True, wirelength=stats0["wirelength"], vias=stats0["vias"])
    assert out["status"] == 0
    X, Y = int(g["meta"][1]), int(g["meta"][2])
    exact = 0
    for net in g["flt_nets"]:
        a = routes2[route2_off[net]:route2_off[net + 1]]
        b = out["routes2"][route2_off[net]:route2_off[net + 1]]
        assert route_geometry(a, X, Y) == route_geometry(b, X, Y), f"net {net}"
        exact += np.array_equal(a[:a[0]], b[:b[0]])
    assert exact >= 0.95 * len(g["flt_nets"])
    r.close()


@pytest.mark.parametrize("mode", ["plain", "persistent"])
@pytest.mark.parametrize("name", NAMES)
def test_flt_block_path_equals_warp_path(name, mode):
    """Nets routed by a whole CTA (a DAG level wider than the threshold) give
    the same route words, demand and statistics as one warp per net: every
    net by one warp (-1), every net by a CTA (0), and a mix (2)."""
    g = load_golden(name)
    need_flt(g)
    dags, _, route2_off = flt_by_net(g)
    out = {}
    for width in (-1, 0, 2):
        r = router_after_lshape(g)
        r.upload_flt(dags, route2_off)
        r.set_plan(g["flt_batch_ids"], g["flt_batch_off"])
        r.set_flt_block_width(width)
        st = r.flt_route(mode, remove_phase_one=True)
        out[width] = (r.read_routes2(), r.read_tables(), st)
        r.close()
    routes_w, tables_w, st_w = out[-1]
    np.testing.assert_array_equal(tables_w["demand_half"], float_demand_to_half(g["flt_after_demand"]))
    for width in (0, 2):
        routes, tables, st = out[width]
        np.testing.assert_array_equal(routes, routes_w)
        np.testing.assert_array_equal(tables["demand_half"], tables_w["demand_half"])
        np.testing.assert_array_equal(tables["timestamp"], tables_w["timestamp"])
        assert (st["wirelength"], st["vias"], st["stamp"]) == (st_w["wirelength"], st_w["vias"], st_w["stamp"])
