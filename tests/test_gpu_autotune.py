"""Autotuned launch shapes (nets per CTA, nets per work-queue grab, by size
bucket) change timing only: every executor still gives the routes, demand and
statistics of the untuned persistent stage, including a design with nets
beyond the shared-memory arena (more than 16 tree nodes)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("workload,n", [("medium_320x320x10", 20000), ("persistent_1600x1600x10", 20000)])
def test_autotune_keeps_results(workload, n):
    from grotor_b200 import Router
    from grotor_b200.synth import WORKLOADS, Design
    d = Design(WORKLOADS[workload].scaled(n, seed=43))
    r = Router(d.grid)
    r.upload_nets(d.nets)
    r.generate_batches_rsmt(d.order, 1000000)
    st0 = r.lshape_route("persistent")
    routes0, dem0 = r.read_routes(), r.read_tables()["demand_half"]
    choice = r.autotune()
    assert all(v in (1, 2, 4, 8) for v in choice["nets_per_cta"] + choice["nets_per_grab"])
    for mode in ("plain", "graph", "persistent"):
        r.reset()
        st = r.lshape_route(mode)
        np.testing.assert_array_equal(r.read_routes(), routes0)
        np.testing.assert_array_equal(r.read_tables()["demand_half"], dem0)
        assert st["wirelength"] == st0["wirelength"] and st["vias"] == st0["vias"]
    r.close()
