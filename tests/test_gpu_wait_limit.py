"""Bounded device waits.  The persistent kernels' grid barriers and the
batching kernel's hand-over counters give up after the context's wait limit:
with a limit far shorter than any wait the kernels actually make, every
block returns, the call reports GRB_ETIMEDOUT, the context stays usable, and
after grb_reset (and a fresh plan) a normal run gives the usual routes.  No
GPU fault is involved: the waits end by their own limit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def design():
    from grotor_b200.synth import WORKLOADS, Design
    return Design(WORKLOADS["medium_320x320x10"].scaled(20000, seed=31))


def test_stage_wait_runs_out_and_context_recovers(design):
    from grotor_b200 import GrbError, Router
    from grotor_b200._abi import GRB_ETIMEDOUT
    d = design
    r = Router(d.grid)
    r.upload_nets(d.nets)
    r.generate_batches_rsmt(d.order, 1000000, 1, "persistent")
    ids, off = r.plan()
    want = r.lshape_route("persistent")
    want_routes = r.read_routes()
    r.reset()
    r.set_wait_limit(1e-9)
    with pytest.raises(GrbError) as e:
        r.lshape_route("persistent")
    assert e.value.code == GRB_ETIMEDOUT
    r.set_wait_limit(20.0)
    r.reset()
    r.set_plan(ids, off)
    got = r.lshape_route("persistent")
    np.testing.assert_array_equal(r.read_routes(), want_routes)
    assert got["wirelength"] == want["wirelength"] and got["vias"] == want["vias"]
    r.close()


def test_batching_wait_runs_out_and_context_recovers(design):
    from grotor_b200 import GrbError, Router
    from grotor_b200._abi import GRB_ETIMEDOUT
    d = design
    r = Router(d.grid)
    r.upload_nets(d.nets)
    want, nb = r.generate_batches_rsmt(d.order, 1000000, 1, "persistent")
    r.set_wait_limit(1e-9)
    with pytest.raises(GrbError) as e:
        r.generate_batches_rsmt(d.order, 1000000, 1, "persistent")
    assert e.value.code == GRB_ETIMEDOUT
    r.set_wait_limit(20.0)
    got, nb2 = r.generate_batches_rsmt(d.order, 1000000, 1, "persistent")
    assert nb2 == nb
    np.testing.assert_array_equal(got, want)
    r.close()
