"""The allocation-free rip-up classification (grb_ripup_classify_noalloc).

Callers that cannot allocate device memory while routing -- a process held to
a fixed device-memory budget next to another framework's caching allocator, or
a steady-state loop that must not pay the synchronisation of cudaMalloc/cudaFree
-- use this entry point; its scratch is a fixed array inside the library.  Its
result must equal the allocating entry point's, call after call (the array is
shared and keeps the previous call's contents), and designs beyond its size
limit must be refused with GRB_ELIMIT.

Collected last so a failure here never hides the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def routed():
    from grotor_b200 import Router
    from grotor_b200.synth import WORKLOADS, Design
    d = Design(WORKLOADS["medium_320x320x10"].scaled(20000, seed=77))
    r = Router(d.grid)
    r.upload_nets(d.nets)
    r.generate_batches_rsmt(d.order, 1000000)
    r.lshape_route("persistent")
    yield r
    r.close()


def test_matches_allocating_entry_point_twice(routed):
    from grotor_b200 import _abi
    lib = _abi.load()
    flagged = 0
    for thr in (0, -2, -5):
        want = routed.ripup(thr)
        flagged += int(want.sum())
        for _ in range(2):  # two calls in a row share and reuse the array
            got = np.zeros_like(want)
            rc = lib.grb_ripup_classify_noalloc(routed._ctx, thr, got.ctypes.data_as(C.c_void_p))
            assert rc == 0, lib.grb_last_error(routed._ctx).decode()
            np.testing.assert_array_equal(got, want)
    assert flagged > 0  # the comparison covered flagged nets


@pytest.fixture(scope="module")
def routed_at_limit():
    """A design of exactly 4,194,304 cells (4 routing layers of 1024 x 1024),
    the largest the fixed array takes, with close to a million nets and low
    capacities: the per-net flags then start right after the last cell word
    the classification uses."""
    from grotor_b200 import Router
    from grotor_b200.synth import SynthParams, Design
    d = Design(SynthParams(1024, 1024, 5, 880000, 1, 3, seed=78))
    assert d.grid.cells == 4 << 20 and 800000 < d.n_subnets <= 1 << 20
    r = Router(d.grid)
    r.upload_nets(d.nets)
    r.generate_batches_rsmt(d.order, 1000000)
    r.lshape_route("persistent")
    yield r
    r.close()


def test_matches_allocating_entry_point_at_the_size_limit(routed_at_limit):
    from grotor_b200 import _abi
    lib = _abi.load()
    r = routed_at_limit
    for thr in (0, -1):
        want = r.ripup(thr)
        assert want.sum() > 0
        for _ in range(2):
            got = np.zeros_like(want)
            rc = lib.grb_ripup_classify_noalloc(r._ctx, thr, got.ctypes.data_as(C.c_void_p))
            assert rc == 0, lib.grb_last_error(r._ctx).decode()
            np.testing.assert_array_equal(got, want)


def test_refuses_designs_beyond_its_limit():
    from grotor_b200 import GrbError, GridArrays, Router
    from grotor_b200._abi import GRB_ELIMIT
    L, X, Y = 9, 1024, 512  # 4.7 M cells > 4,194,304
    grid = GridArrays(L, X, Y, 1, 1.0, 2.0, np.ones(L), np.ones(X - 1, np.int32), np.ones(Y - 1, np.int32),
                      np.full((L, X, Y), 5.0, np.float32))
    r = Router(grid)
    with pytest.raises(GrbError) as e:
        r.ripup_noalloc(0)
    assert e.value.code == GRB_ELIMIT and "at most" in str(e.value)
    r.close()
