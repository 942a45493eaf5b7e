"""GPU first-fit batching equals the reference's CPU batching exactly.

The reference accepts RT-core batches only if the lists equal the CPU's
(generate_batches.hpp:113-131); the same bar applies to the grid kernels here,
in both execution forms, with small batch limits and sparsity > 1.
"""
import numpy as np
import pytest

import oracle
from helpers import golden_nets, load_golden

pytestmark = pytest.mark.gpu


def _check(router, order, nets, X, Y, limit, sparsity, mode):
    from grotor_b200 import plan_from_batches
    bo_ref, nb_ref = oracle.batches(X, Y, order, nets.point_off, nets.points, nets.hseg_off, nets.hsegs,
                                    nets.vseg_off, nets.vsegs, limit, sparsity)
    bo, nb = router.generate_batches_rsmt(order, limit, sparsity, mode)
    assert nb == nb_ref
    np.testing.assert_array_equal(bo, bo_ref)
    ids, off = router.plan()
    ids_ref, off_ref = plan_from_batches(order, bo_ref, nb_ref)
    np.testing.assert_array_equal(off, off_ref)
    np.testing.assert_array_equal(ids, ids_ref)


@pytest.mark.parametrize("mode", ["plain", "persistent"])
@pytest.mark.parametrize("limit,sparsity", [(1000000, 1), (37, 1), (1000000, 3), (1, 1)])
def test_synthetic(mode, limit, sparsity):
    from grotor_b200 import Router
    from grotor_b200.synth import WORKLOADS, Design
    d = Design(WORKLOADS["small_64x64x5"].scaled(3000 if limit > 1 else 700, seed=31))
    r = Router(d.grid)
    r.upload_nets(d.nets)
    _check(r, d.order, d.nets, d.grid.X, d.grid.Y, limit, sparsity, mode)
    r.close()


@pytest.mark.parametrize("mode", ["plain", "persistent"])
def test_medium_many_chunks(mode):
    """Several thousand nets across many 512-net chunks, big nets included."""
    from grotor_b200 import Router
    from grotor_b200.synth import WORKLOADS, Design
    d = Design(WORKLOADS["medium_320x320x10"].scaled(20000, seed=32))
    r = Router(d.grid)
    r.upload_nets(d.nets)
    _check(r, d.order, d.nets, d.grid.X, d.grid.Y, 1000000, 1, mode)
    r.close()


@pytest.mark.parametrize("name", ["ref_64x64x10_2k", "ref_32x32x10_400"])
def test_reference_geometry(name):
    """On the reference's own FLUTE geometry the GPU reproduces the
    reference's batch lists."""
    from grotor_b200 import Router
    from helpers import golden_grid
    g = load_golden(name)
    grid, nets = golden_grid(g), golden_nets(g)
    r = Router(grid)
    r.upload_nets(nets)
    bo, nb = r.generate_batches_rsmt(g["order"], 1000000, 1, "persistent")
    np.testing.assert_array_equal(bo, g["batch_of"])
    ids, off = r.plan()
    np.testing.assert_array_equal(ids, g["ids"])
    np.testing.assert_array_equal(off, g["batch_off"])
    r.close()


def test_empty_and_single():
    from grotor_b200 import Router
    from grotor_b200.synth import WORKLOADS, Design
    d = Design(WORKLOADS["small_64x64x5"].scaled(50, seed=33))
    r = Router(d.grid)
    r.upload_nets(d.nets)
    bo, nb = r.generate_batches_rsmt(np.zeros(0, np.int32), 10)
    assert nb == 0 and len(bo) == 0
    bo, nb = r.generate_batches_rsmt(d.order[:1], 10)
    assert nb == 1 and bo.tolist() == [0]
    r.close()
