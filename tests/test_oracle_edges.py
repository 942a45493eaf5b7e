"""Edge cases of the oracle's first-fit batching that hold whatever the
conflict rule: an empty order, a single net, the batch-size limit, and the
first-fit shape of the result (a net opens at most one new batch, and never
skips one)."""
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
