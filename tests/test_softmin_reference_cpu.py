"""The dense PyTorch soft-min reference on the CPU: its autograd gradient
matches FP64 central finite differences, and at tau = 0 it is the hard DP."""
import numpy as np
import pytest
import torch

import softmin_reference as R


@pytest.fixture(scope="module")
def small():
    from grotor_b200.synth import WORKLOADS, Design
    d = Design(WORKLOADS["softmin_check_32x32x4"].scaled(25))
    return d.grid, d.nets


def test_reference_gradient_matches_fd(small):
    g, nets = small
    dem = np.zeros(g.L * g.X * g.Y, np.int32)
    cap = torch.tensor(np.asarray(g.capacity, np.float64), requires_grad=True)
    uw = torch.full((g.L * g.X * g.Y,), float(g.unit_wire), dtype=torch.float64, requires_grad=True)
    uv = torch.tensor(float(g.unit_via), dtype=torch.float64, requires_grad=True)
    F = R.total_cost(g, dem, nets, cap, uw, uv, 0.5)
    F.backward()
    h = 1e-4
    for k in torch.topk(cap.grad.abs(), 5).indices.tolist():
        c = cap.detach().clone()
        c[k] += h
        fp = R.total_cost(g, dem, nets, c, uw.detach(), uv.detach(), 0.5)
        c[k] -= 2 * h
        fm = R.total_cost(g, dem, nets, c, uw.detach(), uv.detach(), 0.5)
        fd = (fp - fm).item() / (2 * h)
        assert abs(fd - cap.grad[k].item()) <= 1e-5 * max(1.0, abs(fd))


def test_reference_tends_to_hard_min(small):
    g, nets = small
    dem = np.zeros(g.L * g.X * g.Y, np.int32)
    cap = torch.tensor(np.asarray(g.capacity, np.float64))
    uw = torch.full((g.L * g.X * g.Y,), float(g.unit_wire), dtype=torch.float64)
    uv = torch.tensor(float(g.unit_via), dtype=torch.float64)
    hard = R.total_cost(g, dem, nets, cap, uw, uv, 0).item()
    soft = R.total_cost(g, dem, nets, cap, uw, uv, 1e-4).item()
    assert soft <= hard + 1e-9
    assert hard - soft < 1e-2
