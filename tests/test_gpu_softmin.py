"""Soft-min routing DAG and its CUDA adjoint (grotor_b200.softmin).

On the 32x32x4, 200-net gradient-check design (at the demand its exact
L-shape stage leaves), and on the same design with 10% blocked cells
(capacity 0: the cost model's zero-capacity branch): the CUDA forward and
adjoint agree with the dense PyTorch reference (tests/softmin_reference.py) to
1e-9 / 1e-7 relative in FP64; the adjoint matches FP64 central finite
differences (h = 1e-4) to 1e-4 relative at tau = 1, 0.1 and 0.01, including
blocked cells on routed paths (capacity gradient 0 there, wire-cost gradient
not); FP32 runs agree with FP64 to 1e-4; and as tau -> 0 the value tends to the
hard DP optimum and the gradient to the chosen routes' indicator.
"""
import numpy as np
import pytest
import torch

import softmin_reference as R

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=["open", "blocked"])
def setup(request):
    from grotor_b200 import Router
    from grotor_b200.synth import WORKLOADS, Design
    w = WORKLOADS["softmin_check_32x32x4"]
    d = Design(w if request.param == "open" else w.scaled(w.n_nets, blockage=0.10, seed=7))
    r = Router(d.grid)
    r.upload_nets(d.nets)
    r.generate_batches_rsmt(d.order, 1000000, 1, "persistent")
    r.lshape_route("persistent")
    dem = r.read_tables()["demand_half"]
    yield d, r, dem
    r.close()


def inputs(d, dtype, dev="cuda"):
    g = d.grid
    n = g.L * g.X * g.Y
    cap = torch.tensor(np.asarray(g.capacity, np.float64), dtype=dtype, device=dev)
    uw = torch.full((n,), float(g.unit_wire), dtype=dtype, device=dev)
    uv = torch.tensor(float(g.unit_via), dtype=dtype, device=dev)
    return cap, uw, uv


def cuda_cost(r, cap, uw, uv, tau):
    from grotor_b200.softmin import routing_cost
    cap = cap.clone().requires_grad_(True)
    uw = uw.clone().requires_grad_(True)
    uv = uv.clone().requires_grad_(True)
    F = routing_cost(r, cap, uw, uv, tau)
    F.backward()
    return F.item(), cap.grad.cpu(), uw.grad.cpu(), uv.grad.item()


def ref_cost(d, dem, tau):
    cap, uw, uv = (t.requires_grad_(True) for t in inputs(d, torch.float64, "cpu"))
    F = R.total_cost(d.grid, dem, d.nets, cap, uw, uv, tau)
    F.backward()
    return F.item(), cap.grad, uw.grad, uv.grad.item()


@pytest.mark.parametrize("tau", [1.0, 0.1, 0.01])
def test_matches_pytorch_reference(setup, tau):
    d, r, dem = setup
    f, gc, gw, gv = cuda_cost(r, *inputs(d, torch.float64), tau)
    fr, gcr, gwr, gvr = ref_cost(d, dem, tau)
    assert abs(f - fr) <= 1e-9 * abs(fr)
    scale = float(gcr.abs().max())
    assert float((gc - gcr).abs().max()) <= 1e-7 * scale
    assert float((gw - gwr).abs().max()) <= 1e-7 * float(gwr.abs().max())
    assert abs(gv - gvr) <= 1e-7 * abs(gvr)


@pytest.mark.parametrize("tau", [1.0, 0.1, 0.01])
def test_adjoint_matches_finite_differences(setup, tau):
    from grotor_b200.softmin import routing_cost
    d, r, dem = setup
    cap, uw, uv = inputs(d, torch.float64)
    f, gc, gw, gv = cuda_cost(r, cap, uw, uv, tau)
    h = 1e-4
    rng = np.random.default_rng(5)
    picks = torch.topk(gc.abs(), 12).indices.tolist()
    picks += rng.choice(np.flatnonzero(gc.numpy() != 0), 4, replace=False).tolist()
    blocked = np.flatnonzero(np.asarray(d.grid.capacity).reshape(-1) <= 0.001)
    if len(blocked):
        # Blocked cells the routes use: the zero-capacity branch does not
        # depend on capacity, so both sides must give 0 there.
        used = blocked[(dem[blocked] > 0)]
        assert len(used) > 0
        for k in rng.choice(used, min(4, len(used)), replace=False).tolist():
            assert gc[k].item() == 0.0
            picks.append(k)

    def F(c=cap, w=uw, v=uv):
        with torch.no_grad():
            return routing_cost(r, c, w, v, tau).item()

    for k in picks:
        cp, cm = cap.clone(), cap.clone()
        cp[k] += h
        cm[k] -= h
        fd = (F(c=cp) - F(c=cm)) / (2 * h)
        assert abs(fd - gc[k].item()) <= 1e-4 * max(abs(fd), 1e-3 * float(gc.abs().max())), (k, fd, gc[k].item())
    wpicks = torch.topk(gw.abs(), 4).indices.tolist()
    if len(blocked):
        # the blocked cells on routed paths with the largest wire-cost gradients
        on = sorted((k for k in used.tolist() if gw[k].item() != 0.0), key=lambda k: -abs(gw[k].item()))
        assert on, "no blocked cell carries a wire-cost gradient"
        wpicks += on[:3]
    wscale = float(gw.abs().max())
    for k in wpicks:
        wp, wm = uw.clone(), uw.clone()
        wp[k] += h
        wm[k] -= h
        fd = (F(w=wp) - F(w=wm)) / (2 * h)
        assert abs(fd - gw[k].item()) <= 1e-4 * max(abs(fd), 1e-3 * wscale), (k, fd, gw[k].item())
    fd = (F(v=uv + h) - F(v=uv - h)) / (2 * h)
    assert abs(fd - gv) <= 1e-4 * abs(fd)


def test_fp32_agrees_with_fp64(setup):
    d, r, _ = setup
    f64, g64, _, _ = cuda_cost(r, *inputs(d, torch.float64), 0.1)
    f32, g32, _, _ = cuda_cost(r, *inputs(d, torch.float32), 0.1)
    assert abs(f32 - f64) <= 1e-4 * abs(f64)
    assert float((g32.double() - g64).abs().max()) <= 1e-3 * float(g64.abs().max())


def test_tends_to_hard_dp_and_chosen_path(setup):
    d, r, dem = setup
    f, gc, gw, gv = cuda_cost(r, *inputs(d, torch.float64), 1e-5)
    fh, gch, gwh, gvh = ref_cost(d, dem, 0)   # hard min: autograd gives the chosen-path indicator
    assert abs(f - fh) <= 1e-3 * abs(fh) and f <= fh + 1e-6
    # d(total)/d(unit wire cost of an edge) = its length times the number of chosen wires over it
    close = (gw - gwh).abs() <= 1e-3
    assert float(close.double().mean()) >= 0.99
    assert abs(gv - gvh) <= 1e-2 * abs(gvh)
