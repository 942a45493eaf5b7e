"""Differentiable routing cost: the soft-min L-shape DAG and its hand-written
adjoint (include/grb.h: grb_softmin_forward / grb_softmin_backward) behind a
``torch.autograd.Function``.

``routing_cost(router, capacity, unit_wire, unit_via, tau)`` returns the total
soft-min routed cost of every net uploaded to ``router`` at its current demand;
its gradient with respect to the per-edge capacity, the per-edge unit wire cost
and the unit via cost comes from the CUDA adjoint (no autograd tape over the
DP).  Tensors are CUDA tensors of shape (L, X, Y) (or flat), float32 or
float64; the computation runs in that precision.  PyTorch only carries the
buffers: the DP and its adjoint are the library's kernels.
"""
from __future__ import annotations

import ctypes as C

import torch

__all__ = ["SoftminRoutingCost", "routing_cost"]


def _dtype_id(t: torch.Tensor) -> int:
    if t.dtype == torch.float64:
        return 1  # GRB_F64
    if t.dtype == torch.float32:
        return 0  # GRB_F32
    raise TypeError("capacity and unit_wire must be float32 or float64")


def _check_input(router, t: torch.Tensor, name: str) -> torch.Tensor:
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor (the soft-min DP has no CPU path)")
    g = router.grid
    if t.numel() != g.L * g.X * g.Y:
        raise ValueError(f"{name} must hold L*X*Y = {g.L * g.X * g.Y} values")
    return t.contiguous()


class SoftminRoutingCost(torch.autograd.Function):
    """total = sum over nets of the tau-soft-min L-shape DP value."""

    @staticmethod
    def forward(ctx, capacity, unit_wire, unit_via, router, tau):
        capacity = _check_input(router, capacity, "capacity")
        unit_wire = _check_input(router, unit_wire, "unit_wire")
        if unit_wire.dtype != capacity.dtype:
            raise TypeError("capacity and unit_wire must have the same dtype")
        dt = _dtype_id(capacity)
        uv = float(unit_via)
        net_cost = torch.empty(router.nets.n, dtype=capacity.dtype, device=capacity.device)
        total = C.c_double(0)
        torch.cuda.current_stream(capacity.device).synchronize()  # inputs written on torch's stream
        router._check(router._lib.grb_softmin_forward(router._ctx, dt, float(tau), C.c_void_p(capacity.data_ptr()),
                                                      C.c_void_p(unit_wire.data_ptr()), uv,
                                                      C.c_void_p(net_cost.data_ptr()), C.byref(total)))
        ctx.save_for_backward(capacity, unit_wire)
        ctx.router, ctx.tau, ctx.uv, ctx.dt = router, float(tau), uv, dt
        ctx.uv_is_tensor = torch.is_tensor(unit_via)
        ctx.net_cost = net_cost
        return torch.tensor(total.value, dtype=capacity.dtype, device=capacity.device)

    @staticmethod
    def backward(ctx, grad):
        capacity, unit_wire = ctx.saved_tensors
        router = ctx.router
        dcap = torch.empty_like(capacity)
        duw = torch.empty_like(unit_wire)
        duv = C.c_double(0)
        g = float(grad)
        router._check(router._lib.grb_softmin_backward(router._ctx, ctx.dt, ctx.tau, C.c_void_p(capacity.data_ptr()),
                                                       C.c_void_p(unit_wire.data_ptr()), ctx.uv, g,
                                                       C.c_void_p(dcap.data_ptr()), C.c_void_p(duw.data_ptr()),
                                                       C.byref(duv)))
        duv_t = torch.tensor(duv.value, dtype=capacity.dtype, device=capacity.device) if ctx.uv_is_tensor else None
        return dcap, duw, duv_t, None, None


def routing_cost(router, capacity: torch.Tensor, unit_wire: torch.Tensor, unit_via, tau: float) -> torch.Tensor:
    """Soft-min total routed cost (differentiable in capacity, unit_wire and,
    when it is a tensor, unit_via)."""
    return SoftminRoutingCost.apply(capacity, unit_wire, unit_via, router, tau)
