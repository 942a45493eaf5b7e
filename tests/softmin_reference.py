"""Dense PyTorch restatement of the soft-min L-shape DAG (test reference).

The same DP as the CUDA kernels in grotor_b200/csrc/device/softmin.cuh, written
with plain torch operations so that autograd gives an independent gradient:
cost tables from capacity / unit costs at a fixed demand (full_update.cuh:9-83
in real arithmetic), then per net the L-shape DP of lshape_thread.cuh:18-171
with every min replaced by a tau-soft-min (tau = 0: the hard min).
"""
from __future__ import annotations

import torch


def tables(grid, demand_half, cap, uw, uv, of_scale=1.0):
    """wire cost, via cost and exclusive wire-cost prefix, each (L, X, Y)."""
    L, X, Y, DIR = grid.L, grid.X, grid.Y, grid.DIR
    d = torch.as_tensor(demand_half, dtype=cap.dtype).reshape(L, X, Y) * 0.5
    cap = cap.reshape(L, X, Y)
    uw = uw.reshape(L, X, Y)
    w = torch.as_tensor(grid.short_costs, dtype=cap.dtype).reshape(L, 1, 1)

    def of(dd):
        a = 0.5 * (dd - cap)
        b = of_scale * 0.5 * (dd - cap)
        pos = torch.exp(torch.minimum(a, b))
        a2 = 1.5 * dd
        zero = torch.where(dd > 0, torch.exp(torch.minimum(a2, of_scale * a2)), torch.zeros_like(dd))
        return torch.where(cap > 0.001, pos, zero)

    def incr(k):
        return torch.clamp(torch.clamp((of(d + k) - of(d)) * w, max=1e12), max=1e12)

    i1, ih = incr(1.0), incr(0.5)
    xlen = torch.zeros(X, dtype=cap.dtype)
    xlen[:X - 1] = torch.as_tensor(grid.x_edge_len, dtype=cap.dtype)
    ylen = torch.zeros(Y, dtype=cap.dtype)
    ylen[:Y - 1] = torch.as_tensor(grid.y_edge_len, dtype=cap.dtype)
    wc, vc, P = [], [], []
    for l in range(L):
        ay = ((l & 1) ^ DIR) == 1
        if ay:
            wl = i1[l] + uw[l] * ylen.reshape(1, Y)
            v = torch.cat([i1[l][:, :1], ih[l][:, 1:Y - 1] + ih[l][:, 0:Y - 2], i1[l][:, Y - 2:Y - 1]], dim=1)
            p = torch.cat([torch.zeros(X, 1, dtype=cap.dtype), torch.cumsum(wl, dim=1)[:, :Y - 1]], dim=1)
        else:
            wl = i1[l] + uw[l] * xlen.reshape(X, 1)
            v = torch.cat([i1[l][:1, :], ih[l][1:X - 1, :] + ih[l][0:X - 2, :], i1[l][X - 2:X - 1, :]], dim=0)
            p = torch.cat([torch.zeros(1, Y, dtype=cap.dtype), torch.cumsum(wl, dim=0)[:X - 1, :]], dim=0)
        wc.append(wl)
        vc.append(v + uv)
        P.append(p)
    return torch.stack(wc), torch.stack(vc), torch.stack(P)


def _smin(vals, tau):
    v = [x for x in vals if x is not None]
    if not v:
        return None
    t = torch.stack(v)
    if tau == 0:
        return torch.min(t)
    return -tau * torch.logsumexp(-t / tau, dim=0)


def net_cost(grid, vc, P, nodes, parents, tau):
    """Soft-min DP of one net (nodes: 3-D ids in DFS order, parents[0] = -1)."""
    L, X, Y, DIR = grid.L, grid.X, grid.Y, grid.DIR
    XY = X * Y
    N = len(nodes)

    def pos(v):
        return int(v) // XY, int(v) % XY // Y, int(v) % Y

    def ay(l):
        return ((l & 1) ^ DIR) == 1

    def wire(l, xmin, xmax, ymin, ymax):
        return P[l, xmax, ymax] - P[l, xmin, ymin]

    dist = []
    for i in range(N):
        lp, x, y = pos(nodes[i])
        d = {}
        for lo in range(L):
            acc = torch.zeros((), dtype=P.dtype)
            for hi in range(lo, L):
                if hi > lo:
                    acc = acc + vc[hi - 1, x, y]
                d[(lo, hi)] = None if (lp < L and (lo > lp or hi < lp)) else acc
        dist.append(d)
    for i in range(N - 1, 0, -1):
        p = int(parents[i])
        _, x, y = pos(nodes[i])
        _, px, py = pos(nodes[p])
        minx, maxx, miny, maxy = min(x, px), max(x, px), min(y, py), max(y, py)
        cur = [_smin([dist[i][(lo, hi)] for lo in range(l + 1) for hi in range(l, L)], tau) for l in range(L)]
        diag = []
        for pl in range(L):
            cands = []
            for cl in range(L):
                if cur[cl] is None:
                    continue
                if x == px or y == py:
                    if cl != pl or (not ay(cl) and y != py) or (ay(cl) and x != px):
                        continue
                    cands.append(cur[cl] + wire(cl, minx, maxx, miny, maxy))
                else:
                    if ((cl ^ pl) & 1) == 0:
                        continue
                    c = wire(cl, x, x, miny, maxy) if ay(cl) else wire(cl, minx, maxx, y, y)
                    c2 = torch.zeros((), dtype=P.dtype)
                    for l in range(min(cl, pl) + 1, max(cl, pl)):
                        c2 = c2 + (vc[l, x, py] if ay(cl) else vc[l, px, y])
                    c2 = c2 + (wire(pl, px, px, miny, maxy) if ay(pl) else wire(pl, minx, maxx, py, py))
                    cands.append(cur[cl] + (c + c2))
            diag.append(_smin(cands, tau))
        for lo in range(L):
            for hi in range(lo, L):
                m = _smin(diag[lo:hi + 1], tau)
                if dist[p][(lo, hi)] is not None:
                    dist[p][(lo, hi)] = None if m is None else dist[p][(lo, hi)] + m
    return _smin([dist[0][(lo, hi)] for lo in range(L) for hi in range(lo, L)], tau)


def total_cost(grid, demand_half, nets, cap, uw, uv, tau):
    """Sum of the soft-min DP over every net of `nets` (NetArrays)."""
    _, vc, P = tables(grid, demand_half, cap, uw, uv)
    total = torch.zeros((), dtype=cap.dtype)
    for i in range(len(nets.node_off) - 1):
        a, b = int(nets.node_off[i]), int(nets.node_off[i + 1])
        if b <= a:
            continue
        c = net_cost(grid, vc, P, nets.nodes[a:b], nets.parents[a:b], tau)
        if c is not None:
            total = total + c
    return total
