"""Shared helpers for the test suite (fixtures, grid/net conversion, checks)."""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
ROUTE_PER_PIN = 12  # router_state.hpp:31


def load_golden(name: str) -> dict:
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def golden_grid(g: dict):
    from grotor_b200.router import GridArrays
    L, X, Y, DIR = (int(v) for v in g["meta"])
    uw, uv = (float(v) for v in g["unit_costs"])
    return GridArrays(L, X, Y, DIR, uw, uv, g["short_costs"], g["x_edge_len"], g["y_edge_len"], g["capacity"])


def golden_nets(g: dict):
    """Reference topology with the reference's route layout (12 words per pin)."""
    from grotor_b200.router import NetArrays
    route_off = g["pin_acc_num"].astype(np.int64) * ROUTE_PER_PIN
    return NetArrays(g["node_off"], g["nodes"], g["parents"], route_off, g["point_off"], g["points"],
                     g["hseg_off"], g["hsegs"], g["vseg_off"], g["vsegs"])


def orc_grid(grid):
    import oracle
    return oracle.OrcGrid(grid.L, grid.X, grid.Y, grid.DIR, grid.unit_wire, grid.unit_via, grid.short_costs,
                          grid.x_edge_len, grid.y_edge_len, grid.capacity, grid.of_cost_scale)


def float_demand_to_half(d: np.ndarray) -> np.ndarray:
    h = d.astype(np.float64) * 2.0
    assert np.all(h == np.round(h)), "reference demand is not a multiple of 0.5"
    return h.astype(np.int32)


def net_routes(routes: np.ndarray, route_off: np.ndarray, i: int) -> np.ndarray:
    r = routes[route_off[i]:route_off[i + 1]]
    return r[:r[0]] if len(r) else r


def check_connected(routes, route_off, node_off, nodes, X, Y, L, ids):
    """Every routed net's segments form one connected 3-D structure that
    touches every pin at its layer (Steiner nodes at any layer)."""
    XY = X * Y
    for i in ids:
        r = net_routes(routes, route_off, i)
        if len(r) == 0:
            continue
        parent = {}

        def find(a):
            while parent.setdefault(a, a) != a:
                parent[a] = parent[parent[a]]
                a = parent[a]
            return a

        def union(a, b):
            parent[find(a)] = find(b)

        for k in range(1, r[0], 2):
            a, b = int(r[k]), int(r[k + 1])
            la, lb = a // XY, b // XY
            if la == lb:
                xa, ya, xb, yb = a % XY // Y, a % Y, b % XY // Y, b % Y
                assert xa == xb or ya == yb, "wire segment is not straight"
                if xa == xb:
                    cells = [la * XY + xa * Y + y for y in range(min(ya, yb), max(ya, yb) + 1)]
                else:
                    cells = [la * XY + x * Y + ya for x in range(min(xa, xb), max(xa, xb) + 1)]
            else:
                assert a % XY == b % XY, "via changes position"
                cells = [l * XY + a % XY for l in range(min(la, lb), max(la, lb) + 1)]
            for c in cells[1:]:
                union(cells[0], c)
        nd = nodes[node_off[i]:node_off[i + 1]]
        roots = set()
        for v in nd:
            l, pos = int(v) // XY, int(v) % XY
            if l >= L:
                continue
            c = l * XY + pos
            if len(nd) > 1:
                assert c in parent, f"net {i}: pin {c} not touched by its route"
            roots.add(find(c) if c in parent else c)
        if parent:
            comps = {find(c) for c in list(parent)}
            assert len(comps) == 1, f"net {i}: route has {len(comps)} components"
