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


# ---- FLT stage fixtures (tests/golden/make_golden.py --flt) -----------------
ROUTE_PER_PIN_PHASE2 = 100  # router_state.hpp:33
FLT_DAG_KEYS = ("node_off", "coord", "depth", "children", "parent_end", "edge_off", "edge_parent", "edge_slot")


def flt_by_net(g: dict):
    """FLT inputs of a fixture re-indexed by net id: DAG CSR (empty for nets
    outside the stage), batching geometry (FLT geometry for stage nets, the
    stage-one geometry otherwise) and phase-two route offsets (100 words per
    pin for stage nets)."""
    n = len(g["node_off"]) - 1
    slot_of = np.full(n, -1, np.int64)
    slot_of[g["flt_nets"]] = np.arange(len(g["flt_nets"]))

    def csr(off_key, data_keys, default_off=None, default_data=None, width=1):
        off = [0]
        data = {k: [] for k in data_keys}
        for i in range(n):
            s = slot_of[i]
            if s >= 0:
                a, b = g[off_key][s], g[off_key][s + 1]
                for k in data_keys:
                    data[k].append(g[k][a * width:b * width])
                off.append(off[-1] + b - a)
            elif default_off is not None:
                a, b = default_off[i], default_off[i + 1]
                for k, dk in zip(data_keys, default_data):
                    data[k].append(dk[a * width:b * width])
                off.append(off[-1] + b - a)
            else:
                off.append(off[-1])
        cat = {k: (np.concatenate(v) if v else np.zeros(0, np.int32)).astype(np.int32) for k, v in data.items()}
        return np.asarray(off, np.int32), cat

    node_off, nd = csr("flt_node_off", ["flt_coord", "flt_depth", "flt_children", "flt_parent_end"])
    edge_off, ed = csr("flt_edge_off", ["flt_edge_parent", "flt_edge_slot"])
    dags = {"node_off": node_off, "coord": nd["flt_coord"], "depth": nd["flt_depth"],
            "children": nd["flt_children"], "parent_end": nd["flt_parent_end"], "edge_off": edge_off,
            "edge_parent": ed["flt_edge_parent"], "edge_slot": ed["flt_edge_slot"]}
    dags["edge_source_slot"] = dags["edge_slot"]
    point_off, pd = csr("flt_point_off", ["flt_points"], g["point_off"], [g["points"]])
    hseg_off, hd = csr("flt_hseg_off", ["flt_hsegs"], g["hseg_off"], [g["hsegs"]], width=2)
    vseg_off, vd = csr("flt_vseg_off", ["flt_vsegs"], g["vseg_off"], [g["vsegs"]], width=2)
    geom = (point_off, pd["flt_points"], hseg_off, hd["flt_hsegs"], vseg_off, vd["flt_vsegs"])
    words = np.where(slot_of >= 0, g["pin_count"].astype(np.int64) * ROUTE_PER_PIN_PHASE2, 0)
    route2_off = np.concatenate([[0], np.cumsum(words)]).astype(np.int64)
    return dags, geom, route2_off


def segment_multiset(r: np.ndarray):
    """Sorted (a, b) pairs of one route record [count, a0, b0, ...]."""
    if len(r) == 0 or r[0] <= 1:
        return []
    w = r[1:r[0]].reshape(-1, 2)
    return sorted(map(tuple, w.tolist()))


def ref_routes2_of(g: dict, net: int) -> np.ndarray:
    base = int(g["flt_pin_acc2"][net]) * ROUTE_PER_PIN_PHASE2
    return g["flt_routes2"][base:base + int(g["pin_count"][net]) * ROUTE_PER_PIN_PHASE2]


def route_geometry(r: np.ndarray, X: int, Y: int):
    """Canonical geometry of one route record: sorted unit wire edges
    (cell ids) and via stacks.  Two records with the same geometry put the
    same demand on the grid and score the same; they may still split a
    straight run into different segments."""
    XY = X * Y
    edges, vias = [], []
    for a, b in segment_multiset(r):
        if a // XY != b // XY:
            vias.append((a, b))
            continue
        l = a // XY
        xa, ya, xb, yb = a % XY // Y, a % Y, b % XY // Y, b % Y
        if xa == xb:
            edges += [l * XY + xa * Y + y for y in range(min(ya, yb), max(ya, yb))]
        else:
            edges += [l * XY + x * Y + ya for x in range(min(xa, xb), max(xa, xb))]
    return sorted(edges), sorted(vias)


class device_exp_table:
    """Context manager: install in the oracle the device's own values of the
    cost model's exponential (grb_cost_exp on cuda:0) for every argument the
    cost model can produce on `og` up to `max_demand_half`, so the oracle's
    cost tables are bit-identical to the device's; removed on exit.  `misses`
    is the number of exponentials the oracle evaluated outside the table."""

    def __init__(self, og, max_demand_half):
        self.og, self.hmax, self.misses = og, int(max_demand_half), None

    def __enter__(self):
        import ctypes as C

        import oracle
        from grotor_b200 import _abi
        x = oracle.exp_args(self.og, self.hmax)
        y = np.empty_like(x)
        rc = _abi.load().grb_cost_exp(0, x.ctypes.data_as(C.c_void_p), len(x), y.ctypes.data_as(C.c_void_p))
        assert rc == 0, f"grb_cost_exp failed ({rc})"
        oracle.set_exp_table(x, y)
        return self

    def __exit__(self, *exc):
        import oracle
        self.misses = oracle.exp_table_misses()
        oracle.set_exp_table()
        return False
