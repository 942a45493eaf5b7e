"""ctypes bindings of liboracle.so (CPU restatement; test infrastructure only)."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")

__all__ = [
    "build", "load", "OrcGrid", "cost_full", "presum", "presum_logstep", "lshape_batch",
    "commit_batch", "batches", "ripup_classify", "congestion_view", "lshape_stage", "flt_stage", "zshape_stage",
    "bbox_batches", "exp_args", "set_exp_table", "exp_table_misses", "build_topology",
]


def build() -> None:
    """Compile liboracle.so in place (g++, no GPU needed)."""
    subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)


_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        _lib = C.CDLL(_LIB)
        _declare(_lib)
    return _lib


class _COrcGrid(C.Structure):
    _fields_ = [
        ("L", C.c_int32), ("X", C.c_int32), ("Y", C.c_int32), ("DIR", C.c_int32),
        ("unit_wire", C.c_double), ("unit_via", C.c_double), ("of_cost_scale", C.c_double),
        ("short_costs", C.c_void_p), ("x_edge_len", C.c_void_p), ("y_edge_len", C.c_void_p),
        ("capacity", C.c_void_p), ("integer_wire", C.c_int32),
    ]


P = C.c_void_p


def _declare(lib):
    lib.orc_cost_full.argtypes = [P, P, P, P]
    lib.orc_presum.argtypes = [P, P, P]
    lib.orc_presum_logstep.argtypes = [P, P, P]
    lib.orc_lshape_batch.argtypes = [P, P, P, C.c_int32, P, P, P, P, P, P]
    lib.orc_lshape_batch.restype = C.c_int
    lib.orc_commit_batch.argtypes = [P, C.c_int32, P, P, P, C.c_int32, C.c_int32, P, P, P, P]
    lib.orc_batches.argtypes = [C.c_int32, C.c_int32, C.c_int32, P, P, P, P, P, P, P, C.c_int32, C.c_int32, P]
    lib.orc_batches.restype = C.c_int32
    lib.orc_ripup_classify.argtypes = [P, P, C.c_int32, C.c_int32, P, P, P]
    lib.orc_congestion_view.argtypes = [P, P, P, P, P]
    lib.orc_build_topology.argtypes = [C.c_int32, C.c_int32, C.c_int32] + [P] * 13
    lib.orc_build_topology.restype = C.c_int
    lib.orc_lshape_stage.argtypes = [P, C.c_int32, P, P, P, P, P, P, P, P, P, P, P, P, C.c_int32]
    lib.orc_lshape_stage.restype = C.c_int
    lib.orc_flt_stage.argtypes = [P, P, C.c_int32, P, P, P, P, P, P, C.c_int32, P, P, P, P, P, C.c_int32]
    lib.orc_flt_stage.restype = C.c_int
    lib.orc_zshape_stage.argtypes = [P, P, C.c_int32, P, P, P, P, P, P, P, P, P]
    lib.orc_zshape_stage.restype = C.c_int
    lib.orc_bbox_batches.argtypes = [C.c_int32, C.c_int32, C.c_int32, P, P, C.c_int32, P, P]
    lib.orc_bbox_batches.restype = C.c_int32
    lib.orc_exp_args.argtypes = [P, C.c_int32, P, C.c_int64]
    lib.orc_exp_args.restype = C.c_int64
    lib.orc_set_exp_table.argtypes = [C.c_int64, P, P]
    lib.orc_exp_table_misses.restype = C.c_int64


class _COrcFlt(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in ("node_off", "coord", "depth", "children", "parent_end", "edge_off",
                                          "edge_parent", "edge_slot")]


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


class OrcGrid:
    """Grid arrays in the oracle's layout (keeps the numpy buffers alive)."""

    def __init__(self, L, X, Y, DIR, unit_wire, unit_via, short_costs, x_edge_len, y_edge_len, capacity,
                 of_cost_scale=1.0, integer_wire=False):
        self.L, self.X, self.Y, self.DIR = int(L), int(X), int(Y), int(DIR)
        self.short_costs = _c(short_costs, np.float64)
        self.x_edge_len = _c(x_edge_len, np.int32)
        self.y_edge_len = _c(y_edge_len, np.int32)
        self.capacity = _c(capacity, np.float32).reshape(-1)
        self.unit_wire, self.unit_via, self.of_cost_scale = float(unit_wire), float(unit_via), float(of_cost_scale)
        self._s = _COrcGrid(self.L, self.X, self.Y, self.DIR, self.unit_wire, self.unit_via, self.of_cost_scale,
                            _p(self.short_costs), _p(self.x_edge_len), _p(self.y_edge_len), _p(self.capacity),
                            int(bool(integer_wire)))

    @property
    def cells(self):
        return self.L * self.X * self.Y

    @property
    def ref(self):
        return C.byref(self._s)


def cost_full(g: OrcGrid, demand_half):
    lib = load()
    d = _c(demand_half, np.int32)
    w = np.empty(g.cells, np.float32)
    v = np.empty(g.cells, np.float32)
    lib.orc_cost_full(g.ref, _p(d), _p(w), _p(v))
    return w, v


def presum(g: OrcGrid, wcost):
    lib = load()
    w = _c(wcost, np.float32)
    out = np.empty(g.cells, np.float64)
    lib.orc_presum(g.ref, _p(w), _p(out))
    return out


def presum_logstep(g: OrcGrid, wcost):
    lib = load()
    w = _c(wcost, np.float32)
    out = np.empty(g.cells, np.float64)
    lib.orc_presum_logstep(g.ref, _p(w), _p(out))
    return out


def lshape_batch(g: OrcGrid, vcost, presum_, ids, node_off, nodes, parents, route_off, routes):
    """Route nets `ids` into `routes` (modified in place); returns status."""
    lib = load()
    ids = _c(ids, np.int32)
    return lib.orc_lshape_batch(g.ref, _p(_c(vcost, np.float32)), _p(_c(presum_, np.float64)), len(ids), _p(ids),
                                _p(_c(node_off, np.int32)), _p(_c(nodes, np.int32)), _p(_c(parents, np.int32)),
                                _p(_c(route_off, np.int64)), _p(routes))


def commit_batch(g: OrcGrid, ids, route_off, routes, stamp, K, demand_half, timestamp, stats=None):
    """Wire then via commit; demand_half/timestamp are int32 arrays modified in place.
    stats: optional dict with 'wirelength' and 'vias' accumulated in place."""
    lib = load()
    ids = _c(ids, np.int32)
    wl = C.c_double(stats["wirelength"] if stats else 0.0)
    vi = C.c_int64(stats["vias"] if stats else 0)
    lib.orc_commit_batch(g.ref, len(ids), _p(ids), _p(_c(route_off, np.int64)), _p(_c(routes, np.int32)),
                         int(stamp), int(K), _p(demand_half), _p(timestamp), C.byref(wl), C.byref(vi))
    if stats is not None:
        stats["wirelength"], stats["vias"] = wl.value, vi.value


def batches(X, Y, order, point_off, points, hseg_off, hsegs, vseg_off, vsegs, limit, sparsity=1):
    lib = load()
    order = _c(order, np.int32)
    out = np.empty(len(order), np.int32)
    nb = lib.orc_batches(int(X), int(Y), len(order), _p(order), _p(_c(point_off, np.int32)), _p(_c(points, np.int32)),
                         _p(_c(hseg_off, np.int32)), _p(_c(hsegs, np.int32)), _p(_c(vseg_off, np.int32)),
                         _p(_c(vsegs, np.int32)), int(limit), int(sparsity), _p(out))
    return out, int(nb)


def ripup_classify(g: OrcGrid, demand_half, threshold, route_off, routes):
    lib = load()
    n = len(route_off) - 1
    out = np.zeros(n, np.uint8)
    lib.orc_ripup_classify(g.ref, _p(_c(demand_half, np.int32)), int(threshold), n, _p(_c(route_off, np.int64)),
                           _p(_c(routes, np.int32)), _p(out))
    return out


def congestion_view(g: OrcGrid, demand_half):
    lib = load()
    xy = g.X * g.Y
    cong = np.empty(xy, np.uint8)
    xs = np.empty(xy, np.float32)
    ys = np.empty(xy, np.float32)
    lib.orc_congestion_view(g.ref, _p(_c(demand_half, np.int32)), _p(cong), _p(xs), _p(ys))
    return cong, xs, ys


def lshape_stage(g: OrcGrid, ids, batch_off, node_off, nodes, parents, route_off, threads=0,
                 demand_half=None, timestamp=None, stamp=0):
    """Full L-shape stage on the CPU; returns dict with routes, demand, timestamps, stats."""
    lib = load()
    ids = _c(ids, np.int32)
    batch_off = _c(batch_off, np.int32)
    route_off = _c(route_off, np.int64)
    routes = np.zeros(int(route_off[-1]), np.int32)
    demand = np.zeros(g.cells, np.int32) if demand_half is None else _c(demand_half, np.int32).copy()
    ts = np.zeros(g.cells, np.int32) if timestamp is None else _c(timestamp, np.int32).copy()
    st = C.c_int32(stamp)
    wl = C.c_double(0)
    vi = C.c_int64(0)
    rc = lib.orc_lshape_stage(g.ref, len(batch_off) - 1, _p(batch_off), _p(ids), _p(_c(node_off, np.int32)),
                              _p(_c(nodes, np.int32)), _p(_c(parents, np.int32)), _p(route_off), _p(routes),
                              _p(demand), _p(ts), C.byref(st), C.byref(wl), C.byref(vi), int(threads))
    return {"status": rc, "routes": routes, "demand_half": demand, "timestamp": ts, "stamp": st.value,
            "wirelength": wl.value, "vias": vi.value}



def flt_stage(g: OrcGrid, dags: dict, ids, batch_off, route_off, routes, route2_off, demand_half, timestamp, stamp,
              remove_phase_one=True, threads=0, wirelength=0.0, vias=0):
    """FLT stage on the CPU.  `dags` holds the CSR arrays by net id (node_off,
    coord, depth, children, parent_end, edge_off, edge_parent, edge_slot)."""
    lib = load()
    keep = {k: _c(dags[k], np.int32) for k, _ in _COrcFlt._fields_}
    d = _COrcFlt(**{k: v.ctypes.data for k, v in keep.items()})
    ids = _c(ids, np.int32)
    batch_off = _c(batch_off, np.int32)
    route2_off = _c(route2_off, np.int64)
    routes2 = np.zeros(int(route2_off[-1]), np.int32)
    demand = _c(demand_half, np.int32).copy()
    ts = _c(timestamp, np.int32).copy()
    st = C.c_int32(stamp)
    wl = C.c_double(wirelength)
    vi = C.c_int64(vias)
    rc = lib.orc_flt_stage(g.ref, C.byref(d), len(batch_off) - 1, _p(batch_off), _p(ids), _p(_c(route_off, np.int64)),
                           _p(_c(routes, np.int32)), _p(route2_off), _p(routes2), int(bool(remove_phase_one)),
                           _p(demand), _p(ts), C.byref(st), C.byref(wl), C.byref(vi), int(threads))
    return {"status": rc, "routes2": routes2, "demand_half": demand, "timestamp": ts, "stamp": st.value,
            "wirelength": wl.value, "vias": vi.value}


class _COrcZTrees(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in ("node_off", "coord", "child")]


def zshape_stage(g: OrcGrid, trees: dict, ids, batch_off, route_off, demand_half=None, timestamp=None, stamp=0,
                 wirelength=0.0, vias=0):
    """Z-shape stage on the CPU (g built with integer_wire=True for the
    reference's GGR cost mode).  `trees`: node_off, coord, child (3 per node)."""
    lib = load()
    keep = {k: _c(trees[k], np.int32) for k, _ in _COrcZTrees._fields_}
    t = _COrcZTrees(**{k: v.ctypes.data for k, v in keep.items()})
    ids = _c(ids, np.int32)
    batch_off = _c(batch_off, np.int32)
    route_off = _c(route_off, np.int64)
    routes = np.zeros(int(route_off[-1]), np.int32)
    demand = np.zeros(g.cells, np.int32) if demand_half is None else _c(demand_half, np.int32).copy()
    ts = np.zeros(g.cells, np.int32) if timestamp is None else _c(timestamp, np.int32).copy()
    st = C.c_int32(stamp)
    wl = C.c_double(wirelength)
    vi = C.c_int64(vias)
    rc = lib.orc_zshape_stage(g.ref, C.byref(t), len(batch_off) - 1, _p(batch_off), _p(ids), _p(route_off),
                              _p(routes), _p(demand), _p(ts), C.byref(st), C.byref(wl), C.byref(vi))
    return {"status": rc, "routes": routes, "demand_half": demand, "timestamp": ts, "stamp": st.value,
            "wirelength": wl.value, "vias": vi.value}


def bbox_batches(X, Y, group, bbox, max_batch=250):
    """Bounding-box refinement of one first-fit group: list of batches."""
    lib = load()
    group = _c(group, np.int32)
    ids = np.empty(len(group), np.int32)
    off = np.empty(len(group) + 1, np.int32)
    nb = lib.orc_bbox_batches(int(X), int(Y), len(group), _p(group), _p(_c(bbox, np.int32)), int(max_batch),
                              _p(ids), _p(off))
    return [ids[off[k]:off[k + 1]].tolist() for k in range(nb)]


def exp_args(g: OrcGrid, max_demand_half: int) -> np.ndarray:
    """Every argument the cost model can pass to the exponential on this grid
    for cell demands up to max_demand_half half-units (ascending, unique)."""
    lib = load()
    n = lib.orc_exp_args(g.ref, int(max_demand_half), None, 0)
    out = np.empty(n, np.float32)
    lib.orc_exp_args(g.ref, int(max_demand_half), _p(out), n)
    return out


def set_exp_table(x=None, y=None) -> None:
    """Install the device's exponential values y = exp(x) (None removes them)."""
    lib = load()
    if x is None:
        lib.orc_set_exp_table(0, None, None)
        return
    x = _c(x, np.float32)
    y = _c(y, np.float32)
    assert x.shape == y.shape
    lib.orc_set_exp_table(len(x), _p(x), _p(y))


def exp_table_misses() -> int:
    return int(load().orc_exp_table_misses())


def build_topology(X, Y, node_off, pos, adj_off, adj):
    """Per-net DP trees and batching geometry from Steiner trees
    (orc_build_topology); returns a dict of the flat arrays."""
    lib = load()
    node_off = _c(node_off, np.int32)
    n = len(node_off) - 1
    nn = int(node_off[-1])
    out = {"node_off": node_off.copy(), "nodes": np.zeros(nn, np.int32), "parents": np.zeros(nn, np.int32),
           "point_off": np.zeros(n + 1, np.int32), "points": np.zeros(3 * nn, np.int32),
           "hseg_off": np.zeros(n + 1, np.int32), "hsegs": np.zeros(4 * nn, np.int32),
           "vseg_off": np.zeros(n + 1, np.int32), "vsegs": np.zeros(4 * nn, np.int32)}
    totals = np.zeros(3, np.int64)
    rc = lib.orc_build_topology(int(X), int(Y), n, _p(node_off), _p(_c(pos, np.int32)), _p(_c(adj_off, np.int32)),
                                _p(_c(adj, np.int32)), _p(out["nodes"]), _p(out["parents"]), _p(out["point_off"]),
                                _p(out["points"]), _p(out["hseg_off"]), _p(out["hsegs"]), _p(out["vseg_off"]),
                                _p(out["vsegs"]), _p(totals))
    if rc:
        raise ValueError(f"net {-rc - 1}: adjacency is not a tree on its nodes")
    out["points"] = out["points"][:totals[0]]
    out["hsegs"] = out["hsegs"][:2 * totals[1]]
    out["vsegs"] = out["vsegs"][:2 * totals[2]]
    return out
