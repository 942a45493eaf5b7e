"""Seeded synthetic designs (wrapper of include/grb_synth.h, libgrb_synth.so).

Five workloads follow the reference benchmark plan (GCell grid, capacity
model, pin-count and bounding-box distributions); ``scaled`` variants keep a
workload's distributions at a smaller net count for tests.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, replace

import numpy as np

from . import _abi
from .router import GridArrays, NetArrays


@dataclass(frozen=True)
class SynthParams:
    X: int
    Y: int
    cap_layers: int
    n_nets: int
    cap_lo: int
    cap_hi: int
    blockage: float = 0.0
    unit_wire: float = 1.0
    unit_via: float = 2.0
    overflow_weight: float = 1.0
    pin_model: int = 0
    two_pin_frac: float = 0.7
    geo_p: float = 0.35
    max_pins: int = 16
    pareto_alpha: float = 1.6
    bbox_model: int = 0
    bbox_median: float = 6.0
    bbox_sigma: float = 0.75
    big_frac: float = 0.0
    big_lo: int = 0
    big_hi: int = 0
    bbox_max: int = 0
    pin_cap_layers: int = 2
    seed: int = 1

    def scaled(self, n_nets: int, **kw) -> "SynthParams":
        return replace(self, n_nets=n_nets, **kw)


# Workloads (grid, capacities, pin and bbox distributions per configuration).
WORKLOADS = {
    # 64x64, 5 metal layers, capacity U{4..12}, 5,000 nets (70% 2-pin, 3+Geom(0.35)<=16), bbox LogNormal(ln 6, .75)
    "small_64x64x5": SynthParams(64, 64, 5, 5000, 4, 12, seed=1),
    # 320x320x10, capacity U{6..20}, 10% blockages, 120K nets (65% 2-pin, tail to 64), median 12, 1% spanning >half
    "medium_320x320x10": SynthParams(320, 320, 10, 120000, 6, 20, blockage=0.10, two_pin_frac=0.65, max_pins=64,
                                     bbox_median=12.0, big_frac=0.01, big_lo=160, big_hi=320, seed=2),
    # 800x800x10, 900K nets with the medium distributions
    "large_800x800x10": SynthParams(800, 800, 10, 900000, 6, 20, blockage=0.10, two_pin_frac=0.65, max_pins=64,
                                    bbox_median=12.0, big_frac=0.01, big_lo=400, big_hi=800, seed=3),
    # 1600x1600x10, 3M nets, pins 2 + floor(Lomax(1.6)) <= 256, bbox log-uniform [1, 1600]
    "persistent_1600x1600x10": SynthParams(1600, 1600, 10, 3000000, 6, 20, blockage=0.10, pin_model=1,
                                           max_pins=256, pareto_alpha=1.6, bbox_model=1, bbox_max=1600, seed=4),
    # soft-min workload (320x320x10, medium distribution) and its 32x32x4 gradient-check case
    "softmin_320x320x10": SynthParams(320, 320, 10, 120000, 6, 20, blockage=0.10, two_pin_frac=0.65, max_pins=64,
                                      bbox_median=12.0, big_frac=0.01, big_lo=160, big_hi=320, seed=5),
    "softmin_check_32x32x4": SynthParams(32, 32, 4, 200, 2, 6, seed=6),
}


class Design:
    """A generated design plus its routing topology (host arrays)."""

    def __init__(self, params: SynthParams, max_subnet_pins: int = 12, threads: int = 0):
        self._lib = _abi.load_synth()
        self.params = params
        s = _abi.GrbSynthParams(**{f: getattr(params, f) for f, _ in _abi.GrbSynthParams._fields_})
        self._d = C.c_void_p(self._lib.grb_synth_generate(C.byref(s)))
        err = self._lib.grb_design_error(self._d).decode()
        if err:
            raise ValueError(err)
        g = _abi.GrbGrid()
        self._lib.grb_design_grid(self._d, C.byref(g))
        L, X, Y = g.L, g.X, g.Y
        self.grid = GridArrays(
            L, X, Y, g.DIR, g.unit_length_wire_cost, g.unit_via_cost,
            _arr(g.unit_length_short_costs, C.c_double, L).copy(),
            _arr(g.x_edge_len, C.c_int32, X - 1).copy(), _arr(g.y_edge_len, C.c_int32, Y - 1).copy(),
            _arr(g.capacity, C.c_float, L * X * Y).copy())
        if self._lib.grb_design_build_topology(self._d, int(max_subnet_pins), int(threads)):
            raise ValueError("topology construction failed")
        n = _abi.GrbNets()
        self._lib.grb_design_nets(self._d, C.byref(n))
        m = n.n
        node_off = _arr(n.node_off, C.c_int32, m + 1).copy()
        point_off = _arr(n.point_off, C.c_int32, m + 1).copy()
        hseg_off = _arr(n.hseg_off, C.c_int32, m + 1).copy()
        vseg_off = _arr(n.vseg_off, C.c_int32, m + 1).copy()
        self.nets = NetArrays(
            node_off, _arr(n.nodes, C.c_int32, node_off[-1]).copy(), _arr(n.parents, C.c_int32, node_off[-1]).copy(),
            _arr(n.route_off, C.c_int64, m + 1).copy(), point_off, _arr(n.points, C.c_int32, point_off[-1]).copy(),
            hseg_off, _arr(n.hsegs, C.c_int32, 2 * hseg_off[-1]).copy(), vseg_off,
            _arr(n.vsegs, C.c_int32, 2 * vseg_off[-1]).copy())
        hp, orig, pc = C.c_void_p(), C.c_void_p(), C.c_void_p()
        self._lib.grb_design_subnet_info(self._d, C.byref(hp), C.byref(orig), C.byref(pc))
        self.hpwl = _arr(hp, C.c_int32, m).copy()
        self.original = _arr(orig, C.c_int32, m).copy()
        self.pin_count = _arr(pc, C.c_int32, m).copy()
        self.order = np.empty(m, np.int32)
        self._lib.grb_design_order(self._d, self.order.ctypes.data_as(C.c_void_p))

    @property
    def n_subnets(self) -> int:
        return self.nets.n

    def zshape_trees(self) -> dict:
        """The same trees in the Z-shape encoding (upload with Router.upload_zshape)."""
        off, crd, ch = C.c_void_p(), C.c_void_p(), C.c_void_p()
        if self._lib.grb_design_zshape_trees(self._d, C.byref(off), C.byref(crd), C.byref(ch)):
            raise ValueError(self._lib.grb_design_error(self._d).decode())
        m = self.nets.n
        o = _arr(off, C.c_int32, m + 1).copy()
        return {"node_off": o, "coord": _arr(crd, C.c_int32, o[-1]).copy(), "child": _arr(ch, C.c_int32, 3 * o[-1]).copy()}

    def pins(self):
        off, pins, n = C.c_void_p(), C.c_void_p(), C.c_int32()
        self._lib.grb_design_pins(self._d, C.byref(off), C.byref(pins), C.byref(n))
        o = _arr(off, C.c_int32, n.value + 1).copy()
        return o, _arr(pins, C.c_int32, o[-1]).copy()

    def write(self, cap_path: str, net_path: str):
        if self._lib.grb_design_write(self._d, cap_path.encode(), net_path.encode()):
            raise OSError("cannot write design files")

    def close(self):
        if self._d:
            self._lib.grb_design_free(self._d)
            self._d = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _arr(ptr, ctype, count):
    count = int(count)
    if count == 0:
        return np.zeros(0, np.dtype(ctype))
    addr = ptr.value if isinstance(ptr, C.c_void_p) else ptr
    return np.ctypeslib.as_array(C.cast(addr, C.POINTER(ctype)), shape=(count,))


def steiner_trees(nets: NetArrays, shuffle_seed: int | None = None):
    """The nets' trees in the form FLUTE leaves them (grb_trees): node
    positions and adjacency lists, from the depth-first arrays.

    Without a seed every node lists its parent first and then its children by
    index, so the depth-first flattening from node 0 gives the arrays back.
    With a seed the nodes of every net are relabelled (node 0 included, which
    re-roots the tree) and every adjacency list is shuffled."""
    from .router import TreeArrays
    node_off = np.asarray(nets.node_off, np.int64)
    n, nn = len(node_off) - 1, int(node_off[-1])
    net_of = np.repeat(np.arange(n, dtype=np.int64), np.diff(node_off))
    local = np.arange(nn, dtype=np.int64) - node_off[net_of]
    parents = np.asarray(nets.parents, np.int64)
    if shuffle_seed is None:
        new_of_old = np.arange(nn, dtype=np.int64)
    else:
        rng = np.random.default_rng(shuffle_seed)
        order = np.lexsort((rng.random(nn), net_of))
        new_of_old = np.empty(nn, np.int64)
        new_of_old[order] = np.arange(nn, dtype=np.int64)
    pos = np.empty(nn, np.int32)
    pos[new_of_old] = np.asarray(nets.nodes, np.int32)
    child = np.flatnonzero(local > 0)
    par = node_off[net_of[child]] + parents[child]
    a, b = new_of_old[child], new_of_old[par]
    src = np.concatenate([a, b])
    dst = np.concatenate([b, a])
    if shuffle_seed is None:
        # Parent entries first (key -1), then children by their index.
        key = np.concatenate([np.full(len(a), -1, np.int64), a])
        perm = np.lexsort((key, src))
    else:
        perm = np.lexsort((rng.random(len(src)), src))
    src, dst = src[perm], dst[perm]
    adj_off = np.zeros(nn + 1, np.int64)
    np.add.at(adj_off, src + 1, 1)
    adj_off = np.cumsum(adj_off).astype(np.int32)
    adj = (dst - node_off[net_of[dst]]).astype(np.int32)
    return TreeArrays(np.asarray(nets.node_off, np.int32), pos, adj_off, adj, np.asarray(nets.route_off, np.int64))


def _main(argv=None):
    """``python -m grotor_b200.synth WORKLOAD CAP NET`` writes a workload's
    design as the reference's .cap and .net input files."""
    import argparse
    ap = argparse.ArgumentParser(prog="python -m grotor_b200.synth")
    ap.add_argument("workload", choices=sorted(WORKLOADS))
    ap.add_argument("cap")
    ap.add_argument("net")
    args = ap.parse_args(argv)
    Design(WORKLOADS[args.workload]).write(args.cap, args.net)


if __name__ == "__main__":
    _main()
