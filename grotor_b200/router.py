"""Host-side mirror of GRotor's routing-path interface over the C ABI.

``Router`` plays the role of ``cudb::RouterState`` (router_state.hpp:182-232)
and exposes the reference's hot-path seams under their reference names:

* ``generate_batches_rsmt``  -- cudb::generate_batches_rsmt (generate_batches_cpu.hpp:7)
* ``refresh_cost``           -- graph::refresh_cost (incremental_update.cuh:98)
* ``route_batch``            -- the Lshape_route_warp launch (lshape.cuh:168)
* ``commit_batch_demand``    -- graph::commit_batch_demand (demand.cuh:313)
* ``lshape_route``           -- Lshape_route::Lshape_route's hot loop (lshape.cuh:153-179)
* ``ripup``                  -- graph::ripup (congestion.cuh:114)

Errors raise ``GrbError`` with the library's message (the reference throws
std::runtime_error from cuda_check, cuda_memory.hpp:12-15).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi

MODE_PLAIN, MODE_GRAPH, MODE_PERSISTENT = _abi.MODE_PLAIN, _abi.MODE_GRAPH, _abi.MODE_PERSISTENT
_MODES = {"plain": MODE_PLAIN, "graph": MODE_GRAPH, "persistent": MODE_PERSISTENT}


class GrbError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{_abi.ERROR_NAMES.get(code, code)}: {message}")
        self.code = code


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def mode_id(mode) -> int:
    return _MODES[mode] if isinstance(mode, str) else int(mode)


@dataclass
class GridArrays:
    L: int
    X: int
    Y: int
    DIR: int
    unit_wire: float
    unit_via: float
    short_costs: np.ndarray
    x_edge_len: np.ndarray
    y_edge_len: np.ndarray
    capacity: np.ndarray
    of_cost_scale: float = 1.0

    @property
    def cells(self) -> int:
        return self.L * self.X * self.Y

    def struct(self) -> _abi.GrbGrid:
        self._keep = [_c(self.short_costs, np.float64), _c(self.x_edge_len, np.int32),
                      _c(self.y_edge_len, np.int32), _c(self.capacity, np.float32).reshape(-1)]
        s = _abi.GrbGrid(self.L, self.X, self.Y, self.DIR, self.unit_wire, self.unit_via, self.of_cost_scale,
                         *[_p(a) for a in self._keep])
        return s


@dataclass
class NetArrays:
    node_off: np.ndarray
    nodes: np.ndarray
    parents: np.ndarray
    route_off: np.ndarray
    point_off: np.ndarray
    points: np.ndarray
    hseg_off: np.ndarray
    hsegs: np.ndarray
    vseg_off: np.ndarray
    vsegs: np.ndarray

    @property
    def n(self) -> int:
        return len(self.node_off) - 1

    def struct(self) -> _abi.GrbNets:
        self._keep = [_c(self.node_off, np.int32), _c(self.nodes, np.int32), _c(self.parents, np.int32),
                      _c(self.route_off, np.int64), _c(self.point_off, np.int32), _c(self.points, np.int32),
                      _c(self.hseg_off, np.int32), _c(self.hsegs, np.int32), _c(self.vseg_off, np.int32),
                      _c(self.vsegs, np.int32)]
        return _abi.GrbNets(self.n, *[_p(a) for a in self._keep])


@dataclass
class TreeArrays:
    """Steiner trees of every net (grb_trees): node positions with their
    layer (L = Steiner point) and each node's adjacency list."""
    node_off: np.ndarray
    pos: np.ndarray
    adj_off: np.ndarray
    adj: np.ndarray
    route_off: np.ndarray

    @property
    def n(self) -> int:
        return len(self.node_off) - 1

    def struct(self) -> _abi.GrbTrees:
        self._keep = [_c(self.node_off, np.int32), _c(self.pos, np.int32), _c(self.adj_off, np.int32),
                      _c(self.adj, np.int32), _c(self.route_off, np.int64)]
        return _abi.GrbTrees(self.n, *[_p(a) for a in self._keep])


class Router:
    """One routing context on one GPU (owns device memory and a CUDA stream)."""

    def __init__(self, grid: GridArrays, device: int = 0):
        self._lib = _abi.load()
        self.grid = grid
        self._ctx = C.c_void_p()
        s = grid.struct()
        rc = self._lib.grb_create(C.byref(s), int(device), C.byref(self._ctx))
        if rc:
            raise GrbError(rc, "grb_create failed")
        self.nets: NetArrays | None = None
        self._n = 0            # nets in the context's store
        self._route_words = 0  # route words of the store

    # -- lifecycle ---------------------------------------------------------
    def close(self):
        if self._ctx:
            self._lib.grb_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int):
        if rc:
            raise GrbError(rc, self._lib.grb_last_error(self._ctx).decode())

    @property
    def stream_handle(self) -> int:
        return int(self._lib.grb_stream(self._ctx) or 0)

    @property
    def kernel_launches(self) -> int:
        return int(self._lib.grb_kernel_launches(self._ctx))

    def reset(self):
        self._check(self._lib.grb_reset(self._ctx))

    def upload_nets(self, nets: NetArrays):
        s = nets.struct()
        self._check(self._lib.grb_upload_nets(self._ctx, C.byref(s)))
        self.nets = nets
        self._n = nets.n
        self._route_words = int(nets.route_off[-1])

    def build_topology(self, trees: "TreeArrays"):
        """Build every net's DP tree and batching geometry on the device from
        its Steiner tree (grb_build_topology)."""
        s = trees.struct()
        self._check(self._lib.grb_build_topology(self._ctx, C.byref(s)))
        self.nets = None
        self._n = trees.n
        self._route_words = int(trees.route_off[-1])

    def _n_nets(self) -> int:
        return self._n

    def read_topology(self) -> dict:
        """The context's net store: trees in DFS order and batching geometry."""
        sizes = np.zeros(4, np.int64)
        self._check(self._lib.grb_topology_sizes(self._ctx, _p(sizes)))
        n1 = self._n_nets() + 1
        nn, npt, nh, nv = (int(v) for v in sizes)
        out = {"node_off": np.empty(n1, np.int32), "nodes": np.empty(nn, np.int32),
               "parents": np.empty(nn, np.int32), "point_off": np.empty(n1, np.int32),
               "points": np.empty(npt, np.int32), "hseg_off": np.empty(n1, np.int32),
               "hsegs": np.empty(2 * nh, np.int32), "vseg_off": np.empty(n1, np.int32),
               "vsegs": np.empty(2 * nv, np.int32)}
        self._check(self._lib.grb_read_topology(self._ctx, *(_p(out[k]) for k in (
            "node_off", "nodes", "parents", "point_off", "points", "hseg_off", "hsegs", "vseg_off", "vsegs"))))
        return out

    def write_out(self, names, pins, extra, subnets, phase2=None) -> bytes:
        """The .out text of output records (graph::output_nets), formatted on
        the device from the context's routes (grb_format_out) and drained to
        the host (grb_drain_out).  Per record: its name, its 3-D pins, its
        extra route pairs (flat 3-D positions) and its subnet ids, with
        per-subnet phase-two flags (default 0)."""
        def csr(lists, dtype):
            off = np.zeros(len(lists) + 1, np.int32)
            off[1:] = np.cumsum([len(v) for v in lists])
            flat = np.concatenate([np.asarray(v, dtype) for v in lists]) if lists else np.zeros(0, dtype)
            return off, np.ascontiguousarray(flat, dtype)
        raw = [n.encode() if isinstance(n, str) else bytes(n) for n in names]
        name_off = np.zeros(len(raw) + 1, np.int64)
        name_off[1:] = np.cumsum([len(b) for b in raw])
        name_buf = np.frombuffer(b"".join(raw) or b"\0", np.uint8)
        pin_off, pin_flat = csr(pins, np.int32)
        extra_off, extra_flat = csr(extra, np.int32)
        sub_off, sub_flat = csr(subnets, np.int32)
        if phase2 is None:
            phase2 = [np.zeros(len(v), np.uint8) for v in subnets]
        _, ph_flat = csr(phase2, np.uint8)
        rec = _abi.GrbOutRecords(len(raw), _p(name_off), _p(name_buf), _p(pin_off), _p(pin_flat), _p(extra_off),
                                 _p(extra_flat), _p(sub_off), _p(sub_flat), _p(ph_flat))
        nbytes = C.c_int64(0)
        self._check(self._lib.grb_format_out(self._ctx, C.byref(rec), C.byref(nbytes)))
        parts = []

        def sink(data, size, _user):
            parts.append(C.string_at(data, size))
            return 0
        cb = _abi.OUT_SINK(sink)
        self._check(self._lib.grb_drain_out(self._ctx, cb, None))
        text = b"".join(parts)
        assert len(text) == nbytes.value
        return text

    # -- batching ------------------------------------------------------------
    def generate_batches_rsmt(self, order, limit: int = 1000000, sparsity: int = 1, mode="persistent"):
        """Exact first-fit batching; installs the reversed, flattened plan and
        returns (batch_of per order position, number of batches)."""
        order = _c(order, np.int32)
        out = np.empty(len(order), np.int32)
        nb = C.c_int32(0)
        self._check(self._lib.grb_plan_batches(self._ctx, _p(order), len(order), int(limit), int(sparsity),
                                               mode_id(mode), _p(out), C.byref(nb)))
        return out, nb.value

    def set_plan(self, ids, batch_off):
        ids = _c(ids, np.int32)
        batch_off = _c(batch_off, np.int32)
        self._check(self._lib.grb_set_plan(self._ctx, _p(ids), len(ids), _p(batch_off), len(batch_off) - 1))

    def plan(self):
        n, nb = C.c_int32(0), C.c_int32(0)
        self._check(self._lib.grb_get_plan(self._ctx, None, None, C.byref(n), C.byref(nb)))
        ids = np.empty(n.value, np.int32)
        off = np.empty(nb.value + 1, np.int32)
        self._check(self._lib.grb_get_plan(self._ctx, _p(ids), _p(off), C.byref(n), C.byref(nb)))
        return ids, off

    # -- per-batch seams -------------------------------------------------------
    def refresh_cost(self):
        self._check(self._lib.grb_refresh_cost(self._ctx))

    def route_batch(self, b: int, stamp: int):
        self._check(self._lib.grb_route_batch(self._ctx, int(b), int(stamp)))

    def commit_batch_demand(self, b: int, stamp: int, K: int = 1):
        self._check(self._lib.grb_commit_batch(self._ctx, int(b), int(stamp), int(K)))

    # -- stage -------------------------------------------------------------------
    def lshape_route(self, mode="persistent") -> dict:
        st = _abi.GrbStats()
        self._check(self._lib.grb_lshape_stage(self._ctx, mode_id(mode), C.byref(st)))
        return _stats_dict(st)

    # ---- FLT stage ----------------------------------------------------------
    def upload_geometry(self, point_off, points, hseg_off, hsegs, vseg_off, vsegs):
        """Replace the batching geometry (net::points and RSMT segments after the
        FLT DAG builder) so that ``generate_batches_rsmt`` batches the FLT stage."""
        a = [_c(v, np.int32) for v in (point_off, points, hseg_off, hsegs, vseg_off, vsegs)]
        self._check(self._lib.grb_upload_geometry(self._ctx, *[_p(v) for v in a]))

    def upload_flt(self, dags: dict, route2_off):
        """Upload FLT DAGs (CSR by net id: node_off, coord, depth, children,
        parent_end, edge_off, edge_parent, edge_source_slot) and the phase-two
        route offsets (int64, n+1)."""
        keep = {k: _c(dags[k], np.int32) for k in ("node_off", "coord", "depth", "children", "parent_end",
                                                    "edge_off", "edge_parent", "edge_source_slot")}
        keep["route2_off"] = _c(route2_off, np.int64)
        d = _abi.GrbFltDags(**{k: v.ctypes.data for k, v in keep.items()})
        self._check(self._lib.grb_upload_flt(self._ctx, C.byref(d)))
        self._route2_words = int(keep["route2_off"][-1])

    def flt_route(self, mode="persistent", remove_phase_one: bool = True) -> dict:
        """route_prepared_topology's batch loop over the current plan."""
        st = _abi.GrbStats()
        self._check(self._lib.grb_flt_stage(self._ctx, int(bool(remove_phase_one)), mode_id(mode), C.byref(st)))
        return _stats_dict(st)

    def set_flt_block_width(self, width: int):
        """Nets whose widest FLT DAG level holds more than `width` nodes are
        routed by a whole CTA (default 32; negative: every net by one warp)."""
        self._check(self._lib.grb_set_flt_block_width(self._ctx, int(width)))

    def read_routes2(self) -> np.ndarray:
        out = np.zeros(getattr(self, "_route2_words", 0), np.int32)
        self._check(self._lib.grb_read_routes2(self._ctx, _p(out)))
        return out

    def autotune(self, plain: bool = True, persistent: bool = True) -> dict:
        """Pick nets-per-CTA (per-batch DP launch) and nets-per-grab (persistent
        work queue) by size bucket (<= 2, <= 8, <= 16, > 16 tree nodes) on the
        current plan; leaves the context reset."""
        per_cta = np.zeros(4, np.int32)
        per_grab = np.zeros(4, np.int32)
        what = (1 if plain else 0) | (2 if persistent else 0)
        self._check(self._lib.grb_autotune(self._ctx, what, _p(per_cta), _p(per_grab)))
        return {"nets_per_cta": per_cta.tolist(), "nets_per_grab": per_grab.tolist()}

    # ---- Z-shape stage (GGR pipeline) ----------------------------------------
    def set_wire_cost_mode(self, integer_wire: bool):
        """True selects the GGR build's integer wire costs (clamped, truncated)."""
        self._check(self._lib.grb_set_wire_cost_mode(self._ctx, int(bool(integer_wire))))

    def upload_zshape(self, trees: dict):
        """Upload Z-shape trees (CSR by net id: node_off, coord, child[3 per node])."""
        keep = {k: _c(trees[k], np.int32) for k in ("node_off", "coord", "child")}
        t = _abi.GrbZshapeTrees(**{k: v.ctypes.data for k, v in keep.items()})
        self._check(self._lib.grb_upload_zshape(self._ctx, C.byref(t)))

    def plan_bbox_batches(self, max_batch: int = 250, bbox=None) -> int:
        """zshape::generate_bbox_batches over every batch of the current plan."""
        nb = C.c_int32(0)
        b = None if bbox is None else _c(bbox, np.int32)
        self._check(self._lib.grb_plan_bbox_batches(self._ctx, _p(b) if b is not None else None, int(max_batch),
                                                    C.byref(nb)))
        return nb.value

    def zshape_route(self, mode="persistent") -> dict:
        st = _abi.GrbStats()
        self._check(self._lib.grb_zshape_stage(self._ctx, mode_id(mode), C.byref(st)))
        return _stats_dict(st)

    def ripup(self, threshold: int = 0) -> np.ndarray:
        out = np.zeros(self._n, np.uint8)
        self._check(self._lib.grb_ripup_classify(self._ctx, int(threshold), _p(out)))
        return out

    def ripup_noalloc(self, threshold: int = 0) -> np.ndarray:
        """Same result as ``ripup``, computed without allocating device memory
        (for callers under a fixed device-memory budget or in loops that must
        not allocate); see grb_ripup_classify_noalloc in include/grb.h for the
        size limits and the rule that overlapping calls race."""
        out = np.zeros(self._n, np.uint8)
        self._check(self._lib.grb_ripup_classify_noalloc(self._ctx, int(threshold), _p(out)))
        return out

    def congestion_view(self):
        xy = self.grid.X * self.grid.Y
        cong = np.empty(xy, np.uint8)
        xs = np.empty(xy, np.float32)
        ys = np.empty(xy, np.float32)
        self._check(self._lib.grb_congestion_view(self._ctx, _p(cong), _p(xs), _p(ys)))
        return cong, xs, ys

    def set_stage_tail(self, ripup: bool = True, view: bool = True, threshold: int = 0):
        """Compute the rip-up classification and/or the congestion view of the
        final demand at the end of every following lshape_route (inside the
        persistent kernel, no host round trip); read with stage_tail()."""
        flags = (_abi.GRB_TAIL_RIPUP if ripup else 0) | (_abi.GRB_TAIL_VIEW if view else 0)
        self._check(self._lib.grb_set_stage_tail(self._ctx, flags, int(threshold)))
        self._tail = flags

    def stage_tail(self):
        """(is_of, (congestion, xsum, ysum)) of the last stage's tail (None for
        parts not computed)."""
        flags = getattr(self, "_tail", 0)
        xy = self.grid.X * self.grid.Y
        is_of = np.zeros(self._n, np.uint8) if flags & _abi.GRB_TAIL_RIPUP else None
        view = (np.empty(xy, np.uint8), np.empty(xy, np.float32), np.empty(xy, np.float32)) \
            if flags & _abi.GRB_TAIL_VIEW else None
        self._check(self._lib.grb_read_stage_tail(self._ctx, _p(is_of), *(_p(v) for v in (view or (None,) * 3))))
        return is_of, view

    # -- readback ----------------------------------------------------------------
    def read_tables(self) -> dict:
        n = self.grid.cells
        out = {"wcost": np.empty(n, np.float32), "vcost": np.empty(n, np.float32),
               "presum": np.empty(n, np.float64), "demand_half": np.empty(n, np.int32),
               "timestamp": np.empty(n, np.int32)}
        self._check(self._lib.grb_read_tables(self._ctx, _p(out["wcost"]), _p(out["vcost"]), _p(out["presum"]),
                                              _p(out["demand_half"]), _p(out["timestamp"])))
        return out

    def read_routes(self, out=None) -> np.ndarray:
        """All route words (route_off order).  ``out`` may be a caller-owned
        int32 buffer of at least that many words (pinned host memory makes the
        copy run at full PCIe rate)."""
        words = self._route_words
        if out is None:
            out = np.zeros(words, np.int32)
        elif out.dtype != np.int32 or not out.flags.c_contiguous or out.size < words:
            raise ValueError(f"out must be a contiguous int32 array of at least {words} words")
        self._check(self._lib.grb_read_routes(self._ctx, _p(out)))
        return out

    def read_routes_used(self, out: np.ndarray) -> np.ndarray:
        """Each net's route words in use (its count word and the words below
        it) into ``out`` (int32, route_off order); its other words are left as
        they were."""
        if out.dtype != np.int32 or not out.flags.c_contiguous or out.size < self._route_words:
            raise ValueError(f"out must be a contiguous int32 array of at least {self._route_words} words")
        self._check(self._lib.grb_read_routes_used(self._ctx, _p(out)))
        return out

    def write_routes_used(self, routes: np.ndarray):
        """Each net's route words in use, read from ``routes`` (count word at
        the net's offset), to the device; the device's other words are kept."""
        routes = np.ascontiguousarray(routes, np.int32)
        if routes.size < self._route_words:
            raise ValueError(f"routes must hold at least {self._route_words} words")
        self._check(self._lib.grb_write_routes_used(self._ctx, _p(routes)))

    def set_stats(self, wirelength: float = 0.0, vias: int = 0):
        self._check(self._lib.grb_set_stats(self._ctx, float(wirelength), int(vias)))

    def stats(self) -> dict:
        st = _abi.GrbStats()
        self._check(self._lib.grb_get_stats(self._ctx, C.byref(st)))
        return _stats_dict(st)

    # Batching: plain form raster / gather / solve / publish; persistent form
    # publish / gather / solve, plus the waits and the raster it overlaps
    # with the solve.  L-shape stage: the next four.
    PHASES = ("batch_raster", "batch_gather", "batch_solve", "batch_publish", "cost_pass1", "dp", "commit",
              "prefix_tree_pass2", "batch_solver_wait", "batch_worker_wait", "flt_edge_tables", "unused11",
              "net_ms_bucket0", "net_ms_bucket1", "net_ms_bucket2", "net_ms_bucket3",
              "longest_net_ms_bucket0", "longest_net_ms_bucket1", "longest_net_ms_bucket2", "longest_net_ms_bucket3")

    def set_wait_limit(self, seconds: float):
        """Limit of every device-side wait of the persistent kernels."""
        self._check(self._lib.grb_set_wait_limit(self._ctx, float(seconds)))

    def set_profiling(self, on: bool = True):
        self._check(self._lib.grb_set_profiling(self._ctx, int(bool(on))))

    def phase_times(self, reset: bool = True) -> dict:
        out = np.zeros(len(self.PHASES), np.float64)
        self._check(self._lib.grb_phase_times(self._ctx, _p(out), len(out), int(reset)))
        return dict(zip(self.PHASES, out.tolist()))

    def sync(self):
        self._check(self._lib.grb_sync(self._ctx))


def _stats_dict(st: _abi.GrbStats) -> dict:
    return {"wirelength": st.total_wirelength, "vias": int(st.total_via_count), "n_batches": st.n_batches,
            "stamp": st.stamp, "batching_ms": st.batching_ms, "dag_ms": st.dag_ms}


def plan_from_batches(order, batch_of, n_batches):
    """Reverse and flatten a first-fit result into execution order
    (lshape.cuh:70-77): batch n_batches-1 runs first, nets keep order."""
    order = np.asarray(order)
    batch_of = np.asarray(batch_of)
    ids, off = [], [0]
    for c in range(n_batches - 1, -1, -1):
        sel = order[batch_of == c]
        ids.append(sel)
        off.append(off[-1] + len(sel))
    return (np.concatenate(ids).astype(np.int32) if ids else np.zeros(0, np.int32)), np.asarray(off, np.int32)
