"""ctypes mirror of include/grb.h and include/grb_synth.h.

The shared library ``libgrb.so`` (the routing path) is built in-tree by
``grotor_b200.build``; loading fails loudly when it is missing: the package has
no CPU fallback.  The seeded workload generator of include/grb_synth.h is a
separate host-only library, ``libgrb_synth.so``, so a process that only needs
synthetic designs (the CPU reference arm of bench.py) never loads the routing
library.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgrb.so")
SYNTH_PATH = os.path.join(_HERE, "libgrb_synth.so")

GRB_OK, GRB_EINVAL, GRB_ENOMEM, GRB_ECUDA, GRB_ETIMEDOUT, GRB_ELIMIT = range(6)
MODE_PLAIN, MODE_GRAPH, MODE_PERSISTENT = 0, 1, 2
GRB_TAIL_RIPUP, GRB_TAIL_VIEW = 1, 2
ERROR_NAMES = {1: "GRB_EINVAL", 2: "GRB_ENOMEM", 3: "GRB_ECUDA", 4: "GRB_ETIMEDOUT", 5: "GRB_ELIMIT"}

P = C.c_void_p


class GrbGrid(C.Structure):
    _fields_ = [
        ("L", C.c_int32), ("X", C.c_int32), ("Y", C.c_int32), ("DIR", C.c_int32),
        ("unit_length_wire_cost", C.c_double), ("unit_via_cost", C.c_double), ("of_cost_scale", C.c_double),
        ("unit_length_short_costs", P), ("x_edge_len", P), ("y_edge_len", P), ("capacity", P),
    ]


class GrbNets(C.Structure):
    _fields_ = [
        ("n", C.c_int32), ("node_off", P), ("nodes", P), ("parents", P), ("route_off", P),
        ("point_off", P), ("points", P), ("hseg_off", P), ("hsegs", P), ("vseg_off", P), ("vsegs", P),
    ]


class GrbTrees(C.Structure):
    _fields_ = [("n", C.c_int32), ("node_off", P), ("pos", P), ("adj_off", P), ("adj", P), ("route_off", P)]


class GrbOutRecords(C.Structure):
    _fields_ = [("n", C.c_int32), ("name_off", P), ("names", P), ("pin_off", P), ("pins", P), ("extra_off", P),
                ("extra", P), ("sub_off", P), ("subnets", P), ("sub_phase2", P)]


OUT_SINK = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int64, C.c_void_p)


class GrbStats(C.Structure):
    _fields_ = [
        ("total_wirelength", C.c_double), ("total_via_count", C.c_int64), ("n_batches", C.c_int32),
        ("stamp", C.c_int32), ("batching_ms", C.c_double), ("dag_ms", C.c_double),
    ]


class GrbFltDags(C.Structure):
    _fields_ = [(k, P) for k in ("node_off", "coord", "depth", "children", "parent_end", "edge_off", "edge_parent",
                                 "edge_source_slot", "route2_off")]


class GrbZshapeTrees(C.Structure):
    _fields_ = [(k, P) for k in ("node_off", "coord", "child")]


class GrbSynthParams(C.Structure):
    _fields_ = [
        ("X", C.c_int32), ("Y", C.c_int32), ("cap_layers", C.c_int32), ("n_nets", C.c_int32),
        ("cap_lo", C.c_int32), ("cap_hi", C.c_int32),
        ("blockage", C.c_double), ("unit_wire", C.c_double), ("unit_via", C.c_double), ("overflow_weight", C.c_double),
        ("pin_model", C.c_int32), ("two_pin_frac", C.c_double), ("geo_p", C.c_double), ("max_pins", C.c_int32),
        ("pareto_alpha", C.c_double), ("bbox_model", C.c_int32), ("bbox_median", C.c_double),
        ("bbox_sigma", C.c_double), ("big_frac", C.c_double), ("big_lo", C.c_int32), ("big_hi", C.c_int32),
        ("bbox_max", C.c_int32), ("pin_cap_layers", C.c_int32), ("seed", C.c_uint64),
    ]


# Every exported entry point: name -> (restype, argtypes).
SIGNATURES = {
    "grb_init_device": (C.c_int, [C.c_int32]),
    "grb_create": (C.c_int, [C.POINTER(GrbGrid), C.c_int32, C.POINTER(P)]),
    "grb_destroy": (None, [P]),
    "grb_last_error": (C.c_char_p, [P]),
    "grb_stream": (P, [P]),
    "grb_reset": (C.c_int, [P]),
    "grb_upload_nets": (C.c_int, [P, C.POINTER(GrbNets)]),
    "grb_build_topology": (C.c_int, [P, C.POINTER(GrbTrees)]),
    "grb_topology_sizes": (C.c_int, [P, P]),
    "grb_read_topology": (C.c_int, [P] + [P] * 9),
    "grb_plan_batches": (C.c_int, [P, P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, P, C.POINTER(C.c_int32)]),
    "grb_set_plan": (C.c_int, [P, P, C.c_int32, P, C.c_int32]),
    "grb_get_plan": (C.c_int, [P, P, P, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "grb_refresh_cost": (C.c_int, [P]),
    "grb_route_batch": (C.c_int, [P, C.c_int32, C.c_int32]),
    "grb_commit_batch": (C.c_int, [P, C.c_int32, C.c_int32, C.c_int32]),
    "grb_lshape_stage": (C.c_int, [P, C.c_int32, C.POINTER(GrbStats)]),
    "grb_ripup_classify": (C.c_int, [P, C.c_int32, P]),
    "grb_ripup_classify_noalloc": (C.c_int, [P, C.c_int32, P]),
    "grb_upload_geometry": (C.c_int, [P, P, P, P, P, P, P]),
    "grb_upload_flt": (C.c_int, [P, C.POINTER(GrbFltDags)]),
    "grb_flt_stage": (C.c_int, [P, C.c_int32, C.c_int32, C.POINTER(GrbStats)]),
    "grb_set_flt_block_width": (C.c_int, [P, C.c_int32]),
    "grb_read_routes2": (C.c_int, [P, P]),
    "grb_write_routes2": (C.c_int, [P, P]),
    "grb_remove_routes": (C.c_int, [P, P, C.c_int32, P]),
    "grb_ripup_classify_phase2": (C.c_int, [P, C.c_int32, P, P]),
    "grb_routing_score": (C.c_int, [P, C.POINTER(C.c_double)]),
    "grb_checkpoint": (C.c_int, [P]),
    "grb_restore": (C.c_int, [P]),
    "grb_format_out": (C.c_int, [P, C.POINTER(GrbOutRecords), C.POINTER(C.c_int64)]),
    "grb_drain_out": (C.c_int, [P, OUT_SINK, P]),
    "grb_set_wire_cost_mode": (C.c_int, [P, C.c_int32]),
    "grb_autotune": (C.c_int, [P, C.c_int32, P, P]),
    "grb_softmin_forward": (C.c_int, [P, C.c_int32, C.c_double, P, P, C.c_double, P, C.POINTER(C.c_double)]),
    "grb_softmin_backward": (C.c_int, [P, C.c_int32, C.c_double, P, P, C.c_double, C.c_double, P, P,
                                       C.POINTER(C.c_double)]),
    "grb_upload_zshape": (C.c_int, [P, C.POINTER(GrbZshapeTrees)]),
    "grb_plan_bbox_batches": (C.c_int, [P, P, C.c_int32, C.POINTER(C.c_int32)]),
    "grb_zshape_stage": (C.c_int, [P, C.c_int32, C.POINTER(GrbStats)]),
    "grb_congestion_view": (C.c_int, [P, P, P, P]),
    "grb_cost_exp": (C.c_int, [C.c_int32, P, C.c_int32, P]),
    "grb_set_stage_tail": (C.c_int, [P, C.c_int32, C.c_int32]),
    "grb_read_stage_tail": (C.c_int, [P, P, P, P, P]),
    "grb_read_tables": (C.c_int, [P, P, P, P, P, P]),
    "grb_read_routes": (C.c_int, [P, P]),
    "grb_read_routes_used": (C.c_int, [P, P]),
    "grb_write_routes_used": (C.c_int, [P, P]),
    "grb_write_routes": (C.c_int, [P, P]),
    "grb_get_stats": (C.c_int, [P, C.POINTER(GrbStats)]),
    "grb_set_stats": (C.c_int, [P, C.c_double, C.c_int64]),
    "grb_sync": (C.c_int, [P]),
    "grb_kernel_launches": (C.c_int64, [P]),
    "grb_set_wait_limit": (C.c_int, [P, C.c_double]),
    "grb_set_profiling": (C.c_int, [P, C.c_int32]),
    "grb_phase_times": (C.c_int, [P, P, C.c_int32, C.c_int32]),
    # grb_prof.h
    "grb_stage_traffic": (C.c_int, [P, C.c_int32, P, P, P, P, P, P, P, P, P, P, P, P, C.c_int32, P]),
    "grb_zshape_traffic": (C.c_int, [P, C.c_int32, P, P, P, P, P, P, P, P]),
    "grb_flt_traffic": (C.c_int, [P, C.c_int32, P, P, P, P, P, P, C.c_int32, P]),
    "grb_dag_reads": (C.c_int, [P, C.c_int32, P, P, P, P, P]),
}

# include/grb_synth.h (libgrb_synth.so)
SYNTH_SIGNATURES = {
    "grb_synth_generate": (P, [C.POINTER(GrbSynthParams)]),
    "grb_design_free": (None, [P]),
    "grb_design_error": (C.c_char_p, [P]),
    "grb_design_grid": (C.c_int, [P, C.POINTER(GrbGrid)]),
    "grb_design_write": (C.c_int, [P, C.c_char_p, C.c_char_p]),
    "grb_design_build_topology": (C.c_int, [P, C.c_int32, C.c_int32]),
    "grb_design_nets": (C.c_int, [P, C.POINTER(GrbNets)]),
    "grb_design_zshape_trees": (C.c_int, [P, C.POINTER(P), C.POINTER(P), C.POINTER(P)]),
    "grb_design_subnet_info": (C.c_int, [P, C.POINTER(P), C.POINTER(P), C.POINTER(P)]),
    "grb_design_order": (C.c_int, [P, P]),
    "grb_design_pins": (C.c_int, [P, C.POINTER(P), C.POINTER(P), C.POINTER(C.c_int32)]),
}

_libs = {}


def _open(path: str, signatures: dict) -> C.CDLL:
    if path not in _libs:
        if not os.path.exists(path):
            raise ImportError(f"grotor_b200 native library missing: {path} (run grotor_b200.build.build())")
        lib = C.CDLL(path)
        for name, (res, args) in signatures.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _libs[path] = lib
    return _libs[path]


def load() -> C.CDLL:
    """Load libgrb.so, the routing path (raises if it has not been built)."""
    return _open(LIB_PATH, SIGNATURES)


def load_synth() -> C.CDLL:
    """Load libgrb_synth.so, the workload generator (host code only)."""
    return _open(SYNTH_PATH, SYNTH_SIGNATURES)
