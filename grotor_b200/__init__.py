"""grotor_b200 -- GRotor's routing hot path, native to NVIDIA B200 (sm_100a).

Exact first-fit net batching, incremental congestion cost with per-track
prefix tables, L-shape pattern routing with layer assignment, and demand
commit / rip-up, as hand-written CUDA behind the C ABI in include/grb.h.
The Python layer here mirrors the reference's host interface over that ABI.
Creating a ``Router`` loads the native library and fails loudly when it is
missing; there is no CPU fallback.  (The package import itself loads nothing,
so the seeded workload generator, ``grotor_b200.synth``, can be used by a
process that must not load the routing library.)
"""
from .router import GrbError, GridArrays, NetArrays, Router, TreeArrays, plan_from_batches  # noqa: F401

__all__ = ["GrbError", "GridArrays", "NetArrays", "Router", "TreeArrays", "plan_from_batches"]
