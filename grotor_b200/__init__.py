"""grotor_b200 -- GRotor's routing hot path, native to NVIDIA B200 (sm_100a).

Exact first-fit net batching, incremental congestion cost with per-track
prefix tables, L-shape pattern routing with layer assignment, and demand
commit / rip-up, as hand-written CUDA behind the C ABI in include/grb.h.
The Python layer here mirrors the reference's host interface over that ABI.
Importing the package loads the native library; there is no CPU fallback.
"""
from ._abi import load as _load_native
from .router import GrbError, GridArrays, NetArrays, Router, plan_from_batches  # noqa: F401

_load_native()

__all__ = ["GrbError", "GridArrays", "NetArrays", "Router", "plan_from_batches"]
