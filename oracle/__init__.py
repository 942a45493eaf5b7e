"""CPU restatement of GRotor's routing hot path -- TEST INFRASTRUCTURE ONLY.

This package is the checker for the CUDA path in ``grotor_b200``.  Only
``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import it; the product never does and has no CPU fallback.
The C++ sources (grb_oracle.cpp) cite the reference file:line they restate.
"""
from .oracle import *  # noqa: F401,F403
