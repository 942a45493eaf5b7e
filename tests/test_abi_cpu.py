"""The C-ABI library loads and exports every entry point its headers declare
(no GPU needed); argument errors come back as codes, not crashes."""
import ctypes as C
import os
import re

import numpy as np

from helpers import ROOT


def _declared(headers):
    names = set()
    for h in headers:
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(grb_[a-z_0-9]+)\s*\(", text))
    return names


def test_every_declared_symbol_is_exported():
    """grb.h and grb_prof.h are the routing library's ABI (libgrb.so),
    grb_synth.h the workload generator's (libgrb_synth.so)."""
    from grotor_b200 import _abi
    headers = sorted(os.listdir(os.path.join(ROOT, "include")))
    assert headers == ["grb.h", "grb_prof.h", "grb_synth.h"]
    lib = _abi.load()
    declared = _declared(["grb.h", "grb_prof.h"])
    assert len(declared) > 20
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python mirror binds every one of them
    assert declared <= set(_abi.SIGNATURES), sorted(declared - set(_abi.SIGNATURES))
    synth = _abi.load_synth()
    declared_synth = _declared(["grb_synth.h"])
    assert len(declared_synth) >= 10
    missing = [n for n in sorted(declared_synth) if not hasattr(synth, n)]
    assert not missing, missing
    assert declared_synth <= set(_abi.SYNTH_SIGNATURES)
    # the generator is not part of the routing library
    assert not any(hasattr(lib, n) for n in declared_synth)


def test_invalid_arguments_return_codes():
    from grotor_b200 import _abi
    lib = _abi.load()
    ctx = C.c_void_p()
    assert lib.grb_create(None, 0, C.byref(ctx)) == _abi.GRB_EINVAL
    g = _abi.GrbGrid(0, 4, 4, 0, 1.0, 1.0, 1.0, None, None, None, None)
    assert lib.grb_create(C.byref(g), 0, C.byref(ctx)) == _abi.GRB_EINVAL
    assert lib.grb_reset(None) == _abi.GRB_EINVAL
    assert lib.grb_lshape_stage(None, 2, None) == _abi.GRB_EINVAL
    assert lib.grb_last_error(None) == b"null context"


def test_create_without_device_reports_cuda_error():
    """On a machine without a GPU the library reports GRB_ECUDA instead of
    falling back to the CPU."""
    import torch
    from grotor_b200 import _abi
    from grotor_b200.router import GridArrays
    lib = _abi.load()
    grid = GridArrays(2, 4, 4, 0, 1.0, 1.0, np.ones(2), np.ones(3, np.int32), np.ones(3, np.int32),
                      np.ones((2, 4, 4), np.float32))
    s = grid.struct()
    ctx = C.c_void_p()
    rc = lib.grb_create(C.byref(s), 0, C.byref(ctx))
    if torch.cuda.is_available():
        assert rc == 0
        lib.grb_destroy(ctx)
    else:
        assert rc == _abi.GRB_ECUDA
