"""The oracle's table of exponential values (the checker's way to reproduce
the device's cost tables bit for bit without restating the device's
exponential).  On the CPU: a table holding the host's own expf values changes
nothing; a table is really used (a planted change in it moves the costs);
arguments outside an installed table are counted; the argument list covers
every exponential the cost model evaluates for the demands it names."""
import ctypes as C

import numpy as np

import oracle
from helpers import orc_grid

LIBM = C.CDLL("libm.so.6")
LIBM.expf.restype = C.c_float
LIBM.expf.argtypes = [C.c_float]


def _design():
    from grotor_b200.synth import WORKLOADS, Design
    return Design(WORKLOADS["small_64x64x5"].scaled(600, seed=5, cap_lo=0, cap_hi=3))


def _demand(g, seed=1):
    return np.random.default_rng(seed).integers(0, 40, g.cells).astype(np.int32)


def test_host_values_change_nothing_and_every_argument_is_listed():
    d = _design()
    og = orc_grid(d.grid)
    dem = _demand(d.grid)
    w0, v0 = oracle.cost_full(og, dem)
    x = oracle.exp_args(og, int(dem.max()))
    assert np.all(np.diff(x) > 0)
    y = np.array([LIBM.expf(float(a)) for a in x], np.float32)
    try:
        oracle.set_exp_table(x, y)
        w1, v1 = oracle.cost_full(og, dem)
        assert oracle.exp_table_misses() == 0
    finally:
        oracle.set_exp_table()
    np.testing.assert_array_equal(w0.view(np.int32), w1.view(np.int32))
    np.testing.assert_array_equal(v0.view(np.int32), v1.view(np.int32))


def test_table_is_used_and_misses_are_counted():
    d = _design()
    og = orc_grid(d.grid)
    dem = _demand(d.grid, 2)
    w0, _ = oracle.cost_full(og, dem)
    x = oracle.exp_args(og, int(dem.max()))
    y = np.array([LIBM.expf(float(a)) for a in x], np.float32) * np.float32(1.001)  # planted on the CPU
    try:
        oracle.set_exp_table(x, y)
        w1, _ = oracle.cost_full(og, dem)
        assert oracle.exp_table_misses() == 0
        assert not np.array_equal(w0, w1)
        oracle.set_exp_table(x[::2], y[::2])  # half the arguments missing
        oracle.cost_full(og, dem)
        assert oracle.exp_table_misses() > 0
    finally:
        oracle.set_exp_table()
    assert oracle.exp_table_misses() == 0
