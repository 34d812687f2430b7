"""The resident forward's tiling and exchange choice through the C ABI, on
the host (plan creation and gb_plan_set/get_resident make no compute call;
without a device the SM count is taken as the B200's 148)."""
import ctypes

import numpy as np
import pytest

from test_capi import lib  # noqa: F401  (module fixture: the built library)


def _plan(lib, nz, nx, nabc, half, n_shots, free_surface=0):
    from geobrain_b200 import _lib
    d = _lib.ModelDesc(nz=nz, nx=nx, nabc=nabc, nt=10, n_shots=n_shots, n_rcv=nx, half=half,
                       free_surface=free_surface, dt=1e-3, dx=10.0)
    # unpadded indices, as the reference's survey gives them
    sx = np.linspace(0, nx - 1, n_shots).astype(np.int64)
    sz = np.ones(n_shots, np.int64)
    rx = np.arange(nx, dtype=np.int64)
    rz = np.ones(nx, np.int64)
    h = ctypes.c_void_p()
    assert lib.gb_plan_create(ctypes.byref(d), sx.ctypes.data, sz.ctypes.data, rx.ctypes.data, rz.ctypes.data,
                              ctypes.byref(h)) == 0, lib.gb_last_error()
    return h


def _resident(lib, h):
    tz, spl, ex = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    assert lib.gb_plan_get_resident(h, ctypes.byref(tz), ctypes.byref(spl), ctypes.byref(ex)) == 0
    return tz.value, spl.value, ex.value


@pytest.mark.parametrize("nz,nx,nabc,half,shots,want", [
    (100, 200, 20, 2, 1, (4, 1, 0)),        # the 100 x 200 workload: 70 tiles of 4 rows
    (400, 1200, 30, 4, 1, (36, 1, 0)),      # one shot of the 400 x 1200 grid: 143 tiles of 36 rows
    (400, 1200, 30, 4, 32, (0, 0, 0)),      # 32 shots: the tile kernel
    (40, 60, 8, 2, 4, (4, 4, 0)),           # small grid, a few shots in one launch
])
def test_automatic_choice(lib, nz, nx, nabc, half, shots, want):
    h = _plan(lib, nz, nx, nabc, half, shots)
    try:
        assert _resident(lib, h) == want
    finally:
        lib.gb_plan_destroy(h)


def test_modes_and_refusals(lib):
    from geobrain_b200 import _lib
    h = _plan(lib, 100, 200, 20, 2, 1)
    h8 = _plan(lib, 100, 200, 20, 4, 1)
    hfs = _plan(lib, 100, 200, 20, 2, 1, free_surface=1)
    try:
        assert lib.gb_plan_set_resident(h, 3, 0) == 0                      # one exchange a step
        assert _resident(lib, h) == (4, 1, 2)
        assert lib.gb_plan_set_resident(h, 2, 0) == 0                      # cluster: at most 16 tiles
        tz, _, ex = _resident(lib, h)
        assert ex == 1 and ((140 + tz - 1) // tz) * 2 <= 16
        assert lib.gb_plan_set_resident(h, 1, 12) == 0
        assert _resident(lib, h)[0] == 12
        assert lib.gb_plan_set_resident(h, 0, 0) == 0
        assert _resident(lib, h) == (0, 0, 0)
        for mode, rows in ((4, 0), (-2, 0), (1, 10), (1, 48)):
            assert lib.gb_plan_set_resident(h, mode, rows) == _lib.GB_E_ARG
        # one exchange a step needs the 4th order without a free surface
        for p in (h8, hfs):
            assert lib.gb_plan_set_resident(p, 3, 0) == _lib.GB_E_UNSUPPORTED
            assert _resident(lib, p)[2] == 0                               # still automatic
    finally:
        for p in (h, h8, hfs):
            lib.gb_plan_destroy(p)
