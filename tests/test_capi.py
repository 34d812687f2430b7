"""The C-ABI library loads and exports every symbol include/geobrain_b200.h
declares; host-side plan validation runs without a GPU (no compute calls)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "geobrain_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gb_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from geobrain_b200 import build, _lib
    build.build()
    return _lib.load()


def test_every_declared_symbol_is_exported(lib):
    from geobrain_b200 import _lib
    names = declared_functions()
    assert len(names) >= 10
    for n in names:
        assert hasattr(lib, n), n
        assert n in _lib.SIGNATURES, f"{n} missing from the ctypes bindings"


def _plan(lib, **over):
    from geobrain_b200 import _lib
    d = dict(nz=40, nx=60, nabc=8, nt=50, n_shots=2, n_rcv=3, half=4, free_surface=0, dt=1e-3, dx=10.0)
    d.update(over)
    desc = _lib.ModelDesc(**d)
    sx = np.array([5, 30], np.int64)
    sz = np.array([1, 1], np.int64)
    rx = np.array([0, 10, 59], np.int64)
    rz = np.array([1, 1, 39], np.int64)
    h = ctypes.c_void_p()
    rc = lib.gb_plan_create(ctypes.byref(desc), sx.ctypes.data, sz.ctypes.data, rx.ctypes.data, rz.ctypes.data,
                            ctypes.byref(h))
    return rc, h


def test_plan_create_and_sizes(lib):
    rc, h = _plan(lib)
    assert rc == 0, lib.gb_last_error()
    fwd = lib.gb_plan_workspace_bytes(h, 0, 0)      # with the resident forward's exchange strips
    grad = lib.gb_plan_workspace_bytes(h, 1, 10)
    grad_rho = lib.gb_plan_workspace_bytes(h, 2, 10)
    assert lib.gb_plan_set_resident(h, 0, 0) == 0
    fwd_tile = lib.gb_plan_workspace_bytes(h, 0, 0)
    assert lib.gb_plan_set_resident(h, -1, 0) == 0
    assert 0 < fwd_tile < fwd and fwd_tile < grad < grad_rho
    ck32 = lib.gb_plan_checkpoint_bytes(h, 10, 0)
    ck16 = lib.gb_plan_checkpoint_bytes(h, 10, 1)
    assert ck16 < ck32 and ck32 == 5 * 2 * 3 * (40 + 16) * 96 * 4
    assert lib.gb_plan_set_tiling(h, 16, 1) == 0
    assert lib.gb_plan_set_tiling(h, 24, 0) != 0
    lib.gb_plan_destroy(h)
    assert lib.gb_version().startswith(b"geobrain_b200")


@pytest.mark.parametrize("bad", [dict(half=3), dict(nabc=2), dict(nt=0), dict(dt=0.0), dict(n_shots=0)])
def test_plan_rejects_bad_geometry(lib, bad):
    rc, h = _plan(lib, **bad)
    assert rc == -1 and not h.value
    assert lib.gb_last_error()


def test_plan_rejects_positions_outside_grid(lib):
    from geobrain_b200 import _lib
    desc = _lib.ModelDesc(nz=40, nx=60, nabc=8, nt=50, n_shots=1, n_rcv=1, half=2, free_surface=0, dt=1e-3,
                          dx=10.0)
    good = np.array([0], np.int64)
    for rx in (60 + 8 - 1, -9):      # vx has Nx - 1 columns; -9 is left of the padding
        h = ctypes.c_void_p()
        bad = np.array([rx], np.int64)
        rc = lib.gb_plan_create(ctypes.byref(desc), good.ctypes.data, good.ctypes.data, bad.ctypes.data,
                                good.ctypes.data, ctypes.byref(h))
        assert rc == -1 and b"receiver" in lib.gb_last_error()


def test_product_path_fails_loudly_without_gpu():
    """No CPU fallback: on a machine without CUDA the kernel entry raises."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("CUDA present")
    from geobrain_b200.wave import acoustic_forward_kernel
    z = torch.zeros(4, 4)
    with pytest.raises((ValueError, RuntimeError)):
        acoustic_forward_kernel(nx=4, nz=4, dx=1.0, dz=1.0, nt=2, dt=1e-3, nabc=2, free_surface=False,
                                src_x=[1], src_z=[1], src_n=1, src_v=torch.zeros(2), rcv_x=[1], rcv_z=[1], rcv_n=1,
                                damp=torch.zeros(8, 8), vp=z, rho=z, device="cuda")
