"""ctypes front end of the CPU oracle (oracle/acoustic_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
as the checker, and by bench.py's cpu_baseline / reference legs as the timed
CPU restatement.  The product package never imports it.

The oracle restates ``geobrain/physics/wave/kernels/acoustic_2d.py``
(``acoustic_forward_kernel`` :294-501 with ``acoustic_step_forward``
:123-291) in plain C, in float64 or float32, for stencil half-width 2 (the
reference's 4th-order scheme) or 4 (8th order), plus the exact discrete
adjoint used as the gradient oracle.  Positions are the unpadded grid indices
the reference takes (it adds ``nabc`` itself, :380-384).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


class OrcDesc(ctypes.Structure):
    _fields_ = [
        ("nz", ctypes.c_int32), ("nx", ctypes.c_int32), ("nabc", ctypes.c_int32), ("nt", ctypes.c_int32),
        ("n_shots", ctypes.c_int32), ("n_rcv", ctypes.c_int32), ("half", ctypes.c_int32),
        ("free_surface", ctypes.c_int32), ("dt", ctypes.c_double), ("dz", ctypes.c_double),
    ]


def build() -> str:
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
    return _lib


def max_threads() -> int:
    return int(lib().orc_max_threads())


def set_threads(n: int) -> None:
    """OpenMP threads of the following oracle calls (n < 1: the default)."""
    lib().orc_set_threads(ctypes.c_int(int(n)))


def fd_coefficients(half: int) -> np.ndarray:
    """Staggered Taylor coefficients of half-width ``half`` (elastic_2d.py:25-68)."""
    out = np.zeros(8, dtype=np.float64)
    rc = lib().orc_fd_coefficients(ctypes.c_int(half), out.ctypes.data_as(ctypes.c_void_p))
    if rc != 0:
        raise ValueError(f"unsupported half-width {half}")
    return out[:half].copy()


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def _prep(arrs, dtype):
    return [np.ascontiguousarray(a, dtype=dtype) for a in arrs]


def _desc(nz, nx, nabc, nt, n_shots, n_rcv, half, free_surface, dt, dz):
    return OrcDesc(int(nz), int(nx), int(nabc), int(nt), int(n_shots), int(n_rcv), int(half),
                   int(bool(free_surface)), float(dt), float(dz))


def forward(*, nz, nx, dz, nt, dt, nabc, free_surface, src_x, src_z, src_v, rcv_x, rcv_z,
            damp, vp, rho, half=2, snapshot_every=0, dtype=np.float64):
    """Forward modelling; returns the dict acoustic_forward_kernel returns
    (numpy arrays): p/vx/vz traces (n_shots, nt, n_rcv), forward_wavefield_*
    (nz, nx) and, with snapshot_every > 0, snapshots."""
    dtype = np.dtype(dtype)
    sfx = "f64" if dtype == np.float64 else "f32"
    vp, rho, damp = _prep((vp, rho, damp), dtype)
    src_v = np.ascontiguousarray(np.broadcast_to(np.asarray(src_v, dtype=dtype),
                                                 (len(np.atleast_1d(src_x)), nt)))
    sx, sz, rx, rz = [np.ascontiguousarray(np.atleast_1d(a), dtype=np.int64)
                      for a in (src_x, src_z, rcv_x, rcv_z)]
    S, NR = sx.size, rx.size
    d = _desc(nz, nx, nabc, nt, S, NR, half, free_surface, dt, dz)
    tr = [np.zeros((S, nt, NR), dtype=dtype) for _ in range(3)]
    en = [np.zeros((nz, nx), dtype=dtype) for _ in range(3)]
    nsnap = (nt + snapshot_every - 1) // snapshot_every if snapshot_every > 0 else 0
    snaps = np.zeros((max(nsnap, 1), nz, nx), dtype=dtype)
    fn = getattr(lib(), f"orc_forward_{sfx}")
    rc = fn(ctypes.byref(d), _ptr(vp), _ptr(rho), _ptr(damp), _ptr(sx), _ptr(sz), _ptr(src_v),
            _ptr(rx), _ptr(rz), *[_ptr(t) for t in tr], *[_ptr(e) for e in en],
            ctypes.c_int(int(snapshot_every)), _ptr(snaps))
    if rc != 0:
        raise ValueError(f"oracle forward failed with code {rc}")
    out = {"p": tr[0], "vx": tr[1], "vz": tr[2], "forward_wavefield_p": en[0],
           "forward_wavefield_vx": en[1], "forward_wavefield_vz": en[2]}
    if snapshot_every > 0:
        out["snapshots"] = snaps[:nsnap]
    return out


def gradient(*, nz, nx, dz, nt, dt, nabc, free_surface, src_x, src_z, src_v, rcv_x, rcv_z,
             damp, vp, rho, res_p, res_vx=None, res_vz=None, half=2, dtype=np.float64):
    """dL/dvp, dL/drho (nz, nx) and dL/dwavelet (n_shots, nt) for adjoint
    sources res_* = dL/d(trace) of shape (n_shots, nt, n_rcv)."""
    dtype = np.dtype(dtype)
    sfx = "f64" if dtype == np.float64 else "f32"
    vp, rho, damp = _prep((vp, rho, damp), dtype)
    sx, sz, rx, rz = [np.ascontiguousarray(np.atleast_1d(a), dtype=np.int64)
                      for a in (src_x, src_z, rcv_x, rcv_z)]
    S, NR = sx.size, rx.size
    src_v = np.ascontiguousarray(np.broadcast_to(np.asarray(src_v, dtype=dtype), (S, nt)))
    zeros = np.zeros((S, nt, NR), dtype=dtype)
    res = [np.ascontiguousarray(r, dtype=dtype) if r is not None else zeros
           for r in (res_p, res_vx, res_vz)]
    d = _desc(nz, nx, nabc, nt, S, NR, half, free_surface, dt, dz)
    g_vp = np.zeros((nz, nx), dtype=dtype)
    g_rho = np.zeros((nz, nx), dtype=dtype)
    g_w = np.zeros((S, nt), dtype=dtype)
    fn = getattr(lib(), f"orc_gradient_{sfx}")
    rc = fn(ctypes.byref(d), _ptr(vp), _ptr(rho), _ptr(damp), _ptr(sx), _ptr(sz), _ptr(src_v),
            _ptr(rx), _ptr(rz), *[_ptr(r) for r in res], _ptr(g_vp), _ptr(g_rho), _ptr(g_w))
    if rc != 0:
        raise ValueError(f"oracle gradient failed with code {rc}")
    return g_vp, g_rho, g_w


def rel_l2(a, b) -> float:
    """||a - b|| / ||b|| in float64."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (nb if nb > 0 else 1.0))
