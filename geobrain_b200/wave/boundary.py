"""Absorbing-boundary damping profile (host side, computed once per propagator).

bc_pml follows geobrain/physics/wave/boundary/pml.py:16-98: a quadratic
profile d(k) = kappa (k dx / a)^2, a = (pml - 1) dx, kappa = -3 vmax ln(R) /
(2 a) with R = 1e-6, on the left/right strips of every row and the
top/bottom strips; in the corners the larger of the two distances wins (the
reference writes the top/bottom strips over a range that shrinks by one
column per layer, which amounts to the same thing).  Only 'pml' is on the
acoustic path: the acoustic step treats damp as a rate (kappa = damp * dt),
so the multiplicative tapers ('gerjan', 'sincos') and the split / 3-D
profiles of the reference are not provided.
"""
from __future__ import annotations

import math

import numpy as np

REFLECTION = 1e-6


def _profile(pml: int, dx: float, vmax: float) -> np.ndarray:
    a = (pml - 1) * dx
    kappa = -3.0 * vmax * math.log(REFLECTION) / (2.0 * a)   # ZeroDivisionError for pml == 1, as the reference
    xa = np.arange(pml, dtype=np.float64) * dx / a
    return kappa * xa * xa


def bc_pml(nx: int, nz: int, dx: float, dz: float, pml: int, vmax: float, free_surface: bool = True) -> np.ndarray:
    """Damping array of shape (nz + 2 pml, nx + 2 pml), or (nz + pml, nx + 2 pml)
    with free_surface (no top layer)."""
    prof = _profile(pml, dx, vmax)
    nxp = nx + 2 * pml
    nzp = nz + (pml if free_surface else 2 * pml)
    # distance (in layers) into the left/right and top/bottom absorbing strips; -1 = interior
    dist_x = np.full(nxp, -1, dtype=np.int64)
    dist_x[:pml] = np.arange(pml - 1, -1, -1)
    dist_x[nxp - pml:] = np.arange(pml)
    dist_z = np.full(nzp, -1, dtype=np.int64)
    if not free_surface:
        dist_z[:pml] = np.arange(pml - 1, -1, -1)
    dist_z[nzp - pml:] = np.arange(pml)
    dist = np.maximum(dist_z[:, None], dist_x[None, :])
    out = np.zeros((nzp, nxp), dtype=np.float64)
    mask = dist >= 0
    out[mask] = prof[dist[mask]]
    return out


def bc_pml_3d(nx: int, ny: int, nz: int, dx: float, dy: float, dz: float, pml: int, vmax: float,
              free_surface: bool = True) -> np.ndarray:
    """3-D quadratic damping (geobrain/physics/wave/boundary/pml.py:101-196):
    the 1-D profile kappa (i dx / a)^2, kappa = -3 vmax ln(1e-6) / (2 a),
    a = (pml - 1) dx, laid on all six faces (the top one only without a free
    surface), the maximum where faces meet.  With a free surface the grid has
    only the bottom PML in z, as in the reference."""
    nxp, nyp = nx + 2 * pml, ny + 2 * pml
    nzp = nz + pml if free_surface else nz + 2 * pml
    a = (pml - 1) * dx
    kappa = -3.0 * vmax * np.log(1e-6) / (2.0 * a)
    prof = np.array([kappa * (i * dx / a) * (i * dx / a) for i in range(pml)], dtype=np.float64)

    def dist(n, lo):
        d = np.full(n, -1, dtype=np.int64)
        if lo:
            d[:pml] = np.arange(pml - 1, -1, -1)
        d[n - pml:] = np.arange(pml)
        return d
    dz_, dy_, dx_ = dist(nzp, not free_surface), dist(nyp, True), dist(nxp, True)
    out = np.zeros((nzp, nyp, nxp), dtype=np.float64)
    for d, shape in ((dx_, (1, 1, nxp)), (dy_, (1, nyp, 1)), (dz_, (nzp, 1, 1))):
        vals = np.where(d >= 0, prof[np.maximum(d, 0)], 0.0).reshape(shape)
        out = np.maximum(out, vals)
    return out


def create_boundary(bc_type: str, nx: int, nz: int, dx: float, dz: float, n_layers: int, vmax: float = None,
                    alpha: float = 0.0053, free_surface: bool = False, ny: int = None, dy: float = None):
    """Factory with the signature of geobrain/physics/wave/boundary/__init__.py:23-116."""
    bc_type = bc_type.lower()
    if ny is not None:
        if bc_type != "pml":
            raise NotImplementedError(f"3-D boundary type '{bc_type}' is not yet supported. "
                                      f"Only 'pml' is available for 3-D.")
        if vmax is None:
            raise ValueError("vmax is required for PML boundary")
        if dy is None:
            raise ValueError("dy is required for 3-D PML boundary")
        return bc_pml_3d(nx, ny, nz, dx, dy, dz, n_layers, vmax, free_surface)
    if bc_type == "pml":
        if vmax is None:
            raise ValueError("vmax is required for PML boundary")
        return bc_pml(nx, nz, dx, dz, n_layers, vmax, free_surface)
    if bc_type in ("pml_xz", "gerjan", "sincos"):
        raise NotImplementedError(f"boundary type '{bc_type}' is not used by the acoustic propagator")
    raise ValueError(f"Unknown boundary type: '{bc_type}'. Choose from: 'pml', 'pml_xz', 'gerjan', 'sincos'")
