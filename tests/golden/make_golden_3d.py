"""Generate the 3-D golden fixtures under tests/golden/ by running the
GeoBrain reference itself (acoustic_forward_kernel_3d, its PyTorch CPU path)
on seeded synthetic inputs.

    python tests/golden/make_golden_3d.py /path/to/GeoBrain

Per case (no free surface, free surface): the inputs, the damping array of
create_boundary('pml', ..., ny=, dy=, free_surface=False) as the propagator
builds it (propagators/acoustic.py:119-148, boundary/pml.py:101-196), and the
traces (p, vx, vy, vz) and energy maps of
geobrain/physics/wave/kernels/acoustic_3d.py:303-476 in float32 and in
float64 (torch.set_default_dtype(float64) + dtype=float64, because
pad_model_3d allocates with the default dtype), and the float64 autograd
gradients dL/dvp, dL/drho (checkpoint_segments=3) of a loss linear in all
four traces, L = sum_k <lin_k, trace_k>.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root: str) -> None:
    sys.path.insert(0, ref_root)
    import torch
    from geobrain.physics.wave import RickerWavelet, create_boundary
    from geobrain.physics.wave.kernels import acoustic_forward_kernel_3d

    nz, ny, nx, nabc, nt, dx, dt = 12, 14, 16, 6, 70, 10.0, 1e-3
    for name, fs, seed in (("small_3d_nofs", False, 3), ("small_3d_fs", True, 4)):
        rng = np.random.default_rng(seed)
        z = np.arange(nz, dtype=np.float64)[:, None, None]
        vp = (1800.0 + 900.0 * z / (nz - 1) + 150.0 * rng.standard_normal((nz, ny, nx))).astype(np.float32)
        rho = (2000.0 + 200.0 * rng.random((nz, ny, nx))).astype(np.float32)
        damp = create_boundary("pml", nx=nx, nz=nz, dx=dx, dz=dx, n_layers=nabc, vmax=float(vp.max()),
                               free_surface=False, ny=ny, dy=dx).astype(np.float32)
        w, _ = RickerWavelet()(f0=25.0, dt=dt)
        w = w.numpy().astype(np.float32)
        w = np.pad(w, (0, max(0, nt - len(w))))[:nt]
        src_x = np.array([4, 11], np.int64)
        src_y = np.array([7, 3], np.int64)
        src_z = np.array([1, 2], np.int64) if not fs else np.array([0, 1], np.int64)
        ry, rx = np.meshgrid(np.arange(0, ny, 3), np.arange(0, nx, 2), indexing="ij")
        rcv_x = np.concatenate([rx.ravel(), [-nabc, nx + nabc - 2]]).astype(np.int64)
        rcv_y = np.concatenate([ry.ravel(), [-nabc, ny + nabc - 2]]).astype(np.int64)
        rcv_z = np.concatenate([np.ones(rx.size, np.int64), [-nabc, nz + nabc - 2]]).astype(np.int64)
        src_v = np.tile(w, (2, 1))
        out = dict(nz=nz, ny=ny, nx=nx, nabc=nabc, nt=nt, dx=dx, dt=dt, free_surface=fs, vp=vp, rho=rho,
                   damp=damp, src_x=src_x, src_y=src_y, src_z=src_z, rcv_x=rcv_x, rcv_y=rcv_y, rcv_z=rcv_z,
                   src_v=src_v)
        for tag, dtype in (("ref32", torch.float32), ("ref64", torch.float64)):
            torch.set_default_dtype(dtype)
            with torch.no_grad():
                res = acoustic_forward_kernel_3d(
                    nx=nx, ny=ny, nz=nz, dx=dx, dy=dx, dz=dx, nt=nt, dt=dt, nabc=nabc, free_surface=fs,
                    src_x=torch.tensor(src_x), src_y=torch.tensor(src_y), src_z=torch.tensor(src_z), src_n=2,
                    src_v=torch.tensor(src_v, dtype=dtype), rcv_x=torch.tensor(rcv_x), rcv_y=torch.tensor(rcv_y),
                    rcv_z=torch.tensor(rcv_z), rcv_n=rcv_x.size, damp=torch.tensor(damp, dtype=dtype),
                    vp=torch.tensor(vp, dtype=dtype), rho=torch.tensor(rho, dtype=dtype), dtype=dtype)
            torch.set_default_dtype(torch.float32)
            for k, v in res.items():
                out[f"{tag}_{k}"] = v.numpy()
        rng_l = np.random.default_rng(seed + 100)
        lin = {k: rng_l.standard_normal((2, nt, rcv_x.size)) for k in ("p", "vx", "vy", "vz")}
        torch.set_default_dtype(torch.float64)
        vp_t = torch.tensor(vp, dtype=torch.float64, requires_grad=True)
        rho_t = torch.tensor(rho, dtype=torch.float64, requires_grad=True)
        res = acoustic_forward_kernel_3d(
            nx=nx, ny=ny, nz=nz, dx=dx, dy=dx, dz=dx, nt=nt, dt=dt, nabc=nabc, free_surface=fs,
            src_x=torch.tensor(src_x), src_y=torch.tensor(src_y), src_z=torch.tensor(src_z), src_n=2,
            src_v=torch.tensor(src_v, dtype=torch.float64), rcv_x=torch.tensor(rcv_x), rcv_y=torch.tensor(rcv_y),
            rcv_z=torch.tensor(rcv_z), rcv_n=rcv_x.size, damp=torch.tensor(damp, dtype=torch.float64), vp=vp_t,
            rho=rho_t, checkpoint_segments=3, dtype=torch.float64)
        loss = sum((torch.tensor(lin[k]) * res[k]).sum() for k in lin)
        loss.backward()
        torch.set_default_dtype(torch.float32)
        out["ref64_grad_vp"] = vp_t.grad.numpy()
        out["ref64_grad_rho"] = rho_t.grad.numpy()
        for k, v in lin.items():
            out[f"lin_{k}"] = v
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(name, {k: v.shape for k, v in out.items() if hasattr(v, "shape") and k.startswith("ref32")})


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GEOBRAIN_REF")
    if not root:
        sys.exit("usage: %s <path to the GeoBrain source tree> (or set GEOBRAIN_REF)" % os.path.basename(__file__))
    main(root)
