"""Generate tests/golden/propagator_gardner.npz by running the GeoBrain
reference's own model / survey / propagator API on its PyTorch CPU path.

    python tests/golden/make_golden_propagator.py /path/to/GeoBrain
    (or GEOBRAIN_REF=/path/to/GeoBrain python tests/golden/make_golden_propagator.py)

What is recorded (two cases, without and with a free surface):
  * AcousticModel(auto_update_rho=True, vp_grad=True)
    (geobrain/physics/wave/models/acoustic.py:164-195): forward() replaces
    rho by Gardner's 310 vp^0.25 before every propagation and keeps it out
    of autograd;
  * AcousticPropagator(model, survey, dtype).forward()
    (propagators/acoustic.py:150-275) in float32, all shots: the traces and
    energy maps;
  * forward(shot_index=1, checkpoint_segments=3) in float64
    (torch.set_default_dtype(float64) as well, since pad_model allocates with
    the default dtype, kernels/acoustic_2d.py:49), then loss.backward() of a
    loss linear in the three traces: model.vp.grad, and the Gardner density
    the model held.
The inputs (vp, survey positions, wavelet, linear weights) are stored with
the outputs, so nothing is regenerated at test time.
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root: str) -> None:
    sys.path.insert(0, ref_root)
    import torch
    from geobrain.physics.wave import (AcousticModel, AcousticPropagator, BoundaryConfig, GridConfig, Receiver,
                                       RickerWavelet, Source, Survey)

    torch.set_num_threads(os.cpu_count() or 1)
    nz, nx, nabc, nt, dt, dx, f0 = 40, 72, 12, 360, 1e-3, 10.0, 18.0
    src_x, src_z = np.array([12, 36, 60]), np.array([2, 3, 2])
    rcv_x = np.arange(0, nx, 2)
    rcv_z = np.full(rcv_x.size, 2)

    for name, free_surface, seed in (("propagator_gardner", False, 11), ("propagator_gardner_fs", True, 12)):
        rng = np.random.default_rng(seed)
        z = np.arange(nz, dtype=np.float64)[:, None]
        vp = 1800.0 + 1400.0 * z / (nz - 1) + 150.0 * rng.standard_normal((nz, nx)).clip(-2, 2)
        vp = vp.astype(np.float32)
        rho0 = np.full((nz, nx), 2000.0, np.float32)
        w, _ = RickerWavelet()(f0=f0, dt=dt)
        w = w.numpy().astype(np.float32)
        w = np.pad(w, (0, nt - len(w))) if len(w) < nt else w[:nt]
        lin = {k: rng.standard_normal((1, nt, rcv_x.size)) for k in ("p", "vx", "vz")}

        def build(dtype):
            grid = GridConfig(nx=nx, nz=nz, dx=dx, dz=dx)
            bnd = BoundaryConfig(type="pml", n_layers=nabc, free_surface=free_surface)
            model = AcousticModel(grid=grid, boundary=bnd, vp=vp.astype(np.float64) if dtype == torch.float64 else vp,
                                  rho=rho0, vp_grad=True, auto_update_rho=True, dtype=dtype)
            src = Source(nt=nt, dt=dt, f0=f0)
            for x, zz in zip(src_x, src_z):
                src.add_source(x=int(x), z=int(zz), wavelet=w)
            rcv = Receiver(nt=nt, dt=dt)
            rcv.add_receivers(x=rcv_x, z=rcv_z, rcv_type="pr")
            return model, AcousticPropagator(model, Survey(src, rcv), device="cpu", dtype=dtype)

        t0 = time.time()
        model32, prop32 = build(torch.float32)
        with torch.no_grad():
            r32 = prop32.forward()
        prev = torch.get_default_dtype()
        torch.set_default_dtype(torch.float64)
        try:
            model64, prop64 = build(torch.float64)
            r64 = prop64.forward(shot_index=1, checkpoint_segments=3)
            loss = sum((torch.tensor(lin[k]) * getattr(r64, k)).sum() for k in ("p", "vx", "vz"))
            loss.backward()
            grad_vp = model64.vp.grad.detach().numpy().copy()
            rho_gardner = model64.rho.detach().numpy().copy()
            r64p = r64.p.detach().numpy().copy()
        finally:
            torch.set_default_dtype(prev)
        np.savez_compressed(
            os.path.join(HERE, f"{name}.npz"),
            nz=nz, nx=nx, nabc=nabc, nt=nt, dt=dt, dx=dx, f0=f0, free_surface=free_surface,
            vp=vp, rho0=rho0, wavelet=w, src_x=src_x, src_z=src_z, rcv_x=rcv_x, rcv_z=rcv_z,
            damp=prop32.damp.numpy(), shot_index=1, checkpoint_segments=3,
            lin_p=lin["p"], lin_vx=lin["vx"], lin_vz=lin["vz"],
            ref32_p=r32.p.numpy(), ref32_vx=r32.vx.numpy(), ref32_vz=r32.vz.numpy(),
            ref32_forward_wavefield_p=r32.forward_wavefield_p.numpy(),
            ref32_forward_wavefield_vx=r32.forward_wavefield_vx.numpy(),
            ref32_forward_wavefield_vz=r32.forward_wavefield_vz.numpy(),
            ref32_rho_gardner=model32.rho.detach().numpy(),
            ref64_shot1_p=r64p, ref64_grad_vp=grad_vp, ref64_rho_gardner=rho_gardner)
        print(f"{name}: {time.time() - t0:.1f}s")


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GEOBRAIN_REF")
    if not root:
        sys.exit("usage: make_golden_propagator.py <path to the GeoBrain source tree> (or set GEOBRAIN_REF)")
    main(root)
