"""Run a short slice of a benchmark workload, for profilers (ncu).

    python -m geobrain_b200.profile_workload --phase forward  --nt 6
    python -m geobrain_b200.profile_workload --phase gradient --nt 6 [--imaging-dtype fp24]
    python -m geobrain_b200.profile_workload --model 3d --phase forward --nt 6
    python -m geobrain_b200.profile_workload --phase gradient --nt 6 --imaging-dtype fp24 --absorbing cpml

Builds the 400 x 1200 / 32-shot / 8th-order model of the benchmark, runs
``nt`` time steps of the forward (or forward + adjoint) once, synchronises
and exits 0.  Everything stays on the device; nothing is timed.  With
--imaging-dtype the gradient keeps every step's imaging fields in that
format (as the benchmark does); without it, one fp32 checkpoint and a
recompute of all steps.  --model 3d runs the 3-D path instead: a 200^3
model with a 20-cell PML and 4 shots, 4th order (acoustic_forward_kernel_3d;
the gradient is that of 0.5 ||p||^2 with one checkpoint).  --absorbing cpml
uses the CPML layers (its gradient needs --imaging-dtype: the adjoint reads
every step's imaging fields).
"""
from __future__ import annotations

import argparse

import numpy as np
import torch

from . import synthetic, wave
from .wave import engine


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--phase", choices=["forward", "gradient"], default="forward")
    ap.add_argument("--nt", type=int, default=6)
    ap.add_argument("--shots", type=int, default=32)
    ap.add_argument("--tile-rows", type=int, default=0)
    ap.add_argument("--shots-per-cta", type=int, default=0)
    ap.add_argument("--energy", action="store_true")
    ap.add_argument("--imaging-dtype", choices=["fp32", "fp24", "bf16"], default=None)
    ap.add_argument("--model", choices=["2d", "3d"], default="2d")
    ap.add_argument("--absorbing", choices=["damping", "cpml"], default="damping")
    args = ap.parse_args()
    dev = torch.device("cuda:0")
    if args.model == "3d":
        run_3d(args, dev)
        torch.cuda.synchronize()
        print("profile_workload: ok")
        return
    w = synthetic.fwi_400x1200(nt=args.nt, n_shots=args.shots)
    damp = torch.tensor(wave.bc_pml(w.nx, w.nz, w.dx, w.dx, w.nabc, float(w.vp.max()), False), dtype=torch.float32,
                        device=dev)
    geo = engine.Geometry(w.nz, w.nx, w.nabc, w.nt, float(w.dt), float(w.dx), w.fd_order // 2, False)
    plan = engine.get_plan(geo, w.src_x, w.src_z, w.rcv_x, w.rcv_z)
    plan.set_absorbing(args.absorbing, float(w.vp.max()) if args.absorbing == "cpml" else 0.0)
    if args.tile_rows or args.shots_per_cta:
        plan.set_tiling(args.tile_rows, args.shots_per_cta)
    vp = torch.tensor(w.vp, device=dev)
    rho = torch.tensor(w.rho, device=dev)
    src_v = torch.tensor(np.tile(w.wavelet, (w.n_shots, 1)), device=dev)
    if args.phase == "forward":
        engine.run_forward(plan, vp, rho, damp, src_v, want_energy=args.energy)
    else:
        K = w.nt
        if args.imaging_dtype:
            img = torch.empty(plan.imaging_bytes(w.nt, False, args.imaging_dtype), dtype=torch.uint8, device=dev)
            store = engine.make_store(None, K, "fp32", img, w.nt, False, args.imaging_dtype)
        else:
            ck = torch.empty(plan.checkpoint_bytes(K, "fp32"), dtype=torch.uint8, device=dev)
            store = engine.make_store(ck, K, "fp32", None, 0, False)
        p, _, _, _, _ = engine.run_forward(plan, vp, rho, damp, src_v, want_energy=args.energy, store=store)
        engine.run_backward(plan, vp, rho, damp, src_v, p, None, None, store, False)
    torch.cuda.synchronize()
    print("profile_workload: ok")


def run_3d(args, dev, nz=200, ny=200, nx=200, shots=4, nabc=20) -> None:
    rng = np.random.default_rng(0)
    nt = args.nt
    vp = torch.tensor((2000 + 1000 * rng.random((nz, ny, nx))).astype(np.float32), device=dev)
    rho = torch.full((nz, ny, nx), 2000.0, device=dev)
    damp = torch.tensor(wave.bc_pml_3d(nx, ny, nz, 10.0, 10.0, 10.0, nabc, 3000.0, free_surface=False)
                        .astype(np.float32), device=dev)
    w, _ = wave.RickerWavelet()(f0=15.0, dt=1e-3)
    w = torch.tensor(np.pad(w.numpy(), (0, nt))[:nt], device=dev)
    kw = dict(nx=nx, ny=ny, nz=nz, dx=10.0, dy=10.0, dz=10.0, nt=nt, dt=1e-3, nabc=nabc, free_surface=False,
              src_x=np.linspace(10, nx - 10, shots).astype(np.int64), src_y=np.full(shots, ny // 2),
              src_z=np.ones(shots, np.int64), src_n=shots, src_v=w, rcv_x=np.arange(0, nx, 2),
              rcv_y=np.full(nx // 2, ny // 2), rcv_z=np.ones(nx // 2, np.int64), rcv_n=nx // 2, damp=damp,
              rho=rho, device=dev)
    if args.phase == "forward":
        with torch.no_grad():
            wave.acoustic_forward_kernel_3d(vp=vp, **kw)
    else:
        v = vp.detach().requires_grad_(True)
        out = wave.acoustic_forward_kernel_3d(vp=v, **kw)
        (0.5 * (out["p"] * out["p"]).sum()).backward()


if __name__ == "__main__":
    main()
