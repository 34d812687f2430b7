"""Run a short slice of a benchmark workload, for profilers (ncu).

    python -m geobrain_b200.profile_workload --phase forward  --nt 6
    python -m geobrain_b200.profile_workload --phase gradient --nt 6 [--imaging-dtype fp24]

Builds the 400 x 1200 / 32-shot / 8th-order model of the benchmark, runs
``nt`` time steps of the forward (or forward + adjoint) once, synchronises
and exits 0.  Everything stays on the device; nothing is timed.  With
--imaging-dtype the gradient keeps every step's imaging fields in that
format (as the benchmark does); without it, one fp32 checkpoint and a
recompute of all steps.
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
    args = ap.parse_args()
    dev = torch.device("cuda:0")
    w = synthetic.fwi_400x1200(nt=args.nt, n_shots=args.shots)
    damp = torch.tensor(wave.bc_pml(w.nx, w.nz, w.dx, w.dx, w.nabc, float(w.vp.max()), False), dtype=torch.float32,
                        device=dev)
    geo = engine.Geometry(w.nz, w.nx, w.nabc, w.nt, float(w.dt), float(w.dx), w.fd_order // 2, False)
    plan = engine.get_plan(geo, w.src_x, w.src_z, w.rcv_x, w.rcv_z)
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


if __name__ == "__main__":
    main()
