"""Generate the golden fixtures under tests/golden/ by running the GeoBrain
reference itself (its PyTorch CPU path) on seeded synthetic inputs.

Run once in a checkout that has the reference source tree:

    python tests/golden/make_golden.py /path/to/GeoBrain

The reference has no tests and no published vectors, so these fixtures are
the pin for both the CPU oracle and the CUDA path.  Each fixture stores the
inputs it was made from, so nothing regenerates inputs at test time.

What is recorded, per case:
  * acoustic_forward_kernel (geobrain/physics/wave/kernels/acoustic_2d.py:294)
    traces and energy maps in float32 (the reference's default path) and in
    float64 (torch.set_default_dtype(float64) + dtype=float64: pad_model
    allocates with the default dtype, acoustic_2d.py:49, so both are needed
    for a true float64 run);
  * snapshots (snapshot_every > 0, :422-428) in float32;
  * the autograd gradient dL/dvp, dL/drho in float64 with
    checkpoint_segments=3 (:448-460) for a loss linear in all three traces;
  * the damping array of create_boundary('pml', ..., free_surface=False)
    (boundary/__init__.py:23, pml.py:16-98), the padded model of pad_model and
    the Ricker wavelet (wavelets/ricker.py:55-95) the inputs were built with;
  * for the 100x200 / 1000-step case, the AcousticPropagator.forward result
    (propagators/acoustic.py:150-275) through the full model/survey API.
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def layered_vp(nz, nx, rng, vtop=1500.0, vbot=3500.0, n_layers=5, dv=300.0):
    z = np.arange(nz, dtype=np.float64)[:, None]
    vp = vtop + (vbot - vtop) * z / max(nz - 1, 1) + np.zeros((nz, nx))
    for _ in range(n_layers):
        top = int(rng.integers(0, nz - 1))
        thick = int(rng.integers(2, max(3, nz // 4)))
        vp[top:top + thick, :] += rng.uniform(-dv, dv)
    return vp.astype(np.float32)


def main(ref_root: str) -> None:
    sys.path.insert(0, ref_root)
    import torch
    from geobrain.physics.wave import (AcousticModel, AcousticPropagator, BoundaryConfig, GridConfig,
                                       Receiver, RickerWavelet, Source, Survey, create_boundary)
    from geobrain.physics.wave.kernels import acoustic_forward_kernel, pad_model

    torch.set_num_threads(os.cpu_count() or 1)

    def ricker(f0, dt, nt):
        w, _ = RickerWavelet()(f0=f0, dt=dt)
        w = w.numpy().astype(np.float32)
        return np.pad(w, (0, nt - len(w))) if len(w) < nt else w[:nt]

    def run_kernel(case, dtype, snapshot_every=0, segments=1, grad=False, lin=None):
        tdt = torch.float64 if dtype == np.float64 else torch.float32
        prev = torch.get_default_dtype()
        torch.set_default_dtype(tdt)
        try:
            vp = torch.tensor(case["vp"], dtype=tdt, requires_grad=grad)
            rho = torch.tensor(case["rho"], dtype=tdt, requires_grad=grad)
            out = acoustic_forward_kernel(
                nx=int(case["nx"]), nz=int(case["nz"]), dx=float(case["dx"]), dz=float(case["dx"]),
                nt=int(case["nt"]), dt=float(case["dt"]), nabc=int(case["nabc"]),
                free_surface=bool(case["free_surface"]),
                src_x=torch.tensor(case["src_x"]), src_z=torch.tensor(case["src_z"]),
                src_n=len(case["src_x"]), src_v=torch.tensor(case["src_v"], dtype=tdt),
                rcv_x=torch.tensor(case["rcv_x"]), rcv_z=torch.tensor(case["rcv_z"]),
                rcv_n=len(case["rcv_x"]), damp=torch.tensor(case["damp"], dtype=tdt),
                vp=vp, rho=rho, checkpoint_segments=segments, device=torch.device("cpu"),
                dtype=tdt, snapshot_every=snapshot_every)
            if grad:
                loss = sum((torch.tensor(lin[k], dtype=tdt) * out[k]).sum() for k in ("p", "vx", "vz"))
                loss.backward()
                return out, vp.grad.detach().numpy().copy(), rho.grad.detach().numpy().copy()
            return out
        finally:
            torch.set_default_dtype(prev)

    def make_case(name, nz, nx, nabc, nt, dt, dx, f0, free_surface, src_x, src_z, rcv_x, rcv_z, seed,
                  rho_var=True, with_grad=True, keep_all=True):
        rng = np.random.default_rng(seed)
        vp = layered_vp(nz, nx, rng)
        if rho_var:
            rho = (2000.0 + 300.0 * rng.standard_normal((nz, nx)).clip(-2, 2)).astype(np.float32)
        else:
            rho = np.full((nz, nx), 2200.0, dtype=np.float32)
        damp = create_boundary("pml", nx=nx, nz=nz, dx=dx, dz=dx, n_layers=nabc,
                               vmax=float(vp.max()), free_surface=False).astype(np.float32)
        w = ricker(f0, dt, nt)
        S = len(src_x)
        case = dict(nz=nz, nx=nx, nabc=nabc, nt=nt, dt=dt, dx=dx, f0=f0, free_surface=free_surface,
                    vp=vp, rho=rho, damp=damp, src_v=np.tile(w, (S, 1)).astype(np.float32),
                    wavelet=w, src_x=np.asarray(src_x, np.int64), src_z=np.asarray(src_z, np.int64),
                    rcv_x=np.asarray(rcv_x, np.int64), rcv_z=np.asarray(rcv_z, np.int64),
                    pad_vp=pad_model(torch.tensor(vp), nabc, nz, nx).numpy())
        t0 = time.time()
        o32 = run_kernel(case, np.float32)
        o64 = run_kernel(case, np.float64)
        keys = ("p", "vx", "vz") if keep_all else ("p",)
        for k in keys:
            case[f"ref32_{k}"] = o32[k].numpy().astype(np.float32)
            case[f"ref64_{k}"] = o64[k].numpy().astype(np.float64 if keep_all else np.float32)
        for k in ("forward_wavefield_p", "forward_wavefield_vx", "forward_wavefield_vz"):
            case[f"ref32_{k}"] = o32[k].numpy().astype(np.float32)
            case[f"ref64_{k}"] = o64[k].numpy().astype(np.float64)
        if keep_all:
            snap_every = max(nt // 5, 1)
            os_ = run_kernel(case, np.float32, snapshot_every=snap_every)
            case["snapshot_every"] = snap_every
            case["ref32_snapshots"] = os_["snapshots"].numpy().astype(np.float32)
        if with_grad:
            lin = {k: rng.standard_normal((S, nt, len(rcv_x))) for k in ("p", "vx", "vz")}
            _, gvp, grho = run_kernel(case, np.float64, segments=3, grad=True, lin=lin)
            for k in lin:
                case[f"lin_{k}"] = lin[k].astype(np.float64)
            case["ref64_grad_vp"] = gvp
            case["ref64_grad_rho"] = grho
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **case)
        print(f"{name}: {time.time() - t0:.1f}s")
        return case

    rx = np.concatenate([np.arange(0, 48, 2), np.arange(1, 48, 4)])
    rz = np.concatenate([np.ones(24, np.int64), np.full(12, 25)])
    make_case("small_nofs", 32, 48, 10, 240, 1e-3, 10.0, 25.0, False,
              [8, 24, 40], [1, 1, 3], rx, rz, seed=1)
    make_case("small_fs", 32, 48, 10, 240, 1e-3, 10.0, 25.0, True,
              [8, 24, 40], [1, 1, 3], rx, rz, seed=2)

    # The 100 x 200, 20-cell PML, 1000-step, one-shot forward workload, run
    # through the reference's own model / survey / propagator API.
    nz, nx, nabc, nt, dt, dx, f0 = 100, 200, 20, 1000, 1e-3, 10.0, 15.0
    rng = np.random.default_rng(0)
    vp = layered_vp(nz, nx, rng)
    rho = np.full((nz, nx), 2200.0, dtype=np.float32)
    w = ricker(f0, dt, nt)
    grid = GridConfig(nx=nx, nz=nz, dx=dx, dz=dx)
    bnd = BoundaryConfig(type="pml", n_layers=nabc, free_surface=False)
    model = AcousticModel(grid=grid, boundary=bnd, vp=vp, rho=rho, auto_update_rho=False)
    src = Source(nt=nt, dt=dt, f0=f0)
    src.add_source(x=100, z=1, wavelet=w)
    rcv = Receiver(nt=nt, dt=dt)
    rcv.add_receivers(x=np.arange(nx), z=np.ones(nx, dtype=int), rcv_type="pr")
    prop = AcousticPropagator(model, Survey(src, rcv), device="cpu", dtype=torch.float32)
    t0 = time.time()
    res = prop.forward()
    el = time.time() - t0
    np.savez_compressed(
        os.path.join(HERE, "layered_100x200.npz"),
        nz=nz, nx=nx, nabc=nabc, nt=nt, dt=dt, dx=dx, f0=f0, free_surface=False,
        vp=vp, rho=rho, wavelet=w, damp=prop.damp.numpy(), src_x=np.array([100]), src_z=np.array([1]),
        rcv_x=np.arange(nx), rcv_z=np.ones(nx, dtype=np.int64),
        ref32_p=res.p.numpy(), ref32_vx=res.vx.numpy(), ref32_vz=res.vz.numpy(),
        ref32_forward_wavefield_p=res.forward_wavefield_p.numpy(),
        ref32_forward_wavefield_vx=res.forward_wavefield_vx.numpy(),
        ref32_forward_wavefield_vz=res.forward_wavefield_vz.numpy(),
        ref_cpu_seconds=el, ref_cpu_threads=torch.get_num_threads())
    print(f"layered_100x200: {el:.1f}s")


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GEOBRAIN_REF")
    if not root:
        sys.exit("usage: %s <path to the GeoBrain source tree> (or set GEOBRAIN_REF)" % os.path.basename(__file__))
    main(root)
