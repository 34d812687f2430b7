#!/usr/bin/env python
"""Benchmark: FWI gradient throughput of the B200 acoustic propagator.

Workload (one "step" = one full gradient evaluation): the 400 x 1200 model,
dx 10 m, dt 0.8 ms, 3000 time steps, 8th-order stencil, 30-cell PML, 32
Ricker shots, 1200 receivers, L2 misfit on pressure against data modelled in
the true model; forward keeping the imaging fields (24-bit by default, so all
3000 steps fit in HBM; checkpoints and recompute for whatever does not fit),
residual, hand-written adjoint, dL/dvp.  Metric: Gcell-updates/s, one unit =
one (shot, padded cell, time step) forward update plus its adjoint update
(recompute not counted).  The gradient's relative L2 difference from the
all-fp32 path (fp32 checkpoints, fp32 recompute, no cache) is measured once
outside the timed region and reported.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
    python bench.py --slice forward|gradient --nt N [...]   (a short slice for ncu)

Prints ONE JSON line on rank 0.  Under torchrun (N > 1) every rank models
its own 32 shots of the same survey (weak scaling) and the per-rank
gradients are summed with one NCCL all-reduce inside the timed step.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FWI gradient Gcell-updates/s (fwd+adjoint, batched) vs plain fwd kernel, 1 B200"
UNIT = "Gcell-updates/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--nt", type=int, default=3000, help="time steps of the workload (3000 = full)")
    ap.add_argument("--no-extras", action="store_true")
    ap.add_argument("--imaging-dtype", default="fp24", choices=["fp32", "fp24", "bf16"],
                    help="storage of the cached imaging fields")
    # a short slice of a workload for profilers (ncu): runs once, times nothing
    ap.add_argument("--slice", choices=["forward", "gradient"], default=None,
                    help="run nt steps of the forward (or forward + adjoint) once and exit (for ncu)")
    ap.add_argument("--shots", type=int, default=32, help="--slice: shots of the 400 x 1200 model")
    ap.add_argument("--model", choices=["2d", "3d", "100x200", "ensemble"], default="2d",
                    help="--slice: which workload")
    ap.add_argument("--models", type=int, default=6, help="--slice --model ensemble: particles of 256 x 512")
    ap.add_argument("--tile-rows", type=int, default=0, help="--slice: tile kernel rows (16 or 32)")
    ap.add_argument("--shots-per-cta", type=int, default=0, help="--slice: shots per CTA of the tile kernel")
    ap.add_argument("--energy", action="store_true", help="--slice: forward with the energy sums")
    ap.add_argument("--absorbing", choices=["damping", "cpml"], default="damping", help="--slice: absorbing layers")
    ap.add_argument("--resident", choices=["auto", "on", "off", "global", "cluster"], default="auto",
                    help="--slice: resident forward (plain forward only) and its exchange")
    ap.add_argument("--resident-rows", type=int, default=0, help="--slice: resident tile rows (0 = automatic)")
    ap.add_argument("--fused3", type=int, default=0, choices=[0, 1, 2],
                    help="--slice --model 3d: the fused 3-D step kernel with 8- (1) or 16-row (2) tiles")
    return ap.parse_args()


def run_slice(args):
    """A short slice of a benchmark workload, for profilers: nt steps of the
    400 x 1200 / 8th-order model (--shots of its 32 shots; --model 100x200 for
    the 4th-order plain forward workload, --model 3d for a 200^3 model with 4
    shots, --model ensemble for --models particles of the 256 x 512 ensemble
    through the batched engine), forward or forward + adjoint, once;
    synchronises and exits 0.  Everything stays on the device; nothing is
    timed.  The gradient keeps
    every step's imaging fields in --imaging-dtype (fp24 by default, as the
    benchmark does); --absorbing cpml uses the CPML layers."""
    import torch
    from geobrain_b200 import synthetic, wave
    from geobrain_b200.wave import engine
    dev = torch.device("cuda:0")
    if args.model == "3d":
        _slice_3d(torch, wave, args, dev)
        torch.cuda.synchronize()
        print("slice: ok")
        return
    if args.model == "ensemble":
        ws = synthetic.ensemble_256x512(n_particles=args.models, nt=args.nt)
        ms = [_model_kwargs(torch, wave, w, dev) for w in ws]
        if args.slice == "forward":
            with torch.no_grad():
                wave.acoustic_forward_batched(ms, fd_order=8, want_energy=args.energy, device=dev)
        else:
            wave.acoustic_gradient_batched(ms, lambda i, p: (0.5 * (p * p).sum(), p), fd_order=8, device=dev,
                                           imaging_dtype=args.imaging_dtype)
        torch.cuda.synchronize()
        print("slice: ok")
        return
    if args.model == "100x200":
        w = synthetic.plain_forward_100x200()
        w.nt = args.nt
        w.wavelet = w.wavelet[:args.nt]
    else:
        w = synthetic.fwi_400x1200(nt=args.nt, n_shots=args.shots)
    damp = torch.tensor(wave.bc_pml(w.nx, w.nz, w.dx, w.dx, w.nabc, float(w.vp.max()), False), dtype=torch.float32,
                        device=dev)
    geo = engine.Geometry(w.nz, w.nx, w.nabc, w.nt, float(w.dt), float(w.dx), w.fd_order // 2, False)
    plan = engine.get_plan(geo, w.src_x, w.src_z, w.rcv_x, w.rcv_z)
    plan.set_absorbing(args.absorbing, float(w.vp.max()) if args.absorbing == "cpml" else 0.0)
    if args.tile_rows or args.shots_per_cta:
        plan.set_tiling(args.tile_rows, args.shots_per_cta)
    plan.set_resident({"auto": "auto", "on": True, "off": False, "global": "global", "cluster": "cluster"}[args.resident],
                      args.resident_rows)
    vp = torch.tensor(w.vp, device=dev)
    rho = torch.tensor(w.rho, device=dev)
    src_v = torch.tensor(np.tile(w.wavelet, (w.n_shots, 1)), device=dev)
    if args.slice == "forward":
        engine.run_forward(plan, vp, rho, damp, src_v, want_energy=args.energy)
    else:
        img = torch.empty(plan.imaging_bytes(w.nt, False, args.imaging_dtype), dtype=torch.uint8, device=dev)
        store = engine.make_store(None, w.nt, "fp32", img, w.nt, False, args.imaging_dtype)
        p, _, _, _, _ = engine.run_forward(plan, vp, rho, damp, src_v, want_energy=args.energy, store=store)
        engine.run_backward(plan, vp, rho, damp, src_v, p, None, None, store, False)
    torch.cuda.synchronize()
    print("slice: ok")


def _slice_3d(torch, wave, args, dev, nz=200, ny=200, nx=200, shots=4, nabc=20):
    if args.fused3:
        from geobrain_b200 import _lib
        _lib.load().gb3_set_fused_step(args.fused3)
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
    if args.slice == "forward":
        with torch.no_grad():
            wave.acoustic_forward_kernel_3d(vp=vp, **kw)
    else:
        v = vp.detach().requires_grad_(True)
        out = wave.acoustic_forward_kernel_3d(vp=v, **kw)
        (0.5 * (out["p"] * out["p"]).sum()).backward()


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(kernel: str):
    """Per-launch DRAM bytes of `kernel` from the committed ncu summary, or None."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    return d.get(kernel, {}).get("dram_bytes_per_launch")


class ClockSampler:
    """nvidia-smi clocks and throttle reasons every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        sms, maxes, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sms.append(float(parts[1]))
                    maxes.append(float(parts[2]))
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        os.unlink(self.path)
        if not sms:
            return None
        return {"sm_mhz": float(np.median(sms)), "sm_max_mhz": float(max(maxes)), "reasons": sorted(reasons),
                "samples": len(sms)}


# ---------------------------------------------------------------------------
# CPU legs (oracle restatement of the reference; never the product path)
# ---------------------------------------------------------------------------
def cpu_gradient_rate(w, n_shots: int, nt: int, reps: int = 1):
    from oracle import oracle as orc
    from geobrain_b200.wave.boundary import bc_pml
    damp = bc_pml(w.nx, w.nz, w.dx, w.dx, w.nabc, float(w.vp.max()), free_surface=False).astype(np.float32)
    S = n_shots
    sx = w.src_x[np.linspace(0, w.n_shots - 1, S).astype(int)]
    kw = dict(nz=w.nz, nx=w.nx, dz=w.dx, nt=nt, dt=w.dt, nabc=w.nabc, free_surface=False, src_x=sx,
              src_z=np.ones(S, np.int64), src_v=np.tile(w.wavelet[:nt], (S, 1)), rcv_x=w.rcv_x, rcv_z=w.rcv_z,
              damp=damp, vp=w.vp, rho=w.rho, half=w.fd_order // 2, dtype=np.float32)
    res = np.random.default_rng(0).standard_normal((S, nt, w.rcv_x.size)).astype(np.float32)
    best = None
    for _ in range(reps):
        t0 = time.perf_counter()
        orc.gradient(**kw, res_p=res)
        el = time.perf_counter() - t0
        best = el if best is None else min(best, el)
    units = S * w.cells * nt
    return units / best / 1e9, orc.max_threads(), f"{S} shots x {nt} steps of the {w.nz}x{w.nx} grid " \
                                                    f"(forward + adjoint, fp32 C oracle, OpenMP)"


def _one_shot_kwargs(torch, wave, w, dev, shots, nt):
    """Keyword arguments of acoustic_forward_kernel for a subset of a
    workload's shots and its first nt steps (the full grid and receivers)."""
    shots = np.asarray(shots)
    damp = wave.bc_pml(w.nx, w.nz, w.dx, w.dx, w.nabc, float(w.vp.max()), free_surface=False)
    S = shots.size
    return dict(nx=w.nx, nz=w.nz, dx=w.dx, dz=w.dx, nt=nt, dt=w.dt, nabc=w.nabc, free_surface=False,
                src_x=w.src_x[shots], src_z=w.src_z[shots], src_n=S,
                src_v=torch.tensor(np.tile(w.wavelet[:nt], (S, 1)), device=dev), rcv_x=w.rcv_x, rcv_z=w.rcv_z,
                rcv_n=w.rcv_x.size, damp=torch.tensor(damp, dtype=torch.float32, device=dev),
                rho=torch.tensor(w.rho, device=dev), device=dev, fd_order=w.fd_order, want_energy=False), damp


def _oracle_kwargs(kw, w, damp, nt):
    return dict(nz=w.nz, nx=w.nx, dz=w.dx, nt=nt, dt=w.dt, nabc=w.nabc, free_surface=False, src_x=kw["src_x"],
                src_z=kw["src_z"], src_v=kw["src_v"].cpu().numpy(), rcv_x=w.rcv_x, rcv_z=w.rcv_z, damp=damp,
                vp=w.vp, rho=w.rho, half=w.fd_order // 2)


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def oracle_check_fwi(torch, wave, w, dev, imaging_dtype, shots=(5, 26), nt=150):
    """Traces and gradient of the benchmark configuration against the float64
    C oracle, untimed: the full 460 x 1260 padded grid, 2 of the 32 shots,
    the first 150 steps, 8th order, imaging fields cached in the benchmark's
    format (all 150 steps fit) and fp32 checkpoints, as timed.  The adjoint
    source is a seeded random residual (loss = sum(res * p))."""
    nt = min(nt, w.nt)             # a shortened run (--nt) checks its own steps
    from oracle import oracle as orc
    kw, damp = _one_shot_kwargs(torch, wave, w, dev, list(shots), nt)
    res = np.random.default_rng(11).standard_normal((len(shots), nt, w.rcv_x.size)).astype(np.float32)
    vp = torch.tensor(w.vp, device=dev, requires_grad=True)
    out = wave.acoustic_forward_kernel(vp=vp, imaging_dtype=imaging_dtype, **kw)
    (out["p"] * torch.tensor(res, device=dev)).sum().backward()
    okw = _oracle_kwargs(kw, w, damp, nt)
    t0 = time.perf_counter()
    ref = orc.forward(**okw, dtype=np.float64)
    gref, _, _ = orc.gradient(**okw, res_p=res.astype(np.float64), dtype=np.float64)
    return {"trace_rel_l2_vs_fp64_oracle": _rel(out["p"].detach().cpu().numpy(), ref["p"]),
            "rel_l2_vs_fp64_oracle": _rel(vp.grad.cpu().numpy(), gref),
            "oracle_case": f"{w.nz}x{w.nx} grid, shots {list(shots)}, {nt} steps, order {w.fd_order}, "
                           f"{imaging_dtype} imaging cache, fp32 checkpoints; adjoint source seeded N(0,1)",
            "oracle_seconds": time.perf_counter() - t0, "oracle_threads": orc.max_threads()}


def large_gradient_check(torch, wave, synthetic, dev, K, formats, shot=7):
    """Gradient error of the memory-capped 1000 x 3000 configuration, untimed:
    the full 1080 x 3080 padded grid, one shot, 2K + 8 steps with the real
    run's segment length K and no imaging cache, so the adjoint restarts
    twice from stored snapshots (fp24 imaging fields, as in the timed run).
    Each snapshot format is compared with the fp32-snapshot run of the same
    problem and with the float64 C oracle.  Adjoint source: a seeded random
    residual."""
    from oracle import oracle as orc
    nt = 2 * K + 8
    w = synthetic.large_1000x3000(nt=nt)
    kw, damp = _one_shot_kwargs(torch, wave, w, dev, [shot], nt)
    res = np.random.default_rng(12).standard_normal((1, nt, w.rcv_x.size)).astype(np.float32)
    res_d = torch.tensor(res, device=dev)

    def grad(fmt):
        vp = torch.tensor(w.vp, device=dev, requires_grad=True)
        out = wave.acoustic_forward_kernel(vp=vp, checkpoint_every=K, snapshot_dtype=fmt, imaging_cache=0,
                                           imaging_dtype="fp24", **kw)
        (out["p"] * res_d).sum().backward()
        return vp.grad.cpu().numpy()

    g = {fmt: grad(fmt) for fmt in ("fp32",) + tuple(formats)}
    t0 = time.perf_counter()
    gref, _, _ = orc.gradient(**_oracle_kwargs(kw, w, damp, nt), res_p=res.astype(np.float64), dtype=np.float64)
    out = {"case": f"{w.nz}x{w.nx} grid, shot {shot}, {nt} steps, checkpoint_every {K} (2 restarts), "
                   f"fp24 imaging, no cache; adjoint source seeded N(0,1)",
           "oracle_seconds": time.perf_counter() - t0, "oracle_threads": orc.max_threads(),
           "fp32_snapshots_rel_l2_vs_fp64_oracle": _rel(g["fp32"], gref)}
    for fmt in formats:
        out[fmt] = {"rel_l2_vs_fp32_snapshots": _rel(g[fmt], g["fp32"]), "rel_l2_vs_fp64_oracle": _rel(g[fmt], gref)}
    return out


def workload_config(w, world, imaging_dtype):
    """The workload's `config`, printed identically by both arms."""
    return {"workload": "fwi_400x1200", "grid": [w.nz, w.nx], "nabc": w.nabc, "dx": w.dx, "dt": w.dt,
            "nt": w.nt, "fd_order": w.fd_order, "n_shots_per_gpu": w.n_shots, "n_receivers": int(w.rcv_x.size),
            "misfit": "L2 on pressure", "checkpoints": "fp32, auto segment length",
            "imaging_cache": f"{imaging_dtype}, auto budget",
            "l2": "inputs larger than L2 (fields 2 x 222 MB per state, no flush needed)",
            "parallelism": f"shots{world}" if world > 1 else "single GPU"}


def run_reference_arm(args):
    """--impl reference: the reference algorithm's CPU restatement on the host
    cores, same metric and config, bounded sample per step."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from geobrain_b200 import synthetic
    w = synthetic.fwi_400x1200(nt=args.nt)
    S, nt = 2, min(60, args.nt)
    for _ in range(max(args.warmup, 0)):
        cpu_gradient_rate(w, S, nt)
    rates = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        r, cores, sample = cpu_gradient_rate(w, S, nt)
        rates.append(r)
    el = time.perf_counter() - t0
    v = float(np.mean(rates))
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Gaussian-field model, Ricker shots)",
        "config": workload_config(w, args.gpus, args.imaging_dtype),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


# ---------------------------------------------------------------------------
# B200 arm
# ---------------------------------------------------------------------------
def main():
    args = parse()
    if args.slice:
        run_slice(args)
        return
    if args.impl == "reference":
        run_reference_arm(args)
        return

    import torch
    import torch.distributed as dist
    from geobrain_b200 import synthetic, wave
    from geobrain_b200.wave import engine, sharding

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    w = synthetic.fwi_400x1200(nt=args.nt)
    S = w.n_shots
    # weak scaling: rank r models shots shifted by r / world of a shot spacing
    if world > 1:
        spacing = (w.nx - 1) / (S + 1)
        w.src_x = np.clip(np.round(w.src_x + rank * spacing / world), 0, w.nx - 1).astype(np.int64)
    damp = wave.bc_pml(w.nx, w.nz, w.dx, w.dx, w.nabc, float(w.vp_true.max()), free_surface=False)
    damp_t = torch.tensor(damp, dtype=torch.float32, device=dev)
    src_v = torch.tensor(np.tile(w.wavelet, (S, 1)), device=dev)
    common = dict(nx=w.nx, nz=w.nz, dx=w.dx, dz=w.dx, nt=w.nt, dt=w.dt, nabc=w.nabc, free_surface=False,
                  src_x=w.src_x, src_z=w.src_z, src_n=S, src_v=src_v, rcv_x=w.rcv_x, rcv_z=w.rcv_z,
                  rcv_n=w.rcv_x.size, damp=damp_t, device=dev, fd_order=w.fd_order)
    rho_t = torch.tensor(w.rho, device=dev)
    with torch.no_grad():
        d_obs = wave.acoustic_forward_kernel(vp=torch.tensor(w.vp_true, device=dev), rho=rho_t, want_energy=False,
                                             **common)["p"].contiguous()

    def gradient_step(vp_dev, d_obs_dev, imaging_dtype=args.imaging_dtype, imaging_cache="auto", d_obs_ready=None):
        vp = vp_dev.detach().requires_grad_(True)
        out = wave.acoustic_forward_kernel(vp=vp, rho=rho_t, imaging_dtype=imaging_dtype,
                                           imaging_cache=imaging_cache, **common)
        if d_obs_ready is not None:       # the observed traces were copied in beside the forward
            torch.cuda.current_stream().wait_event(d_obs_ready)
        res = out["p"] - d_obs_dev
        loss = 0.5 * (res * res).sum()
        loss.backward()
        g = vp.grad
        if world > 1:      # one packed NCCL all-reduce of the gradient and the misfit
            loss, g = sharding.allreduce_packed([loss.detach().reshape(1), g])
            loss = loss.reshape(())
        return g, loss

    vp0 = torch.tensor(w.vp, device=dev)
    geo = engine.Geometry(w.nz, w.nx, w.nabc, w.nt, float(w.dt), float(w.dx), w.fd_order // 2, False)
    plan = engine.get_plan(geo, w.src_x, w.src_z, w.rcv_x, w.rcv_z)

    # CPU baseline first (rank 0, N = 1 only), outside every timed region
    cpu = None
    if rank == 0 and world == 1:
        v, cores, sample = cpu_gradient_rate(w, 2, min(60, w.nt))
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample}

    for _ in range(max(args.warmup, 3)):
        gradient_step(vp0, d_obs)
    torch.cuda.synchronize()

    def timed(fn, steps):
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        ms = torch.tensor([e0.elapsed_time(e1)], device=dev)
        if world > 1:
            dist.all_reduce(ms, op=dist.ReduceOp.MAX)
        return float(ms.item())

    plan.set_profiling(True)
    with ClockSampler(local) as clk:
        ms_total = timed(lambda: gradient_step(vp0, d_obs), args.steps)
    prof = plan.profile()
    plan.set_profiling(False)
    clocks = clk.summary()

    units = S * w.cells * w.nt * world
    ms_step = ms_total / args.steps
    value = units / (ms_step * 1e-3) / 1e9

    # end to end: pinned host inputs copied in, gradient and loss read back,
    # every step.  The observed traces (460 MB) travel on a second stream
    # while the forward runs; the misfit waits for them.  Each step ends on
    # the loss read, so the next step's copies never overwrite traces still
    # in use.
    vp_host = torch.tensor(w.vp).pin_memory()
    dobs_host = d_obs.cpu().pin_memory()
    g_host = torch.empty((w.nz, w.nx), dtype=torch.float32).pin_memory()
    dobs_dev = torch.empty_like(d_obs)
    copy_stream = torch.cuda.Stream(device=dev)
    dobs_in = torch.cuda.Event()

    def e2e_step():
        vp_d = vp_host.to(dev, non_blocking=True)
        with torch.cuda.stream(copy_stream):
            dobs_dev.copy_(dobs_host, non_blocking=True)
            dobs_in.record(copy_stream)
        g, loss = gradient_step(vp_d, dobs_dev, d_obs_ready=dobs_in)
        g_host.copy_(g, non_blocking=True)
        return float(loss.item())

    e2e_step()
    ms_e2e = timed(e2e_step, args.steps) / args.steps
    h2d = vp_host.numel() * 4 + dobs_host.numel() * 4
    d2h = g_host.numel() * 4 + 4

    # roofline of the kernels, from the CUDA-event phase timings of the timed region
    peak, peak_kind = measured_peaks()
    nt, cells = w.nt, w.cells
    # ms per time step of each phase (all shot groups of a step together)
    per_step_fwd = prof["forward_ms"] / max(prof["forward_steps"], 1)
    per_step_rec = prof["recompute_ms"] / max(prof["recompute_steps"], 1)
    per_step_adj = prof["adjoint_ms"] / max(prof["adjoint_steps"], 1)
    cached_frac = 1.0 - prof["recompute_steps"] / max(prof["adjoint_steps"], 1)
    eb = {"fp32": 4, "fp24": 3, "bf16": 2}[args.imaging_dtype]   # bytes per cached imaging value
    # per time step: fields r+w, a1 / a2 shared by the shots; the forward
    # writes the imaging field of cached steps, the recompute of the others;
    # the adjoint reads it (cached or recomputed), coefficients, gradient sums
    b_fwd = S * cells * (24 + 8 / S + eb * cached_frac)
    b_rec = S * cells * (24 + 4 + 8 / S)
    b_adj = S * cells * (24 + 16 / S + eb * cached_frac + 4 * (1 - cached_frac))
    kern = {
        "fwd_step (forward)": {"ms_per_launch": per_step_fwd, "bytes_per_launch": b_fwd},
        "fwd_step (recompute)": {"ms_per_launch": per_step_rec, "bytes_per_launch": b_rec},
        "adj_step": {"ms_per_launch": per_step_adj, "bytes_per_launch": b_adj},
    }
    for k, v in kern.items():
        v["achieved_gbs"] = v["bytes_per_launch"] / (v["ms_per_launch"] * 1e-3) / 1e9 if v["ms_per_launch"] else 0
        v["frac"] = v["achieved_gbs"] / peak
    # dominant kernel by share of the timed region; fwd_step runs twice per
    # gradient (forward pass and recompute), adj_step once
    t_fwd = prof["forward_ms"] + prof["recompute_ms"]
    t_adj = prof["adjoint_ms"]
    if t_fwd >= t_adj:
        tname = "fwd_step"
        n_f, n_r = prof["forward_steps"], prof["recompute_steps"]
        achieved = (b_fwd * n_f + b_rec * n_r) / (t_fwd * 1e-3) / 1e9
    else:
        tname = "adj_step"
        achieved = b_adj / (per_step_adj * 1e-3) / 1e9
    roofline = {"kernel": tname, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak,
                "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                else "fallback 6.65 TB/s",
                "share_of_step": max(t_fwd, t_adj) / args.steps / ms_step, "traffic": ncu_traffic(tname)}
    grad_bytes = units / world * (56 + 16 / S)
    grad_roof = {"algorithmic_bytes_per_unit": 56 + 16 / S, "kernels": "fwd_step + adj_step (+ recompute)",
                 "achieved": grad_bytes / (ms_step * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                 "frac": grad_bytes / (ms_step * 1e-3) / 1e9 / peak}

    # accuracy of the timed configuration: gradient against the all-fp32 path
    g_fast, _ = gradient_step(vp0, d_obs)
    g_ref, _ = gradient_step(vp0, d_obs, imaging_dtype="fp32", imaging_cache=0)
    grad_check = {"rel_l2_vs_fp32_storage": float(torch.linalg.vector_norm(g_fast - g_ref) /
                                                  torch.linalg.vector_norm(g_ref)),
                  "reference_path": "fp32 checkpoints, fp32 recompute of every step, no imaging cache"}
    del g_fast, g_ref
    if rank == 0 and world == 1:
        grad_check.update(oracle_check_fwi(torch, wave, w, dev, args.imaging_dtype))

    extras = {}
    if not args.no_extras and world == 1:
        extras = plain_forward_rates(torch, wave, synthetic, dev)
        extras.update(batch_rates(torch, wave, synthetic, dev))
        extras.update(large_gradient_rate(torch, wave, synthetic, dev))
        extras.update(rates_3d(torch, wave, dev))
        extras.update(cpml_gradient_rate(torch, wave, synthetic, dev))
        extras.update(reference_gpu_rates(torch, wave, synthetic, dev))

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Gaussian-field model, Ricker shots)",
        "config": workload_config(w, world, args.imaging_dtype),
        "e2e": {"value": units / (ms_e2e * 1e-3) / 1e9, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "ms_per_step": ms_e2e},
        "roofline": roofline,
        "gradient_roofline": grad_roof,
        "kernels": kern,
        "phase_ms_per_step": {k: prof[k] / args.steps for k in ("forward_ms", "recompute_ms", "adjoint_ms")},
        "imaging_cache_fraction": cached_frac,
        "gradient_check": grad_check,
        "gpu_launches": int(prof["launches"]),
        "clocks": clocks,
        "cpu_baseline": cpu,
        "extras": extras,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def plain_forward_rates(torch, wave, synthetic, dev):
    """Plain forward kernel rates beside the gradient: the 400 x 1200 grid
    with one shot and with 32 shots (damping layers, and the CPML option),
    and the 100 x 200 4th-order workload.  Roofline fraction at the damping
    scheme's algorithmic bytes, 24 + 8 / shots per unit (the CPML option
    moves more in its layers)."""
    peak, _ = measured_peaks()
    out = {}
    for name, w, absorbing in (("fwd_400x1200_1shot", synthetic.fwi_400x1200(nt=3000, n_shots=1), "damping"),
                               ("fwd_400x1200_32shots", synthetic.fwi_400x1200(nt=1000), "damping"),
                               ("fwd_400x1200_32shots_cpml", synthetic.fwi_400x1200(nt=1000), "cpml"),
                               ("fwd_100x200_1shot", synthetic.plain_forward_100x200(), "damping")):
        damp = torch.tensor(wave.bc_pml(w.nx, w.nz, w.dx, w.dx, w.nabc, float(w.vp.max()), False),
                            dtype=torch.float32, device=dev)
        kw = dict(nx=w.nx, nz=w.nz, dx=w.dx, dz=w.dx, nt=w.nt, dt=w.dt, nabc=w.nabc, free_surface=False,
                  src_x=w.src_x, src_z=w.src_z, src_n=w.n_shots,
                  src_v=torch.tensor(np.tile(w.wavelet, (w.n_shots, 1)), device=dev), rcv_x=w.rcv_x,
                  rcv_z=w.rcv_z, rcv_n=w.rcv_x.size, damp=damp, vp=torch.tensor(w.vp, device=dev),
                  rho=torch.tensor(w.rho, device=dev), device=dev, fd_order=w.fd_order, absorbing=absorbing)
        for _ in range(2):
            wave.acoustic_forward_kernel(**kw)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        reps = 3
        for _ in range(reps):
            wave.acoustic_forward_kernel(**kw)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        rate = w.cell_updates() / (ms * 1e-3) / 1e9
        # p, vx, vz read and written once per step; a1, a2 read once per shot group
        b_unit = 24 + 8 / w.n_shots
        from geobrain_b200.wave import engine
        plan = engine.get_plan(engine.Geometry(w.nz, w.nx, w.nabc, w.nt, float(w.dt), float(w.dx), w.fd_order // 2,
                                               False), w.src_x, w.src_z, w.rcv_x, w.rcv_z)
        res = plan.resident()
        out[name] = {"gcell_updates_per_s": rate, "ms": ms, "fd_order": w.fd_order, "nt": w.nt,
                     "shots": w.n_shots, "absorbing": absorbing, "bytes_per_unit": b_unit,
                     "achieved_gbs": rate * b_unit, "frac": rate * b_unit / peak,
                     "kernel": (f"resident ({res['tile_rows']}-row tiles, {res['exchange']} exchange, "
                                "one launch)" if res["tile_rows"] else "tile kernel, one launch per step")}
    return out


def cpml_gradient_rate(torch, wave, synthetic, dev, nt=1000):
    """The CPML option's gradient through the public API: the 400 x 1200
    grid, 32 shots, 8th order, nt truncated to 1000 steps (its adjoint reads
    every step's fp24 imaging field: 56 GB here), loss 0.5 ||p - d_obs||^2."""
    w = synthetic.fwi_400x1200(nt=nt)
    kw = _model_kwargs(torch, wave, w, dev)
    kw.pop("vp")
    vp0 = torch.tensor(w.vp, device=dev)
    common = dict(dx=w.dx, dz=w.dx, nt=w.nt, dt=w.dt, nabc=w.nabc, device=dev, fd_order=w.fd_order,
                  absorbing="cpml", imaging_dtype="fp24")
    kw = {k: v for k, v in kw.items() if k not in common}
    with torch.no_grad():
        d_obs = wave.acoustic_forward_kernel(vp=vp0 * 1.02, **kw, **common)["p"]

    def grad():
        v = vp0.clone().requires_grad_(True)
        r = wave.acoustic_forward_kernel(vp=v, **kw, **common)["p"] - d_obs
        (0.5 * (r * r).sum()).backward()

    ms = _timed(torch, grad, 1)
    return {"cpml_gradient_400x1200_32shots": {"gcell_updates_per_s": w.cell_updates() / (ms * 1e-3) / 1e9,
                                               "ms": ms, "nt": nt, "shots": w.n_shots, "fd_order": w.fd_order,
                                               "imaging": "fp24, every step"}}


def reference_gpu_rates(torch, wave, synthetic, dev, nt=100, segments=4):
    """The reference's own PyTorch path on the B200, for comparison: its
    acoustic_forward_kernel (geobrain/physics/wave/kernels/acoustic_2d.py
    :294-501, installed unmodified under baseline/_ref) on the benchmark's
    400 x 1200 grid, 30-cell PML and 32 shots at its only order (4), nt
    truncated to 100 steps.  Forward without autograd, and the gradient of
    0.5 ||p - d_obs||^2 by loss.backward() through its checkpointed step loop
    (checkpoint_segments = 4, as examples/07 uses); one unit = one forward
    plus one adjoint step of a (shot, padded cell), as for the headline."""
    ref_dir = os.path.join(ROOT, "baseline", "_ref")
    if not os.path.isdir(os.path.join(ref_dir, "geobrain")):
        return {"reference_pytorch_gpu": {"unavailable": "the reference is not installed under baseline/_ref"}}
    sys.path.insert(0, ref_dir)
    try:
        from geobrain.physics.wave.kernels import acoustic_forward_kernel as ref_kernel
    finally:
        sys.path.remove(ref_dir)
    w = synthetic.fwi_400x1200(nt=nt)
    S = w.n_shots
    damp = torch.tensor(wave.bc_pml(w.nx, w.nz, w.dx, w.dx, w.nabc, float(w.vp.max()), False),
                        dtype=torch.float32, device=dev)
    kw = dict(nx=w.nx, nz=w.nz, dx=w.dx, dz=w.dx, nt=nt, dt=w.dt, nabc=w.nabc, free_surface=False,
              src_x=torch.tensor(w.src_x, dtype=torch.long, device=dev),
              src_z=torch.tensor(w.src_z, dtype=torch.long, device=dev), src_n=S,
              src_v=torch.tensor(np.tile(w.wavelet[:nt], (S, 1)), device=dev),
              rcv_x=torch.tensor(w.rcv_x, dtype=torch.long, device=dev),
              rcv_z=torch.tensor(w.rcv_z, dtype=torch.long, device=dev), rcv_n=int(w.rcv_x.size), damp=damp,
              rho=torch.tensor(w.rho, device=dev), device=dev, dtype=torch.float32)
    vp = torch.tensor(w.vp, device=dev)
    units = S * (w.nz + 2 * w.nabc) * (w.nx + 2 * w.nabc) * nt
    with torch.no_grad():
        d_obs = ref_kernel(vp=vp * 1.02, **kw)["p"]

    def fwd():
        with torch.no_grad():
            ref_kernel(vp=vp, **kw)

    def grad():
        v = vp.clone().requires_grad_(True)
        r = ref_kernel(vp=v, checkpoint_segments=segments, **kw)["p"] - d_obs
        (0.5 * (r * r).sum()).backward()

    ms_f, ms_g = _timed(torch, fwd, 2), _timed(torch, grad, 1)

    # this library on the identical inputs and order, through the same call
    def fwd_b200():
        with torch.no_grad():
            wave.acoustic_forward_kernel(vp=vp, **kw)

    def grad_b200():
        v = vp.clone().requires_grad_(True)
        r = wave.acoustic_forward_kernel(vp=v, checkpoint_segments=segments, **kw)["p"] - d_obs
        (0.5 * (r * r).sum()).backward()

    ms_fb, ms_gb = _timed(torch, fwd_b200, 2), _timed(torch, grad_b200, 2)
    return {"reference_pytorch_gpu": {
        "forward_gcell_updates_per_s": units / (ms_f * 1e-3) / 1e9, "forward_ms": ms_f,
        "gradient_gcell_updates_per_s": units / (ms_g * 1e-3) / 1e9, "gradient_ms": ms_g,
        "nt": nt, "shots": S, "fd_order": 4, "checkpoint_segments": segments,
        "sample": "400x1200 grid, 30-cell PML, 32 shots, nt truncated to 100 (the reference has no 8th order)",
        "b200_same_inputs": {"forward_gcell_updates_per_s": units / (ms_fb * 1e-3) / 1e9, "forward_ms": ms_fb,
                             "gradient_gcell_updates_per_s": units / (ms_gb * 1e-3) / 1e9, "gradient_ms": ms_gb,
                             "fd_order": 4, "note": "acoustic_forward_kernel of this library, same arguments"}}}


def _model_kwargs(torch, wave, w, dev, vp=None):
    damp = torch.tensor(wave.bc_pml(w.nx, w.nz, w.dx, w.dx, w.nabc, float(w.vp.max()), False),
                        dtype=torch.float32, device=dev)
    return dict(nx=w.nx, nz=w.nz, dx=w.dx, dz=w.dx, nt=w.nt, dt=w.dt, nabc=w.nabc, free_surface=False,
                src_x=w.src_x, src_z=w.src_z, src_n=w.n_shots,
                src_v=torch.tensor(np.tile(w.wavelet, (w.n_shots, 1)), device=dev), rcv_x=w.rcv_x, rcv_z=w.rcv_z,
                rcv_n=w.rcv_x.size, damp=damp, vp=vp if vp is not None else torch.tensor(w.vp, device=dev),
                rho=torch.tensor(w.rho, device=dev))


def _timed(torch, fn, reps=1):
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def _plans_of(engine, ws):
    """The distinct plans (8th order, no free surface) of a list of workloads."""
    out = {}
    for w in ws:
        p = engine.get_plan(engine.Geometry(w.nz, w.nx, w.nabc, w.nt, float(w.dt), float(w.dx), 4, False),
                            w.src_x, w.src_z, w.rcv_x, w.rcv_z)
        out[id(p)] = p
    return list(out.values())


def _profiled(plans, fn):
    """Run fn with phase profiling on every plan; the summed phase split."""
    for p in plans:
        p.set_profiling(True)
    fn()
    tot = {}
    for p in plans:
        for k, v in p.profile().items():
            tot[k] = tot.get(k, 0) + v
        p.set_profiling(False)
    return tot


def batch_rates(torch, wave, synthetic, dev):
    """Batched engine (one launch per time step for all models of a batch):
    the 50 particles of 256 x 512 (8 shots, 2000 steps) and the 24 uneven
    models (128 x 256 .. 512 x 1024, 1000 .. 3000 steps, 4 .. 16 shots).
    Forward; gradient (forward + adjoint of 0.5 ||p||^2, fp24 imaging fields)
    by acoustic_gradient_batched, which applies the misfit between the
    forward and the adjoint and runs memory-sized sub-batches that keep
    every step's imaging fields; and, for comparison, the same gradient by
    autograd through acoustic_forward_batched, whose stores must all live
    until the backward, so the steps that do not fit are recomputed."""
    from geobrain_b200.wave import engine
    peak, _ = measured_peaks()
    out = {}
    for name, ws in (("ensemble_256x512_50particles", synthetic.ensemble_256x512()),
                     ("uneven_batch_24models", synthetic.uneven_batch())):
        units = sum(w.cell_updates() for w in ws)
        plans = _plans_of(engine, ws)

        def fwd():
            with torch.no_grad():
                wave.acoustic_forward_batched([_model_kwargs(torch, wave, w, dev) for w in ws], fd_order=8,
                                              want_energy=False, device=dev)

        def grad():
            ms = [_model_kwargs(torch, wave, w, dev) for w in ws]
            return wave.acoustic_gradient_batched(ms, lambda i, p: (0.5 * (p * p).sum(), p), fd_order=8,
                                                  device=dev, imaging_dtype="fp24")

        def grad_autograd():
            ms = [_model_kwargs(torch, wave, w, dev, torch.tensor(w.vp, device=dev, requires_grad=True)) for w in ws]
            outs = wave.acoustic_forward_batched(ms, fd_order=8, want_energy=False, device=dev, imaging_dtype="fp24")
            loss = sum(0.5 * (o["p"] * o["p"]).sum() for o in outs)
            loss.backward()
            return [m["vp"].grad for m in ms]

        ms_f = _timed(torch, fwd)
        ms_g = _timed(torch, grad)
        prof = _profiled(plans, grad)
        ms_a = _timed(torch, grad_autograd)
        prof_a = _profiled(plans, grad_autograd)
        b_grad = sum(w.cell_updates() * (56 + 16 / w.n_shots) for w in ws)
        b_fwd = sum(w.cell_updates() * (24 + 8 / w.n_shots) for w in ws)
        split = lambda p: {"phase_ms": {k: p[k] for k in ("forward_ms", "recompute_ms", "adjoint_ms")},
                           "phase_steps": {k: p[k] for k in ("forward_steps", "recompute_steps", "adjoint_steps")},
                           "launches": p["launches"]}
        out[name] = {"forward_gcell_updates_per_s": units / (ms_f * 1e-3) / 1e9, "forward_ms": ms_f,
                     "forward_frac": b_fwd / (ms_f * 1e-3) / 1e9 / peak,
                     "gradient_gcell_updates_per_s": units / (ms_g * 1e-3) / 1e9, "gradient_ms": ms_g,
                     "gradient_frac": b_grad / (ms_g * 1e-3) / 1e9 / peak,
                     "gradient": dict(split(prof), api="acoustic_gradient_batched (fused misfit, sub-batches, "
                                                          "no recompute)"),
                     "autograd_gradient_gcell_updates_per_s": units / (ms_a * 1e-3) / 1e9, "autograd_gradient_ms": ms_a,
                     "autograd_gradient": dict(split(prof_a), api="acoustic_forward_batched + loss.backward()"),
                     "models": len(ws), "cell_updates": units, "launch": "batched (one launch per step)"}
    return out


# snapshot format of the memory-capped run: 16 bits with one scale per
# snapshot field (fp16 keeps 11 significant bits; bf16's 8 miss the 1e-3 bar)
LARGE_SNAPSHOTS = "fp16"


def large_gradient_rate(torch, wave, synthetic, dev, cap_bytes=60 * 10**9, snapshot_dtype=LARGE_SNAPSHOTS):
    """1000 x 3000 (1080 x 3080 padded), 16 shots, 8000 steps, 8th order:
    gradient within a 60 GB device-memory cap, with 16-bit checkpoints (one
    scale per snapshot field), fp24 imaging fields, and as many cached steps
    as the cap leaves room for; then, untimed, the gradient error of that
    storage on a truncated problem with the same segment length."""
    w = synthetic.large_1000x3000()
    kw = _model_kwargs(torch, wave, w, dev)
    kw.pop("vp")
    vp0 = torch.tensor(w.vp, device=dev)
    from geobrain_b200.wave import engine
    torch.cuda.synchronize()
    base = torch.cuda.memory_allocated(dev)
    torch.cuda.reset_peak_memory_stats(dev)

    def grad():
        vp = vp0.detach().requires_grad_(True)
        out = wave.acoustic_forward_kernel(vp=vp, **kw, device=dev, fd_order=8, want_energy=False,
                                           snapshot_dtype=snapshot_dtype, imaging_dtype="fp24",
                                           memory_budget=cap_bytes)
        (0.5 * (out["p"] * out["p"]).sum()).backward()
        return vp.grad

    ms = _timed(torch, grad)
    peak = torch.cuda.max_memory_allocated(dev) - base
    geo = engine.Geometry(w.nz, w.nx, w.nabc, w.nt, float(w.dt), float(w.dx), 4, False)
    plan = engine.get_plan(geo, w.src_x, w.src_z, w.rcv_x, w.rcv_z)
    K = engine.choose_checkpoint_every(plan, 1, 0, snapshot_dtype, False, "fp24")
    del kw, vp0
    torch.cuda.empty_cache()
    check = large_gradient_check(torch, wave, synthetic, dev, K, (snapshot_dtype,) + tuple(
        f for f in ("fp24", "bf16", "fp16") if f != snapshot_dtype))
    return {"large_1000x3000_16shots_gradient": {
        "gcell_updates_per_s": w.cell_updates() / (ms * 1e-3) / 1e9, "ms": ms, "nt": w.nt, "shots": w.n_shots,
        "memory_cap_bytes": cap_bytes, "peak_bytes_above_inputs": int(peak), "checkpoint_every": K,
        "checkpoints": f"{snapshot_dtype}, one scale per (checkpoint, shot, field)" if snapshot_dtype in
        ("fp16", "bf16") else snapshot_dtype, "imaging": "fp24",
        "gradient_check": check}}


def rates_3d(torch, wave, dev, nz=200, ny=200, nx=200, shots=4, nt=200, nabc=20):
    """The 3-D path (acoustic_forward_kernel_3d, 4th order): forward and
    gradient (forward + adjoint of 0.5 ||p||^2; every step's imaging fields kept) on a
    200^3 model with a 20-cell PML and 4 shots, seeded random velocities."""
    rng = np.random.default_rng(0)
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
    units = shots * (nz + 2 * nabc) * (ny + 2 * nabc) * (nx + 2 * nabc) * nt

    def fwd():
        with torch.no_grad():
            wave.acoustic_forward_kernel_3d(vp=vp, **kw)

    def grad():
        v = vp.detach().requires_grad_(True)
        out = wave.acoustic_forward_kernel_3d(vp=v, **kw)
        (0.5 * (out["p"] * out["p"]).sum()).backward()

    ms_f, ms_g = _timed(torch, fwd, 2), _timed(torch, grad, 1)
    return {"3d_200x200x200_4shots": {"forward_gcell_updates_per_s": units / (ms_f * 1e-3) / 1e9,
                                      "forward_ms": ms_f, "gradient_gcell_updates_per_s": units / (ms_g * 1e-3) / 1e9,
                                      "gradient_ms": ms_g, "nt": nt, "fd_order": 4}}


if __name__ == "__main__":
    main()
