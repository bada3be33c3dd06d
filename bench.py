#!/usr/bin/env python
"""Benchmark of the INS2D explicit RK hot path on B200.

Metric: cell-updates/s per RK4 step including all Poisson solves
(Npx*Npy*steps / time), plus CG iterations per solve on the PCG path.

Default workload: decaying 2D turbulence on a periodic 2048x2048 uniform grid,
Re=2000, RK44, CFL 0.5, FFT pressure solve, FP64 (seeded random-phase
streamfunction IC, E(k) ~ k^4 exp(-2(k/10)^2), unit kinetic energy).  The
working set of a step (about 0.5 GB of FP64 fields, 32 MiB each) is larger
than the 126 MB L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload turb2048|turb2048_fp32|turb2048_pcg|turb2048_pcg_fp32|tg512|ldc64|ens256]
                  [--members M]

--impl reference times the reference algorithm's CPU restatement (the oracle
port; the MATLAB reference itself cannot run here) on the host cores.
Multi-GPU (torchrun): single-grid workloads run one independent replica per
rank (weak scaling, no data-path collective); the ensemble workload splits
its members over the ranks (strong scaling); time = max over ranks.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: (N, domain, Re, poisson, precision, description)
    "turb2048": dict(N=2048, L=1.0, Re=2000.0, poisson=6, precision="fp64", ic="turbulence",
                     desc="decaying 2D turbulence 2048x2048 periodic, Re=2000, RK44, CFL 0.5, FFT Poisson, FP64"),
    "turb2048_fp32": dict(N=2048, L=1.0, Re=2000.0, poisson=6, precision="fp32", ic="turbulence",
                          desc="decaying 2D turbulence 2048x2048, FP32 stencils + FP64 Poisson/projection"),
    "turb2048_pcg": dict(N=2048, L=1.0, Re=2000.0, poisson=4, precision="fp64", ic="turbulence", CG_acc=1e-10,
                         compare_plain=True,
                         desc="decaying 2D turbulence 2048x2048, PCG Poisson to 1e-10 with the default preconditioner "
                              "(fast diagonalization; on this periodic uniform grid its Fourier basis, the FFT "
                              "solve), FP64"),
    "turb2048_pcg_mg": dict(N=2048, L=1.0, Re=2000.0, poisson=4, precision="fp64", ic="turbulence", CG_acc=1e-10,
                            precond="mg",
                            desc="decaying 2D turbulence 2048x2048, PCG Poisson to 1e-10, multigrid-preconditioned, "
                                 "FP64"),
    "turb2048_pcg_fp32": dict(N=2048, L=1.0, Re=2000.0, poisson=4, precision="fp32", ic="turbulence", CG_acc=1e-10,
                              compare_plain=True,
                              desc="decaying 2D turbulence 2048x2048, FP32 stencils, PCG to 1e-10 with the default "
                                   "preconditioner, FP64 Poisson/projection"),
    "turb2048_pcg_fp32_learned": dict(N=2048, L=1.0, Re=2000.0, poisson=4, precision="fp32", ic="turbulence",
                                      CG_acc=1e-10, compare_plain=True,
                                      learned=dict(record_steps=12, pairs=60, train_steps=200, batch=2, lr=2e-3,
                                                   seed=0),
                                      desc="decaying 2D turbulence 2048x2048, FP32 stencils, PCG to 1e-10 with the "
                                           "default preconditioner started from the learned guess (CNN trained on "
                                           "the GPU on the first steps' solves), FP64 Poisson/projection"),
    "tg512": dict(N=512, L=2 * math.pi, Re=1e100, poisson=6, precision="fp64", ic="tg", dt=1e-3,
                  desc="inviscid Taylor-Green 512x512 periodic [0,2pi]^2, RK44 dt=1e-3, FFT Poisson, FP64"),
    "ldc64": dict(N=64, L=1.0, Re=1000.0, poisson=4, precision="fp64", ic="rest", dt=1e-3, CG_acc=1e-12,
                  desc="lid-driven cavity 64x64, Re=1000, RK44 dt=1e-3, PCG to 1e-12 with the default "
                       "preconditioner (fast diagonalization), FP64"),
    "ldc64_mg": dict(N=64, L=1.0, Re=1000.0, poisson=4, precision="fp64", ic="rest", dt=1e-3, CG_acc=1e-12,
                     precond="mg",
                     desc="lid-driven cavity 64x64, Re=1000, RK44 dt=1e-3, multigrid PCG to 1e-12, FP64"),
    "bfs1024": dict(N=1024, ic="bfs", Re=800.0, poisson=4, precision="fp64", dt=1e-3, CG_acc=1e-10,
                    desc="backward-facing step 1024x1024, x in [0,30], y in [-0.5,0.5], tanh-stretched 1.02, "
                         "inflow u=24y(0.5-y) for y>=0, outflow p=0, Re=800, RK44 with dt = min(1e-3, 0.7 x the "
                         "explicit stability limit on the smallest cells), PCG to 1e-10 with the default "
                         "preconditioner (fast diagonalization), FP64"),
    "bfs1024_mg": dict(N=1024, ic="bfs", Re=800.0, poisson=4, precision="fp64", dt=1e-3, CG_acc=1e-10, precond="mg",
                       desc="backward-facing step 1024x1024 as bfs1024, multigrid PCG to 1e-10, FP64"),
    "bfs1024_learned": dict(N=1024, ic="bfs", Re=800.0, poisson=4, precision="fp64", dt=1e-3, CG_acc=1e-10,
                            learned=dict(record_steps=24, pairs=120, train_steps=300, batch=4, lr=2e-3, seed=0),
                            desc="backward-facing step 1024x1024 (as bfs1024) with the learned initial guess: "
                                 "a 6-layer 32-channel BF16 CNN trained on the GPU on the (f, dp) pairs of the "
                                 "first steps' solves; PCG with the default preconditioner to the same 1e-10"),
    "turb2048_slab": dict(kind="slab", N=2048, L=1.0, Re=2000.0, poisson=6, precision="fp64", ic="turbulence",
                          desc="decaying 2D turbulence 2048x2048 periodic, Re=2000, RK44, CFL 0.5, FFT Poisson, FP64, "
                               "the one grid split into y-slabs over the ranks (halo exchanges and all-to-all "
                               "transposes over NCCL)"),
    "ens256": dict(kind="ensemble", n=256, sizes=(64, 96, 128, 192, 256), stretch=1.05, dt=5e-4, CG_acc=1e-10,
                   poisson=4, precision="fp64",
                   desc="ensemble of 256 cavity/channel flows, tanh-stretched 1.05, nx,ny in {64..256}, "
                        "Re U[100,5000], lid/inflow U[0.5,1.5], from rest, RK44 dt=5e-4, PCG to 1e-10, FP64; "
                        "members sharded over ranks longest-first; the batched solves use fast "
                        "diagonalization"),
    "ens256_mg": dict(kind="ensemble", n=256, sizes=(64, 96, 128, 192, 256), stretch=1.05, dt=5e-4, CG_acc=1e-10,
                      poisson=4, precision="fp64", precond="mg",
                      desc="ens256 with the members' multigrid preconditioner (solve form chosen by the tuner)"),
}

# Algorithmic DRAM bytes per pressure cell of one launch of each kernel
# family, averaged over the family's launches in an RK44 step with steady
# boundary conditions (each array read or written once per launch).
# FP64 storage:
#   stage:    stages 2-3 (V_s, Vn in; Wt, kV out: 64 each), stage 4 (V_s, Vn,
#             three earlier kV in; Wt out: 96)            -> 224 / 3 launches
#   residual: V, p in; w, kV_next out                      -> 56
#   project:  the first stage from the cached residual fused into its
#             projection (Vn, kV0, p in; V_s out: 56), stages 2-4 (Wt, dp in;
#             V out: 40 each)                              -> 176 / 4
#   poisson_fft: rows with the divergence fused in (W in 16, half spectrum out
#             8), columns (8 + 8), rows back (8 in, dp out 8; + 8 for the
#             accumulating additional solve)               -> (3*56 + 64) / 4
# FP32 storage of the stage quantities (FP32-stencil contexts; no launch for
# the cached first stage):
#   stage:    stages 2-3 (V_s 4+4 in, kV 8 out: 16 each), stage 4 (V_s 8, three
#             kV 24 in, Vtemp 8 out: 40)                   -> 72 / 3
#   residual: V 16, p 8 in; w 16, kV_next 8 out            -> 48
#   project:  Vn 16, Vtemp 8, dp 8 in; V_s 8 out (stages 1-3) or V 16 (stage 4)
#                                                          -> 168 / 4
#   poisson_fft: rows from Vn 16 + Vtemp 8 (stage solves) or w 16 (additional
#             solve) -> 3*64 + 64 over 4 solves
FAMILY_BYTES = {
    "fp64": {"stage": 224 / 3.0, "residual": 56.0, "project": 176 / 4.0, "poisson_fft": (3 * 56 + 64) / 4.0,
             "div": 24.0},
    "fp32": {"stage": 72 / 3.0, "residual": 48.0, "project": 168 / 4.0, "poisson_fft": 64.0, "div": 32.0},
}
# per RK44 step: all launches of the families above
STEP_BYTES = {"fp64": 224 + 56 + 176 + (3 * 56 + 64), "fp32": 72 + 48 + 168 + 4 * 64}
# the same step in the reference's operator decomposition (fused stage + divergence
# 88, projection 40, FFT solve 64 per stage, additional solve 40 + solve)
STEP_BYTES_REFERENCE_DECOMPOSITION = 808


def family_bytes_per_cell(fam, precision="fp64"):
    return FAMILY_BYTES[precision].get(fam)


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.out = tempfile.NamedTemporaryFile(prefix="clocks_", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "50"], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.close()
        rows = []
        with open(self.out.name) as fh:
            for line in fh:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.out.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if "Active" in r[5 + k] and "Not" not in r[5 + k]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def bfs_profile(y):
    """inflow above the step (y >= 0): u = 24 y (0.5 - y)"""
    y = np.asarray(y, dtype=np.float64)
    return np.where(y >= 0.0, 24.0 * y * (0.5 - y), 0.0)


def bfs_dt(x, y, Re, dt_max, umax=1.5, safety=0.7):
    """The backward-facing step's nominal dt = 1e-3 is beyond explicit RK4's stability limit
    on a 1024-cell unit height (diffusion: |lambda dt| = 4 dt (1/hx^2 + 1/hy^2)
    / Re must stay below 2.78, convection: umax dt (1/hx + 1/hy) below 2.83),
    so the step is the smaller of dt_max and 0.7 times those limits on the
    smallest cells."""
    hx, hy = float(np.min(np.diff(x))), float(np.min(np.diff(y)))
    lim_d = 2.78 / (4.0 / Re * (1.0 / hx ** 2 + 1.0 / hy ** 2))
    lim_c = 2.83 / (umax * (1.0 / hx + 1.0 / hy))
    return min(dt_max, safety * min(lim_d, lim_c))


def setup_case(wl, device=0):
    import ins2d_b200
    from ins2d_b200 import cases
    if wl["ic"] == "bfs":
        N = wl["N"]
        x = cases.tanh_grid(N, 0.0, 30.0, 1.02)
        y = cases.tanh_grid(N, -0.5, 0.5, 1.02)
        opts = ins2d_b200.Options(x, y, cases.BC_CHANNEL, Re=wl["Re"], poisson=wl["poisson"],
                                  CG_acc=wl.get("CG_acc", 1e-10), CG_maxit=50000, uBC=cases.channel_uBC(bfs_profile),
                                  RK="RK44", precision=wl["precision"], device=device,
                                  precond=wl.get("precond", "default"))
        V = np.r_[bfs_profile(opts.yu), np.zeros(opts.Nv)]
        V = opts.initial_projection(V, 0.0)
        return opts, V, bfs_dt(x, y, wl["Re"], wl["dt"])
    N, L = wl["N"], wl["L"]
    x = cases.uniform_grid(N, 0.0, L)
    if wl["ic"] == "rest":
        bc = cases.BC_CAVITY
        uBC = cases.lid_uBC(1.0, L)
    else:
        bc = cases.BC_PERIODIC
        uBC = None
    opts = ins2d_b200.Options(x, x.copy(), bc, Re=wl["Re"], poisson=wl["poisson"], CG_acc=wl.get("CG_acc", 1e-12),
                              CG_maxit=50000, uBC=uBC, RK="RK44", precision=wl["precision"], device=device,
                              precond=wl.get("precond", "default"))
    if wl["ic"] == "turbulence":
        V = cases.decaying_turbulence_ic(opts, k0=10.0, seed=2048)
        dt = cases.cfl_dt(opts, V, 0.5)
    elif wl["ic"] == "tg":
        V = cases.taylor_green(opts)
        dt = wl["dt"]
    else:
        V = np.zeros(opts.NV)
        dt = wl["dt"]
    return opts, V, dt


def setup_learned(opts, lw, Vd, pd, t, dt, stream, device):
    """Records the (f, dp) pairs of the first steps' PCG solves, trains the
    network on them on the GPU and attaches it as the initial guess.  Returns
    the time reached and a description of the training."""
    import torch
    from ins2d_b200 import learned
    f_buf, p_buf = learned.record_pairs(opts, lw["pairs"])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    _, _, rst = opts.time_ERK(Vd, pd, t, dt, nsteps=lw["record_steps"], return_stats=True)
    torch.cuda.synchronize()
    rec_s = time.perf_counter() - t0
    t += lw["record_steps"] * dt
    n = learned.recorded_pairs(opts)
    learned.stop_recording(opts)
    inp, tgt = learned.prepare_pairs(opts, f_buf[:n], p_buf[:n])
    del f_buf, p_buf
    torch.cuda.empty_cache()
    net = learned.ConvNet(device=device, seed=lw.get("seed", 0))
    net.set_stream(stream.cuda_stream)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    losses = learned.train(net, inp, None, steps=lw["train_steps"], batch=lw["batch"], lr=lw["lr"],
                           seed=lw.get("seed", 0), options=opts)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    del inp, tgt
    torch.cuda.empty_cache()
    learned.attach(opts, net)
    info = {"pairs": n, "record_steps": lw["record_steps"], "record_s": round(rec_s, 3),
            "record_cg_iters_per_solve": rst["iters_total"] / max(rst["n_solves"], 1),
            "train_steps": lw["train_steps"], "batch": lw["batch"], "train_s": round(train_s, 3),
            "loss_rel_first": float(np.mean(losses[:5])), "loss_rel_last": float(np.mean(losses[-10:]))}
    return t, info, net


def load_tensor_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["bf16_tflops"]), "measured bf16 burst (MEASURED_PEAKS.json)"
    except Exception:
        return 1590.0, "fallback"


def run_ours(args, wl, rank, world, local_rank):
    import torch
    import ins2d_b200
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    opts, V0, dt = setup_case(wl, device=local_rank)
    stream = torch.cuda.current_stream()
    opts.set_stream(stream.cuda_stream)
    Vd = torch.tensor(V0, dtype=torch.float64, device="cuda")
    pd = torch.zeros(opts.Np, dtype=torch.float64, device="cuda")
    pd = opts.pressure_additional_solve(Vd, pd, 0.0)  # p_initial (input_check.m:126-128)
    t = 0.0
    lw = wl.get("learned")
    learned_info = None
    if lw:
        t, learned_info, net = setup_learned(opts, lw, Vd, pd, t, dt, stream, local_rank)
    state0 = (Vd.clone(), pd.clone(), t) if lw else None
    # warm-up
    _, _, st = opts.time_ERK(Vd, pd, t, dt, nsteps=args.warmup, return_stats=True)
    t += args.warmup * dt
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)  # let nvidia-smi start sampling before the timed region
    opts.profile(False)  # resets launch counters
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    _, _, st = opts.time_ERK(Vd, pd, t, dt, nsteps=args.steps, return_stats=True)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    prof = opts.profile_read()
    launches = sum(n for _, n in prof.values())
    t += args.steps * dt
    if dist:
        dist.barrier()
    clk = clocks.stop()
    ms_max = ms
    if dist:
        tt = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms_max = float(tt.item())
    cells = opts.Npx * opts.Npy
    value = cells * args.steps * world / (ms_max / 1e3)

    # end to end through the public API with host buffers: every step copies
    # V and p from pinned host memory and reads them back
    hV = torch.empty(opts.NV, dtype=torch.float64, pin_memory=True)
    hp = torch.empty(opts.Np, dtype=torch.float64, pin_memory=True)
    hV.copy_(Vd.cpu())
    hp.copy_(pd.cpu())
    hVn, hpn = hV.numpy(), hp.numpy()
    from ins2d_b200 import _lib
    import ctypes
    lib = _lib.load()
    ss = _lib.StepStats()
    e_steps = max(2, min(args.steps, 20))
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0.record(stream)
    tw0 = time.perf_counter()
    for n in range(e_steps):
        rc = lib.ins2d_erk_step(opts._ctx, hVn.ctypes.data, hpn.ctypes.data, t + n * dt, dt, ctypes.byref(ss),
                                _lib.MEM_HOST)
        if rc:
            raise RuntimeError(opts._err())
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max(e0.elapsed_time(e1), (time.perf_counter() - tw0) * 1e3)
    if dist:
        tt = torch.tensor([e2e_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_ms = float(tt.item())
    e2e_value = cells * e_steps * world / (e2e_ms / 1e3)

    # the step with process_iteration.m's per-step diagnostics (one more F for
    # the residual, process_iteration.m:4, and check_conservation, :22): each
    # step followed by both calls on the device state
    nd = max(2, min(args.steps, 10))
    torch.cuda.synchronize()
    e0.record(stream)
    for n in range(nd):
        opts.time_ERK(Vd, pd, t + n * dt, dt, nsteps=1)
        opts.F(Vd, None, pd, t + (n + 1) * dt)
        opts.check_conservation(Vd, t + (n + 1) * dt)
    e1.record(stream)
    torch.cuda.synchronize()
    diag_ms = e0.elapsed_time(e1) / nd
    t += nd * dt
    diagnostics = {"steps": nd, "ms_per_step": round(diag_ms, 4), "value": cells / (diag_ms / 1e3),
                   "note": "each step an ins2d_erk_step call followed by ins2d_F (maxres) and "
                           "ins2d_conservation, as process_iteration.m runs them every step"}

    # per-family device time (a separate profiled run; events add a little overhead)
    nprof = max(2, min(args.steps, 10))
    opts.profile(True)
    opts.time_ERK(Vd, pd, t, dt, nsteps=nprof)
    fam = opts.profile_read()
    opts.profile(False)
    peak, peak_kind = load_peaks()
    fam_ms = {k: v[0] for k, v in fam.items()}
    dom = max(fam_ms, key=fam_ms.get)
    dom_launch_ms = fam[dom][0] / max(fam[dom][1], 1)
    fkey = "poisson_fft" if (dom == "poisson" and wl["poisson"] == 6) else dom
    prec = wl["precision"]
    bpc = family_bytes_per_cell(fkey, prec)
    roof = None
    if bpc is not None:
        if dom == "poisson":
            launch_ms = fam[dom][0] / max(nprof * 4, 1)  # one solve = 3 passes
        else:
            launch_ms = dom_launch_ms
        achieved = bpc * cells / (launch_ms / 1e3) / 1e9
        traffic = None
        tpath = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tpath):
            try:
                with open(tpath) as fh:
                    traffic = json.load(fh).get(args.workload, {}).get(fkey)
            except Exception:
                traffic = None
        per_family = {}
        for k, (fms, nl) in fam.items():
            kk = "poisson_fft" if (k == "poisson" and wl["poisson"] == 6) else k
            b = family_bytes_per_cell(kk, prec)
            if b is None or nl == 0 or fms <= 0:
                continue
            lms = fms / (nprof * 4) if k == "poisson" else fms / nl
            gbs = b * cells / (lms / 1e3) / 1e9
            per_family[kk] = {"ms_per_launch": round(lms, 5), "bytes_per_cell": b, "achieved_gbs": round(gbs, 1),
                              "frac": round(gbs / peak, 4)}
        step_ms = ms_max / args.steps
        roof = {"bound": "hbm", "kernel": fkey, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_kind": peak_kind, "traffic": traffic,
                "bytes_per_launch": bpc * cells, "launch_ms": round(launch_ms, 5),
                "family_ms_per_step": {k: round(v / nprof, 4) for k, v in fam_ms.items()},
                "families": per_family,
                "step": {"bytes_per_cell": STEP_BYTES[prec],
                         "achieved_gbs": round(STEP_BYTES[prec] * cells / step_ms / 1e6, 1),
                         "frac": round(STEP_BYTES[prec] * cells / step_ms / 1e6 / peak, 4),
                         "bytes_per_cell_reference_decomposition": STEP_BYTES_REFERENCE_DECOMPOSITION,
                         "frac_reference_decomposition":
                             round(STEP_BYTES_REFERENCE_DECOMPOSITION * cells / step_ms / 1e6 / peak, 4)}}
    # accuracy of this run: kinetic energy drift and divergence; for the FP32
    # stencil workload also the deviation from the FP64 path over the same steps
    total_steps = (lw["record_steps"] if lw else 0) + args.warmup + args.steps + nd + nprof
    acc = None
    if rank == 0:
        c0 = opts.check_conservation(torch.tensor(V0, dtype=torch.float64, device="cuda"), 0.0)
        c1 = opts.check_conservation(Vd, t)
        acc = {"steps": total_steps, "k0": c0[3], "k": c1[3],
               "energy_change_rel": (c1[3] - c0[3]) / c0[3] if c0[3] != 0 else None, "maxdiv": c1[0]}
        if wl["precision"] == "fp32":
            ref_wl = dict(wl, precision="fp64")
            o64, V64_0, _ = setup_case(ref_wl, device=local_rank)
            o64.set_stream(stream.cuda_stream)
            V64 = torch.tensor(V64_0, dtype=torch.float64, device="cuda")
            p64 = o64.pressure_additional_solve(V64, torch.zeros(o64.Np, dtype=torch.float64, device="cuda"), 0.0)
            o64.time_ERK(V64, p64, 0.0, dt, nsteps=(lw["record_steps"] if lw else 0) + args.warmup + args.steps)
            o64.time_ERK(V64, p64, 0.0, dt, nsteps=nd + nprof)
            k64 = o64.check_conservation(V64, t)[3]
            acc.update({"fp64_k": k64, "energy_vs_fp64_rel": abs(c1[3] - k64) / k64,
                        "velocity_l2_vs_fp64_rel": float(torch.linalg.norm(Vd - V64) / torch.linalg.norm(V64))})
            o64.close()
    # the plain FP64 PCG (Jacobi preconditioner) on the same case, same
    # tolerance: one timed step after one warm-up step
    plain = None
    if rank == 0 and wl.get("compare_plain"):
        pwl = dict(wl, precision="fp64", precond="jacobi")
        op, Vp0, _ = setup_case(pwl, device=local_rank)
        op.set_stream(stream.cuda_stream)
        Vp = torch.tensor(Vp0, dtype=torch.float64, device="cuda")
        pp = op.pressure_additional_solve(Vp, torch.zeros(op.Np, dtype=torch.float64, device="cuda"), 0.0)
        op.time_ERK(Vp, pp, 0.0, dt, nsteps=1)
        torch.cuda.synchronize()
        e0.record(stream)
        _, _, pst = op.time_ERK(Vp, pp, dt, dt, nsteps=1, return_stats=True)
        e1.record(stream)
        torch.cuda.synchronize()
        pms = e0.elapsed_time(e1)
        plain = {"precond": "jacobi", "dtype": "f64", "ms_per_step": pms,
                 "cg_iters_per_solve": pst["iters_total"] / max(pst["n_solves"], 1),
                 "value": cells / (pms / 1e3), "speedup_of_this_run": (cells / (pms / 1e3)) and value / (cells / (pms / 1e3))}
        op.close()
    # the learned guess's effect: the same steps from the same state without
    # the network (multigrid PCG from zero), and the network's own forward time
    if lw:
        from ins2d_b200 import learned
        tc = state0[2]
        learned.attach(opts, None)
        Vc, pc = state0[0].clone(), state0[1].clone()
        opts.time_ERK(Vc, pc, tc, dt, nsteps=args.warmup)
        torch.cuda.synchronize()
        e0.record(stream)
        _, _, wst = opts.time_ERK(Vc, pc, tc + args.warmup * dt, dt, nsteps=args.steps, return_stats=True)
        e1.record(stream)
        torch.cuda.synchronize()
        wms = e0.elapsed_time(e1)
        learned_info["without"] = {"ms_per_step": wms / args.steps, "value": cells * args.steps / (wms / 1e3),
                                   "cg_iters_per_solve": wst["iters_total"] / max(wst["n_solves"], 1)}
        learned_info["with"] = {"ms_per_step": ms_max / args.steps, "value": value,
                                "cg_iters_per_solve": st["iters_total"] / max(st["n_solves"], 1)}
        learned_info["speedup"] = learned_info["without"]["ms_per_step"] / learned_info["with"]["ms_per_step"]
        # forward pass of the network on one field of the grid (tensor-core layers)
        x_in = torch.randn(1, opts.Npy, opts.Npx, dtype=torch.float32, device="cuda")
        for _ in range(3):
            net.forward(x_in)
        nrep = 10
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(nrep):
            net.forward(x_in)
        e1.record(stream)
        torch.cuda.synchronize()
        fms = e0.elapsed_time(e1) / nrep
        flops = 2 * 9 * (1 * 32 + 4 * 32 * 32 + 32 * 1) * cells
        tpk = load_tensor_peak()
        learned_info["forward"] = {"ms": round(fms, 4), "flops": flops, "achieved_tflops": round(flops / fms / 1e9, 2),
                                   "peak_tflops": tpk[0], "peak_kind": tpk[1],
                                   "frac": round(flops / fms / 1e9 / tpk[0], 4),
                                   "note": "ms includes the host synchronisation of each ins2d_cnn_forward call"}
        del net
    # the configuration's target comparison (default workload only): FP32
    # stencils + learned guess against the default FP64 path at the same CG
    # residual 1e-10 (multigrid PCG), a few steps each
    target = None
    if rank == 0 and args.workload == "turb2048" and not args.no_target:
        target = target_comparison(local_rank, stream)
    # CPU baseline on rank 0 only at N=1
    cpu = None
    if world == 1 and rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_baseline(wl, budget_s=args.cpu_budget)
    res = {
        "metric": "cell-updates/s per RK4 step incl. Poisson solve",
        "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if wl["precision"] == "fp64" else "f32-stencil/f64-poisson", "data": "synthetic",
        "config": {"workload": args.workload, "desc": wl["desc"], "grid": [opts.Npx, opts.Npy], "dt": dt,
                   "cells": cells, "l2": "working set > 126 MB L2 (no flush)" if cells >= 1 << 20 else
                   "small grid: L2-resident", "parallelism": f"replicas{world}"},
        "cg_iters_per_solve": (st["iters_total"] / st["n_solves"]) if (st and st["n_solves"] and wl["poisson"] != 6)
        else None,
        "e2e": {"value": e2e_value, "unit": "cell-updates/s", "steps": e_steps,
                "h2d_bytes_per_step": 8 * (opts.NV + opts.Np), "d2h_bytes_per_step": 8 * (opts.NV + opts.Np)},
        "gpu_launches": launches,
        "roofline": roof,
        "cpu_baseline": cpu,
        "accuracy": acc,
        "with_process_iteration": diagnostics,
        "target": target,
        "plain_pcg": plain,
        "learned": learned_info,
        "clocks": clk,
    }
    if rank == 0:
        print(json.dumps(res), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def timed_steps(opts, Vd, pd, t, dt, n, stream):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    _, _, st = opts.time_ERK(Vd, pd, t, dt, nsteps=n, return_stats=True)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / n, st["iters_total"] / max(st["n_solves"], 1)


def target_comparison(device, stream, nsteps=4):
    """North-star comparison on the 2048^2 turbulence: the default FP64 path
    (PCG with the default preconditioner) against FP32 stencils and against
    FP32 stencils with the learned initial guess, every solve to the same
    relative residual 1e-10; the FP64 multigrid PCG for reference.
    Each form: one warm-up step, then nsteps timed steps from the same state;
    the network is trained first on the pairs of the FP32 run's first steps."""
    import torch
    out = {"workload": "decaying turbulence 2048x2048, PCG to 1e-10", "steps": nsteps}
    forms = (("fp64", "turb2048_pcg", None), ("fp64_multigrid", "turb2048_pcg_mg", None),
             ("fp32", "turb2048_pcg_fp32", None), ("fp32_learned", "turb2048_pcg_fp32_learned", "learned"))
    for name, wkey, kind in forms:
        wl = WORKLOADS[wkey]
        opts, V0, dt = setup_case(wl, device=device)
        opts.set_stream(stream.cuda_stream)
        Vd = torch.tensor(V0, dtype=torch.float64, device="cuda")
        pd = opts.pressure_additional_solve(Vd, torch.zeros(opts.Np, dtype=torch.float64, device="cuda"), 0.0)
        t = 0.0
        info = {}
        net = None
        if kind == "learned":
            t, linfo, net = setup_learned(opts, wl["learned"], Vd, pd, t, dt, stream, device)
            info = {"train_s": linfo["train_s"], "pairs": linfo["pairs"]}
        opts.time_ERK(Vd, pd, t, dt, nsteps=1)
        t += dt
        ms, it = timed_steps(opts, Vd, pd, t, dt, nsteps, stream)
        out[name] = dict(info, ms_per_step=round(ms, 3), cg_iters_per_solve=round(it, 2),
                         value=opts.Npx * opts.Npy / (ms / 1e3))
        if net is not None:
            from ins2d_b200 import learned
            learned.attach(opts, None)
            net.close()
        opts.close()
        torch.cuda.empty_cache()
    base = out["fp64"]["ms_per_step"]
    for name in ("fp64_multigrid", "fp32", "fp32_learned"):
        out[name]["speedup_vs_fp64"] = round(base / out[name]["ms_per_step"], 3)
    out["target_speedup"] = 2.0
    out["met"] = out["fp32_learned"]["speedup_vs_fp64"] >= 2.0
    return out


def run_slab(args, wl, rank, world, local_rank):
    """One grid split into y-slabs over the ranks (ins2d_b200/slab.py): each
    rank advances its rows; halos and the FFT's transposes move over NCCL.
    value = the grid's cell-updates / max-over-ranks time (strong scaling)."""
    import datetime
    import torch
    from ins2d_b200 import cases, slab
    from ins2d_b200.rk import getRKmethod
    torch.cuda.set_device(local_rank)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    N, L = wl["N"], wl["L"]
    V0, dt = periodic_case_host(wl)
    part = slab.SlabPartition(N, world, rank)
    rows = part.global_rows()
    dev = torch.device("cuda", local_rank)
    u = torch.tensor(V0[:N * N].reshape(N, N)[rows], device=dev)
    v = torch.tensor(V0[N * N:].reshape(N, N)[rows], device=dev)
    p = torch.zeros((part.nL, N), dtype=torch.float64, device=dev)
    ops = slab.DeviceSlabOps(N, N, L, L, wl["Re"], part, device=local_rank)
    A, b, c = getRKmethod("RK44")
    ex = slab.Exchange(part)
    erk = slab.SlabERK(ops, part, ex, A, b, c, solver="fft")
    stream = torch.cuda.current_stream()
    t = 0.0
    for n in range(args.warmup):
        erk.step(u, v, p, t, dt)
        t += dt
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for n in range(args.steps):
        erk.step(u, v, p, t, dt)
        t += dt
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    tt = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    ms_max = float(tt.item())
    cells = N * N
    value = cells * args.steps / (ms_max / 1e3)
    # end to end: each rank's slab from pinned host memory in, one step, back out
    I = part.interior()
    hu = torch.empty((part.n, N), dtype=torch.float64, pin_memory=True)
    hv = torch.empty_like(hu)
    hp = torch.empty_like(hu)
    hu.copy_(u[I].cpu())
    hv.copy_(v[I].cpu())
    hp.copy_(p[I].cpu())
    e_steps = max(2, min(args.steps, 5))
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0.record(stream)
    tw0 = time.perf_counter()
    for n in range(e_steps):
        u[I].copy_(hu, non_blocking=True)
        v[I].copy_(hv, non_blocking=True)
        p[I].copy_(hp, non_blocking=True)
        erk.step(u, v, p, t, dt)
        t += dt
        hu.copy_(u[I])
        hv.copy_(v[I])
        hp.copy_(p[I])
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max(e0.elapsed_time(e1), (time.perf_counter() - tw0) * 1e3)
    te = torch.tensor([e2e_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_ms = float(te.item())
    nbytes = 8 * 3 * part.n * N
    # divergence of the final field on this rank's rows, maximum over the ranks
    f = ops.div(u, v)
    md = torch.tensor([float(f[I].abs().max())], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(md, op=dist.ReduceOp.MAX)
    cpu = None
    if world == 1 and rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_baseline(WORKLOADS["turb2048"], budget_s=args.cpu_budget)
    res = {
        "metric": "cell-updates/s per RK4 step incl. Poisson solve", "value": value, "unit": "cell-updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "desc": wl["desc"], "grid": [N, N], "dt": dt, "cells": cells,
                   "rows_per_rank": part.counts, "l2": "working set > 126 MB L2 (no flush)",
                   "parallelism": f"y-slabs over {world} rank(s)"},
        "e2e": {"value": cells * e_steps / (e2e_ms / 1e3), "unit": "cell-updates/s", "steps": e_steps,
                "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes},
        # per RK4 step on each rank: 4 right-hand sides (F), 4 projections' gradients, 4 divergences, and
        # the 3 + 1 solves of three transform passes each (the rest are torch element-wise operations)
        "gpu_launches": args.steps * (4 + 4 + 4 + 4 * 3),
        "roofline": None,
        "cpu_baseline": cpu,
        "accuracy": {"maxdiv": float(md.item())},
        "clocks": clk,
    }
    if rank == 0:
        print(json.dumps(res), flush=True)
    ops.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_ensemble(args, wl, rank, world, local_rank):
    """The batching workload: a fixed ensemble of wl['n'] members split over
    the ranks (LPT by cells); each rank advances its share as one ensemble.
    value = all members' cell-updates / max-over-ranks time (strong scaling)."""
    import torch
    import ins2d_b200
    from ins2d_b200 import ensembles
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    members = ensembles.random_members(args.members or wl["n"], seed=4, sizes=wl["sizes"], stretch=wl["stretch"],
                                       CG_acc=wl["CG_acc"], precision=wl["precision"],
                                       precond=wl.get("precond", "default"))
    costs = [ensembles.member_cost(kw) for kw in members]
    mine = ensembles.lpt_partition(costs, world)[rank]
    t0 = time.perf_counter()
    ens = ins2d_b200.Ensemble([dict(members[m], device=local_rank) for m in mine])
    dt = wl["dt"]
    # members whose explicit RK4 limit is below dt advance with their own stable step
    reduced = 0
    for k, m in enumerate(mine):
        dtm = ensembles.stable_dt(members[m], members[m]["_U"])
        if dtm < dt:
            ens.set_member_dt(k, dtm)
            reduced += 1
    setup_s = time.perf_counter() - t0
    stream = torch.cuda.current_stream()
    ens.set_stream(stream.cuda_stream)
    cells = sum(costs[m] for m in mine)
    total_cells = sum(costs)
    ens.time_ERK(0.0, dt, args.warmup)  # includes the solve-shape tuning and the graph capture
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    stats = ens.time_ERK(args.warmup * dt, dt, args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    ms_max = ms
    if dist:
        tt = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms_max = float(tt.item())
    value = total_cells * args.steps / (ms_max / 1e3)
    # end to end: every member's state from pinned host memory in, one step, back out
    hostV = [torch.empty(ens.member(k).NV, dtype=torch.float64, pin_memory=True) for k in range(len(mine))]
    hostp = [torch.empty(ens.member(k).Np, dtype=torch.float64, pin_memory=True) for k in range(len(mine))]
    for k in range(len(mine)):
        V, p = ens.get_state(k)
        hostV[k].numpy()[:] = V
        hostp[k].numpy()[:] = p
    e_steps = 3
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0.record(stream)
    tw0 = time.perf_counter()
    for _ in range(e_steps):
        for k in range(len(mine)):
            ens.set_state(k, hostV[k].numpy(), hostp[k].numpy())
        ens.time_ERK(0.0, dt, 1)
        for k in range(len(mine)):
            ens.get_state(k, hostV[k].numpy(), hostp[k].numpy())
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max(e0.elapsed_time(e1), (time.perf_counter() - tw0) * 1e3)
    if dist:
        tt = torch.tensor([e2e_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_ms = float(tt.item())
    nbytes = sum(8 * (ens.member(k).NV + ens.member(k).Np) for k in range(len(mine)))
    local = [dict(s, cells=costs[m]) for s, m in zip(stats, mine)]
    all_stats = ensembles.gather_stats(local, mine, len(members)) if dist else local
    it_mean = sum(s["iters_total"] for s in all_stats) / max(sum(s["n_solves"] for s in all_stats), 1)
    it_max = max(s["iters_max"] for s in all_stats)
    # whole-step roofline in the CG-path decomposition (552 + 4 (16 + 88 iters)
    # B per cell and RK44 step: stages, projections and residual, plus the CG
    # vectors of each solve; the V-cycle's own traffic is not counted)
    peak, peak_kind = load_peaks()
    step_bpc = 552 + 4 * (16 + 88 * it_mean)
    ach = step_bpc * total_cells / (ms_max / args.steps / 1e3) / 1e9
    roof = {"bound": "hbm", "kernel": "whole RK44 step (CG-path decomposition)", "achieved": round(ach, 1),
            "peak": peak, "unit": "GB/s", "frac": round(ach / peak, 4), "peak_kind": peak_kind, "traffic": None,
            "bytes_per_cell": round(step_bpc, 1)}
    cpu = None
    if world == 1 and rank == 0 and not args.no_cpu_baseline:
        cpu = ensemble_cpu_baseline(wl)
    res = {
        "metric": "cell-updates/s per RK4 step incl. Poisson solve (sum over ensemble members)",
        "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "desc": wl["desc"], "members": len(members),
                   "members_this_rank": len(mine), "cells_total": total_cells, "dt": dt,
                   "l2": "working set > 126 MB L2 (no flush)", "parallelism": f"members sharded over {world} rank(s)",
                   "setup_s": round(setup_s, 1), "solve_shape": ens.solve_shape(),
                   "members_with_reduced_dt_this_rank": reduced},
        "cg_iters_per_solve": it_mean, "cg_iters_max": it_max,
        "e2e": {"value": total_cells * e_steps / (e2e_ms / 1e3), "unit": "cell-updates/s", "steps": e_steps,
                "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes},
        # per RK4 step: 2 walker launches (interior / boundary tiles) for 3 stages and the
        # residual, 1 cached first stage, 3 divergence + 3 solve launches for stages 2-4,
        # 4 projections, 1 divergence + 1 solve for the additional solve
        "gpu_launches": args.steps * 21,
        "roofline": roof,
        "cpu_baseline": cpu,
        "clocks": clk,
    }
    if rank == 0:
        print(json.dumps(res), flush=True)
    ens.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def cpu_model():
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def host_threads():
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)


def periodic_case_host(wl):
    """(V0, dt) of a periodic workload computed on the host alone: the same
    seeded spectral field (turbulence) or Taylor-Green field as the GPU arm."""
    from ins2d_b200 import cases
    N, L = wl["N"], wl["L"]
    if wl["ic"] == "turbulence":
        V = cases.decaying_turbulence_ic_host(N, L, k0=10.0, seed=2048)
        h = L / N
        dt = 0.5 * h / float(np.max(np.abs(V)))  # cases.cfl_dt
    else:
        x = cases.uniform_grid(N, 0.0, L)
        xp = (x[:-1] + x[1:]) / 2
        xu, yu = np.tile(x[:-1], N), np.repeat(xp, N)
        xv, yv = np.tile(xp, N), np.repeat(x[:-1], N)
        V = np.r_[np.sin(xu) * np.cos(yu), -np.cos(xv) * np.sin(yv)]
        dt = wl["dt"]
    return V, dt


CPU_SAMPLE_N = 256  # largest grid the scipy restatement of a PCG workload is timed on


def cpu_baseline(wl, budget_s=25.0, steps=None, warmup=1):
    """The reference algorithm on the host cores, on a bounded sample (RK44
    steps of the same workload from the same initial field).  Periodic FFT
    workloads: the OpenMP C restatement oracle/erk_periodic.c on all host
    threads (checked against the scipy restatement in
    tests/test_oracle_pins.py); other workloads: the scipy/numpy restatement
    (single-threaded sparse matvecs, cg.F's DIC-PCG in C).  steps: the timed
    step count (capped so the timed part stays near budget_s)."""
    from oracle import ins2d_ref as R
    from ins2d_b200 import cases
    if wl["ic"] == "bfs":
        return bfs_cpu_baseline(wl, budget_s, steps)
    N, L = wl["N"], wl["L"]
    if wl.get("poisson") == 6 and wl["ic"] in ("turbulence", "tg"):
        threads = host_threads()
        V, dt = periodic_case_host(wl)
        p = np.zeros(N * N)
        if warmup > 0:
            V, p = R.erk_periodic_c(V, p, N, N, L, L, wl["Re"], dt, warmup, threads=threads)
        t0 = time.perf_counter()
        V, p = R.erk_periodic_c(V, p, N, N, L, L, wl["Re"], dt, 1, threads=threads)
        t1 = time.perf_counter() - t0
        want = steps if steps is not None else 50
        n_more = max(0, min(want - 1, int(budget_s / max(t1, 1e-9))))
        t0 = time.perf_counter()
        if n_more:
            V, p = R.erk_periodic_c(V, p, N, N, L, L, wl["Re"], dt, n_more, threads=threads)
        el = t1 + (time.perf_counter() - t0)
        n = 1 + n_more
        return {"value": N * N * n / el, "unit": "cell-updates/s", "cores": threads, "kind": "port",
                "steps": n, "cpu_model": cpu_model(), "dt": dt,
                "sample": f"{n} RK44 step(s) (after {warmup} untimed) of the {N}x{N} periodic workload from its own "
                          f"initial field, with the OpenMP C restatement of the reference algorithm "
                          f"(oracle/erk_periodic.c, FFT pressure solve), {threads} threads"}
    if N > CPU_SAMPLE_N:
        # the single-threaded scipy restatement's DIC-PCG on a 2048^2 grid
        # takes minutes per step: the same case on a CPU_SAMPLE_N^2 grid
        res = cpu_baseline(dict(wl, N=CPU_SAMPLE_N), budget_s, steps, warmup)
        res["sample"] = (f"the {N}x{N} workload's case on a {CPU_SAMPLE_N}x{CPU_SAMPLE_N} grid (the size the "
                         f"single-threaded restatement finishes in seconds): " + res["sample"])
        return res
    x = cases.uniform_grid(N, 0.0, L)
    bc = cases.BC_CAVITY if wl["ic"] == "rest" else cases.BC_PERIODIC
    uBC = cases.lid_uBC(1.0, L) if wl["ic"] == "rest" else None
    poisson = 6 if wl["poisson"] == 6 else 4
    t0 = time.perf_counter()
    o = R.make_options(x, x.copy(), bc, Re=wl["Re"], poisson=poisson, CG_acc=wl.get("CG_acc", 1e-12),
                       CG_maxit=100000, uBC=uBC, RK="RK44")
    setup_s = time.perf_counter() - t0
    g = o.grid
    dt = wl.get("dt", 1e-4)
    if wl["ic"] == "rest":
        V = np.zeros(g.NV)
    elif wl["ic"] == "tg":
        V = np.r_[np.sin(g.xu) * np.cos(g.yu), -np.cos(g.xv) * np.sin(g.yv)]
    else:
        V, dt = periodic_case_host(wl)
    p = np.zeros(g.Np)
    for n in range(warmup):
        V, p = R.time_ERK(V, p, n * dt, dt, o)
    n = 0
    t0 = time.perf_counter()
    while True:
        V, p = R.time_ERK(V, p, n * dt, dt, o)
        n += 1
        el = time.perf_counter() - t0
        if (steps is not None and n >= steps) or el > budget_s or (steps is None and n >= 50):
            break
    return {"value": g.Npx * g.Npy * n / el, "unit": "cell-updates/s", "cores": 1, "kind": "port", "steps": n,
            "cpu_model": cpu_model(), "dt": dt,
            "sample": f"{n} RK44 step(s) (after {warmup} untimed) of the {N}x{N} workload with the scipy/numpy "
                      f"restatement (sparse matvecs single-threaded, cg.F's DIC-PCG in C; operator setup "
                      f"{setup_s:.1f}s excluded)"}


def bfs_cpu_baseline(wl, budget_s=25.0, steps=None, n_sample=128):
    """The scipy restatement (single-threaded sparse matvecs, cg.F's DIC-PCG
    in C) on a bounded sample of the backward-facing-step workload: the same
    case on a 128x128 grid (the 1024x1024 grid's DIC-PCG takes minutes per
    step on one core), from the projected inflow profile."""
    from oracle import ins2d_ref as R
    from ins2d_b200 import cases
    x = cases.tanh_grid(n_sample, 0.0, 30.0, 1.02)
    y = cases.tanh_grid(n_sample, -0.5, 0.5, 1.02)
    t0 = time.perf_counter()
    o = R.make_options(x, y, cases.BC_CHANNEL, Re=wl["Re"], poisson=4, CG_acc=wl.get("CG_acc", 1e-10),
                       CG_maxit=100000, uBC=cases.channel_uBC(bfs_profile), RK="RK44")
    setup_s = time.perf_counter() - t0
    g = o.grid
    V = R.initial_projection(np.r_[bfs_profile(g.yu), np.zeros(g.Nv)], 0.0, o)
    p = np.zeros(g.Np)
    dt = bfs_dt(x, y, wl["Re"], wl["dt"])
    n = 0
    t0 = time.perf_counter()
    while True:
        V, p = R.time_ERK(V, p, n * dt, dt, o)
        n += 1
        el = time.perf_counter() - t0
        if (steps is not None and n >= steps) or (steps is None and (el > budget_s or n >= 50)):
            break
    return {"value": g.Npx * g.Npy * n / el, "unit": "cell-updates/s", "cores": 1, "kind": "port",
            "sample": f"{n} RK44 step(s) of the backward-facing step on a {n_sample}x{n_sample} grid (the "
                      f"{wl['N']}x{wl['N']} workload's case at a size the single-threaded scipy restatement "
                      f"finishes in seconds; operator setup {setup_s:.1f}s excluded)"}


def ensemble_cpu_baseline(wl, nmembers=2, steps=2):
    """The scipy restatement on a bounded sample of the ensemble: the first
    members of the same seeded ensemble, a few RK44 steps each."""
    from oracle import ins2d_ref as R
    from ins2d_b200 import ensembles
    members = ensembles.random_members(nmembers, seed=4, sizes=wl["sizes"], stretch=wl["stretch"],
                                       CG_acc=wl["CG_acc"])
    cells, el = 0, 0.0
    for kw in members:
        o = R.make_options(kw["x"], kw["y"], kw["BC"], Re=kw["Re"], poisson=4, CG_acc=kw["CG_acc"],
                           CG_maxit=100000, uBC=kw["uBC"], RK="RK44")
        V, p = np.zeros(o.grid.NV), np.zeros(o.grid.Np)
        dt = min(wl["dt"], ensembles.stable_dt(kw, kw["_U"]))
        t0 = time.perf_counter()
        for n in range(steps):
            V, p = R.time_ERK(V, p, n * dt, dt, o)
        el += time.perf_counter() - t0
        cells += o.grid.Npx * o.grid.Npy * steps
    return {"value": cells / el, "unit": "cell-updates/s", "cores": 1, "kind": "port", "steps": steps,
            "cpu_model": cpu_model(),
            "sample": f"{steps} RK44 steps of each of the first {nmembers} members with the scipy/numpy "
                      f"restatement (cg.F's DIC-PCG in C, single-threaded)"}


def run_reference(args, wl, rank, world):
    """The reference algorithm's CPU restatement (the reference itself is
    MATLAB, not runnable here) on the same workload, metric and config as the
    GPU arm: args.warmup untimed steps, then args.steps timed steps (capped
    to --ref-budget seconds of timed work; the cap is stated in the line)."""
    if rank != 0:
        return
    if wl.get("kind") == "ensemble":
        cb = ensemble_cpu_baseline(wl)
        config = {"workload": args.workload, "desc": wl["desc"], "members": wl["n"],
                  "sample": cb["sample"]}
        steps = cb.get("steps")
    else:
        cb = cpu_baseline(wl, budget_s=args.ref_budget, steps=max(1, args.steps), warmup=args.warmup)
        steps = cb["steps"]
        N = wl["N"]
        cells = N * N
        config = {"workload": args.workload, "desc": wl["desc"], "grid": [N, N], "dt": cb.get("dt"),
                  "cells": cells, "l2": "working set > 126 MB L2 (no flush)" if cells >= 1 << 20 else
                  "small grid: L2-resident", "parallelism": "host threads"}
        if wl["ic"] == "bfs":
            config["sample"] = cb["sample"]
    res = {
        "impl": "reference", "metric": "cell-updates/s per RK4 step incl. Poisson solve", "value": cb["value"],
        "unit": "cell-updates/s", "n_gpus": world, "steps": steps, "warmup": args.warmup, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config,
        "steps_requested": args.steps,
        "cpu_baseline": cb,
        "e2e": {"value": cb["value"], "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(res), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="turb2048", choices=sorted(WORKLOADS))
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--ref-budget", type=float, default=150.0,
                    help="--impl reference: seconds of timed CPU work at most")
    ap.add_argument("--no-target", action="store_true",
                    help="skip the FP32 + learned vs FP64 multigrid comparison of the default workload")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--members", type=int, default=None, help="ensemble workloads: number of members")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    wl = WORKLOADS[args.workload]
    if args.impl == "reference":
        run_reference(args, wl, rank, world)
    elif wl.get("kind") == "ensemble":
        run_ensemble(args, wl, rank, world, local_rank)
    elif wl.get("kind") == "slab":
        run_slab(args, wl, rank, world, local_rank)
    else:
        run_ours(args, wl, rank, world, local_rank)


if __name__ == "__main__":
    main()
