#!/usr/bin/env python
"""Throughput benchmark of the PowerLLEL_Channel DNS time step on B200.

Metric: grid-points x steps per second of the full time step (RK2 stencils,
FFT + tridiagonal Poisson projection, bulk forcing, boundary updates and the
NaN/CFL/divergence checks every nt_check steps) on the Re_tau ~ 550 channel
768 x 384 x 256 (domain 2pi x pi x 2, tanh stretching 1.8, Re_b = 20000,
CFL-controlled dt with CFL 0.5), FP64, seeded laminar + noise initial field
generated on the device.  Every field (613 MB) is larger than the 126 MB L2,
so no L2 flush is needed between steps.  The line's "mixed" object reports
the mixed-precision form on the same workload (FP32 fields) with its
speed-up over the FP64 form and its 10-step error against it; its
"ensemble" object a batch of 16 uneven channels (64x48x48 to 256x192x128,
mixed form) stepped as one graph launch per ensemble step, split over the
GPUs by the cost model when N > 1; its "spinup" object the steps and
seconds to a stationary turbulent state at 256x192x128, Re_tau 180, from the
learned initialiser against the laminar fallbacks (rank 0).

  python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]

One process per GPU (torchrun for N > 1); each GPU runs an independent
replica of the channel (the single-channel path does not shard), so the
scaling is weak and no collective touches the data path: the ranks only meet
in a barrier and in the max-over-ranks reduction of the timed region.

``--impl reference`` times the reference's CPU path on all host cores, rank
0 only: the reference's own time-step modules, compiled from its sources for
the CPU over host stand-ins for SYCL (OpenMP), one-rank MPI and the oneMKL
DFT (``oracle/_ref``, built by ``oracle/reference_cpu``), or -- where that
build is absent -- the FP64 oracle restatement in ``oracle/``.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

WORKLOADS = {
    # Re_tau ~ 550 channel (the headline throughput configuration)
    "re550": dict(nx=768, ny=384, nz=256, lx=2 * math.pi, ly=math.pi, lz=2.0, stretch_ratio=1.8,
                  re=10000.0, dt=1e-3, cfl_target=0.5),
    # same physics on 512 x 256 x 128 (fields 138 MB, > L2): the ncu capture case
    "prof": dict(nx=512, ny=256, nz=128, lx=2 * math.pi, ly=math.pi, lz=2.0, stretch_ratio=1.8,
                 re=10000.0, dt=1e-3, cfl_target=0.5),
    # Re_tau ~ 180 channel, 128 x 64 x 64 (the reference's CPU-runnable case)
    "re180": dict(nx=128, ny=64, nz=64, lx=4 * math.pi, ly=2 * math.pi, lz=2.0, stretch_ratio=1.5,
                  re=2800.0, dt=2e-3, cfl_target=0.0),
}

# Algorithmic HBM bytes per grid point of each kernel of the fused FP64 step:
# every distinct array a kernel must read counted once, every array it writes
# counted once (halos and 1-D coefficients excluded).
KERNEL_BYTES_PER_POINT = {
    "rk1+bound(u1)": 48,          # read u,v,w; write u1,v1,w1
    "rk2+bound(u)": 72,           # read u1,v1,w1,u,v,w; write u,v,w
    "calcRHS+fft_x_fwd": 32,      # read u,v,w; write spectral array
    "fft_y_fwd": 16,              # spectral array in place
    "trid_z": 16,                 # spectral array in place (pivot table excluded)
    "fft_y_bwd": 16,
    "fft_x_bwd+bound(p)": 16,     # read spectral array; write p
    "correct+mean": 56,           # read p,u,v,w; write u,v,w
    "force+bound(u)": 16,         # read u; write u
}
STEP_BYTES_PER_POINT = sum(KERNEL_BYTES_PER_POINT.values())  # 288
# the mixed form stores every field in FP32 (half the bytes; the pivot table
# excluded, as above); its RK2 also sums the bulk mean and its correction
# applies the forcing, so it has no separate forcing pass
MIXED_BYTES_PER_POINT = {
    "rk1+bound(u1)": 24,          # read u,v,w; write u1,v1,w1
    "rk2+bound(u)+mean": 36,      # read u1,v1,w1,u,v,w; write u,v,w
    "calcRHS+fft_x_fwd": 16,      # read u,v,w; write spectral array
    "fft_y_fwd": 8,
    "trid_z": 8,
    "fft_y_bwd": 8,
    "fft_x_bwd+bound(p)": 8,
    "correct+force+bound(u)": 28,  # read p,u,v,w; write u,v,w
}
MIXED_STEP_BYTES_PER_POINT = sum(MIXED_BYTES_PER_POINT.values())  # 136


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_traffic(workload, form, kernel, npts):
    """ncu DRAM read+write bytes per launch of a step kernel: the committed
    bytes per point (from a capture of this workload, else of the 512x256x128
    case -- the traffic of these streaming kernels grows with the points)
    times the points of the workload.  Returns (bytes, source) or (None, None)."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
    except Exception:
        return None, None
    for wl in (workload, "prof"):
        bpp = d.get(wl, {}).get(form, {}).get(kernel)
        if bpp is not None:
            return bpp * npts, f"ncu capture of the {wl} workload, {bpp:.1f} B/pt"
    return None, None


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
            # the sampler is running before the timed region starts: its
            # samples from here on fall inside the region
            t0 = time.perf_counter()
            while not self.lines and time.perf_counter() - t0 < 5.0:
                time.sleep(0.01)
            self.lines.clear()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


class nvtx_range:
    """NVTX range around a timed region (lets a profiler select the step's
    kernels: ncu --nvtx --nvtx-include fp64_step/); a no-op without torch."""

    def __init__(self, name):
        self.name = name

    def __enter__(self):
        try:
            import torch
            torch.cuda.nvtx.range_push(self.name)
            self.ok = True
        except Exception:
            self.ok = False
        return self

    def __exit__(self, *exc):
        if self.ok:
            import torch
            torch.cuda.nvtx.range_pop()


def channel_params(wl, nt_check, precision="fp64", cfl_target=None):
    from powerllel_channel_sycl_b200 import make_params
    return make_params(
        nx=wl["nx"], ny=wl["ny"], nz=wl["nz"], lx=wl["lx"], ly=wl["ly"], lz=wl["lz"],
        mesh_type=1, stretch_func=0, stretch_ratio=wl["stretch_ratio"], re=wl["re"], u_ref=1.0,
        l_ref=1.0, dt=wl["dt"], nt_check=nt_check, cfl_limit=1.0, div_limit=1e-9,
        initial_field="poi", init_with_noise=1, noise_intensity=0.1, is_forced=[1, 0, 0],
        vel_force=[1.0, 0.0, 0.0],
        cfl_target=wl["cfl_target"] if cfl_target is None else cfl_target, precision=precision)


def run_mixed(args, wl, world, local, pg, fp64_ms):
    """The mixed-precision form on the same workload: throughput, per-kernel
    times, and its 10-step error against the FP64 form from the same initial
    field (fixed dt, so that both forms take identical steps)."""
    import torch
    from powerllel_channel_sycl_b200 import Channel

    npts = wl["nx"] * wl["ny"] * wl["nz"]
    ch = Channel(channel_params(wl, args.nt_check, precision="mixed"), device=local)
    ch.initFlow()
    ch.step(args.warmup)
    ch.sync()
    torch.cuda.synchronize(local)
    barrier(pg, local)
    with nvtx_range("mixed_step"):
        ms = ch.step_timed(args.steps)
    torch.cuda.synchronize(local)
    barrier(pg, local)
    ms_max = max_over_ranks(ms, pg, local)
    value = world * npts * args.steps / (ms_max / 1e3)
    ok, cfl, div = ch.check()
    tiles = dict(ch.fft_tiles, rk_kchunk=ch.rk_kchunk, rk2_carry=ch.rk2_carry)
    prof_steps = max(2, min(5, args.steps))
    prof = ch.profile_step(prof_steps)
    total = sum(prof.values())
    kernels = {k: {"ms": v / prof_steps, "share": v / total,
                   "gbs": MIXED_BYTES_PER_POINT[k] * npts / (v / prof_steps / 1e3) / 1e9}
               for k, v in prof.items()}
    ch.close()
    peak, peak_kind = load_peaks()
    dom = max(prof, key=prof.get)
    achieved = kernels[dom]["gbs"]
    traffic, traffic_src = load_traffic(args.workload, "mixed", dom, npts)

    # accuracy: 10 steps of both forms from the same laminar + noise field
    nerr = 10
    a = Channel(channel_params(wl, 0, precision="fp64", cfl_target=0.0), device=local)
    b = Channel(channel_params(wl, 0, precision="mixed", cfl_target=0.0), device=local)
    a.initFlow()
    b.initFlow()
    a.step(nerr)
    b.step(nerr)
    err = rel_errors(a, b)
    _, _, div_b = b.check()
    a.close()
    b.close()
    developed = (mixed_error_developed(wl, local, nerr, args.developed_steps)
                 if args.developed_steps > 0 else None)
    return {
        "value": value, "unit": "grid-pt*step/s", "ms_per_step": ms_max / args.steps,
        "speedup_vs_fp64": fp64_ms / ms_max, "dtype": "f32 fields, f64 scalars/reductions/trid",
        "step_roofline": {"bytes_per_point_step": MIXED_STEP_BYTES_PER_POINT,
                          "achieved_gbs": MIXED_STEP_BYTES_PER_POINT * value / world / 1e9,
                          "frac": MIXED_STEP_BYTES_PER_POINT * value / world / 1e9 / peak},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": traffic, "traffic_source": traffic_src,
                     "bytes_per_point": MIXED_BYTES_PER_POINT[dom]},
        "kernels": kernels,
        "checks": {"nan_free": ok, "cfl_max": cfl[0], "div_max": div[0]},
        "fft_tiles": tiles,
        "error_vs_fp64": {"steps": nerr, "dt": wl["dt"], "vel_rel_l2": err,
                          "div_max_mixed": div_b[0]},
        "error_vs_fp64_developed": developed,
    }


def rel_errors(a, b):
    """Relative L2 errors of b's u, v, w against a's (interiors), and of the
    plane-mean u profile (max over planes, relative to the profile's max)."""
    err = {}
    for name in "uvw":
        x = a.download(name)[1:-1, 1:-1, 1:-1]
        y = b.download(name)[1:-1, 1:-1, 1:-1]
        err[name] = float(np.linalg.norm((y - x).ravel()) / np.linalg.norm(x.ravel()))
        if name == "u":
            mx, my = x.mean(axis=(1, 2)), y.mean(axis=(1, 2))
            err["u_mean_profile_max_rel"] = float(np.max(np.abs(my - mx)) / np.max(np.abs(mx)))
        del x, y
    return err


def mixed_error_developed(wl, local, nerr, spin):
    """The mixed form's 10-step error against FP64 from a developed turbulent
    state of the same workload: laminar + noise + streamwise vortices
    (amplitude 0.15) spun up in the mixed form under CFL control until the
    flow is turbulent (Re_tau well above its laminar value), then the state
    copied into an FP64 and a fresh mixed context and both stepped nerr times
    with the last dt fixed."""
    from powerllel_channel_sycl_b200 import Channel
    prm = channel_params(wl, 50, precision="mixed")
    prm.init_vortex_amp = 0.15
    ch = Channel(prm, device=local)
    ch.initFlow()
    t0 = time.perf_counter()
    ch.step(spin)
    wall = time.perf_counter() - t0
    re_tau, dt = ch.re_tau(), ch.dt
    state = {name: ch.download(name) for name in "uvwp"}
    ch.close()
    out = {"spin_steps": spin, "spin_wall_s": wall, "re_tau": re_tau, "dt": dt, "steps": nerr}
    a = Channel(channel_params(wl, 0, precision="fp64", cfl_target=0.0), device=local)
    b = Channel(channel_params(wl, 0, precision="mixed", cfl_target=0.0), device=local)
    for c in (a, b):
        for name in "uvwp":
            c.upload(name, state[name])
        c.dt = dt
    del state
    a.step(nerr)
    b.step(nerr)
    out["vel_rel_l2"] = rel_errors(a, b)
    out["div_max_mixed"] = b.check()[2][0]
    a.close()
    b.close()
    return out


def cpu_reference_rate(wl, budget_s: float, max_steps: int, warmup: int):
    """The reference's CPU path on the host cores, in grid-pt*steps/s.

    Where the reference's own modules were built from its sources
    (oracle/_ref, test infrastructure: its mod_calcVel, mod_calcRHS,
    mod_updateBound, mod_poisson_solver, mod_fft, ... over host stand-ins for
    SYCL with OpenMP, one-rank MPI and the oneMKL DFT), those run main.cc's
    loop ("reference"); otherwise the oracle restatement does ("port").
    `warmup` untimed steps, then min(max_steps, what fits in budget_s) timed
    steps.  Returns (rate, steps, warmup, threads, kind)."""
    import oracle
    from oracle import reference_modules as refmod
    threads = os.cpu_count() or 1
    npts = wl["nx"] * wl["ny"] * wl["nz"]
    kw = dict(lx=wl["lx"], ly=wl["ly"], lz=wl["lz"], dt=wl["dt"], re=wl["re"],
              stretch_ratio=wl["stretch_ratio"])
    if os.path.exists(refmod.LIB_PATH):
        refmod.set_threads(threads)
        m = refmod.ReferenceModules(wl["nx"], wl["ny"], wl["nz"], **kw)
        m.init_flow("poi", noise_intensity=0.1)
        step = m.step
        kind = "reference"
    else:
        oracle.set_threads(threads)
        case = oracle.Case(wl["nx"], wl["ny"], wl["nz"], **kw)
        f = list(case.init_flow("poi", noise_intensity=0.1))
        f += [case.zeros(), case.zeros(), case.zeros(), case.zeros()]
        _ = case.ps
        step = lambda n: case.step(*f, nsteps=n)  # noqa: E731
        m, kind = None, "port"
    t_one = None
    for _ in range(max(0, warmup)):
        t0 = time.perf_counter()
        step(1)
        t_one = time.perf_counter() - t0
    if t_one is None:
        t0 = time.perf_counter()
        step(1)
        t_one = time.perf_counter() - t0
        warmup = 1
    nsteps = int(max(1, min(max_steps, budget_s // max(t_one, 1e-9))))
    t0 = time.perf_counter()
    step(nsteps)
    dt = time.perf_counter() - t0
    if m is not None:
        m.close()
    return npts * nsteps / dt, nsteps, warmup, threads, kind


def dist_setup(n_gpus):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        backend = "nccl" if _cuda_ok() else "gloo"
        if backend == "nccl":
            import torch
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
        pg = dist
    return rank, world, local, pg


def _cuda_ok():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def max_over_ranks(value: float, pg, local: int) -> float:
    if pg is None:
        return value
    import torch
    dev = torch.device("cuda", local) if _cuda_ok() else torch.device("cpu")
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg, local):
    if pg is not None:
        import torch
        if _cuda_ok():
            pg.barrier(device_ids=[local])
        else:
            pg.barrier()


def run_reference(args, wl, rank, world, pg):
    if rank != 0:
        return None
    warmup = max(args.warmup, 3)  # the GPU arm's warm-up
    rate, nsteps, warmup, threads, kind = cpu_reference_rate(
        wl, budget_s=args.ref_budget, max_steps=args.steps, warmup=warmup)
    npts = wl["nx"] * wl["ny"] * wl["nz"]
    what = ("the reference's own modules built from its sources for the CPU (SYCL kernels "
            "on OpenMP threads, one-rank MPI, the oneMKL DFT restated by a stand-in FFT)"
            if kind == "reference" else "the oracle restatement of the reference path")
    sample = (f"{nsteps} full FP64 steps (of {args.steps} requested, bounded by "
              f"{args.ref_budget:.0f} s) of the {wl['nx']}x{wl['ny']}x{wl['nz']} channel after "
              f"{warmup} warm-up steps, main.cc's loop by {what}, {threads} threads")
    line = {
        "impl": "reference",
        "metric": "grid-pts*steps/s", "value": rate, "unit": "grid-pt*step/s",
        "n_gpus": world, "steps": nsteps, "warmup": warmup,
        "ms_per_step": 1e3 * npts / rate, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args, wl),
        "cpu_baseline": {"value": rate, "unit": "grid-pt*step/s", "cores": threads, "kind": kind,
                         "sample": sample},
        "e2e": {"value": rate, "unit": "grid-pt*step/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "gpu_launches": 0,
    }
    return line


def workload_config(args, wl):
    return {"workload": (f"channel DNS step {wl['nx']}x{wl['ny']}x{wl['nz']}, "
                         f"Re_b={2 * wl['re']:.0f}, FP64 plain form"
                         + (f", CFL-controlled dt (CFL {wl['cfl_target']})" if wl["cfl_target"] else
                            f", dt={wl['dt']}")),
            "nx": wl["nx"], "ny": wl["ny"], "nz": wl["nz"], "precision": "fp64",
            "nt_check": args.nt_check, "parallelism": f"replicas x{args.gpus}",
            "l2": "fields (613 MB each) larger than L2; no flush"
            if wl["nx"] * wl["ny"] * wl["nz"] > 20_000_000 else "working set partly L2-resident"}


def ensemble_members(seed=3, n=16):
    """16 uneven channels: grids between 64x48x48 and 256x192x128 (2^a 3^b),
    Re_tau ~ U[120, 400] (re = (Re_tau / 0.09)^(1/0.88) / 2), independent
    seeds, mixed precision, CFL-controlled dt."""
    rng = np.random.default_rng(seed)
    out = []
    for m in range(n):
        nx = int(rng.choice([64, 96, 128, 192, 256]))
        ny = int(rng.choice([48, 64, 96, 128, 192]))
        nz = int(rng.choice([48, 64, 96, 128]))
        re_tau = float(rng.uniform(120.0, 400.0))
        out.append(dict(nx=nx, ny=ny, nz=nz, lx=4 * math.pi, ly=2 * math.pi, lz=2.0,
                        stretch_ratio=1.5, re=0.5 * (re_tau / 0.09) ** (1 / 0.88), dt=1e-4,
                        cfl_target=0.5, re_tau=re_tau))
    return out


def run_ensemble(args, world, rank, local, pg):
    """Batched ensemble: this rank's share of the 16 channels (placed by the
    cost model) stepped as one graph launch per ensemble step."""
    import torch
    from powerllel_channel_sycl_b200 import Ensemble
    from powerllel_channel_sycl_b200.ensemble import members_of_rank

    specs = ensemble_members()
    costs = [float(s["nx"] * s["ny"] * s["nz"]) for s in specs]
    mine = members_of_rank(costs, rank, world)
    ens_ntc = args.nt_check if args.ens_nt_check is None else args.ens_nt_check
    prms = [channel_params(specs[i], ens_ntc, precision="mixed") for i in mine]
    ens = Ensemble(prms, device=local)
    ens.initFlow()
    tune = ens.autotune(steps=5)
    # warm-up up to a check step, so that the timed steps run in whole check
    # blocks (one graph launch per nt_check steps, the checks inside it), and
    # through one such block at least
    ntc = ens_ntc if ens_ntc > 0 else 1
    ens.step(-(-max(args.warmup, 2 * ntc) // ntc) * ntc)
    # whole check periods, so that the timed steps carry their share of checks
    steps = -(-args.steps // ntc) * ntc
    torch.cuda.synchronize(local)
    barrier(pg, local)
    with nvtx_range("ensemble_step"):
        ms = ens.step_timed(steps)
    torch.cuda.synchronize(local)
    barrier(pg, local)
    ms_max = max_over_ranks(ms, pg, local)
    total_pts = sum(costs)
    value = total_pts * steps / (ms_max / 1e3)
    sched, groups, budgets = ens.schedule()
    seq = tune.get("sequential")
    mine_pts = sum(costs[i] for i in mine)
    out = {
        "value": value, "unit": "grid-pt*step/s", "ms_per_step": ms_max / steps,
        "steps": steps, "nt_check": ens_ntc, "members": len(specs), "members_this_rank": len(mine), "points": int(total_pts),
        "grids": [f"{s['nx']}x{s['ny']}x{s['nz']}" for s in specs],
        "dtype": "f32 fields (mixed form)", "scaling": "strong",
        "schedule": sched, "sm_budgets": budgets, "groups": groups,
        "autotune_ms_per_step": tune,
        "batch_choice": ens.batch_choice() if sched == "batched" else None,
        "speedup_vs_sequential": (seq / (ms / steps)) if seq else None,
        "sequential_value_this_rank": (mine_pts / (seq / 1e3)) if seq else None,
    }
    ens.close()
    return out


def run_spinup(args, local):
    """Spin-up to a stationary turbulent state at 256 x 192 x 128, Re_tau 180
    (mixed form, CFL 0.4): from the learned initialiser's proposal, from the
    laminar + noise + vortices fallback, and from the reference's laminar +
    noise recipe (capped at 7x the generator's steps; it relaminarises)."""
    from powerllel_channel_sycl_b200 import Channel
    from powerllel_channel_sycl_b200 import learned as L
    rt = 180.0
    spec = dict(nx=256, ny=192, nz=128, re=L.re_from_re_tau(rt))
    gen = L.load_weights(device=local)
    out = {"re_tau": rt, "grid": "256x192x128", "precision": "mixed", "cfl": 0.4,
           "criterion": "Re_tau and mean u profile over a 2000-step window within 1% of the "
                        "previous window's, Re_tau >= 0.75 x target"}
    runs = {}
    for method in ("generator", "vortices", "laminar_noise"):
        ch = Channel(L.channel_params_for(spec, vortices=0.15 if method == "vortices" else 0.0),
                     device=local)
        ch.initFlow()
        t0 = time.perf_counter()
        if method == "generator":
            gen.propose(ch, rt, seed=1)
        t_init = time.perf_counter() - t0
        cap = 60000 if method != "laminar_noise" else 7 * max(runs["generator"]["steps"] or 0, 2000)
        r = L.spinup(ch, cap, min_re_tau=0.75 * rt)
        runs[method] = {"steps": r["steps"], "steps_run": r["steps_run"],
                        "wall_s": r["wall_s"] + t_init, "re_tau_end": float(r["re_tau"][-1])}
        ch.close()
    gen.close()
    out["runs"] = runs
    g = runs["generator"]
    if g["steps"]:
        if runs["vortices"]["steps"]:
            out["steps_ratio_vs_vortices"] = runs["vortices"]["steps"] / g["steps"]
            out["wall_ratio_vs_vortices"] = runs["vortices"]["wall_s"] / g["wall_s"]
        lam = runs["laminar_noise"]
        # the laminar + noise run never became turbulent within its cap: a lower bound
        out["steps_ratio_vs_laminar_noise_at_least"] = (
            lam["steps_run"] / g["steps"] if lam["steps"] is None else lam["steps"] / g["steps"])
        out["wall_ratio_vs_laminar_noise_at_least"] = lam["wall_s"] / g["wall_s"]
    return out


def run_ours(args, wl, rank, world, local, pg):
    import torch  # noqa: F401  (device init; the library owns its stream)
    from powerllel_channel_sycl_b200 import Channel
    from powerllel_channel_sycl_b200._lib import lib
    import ctypes as C

    npts = wl["nx"] * wl["ny"] * wl["nz"]
    ch = Channel(channel_params(wl, args.nt_check), device=local)
    ch.initFlow()
    ch.step(args.warmup)
    ch.sync()
    torch.cuda.synchronize(local)
    barrier(pg, local)
    torch.cuda.synchronize(local)
    with ClockSampler(local) as clk, nvtx_range("fp64_step"):
        ms = ch.step_timed(args.steps)
    torch.cuda.synchronize(local)
    barrier(pg, local)
    ms_max = max_over_ranks(ms, pg, local)
    value = world * npts * args.steps / (ms_max / 1e3)
    ok, cfl, div = ch.check()  # NaN / CFL / divergence of the state after the timed steps
    tiles = dict(ch.fft_tiles, rk_kchunk=ch.rk_kchunk)

    # per-kernel device times of the same fused kernels (plain launches with
    # CUDA events between them on the library's stream)
    prof_steps = max(2, min(5, args.steps))
    prof = ch.profile_step(prof_steps)
    total = sum(prof.values())
    dom = max(prof, key=prof.get)
    dom_ms = prof[dom] / prof_steps
    peak, peak_kind = load_peaks()
    achieved = KERNEL_BYTES_PER_POINT[dom] * npts / (dom_ms / 1e3) / 1e9
    traffic, traffic_src = load_traffic(args.workload, "fp64", dom, npts)
    kernels = {k: {"ms": v / prof_steps, "share": v / total,
                   "gbs": KERNEL_BYTES_PER_POINT[k] * npts / (v / prof_steps / 1e3) / 1e9}
               for k, v in prof.items()}

    # end to end through the C ABI with host buffers: upload the state from
    # pinned host memory, K steps each followed by a device->host read of the
    # step's result (its bulk mean and forcing; the NaN/CFL/divergence check
    # runs inside the step every nt_check steps), download the final u, v, w, p
    nfield = (wl["nx"] + 2) * (wl["ny"] + 2) * (wl["nz"] + 2)
    L = lib()
    hbuf = {}
    for name in ("u", "v", "w", "p"):
        ptr = C.c_void_p()
        rc = L.plc_host_alloc(nfield * 8, C.byref(ptr))
        if rc != 0:
            raise RuntimeError("plc_host_alloc failed")
        hbuf[name] = ptr
    fid = {"u": 0, "v": 1, "w": 2, "p": 6}
    for name in ("u", "v", "w"):
        L.plc_download(ch._ctx, fid[name], hbuf[name])
    torch.cuda.synchronize(local)
    barrier(pg, local)
    t0 = time.perf_counter()
    for name in ("u", "v", "w"):
        rc = L.plc_upload(ch._ctx, fid[name], hbuf[name])
        assert rc == 0
    fm = (C.c_double * 3)()
    ff = (C.c_double * 3)()
    for _ in range(args.steps):
        ch.step(1)
        rc = L.plc_step_forcing(ch._ctx, fm, ff)  # device->host read of the step's result
        assert rc == 0
    for name in ("u", "v", "w", "p"):
        rc = L.plc_download(ch._ctx, fid[name], hbuf[name])
        assert rc == 0
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s, pg, local)
    for name in hbuf:
        L.plc_host_free(hbuf[name])
    e2e_value = world * npts * args.steps / e2e_s
    h2d = 3 * nfield * 8 / args.steps
    d2h = (4 * nfield * 8 + args.steps * 48) / args.steps

    line = {
        "metric": "grid-pts*steps/s", "value": value, "unit": "grid-pt*step/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args, wl),
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": traffic, "traffic_source": traffic_src,
                     "bytes_per_point": KERNEL_BYTES_PER_POINT[dom]},
        "step_roofline": {"bytes_per_point_step": STEP_BYTES_PER_POINT,
                          "achieved_gbs": STEP_BYTES_PER_POINT * value / world / 1e9,
                          "frac": STEP_BYTES_PER_POINT * value / world / 1e9 / peak},
        "kernels": kernels,
        "e2e": {"value": e2e_value, "unit": "grid-pt*step/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "steps": args.steps,
                "copies": ("u, v, w uploaded once and u, v, w, p downloaded once per run, "
                           f"amortised over {args.steps} steps; every step is followed by a "
                           "48-byte read of its forcing")},
        "gpu_launches": args.steps * ch.kernels_per_step + (args.steps // args.nt_check
                                                            if args.nt_check else 0),
        "clocks": clk.summary(),
        "checks": {"nan_free": ok, "cfl_max": cfl[0], "div_max": div[0], "dt": ch.dt},
        "fft_tiles": tiles,
    }
    ch.close()
    if not args.no_mixed:
        line["mixed"] = run_mixed(args, wl, world, local, pg, ms_max)
        line["gpu_launches"] += args.steps * len(MIXED_BYTES_PER_POINT)
    if not args.no_ensemble:
        ens = run_ensemble(args, world, rank, local, pg)
        line["ensemble"] = ens
        if ens["schedule"] == "batched":
            # per chain and step: RK1, RK2, forcing, Thomas sweep and correction,
            # plus one launch per line-length group of each transform (at most);
            # one check launch per check period
            g = ens["batch_choice"]["fft_groups"]
            per_step = ens["batch_choice"]["chains"] * (5 + g[0] + g[1] + 2 * g[2])
            line["gpu_launches"] += (ens["steps"] * per_step
                                     + ens["steps"] // max(ens["nt_check"], 1))
        else:
            line["gpu_launches"] += (ens["steps"] * ens["members_this_rank"]
                                     * len(MIXED_BYTES_PER_POINT))
    if rank == 0 and not args.no_spinup:
        line["spinup"] = run_spinup(args, local)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # 10 timed steps after 2 warm-up steps (bounded by --cpu-budget)
        rate, nsteps, cw, threads, kind = cpu_reference_rate(
            wl, budget_s=args.cpu_budget, max_steps=10, warmup=2)
        line["cpu_baseline"] = {
            "value": rate, "unit": "grid-pt*step/s", "cores": threads, "kind": kind,
            "sample": (f"{nsteps} full FP64 steps after {cw} warm-up steps of the same "
                       f"{wl['nx']}x{wl['ny']}x{wl['nz']} case by "
                       + ("the reference's own modules built for the CPU"
                          if kind == "reference" else "the oracle restatement")
                       + f" ({threads} threads)")}
    return line if rank == 0 else None


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawTextHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="re550")
    ap.add_argument("--nt-check", type=int, default=10)
    ap.add_argument("--ens-nt-check", type=int, default=None,
                    help="check period of the ensemble's channels (default: --nt-check; the "
                         "reference's template param.json uses 100)")
    ap.add_argument("--cpu-budget", type=float, default=60.0)
    ap.add_argument("--ref-budget", type=float, default=120.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true",
                    help="skip the mixed-precision measurement")
    ap.add_argument("--no-ensemble", action="store_true",
                    help="skip the 16-channel ensemble measurement")
    ap.add_argument("--no-spinup", action="store_true",
                    help="skip the learned-initialiser spin-up comparison")
    ap.add_argument("--developed-steps", type=int, default=4000,
                    help="spin-up steps of the developed state the mixed form's error is "
                         "measured from (0: skip)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    wl = WORKLOADS[args.workload]
    rank, world, local, pg = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            line = run_reference(args, wl, rank, world, pg)
        else:
            line = run_ours(args, wl, rank, world, local, pg)
        if line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
