"""Benchmark: coupled surface-subsurface flow steps per second on B200.

Workload (default): one 512x512x40 hillslope domain (10,485,760 cells),
mixed precision (FP32 inner Krylov iterations, FP64 refinement, FP64 closure
and mass accumulator), rain 20 mm/h for 2 h then 2 h recession, dt = 60 s;
the timed region is K time steps from the initial state (K = 240 is the whole
storm).  A "step" is one time step of the coupled model for the domain: the
Picard loop (assembly, persistent Krylov solve, convergence check), the step
epilogue, and the overland solve.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (launched by torchrun) every rank runs an independent replica of
the domain on its own GPU ("replicas only": the single-domain solve does not
shard); value is the aggregate over ranks, timed as the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-steps/s mixed vs FP64 on 1 B200 at <=1e-8 mass error; adjoint/fwd time"
UNIT = "cell-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=240)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nx", type=int, default=512)
    ap.add_argument("--nz", type=int, default=40)
    ap.add_argument("--fp64-steps", type=int, default=20)
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--adjoint-steps", type=int, default=120)
    ap.add_argument("--fd-steps", type=int, default=20)
    ap.add_argument("--ensemble-steps", type=int, default=120)
    ap.add_argument("--ensemble-halving-steps", type=int, default=4)
    ap.add_argument("--schedule-steps", type=int, default=10)
    ap.add_argument("--autotune", type=int, default=1)
    return ap.parse_args()


# ----------------------------------------------------------------- helpers
class ClockSampler:
    """nvidia-smi clock/throttle samples every 200 ms during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.lines = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic_ratio():
    """DRAM bytes per algorithmic byte of k_krylov, measured by ncu over every
    k_krylov launch of a short run of this workload (profiles/krylov_traffic.json);
    the traffic of a timed launch is this ratio times its algorithmic bytes."""
    p = os.path.join(ROOT, "profiles", "krylov_traffic.json")
    try:
        with open(p) as f:
            return json.load(f)
    except Exception:
        return None


def dist_init(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        import torch
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    """Max of a per-rank value over all ranks (device tensor under NCCL, host
    tensor under gloo)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(cells_per_rank, steps, ms, world):
    """Whole-job cell-steps/s of `world` independent replicas: all ranks'
    cells x steps over the slowest rank's time."""
    ms_max = max_over_ranks(ms, world)
    return world * cells_per_rank * steps / (ms_max / 1e3), ms_max


# ------------------------------------------------------------------ ours
def run_ours(args, world, rank, local):
    import torch
    import dhara_b200 as db
    from dhara_b200 import inputs

    torch.cuda.set_device(local)
    dom = inputs.mixed_512x512x40(nx=args.nx, ny=args.nx, nz=args.nz, nsteps=max(args.steps, 1))
    N = dom.ncells
    p = dom.params

    def fresh(precision=db.MIXED):
        q = type(p).from_buffer_copy(p)
        q.precision = precision
        s = db.Solver(q, device=local)
        s.load(dom)
        s.prepare()
        return s

    def timed(s, nsteps, graph=False, kernel_timing=False):
        stream = torch.cuda.ExternalStream(s.stream, device=local)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        s.synchronize()
        if kernel_timing:
            s.set_kernel_timing(True)
            s.reset_kernel_timing()
        lc0 = s.launch_count()
        barrier(world)
        torch.cuda.synchronize()
        e0.record(stream)
        s.step(nsteps, graph=graph)
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        barrier(world)
        ms = e0.elapsed_time(e1)
        return ms, s.launch_count() - lc0

    # warm-up on a separate handle (same shapes), then a fresh state for timing;
    # the block schedule is autotuned on the warm-up handle's state
    s = fresh()
    s.step(args.warmup)
    s.synchronize()
    launch_cfg = s.autotune(2) if args.autotune else s.launch_config()
    s.close()

    def fresh_tuned(precision=db.MIXED, fused=None):
        s_ = fresh(precision)
        s_.set_launch_config(launch_cfg["krylov_blocks_per_sm"], launch_cfg["overland_resident"],
                             launch_cfg["overland_blocks_per_sm"], launch_cfg["tile_shape"],
                             launch_cfg["fused_step"] if fused is None else fused)
        return s_

    s = fresh_tuned()
    clocks = ClockSampler(local)
    clocks.start()
    ms, launches = timed(s, args.steps)
    clk = clocks.stop()
    dg = s.diagnostics()
    s.close()
    value, ms_max = replica_throughput(N, args.steps, ms, world)
    # per-kernel times (the Krylov roofline) from the same steps run as a
    # launch per kernel: the fused step runs the same per-tile code, but one
    # launch cannot be timed phase by phase
    s = fresh_tuned(fused=0)
    ms_k, _ = timed(s, args.steps, kernel_timing=True)
    kn, kms = s.kernel_timing("krylov")
    kbytes, kiters = s.krylov_traffic()
    timing = {k: s.kernel_timing(k) for k in db.KERNELS}
    s.close()

    # FP64 solver on the same workload (bounded number of steps)
    fp64_value = None
    if args.fp64_steps > 0:
        s64 = fresh(db.FP64)
        s64.step(1)
        s64.synchronize()
        s64.close()
        s64 = fresh(db.FP64)
        ms64, _ = timed(s64, min(args.fp64_steps, args.steps))
        s64.close()
        ms64 = max_over_ranks(ms64, world)
        fp64_value = world * N * min(args.fp64_steps, args.steps) / (ms64 / 1e3)
    # the same mixed steps for comparison over the same horizon
    s2 = fresh_tuned()
    ms_h, _ = timed(s2, min(args.fp64_steps, args.steps))
    s2.close()
    ms_h = max_over_ranks(ms_h, world)
    mixed_same_horizon = world * N * min(args.fp64_steps, args.steps) / (ms_h / 1e3)
    # and with the constitutive closure in FP32 (closure_fp32; its parity
    # against the oracle is in error_vs_oracle)
    closure_fp32 = None
    if args.fp64_steps > 0:
        q4 = type(p).from_buffer_copy(p)
        q4.closure_fp32 = 1
        s4 = db.Solver(q4, device=local)
        s4.load(dom)
        s4.prepare()
        s4.set_launch_config(launch_cfg["krylov_blocks_per_sm"], launch_cfg["overland_resident"],
                             launch_cfg["overland_blocks_per_sm"], launch_cfg["tile_shape"], launch_cfg["fused_step"])
        ms_c, _ = timed(s4, min(args.fp64_steps, args.steps))
        dg4 = s4.diagnostics()
        s4.close()
        ms_c = max_over_ranks(ms_c, world)
        closure_fp32 = {"value": world * N * min(args.fp64_steps, args.steps) / (ms_c / 1e3),
                        "speedup_vs_fp64": None,
                        "mass_error_over_inflow": (dg4["storage_change_cum"] - (dg4["top_inflow_cum"] -
                                                   dg4["bottom_outflow_cum"])) / dg4["top_inflow_cum"]}

    # end to end through the public API: per step upload the step's rain field
    # from pinned host memory, advance, read back the ponded depth and the
    # diagnostics record.
    C = p.nx * p.ny
    e2e = None
    if args.e2e_steps > 0:
        s3 = fresh_tuned()
        q = type(p).from_buffer_copy(p)
        rain_pinned = torch.empty(C, dtype=torch.float64, pin_memory=True).numpy()
        pond_pinned = torch.empty(C, dtype=torch.float64, pin_memory=True).numpy()
        ne = min(args.e2e_steps, args.steps)
        # the rain field replaces the schedule: clear the schedule for this handle
        s3.set_rain_schedule(np.zeros(0))
        stream = torch.cuda.ExternalStream(s3.stream, device=local)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        barrier(world)
        torch.cuda.synchronize()
        e0.record(stream)
        t0 = time.perf_counter()
        for t in range(ne):
            rain_pinned[:] = dom.rain_mm[t]
            s3.upload("ppt", rain_pinned)
            s3.step(1)
            import ctypes as ct
            rc = db.lib().dhara_download(s3.h, 0, db._abi.F["ponding"],
                                         pond_pinned.ctypes.data_as(ct.POINTER(ct.c_double)), C)
            if rc != 0:
                raise RuntimeError(db.lib().dhara_last_error().decode())
            s3.diagnostics()
        e1.record(stream)
        e1.synchronize()
        wall = time.perf_counter() - t0
        barrier(world)
        ms_e = max_over_ranks(max(e0.elapsed_time(e1), wall * 1e3), world)
        s3.close()
        e2e = {"value": world * N * ne / (ms_e / 1e3), "unit": UNIT, "steps": ne,
               "h2d_bytes_per_step": C * 8, "d2h_bytes_per_step": C * 8 + 312,
               "path": "dhara_upload(ppt) + dhara_step(1) + dhara_download(ponding) + "
                       "dhara_get_diagnostics, pinned host buffers"}

    # roofline of the dominant kernel (the persistent Krylov solve)
    peak, peak_kind = measured_peak()
    # algorithmic bytes of the timed region only (the counter is cumulative
    # per handle and this handle was created fresh for the timed region)
    achieved = (kbytes / (kms / 1e3)) / 1e9 if kms > 0 else None
    ncu = ncu_traffic_ratio()
    traffic = None
    if ncu and kn > 0 and ncu.get("workload") == f"mixed_{p.nx}x{p.ny}x{p.nz}":
        traffic = ncu["dram_bytes_per_algorithmic_byte"] * kbytes / kn
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                "peak_source": f"{peak_kind} hbm_gbs", "kernel": "k_krylov<float>",
                "algorithmic_bytes_per_launch": kbytes / kn if kn else None,
                "avg_launch_ms": kms / kn if kn else None,
                "launches": kn, "share_of_step": kms / ms_k if ms_k else None,
                "timed_in": "launch-per-kernel run of the same steps (fused_step 0), %.2f ms/step" %
                            (ms_k / args.steps)}
    # the storm's Krylov work depends on the chaotic Picard trajectory, so the
    # kernel's speed is also given per inner (FP32 CG) iteration
    krylov_ms_per_inner = kms / kiters if kiters else None

    adjoint = run_adjoint(args, local) if args.adjoint_steps > 0 else None
    ensemble = run_ensemble(args, local, world, rank) if args.ensemble_steps > 0 else None
    ensemble_halving = (run_ensemble_halving(args, local, world, rank)
                        if args.ensemble_halving_steps > 0 else None)

    mass_err = dg["storage_change_cum"] - (dg["top_inflow_cum"] - dg["bottom_outflow_cum"])
    inflow = dg["top_inflow_cum"]
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 inner Krylov + f64 refinement/closure",
        "data": "synthetic (seeded GRF topography, lognormal Ks; no public dataset)",
        "config": {"workload": f"mixed_{p.nx}x{p.ny}x{p.nz}", "cells": N, "dt_s": p.dt,
                   "storm": "20 mm/h for 2 h then recession", "precision": "mixed",
                   "picard": "absolute 1e-6 m, max 10, am 0.25", "krylov_tol": p.krylov_tol,
                   "l2": "inputs larger than L2 (~0.8 GB working set per step)",
                   "parallelism": f"replicas x{world}"},
        "fp64_value": fp64_value, "mixed_same_horizon": mixed_same_horizon,
        "mixed_closure_fp32": (dict(closure_fp32, speedup_vs_fp64=closure_fp32["value"] / fp64_value)
                               if closure_fp32 and fp64_value else closure_fp32),
        "speedup_mixed_vs_fp64": (mixed_same_horizon / fp64_value) if fp64_value else None,
        "mass_error_over_inflow": mass_err / inflow if inflow else None,
        "picard_iters": dg["picard_iters_total"], "krylov_inner_iters": dg["krylov_iters_total"],
        "refine_cycles": dg["refine_iters_total"], "overland_iters": dg["overland_iters_total"],
        "krylov_ms_per_inner_iter": krylov_ms_per_inner,
        "krylov_solves_at_cap": dg["krylov_nonconverged"], "overland_solves_at_cap": dg["overland_nonconverged"],
        "picard_steps_at_cap": dg["picard_nonconverged"],
        "adjoint_over_forward": adjoint["adjoint_over_forward"] if adjoint else None,
        "adjoint": adjoint,
        "ensemble": ensemble,
        "ensemble_dt_halving": ensemble_halving,
        "kernel_ms": {k: v[1] for k, v in timing.items()},
        "gpu_launches": launches, "clocks": clk, "roofline": roofline, "e2e": e2e,
        "launch_config": launch_cfg,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(args)
        out["error_vs_oracle"] = error_vs_oracle(args, local)
    return out


# -------------------------------------------------------------- ensemble
def run_ensemble(args, local, world=1, rank=0):
    """256 independent domains of uneven size (16x16x20 .. 128x128x40), each
    with its own seeded topography, Ks field, van Genuchten parameters and
    rain, advanced together by one handle: every launch of a step covers all
    domains (the persistent solvers schedule their tiles), and the step is
    replayed from a CUDA graph.  Timed over the 120-step run after warm-up.
    With N ranks the domains are sharded over them (dhara_b200.ensemble: a
    greedy bin-pack on cell count, nothing exchanged while stepping); the time
    is the slowest rank's and the value counts every domain (the ensemble is
    fixed, so this is strong scaling)."""
    from dhara_b200 import ensemble as ens
    from dhara_b200 import inputs
    nsteps = args.ensemble_steps
    doms = inputs.ensemble(256, nsteps=max(nsteps, 1))
    cells = sum(d.ncells for d in doms)
    if args.warmup > 0:
        ens.run_sharded(doms, args.warmup, rank, world, device=local)
    barrier(world)
    ms, launches, diags = ens.run_sharded(doms, nsteps, rank, world, device=local, autotune=2 if args.autotune else 0)
    ms_max = max_over_ranks(ms, world)
    # the two step schedules on the same first steps: one launch per subsurface
    # step (fused) and a launch per kernel
    schedules = {}
    if world == 1 and args.schedule_steps > 0:
        import torch
        import dhara_b200 as db
        for fused in (1, 0):
            s = db.Solver([d.params for d in doms], device=local)
            for i, d in enumerate(doms):
                s.load(d, i)
            s.prepare()
            c = s.launch_config()
            s.set_launch_config(c["krylov_blocks_per_sm"], c["overland_resident"], c["overland_blocks_per_sm"],
                                fused_step=fused)
            stream = torch.cuda.ExternalStream(s.stream, device=local)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            s.synchronize()
            n0 = s.launch_count()
            e0.record(stream)
            s.step(args.schedule_steps, graph=True)
            e1.record(stream)
            e1.synchronize()
            schedules["fused_step" if fused else "launch_per_kernel"] = {
                "ms_per_step": e0.elapsed_time(e1) / args.schedule_steps,
                "launches_per_step": (s.launch_count() - n0) / args.schedule_steps}
            if not fused:
                # where a step's time goes: the same steps again with per-kernel events
                s.set_kernel_timing(True)
                s.reset_kernel_timing()
                s.step(args.schedule_steps)
                s.synchronize()
                schedules["kernel_ms_per_step"] = {k: s.kernel_timing(k)[1] / args.schedule_steps
                                                   for k in db.KERNELS if s.kernel_timing(k)[0]}
            s.close()
        schedules["steps"] = args.schedule_steps
    worst_mass = 0.0
    kry_nc = olf_nc = solves = 0
    runaway = 0
    for i in range(len(doms)):
        dg = diags[i]
        if dg.get("psi_abs_max", 0.0) > 1e3:
            runaway += 1
        inflow = dg["top_inflow_cum"]
        if inflow:
            worst_mass = max(worst_mass, abs(dg["storage_change_cum"] - (inflow - dg["bottom_outflow_cum"])) / inflow)
        kry_nc += dg["krylov_nonconverged"]
        olf_nc += dg["overland_nonconverged"]
        solves += dg["picard_iters_total"]
    return {"workload": "ensemble_256_domains_16x16x20_to_128x128x40", "domains": len(doms), "cells": cells,
            "steps": nsteps, "ms_per_step": ms_max / nsteps, "value": cells * nsteps / (ms_max / 1e3),
            "unit": "cell-steps/s", "graph": True, "ranks": world,
            "scaling": "strong" if world > 1 else None,
            "shard_balance": ens.balance([d.ncells for d in doms], world),
            "gpu_launches": launches, "gpu_launches_note": "this rank's" if world > 1 else None,
            "launches_per_step": launches / nsteps if nsteps else None,
            "launch_config": diags[0].get("launch_config"),
            "worst_mass_error_over_inflow": worst_mass, "subsurface_solves": solves,
            "subsurface_solves_at_cap": kry_nc, "overland_solves_at_cap": olf_nc,
            "picard_steps_at_cap": sum(diags[i]["picard_nonconverged"] for i in range(len(doms))),
            "domain_steps": len(doms) * nsteps,
            "domains_with_abs_psi_above_1e3_m": runaway,
            "schedules": schedules,
            "note": "the reference's modified Picard iteration diverges on most of these rain-on-dry-soil domains, "
                    "in the oracle exactly as here; the rate measures the path's work, not a physical result"}


def run_ensemble_halving(args, local, world=1, rank=0):
    """The same 256 domains with time-step halving (dt_halvings 6: a step
    whose Picard iteration does not converge is redone as two half steps,
    down to dt/64), the opt-in converging variant of the reference's scheme,
    over the first steps (a bounded sample: the Picard iteration of the
    saturated zone stalls at any step length in many of these domains, so
    most of their sub-steps end at the smallest length).  The rate counts full
    steps; the sub-steps and all attempts (undone ones included) are reported
    beside it."""
    from dhara_b200 import ensemble as ens
    from dhara_b200 import inputs
    nsteps = args.ensemble_halving_steps
    doms = inputs.ensemble(256, nsteps=max(nsteps, 1))
    for d in doms:
        d.params.dt_halvings = 6
    cells = sum(d.ncells for d in doms)
    barrier(world)
    ms, launches, diags = ens.run_sharded(doms, nsteps, rank, world, device=local, autotune=0)
    ms_max = max_over_ranks(ms, world)
    worst_mass = 0.0
    runaway = capped = sub = att = 0
    for i in range(len(doms)):
        dg = diags[i]
        runaway += dg.get("psi_abs_max", 0.0) > 1e3
        capped += dg["picard_nonconverged"]
        sub += dg["substeps_total"]
        att += dg["step_attempts_total"]
        inflow = dg["top_inflow_cum"]
        if inflow:
            worst_mass = max(worst_mass, abs(dg["storage_change_cum"] - (inflow - dg["bottom_outflow_cum"])) / inflow)
    return {"workload": "ensemble_256_domains_dt_halving_6", "domains": len(doms), "cells": cells,
            "steps": nsteps, "ms_per_step": ms_max / nsteps, "value": cells * nsteps / (ms_max / 1e3),
            "unit": "cell-steps/s (full steps)", "ranks": world, "domain_steps": len(doms) * nsteps,
            "substeps_total": sub, "step_attempts_total": att, "picard_steps_at_cap": capped,
            "domains_with_abs_psi_above_1e3_m": runaway, "worst_mass_error_over_inflow": worst_mass,
            "gpu_launches": launches}


# --------------------------------------------------------------- adjoint
def run_adjoint(args, local):
    """Calibration gradient on the 128x128x30 domain: the loss is the misfit
    of the top three layers' moisture and of the outflow into the boundary
    ring against a seeded target run with perturbed log Ks; the gradient with
    respect to per-cell log Ks, alpha and n comes from dhara_adjoint with a
    checkpoint every 10 steps.  Reports the gradient's wall time over the
    forward run's (medians of three runs each), and central differences on
    random cells over the run's first steps (fd_check)."""
    import dhara_b200 as db
    from dhara_b200 import inputs
    nsteps = args.adjoint_steps
    dom = inputs.adjoint_128x128x30(nsteps=max(nsteps, 1))
    p = dom.params
    C = p.nx * p.ny

    def solver(d):
        s = db.Solver(d.params, device=local)
        s.load(d)
        s.prepare()
        return s

    # target: the same domain with log Ks perturbed by 0.3 N(0, 1)
    rng = np.random.default_rng(11)
    tgt = inputs.Domain(params=p, fields={k: v.copy() for k, v in dom.fields.items()},
                        int_fields=dom.int_fields, rain_mm=dom.rain_mm)
    tgt.fields["ksat"] = tgt.fields["ksat"] * np.exp(0.3 * rng.standard_normal(dom.ncells))
    s = solver(tgt)
    th_t = np.zeros((nsteps, 3, C))
    q_t = np.zeros(nsteps)
    prev = s.diagnostics()["overland_boundary_out_cum"]
    for t in range(nsteps):
        s.step(1)
        th_t[t] = s.download("theta")[:3 * C].reshape(3, C)
        cur = s.diagnostics()["overland_boundary_out_cum"]
        q_t[t] = cur - prev
        prev = cur
    s.close()

    def timed_call(fn):
        import torch
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = fn()
        torch.cuda.synchronize()
        return out, time.perf_counter() - t0

    s = solver(dom)   # warm-up of both paths on a short horizon
    s.adjoint(th_t[:2], q_t[:2], 2, checkpoint_every=1)
    s.close()
    s = solver(dom)
    _, t_step = timed_call(lambda: s.step(nsteps))
    s.close()
    # forward-only and gradient runs alternate, three of each; the medians
    # are reported (single wall-clock runs vary by up to 25 % on a shared box)
    t_fwds, t_grads = [], []
    for _ in range(3):
        s = solver(dom)
        loss_fwd, t = timed_call(lambda: s.adjoint(th_t, q_t, nsteps, checkpoint_every=10, gradients=False))
        t_fwds.append(t)
        s.close()
        s = solver(dom)
        (loss, g_lk, g_al, g_n), t = timed_call(lambda: s.adjoint(th_t, q_t, nsteps, checkpoint_every=10))
        t_grads.append(t)
        s.close()
    t_fwd, t_grad = float(np.median(t_fwds)), float(np.median(t_grads))
    s = solver(dom)
    s.set_kernel_timing(True)
    s.adjoint(th_t, q_t, nsteps, checkpoint_every=10)
    breakdown = {k: s.kernel_timing(k)[1] for k in db.KERNELS}
    s.close()
    fd = fd_check(dom, th_t, q_t, min(nsteps, args.fd_steps), local) if args.fd_steps > 0 else None
    return {"workload": f"adjoint_{p.nx}x{p.ny}x{p.nz}", "steps": nsteps, "checkpoint_every": 10,
            "precision": "mixed", "loss": loss, "loss_forward_only": loss_fwd,
            "forward_s": t_fwd, "forward_step_only_s": t_step, "gradient_s": t_grad,
            "forward_s_runs": t_fwds, "gradient_s_runs": t_grads,
            "adjoint_over_forward": t_grad / t_fwd, "gradient_kernel_ms": breakdown,
            "grad_norm": {"log_ks": float(np.linalg.norm(g_lk)), "alpha": float(np.linalg.norm(g_al)),
                          "n": float(np.linalg.norm(g_n))},
            "fd_check": fd}


def fd_check(dom, th_t, q_t, nsteps, local, ncells=32, steps=(1e-4, 1e-5, 1e-6)):
    """Central differences of the FP64 loss on `ncells` random cells (log Ks)
    and 8 each for alpha and n, over the first `nsteps` steps of the
    calibration run, against the FP64 adjoint gradient of the same run.  A
    difference counts only for a step h whose +h and -h runs took every
    branch of the unperturbed run (dhara_diagnostics.branch_signature: the
    top-flux selection, ponding and depth clips, Manning's wet test and
    saturation are switches of the reference scheme, where the loss is not
    differentiable)."""
    import dhara_b200 as db
    from dhara_b200 import inputs
    p = type(dom.params).from_buffer_copy(dom.params)
    p.precision = db.FP64
    # the loss's switches (not saturation: theta and K are continuous there) and the
    # overland iteration counts (a CG stopped at another iteration is another map)
    p.record_branches = 1 | 2 | 4 | 8 | 32 | 64
    p.krylov_tol, p.krylov_maxiter, p.overland_tol, p.overland_maxiter = 1e-13, 5000, 1e-12, 50000
    d = inputs.Domain(params=p, fields=dom.fields, int_fields=dom.int_fields, rain_mm=dom.rain_mm)
    th, q = th_t[:nsteps], q_t[:nsteps]

    def run(dd, gradients):
        s = db.Solver(dd.params, device=local)
        s.load(dd)
        s.prepare()
        out = s.adjoint(th, q, nsteps, checkpoint_every=5, gradients=gradients)
        sig = s.diagnostics()["branch_signature"]
        s.close()
        return out, sig

    (L, g_lk, g_al, g_n), base = run(d, True)
    rng = np.random.default_rng(2024)
    out = {"steps": nsteps, "precision": "fp64", "solves": "3D 1e-13, overland 1e-12", "h_tried": list(steps),
           "rule": "accepted h: +h and -h runs keep every branch of the unperturbed run; "
                   "error relative to |fd| where |fd| >= 1e-3 max|g|, else relative to max|g|"}
    for name, g, field, n in (("log_ks", g_lk, "ksat", ncells), ("alpha", g_al, "alpha", 8), ("n", g_n, "nvg", 8)):
        scale = float(np.max(np.abs(g)))
        rows = []
        for c in rng.choice(d.ncells, n, replace=False):
            c = int(c)
            row = {"cell": c, "adjoint": float(g[c]), "h": None, "fd": None, "err": None}
            for h in steps:
                vals, sigs = [], []
                for sgn in (1, -1):
                    f = {k: v.copy() for k, v in d.fields.items()}
                    if field == "ksat":
                        f["ksat"][c] *= np.exp(sgn * h)
                    else:
                        f[field] = f.get(field, np.full(d.ncells, p.alpha if field == "alpha" else p.n)).copy()
                        f[field][c] += sgn * h
                    dd = inputs.Domain(params=p, fields=f, int_fields=d.int_fields, rain_mm=d.rain_mm)
                    (Lh, sig) = run(dd, False)
                    vals.append(Lh)
                    sigs.append(sig)
                if sigs[0] == base and sigs[1] == base:
                    fdv = (vals[0] - vals[1]) / (2 * h)
                    row.update(h=h, fd=fdv,
                               err=abs(g[c] - fdv) / (abs(fdv) if abs(fdv) >= 1e-3 * scale else scale))
                    break
            rows.append(row)
        acc = [r for r in rows if r["h"] is not None]
        out[name] = {"cells": n, "accepted": len(acc), "worst_err": max((r["err"] for r in acc), default=None),
                     "within_1e-4": sum(1 for r in acc if r["err"] <= 1e-4), "rows": rows}
    return out


# ------------------------------------------------------------ CPU oracle
CPU_PATCH = 64


def cpu_sample_domain(args, n=CPU_PATCH, nsteps=None):
    """The bounded CPU sample: the same physics, solver settings and forcing on
    an n x n patch (same nz) of the benchmark domain's configuration."""
    from dhara_b200 import inputs
    return inputs.mixed_512x512x40(nx=n, ny=n, nz=args.nz, precision=0,
                                   nsteps=nsteps or max(args.steps, 8))


def patch_name(d):
    return f"mixed_patch_{d.params.nx}x{d.params.ny}x{d.params.nz}"


def cpu_baseline(args, sample_steps=8, threads=None):
    import oracle
    threads = threads or os.cpu_count() or 1
    oracle.set_threads(threads)
    d = cpu_sample_domain(args)
    o = oracle.Oracle(d.params, oracle.SOLVER_BICGSTAB, oracle.SOLVER_CG)
    o.load(d)
    o.prepare()
    t0 = time.perf_counter()
    for t in range(sample_steps):
        o.step(d.rain_mm[t])
    dt = time.perf_counter() - t0
    o.close()
    n = d.ncells * sample_steps
    return {"value": n / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"FP64 oracle (reference algorithm: unpreconditioned BiCGSTAB, CUSP rules) "
                      f"on the {patch_name(d)} patch of the workload, "
                      f"{sample_steps} step(s), {dt:.2f} s, {threads} OpenMP threads"}


def error_vs_oracle(args, local, nsteps=8):
    """The GPU solver as benchmarked (mixed, and FP64) against the FP64 oracle
    of the same method with converged solves (column-preconditioned CG to a
    relative residual of 1e-12) on the CPU-baseline patch: the free-running
    difference after nsteps, and the largest one-step difference along the
    way (oracle/shadow.py).  Norm-wise relative errors max|gpu - oracle| /
    max|oracle|.  Beside them, `oracle_spread`: the free-running difference of
    the oracle against itself with another converged 3D solver (plain CG,
    also to 1e-12) -- on this physics the reference's Picard iteration does
    not converge and the step map is chaotic, so the free-running GPU error
    is to be read against that spread, and the one-step errors are the
    parity figure."""
    import dhara_b200 as db
    import oracle
    from oracle import shadow as sh
    oracle.set_threads(os.cpu_count() or 1)
    d = cpu_sample_domain(args, nsteps=nsteps)
    q = type(d.params).from_buffer_copy(d.params)
    q.krylov_tol, q.krylov_maxiter = 1e-12, 20000
    from dhara_b200 import inputs
    d_or = inputs.Domain(params=q, fields=d.fields, int_fields=d.int_fields, rain_mm=d.rain_mm)
    o, _, _ = oracle.run(d_or, nsteps, solver3d=oracle.SOLVER_PCG_COLUMN)
    out = {"patch": patch_name(d), "steps": nsteps,
           "oracle": "FP64, column-preconditioned CG to 1e-12 relative residual, CG overland",
           "oracle_spread": sh.free_run_drift(d_or, nsteps, oracle.SOLVER_CG, oracle.SOLVER_PCG_COLUMN)}
    fields = ("psi", "theta", "ponding", "waterelev")
    for name, prec, cf32 in (("mixed", db.MIXED, 0), ("fp64", db.FP64, 0), ("mixed_closure_fp32", db.MIXED, 1)):
        p = type(d.params).from_buffer_copy(d.params)
        p.precision = prec
        p.closure_fp32 = cf32
        dd = inputs.Domain(params=p, fields=d.fields, int_fields=d.int_fields, rain_mm=d.rain_mm)
        g, _, _ = db.run(dd, nsteps=nsteps, device=local)
        s = db.Solver(p, device=local)
        s.load(dd)
        s.prepare()
        r = sh.shadow(s, dd, nsteps)
        s.close()
        out[name] = {"free_run": {k: sh.rel_err(g[k], o[k]) for k in fields},
                     "max_one_step": {k: r["max"][k] for k in fields}}
    return out


def run_reference(args, world, rank):
    """The reference's algorithm on the host cores (the reference's own CPU
    path does not exist and its CUSP dependency does not build here, so the
    FP64 oracle port stands in); each step is one time step of the same
    bounded patch of the workload the cpu_baseline leg times."""
    if rank != 0:
        return None
    import oracle
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    d = cpu_sample_domain(args)
    o = oracle.Oracle(d.params, oracle.SOLVER_BICGSTAB, oracle.SOLVER_CG)
    o.load(d)
    o.prepare()
    for t in range(args.warmup):
        o.step(d.rain_mm[t % len(d.rain_mm)])
    o.close()
    o = oracle.Oracle(d.params, oracle.SOLVER_BICGSTAB, oracle.SOLVER_CG)
    o.load(d)
    o.prepare()
    budget_s = 240.0
    t0 = time.perf_counter()
    done = 0
    for t in range(args.steps):
        o.step(d.rain_mm[t % len(d.rain_mm)])
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    o.close()
    v = d.ncells * done / dt
    sample = (f"FP64 oracle port of the reference algorithm (unpreconditioned BiCGSTAB, CUSP rules) on the "
              f"{patch_name(d)} patch of the workload, {done} of {args.steps} steps timed "
              f"({dt:.1f} s), {threads} OpenMP threads")
    return {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": done,
            "warmup": args.warmup, "ms_per_step": dt * 1e3 / max(done, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": patch_name(d), "cells": d.ncells,
                       "full_workload": f"mixed_{args.nx}x{args.nx}x{args.nz}",
                       "full_workload_cells": args.nx * args.nx * args.nz,
                       "precision": "fp64 (the reference's)", "parallelism": f"{threads} host threads"},
            "impl": "reference",
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    world, rank, local = dist_init(args)
    try:
        if args.impl == "reference":
            out = run_reference(args, world, rank)
        else:
            out = run_ours(args, world, rank, local)
        if rank == 0 and out is not None:
            print(json.dumps(out), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
