"""Benchmark of the B200 FUGU-2D coupled step (one JSON line on rank 0).

Workload (the configuration the headline metric is quoted on): static
two-phase droplet on the unit square, 256 x 256 MAC grid, R = 0.25 centred,
inside rho = 1, mu = 0.1, outside rho = 0.1, mu = 0.01, sigma = 1, no gravity,
colour from 16 x 16 sub-sampled area fractions, BDF2, dt = 1e-4, each coupled
step solved to a true relative residual |B - AX| / |B| < 1e-8.  A "step" is
one advance_coupled_step.  Synthetic inputs: the case is fully determined by
these parameters (no dataset).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

value : mixed form (FP32 inner flexible GMRES(30) + PCD inside the FP64
        defect correction, each Arnoldi step replayed from a CUDA graph; the
        PCD's Schur step carries the viscous (Cahouet-Chabard) term),
        device-resident state, CUDA events on the library's stream around
        each timed step, L2 flushed (256 MiB write) between timed steps.
e2e   : the same steps through the drop-in C entry fugu_advance_coupled_step
        with pinned host arrays (state uploaded and downloaded every step).
Also reported: the FP64-inner form of the same solver ("fp64"), the same
mixed form with the reference's PCD (no viscous term), and the reference
algorithm as written (BiCGStab + PCD, preconditioned residual, max 500
iterations) with the residual it actually reaches.

Multi-GPU (torchrun): the case does not shard; every rank runs an
independent replica ("replicas only", weak scaling); value = all ranks'
steps / max over ranks of the timed region.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "coupled steps/s at 1e-8 residual: FP32+refine vs FP64 on B200; % HBM roofline"
UNIT = "coupled steps/s"
N = 256
DT = 1e-4
TOL = 1e-8


# inner solve of the FP64 defect correction: flexible GMRES (refine 2) or the
# step's BiCGStab(2) (refine 1); both around the same PCD preconditioner.
# With flexible GMRES the PCD's Schur step carries the viscous
# (Cahouet-Chabard) term (pcd_visc_scale 1), the PCG inside PCD starts capped
# at 80 iterations and the velocity smoothing at 6 Jacobi sweeps; an inner
# solve that misses its tolerance doubles the cap (up to the reference's
# 150), then the sweeps (up to 24).  BiCGStab keeps the reference's fixed
# preconditioner.
INNER = {"fgmres": 2, "bicgstab2": 1}
INNER_NAME = {2: "flexible GMRES(30)", 1: "BiCGStab(2)"}
PCG_CAP_START = 80
PCD_SWEEPS, PCD_SWEEPS_MAX = 6, 24
VISC_SCALE = 1.0
# the reference's PCD (no viscous term), measured beside the headline; its
# PCG cap starts at 40, where that preconditioner is fastest
REF_PCD_CAP_START = 40


def case_params(refine=2):
    from coupled_codefort_2d_b200.params import Params

    fg = refine == 2
    return Params(rho1=1.0, rho2=0.1, mu1=0.1, mu2=0.01, sigma=1.0, gx=0.0, gy=0.0, time_order=2,
                  tol_bicgstab2=TOL, max_iter_bicgstab2=500, refine=refine, refine_inner_tol=1e-2,
                  refine_max_inner=30, refine_max_outer=60, krylov_bc_fix=1,
                  pcg_cap_start=PCG_CAP_START if fg else 0, pcd_sweeps=PCD_SWEEPS if fg else 3,
                  pcd_sweeps_max=PCD_SWEEPS_MAX if fg else 0, graphs=1,
                  pcd_visc_scale=VISC_SCALE if fg else 0.0)


def reference_pcd_params(prm):
    return prm.with_(pcd_visc_scale=0.0, pcg_cap_start=REF_PCD_CAP_START)


def solver_name(refine):
    if refine != 2:
        return f"{INNER_NAME[refine]}+PCD (inner tol 1e-2)"
    return (f"{INNER_NAME[refine]}+PCD with the viscous Schur term (inner tol 1e-2, pcd_visc_scale {VISC_SCALE}, "
            f"PCG cap adaptive {PCG_CAP_START}-150, sweeps {PCD_SWEEPS}-{PCD_SWEEPS_MAX}; Arnoldi steps replayed "
            "from CUDA graphs)")


def initial_state(g, prm):
    from coupled_codefort_2d_b200 import cases
    from coupled_codefort_2d_b200._lib import FIELD_KIND

    c0 = cases.circle_fraction(g, 0.5, 0.5, 0.25, inside=1.0, ns=16)
    st = {k: g.zeros(FIELD_KIND[k]) for k in ("u_vel", "v_vel", "p_field", "c_field", "u_prev", "v_prev", "rho_c",
                                              "rho_u", "rho_v", "kappa", "zeta", "eta", "kappa_curv",
                                              "f_sigma_u", "f_sigma_v")}
    st["c_field"][...] = c0
    return st


def workload_config(solver_name):
    return {
        "workload": f"static_droplet_{N}x{N}", "grid": [N, N], "radius": 0.25, "rho_in_out": [1.0, 0.1],
        "mu_in_out": [0.1, 0.01], "sigma": 1.0, "time_scheme": "BDF2", "dt": DT,
        "residual": "true |B-AX|/|B| < 1e-8 (coupled_dot norm)",
        "solver": solver_name, "l2": "flushed between timed steps (256 MiB write)",
    }


# --------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples during the timed region (clocks and throttle reasons)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        for line in (self.out or "").strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None
        loaded = [s for s in sm if smax and s > 0.5 * smax] or sm
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for nm, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(loaded)) if loaded else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(rows)}


# --------------------------------------------------------------- GPU arm
def gpu_arm(args, rank, world, local_rank):
    import torch

    from coupled_codefort_2d_b200 import build
    from coupled_codefort_2d_b200._lib import FIELD_KIND, MIXED, FP64
    from coupled_codefort_2d_b200.context import Context
    from coupled_codefort_2d_b200.layout import Grid

    build.build()
    torch.cuda.set_device(local_rank)
    g = Grid(N, N)
    prm = case_params(INNER[args.inner])
    st0 = initial_state(g, prm)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local_rank}")

    def run_form(precision, steps, warmup, use_b2=True, prm_=None, profile=False, sampler=None):
        p = prm_ or prm
        with Context(g, p, device=local_rank, precision=precision) as ctx:
            ctx.upload_state(st0)
            # properties from C (the drivers' set-up, main.f90:185-186)
            pr = {k: g.zeros(FIELD_KIND[k]) for k in ("rho_c", "rho_u", "rho_v", "kappa", "zeta", "eta")}
            ctx.compute_mixture_densities(st0["c_field"], pr["rho_c"], pr["rho_u"], pr["rho_v"])
            ctx.compute_mixture_viscosities(st0["c_field"], pr["kappa"], pr["zeta"], pr["eta"])
            for k, a in pr.items():
                ctx.upload(k, a)
            opts = ctx.step_opts(use_bicgstab2=use_b2)
            stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=f"cuda:{local_rank}")
            stats = []
            for s in range(1, warmup + 1):
                stats.append(ctx.step(DT, s, opts))
            if world > 1:
                torch.distributed.barrier()
            torch.cuda.synchronize()
            if profile:
                ctx.profile(1)
            times = []
            ctx_s = sampler if sampler is not None else _Null()
            with ctx_s:
                for s in range(warmup + 1, warmup + steps + 1):
                    with torch.cuda.stream(stream):
                        flush.zero_()
                        e0 = torch.cuda.Event(enable_timing=True)
                        e1 = torch.cuda.Event(enable_timing=True)
                        e0.record(stream)
                    r = ctx.step(DT, s, opts)
                    with torch.cuda.stream(stream):
                        e1.record(stream)
                    e1.synchronize()
                    times.append(e0.elapsed_time(e1))
                    stats.append(r)
            torch.cuda.synchronize()
            prof = ctx.profile(0) if profile else None
            state = ctx.download_state(["u_vel", "v_vel", "p_field", "c_field", "u_prev", "v_prev", "rho_c", "rho_u",
                                        "rho_v", "kappa", "zeta", "eta", "kappa_curv", "f_sigma_u", "f_sigma_v"])
        return times, stats, prof, state

    sampler = ClockSampler(local_rank)
    t_mixed, s_mixed, prof, state_w = run_form(MIXED, args.steps, args.warmup, profile=True, sampler=sampler)
    total_ms = float(np.sum(t_mixed))
    # max over ranks of the timed region
    if world > 1:
        tt = torch.tensor([total_ms], device=f"cuda:{local_rank}", dtype=torch.float64)
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(tt.item())
    out = {"t_mixed": t_mixed, "s_mixed": s_mixed, "prof": prof, "total_ms": total_ms, "clocks": sampler.summary()}

    if not args.quick:  # every rank: the ensemble is sharded over the ranks
        peaks = {}
        pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
        if os.path.exists(pk):
            peaks = json.load(open(pk))
        out["batched"] = batched_arm(world, rank, local_rank, peaks)

    if rank == 0 and not args.quick:
        # FP64 inner form of the same solver, same steps
        t64, s64, _, _ = run_form(FP64, args.steps, args.warmup)
        out["t_fp64"], out["s_fp64"] = t64, s64
        out["e2e"] = e2e_arm(args, g, prm, st0, local_rank)
        out["state_w"] = state_w
        # the reference algorithm as written (preconditioned residual, max 500 its,
        # the reference's 3 PCD sweeps and uncapped PCG)
        pref = prm.with_(refine=0, krylov_bc_fix=0, pcd_sweeps=3, pcd_sweeps_max=0, pcg_cap_start=0,
                         pcd_visc_scale=0.0)
        tref, sref, _, _ = run_form(FP64, 2, 1, use_b2=False, prm_=pref)
        out["t_ref"], out["s_ref"] = tref, sref
        # last, guarded: the same mixed form with the reference's PCD (no
        # viscous term).  A failure is reported in the line; a CUDA error that
        # leaves the context unusable cannot reach the arms above any more.
        if INNER[args.inner] == 2:
            try:
                tv, sv, _, _ = run_form(MIXED, args.steps, args.warmup, prm_=reference_pcd_params(prm))
                out["t_refpcd"], out["s_refpcd"] = tv, sv
            except Exception as exc:  # noqa: BLE001
                out["refpcd_error"] = f"{type(exc).__name__}: {exc}"
    return out


# the batched line: the whole rising-bubble ensemble of the configuration
# (256 cases per GPU), mixed form, device-timed steps after warm-up, in both
# batched forms: the lockstep batch (groups of at most BATCH_GROUP cases of
# one PCG grid class) and the thread-pool batch; the faster is the line's value
BATCH_CASES_PER_GPU = 256
BATCH_STEPS, BATCH_WARMUP = 20, 2
BATCH_GROUP = 4
# the like-for-like comparison with the plain FP64 single-case form: the same
# cases and the same steps in both forms
SAME_CASES, SAME_STEPS, SAME_WARMUP = 32, 3, 1


def _fp64_single(specs, steps, warmup, local_rank):
    """The plain FP64 form of the same solver, one context at a time: CUDA
    events on each context's stream around its timed steps, summed."""
    import torch

    from coupled_codefort_2d_b200 import ensemble
    from coupled_codefort_2d_b200._lib import FP64
    from coupled_codefort_2d_b200.batch import ensemble_params, initial_bubble_state
    from coupled_codefort_2d_b200.context import Context

    ms, n, res = 0.0, 0, 0.0
    for s in specs:
        with Context(s["grid"], ensemble_params(s, **ensemble.SOLVER), device=local_rank, precision=FP64) as ctx:
            initial_bubble_state(ctx, s)
            o = ctx.step_opts(use_bicgstab2=True)
            for k in range(1, warmup + 1):
                ctx.step(ensemble.DT, k, o)
            stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=f"cuda:{local_rank}")
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            for k in range(warmup + 1, warmup + steps + 1):
                r = ctx.step(ensemble.DT, k, o)
                res = max(res, r["res"])
            e1.record(stream)
            e1.synchronize()
            ms += e0.elapsed_time(e1)
            n += steps
    return {"value": 1000.0 * n / ms, "unit": "case-steps/s", "case_steps": n, "max_true_residual": res}


def batched_arm(world, rank, local_rank, peaks):
    """The batched form on the rising-bubble ensemble of the configuration
    (256 x N cases of the seeded ensemble, grids 64x128 .. 256x512, density
    ratios 10-1000), sharded over the N ranks, lockstep mixed precision,
    device-timed.  Beside it, on rank 0, the same comparison on equal work:
    the first 32 cases, the same steps, lockstep mixed against the plain
    FP64 single-case form one context at a time."""
    from coupled_codefort_2d_b200 import cases, ensemble

    specs = cases.bubble_ensemble(BATCH_CASES_PER_GPU * world)
    if world > 1:
        barrier, max_reduce, gather = ensemble._dist_ops()
    else:
        barrier, max_reduce, gather = (lambda: None), (lambda x: x), (lambda o: [o])
    forms = {}
    for form, lockstep in (("lockstep", True), ("thread_pool", False)):
        res = ensemble.run_ensemble(
            specs, BATCH_STEPS, rank, world,
            lambda idx: ensemble.run_shard_gpu(specs, idx, BATCH_STEPS, local_rank, nthreads=0, warmup=BATCH_WARMUP,
                                               lockstep=lockstep, lockstep_group=BATCH_GROUP),
            barrier, max_reduce, gather)
        forms[form] = res
    if rank != 0:
        return None
    peak = (peaks or {}).get("hbm_gbs")
    src = "measured" if peak else "fallback"
    peak = peak or 6650.0
    summary = {}
    for form, res in forms.items():
        rows = res["rows"]
        summary[form] = {"value": res["case_steps_per_s"], "seconds": res["seconds"],
                         "max_true_residual": max(r["max_res"] for r in rows),
                         "failed_cases": [r["case"] for r in rows if r["status"] != 0],
                         "gpu_launches_rank0": rows[0].get("shard_launches"),
                         "algorithmic_gb_per_s": res["algorithmic_gb_per_s"] / world}
    best = max(summary, key=lambda f: summary[f]["value"])
    b = summary[best]
    out = {"workload": f"rising_bubble_ensemble_{len(specs)} (seed {cases.ENSEMBLE_SEED})",
           "value": b["value"], "unit": "case-steps/s", "form": best, "steps": BATCH_STEPS, "warmup": BATCH_WARMUP,
           "seconds": b["seconds"], "dtype": "f32 inner / f64 outer",
           "max_true_residual": max(v["max_true_residual"] for v in summary.values()),
           "failed_cases": sorted(set(sum((v["failed_cases"] for v in summary.values()), []))),
           "solver": "FP64 defect correction around flexible GMRES(30) + PCD with the viscous Schur term (PCG cap "
                     "adaptive 40-150, red-black SOR velocity smoother omega 1.5, sweeps adaptive 6-24); all "
                     "timed steps in one batch run per form",
           "solver_params": ensemble.SOLVER,
           "forms": {"lockstep": dict(summary["lockstep"], group=f"<= {BATCH_GROUP} cases of one PCG grid class, "
                                                                 "one launch per kernel family per group"),
                     "thread_pool": dict(summary["thread_pool"], note="host threads stepping contexts")},
           "gpu_launches_rank0": b["gpu_launches_rank0"],
           "roofline": {"bound": "hbm", "achieved": b["algorithmic_gb_per_s"], "peak": peak,
                        "peak_source": src, "unit": "GB/s", "frac": b["algorithmic_gb_per_s"] / peak,
                        "traffic": None,
                        "bytes": "algorithmic bytes of every case's solves (ensemble.solve_bytes: PCG iterations, "
                                 "Arnoldi steps with PCD, matvec and Gram-Schmidt, outer passes; smoother sweeps at "
                                 "their minimum) / device time, per GPU"},
           "timing": "CUDA events on the batch stream around the timed steps, max over ranks"}
    if world == 1:
        same = specs[:SAME_CASES]
        r2 = ensemble.run_ensemble(
            same, SAME_STEPS, 0, 1,
            lambda idx: ensemble.run_shard_gpu(same, idx, SAME_STEPS, local_rank, nthreads=0, warmup=SAME_WARMUP,
                                               lockstep=best == "lockstep", lockstep_group=BATCH_GROUP),
            barrier, max_reduce, gather)
        f64 = _fp64_single(same, SAME_STEPS, SAME_WARMUP, local_rank)
        out["equal_work"] = {"cases": len(same), "steps": SAME_STEPS, "warmup": SAME_WARMUP,
                             "batched_mixed": r2["case_steps_per_s"], "batched_form": best,
                             "fp64_single_case": f64,
                             "batched_mixed_over_fp64_single": r2["case_steps_per_s"] / f64["value"],
                             "note": "the same cases and steps in both forms, device-timed"}
    return out


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        pass


def pinned_field(g, kind):
    import torch

    shp = g.shape(kind)
    t = torch.zeros((shp[1], shp[0]), dtype=torch.float64, pin_memory=True)
    return t, t.numpy().T  # Fortran-ordered view of pinned memory


def e2e_arm(args, g, prm, st0, local_rank):
    """fugu_advance_coupled_step (the drop-in C entry) on pinned host arrays."""
    import torch

    from coupled_codefort_2d_b200._lib import FIELD_KIND, MIXED
    from coupled_codefort_2d_b200.context import Context

    names = ["u_vel", "v_vel", "p_field", "c_field", "u_prev", "v_prev", "rho_c", "rho_u", "rho_v", "kappa",
             "zeta", "eta", "kappa_curv", "f_sigma_u", "f_sigma_v"]
    keep, host = [], {}
    for k in names:
        t, a = pinned_field(g, FIELD_KIND[k])
        a[...] = st0[k]
        keep.append(t)
        host[k] = a
    nbytes = sum(a.nbytes for a in host.values())
    with Context(g, prm, device=local_rank, precision=MIXED) as ctx:
        ctx.compute_mixture_densities(host["c_field"], host["rho_c"], host["rho_u"], host["rho_v"])
        ctx.compute_mixture_viscosities(host["c_field"], host["kappa"], host["zeta"], host["eta"])
        stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=f"cuda:{local_rank}")
        times = []
        for s in range(1, args.warmup + args.steps + 1):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r = ctx.advance_coupled_step(*[host[k] for k in names], DT, s, use_bicgstab2=True)
            e1.record(stream)
            e1.synchronize()
            if s > args.warmup:
                times.append(e0.elapsed_time(e1))
            assert r["res"] < TOL, r
    ms = float(np.mean(times))
    return {"value": 1000.0 / ms, "unit": UNIT, "h2d_bytes_per_step": int(nbytes), "d2h_bytes_per_step": int(nbytes),
            "ms_per_step": ms, "entry": "fugu_advance_coupled_step (pinned host arrays, reference layout)"}


# --------------------------------------------------------------- CPU legs
def cpu_step_time(state, step_idx, prm, nsteps=1):
    """The oracle (a C restatement of the reference) on the same inputs."""
    from coupled_codefort_2d_b200.layout import Grid
    from oracle import oracle

    g = Grid(N, N)
    o = oracle.Oracle(g, prm)
    st = {k: a.copy(order="F") for k, a in state.items()}
    t0 = time.perf_counter()
    stats = []
    for s in range(step_idx, step_idx + nsteps):
        stats.append(o.step(st, DT, s, use_bicgstab2=True))
    return (time.perf_counter() - t0) / nsteps, stats


def _replica_run(args_tuple):
    """One independent replica of the workload on one host core: its own
    warm-up steps, then the timed steps, each timed inside this process (no
    inter-process traffic inside the timed region)."""
    warmup, steps, inner = args_tuple
    from coupled_codefort_2d_b200.layout import Grid
    from oracle import oracle

    g = Grid(N, N)
    prm = case_params(inner)
    st = initial_state(g, prm)
    o = oracle.Oracle(g, prm)
    o.densities(st["c_field"], st["rho_c"], st["rho_u"], st["rho_v"])
    o.viscosities(st["c_field"], st["kappa"], st["zeta"], st["eta"])
    for s in range(1, warmup + 1):
        o.step(st, DT, s, use_bicgstab2=True)
    times, res = [], []
    for s in range(warmup + 1, warmup + steps + 1):
        t0 = time.perf_counter()
        r = o.step(st, DT, s, use_bicgstab2=True)
        times.append(time.perf_counter() - t0)
        res.append(r.res)
    return times, res


def reference_toolchain():
    """Where the host could build and run the Fortran/MPI reference: the
    compilers and launcher its Makefile and README use (None when absent),
    and the host's cores."""
    tools = {t: shutil.which(t) for t in ("gfortran", "mpifort", "mpirun")}
    return {**tools, "cores": os.cpu_count() or 1}


def reference_arm(args, rank, world):
    """The reference's CPU path on the host cores: the oracle port (the
    Fortran/MPI reference cannot be built here), one independent replica per
    host core running the whole workload; each replica times its own steps,
    and the aggregate rate is replicas x steps / the slowest replica's time."""
    if rank != 0:
        return
    from oracle import oracle

    oracle.build()
    tc = reference_toolchain()
    inner = INNER[args.inner]
    cores = os.cpu_count() or 1
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        runs = pool.map(_replica_run, [(args.warmup, args.steps, inner)] * cores, chunksize=1)
    slowest = max(sum(t) for t, _ in runs)
    value = cores * args.steps / slowest
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 * slowest / args.steps / cores, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(f"FP64 defect correction around {solver_name(inner)} (oracle port of the "
                                  "reference modules)"),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{cores} independent replicas x 1 thread, each {args.warmup} warm-up + "
                                   f"{args.steps} timed steps of the {N}^2 droplet, timed inside the replica"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "max_true_residual": max(max(r) for _, r in runs),
        "reference_toolchain": tc,
        "note": ("the Fortran/MPI reference is not built (probed on this host: "
                 + ", ".join(f"{t} {'at ' + tc[t] if tc[t] else 'absent'}" for t in ("gfortran", "mpifort", "mpirun"))
                 + "); the C oracle restates its hot path"),
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------- main
# algorithmic values moved per cell and PCG iteration by a fused streaming
# implementation: reads of p, cx, cy, dinv, phi, r and writes of p, phi, r
PCG_VALUES_PER_CELL = 9


def roofline(prof, peaks):
    """Dominant kernel: the persistent PCG of the PCD preconditioner (FP32 in
    the mixed form).  Algorithmic bytes per PCG iteration and cell: the fused
    minimum, reads of p, cx, cy, dinv, phi, r and writes of p, phi, r = 9
    values (the kernel itself keeps them on chip).
    The timed launches are the PCG of the first Arnoldi step of every
    flexible-GMRES cycle in the timed steps (CUDA events recorded by the
    replayed graph), with their own iteration counts."""
    if not prof or not prof["pcg_launches"]:
        return None
    elt = 4  # FP32 inner solve
    bytes_per_launch = PCG_VALUES_PER_CELL * elt * prof["pcg_cells"] * prof["pcg_iters_timed"] / prof["pcg_launches"]
    ms_per_launch = prof["pcg_ms"] / prof["pcg_launches"]
    achieved = bytes_per_launch / (ms_per_launch * 1e-3) / 1e9
    peak = peaks.get("hbm_gbs") if peaks else None
    src = "measured" if peak else "fallback"
    peak = peak or 6650.0
    traffic = None
    tf = os.path.join(ROOT, "profiles", "pcg_traffic.json")
    if os.path.exists(tf):
        try:
            t = json.load(open(tf))
            traffic = t.get("dram_bytes_per_launch")
        except Exception:
            traffic = None
    return {"kernel": "k_pcg_cluster<float> (cluster-resident Jacobi-PCG of the PCD pressure step)", "bound": "hbm",
            "achieved": achieved, "peak": peak, "peak_source": src, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "bytes_per_launch": bytes_per_launch, "ms_per_launch": ms_per_launch,
            "iters_per_launch": prof["pcg_iters_timed"] / prof["pcg_launches"],
            "timed_launches": prof["pcg_launches"],
            "timing": "CUDA events on the library's stream around the PCG of the first Arnoldi step of each "
                      "flexible-GMRES cycle in the timed steps"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gpu", choices=["gpu", "reference"])
    ap.add_argument("--quick", action="store_true", help="skip the secondary arms")
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline sample")
    ap.add_argument("--inner", default="fgmres", choices=sorted(INNER),
                    help="inner solve of the FP64 defect correction")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch

        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    if args.impl == "reference":
        reference_arm(args, rank, world)
        if world > 1:
            import torch

            torch.distributed.destroy_process_group()
        return

    out = gpu_arm(args, rank, world, local_rank)
    if world > 1:
        import torch

        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank != 0:
        return
    peaks = {}
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = json.load(open(pk))
    total_ms = out["total_ms"]
    value = world * args.steps * 1000.0 / total_ms
    s_m = out["s_mixed"][args.warmup:]
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 inner / f64 outer",
        "data": "synthetic (droplet case fully determined by its parameters)",
        "config": workload_config(f"FP64 defect correction around FP32 {solver_name(INNER[args.inner])}"),
        "max_true_residual": max(r["res"] for r in s_m),
        "per_step": {"outer": [r["outer"] for r in s_m], "inner_iters": [r["iter"] for r in s_m],
                     "pcg_calls": [r["pcg_calls"] for r in s_m], "pcg_iters": [r["pcg_iters"] for r in s_m]},
        "roofline": roofline(out["prof"], peaks),
        "gpu_launches": int(out["prof"]["kernel_launches"]) if out["prof"] else None,
        "clocks": out["clocks"],
    }
    if "t_fp64" in out:
        s64 = out["s_fp64"][args.warmup:]
        line["fp64"] = {"value": 1000.0 * len(out["t_fp64"]) / float(np.sum(out["t_fp64"])), "unit": UNIT,
                        "max_true_residual": max(r["res"] for r in s64),
                        "solver": f"FP64 defect correction around FP64 {solver_name(INNER[args.inner])}"}
        line["mixed_over_fp64"] = value / world / line["fp64"]["value"]
        sref = out["s_ref"][1:]
        line["reference_algorithm_fp64"] = {
            "value": 1000.0 * len(out["t_ref"]) / float(np.sum(out["t_ref"])), "unit": UNIT,
            "iterations": [r["iter"] for r in sref], "preconditioned_residual": [r["res"] for r in sref],
            "status": ["converged" if r["status"] == 0 else "max-iter/breakdown" for r in sref],
            "solver": "bicgstab_solve + PCD exactly as the reference (tol 1e-8 on the preconditioned residual)"}
    if "t_refpcd" in out:
        sv = out["s_refpcd"][args.warmup:]
        line["reference_pcd"] = {
            "value": 1000.0 * len(out["t_refpcd"]) / float(np.sum(out["t_refpcd"])), "unit": UNIT,
            "max_true_residual": max(r["res"] for r in sv), "inner_iters": [r["iter"] for r in sv],
            "outer": [r["outer"] for r in sv], "status": [r["status"] for r in sv],
            "solver": f"as value, with the reference's PCD Schur step (no viscous term) and the PCG cap adaptive "
                      f"from {REF_PCD_CAP_START}",
            "timing": "CUDA events on the library's stream, same steps and L2 flush as value, no profiling"}
    elif "refpcd_error" in out:
        line["reference_pcd"] = {"error": out["refpcd_error"]}
    if "e2e" in out:
        line["e2e"] = out["e2e"]
    if out.get("batched"):
        line["batched"] = out["batched"]
    if not args.no_cpu and "state_w" in out:
        nxt = args.warmup + args.steps + 1
        dt_cpu, st_cpu = cpu_step_time(out["state_w"], nxt, case_params(INNER[args.inner]))
        line["cpu_baseline"] = {
            "value": 1.0 / dt_cpu, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"1 coupled step (step {nxt}) of the same workload from the GPU run's state, "
                      f"oracle C port, FP64 defect correction around {solver_name(INNER[args.inner])}, 1 thread",
            "true_residual": st_cpu[0].res}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
