"""The batched ensemble across GPUs: independent cases sharded over ranks.

One process per GPU (``torchrun``); every rank advances its own shard of the
cases with a :class:`~coupled_codefort_2d_b200.batch.Batch` on its GPU (the
lockstep form by default: one launch per kernel family for all its cases).
Cases never exchange data, so the data path has no collective: the ranks
meet only at the barriers around the timed region, in one max-reduction of
the elapsed time, and in a final gather of per-case scalars (status,
largest residual, iterations, bubble centroid) to rank 0.  The reference
runs one case per ``mpirun`` and has no counterpart.

    torchrun --nproc-per-node 8 --master-addr 127.0.0.1 -m coupled_codefort_2d_b200.ensemble \
        --cases 256 --steps 200
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import cases

# flexible GMRES(30) inside the FP64 defect correction; the PCD's PCG cap
# adapts from 40 and its velocity smoothing from 6 sweeps of red-black SOR
# (omega 1.5), which on the hard high-density-ratio cases needs fewer Arnoldi
# steps than the reference's damped Jacobi at four times the sweeps; the
# PCD's Schur step carries the viscous (Cahouet-Chabard) term, which the
# viscous-dominated bubbles need most; every Arnoldi step is replayed from a
# CUDA graph (one launch per step)
SOLVER = dict(tol_bicgstab2=1e-8, max_iter_bicgstab2=500, refine=2, refine_inner_tol=1e-2, refine_max_inner=30,
              refine_max_outer=60, krylov_bc_fix=1, pcg_cap_start=40, pcd_sweeps=6, pcd_sweeps_max=24,
              pcd_smoother=1, pcd_sor_omega=1.5, graphs=1, pcd_visc_scale=1.0)
DT = 5e-4


def partition(costs, world: int) -> list[list[int]]:
    """Greedy longest-processing-time split of case indices over ``world``
    ranks: cases in decreasing cost (ties by index) go to the least-loaded
    rank (ties by rank).  Deterministic, so every rank computes the same
    split without communicating."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    shards = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        shards[r].append(i)
        load[r] += costs[i]
    return [sorted(s) for s in shards]


def case_cost(spec: dict) -> float:
    """Cost model of a case: its cell count (the work of every kernel of a
    step scales with it)."""
    return float(spec["grid"].ncells)


def solve_bytes(spec: dict, steps: list, solver: dict | None = None, inner_bytes: int = 4) -> float:
    """Algorithmic bytes of one case's coupled solves over its steps: each
    distinct array read once and written once per kernel invocation, over the
    case's nx * ny cells (N) and its 3N coupled unknowns.  Counted per step
    from its statistics (``steps``: dicts with iter = Arnoldi steps, outer =
    defect-correction passes, pcg_iters; per step, or summed over a run):

    - PCG: 9 values per cell and iteration (reads of p, cx, cy, dinv, phi, r;
      writes of p, phi, r);
    - per Arnoldi step j (taken as the mean j of a cycle of ``iter / outer``
      steps): PCD Schur step 6 values, residual update 5, cross term 4,
      zeroing 4; the velocity smoother at least ``pcd_sweeps`` sweeps of both
      components at 7 values per face (u, rhs, rho, kappa, zeta, eta read, u
      written; the adaptive count can only be higher); the coupled matvec 14
      values; classical Gram-Schmidt twice: (j + 2) vectors read by each dot,
      (j + 3) moved by each update, the norm and the scaling of the new basis
      vector (3 vectors);
    - per outer pass: the FP64 matvec (14 values at 8 B), the defect and its
      norm (4 FP64 vectors), its conversion and the accumulation.

    A lower bound where counts are not reported (the smoother's adaptive
    sweeps), exact otherwise."""
    sv = SOLVER if solver is None else solver
    n = float(spec["grid"].ncells)
    n3 = 3.0 * n
    b = float(inner_bytes)
    sweeps = sv.get("pcd_sweeps", 6)
    total = 0.0
    for st in steps:
        a = float(st["iter"])
        outer = max(int(st["outer"]), 1)
        jbar = 0.5 * (a / outer - 1.0) if a > 0 else 0.0
        pcd = (6 + 5 + 4 + 4) * n * b + 2 * sweeps * 7 * n * b
        matvec = 14 * n * b
        cgs2 = (2 * (jbar + 2) + 2 * (jbar + 3) + 1 + 3) * n3 * b
        total += a * (pcd + matvec + cgs2) + 9 * n * b * float(st["pcg_iters"])
        total += outer * (14 * n * 8 + 4 * n3 * 8 + n3 * (8 + 4) + n3 * (8 + 8 + 4))
    return total


def run_shard_gpu(specs, idx, nsteps, device, nthreads=0, precision=None, warmup=0, solver=None, lockstep=True,
                  lockstep_group=0):
    """Advance the cases ``idx`` on ``device`` and return their per-case
    scalars and the elapsed seconds of the stepping, timed with CUDA events
    on the batch stream (barrier-free; the caller brackets it).  ``warmup``
    untimed steps come first (work space allocation, the adaptive PCG cap
    settling).  ``solver`` overrides the solver settings (default
    ``SOLVER``); ``lockstep`` selects the lockstep batch (one launch per
    kernel family for the cases of a group) over the thread-pool batch,
    ``lockstep_group`` its largest group (0: one group per PCG grid class).
    The timed steps are one batch run, so no case waits for the others
    between its steps."""
    import torch

    from ._lib import MIXED
    from .batch import Batch, ensemble_params, initial_bubble_state

    prec = MIXED if precision is None else precision
    sub = [specs[i] for i in idx]
    if not sub:  # more ranks than cases: this rank only takes part in the collectives
        yield "ready", None
        yield "done", ([], 0.0)
        return
    sv = SOLVER if solver is None else solver
    with Batch([(s["grid"], ensemble_params(s, **sv), prec) for s in sub], device=device,
               nthreads=nthreads, lockstep=lockstep, lockstep_group=lockstep_group) as b:
        for k, s in enumerate(sub):
            initial_bubble_state(b.case(k), s)
        opts = b.case(0).step_opts(use_bicgstab2=True)
        if warmup:
            b.run(warmup, DT, 1, opts)
        torch.cuda.synchronize(device)
        stream = torch.cuda.ExternalStream(b.stream_handle(), device=f"cuda:{device}")
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        yield "ready", None
        n0 = b.launches()
        t0 = time.perf_counter()
        e0.record(stream)
        out = b.run(nsteps, DT, warmup + 1, opts)
        e1.record(stream)
        e1.synchronize()
        elapsed = e0.elapsed_time(e1) / 1000.0
        wall = time.perf_counter() - t0
        launches = b.launches() - n0
        torch.cuda.synchronize(device)
        rows = []
        for k, s in enumerate(sub):
            st = b.case(k).download_state(["c_field", "v_vel"])
            ycm, vr = cases.bubble_centroid_velocity(s["grid"], st["c_field"], st["v_vel"])
            tot = out["total"][k]
            rows.append({"case": s["case"], "status": out["status"][k], "max_res": out["max_res"][k],
                         "arnoldi_steps": tot["iter"], "outer": tot["outer"], "pcg_iters": tot["pcg_iters"],
                         "bytes": solve_bytes(s, [tot], sv, 4 if prec == MIXED else 8),
                         "y_centroid": ycm, "rise_velocity": vr, "host_wall_s": wall,
                         "shard_launches": launches})
        yield "done", (rows, elapsed)


def run_ensemble(specs, nsteps, rank, world, runner, barrier, max_reduce, gather):
    """Shard, run, time and gather.  ``runner(idx)`` is a generator that
    yields ("ready", None) once its cases are set up and ("done", (rows,
    seconds)) after stepping them; ``barrier``, ``max_reduce(x)`` and
    ``gather(obj) -> list | None`` are the process-group operations (rank 0
    receives the list).  Every rank takes the same collective steps in the
    same order, whatever its shard holds."""
    shards = partition([case_cost(s) for s in specs], world)
    mine = shards[rank]
    it = runner(mine)
    tag, _ = next(it)
    assert tag == "ready"
    barrier()
    tag, (rows, elapsed) = next(it)
    assert tag == "done"
    it.close()  # releases the shard's batch before the collectives
    barrier()
    slowest = max_reduce(elapsed)
    all_rows = gather(rows)
    if rank != 0:
        return None
    merged = sorted((r for part in all_rows for r in part), key=lambda r: r["case"])
    total_bytes = sum(r.get("bytes", 0.0) for r in merged)
    return {"cases": len(specs), "steps": nsteps, "world": world, "seconds": slowest,
            "case_steps_per_s": len(specs) * nsteps / slowest if slowest > 0 else float("inf"),
            "algorithmic_gb_per_s": total_bytes / slowest / 1e9 if slowest > 0 else 0.0,
            "shard_cells": [sum(specs[i]["grid"].ncells for i in s) for s in shards], "rows": merged}


def _dist_ops():
    import torch
    import torch.distributed as dist

    def barrier():
        dist.barrier()

    def max_reduce(x):
        t = torch.tensor([x], dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def gather(obj):
        out = [None] * dist.get_world_size()
        dist.all_gather_object(out, obj)
        return out

    return barrier, max_reduce, gather


def solver_from_args(args) -> dict:
    """SOLVER with the command line's overrides (None keeps a setting)."""
    solver = dict(SOLVER)
    if args.smoother:
        solver["pcd_smoother"] = 1 if args.smoother == "rbsor" else 0
    for key, val in (("pcd_sor_omega", args.omega), ("pcd_sweeps", args.sweeps), ("pcd_sweeps_max", args.sweeps_max),
                     ("graphs", args.graphs)):
        if val is not None:
            solver[key] = val
    return solver


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--cases", type=int, default=256)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--seed", type=int, default=cases.ENSEMBLE_SEED)
    ap.add_argument("--threads", type=int, default=0, help="host threads per rank (0: one per host core)")
    ap.add_argument("--out", default=None, help="write the per-case table (JSON) here")
    ap.add_argument("--warmup", type=int, default=0, help="untimed steps first")
    ap.add_argument("--smoother", choices=["jacobi", "rbsor"], default=None,
                    help="the PCD's velocity smoother (default: the SOLVER setting)")
    ap.add_argument("--omega", type=float, default=None, help="red-black SOR over-relaxation")
    ap.add_argument("--sweeps", type=int, default=None, help="PCD velocity sweeps")
    ap.add_argument("--sweeps-max", type=int, default=None, help="adaptive sweeps ceiling (0: fixed)")
    ap.add_argument("--graphs", type=int, choices=[0, 1], default=None,
                    help="replay the Arnoldi steps from CUDA graphs (default: the SOLVER setting)")
    ap.add_argument("--thread-pool", action="store_true",
                    help="step the cases from host threads instead of in lockstep")
    ap.add_argument("--lockstep-group", type=int, default=0,
                    help="largest lockstep group (0: one group per PCG grid class)")
    args = ap.parse_args(argv)
    solver = solver_from_args(args)
    import datetime

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        barrier, max_reduce, gather = _dist_ops()
    else:
        barrier, max_reduce, gather = (lambda: None), (lambda x: x), (lambda o: [o])
    specs = cases.bubble_ensemble(args.cases, seed=args.seed)
    res = run_ensemble(specs, args.steps, rank, world,
                       lambda idx: run_shard_gpu(specs, idx, args.steps, local, args.threads, warmup=args.warmup,
                                                 solver=solver, lockstep=not args.thread_pool,
                                                 lockstep_group=args.lockstep_group),
                       barrier, max_reduce, gather)
    if world > 1:
        dist.destroy_process_group()
    if rank == 0:
        rows = res.pop("rows")
        res["failed"] = [r["case"] for r in rows if r["status"] != 0]
        res["max_res"] = max(r["max_res"] for r in rows)
        res["form"] = "thread pool" if args.thread_pool else f"lockstep (group <= {args.lockstep_group or 'class'})"
        res["launches_rank0"] = rows[0].get("shard_launches") if rows else None
        res["solver"] = solver
        print(json.dumps(res), flush=True)
        if args.out:
            with open(args.out, "w") as f:
                json.dump(rows, f, indent=1)


if __name__ == "__main__":
    main()
