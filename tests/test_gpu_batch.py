"""Batched form (``fugu_batch_*``): independent cases of different grids and
physics stepped together from a pool of host threads.

With the single-context cluster plan (max_cluster 16) a batch must give, case
by case, the same bits as a context running that case alone: the cases share
nothing but the device.  With the autotuned cluster sizes every case still
reaches the FP64 true-residual tolerance, and its state stays within the
mixed-precision bound (1e-6 relative L2) of the lone run.
"""
import numpy as np
import pytest

from coupled_codefort_2d_b200 import cases
from coupled_codefort_2d_b200._lib import FP64, MIXED, FuguError
from coupled_codefort_2d_b200.batch import STATE_FIELDS, Batch, ensemble_params, initial_bubble_state
from coupled_codefort_2d_b200.context import Context

pytestmark = pytest.mark.gpu

SOLVER = dict(tol_bicgstab2=1e-8, max_iter_bicgstab2=200, refine=1, refine_inner_tol=1e-2, refine_max_inner=30,
              refine_max_outer=40, krylov_bc_fix=1)
SMALL_GRIDS = ((16, 32), (24, 48), (32, 64))
DT, NSTEPS = 5e-4, 3


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def alone(spec, prm, prec):
    with Context(spec["grid"], prm, precision=prec) as ctx:
        initial_bubble_state(ctx, spec)
        o = ctx.step_opts(use_bicgstab2=True)
        stats = [ctx.step(DT, s, o) for s in range(1, NSTEPS + 1)]
        return stats, ctx.download_state(list(STATE_FIELDS))


def batched(specs, prms, prec, **kw):
    with Batch([(s["grid"], p, prec) for s, p in zip(specs, prms)], **kw) as b:
        for i, s in enumerate(specs):
            initial_bubble_state(b.case(i), s)
        out = b.run(NSTEPS, DT, 1, b.case(0).step_opts(use_bicgstab2=True))
        states = [b.case(i).download_state(list(STATE_FIELDS)) for i in range(len(specs))]
        prof = [b.case(i).profile(-1) for i in range(len(specs))]
    return out, states, prof


# the batched ensemble's own solver: flexible GMRES, adaptive PCD with the
# red-black SOR velocity smoother, Arnoldi steps replayed from CUDA graphs
ENSEMBLE_LIKE = dict(tol_bicgstab2=1e-8, max_iter_bicgstab2=200, refine=2, refine_inner_tol=1e-2, refine_max_inner=30,
                     refine_max_outer=40, krylov_bc_fix=1, pcg_cap_start=4, pcd_sweeps=2, pcd_sweeps_max=8,
                     pcd_smoother=1, pcd_sor_omega=1.5, graphs=1)


@pytest.mark.parametrize("prec,solver", [(FP64, SOLVER), (MIXED, SOLVER), (MIXED, ENSEMBLE_LIKE)])
def test_batch_equals_lone_contexts_bitwise(gpu, prec, solver):
    specs = cases.bubble_ensemble(4, grids=SMALL_GRIDS)
    prms = [ensemble_params(s, **solver) for s in specs]
    out, states, _ = batched(specs, prms, prec, nthreads=4, max_cluster=16)
    assert out["status"] == [0] * len(specs)
    for i, (s, p) in enumerate(zip(specs, prms)):
        stats, ref = alone(s, p, prec)
        assert out["last"][i]["iter"] == stats[-1]["iter"]
        assert out["last"][i]["res"] == stats[-1]["res"]
        assert out["max_res"][i] == max(st["res"] for st in stats)
        for k in STATE_FIELDS:
            np.testing.assert_array_equal(states[i][k], ref[k], err_msg=f"case {i} {k}")


def test_autotuned_batch_reaches_tolerance(gpu):
    specs = cases.bubble_ensemble(6, grids=SMALL_GRIDS)
    prms = [ensemble_params(s, **SOLVER) for s in specs]
    out, states, prof = batched(specs, prms, MIXED, nthreads=3)
    assert out["status"] == [0] * len(specs)
    for i, (s, p) in enumerate(zip(specs, prms)):
        assert out["max_res"][i] < 1e-8
        assert prof[i]["pcg_cluster_fp32"] in (2, 4, 8, 16)
        _, ref = alone(s, p, MIXED)
        num = sum(float(np.sum((states[i][k] - ref[k]) ** 2)) for k in ("u_vel", "v_vel"))
        den = sum(float(np.sum(ref[k] ** 2)) for k in ("u_vel", "v_vel"))
        assert (num / den) ** 0.5 <= 1e-6
        assert rel(states[i]["c_field"], ref["c_field"]) <= 1e-6


def test_batch_rejects_bad_run_arguments(gpu):
    specs = cases.bubble_ensemble(2, grids=SMALL_GRIDS)
    prms = [ensemble_params(s, **SOLVER) for s in specs]
    with Batch([(s["grid"], p, FP64) for s, p in zip(specs, prms)], max_cluster=4) as b:
        with pytest.raises(FuguError):
            b.run(-1, DT, 1, b.case(0).step_opts())
