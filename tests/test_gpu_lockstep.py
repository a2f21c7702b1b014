"""The lockstep batch (``fugu_batch_opts.lockstep``): the coupled solves of
many cases of uneven grids advance together, one launch per kernel family
serving every case still running.

Per case, a virtual block of a lockstep kernel does what one CTA of the
single-case kernel does (same element functions, same reduction partition,
same merge order), so every case must reproduce the thread-pool batch -- and
with it a context running the case alone -- bit for bit: state, iteration
counts, outer passes, residual, PCG iterations and matvecs.  Both batches use
the same PCG cluster size (max_cluster), since the FP32 PCG's sums depend on
it.  The cases cover three grid classes (three PCG launches side by side),
cases that converge in different passes and Arnoldi steps, the adaptive PCG
cap and sweeps, both velocity smoothers (the fused red-black sweep and damped
Jacobi), FP64 and mixed precision, and a periodic case (ghost-cell launches,
red-black colours in two launches).
"""
import dataclasses

import numpy as np
import pytest

from coupled_codefort_2d_b200 import cases
from coupled_codefort_2d_b200._lib import FP64, MIXED, FuguError
from coupled_codefort_2d_b200.batch import STATE_FIELDS, Batch, ensemble_params, initial_bubble_state

pytestmark = pytest.mark.gpu

SMALL_GRIDS = ((16, 32), (24, 48), (32, 64))
DT, NSTEPS = 5e-4, 3
# the ensemble's solver shape with small caps, so that the adaptive PCG cap
# and sweeps both move within a few steps
SOLVER = dict(tol_bicgstab2=1e-8, max_iter_bicgstab2=200, refine=2, refine_inner_tol=1e-2, refine_max_inner=30,
              refine_max_outer=40, krylov_bc_fix=1, pcg_cap_start=4, pcd_sweeps=2, pcd_sweeps_max=8,
              pcd_smoother=1, pcd_sor_omega=1.5, graphs=1, pcd_visc_scale=1.0)
STATS = ("iter", "res", "outer", "status", "pcg_iters", "pcg_calls", "matvecs", "svof_iters")


def specs_with_periodic(n):
    """n ensemble cases; the second becomes periodic in x (same size)."""
    specs = cases.bubble_ensemble(n, grids=SMALL_GRIDS)
    g = specs[1]["grid"]
    specs[1] = dict(specs[1], grid=dataclasses.replace(g, periodic_x=True))
    return specs


def run(specs, prms, prec, lockstep, nsteps=NSTEPS, one_call=False, group=0):
    with Batch([(s["grid"], p, prec) for s, p in zip(specs, prms)], nthreads=4, max_cluster=8,
               lockstep=lockstep, lockstep_group=group) as b:
        for i, s in enumerate(specs):
            initial_bubble_state(b.case(i), s)
        o = b.case(0).step_opts(use_bicgstab2=True)
        if one_call:  # every step in one run: the cases move through their steps at their own pace
            outs = [b.run(nsteps, DT, 1, o)]
        else:
            outs = [b.run(1, DT, k, o) for k in range(1, nsteps + 1)]
        states = [b.case(i).download_state(list(STATE_FIELDS)) for i in range(len(specs))]
        launches = b.launches()
    return outs, states, launches


@pytest.mark.parametrize("prec,smoother,periodic", [(MIXED, 1, False), (FP64, 1, False), (MIXED, 0, False),
                                                    (MIXED, 1, True)])
def test_lockstep_equals_thread_pool_bitwise(gpu, prec, smoother, periodic):
    specs = specs_with_periodic(6) if periodic else cases.bubble_ensemble(6, grids=SMALL_GRIDS)
    prms = [ensemble_params(s, **dict(SOLVER, pcd_smoother=smoother)) for s in specs]
    if periodic:
        prms[1] = dataclasses.replace(prms[1], free_slip_x=0)
    ref_out, ref_states, ref_launches = run(specs, prms, prec, lockstep=False)
    out, states, launches = run(specs, prms, prec, lockstep=True)
    for step, (o, r) in enumerate(zip(out, ref_out)):
        assert o["status"] == r["status"] == [0] * len(specs)
        for i in range(len(specs)):
            for k in STATS:
                assert o["last"][i][k] == r["last"][i][k], (step, i, k, o["last"][i], r["last"][i])
            assert o["last"][i]["res"] < 1e-8
    for i in range(len(specs)):
        for k in STATE_FIELDS:
            np.testing.assert_array_equal(states[i][k], ref_states[i][k], err_msg=f"case {i} {k}")
    assert 0 < launches < ref_launches  # one launch per kernel family for all cases


@pytest.mark.parametrize("smoother,periodic,group", [(1, False, 0), (0, True, 0), (1, False, 1), (1, False, 2)])
def test_lockstep_continuous_run_equals_thread_pool_bitwise(gpu, smoother, periodic, group):
    """All steps in one run: a case whose solve ends at a pass takes its next
    step's explicit stages while the others keep solving, and joins the
    lockstep solve at the following pass, so within the run the cases are at
    different steps.  The cases form lockstep groups by PCG grid class (group
    0: one group per class; 1 and 2: at most that many cases per group), each
    run by its own host thread.  Every case still follows its own sequence of
    operations, so the final states, the last step's and the run's summed
    statistics equal the thread-pool batch's bit for bit."""
    specs = specs_with_periodic(6) if periodic else cases.bubble_ensemble(6, grids=SMALL_GRIDS)
    prms = [ensemble_params(s, **dict(SOLVER, pcd_smoother=smoother)) for s in specs]
    if periodic:
        prms[1] = dataclasses.replace(prms[1], free_slip_x=0)
    nsteps = 4
    (ref,), ref_states, _ = run(specs, prms, MIXED, lockstep=False, nsteps=nsteps, one_call=True)
    (out,), states, _ = run(specs, prms, MIXED, lockstep=True, nsteps=nsteps, one_call=True, group=group)
    assert out["status"] == ref["status"] == [0] * len(specs)
    assert out["max_res"] == ref["max_res"]
    for i in range(len(specs)):
        for k in STATS:
            assert out["last"][i][k] == ref["last"][i][k], (i, k, out["last"][i], ref["last"][i])
            assert out["total"][i][k] == ref["total"][i][k], (i, k, out["total"][i], ref["total"][i])
        assert out["total"][i]["iter"] > out["last"][i]["iter"]
        for k in STATE_FIELDS:
            np.testing.assert_array_equal(states[i][k], ref_states[i][k], err_msg=f"case {i} {k}")


def test_lockstep_rejects_cases_it_cannot_run(gpu):
    specs = cases.bubble_ensemble(2, grids=SMALL_GRIDS)
    prms = [ensemble_params(s, **SOLVER) for s in specs]
    prms[1] = dataclasses.replace(prms[1], refine=1)  # BiCGStab(2) inner solve: not a lockstep solve
    with pytest.raises(FuguError) as ei:
        Batch([(s["grid"], p, MIXED) for s, p in zip(specs, prms)], lockstep=True)
    assert ei.value.code == -1
