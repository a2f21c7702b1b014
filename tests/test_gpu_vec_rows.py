"""The vectorised row kernels (``fugu_params.vec_rows``): the damped-Jacobi
sweeps and the PCD's Schur, residual and cross steps with 16-byte vector
accesses, four floats or two doubles of a box row per thread.  They read the
same operands through a window of registers and keep every formula's operand
order, so the bar is bit identity:

- FP64 routines (``solve_helmholtz_u/v``, ``apply_pcd_precond``) against the
  CPU oracle on every routine grid, walls and periodic boxes, with and
  without the Darcy penalty;
- the mixed form (FP32 inner solve) with vec_rows = 1 against vec_rows = -1
  (the one-thread-per-element kernels): same states and iteration counts;
- the size rule (vec_rows = 0 takes the vector kernels from 2^20 box points,
  the sweeps of wall-bounded cases from 2^21) on a 1024 x 1024 PCD
  application against vec_rows = -1.
"""
import numpy as np
import pytest

from conftest import GRIDS, colour, rfield, two_phase_params
from coupled_codefort_2d_b200.context import Context
from coupled_codefort_2d_b200.layout import Grid
from test_gpu_step import STATE, _device_run

pytestmark = pytest.mark.gpu

VEC_GRIDS = {**GRIDS, "walls_61x47": Grid(61, 47, 1.3, 1.0), "walls_256x256": Grid(256, 256)}


@pytest.fixture(params=list(VEC_GRIDS))
def grid(request):
    return VEC_GRIDS[request.param]


def _props(o, g, rng):
    return o.properties(colour(rng, g))


@pytest.mark.parametrize("use_pen", [False, True])
def test_helmholtz_sweeps_vec_rows(gpu, oracle_mod, grid, use_pen):
    """n damped-Jacobi sweeps, odd n included (the result is copied back)."""
    rng = np.random.default_rng(61)
    prm = two_phase_params(vec_rows=1)
    o = oracle_mod.Oracle(grid, prm)
    pr = _props(o, grid, rng)
    with Context(grid, prm) as ctx:
        for kind, gfn, ofn in (("u", ctx.solve_helmholtz_u, o.helmholtz_u), ("v", ctx.solve_helmholtz_v, o.helmholtz_v)):
            sol, rhs = rfield(rng, grid, kind), rfield(rng, grid, kind)
            pen = rfield(rng, grid, kind, 0, 1e6) if use_pen else None
            rho = pr["rho_u"] if kind == "u" else pr["rho_v"]
            for n in (1, 2, 5):
                s, r = sol.copy(order="F"), sol.copy(order="F")
                gfn(s, rhs, rho, pr["kappa"], pr["zeta"], pr["eta"], 2e-3, n, pen)
                ofn(r, rhs, pr, 2e-3, n, pen)
                np.testing.assert_array_equal(s, r, err_msg=f"{kind} n={n}")


@pytest.mark.parametrize("penalty,visc", [(False, 0.0), (True, 0.0), (False, 1.0)])
def test_pcd_precond_vec_rows(gpu, oracle_mod, grid, penalty, visc):
    """apply_pcd_precond with the Schur step (plain and with the viscous
    term), the residual update, the v sweeps, the cross term and the u
    sweeps all on the vector kernels."""
    rng = np.random.default_rng(62)
    prm = two_phase_params(pcd_sweeps=3, pcd_visc_scale=visc, vec_rows=1)
    o = oracle_mod.Oracle(grid, prm)
    pr = _props(o, grid, rng)
    z = [rfield(rng, grid, k) for k in ("u", "v", "cell")]
    ua, va = rfield(rng, grid, "u"), rfield(rng, grid, "v")
    pen = (np.abs(rfield(rng, grid, "u")) * 1e3, np.abs(rfield(rng, grid, "v")) * 1e3) if penalty else (None, None)
    rg = [grid.zeros(k) for k in ("u", "v", "cell")]
    ro = [grid.zeros(k) for k in ("u", "v", "cell")]
    with Context(grid, prm) as ctx:
        ctx.apply_pcd_precond(*z, *rg, ua, va, pr["rho_u"], pr["rho_v"], pr["kappa"], pr["zeta"], pr["eta"], 2e-3,
                              *pen)
    o.pcd(*z, *ro, ua, va, pr, 2e-3, *pen)
    for a, b in zip(rg, ro):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("name", ["droplet", "bubble_freeslip", "poiseuille"])
def test_mixed_form_vec_rows_bitwise(gpu, name):
    """The FP32 inner solve (flexible GMRES + PCD, FMA in the sweeps) with the
    vector kernels gives the bits and iteration counts of the scalar ones."""
    over = dict(refine=2, refine_inner_tol=1e-2, refine_max_inner=30, refine_max_outer=30, krylov_bc_fix=1,
                tol_bicgstab2=1e-9, pcg_cap_start=4, pcd_sweeps=3, pcd_sweeps_max=12, pcd_visc_scale=1.0, graphs=1)
    runs = {m: _device_run(name, dict(over, vec_rows=m), 1, False) for m in (-1, 1)}
    (s0, h0, _), (s1, h1, _) = runs[-1], runs[1]
    for a, b in zip(h0, h1):
        assert a == b
    for k in STATE:
        np.testing.assert_array_equal(s0[k], s1[k], err_msg=k)


def test_size_rule_takes_vector_kernels_bitwise(gpu):
    """A 1024 x 1024 box has 1040 x 1029 = 1,070,160 points, above the 2^20
    of the size rule for the PCD's Schur, residual and cross steps and below
    the 2^21 of the wall-bounded sweeps: one PCD application with vec_rows =
    0 equals the one with the scalar kernels (vec_rows = -1) bit for bit, in
    FP64."""
    g = Grid(1024, 1024)
    rng = np.random.default_rng(63)
    pitch = (g.nx + 5 + 15) // 16 * 16  # the box: rows padded to 16 elements, ny + 5 rows
    assert pitch * (g.ny + 5) >= 1 << 20
    from oracle import oracle as o  # the coefficient fields only

    base = two_phase_params(pcd_sweeps=4, pcd_visc_scale=1.0)
    pr = o.Oracle(g, base).properties(colour(rng, g))
    z = [rfield(rng, g, k) for k in ("u", "v", "cell")]
    ua, va = rfield(rng, g, "u"), rfield(rng, g, "v")
    out = {}
    for m in (-1, 0):
        r = [g.zeros(k) for k in ("u", "v", "cell")]
        with Context(g, base.with_(vec_rows=m)) as ctx:
            ctx.apply_pcd_precond(*z, *r, ua, va, pr["rho_u"], pr["rho_v"], pr["kappa"], pr["zeta"], pr["eta"],
                                  2e-3, None, None)
        out[m] = r
    for a, b in zip(out[-1], out[0]):
        np.testing.assert_array_equal(a, b)
