"""Routine-level parity: every CUDA routine of the hot path against the CPU
oracle on identical seeded inputs (ghost cells included, because ghost
contents are part of the reference's operator semantics).

Tolerance: BIT-EXACT for every routine.  Element-wise kernels are compiled
without FMA contraction and keep the reference's operand order; reductions
(coupled_dot, the PCG scalars) accumulate a double-double on both sides and
round once, which on these inputs gives the correctly rounded sum in any
summation order.  The same routines are bit-exact at 256^2 and 320 x 640
too; whole solves at those sizes are compared within tolerance in
``test_gpu_configs.py``.
"""
import numpy as np
import pytest

from conftest import GRIDS, colour, rfield, two_phase_params
from coupled_codefort_2d_b200.context import Context
from coupled_codefort_2d_b200.layout import Grid
from coupled_codefort_2d_b200.params import Params

pytestmark = pytest.mark.gpu

# the small grids plus the droplet and rising-bubble sizes (256^2 takes the
# cluster-resident PCG, 320 x 640 the grid-wide one)
ROUTINE_GRIDS = {**GRIDS, "walls_256x256": Grid(256, 256), "walls_320x640": Grid(320, 640, 1.0, 2.0)}
GRID_IDS = list(ROUTINE_GRIDS)


def exact(a, b):
    np.testing.assert_array_equal(a, b)


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(params=GRID_IDS)
def grid(request):
    return ROUTINE_GRIDS[request.param]


def props(o, g, rng, prm):
    c = colour(rng, g)
    return c, o.properties(c)


def test_halo_exchange(gpu, oracle_mod, grid):
    rng = np.random.default_rng(1)
    prm = Params()
    o = oracle_mod.Oracle(grid, prm)
    with Context(grid, prm) as ctx:
        for kind in ("cell", "u", "v"):
            a = rfield(rng, grid, kind)
            ref = a.copy(order="F")
            o.halo(kind, ref)
            ctx.halo(kind, a)
            exact(a, ref)


def test_properties(gpu, oracle_mod, grid):
    rng = np.random.default_rng(2)
    for prm in (two_phase_params(), Params(mu1=0.1, mu2=0.1, rho1=1.0, rho2=1.0)):
        o = oracle_mod.Oracle(grid, prm)
        c = colour(rng, grid)
        ref = o.properties(c)
        with Context(grid, prm) as ctx:
            out = {k: grid.zeros(v) for k, v in (("rho_c", "cell"), ("rho_u", "u"), ("rho_v", "v"),
                                                  ("kappa", "cell"), ("zeta", "vert"), ("eta", "vert"))}
            ctx.compute_mixture_densities(c, out["rho_c"], out["rho_u"], out["rho_v"])
            ctx.compute_mixture_viscosities(c, out["kappa"], out["zeta"], out["eta"])
        for k in out:
            exact(out[k], ref[k])


def test_operators(gpu, oracle_mod, grid):
    rng = np.random.default_rng(3)
    prm = two_phase_params()
    o = oracle_mod.Oracle(grid, prm)
    c, pr = props(o, grid, rng, prm)
    u, v, p = rfield(rng, grid, "u"), rfield(rng, grid, "v"), rfield(rng, grid, "cell")
    ua, va = rfield(rng, grid, "u"), rfield(rng, grid, "v")
    mdu, mdv = rfield(rng, grid, "u", 0, 5), rfield(rng, grid, "v", 0, 5)
    with Context(grid, prm) as ctx:
        d_g, d_o = grid.zeros("cell"), grid.zeros("cell")
        ctx.op_divergence(u, v, d_g)
        o.divergence(u, v, d_o)
        exact(d_g, d_o)
        gu, gv, ou, ov = grid.zeros("u"), grid.zeros("v"), grid.zeros("u"), grid.zeros("v")
        ctx.op_grad_pressure(p, gu, gv)
        o.grad_pressure(p, ou, ov)
        exact(gu, ou)
        exact(gv, ov)
        ctx.op_viscous_stress(u, v, pr["kappa"], pr["zeta"], pr["eta"], gu, gv)
        o.viscous_stress(u, v, pr["kappa"], pr["zeta"], pr["eta"], ou, ov)
        exact(gu, ou)
        exact(gv, ov)
        for cons in (False, True):
            m = (mdu, mdv) if cons else (None, None)
            ctx.op_advection(ua, va, pr["rho_c"], pr["rho_u"], pr["rho_v"], u, v, gu, gv, *m)
            o.advection(ua, va, pr["rho_c"], pr["rho_u"], pr["rho_v"], u, v, ou, ov, *m)
            exact(gu, ou)
            exact(gv, ov)


@pytest.mark.parametrize("lid", [None, 1.0])
@pytest.mark.parametrize("free_slip", [0, 1])
def test_velocity_bcs(gpu, oracle_mod, grid, lid, free_slip):
    rng = np.random.default_rng(4)
    prm = Params(free_slip_x=free_slip)
    o = oracle_mod.Oracle(grid, prm)
    u, v = rfield(rng, grid, "u"), rfield(rng, grid, "v")
    ru, rv = u.copy(order="F"), v.copy(order="F")
    with Context(grid, prm) as ctx:
        ctx.apply_velocity_bcs(u, v, lid)
    o.velocity_bcs(ru, rv, lid)
    exact(u, ru)
    exact(v, rv)


@pytest.mark.parametrize("variant", ["plain", "no_adv", "penalty", "amp"])
def test_matvec_coupled(gpu, oracle_mod, grid, variant):
    rng = np.random.default_rng(5)
    prm = two_phase_params()
    o = oracle_mod.Oracle(grid, prm)
    c, pr = props(o, grid, rng, prm)
    X = [rfield(rng, grid, k) for k in ("u", "v", "cell")]
    Xo = [a.copy(order="F") for a in X]
    ua, va = rfield(rng, grid, "u"), rfield(rng, grid, "v")
    pen = (rfield(rng, grid, "u", 0, 1e12), rfield(rng, grid, "v", 0, 1e12)) if variant == "penalty" else (None, None)
    amp = (rfield(rng, grid, "u", 0, 5), rfield(rng, grid, "v", 0, 5)) if variant == "amp" else (None, None)
    Yg = [grid.zeros(k) for k in ("u", "v", "cell")]
    Yo = [grid.zeros(k) for k in ("u", "v", "cell")]
    dt = 3.7e-3
    with Context(grid, prm) as ctx:
        ctx.matvec_coupled(*X, *Yg, ua, va, pr["rho_c"], pr["rho_u"], pr["rho_v"], pr["kappa"], pr["zeta"],
                           pr["eta"], dt, variant != "no_adv", pen[0], pen[1], amp[0], amp[1])
    o.matvec(*Xo, *Yo, ua, va, pr, dt, variant != "no_adv", pen[0], pen[1], amp[0], amp[1])
    for a, b in zip(Yg, Yo):
        exact(a, b)
    for a, b in zip(X, Xo):  # X is intent(inout): halo'd ghosts must match
        exact(a, b)


@pytest.mark.parametrize("use_pen", [False, True])
@pytest.mark.parametrize("smoother", [0, 1])
def test_helmholtz_sweeps(gpu, oracle_mod, grid, use_pen, smoother):
    """damped Jacobi (the reference) and the red-black SOR extension"""
    rng = np.random.default_rng(6)
    prm = two_phase_params(pcd_smoother=smoother, pcd_sor_omega=1.5)
    o = oracle_mod.Oracle(grid, prm)
    c, pr = props(o, grid, rng, prm)
    with Context(grid, prm) as ctx:
        for kind, gfn, ofn in (("u", ctx.solve_helmholtz_u, o.helmholtz_u), ("v", ctx.solve_helmholtz_v, o.helmholtz_v)):
            sol, rhs = rfield(rng, grid, kind), rfield(rng, grid, kind)
            pen = rfield(rng, grid, kind, 0, 1e6) if use_pen else None
            ref = sol.copy(order="F")
            for n in (1, 3, 4):
                s = sol.copy(order="F")
                r = ref.copy(order="F")
                rho = pr["rho_u"] if kind == "u" else pr["rho_v"]
                gfn(s, rhs, rho, pr["kappa"], pr["zeta"], pr["eta"], 2e-3, n, pen)
                ofn(r, rhs, pr, 2e-3, n, pen)
                exact(s, r)


def test_vof_advection(gpu, oracle_mod, grid):
    rng = np.random.default_rng(7)
    for lim in (0, 1):
        prm = Params(limiter=lim)
        o = oracle_mod.Oracle(grid, prm)
        c = colour(rng, grid)
        u, v = rfield(rng, grid, "u", -2, 2), rfield(rng, grid, "v", -2, 2)
        dt = 0.2 * min(grid.dx, grid.dy) / 2
        cg, co = grid.zeros("cell"), grid.zeros("cell")
        fxg, fyg, fxo, fyo = grid.zeros("u"), grid.zeros("v"), grid.zeros("u"), grid.zeros("v")
        with Context(grid, prm) as ctx:
            ctx.vof_advection_tvd(c, cg, u, v, dt, fxg, fyg)
        o.vof(c, co, u, v, dt, fxo, fyo)
        exact(cg, co)
        exact(fxg, fxo)
        exact(fyg, fyo)


def test_svof_curvature_csf(gpu, oracle_mod, grid):
    from coupled_codefort_2d_b200 import cases

    prm = Params(sigma=1.3)
    o = oracle_mod.Oracle(grid, prm)
    c = cases.binary_circle(grid, 0.5 * grid.Lx, 0.5 * grid.Ly, 0.3 * min(grid.Lx, grid.Ly), 1.0)
    delta = 1.5 * min(grid.dx, grid.dy)
    cs_g, cs_o = grid.zeros("cell"), grid.zeros("cell")
    with Context(grid, prm) as ctx:
        it_g = ctx.svof_helmholtz_filter(c, cs_g, delta, 150, 1e-7)
        it_o = o.svof(c, cs_o, delta, 150, 1e-7)
        assert it_g == it_o
        exact(cs_g, cs_o)
        kg, ko = grid.zeros("cell"), grid.zeros("cell")
        ctx.compute_interface_curvature(cs_g, kg)
        o.curvature(cs_o, ko)
        exact(kg, ko)
        fu, fv, gu, gv = grid.zeros("u"), grid.zeros("v"), grid.zeros("u"), grid.zeros("v")
        ctx.compute_csf_force(c, kg, fu, fv)
        o.csf(c, ko, gu, gv)
        exact(fu, gu)
        exact(fv, gv)


def test_cylinder_mask_and_dt(gpu, oracle_mod, grid):
    rng = np.random.default_rng(8)
    prm = two_phase_params()
    o = oracle_mod.Oracle(grid, prm)
    with Context(grid, prm) as ctx:
        pu, pv = ctx.build_cylinder_mask(0.5, 0.4, 0.2)
        ou, ov = o.cylinder_mask(0.5, 0.4, 0.2)
        exact(pu, ou)
        exact(pv, ov)
        u, v = rfield(rng, grid, "u"), rfield(rng, grid, "v")
        assert ctx.compute_adaptive_dt(u, v, 1e-2) == o.adaptive_dt(u, v, 1e-2)


def test_coupled_dot(gpu, oracle_mod, grid):
    rng = np.random.default_rng(9)
    prm = Params()
    o = oracle_mod.Oracle(grid, prm)
    a = [rfield(rng, grid, k) for k in ("u", "v", "cell")]
    b = [rfield(rng, grid, k) for k in ("u", "v", "cell")]
    with Context(grid, prm) as ctx:
        dg = ctx.coupled_dot(*a, *b)
    do = o.coupled_dot(a, b)
    assert dg == do, (dg, do)


@pytest.fixture(params=["auto", "grid"])
def pcg_variant(request, monkeypatch):
    """auto: the cluster-resident PCG when the grid fits one thread-block
    cluster (all the grids here do); grid: the grid-wide persistent kernel."""
    monkeypatch.setenv("FUGU_PCG", request.param)
    return request.param


@pytest.mark.parametrize("zero_init", [True, False])
def test_poisson_pcg(gpu, oracle_mod, grid, zero_init, pcg_variant):
    rng = np.random.default_rng(10)
    prm = two_phase_params()
    o = oracle_mod.Oracle(grid, prm)
    c, pr = props(o, grid, rng, prm)
    rhs = rfield(rng, grid, "cell")
    phi0 = grid.zeros("cell") if zero_init else rfield(rng, grid, "cell", -0.1, 0.1)
    pg, po = phi0.copy(order="F"), phi0.copy(order="F")
    with Context(grid, prm) as ctx:
        itg, resg = ctx.solve_poisson_pressure(pg, rhs, pr["rho_u"], pr["rho_v"], 1e-5, 150)
    ito, reso = o.poisson(po, rhs, pr["rho_u"], pr["rho_v"], 1e-5, 150)
    assert (itg, resg) == (ito, reso)
    exact(pg, po)


@pytest.mark.parametrize("sweeps,penalty,smoother,visc", [(3, False, 0, 0.0), (4, True, 0, 0.0), (3, True, 1, 0.0),
                                                         (3, False, 0, 1.0)])
def test_pcd_precond(gpu, oracle_mod, grid, pcg_variant, sweeps, penalty, smoother, visc):
    """apply_pcd_precond: 3 sweeps (odd: the Jacobi result is copied back),
    4 sweeps with the Darcy penalty diagonal, 3 red-black SOR sweeps, and the
    viscous (Cahouet-Chabard) term in the Schur step."""
    rng = np.random.default_rng(11)
    prm = two_phase_params(pcd_sweeps=sweeps, pcd_smoother=smoother, pcd_sor_omega=1.5, pcd_visc_scale=visc)
    o = oracle_mod.Oracle(grid, prm)
    c, pr = props(o, grid, rng, prm)
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
        exact(a, b)
