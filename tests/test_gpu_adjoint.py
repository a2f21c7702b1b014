"""Discrete adjoint of the coupled solve (extension; the reference has none).

1. The probed transpose is the transpose: <A x, y> = <x, A^T y> over the owned
   unknowns, for wall-bounded and periodic grids, with penalty and AMP
   coefficients, to 1e-12 relative (the probe reproduces the operator exactly;
   the two sums differ by rounding only).
2. The adjoint solve is dual to the forward solve: for A X = B and
   A^T lambda = g, g . X = lambda . B to 1e-9, with flexible GMRES and with
   BiCGStab(2) as the inner solver of the defect correction.
3. The steady two-phase Poiseuille gradient dJ/dmu (J = mean velocity) from
   the adjoint equals central finite differences of the GPU forward solve
   (h = 1e-5 relative) to 1e-6, and the analytic derivative of the two-layer
   profile to the discretisation error (2 %), also through the
   torch.autograd.Function harness.
4. The start-up of the same channel over 12 BDF steps: the harness's time
   stepping equals fugu_step on the device state, and the multi-step adjoint
   with checkpointing (every 4th state kept, the rest recomputed) equals
   central finite differences to 1e-6.
"""
import numpy as np
import pytest

from conftest import GRIDS, colour, rfield, two_phase_params
from coupled_codefort_2d_b200 import adjoint
from coupled_codefort_2d_b200.context import Context
from coupled_codefort_2d_b200.layout import Grid
from coupled_codefort_2d_b200.params import Params

pytestmark = pytest.mark.gpu


def coefs(ctx, g, rng):
    c = colour(rng, g)
    pr = {k: g.zeros(kd) for k, kd in (("rho_c", "cell"), ("rho_u", "u"), ("rho_v", "v"), ("kappa", "cell"),
                                        ("zeta", "vert"), ("eta", "vert"))}
    ctx.compute_mixture_densities(c, pr["rho_c"], pr["rho_u"], pr["rho_v"])
    ctx.compute_mixture_viscosities(c, pr["kappa"], pr["zeta"], pr["eta"])
    ua, va = rfield(rng, g, "u"), rfield(rng, g, "v")
    return ua, va, pr


def owned_random(rng, g):
    return [np.where(m, rfield(rng, g, k), 0.0) for m, k in zip(adjoint.owned_masks(g), ("u", "v", "cell"))]


@pytest.mark.parametrize("name", ["walls_13x9", "walls_32x24", "px_16x12", "py_12x16", "pxy_10x14"])
@pytest.mark.parametrize("extra", ["plain", "penalty", "amp"])
def test_transpose_dot_product(gpu, name, extra):
    g = GRIDS[name]
    rng = np.random.default_rng(31)
    prm = two_phase_params()
    with Context(g, prm) as ctx:
        ua, va, pr = coefs(ctx, g, rng)
        kw = {}
        if extra == "penalty":
            kw = dict(penalty_u=np.abs(rfield(rng, g, "u")) * 1e3, penalty_v=np.abs(rfield(rng, g, "v")) * 1e3)
        if extra == "amp":
            kw = dict(mdot_u_cons=rfield(rng, g, "u"), mdot_v_cons=rfield(rng, g, "v"))
        x, y = owned_random(rng, g), owned_random(rng, g)
        xb = [a.copy(order="F") for a in x]
        ctx.apply_velocity_bcs(xb[0], xb[1], None)
        Ax = [g.zeros(k) for k in ("u", "v", "cell")]
        ctx.matvec_coupled(*xb, *Ax, ua, va, pr["rho_c"], pr["rho_u"], pr["rho_v"], pr["kappa"], pr["zeta"],
                           pr["eta"], 2e-3, **kw)
        ATy = [g.zeros(k) for k in ("u", "v", "cell")]
        ctx.matvec_coupled_t(*y, *ATy, ua, va, pr["rho_c"], pr["rho_u"], pr["rho_v"], pr["kappa"], pr["zeta"],
                             pr["eta"], 2e-3, **kw)
    lhs = adjoint.owned_dot(g, Ax, y)
    rhs = adjoint.owned_dot(g, x, ATy)
    scale = sum(float(np.sum(np.abs(a[m]) * np.abs(b[m]))) for a, b, m in zip(Ax, y, adjoint.owned_masks(g)))
    assert abs(lhs - rhs) <= 1e-12 * scale, (lhs, rhs)
    # nothing outside the owned set
    for a, m in zip(ATy, adjoint.owned_masks(g)):
        assert not np.any(a[~m])


@pytest.mark.parametrize("refine", [2, 1])
def test_adjoint_solve_is_dual_to_the_forward_solve(gpu, refine):
    """A two-phase system of a step: a circular interface (density ratio 10)
    and a mild advecting velocity; random right-hand sides.  refine 2: both
    solves are the defect correction around flexible GMRES; refine 1: around
    BiCGStab(2), the forward solve on A and the adjoint one on S A^T S."""
    from coupled_codefort_2d_b200 import cases

    g = Grid(24, 32, periodic_x=True)
    rng = np.random.default_rng(32)
    prm = two_phase_params(refine=refine, refine_inner_tol=1e-2, refine_max_inner=30, refine_max_outer=200,
                           krylov_bc_fix=1, tol_bicgstab2=1e-10)
    with Context(g, prm) as ctx:
        c = cases.binary_circle(g, 0.5, 0.5, 0.25, inside=1.0)
        pr = {k: g.zeros(kd) for k, kd in (("rho_c", "cell"), ("rho_u", "u"), ("rho_v", "v"), ("kappa", "cell"),
                                            ("zeta", "vert"), ("eta", "vert"))}
        ctx.compute_mixture_densities(c, pr["rho_c"], pr["rho_u"], pr["rho_v"])
        ctx.compute_mixture_viscosities(c, pr["kappa"], pr["zeta"], pr["eta"])
        ua, va = 0.1 * rfield(rng, g, "u"), 0.1 * rfield(rng, g, "v")
        co = (ua, va, pr["rho_c"], pr["rho_u"], pr["rho_v"], pr["kappa"], pr["zeta"], pr["eta"])
        B = owned_random(rng, g)
        B[2][...] = 0.0  # compatible with the pressure null space
        gv = owned_random(rng, g)
        gv[2][...] = 0.0
        X = [g.zeros(k) for k in ("u", "v", "cell")]
        st = ctx.bicgstab2_solve(*X, *B, *co, 2e-3, tol_in=1e-10, max_iter_in=500)
        lam = [g.zeros(k) for k in ("u", "v", "cell")]
        ast = ctx.adjoint_solve(*gv, *lam, *co, 2e-3, tol=1e-10)
        assert st["res"] < 1e-10 and st["status"] == 0, st
        assert ast["res"] < 1e-10 and ast["status"] == 0, ast
        r = [g.zeros(k) for k in ("u", "v", "cell")]
        ctx.matvec_coupled_t(*lam, *r, *co, 2e-3)
    res = np.sqrt(sum(float(np.sum((a[m] - b[m]) ** 2)) for a, b, m in zip(r, gv, adjoint.owned_masks(g))))
    assert res <= 1e-8 * np.sqrt(adjoint.owned_dot(g, gv, gv))
    # g.X - lambda.B = (g - A^T lambda).X + lambda.(A X - B): bounded by the
    # two residuals times the other vector
    gx, lb = adjoint.owned_dot(g, gv, X), adjoint.owned_dot(g, lam, B)

    def nrm(t):
        return np.sqrt(adjoint.owned_dot(g, t, t))

    assert abs(gx - lb) <= 1e-9 * (nrm(gv) * nrm(X) + nrm(lam) * nrm(B)), (gx, lb)


@pytest.fixture(scope="module")
def poiseuille(gpu):
    p = adjoint.SteadyPoiseuille(nx=32, ny=64)
    yield p
    p.close()


def test_poiseuille_gradient_matches_fd_and_analytic(poiseuille):
    mu1, mu2 = 1.0, 0.1  # viscosity ratio 10
    J, grads, st = poiseuille.value_and_grad(mu1, mu2)
    assert st["forward"]["status"] == 0 and st["adjoint"]["status"] == 0
    h1, h2 = 1e-5 * mu1, 1e-5 * mu2
    fd1 = (poiseuille.value(mu1 + h1, mu2) - poiseuille.value(mu1 - h1, mu2)) / (2 * h1)
    fd2 = (poiseuille.value(mu1, mu2 + h2) - poiseuille.value(mu1, mu2 - h2)) / (2 * h2)
    assert abs(grads[0] - fd1) <= 1e-6 * abs(fd1), (grads[0], fd1)
    assert abs(grads[1] - fd2) <= 1e-6 * abs(fd2), (grads[1], fd2)
    a1, a2 = adjoint.analytic_grad(mu1, mu2)
    assert abs(J - adjoint.analytic_mean_velocity(mu1, mu2)) <= 2e-2 * abs(J)
    assert abs(grads[0] - a1) <= 2e-2 * abs(a1), (grads[0], a1)
    assert abs(grads[1] - a2) <= 2e-2 * abs(a2), (grads[1], a2)
    # d J / d(mu ratio) with mu1 fixed: mu2 = mu1 / r
    r = mu1 / mu2
    dJ_dr = -grads[1] * mu1 / r ** 2
    assert np.sign(dJ_dr) == np.sign(-a2 * mu1 / r ** 2)


def test_torch_autograd_harness(poiseuille):
    import torch

    f = adjoint.torch_flux_function(poiseuille)
    mu = torch.tensor([1.0, 0.1], dtype=torch.float64, requires_grad=True)
    J = f(mu)
    (2.0 * J).backward()
    _, grads, _ = poiseuille.value_and_grad(1.0, 0.1)
    np.testing.assert_allclose(mu.grad.numpy(), 2.0 * np.array(grads), rtol=1e-12)


@pytest.fixture(scope="module")
def startup(gpu):
    p = adjoint.StartupPoiseuille(nx=16, ny=32, nsteps=12, dt=0.05, checkpoint=4)
    yield p
    p.close()


def test_startup_forward_is_the_device_step(startup):
    """The multi-step harness's time stepping equals advance_coupled_step on
    the device-resident state (fugu_step): the coefficients it holds fixed do
    not move in this flow."""
    from coupled_codefort_2d_b200 import cases
    from oracle import oracle as O

    mu1, mu2 = 1.0, 0.1
    J, XN = startup.trajectory_value(mu1, mu2)
    g = startup.g
    p = startup.params(mu1, mu2)
    st = O.new_state(g, cases.initial_colour(g, "poiseuille"), p)
    with Context(g, p) as ctx:
        ctx.upload_state(st)
        opts = ctx.step_opts(use_bicgstab2=True)
        for s in range(1, startup.nsteps + 1):
            ctx.step(startup.dt, s, opts)
        u = ctx.download("u_vel")
        c = ctx.download("c_field")
    mu_, _, _ = adjoint.owned_masks(g)
    assert np.linalg.norm(u[mu_] - XN[0][mu_]) <= 1e-9 * np.linalg.norm(XN[0][mu_])
    np.testing.assert_allclose(c, st["c_field"], rtol=0, atol=1e-12)  # the layers do not move


def test_startup_gradient_with_checkpointing_matches_fd(startup):
    mu1, mu2 = 1.0, 0.1
    J, grads, _ = startup.value_and_grad(mu1, mu2)
    assert startup.kept_states < startup.nsteps and startup.recomputed_steps > 0
    h1, h2 = 1e-5 * mu1, 1e-5 * mu2
    fd1 = (startup.value(mu1 + h1, mu2) - startup.value(mu1 - h1, mu2)) / (2 * h1)
    fd2 = (startup.value(mu1, mu2 + h2) - startup.value(mu1, mu2 - h2)) / (2 * h2)
    assert abs(grads[0] - fd1) <= 1e-6 * abs(fd1), (grads[0], fd1)
    assert abs(grads[1] - fd2) <= 1e-6 * abs(fd2), (grads[1], fd2)
    # the start-up is still far from the steady profile: the gradient differs from the steady one
    assert J < adjoint.analytic_mean_velocity(mu1, mu2)
