"""Numerical failure paths of the coupled step, on the GPU, without faulting
it.  The reference's solvers leave their loops silently on breakdown or at
the iteration cap (``src/mod_bicgstab2.f90:148,197,240``); here every device
loop has a cap and the step reports a status word that the host reads:
FUGU_CONVERGED 0, FUGU_MAXITER 1, FUGU_BREAKDOWN 2, FUGU_NAN 3.

- a NaN planted in an input field is reported as FUGU_NAN, and the same
  context then steps a clean state to the oracle's bits;
- an iteration cap below what the tolerance needs is reported as FUGU_MAXITER
  after exactly that many iterations, with the oracle's state;
- a zero right-hand side converges at once to the zero solution, as in the
  oracle;
- a grid barrier of the persistent PCG kernel that waits in vain (the test
  hook makes it wait for one CTA more than the launch has) gives up after its
  poll limit: the call reports FUGU_ETIMEOUT with a message, and the same
  context then solves a clean case to the oracle's bits.  No wait is
  unbounded, so nothing hangs the GPU.
"""
import numpy as np
import pytest

from conftest import GRIDS, rfield, two_phase_params
from coupled_codefort_2d_b200._lib import FuguError
from coupled_codefort_2d_b200.context import Context
from coupled_codefort_2d_b200.layout import Grid
from coupled_codefort_2d_b200.params import Params

pytestmark = pytest.mark.gpu

STATE = ["u_vel", "v_vel", "p_field", "c_field", "u_prev", "v_prev", "rho_c", "rho_u", "rho_v", "kappa",
         "zeta", "eta", "kappa_curv", "f_sigma_u", "f_sigma_v"]
FUGU_CONVERGED, FUGU_MAXITER, FUGU_NAN = 0, 1, 3
FUGU_ETIMEOUT = -5


def cavity():
    g = Grid(24, 24)
    p = Params(rho1=1.0, rho2=1.0, mu1=0.01, mu2=0.01, sigma=0.0, gx=0.0, gy=0.0, time_order=1,
               tol_bicgstab2=1e-8, max_iter_bicgstab2=100)
    return g, p


def test_nan_input_is_reported_and_the_context_recovers(gpu, oracle_mod):
    g, p = cavity()
    st_o = oracle_mod.new_state(g, g.full("cell", 1.0), p)
    bad = {k: a.copy(order="F") for k, a in st_o.items()}
    bad["u_vel"][8, 9] = np.nan  # an interior u face
    clean = {k: a.copy(order="F") for k, a in st_o.items()}
    o = oracle_mod.Oracle(g, p)
    with Context(g, p) as ctx:
        r = ctx.advance_coupled_step(*[bad[k] for k in STATE], 1e-2, 1, use_bicgstab2=False, u_top_lid=1.0)
        assert r["status"] == FUGU_NAN, r
        r = ctx.advance_coupled_step(*[clean[k] for k in STATE], 1e-2, 1, use_bicgstab2=False, u_top_lid=1.0)
    so = o.step(st_o, 1e-2, 1, use_bicgstab2=False, u_top_lid=1.0)
    assert r["status"] == FUGU_CONVERGED and r["iter"] == so.iter
    for k in STATE:
        np.testing.assert_array_equal(clean[k], st_o[k], err_msg=k)


@pytest.mark.parametrize("use_b2", [False, True])
def test_iteration_cap_is_reported(gpu, oracle_mod, use_b2):
    g, p = cavity()
    st_o = oracle_mod.new_state(g, g.full("cell", 1.0), p)
    st_g = {k: a.copy(order="F") for k, a in st_o.items()}
    o = oracle_mod.Oracle(g, p)
    with Context(g, p) as ctx:
        r = ctx.advance_coupled_step(*[st_g[k] for k in STATE], 1e-2, 1, use_bicgstab2=use_b2, u_top_lid=1.0,
                                     tol_in=1e-14, max_iter_in=2)
    so = o.step(st_o, 1e-2, 1, use_bicgstab2=use_b2, u_top_lid=1.0, tol=1e-14, max_iter=2)
    assert r["status"] == FUGU_MAXITER, r
    assert r["iter"] == so.iter == 2
    for k in STATE:
        np.testing.assert_array_equal(st_g[k], st_o[k], err_msg=k)


def test_zero_right_hand_side_converges_at_once(gpu, oracle_mod):
    g, p = cavity()
    st_o = oracle_mod.new_state(g, g.full("cell", 1.0), p)
    st_g = {k: a.copy(order="F") for k, a in st_o.items()}
    o = oracle_mod.Oracle(g, p)
    with Context(g, p) as ctx:  # at rest, no lid, no body force, no surface tension: B = 0
        r = ctx.advance_coupled_step(*[st_g[k] for k in STATE], 1e-2, 1, use_bicgstab2=False)
    so = o.step(st_o, 1e-2, 1, use_bicgstab2=False)
    assert r["status"] == FUGU_CONVERGED, r
    assert r["iter"] == so.iter
    for k in ("u_vel", "v_vel", "p_field"):
        assert not np.any(st_g[k]), k
        np.testing.assert_array_equal(st_g[k], st_o[k], err_msg=k)


def poisson_case(o, g, seed):
    rng = np.random.default_rng(seed)
    c = np.asfortranarray(rng.uniform(0.0, 1.0, size=g.shape("cell")))
    pr = o.properties(c)
    rhs = rfield(rng, g, "cell")
    phi0 = rfield(rng, g, "cell", -0.1, 0.1)
    return pr, rhs, phi0


def test_grid_barrier_timeout_is_reported_and_the_context_recovers(gpu, oracle_mod):
    g, prm = GRIDS["walls_32x24"], two_phase_params()
    o = oracle_mod.Oracle(g, prm)
    pr, rhs, phi0 = poisson_case(o, g, 31)
    with Context(g, prm) as ctx:
        ctx.arm_barrier_timeout(1000)
        with pytest.raises(FuguError) as ei:
            ctx.solve_poisson_pressure(phi0.copy(order="F"), rhs, pr["rho_u"], pr["rho_v"], 1e-5, 150)
        assert ei.value.code == FUGU_ETIMEOUT and "gave up" in str(ei.value)
        pg = phi0.copy(order="F")
        itg, resg = ctx.solve_poisson_pressure(pg, rhs, pr["rho_u"], pr["rho_v"], 1e-5, 150)
    po = phi0.copy(order="F")
    ito, reso = o.poisson(po, rhs, pr["rho_u"], pr["rho_v"], 1e-5, 150)
    assert (itg, resg) == (ito, reso)
    np.testing.assert_array_equal(pg, po)


def test_grid_barrier_timeout_inside_a_step(gpu, oracle_mod):
    """The hook armed before a whole step: its first PCG launch gives up, the
    step reports FUGU_ETIMEOUT, and the next step on clean inputs equals the
    oracle's bit for bit."""
    g, p = cavity()
    st_o = oracle_mod.new_state(g, g.full("cell", 1.0), p)
    clean = {k: a.copy(order="F") for k, a in st_o.items()}
    first = {k: a.copy(order="F") for k, a in st_o.items()}
    o = oracle_mod.Oracle(g, p)
    with Context(g, p) as ctx:
        ctx.arm_barrier_timeout(1000)
        with pytest.raises(FuguError) as ei:
            ctx.advance_coupled_step(*[first[k] for k in STATE], 1e-2, 1, use_bicgstab2=False, u_top_lid=1.0)
        assert ei.value.code == FUGU_ETIMEOUT
        r = ctx.advance_coupled_step(*[clean[k] for k in STATE], 1e-2, 1, use_bicgstab2=False, u_top_lid=1.0)
    so = o.step(st_o, 1e-2, 1, use_bicgstab2=False, u_top_lid=1.0)
    assert r["status"] == FUGU_CONVERGED and r["iter"] == so.iter
    for k in STATE:
        np.testing.assert_array_equal(clean[k], st_o[k], err_msg=k)
