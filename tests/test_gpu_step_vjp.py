"""The vector-Jacobian product of one coupled step (``fugu_step_vjp``) and the
multi-step rising-bubble gradient built on it, against central differences
of the GPU forward step.

The step clips C to [0, 1] after transport, and a cell of pure fluid 1 sits
on that clip: its new value is 1 - dt div(u), with div(u) at the solve's
tolerance.  A perturbation of u that changes div(u) by more than that crosses
the clip, so central differences along it mix two branches.  Velocity
directions are therefore divergence-free (from a stream function that
vanishes on the walls), as the solve's own responses are; the colour is
perturbed on interface cells only.  The adjoint is the derivative of the
branches the step took.

Tolerances: relative 1e-5 for one step (h = 1e-5), 1e-5 for the gradient of
the centroid height after 8 steps (h = 1e-4 relative; 1e-6 leaves the
central difference with solver noise of the same size as the error sought).
"""
import numpy as np
import pytest

from coupled_codefort_2d_b200.adjoint import RisingBubble
from coupled_codefort_2d_b200.context import VJP_STATE, Context
from coupled_codefort_2d_b200._lib import FuguError
from coupled_codefort_2d_b200.layout import Grid, at
from coupled_codefort_2d_b200.params import Params

pytestmark = pytest.mark.gpu

DT = 2.5e-3


def bubble(nsteps, checkpoint=3):
    return RisingBubble(nx=24, ny=48, nsteps=nsteps, T=nsteps * DT, checkpoint=checkpoint, tol=1e-13)


def divergence_free(rng, g):
    """(u, v) = (d psi/dy, -d psi/dx) on the MAC faces, psi random at the
    vertices and zero on the walls: the discrete divergence vanishes and so
    do the wall faces."""
    psi = np.zeros((g.nx + 1, g.ny + 1))
    psi[1:-1, 1:-1] = rng.standard_normal((g.nx - 1, g.ny - 1))
    du, dv = g.zeros("u"), g.zeros("v")
    at(du, "u", slice(0, g.nx), slice(1, g.ny))[...] = (psi[:, 1:] - psi[:, :-1]) / g.dy
    at(dv, "v", slice(1, g.nx), slice(0, g.ny))[...] = -(psi[1:, :] - psi[:-1, :]) / g.dx
    s = max(np.abs(du).max(), np.abs(dv).max())  # unit entries: h d stays well below u
    return du / s, dv / s


def interface_cells(g, c, rng):
    d = g.zeros("cell")
    ci = at(c, "cell", slice(1, g.nx), slice(1, g.ny))
    m = (ci > 0.02) & (ci < 0.98)
    at(d, "cell", slice(1, g.nx), slice(1, g.ny))[...] = np.where(m, rng.standard_normal(ci.shape), 0.0)
    return d


@pytest.fixture(scope="module")
def one_step(gpu):
    """The state before step 4 of the small bubble, random adjoints of the
    state after it, and the step's VJP."""
    pb = bubble(3)
    g = pb.g
    rng = np.random.default_rng(3)
    ctx = Context(g, pb.params())
    opts = ctx.step_opts()
    pb._put(ctx, pb._state0(None))
    for s in range(1, 4):
        ctx.step(DT, s, opts)
    x = pb._get(ctx)
    ybar = {k: np.asfortranarray(rng.standard_normal(g.shape(kind))) for k, kind in VJP_STATE}
    pb._put(ctx, x)
    bar, theta, st = ctx.step_vjp(DT, 4, opts, ybar)
    yield pb, ctx, opts, x, ybar, bar, theta, st, rng
    ctx.close()


def phi(pb, ctx, opts, x, ybar):
    pb._put(ctx, x)
    st = ctx.step(DT, 4, opts)
    assert st["status"] == 0
    out = pb._get(ctx)
    return sum(float(np.sum(ybar[k] * out[k])) for k, _ in VJP_STATE)


def central(pb, ctx, opts, x, ybar, dirs, h=1e-5):
    vals = []
    for sgn in (1.0, -1.0):
        xx = {k: a.copy(order="F") for k, a in x.items()}
        for k, d in dirs.items():
            xx[k] = xx[k] + sgn * h * d
        vals.append(phi(pb, ctx, opts, xx, ybar))
    return (vals[0] - vals[1]) / (2 * h)


def test_step_vjp_converges(one_step):
    *_, st, _ = one_step
    assert st["status"] == 0 and st["res"] < 1e-13 and st["svof_iters"] == 150


@pytest.mark.parametrize("which", ["velocity", "colour", "previous_velocity", "all"])
def test_step_vjp_matches_central_differences(one_step, which):
    pb, ctx, opts, x, ybar, bar, _, _, _ = one_step
    g = pb.g
    rng = np.random.default_rng({"velocity": 1, "colour": 2, "previous_velocity": 4, "all": 5}[which])
    dirs = {}
    if which in ("velocity", "all"):
        dirs["u_vel"], dirs["v_vel"] = divergence_free(rng, g)
    if which in ("colour", "all"):
        dirs["c_field"] = interface_cells(g, x["c_field"], rng)
    if which in ("previous_velocity", "all"):
        dirs["u_prev"] = np.asfortranarray(rng.standard_normal(g.shape("u")))
        dirs["v_prev"] = np.asfortranarray(rng.standard_normal(g.shape("v")))
    ad = sum(float(np.sum(bar[k] * d)) for k, d in dirs.items())
    fd = central(pb, ctx, opts, x, ybar, dirs)
    assert abs(ad - fd) <= 1e-5 * abs(fd), (ad, fd)


@pytest.mark.parametrize("q,name", list(enumerate(RisingBubble.PARAMS)))
def test_step_vjp_parameters(one_step, q, name):
    pb, ctx, opts, x, ybar, _, theta, _, _ = one_step
    v0 = pb.phys[name]
    h = 1e-5 * v0
    vals = []
    for sgn in (1.0, -1.0):
        ctx.set_params(pb.params(**{name: v0 + sgn * h}))
        vals.append(phi(pb, ctx, opts, x, ybar))
    ctx.set_params(pb.params())
    fd = (vals[0] - vals[1]) / (2 * h)
    assert abs(theta[q] - fd) <= 1e-5 * abs(fd), (theta[q], fd)


@pytest.fixture(scope="module")
def gradient(gpu):
    pb = bubble(8)
    return pb, pb.value_and_grad()


def test_bubble_value_matches_forward_run(gradient):
    pb, (J, _, _) = gradient
    assert J == pb.value()
    assert 0.5 < J < 0.51  # the bubble has started to rise


@pytest.mark.parametrize("name", ["sigma", "mu1"])
def test_bubble_parameter_gradient(gradient, name):
    pb, (_, grads, _) = gradient
    v0 = pb.phys[name]
    h = 1e-4 * v0
    fd = (pb.value(**{name: v0 + h}) - pb.value(**{name: v0 - h})) / (2 * h)
    assert abs(grads[name] - fd) <= 1e-5 * abs(fd), (grads[name], fd)


def test_bubble_initial_colour_gradient(gradient):
    pb, (_, _, dc0) = gradient
    g = pb.g
    ci = at(pb.c0, "cell", slice(1, g.nx), slice(1, g.ny))
    cells = np.argwhere((ci > 0.1) & (ci < 0.9))[::7][:3]
    for i0, j0 in cells:
        k = (i0 + 2, j0 + 2)  # interior (i0 + 1, j0 + 1) in the cell array (lower bound -1)
        h = 1e-4
        cp, cm = pb.c0.copy(order="F"), pb.c0.copy(order="F")
        cp[k] += h
        cm[k] -= h
        fd = (pb.value(c0=cp) - pb.value(c0=cm)) / (2 * h)
        assert abs(dc0[k] - fd) <= 1e-6 * abs(fd), (k, dc0[k], fd)


def test_bubble_gradient_independent_of_checkpointing(gradient):
    pb, (J, grads, dc0) = gradient
    J2, grads2, dc02 = bubble(8, checkpoint=8).value_and_grad()
    assert J2 == J
    assert grads2 == grads
    np.testing.assert_array_equal(dc02, dc0)


def test_step_vjp_rejects_unsupported_cases(gpu):
    g = Grid(16, 16, periodic_x=True)
    with Context(g, Params(sigma=1.0)) as ctx:
        with pytest.raises(FuguError):
            ctx.step_vjp(1e-3, 1, ctx.step_opts(), {})
    g = Grid(16, 16)
    with Context(g, Params(sigma=1.0)) as ctx:
        with pytest.raises(FuguError):
            ctx.step_vjp(1e-3, 1, ctx.step_opts(consistent_amp=True), {})


@pytest.mark.slow
def test_bubble_gradient_c5_like_size(gpu):
    """The rising-bubble gradient of the adjoint configuration's run (400 BDF2
    steps of dt = 2.5e-3 to T = 1, checkpoints every 20, FP64 solves to
    1e-12) on 80 x 160: dJ/dsigma, dJ/dmu1 and the derivative along a smooth
    interface direction of C0.  dJ/dsigma and dJ/dmu1 within 1e-6 relative
    of a central difference on the plateau of the h sweep (configs c5
    --sweep); the C0 derivative converging to the adjoint's linearly in h
    (below).  Both the adjoint and J carry errors of a few 1e-12 in absolute
    terms (the solves' tolerance, J's noise of ~3e-14 over 2h); at T = 1
    every derivative is large enough for that to stay below 1e-7 relative,
    while at shorter horizons dJ/dsigma (~8e-7 at T = 0.25) is not.  sigma
    uses the fourth-order difference (J at +-h and +-2h, h = 1e-3 relative),
    mu1 and C0 the two-point one (h = 1e-4 relative for mu1; absolute along
    the unit-maximum direction for C0)."""
    from coupled_codefort_2d_b200.configs import smooth_interface_direction

    def fd2(f, h):
        return (f(h) - f(-h)) / (2.0 * h)

    def fd4(f, h):
        return (8.0 * (f(h) - f(-h)) - (f(2 * h) - f(-2 * h))) / (12.0 * h)

    pb = RisingBubble(nx=80, ny=160, nsteps=400, T=400 * DT, checkpoint=20, tol=1e-12)
    J, grads, dc0 = pb.value_and_grad()
    assert J > 0.5
    for name, fd_of, hrel in (("sigma", fd4, 1e-3), ("mu1", fd2, 1e-4)):
        v0 = pb.phys[name]
        fd = fd_of(lambda h: pb.value(**{name: v0 + h}), hrel * v0)
        print(f"dJ/d{name}: adjoint {grads[name]:.12e}, central difference {fd:.12e}, "
              f"relative {abs(grads[name] - fd) / abs(fd):.2e}")
        assert abs(grads[name] - fd) <= 1e-6 * abs(fd), (name, grads[name], fd)
    # J is only piecewise smooth in C0: a perturbation of the colour moves
    # cells across the flux limiter's and the [0, 1] clip's branch points in
    # later steps, in number proportional to h, so the central difference
    # converges to the derivative of the branch taken (what the adjoint
    # computes) linearly in h, not on a plateau: the relative difference must
    # shrink about tenfold from h = 1e-4 to 1e-5 (the noise's share there is
    # ~5e-7) and end below 1e-5
    d = smooth_interface_direction(pb)
    ad = float(np.sum(dc0 * d))
    err = {}
    for h in (1e-4, 1e-5):
        fd = fd2(lambda t: pb.value(c0=pb.c0 + t * d), h)
        err[h] = abs(ad - fd) / abs(fd)
        print(f"dJ/dC0 . dir: adjoint {ad:.12e}, central difference (h = {h:g}) {fd:.12e}, relative {err[h]:.2e}")
    assert err[1e-5] <= 1e-5 and err[1e-5] <= err[1e-4] / 4, err
