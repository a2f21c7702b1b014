"""Host side of the adjoint harness, no GPU: the closed-form mean velocity of
the two-layer Poiseuille profile equals a quadrature of the profile the
reference's test uses (tests/test_poiseuille_twophase.f90:307-323), its
complex-step derivative equals central differences, the mixture-law
derivatives recover d mu / d mu_k, and the rising-bubble objective's seed
dJ/dC equals central differences."""
import numpy as np

from coupled_codefort_2d_b200 import adjoint
from refcases import poiseuille_exact


def test_closed_form_mean_velocity_matches_quadrature():
    for mu1, mu2 in ((1.0, 0.25), (1.0, 0.1), (0.3, 2.0)):
        y = (np.arange(200000) + 0.5) / 200000
        quad = float(np.mean(poiseuille_exact(y, 1.0, mu1, mu2)))
        assert abs(adjoint.analytic_mean_velocity(mu1, mu2) - quad) <= 1e-9 * abs(quad)


def test_complex_step_derivative_matches_central_difference():
    mu1, mu2 = 1.0, 0.1
    d1, d2 = adjoint.analytic_grad(mu1, mu2)
    h = 1e-6
    f = adjoint.analytic_mean_velocity
    assert abs(d1 - (f(mu1 + h, mu2) - f(mu1 - h, mu2)) / (2 * h)) <= 1e-7 * abs(d1)
    assert abs(d2 - (f(mu1, mu2 + h) - f(mu1, mu2 - h)) / (2 * h)) <= 1e-7 * abs(d2)


def test_mixture_derivatives():
    mu1, mu2 = 1.0, 0.1
    C = np.linspace(0.0, 1.0, 11)

    def mu(c, a, b):
        return a * b / (b * c + a * (1.0 - c))

    field = 2.0 * mu(C, mu1, mu2)
    d1, d2 = adjoint.mixture_derivatives(field, mu1, mu2, 2.0)
    h = 1e-7
    np.testing.assert_allclose(d1, 2.0 * (mu(C, mu1 + h, mu2) - mu(C, mu1 - h, mu2)) / (2 * h), rtol=1e-6, atol=1e-12)
    np.testing.assert_allclose(d2, 2.0 * (mu(C, mu1, mu2 + h) - mu(C, mu1, mu2 - h)) / (2 * h), rtol=1e-6, atol=1e-12)


def test_centroid_objective_gradient():
    """dJ/dC of the centroid height of fluid 2 (the rising-bubble adjoint's
    seed) equals central differences, and is zero off the interior."""
    pb = adjoint.RisingBubble(nx=12, ny=24, nsteps=1)
    g = pb.g
    rng = np.random.default_rng(0)
    c = pb.c0 + 0.01 * rng.standard_normal(pb.c0.shape)
    c = np.asfortranarray(c)
    grad = pb.objective_grad(c)
    for k in ((3, 4), (7, 20), (10, 13)):
        cp, cm = c.copy(order="F"), c.copy(order="F")
        cp[k] += 1e-6
        cm[k] -= 1e-6
        fd = (pb.objective(cp) - pb.objective(cm)) / 2e-6
        assert abs(grad[k] - fd) <= 1e-8 * abs(fd)
    assert not grad[0, :].any() and not grad[:, -1].any()
    assert pb.params().svof_tol == 0.0 and abs(pb.dt - 1.0) < 1e-15
