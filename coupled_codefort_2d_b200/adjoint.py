"""Discrete adjoint of the coupled solve, and a torch.autograd harness.

The Krylov solvers see the linear map A: x -> matvec_coupled(BC(x)) on the
owned unknowns (``mod_operators.f90:341-443`` after the homogeneous wall BCs of
``:254-333``).  ``fugu_matvec_coupled_t`` applies A^T and ``fugu_adjoint_solve``
solves A^T lambda = g on the GPU.  For a functional J = g . X of the solution
of A(theta) X = B(theta),

    dJ/dtheta = lambda . (dB/dtheta - (dA/dtheta) X).

The viscous part of A is linear in the property fields (kappa, zeta, eta), so
(dA/dtheta) X is one more matvec with the property derivatives in place of
the properties, minus the same matvec with zero viscosity.  The property
derivatives follow from the mixture law mu(C) = mu1 mu2 / (mu2 C + mu1 (1 - C))
(``mod_viscosity.f90:28-46``).

The check case is the steady two-phase Poiseuille channel of
``tests/test_poiseuille_twophase.f90`` (periodic in x, no-slip walls in y,
fluid 1 below y = Ly/2, body force gx): one backward-Euler solve with a very
large time step is the steady coupled system.  No counterpart in the
reference, which has no adjoint.
"""
from __future__ import annotations

import numpy as np

from . import cases
from .context import Context
from .layout import Grid, at
from .params import Params

DT_STEADY = 1.0e8  # backward Euler with this step is the steady coupled system


def owned_masks(g: Grid):
    """Boolean masks (reference layout) of the owned unknowns: interior u faces
    (i = 1..imax), v faces (j = 1..jmax) and cells."""
    imax = g.nx if g.periodic_x else g.nx - 1
    jmax = g.ny if g.periodic_y else g.ny - 1
    mu, mv, mp = (np.zeros(g.shape(k), dtype=bool, order="F") for k in ("u", "v", "cell"))
    at(mu, "u", slice(1, imax), slice(1, g.ny))[...] = True
    at(mv, "v", slice(1, g.nx), slice(1, jmax))[...] = True
    at(mp, "cell", slice(1, g.nx), slice(1, g.ny))[...] = True
    return mu, mv, mp


def owned_dot(g: Grid, a, b) -> float:
    """Euclidean product of two (u, v, p) triples over the owned unknowns."""
    return float(sum(np.sum(x[m] * y[m]) for x, y, m in zip(a, b, owned_masks(g))))


def mixture_derivatives(field, mu1, mu2, scale):
    """d(field)/d(mu1), d(field)/d(mu2) for field = scale * mu(C), recovering C
    from the field itself (mu1 != mu2)."""
    mu = field / scale
    D = mu1 * mu2 / mu
    C = (D - mu1) / (mu2 - mu1)
    return scale * mu2 * mu2 * C / (D * D), scale * mu1 * mu1 * (1.0 - C) / (D * D)


class SteadyPoiseuille:
    """J(mu1, mu2) = mean streamwise velocity of the steady two-phase
    Poiseuille channel, with its adjoint gradient.  ``nx`` x ``ny`` cells,
    unit box, gx body force, densities rho (both fluids)."""

    def __init__(self, nx=32, ny=64, gx=1.0, rho=1.0, tol=1e-13, device=0):
        self.g = Grid(nx, ny, periodic_x=True)
        self.gx, self.rho, self.tol = gx, rho, tol
        self.c0 = cases.initial_colour(self.g, "poiseuille")
        self.ctx = Context(self.g, self.params(1.0, 0.1), device=device)

    def params(self, mu1, mu2) -> Params:
        return Params(rho1=self.rho, rho2=self.rho, mu1=mu1, mu2=mu2, sigma=0.0, gx=self.gx, gy=0.0,
                      time_order=1, tol_bicgstab2=self.tol, refine=2, refine_inner_tol=1e-2, refine_max_inner=30,
                      refine_max_outer=200, krylov_bc_fix=1)

    def close(self):
        self.ctx.close()

    def _setup(self, mu1, mu2):
        g = self.g
        self.ctx.set_params(self.params(mu1, mu2))
        pr = {k: g.zeros(kd) for k, kd in (("rho_c", "cell"), ("rho_u", "u"), ("rho_v", "v"), ("kappa", "cell"),
                                            ("zeta", "vert"), ("eta", "vert"))}
        self.ctx.compute_mixture_densities(self.c0, pr["rho_c"], pr["rho_u"], pr["rho_v"])
        self.ctx.compute_mixture_viscosities(self.c0, pr["kappa"], pr["zeta"], pr["eta"])
        pr["u_adv"], pr["v_adv"] = g.zeros("u"), g.zeros("v")
        mu_, mv_, _ = owned_masks(g)
        B = [g.zeros("u"), g.zeros("v"), g.zeros("cell")]
        B[0][mu_] = (pr["rho_u"] * self.gx)[mu_]  # mod_solver_coupled.f90:268-303 with u^n = 0
        return pr, B

    def _coef(self, pr):
        return (pr["u_adv"], pr["v_adv"], pr["rho_c"], pr["rho_u"], pr["rho_v"], pr["kappa"], pr["zeta"], pr["eta"])

    def solve(self, mu1, mu2):
        g = self.g
        pr, B = self._setup(mu1, mu2)
        X = [g.zeros("u"), g.zeros("v"), g.zeros("cell")]
        st = self.ctx.bicgstab2_solve(*X, *B, *self._coef(pr), DT_STEADY, tol_in=self.tol, max_iter_in=500)
        return X, B, pr, st

    def functional(self):
        """g with J = g . X: the mean of u over the channel (owned u faces)."""
        g = self.g
        mu_, _, _ = owned_masks(g)
        gu = g.zeros("u")
        gu[mu_] = 1.0 / mu_.sum()
        return [gu, g.zeros("v"), g.zeros("cell")]

    def value(self, mu1, mu2) -> float:
        X, _, _, st = self.solve(mu1, mu2)
        return owned_dot(self.g, self.functional(), X)

    def value_and_grad(self, mu1, mu2):
        """J and (dJ/dmu1, dJ/dmu2) by the discrete adjoint."""
        g = self.g
        X, B, pr, st = self.solve(mu1, mu2)
        gJ = self.functional()
        J = owned_dot(g, gJ, X)
        lam = [g.zeros("u"), g.zeros("v"), g.zeros("cell")]
        ast = self.ctx.adjoint_solve(*gJ, *lam, *self._coef(pr), DT_STEADY, tol=self.tol)
        grads = []
        for which in (0, 1):
            dk = mixture_derivatives(pr["kappa"], mu1, mu2, 2.0)[which]
            dz = mixture_derivatives(pr["zeta"], mu1, mu2, 2.0)[which]
            de = mixture_derivatives(pr["eta"], mu1, mu2, 1.0)[which]
            grads.append(-owned_dot(g, lam, self._dA_X(X, pr, dk, dz, de)))
        return J, grads, {"forward": st, "adjoint": ast}

    def _dA_X(self, X, pr, dk, dz, de):
        """(dA/dtheta) X: the matvec with the property derivatives minus the
        matvec with zero viscosity (the viscous part is linear in them)."""
        g = self.g
        Xb = [a.copy(order="F") for a in X]
        self.ctx.apply_velocity_bcs(Xb[0], Xb[1], None)

        def mv(k, z, e):
            Y = [g.zeros("u"), g.zeros("v"), g.zeros("cell")]
            Xc = [a.copy(order="F") for a in Xb]
            self.ctx.matvec_coupled(*Xc, *Y, pr["u_adv"], pr["v_adv"], pr["rho_c"], pr["rho_u"], pr["rho_v"], k, z,
                                    e, DT_STEADY)
            return Y

        Y1 = mv(dk, dz, de)
        Y0 = mv(g.zeros("cell"), g.zeros("vert"), g.zeros("vert"))
        return [a - b for a, b in zip(Y1, Y0)]


def analytic_mean_velocity(mu1, mu2, G=1.0, Ly=1.0):
    """Mean velocity of the exact two-layer profile
    (tests/test_poiseuille_twophase.f90:307-323), integrated in closed form;
    complex arguments give exact complex-step derivatives."""
    yi = 0.5 * Ly
    A1 = G * (yi ** 2 / (2 * mu1) + (Ly ** 2 - yi ** 2) / (2 * mu2)) / (yi + (mu1 / mu2) * (Ly - yi))
    A2 = (mu1 / mu2) * A1
    B2 = G * Ly ** 2 / (2 * mu2) - A2 * Ly
    low = -(G / (6 * mu1)) * yi ** 3 + 0.5 * A1 * yi ** 2
    up = (-(G / (6 * mu2)) * (Ly ** 3 - yi ** 3) + 0.5 * A2 * (Ly ** 2 - yi ** 2) + B2 * (Ly - yi))
    return (low + up) / Ly


def analytic_grad(mu1, mu2, G=1.0):
    h = 1e-30
    d1 = analytic_mean_velocity(mu1 + 1j * h, mu2, G).imag / h
    d2 = analytic_mean_velocity(mu1, mu2 + 1j * h, G).imag / h
    return d1, d2


def torch_flux_function(problem: SteadyPoiseuille):
    """A torch.autograd.Function J(mu) with mu = tensor([mu1, mu2]) (float64):
    forward by the GPU solve, backward by the GPU adjoint."""
    import torch

    class SteadyFlux(torch.autograd.Function):
        @staticmethod
        def forward(ctx, mu):
            J, grads, _ = problem.value_and_grad(float(mu[0]), float(mu[1]))
            ctx.save_for_backward(torch.tensor(grads, dtype=torch.float64))
            return torch.tensor(J, dtype=torch.float64)

        @staticmethod
        def backward(ctx, gout):
            (grads,) = ctx.saved_tensors
            return gout * grads

    return SteadyFlux.apply
