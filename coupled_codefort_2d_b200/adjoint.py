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
from ._lib import FIELD_KIND, FuguError
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


class StartupPoiseuille(SteadyPoiseuille):
    """The two-phase Poiseuille channel started from rest: N steps of
    advance_coupled_step's time discretisation (BDF1 first, then BDF2:
    ``mod_solver_coupled.f90:196-201, 268-303``), J = g . u^N (the mean
    velocity after N steps), and its gradient by the multi-step discrete
    adjoint with checkpointing.

    Step s solves A_s X^s = B_s with B_s = M (c1 u^(s-1) + c0 u^(s-2)) + rho g
    (M = rho/dt on the velocity rows; c1, c0 = 1, 0 for BDF1 and 2, -1/2 for
    BDF2) and A_s the coupled operator at dt_eff (dt, then dt/1.5), its
    advecting velocity the AB extrapolation 2u^(s-1) - u^(s-2).  The adjoint
    runs backwards:

        A_s^T lam^s = [s = N] g + M (c1_(s+1) lam^(s+1) + c0_(s+2) lam^(s+2)),
        dJ/dtheta   = -sum_s lam^s . (dA_s/dtheta) X^s.

    The coefficient fields (colour, densities, viscosities, advecting
    velocity) are held at their forward values: exact here, where the flow
    stays parallel to the layers, so C does not move and the advection terms
    vanish along every sensitivity (checked against ``fugu_step`` and finite
    differences in the tests).  States X^s are kept every ``checkpoint``
    steps and recomputed in between during the backward sweep.
    """

    def __init__(self, nx=16, ny=32, nsteps=20, dt=0.05, checkpoint=5, **kw):
        super().__init__(nx=nx, ny=ny, **kw)
        self.nsteps, self.dt, self.checkpoint = nsteps, dt, checkpoint
        self.recomputed_steps = 0

    def params(self, mu1, mu2) -> Params:
        return super().params(mu1, mu2).with_(time_order=2)

    def _coeffs(self, s):
        bdf2 = s >= 2
        return (2.0, -0.5, self.dt / 1.5) if bdf2 else (1.0, 0.0, self.dt)

    def _step(self, pr, s, u1, u2):
        """X^s from u^(s-1) (u1) and u^(s-2) (u2), triples of host arrays."""
        g = self.g
        c1, c0, dt_eff = self._coeffs(s)
        mu_, mv_, _ = owned_masks(g)
        B = [g.zeros("u"), g.zeros("v"), g.zeros("cell")]
        B[0][mu_] = ((pr["rho_u"] / self.dt) * (c1 * u1[0] + c0 * u2[0]) + pr["rho_u"] * self.gx)[mu_]
        B[1][mv_] = ((pr["rho_v"] / self.dt) * (c1 * u1[1] + c0 * u2[1]))[mv_]
        ua = u1[0] if s == 1 else 2.0 * u1[0] - u2[0]
        va = u1[1] if s == 1 else 2.0 * u1[1] - u2[1]
        X = [a.copy(order="F") for a in u1]  # the previous step's state is the initial guess
        self.ctx.bicgstab2_solve(*X, *B, np.asfortranarray(ua), np.asfortranarray(va), pr["rho_c"], pr["rho_u"],
                                 pr["rho_v"], pr["kappa"], pr["zeta"], pr["eta"], dt_eff, tol_in=self.tol,
                                 max_iter_in=500)
        self.ctx.apply_velocity_bcs(X[0], X[1], None)
        return X, (np.asfortranarray(ua), np.asfortranarray(va), dt_eff)

    def _run(self, pr, s0, X_prev, X_prev2, s1, keep=None):
        """States from step s0 to s1 (inclusive) given X^(s0-1), X^(s0-2)."""
        out = {}
        for s in range(s0, s1 + 1):
            X, _ = self._step(pr, s, X_prev, X_prev2)
            if keep is None or s in keep:
                out[s] = X
            X_prev2, X_prev = X_prev, X
        return out, X_prev, X_prev2

    def trajectory_value(self, mu1, mu2):
        g = self.g
        pr, _ = self._setup(mu1, mu2)
        zero = [g.zeros("u"), g.zeros("v"), g.zeros("cell")]
        _, XN, _ = self._run(pr, 1, zero, zero, self.nsteps, keep=set())
        return owned_dot(g, self.functional(), XN), XN

    def value(self, mu1, mu2) -> float:
        return self.trajectory_value(mu1, mu2)[0]

    def value_and_grad(self, mu1, mu2):
        g = self.g
        N, K = self.nsteps, self.checkpoint
        pr, _ = self._setup(mu1, mu2)
        zero = [g.zeros("u"), g.zeros("v"), g.zeros("cell")]
        # forward sweep: keep every K-th state and the one before it (BDF2
        # restarts from the pair)
        keep = {s for s in range(1, N + 1) if s % K == 0 or s % K == K - 1}
        ck, XN, _ = self._run(pr, 1, zero, zero, N, keep=keep)
        ck[0] = ck[-1] = zero
        self.kept_states = len(keep)
        gJ = self.functional()
        J = owned_dot(g, gJ, XN)
        dk = [mixture_derivatives(pr["kappa"], mu1, mu2, 2.0)[w] for w in (0, 1)]
        dz = [mixture_derivatives(pr["zeta"], mu1, mu2, 2.0)[w] for w in (0, 1)]
        de = [mixture_derivatives(pr["eta"], mu1, mu2, 1.0)[w] for w in (0, 1)]
        grads = [0.0, 0.0]
        lam_next, lam_next2 = None, None  # lambda^(s+1), lambda^(s+2)
        segment = {0: zero, -1: zero}
        self.recomputed_steps = 0
        for s in range(N, 0, -1):
            if any(k not in segment for k in (s, s - 1, s - 2) if k >= 1):
                # recompute the checkpoint segment that ends at s from its stored pair
                start = (s - 1) // K * K
                if start >= 1 and s - 2 < start:  # X^(s-2) lies in the segment before
                    start = (start - 1) // K * K
                base1, base2 = ck[start], ck[start - 1]
                segment, _, _ = self._run(pr, start + 1, base1, base2, s)
                self.recomputed_steps += s - start
                segment.update({start: base1, start - 1: base2, 0: zero, -1: zero})
            X, X1, X2 = segment[s], segment[s - 1], segment[s - 2]
            ua = X1[0] if s == 1 else 2.0 * X1[0] - X2[0]
            va = X1[1] if s == 1 else 2.0 * X1[1] - X2[1]
            _, _, dt_eff = self._coeffs(s)
            rhs = [a.copy(order="F") for a in (gJ if s == N else zero)]
            for lam, sp in ((lam_next, s + 1), (lam_next2, s + 2)):
                if lam is None or sp > N:
                    continue
                c1, c0, _ = self._coeffs(sp)
                c = c1 if sp == s + 1 else c0
                rhs[0] = rhs[0] + c * (pr["rho_u"] / self.dt) * lam[0]
                rhs[1] = rhs[1] + c * (pr["rho_v"] / self.dt) * lam[1]
            mu_, mv_, mp_ = owned_masks(g)
            rhs = [np.asfortranarray(np.where(m, a, 0.0)) for a, m in zip(rhs, (mu_, mv_, mp_))]
            lam = [g.zeros("u"), g.zeros("v"), g.zeros("cell")]
            co = (np.asfortranarray(ua), np.asfortranarray(va), pr["rho_c"], pr["rho_u"], pr["rho_v"], pr["kappa"],
                  pr["zeta"], pr["eta"])
            self.ctx.adjoint_solve(*rhs, *lam, *co, dt_eff, tol=self.tol)
            for w in (0, 1):
                grads[w] -= owned_dot(g, lam, self._dA_X_dt(X, co, dk[w], dz[w], de[w], dt_eff))
            lam_next2, lam_next = lam_next, lam
        return J, grads, {}

    def _dA_X_dt(self, X, co, dk, dz, de, dt_eff):
        g = self.g
        Xb = [a.copy(order="F") for a in X]
        self.ctx.apply_velocity_bcs(Xb[0], Xb[1], None)

        def mv(k, z, e):
            Y = [g.zeros("u"), g.zeros("v"), g.zeros("cell")]
            Xc = [a.copy(order="F") for a in Xb]
            self.ctx.matvec_coupled(*Xc, *Y, co[0], co[1], co[2], co[3], co[4], k, z, e, dt_eff)
            return Y

        Y1 = mv(dk, dz, de)
        Y0 = mv(g.zeros("cell"), g.zeros("vert"), g.zeros("vert"))
        return [a - b for a, b in zip(Y1, Y0)]


class RisingBubble:
    """The rising bubble of the adjoint check: a 1 x 2 wall-bounded box,
    fluid 2 (C = 0) a disc of radius 0.25 at (0.5, 0.5) given by area
    fractions, BDF2 steps of advance_coupled_step to time T, and
    J = the centroid height of fluid 2 at T (``test_rising_bubble.f90:134-155``).

    ``value_and_grad`` returns J and its derivatives with respect to sigma,
    mu1 (the outer fluid), mu2, rho1, rho2 and every entry of the initial
    colour field, by the step's vector-Jacobian product (``fugu_step_vjp``)
    run backwards over the steps.  The forward run stores the state every
    ``checkpoint`` steps; the backward sweep recomputes each segment from its
    checkpoint.  The solves run to ``tol`` and the SVOF filter to
    ``svof_tol`` (0: always its 150 sweeps, so that J is a smooth function of
    the inputs apart from the limiter and clip branches).  No counterpart in
    the reference, which has no adjoint.
    """

    PARAMS = ("sigma", "mu1", "mu2", "rho1", "rho2")
    STATE = ("u_vel", "v_vel", "p_field", "c_field", "u_prev", "v_prev")

    def __init__(self, nx=160, ny=320, nsteps=400, T=1.0, checkpoint=20, tol=1e-12, svof_tol=0.0, device=0,
                 **phys):
        self.g = Grid(nx, ny, 1.0, 2.0)
        self.nsteps, self.dt, self.checkpoint = int(nsteps), T / nsteps, int(checkpoint)
        self.phys = dict(rho1=1000.0, rho2=100.0, mu1=10.0, mu2=1.0, sigma=24.5)
        self.phys.update(phys)
        self.tol, self.svof_tol, self.device = tol, svof_tol, device
        self.c0 = cases.circle_fraction(self.g, 0.5, 0.5, 0.25, inside=0.0, ns=16)

    def params(self, **over) -> Params:
        ph = {**self.phys, **over}
        return Params(gx=0.0, gy=-0.98, time_order=2, tol_bicgstab2=self.tol, max_iter_bicgstab2=500,
                      svof_tol=self.svof_tol, refine=2, refine_inner_tol=1e-2, refine_max_inner=30,
                      refine_max_outer=100, krylov_bc_fix=1, **ph)

    def objective(self, c) -> float:
        ci = at(c, "cell", slice(1, self.g.nx), slice(1, self.g.ny))
        _, Y = cases.cell_centres_interior(self.g)
        return float(np.sum((1.0 - ci) * Y) / np.sum(1.0 - ci))

    def objective_grad(self, c) -> np.ndarray:
        """dJ/dC over the cell extent (nonzero on the interior only)."""
        g = self.g
        ci = at(c, "cell", slice(1, g.nx), slice(1, g.ny))
        _, Y = cases.cell_centres_interior(g)
        S = np.sum(1.0 - ci)
        J = np.sum((1.0 - ci) * Y) / S
        out = g.zeros("cell")
        at(out, "cell", slice(1, g.nx), slice(1, g.ny))[...] = (J - Y) / S
        return out

    def _state0(self, c0):
        g = self.g
        st = {k: g.zeros(FIELD_KIND[k]) for k in self.STATE}
        st["c_field"][...] = self.c0 if c0 is None else c0
        return st

    def _put(self, ctx, st):
        for k in self.STATE:
            ctx.upload(k, st[k])

    def _get(self, ctx):
        return {k: ctx.download(k) for k in self.STATE}

    @staticmethod
    def _check(st, what):
        if st["status"] != 0:
            raise FuguError(f"{what}: status {st['status']} (residual {st['res']:.3e})")

    def value(self, c0=None, **over) -> float:
        with Context(self.g, self.params(**over), device=self.device) as ctx:
            self._put(ctx, self._state0(c0))
            opts = ctx.step_opts(use_bicgstab2=True)
            for s in range(1, self.nsteps + 1):
                self._check(ctx.step(self.dt, s, opts), f"step {s}")
            return self.objective(ctx.download("c_field"))

    def value_and_grad(self, c0=None, **over):
        """(J, {parameter: dJ/dparameter}, dJ/dC0 over the cell extent)."""
        N, K = self.nsteps, self.checkpoint
        with Context(self.g, self.params(**over), device=self.device) as ctx:
            opts = ctx.step_opts(use_bicgstab2=True)
            chk = {0: self._state0(c0)}
            self._put(ctx, chk[0])
            for s in range(1, N + 1):
                self._check(ctx.step(self.dt, s, opts), f"step {s}")
                if s % K == 0 and s < N:
                    chk[s] = self._get(ctx)
            c_end = ctx.download("c_field")
            J = self.objective(c_end)
            bar = {"c_field": self.objective_grad(c_end)}
            theta = np.zeros(len(self.PARAMS))
            for s0 in sorted(chk, reverse=True):
                s1 = min(s0 + K, N)
                # the states before steps s0 + 1 .. s1, recomputed from the checkpoint
                pre = [chk[s0]]
                self._put(ctx, chk[s0])
                for s in range(s0 + 1, s1):
                    self._check(ctx.step(self.dt, s, opts), f"recomputed step {s}")
                    pre.append(self._get(ctx))
                for s in range(s1, s0, -1):
                    self._put(ctx, pre[s - s0 - 1])
                    bar, th, st = ctx.step_vjp(self.dt, s, opts, bar)
                    self._check(st, f"adjoint of step {s}")
                    theta += th
        return J, dict(zip(self.PARAMS, theta)), bar["c_field"]
