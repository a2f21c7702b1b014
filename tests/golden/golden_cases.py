"""Seeded cases of the golden fixtures (``oracle_golden.npz``).

Each case builds its inputs from a fixed seed and runs one routine or a few
coupled steps on one side: ``"oracle"`` (the CPU restatement in ``oracle/``)
or ``"gpu"`` (the CUDA path through the C ABI).  ``make_golden.py`` stores the
oracle side's outputs; ``tests/test_golden_cpu.py`` checks that the oracle
still reproduces them bit for bit, and ``tests/test_gpu_golden.py`` that the
CUDA path does, without running the oracle.  Inputs are regenerated, not
stored: numpy's PCG64 streams are stable across versions.
"""
from __future__ import annotations

import numpy as np

from coupled_codefort_2d_b200 import cases
from coupled_codefort_2d_b200.layout import Grid
from coupled_codefort_2d_b200.params import Params

PHYS = dict(rho1=1000.0, rho2=100.0, mu1=10.0, mu2=1.0, sigma=24.5, gx=0.0, gy=-0.98)
STATE = ("u_vel", "v_vel", "p_field", "c_field", "u_prev", "v_prev", "rho_c", "rho_u", "rho_v", "kappa", "zeta",
         "eta", "kappa_curv", "f_sigma_u", "f_sigma_v")
KIND = {"u_vel": "u", "v_vel": "v", "p_field": "cell", "c_field": "cell", "u_prev": "u", "v_prev": "v",
        "rho_c": "cell", "rho_u": "u", "rho_v": "v", "kappa": "cell", "zeta": "vert", "eta": "vert",
        "kappa_curv": "cell", "f_sigma_u": "u", "f_sigma_v": "v"}


def _field(rng, g, kind, lo=-1.0, hi=1.0):
    return np.asfortranarray(rng.uniform(lo, hi, size=g.shape(kind)))


class _Side:
    """the routines a case needs, on the oracle or through the C ABI"""

    def __init__(self, side, g, prm, precision=0):
        self.side, self.g, self.prm = side, g, prm
        if side == "oracle":
            from oracle import oracle

            self.o = oracle.Oracle(g, prm)
            self.ctx = None
        else:
            from coupled_codefort_2d_b200.context import Context

            self.ctx = Context(g, prm, precision=precision)

    def close(self):
        if self.ctx is not None:
            self.ctx.close()

    def properties(self, c):
        g = self.g
        pr = {k: g.zeros(KIND[k]) for k in ("rho_c", "rho_u", "rho_v", "kappa", "zeta", "eta")}
        if self.ctx is None:
            self.o.densities(c, pr["rho_c"], pr["rho_u"], pr["rho_v"])
            self.o.viscosities(c, pr["kappa"], pr["zeta"], pr["eta"])
        else:
            self.ctx.compute_mixture_densities(c, pr["rho_c"], pr["rho_u"], pr["rho_v"])
            self.ctx.compute_mixture_viscosities(c, pr["kappa"], pr["zeta"], pr["eta"])
        return pr


def case_matvec_penalty(side):
    """matvec_coupled on 13 x 9 walls with advection and the Darcy penalty"""
    g = Grid(13, 9, 1.0, 0.7)
    rng = np.random.default_rng(101)
    prm = Params(**PHYS)
    s = _Side(side, g, prm)
    try:
        pr = s.properties(np.asfortranarray(rng.uniform(-0.05, 1.05, size=g.shape("cell"))))
        X = [_field(rng, g, k) for k in ("u", "v", "cell")]
        ua, va = _field(rng, g, "u"), _field(rng, g, "v")
        pen = (_field(rng, g, "u", 0, 1e12), _field(rng, g, "v", 0, 1e12))
        Y = [g.zeros(k) for k in ("u", "v", "cell")]
        if side == "oracle":
            s.o.matvec(*X, *Y, ua, va, pr, 3.7e-3, True, pen[0], pen[1])
        else:
            s.ctx.matvec_coupled(*X, *Y, ua, va, pr["rho_c"], pr["rho_u"], pr["rho_v"], pr["kappa"], pr["zeta"],
                                 pr["eta"], 3.7e-3, True, pen[0], pen[1])
        return {"Yu": Y[0], "Yv": Y[1], "Yp": Y[2]}
    finally:
        s.close()


def case_pcd_periodic(side):
    """apply_pcd_precond on a 16 x 12 box periodic in x, 3 damped-Jacobi sweeps"""
    g = Grid(16, 12, periodic_x=True)
    rng = np.random.default_rng(102)
    prm = Params(**PHYS, pcd_sweeps=3)
    s = _Side(side, g, prm)
    try:
        pr = s.properties(np.asfortranarray(rng.uniform(-0.05, 1.05, size=g.shape("cell"))))
        z = [_field(rng, g, k) for k in ("u", "v", "cell")]
        ua, va = _field(rng, g, "u"), _field(rng, g, "v")
        r = [g.zeros(k) for k in ("u", "v", "cell")]
        if side == "oracle":
            s.o.pcd(*z, *r, ua, va, pr, 2e-3)
        else:
            s.ctx.apply_pcd_precond(*z, *r, ua, va, pr["rho_u"], pr["rho_v"], pr["kappa"], pr["zeta"], pr["eta"],
                                    2e-3)
        return {"r_u": r[0], "r_v": r[1], "r_p": r[2]}
    finally:
        s.close()


def case_transport(side):
    """vof_advection_tvd (Superbee), svof_helmholtz_filter, curvature and CSF
    on a 32 x 32 disc with a seeded velocity field"""
    g = Grid(32, 32)
    rng = np.random.default_rng(103)
    prm = Params(limiter=1, sigma=1.3)
    s = _Side(side, g, prm)
    try:
        c = cases.circle_fraction(g, 0.5, 0.5, 0.25, inside=1.0, ns=8)
        u, v = _field(rng, g, "u", -2, 2), _field(rng, g, "v", -2, 2)
        dt = 0.2 * g.dx / 2
        c1, fx, fy = g.zeros("cell"), g.zeros("u"), g.zeros("v")
        cs, kc, fu, fv = g.zeros("cell"), g.zeros("cell"), g.zeros("u"), g.zeros("v")
        delta = 1.5 * g.dx
        if side == "oracle":
            s.o.vof(c, c1, u, v, dt, fx, fy)
            it = s.o.svof(c1, cs, delta, 150, 1e-7)
            s.o.curvature(cs, kc)
            s.o.csf(c1, kc, fu, fv)
        else:
            s.ctx.vof_advection_tvd(c, c1, u, v, dt, fx, fy)
            it = s.ctx.svof_helmholtz_filter(c1, cs, delta, 150, 1e-7)
            s.ctx.compute_interface_curvature(cs, kc)
            s.ctx.compute_csf_force(c1, kc, fu, fv)
        return {"c_new": c1, "flux_x": fx, "flux_y": fy, "c_smooth": cs, "kappa_curv": kc, "f_sigma_u": fu,
                "f_sigma_v": fv, "svof_iters": np.array([it])}
    finally:
        s.close()


def _steps(side, g, prm, c0, dt, nsteps, **kw):
    s = _Side(side, g, prm)
    try:
        st = {k: g.zeros(KIND[k]) for k in STATE}
        st["c_field"][...] = c0
        pr = s.properties(st["c_field"])
        for k, a in pr.items():
            st[k][...] = a
        its = []
        for step in range(1, nsteps + 1):
            if side == "oracle":
                r = s.o.step(st, dt, step, **kw)
                its.append((r.iter, r.outer))
            else:
                r = s.ctx.advance_coupled_step(*[st[k] for k in STATE], dt, step, **kw)
                its.append((r["iter"], r["outer"]))
        out = {k: st[k] for k in ("u_vel", "v_vel", "p_field", "c_field")}
        out["iterations"] = np.array(its)
        return out
    finally:
        s.close()


def case_steps_droplet(side):
    """three plain-FP64 BDF2 steps of a 32 x 32 static droplet (BiCGStab + PCD)"""
    g = Grid(32, 32)
    prm = Params(rho1=1.0, rho2=0.1, mu1=0.1, mu2=0.01, sigma=1.0, gx=0.0, gy=0.0, time_order=2,
                 tol_bicgstab2=1e-6, max_iter_bicgstab2=100)
    c0 = cases.circle_fraction(g, 0.5, 0.5, 0.25, inside=1.0, ns=8)
    return _steps(side, g, prm, c0, 1e-4, 3, use_bicgstab2=False)


def case_steps_bubble_fgmres(side):
    """three FP64 steps of a 16 x 32 free-slip rising bubble, defect correction
    around flexible GMRES with the adaptive PCG cap and red-black SOR smoothing"""
    g = Grid(16, 32, 1.0, 2.0)
    prm = Params(**PHYS, time_order=2, tol_bicgstab2=1e-9, max_iter_bicgstab2=100, free_slip_x=1, refine=2,
                 refine_inner_tol=1e-2, refine_max_inner=30, refine_max_outer=30, krylov_bc_fix=1, pcg_cap_start=4,
                 pcd_smoother=1, pcd_sor_omega=1.5)
    c0 = cases.initial_colour(g, "rising_bubble")
    return _steps(side, g, prm, c0, 1e-3, 3, use_bicgstab2=False)


CASES = {
    "matvec_penalty": case_matvec_penalty,
    "pcd_periodic": case_pcd_periodic,
    "transport": case_transport,
    "steps_droplet": case_steps_droplet,
    "steps_bubble_fgmres": case_steps_bubble_fgmres,
}
