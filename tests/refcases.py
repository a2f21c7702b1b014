"""The reference's own validation programs (tests/test_*.f90), restated as
functions of a backend: the CPU oracle (``oracle.oracle.Oracle``) or the CUDA
path through :class:`GpuBackend`.  Each returns the diagnostics the Fortran
test prints; the pytest files assert the Fortran test's pass criterion.
"""
import math

import numpy as np

from coupled_codefort_2d_b200 import cases
from coupled_codefort_2d_b200.layout import Grid, at
from coupled_codefort_2d_b200.params import Params

STATE_KINDS = {
    "u_vel": "u", "v_vel": "v", "p_field": "cell", "c_field": "cell", "u_prev": "u", "v_prev": "v",
    "rho_c": "cell", "rho_u": "u", "rho_v": "v", "kappa": "cell", "zeta": "vert", "eta": "vert",
    "kappa_curv": "cell", "f_sigma_u": "u", "f_sigma_v": "v",
}
STATE = list(STATE_KINDS)


class GpuBackend:
    """The CUDA context with the oracle's method names."""

    def __init__(self, g, prm, precision=0):
        from coupled_codefort_2d_b200.context import Context

        self.g = g
        self.ctx = Context(g, prm, precision=precision)

    def close(self):
        self.ctx.close()

    def halo(self, kind, a):
        self.ctx.halo(kind, a)

    def properties(self, c):
        g = self.g
        out = {k: g.zeros(kd) for k, kd in (("rho_c", "cell"), ("rho_u", "u"), ("rho_v", "v"),
                                             ("kappa", "cell"), ("zeta", "vert"), ("eta", "vert"))}
        self.ctx.compute_mixture_densities(c, out["rho_c"], out["rho_u"], out["rho_v"])
        self.ctx.compute_mixture_viscosities(c, out["kappa"], out["zeta"], out["eta"])
        return out

    def divergence(self, u, v, d):
        self.ctx.op_divergence(u, v, d)

    def grad_pressure(self, p, gu, gv):
        self.ctx.op_grad_pressure(p, gu, gv)

    def viscous_stress(self, u, v, k, z, e, vu, vv):
        self.ctx.op_viscous_stress(u, v, k, z, e, vu, vv)

    def matvec(self, Xu, Xv, Xp, Yu, Yv, Yp, ua, va, pr, dt, include_adv=True):
        self.ctx.matvec_coupled(Xu, Xv, Xp, Yu, Yv, Yp, ua, va, pr["rho_c"], pr["rho_u"], pr["rho_v"],
                                pr["kappa"], pr["zeta"], pr["eta"], dt, include_adv)

    def svof(self, c, cs, delta, max_iter=100, tol=1e-6):
        return self.ctx.svof_helmholtz_filter(c, cs, delta, max_iter, tol)

    def curvature(self, cs, kc):
        self.ctx.compute_interface_curvature(cs, kc)

    def csf(self, c, kc, fu, fv):
        self.ctx.compute_csf_force(c, kc, fu, fv)

    def adaptive_dt(self, u, v, dt_max):
        return self.ctx.compute_adaptive_dt(u, v, dt_max)

    def cylinder_mask(self, xc, yc, rad):
        return self.ctx.build_cylinder_mask(xc, yc, rad)

    def krylov(self, solver, X, B, ua, va, pr, dt, tol, max_iter, u_lid=None):
        fn = self.ctx.bicgstab2_solve if solver == 2 else self.ctx.bicgstab_solve
        st = fn(*X, *B, ua, va, pr["rho_c"], pr["rho_u"], pr["rho_v"], pr["kappa"], pr["zeta"], pr["eta"], dt,
                tol, max_iter, u_lid)
        return st["iter"], st["res"], st

    def step(self, st, dt, step_idx, use_bicgstab2=True, u_top_lid=None, tol=None, max_iter=None,
             consistent_amp=False, phi_s=None, u_solid=None, v_solid=None):
        r = self.ctx.advance_coupled_step(
            *[st[k] for k in STATE], dt, step_idx, use_bicgstab2=use_bicgstab2, u_top_lid=u_top_lid,
            tol_in=tol, max_iter_in=max_iter, consistent_amp=consistent_amp,
            phi_s_u=None if phi_s is None else phi_s[0], phi_s_v=None if phi_s is None else phi_s[1],
            u_solid_in=u_solid, v_solid_in=v_solid)

        class S:
            pass

        s = S()
        for k, v in r.items():
            setattr(s, k, v)
        return s


def new_state(be, g, c0):
    st = {k: g.zeros(kind) for k, kind in STATE_KINDS.items()}
    st["c_field"][...] = c0
    pr = be.properties(st["c_field"])
    for k, a in pr.items():
        st[k][...] = a
    return st


def make(backend_cls, g, prm):
    return backend_cls(g, prm)


# ---------------------------------------------------------------- the tests
def halo_exchange(be_cls):
    """tests/test_halo_exchange.f90:19-119 (periodic 64^2, one rank)."""
    g = Grid(64, 64, periodic_x=True, periodic_y=True)
    be = make(be_cls, g, Params())
    phi = g.zeros("cell")
    x = (np.arange(1, 65) - 0.5) * g.dx
    X, Y = np.meshgrid(x, x, indexing="ij")
    at(phi, "cell", slice(1, 64), slice(1, 64))[...] = np.sin(2 * np.pi * X) * np.cos(2 * np.pi * Y)
    be.halo("cell", phi)
    err = 0.0
    for jl in range(-1, 67):
        jg = jl + 64 if jl < 1 else (jl - 64 if jl > 64 else jl)
        y = (jg - 0.5) * g.dy
        for il in list(range(-1, 1)) + list(range(65, 67)):
            ig = il + 64 if il < 1 else il - 64
            xx = (ig - 0.5) * g.dx
            err = max(err, abs(at(phi, "cell", il, jl) - math.sin(2 * math.pi * xx) * math.cos(2 * math.pi * y)))
    for il in range(1, 65):
        xx = (il - 0.5) * g.dx
        for jl in list(range(-1, 1)) + list(range(65, 67)):
            jg = jl + 64 if jl < 1 else jl - 64
            y = (jg - 0.5) * g.dy
            err = max(err, abs(at(phi, "cell", il, jl) - math.sin(2 * math.pi * xx) * math.cos(2 * math.pi * y)))
    _close(be)
    return {"err": err}


def operators(be_cls):
    """tests/test_operators.f90:39-240 (Taylor-Green 64^2 periodic)."""
    g = Grid(64, 64, periodic_x=True, periodic_y=True)
    prm = Params(rho1=1.0, rho2=1.0, mu1=1.0, mu2=1.0)
    be = make(be_cls, g, prm)
    u, v, p, c = g.zeros("u"), g.zeros("v"), g.zeros("cell"), g.full("cell", 1.0)
    ju = np.arange(-1, 67)
    iu = np.arange(-2, 67)
    XF, YN = np.meshgrid(iu * g.dx, (ju - 0.5) * g.dy, indexing="ij")
    u[...] = np.sin(2 * np.pi * XF) * np.cos(2 * np.pi * YN)
    iv, jv = np.arange(-1, 67), np.arange(-2, 67)
    XN, YF = np.meshgrid((iv - 0.5) * g.dx, jv * g.dy, indexing="ij")
    v[...] = -np.cos(2 * np.pi * XN) * np.sin(2 * np.pi * YF)
    ic = np.arange(-1, 67)
    XC, YC = np.meshgrid((ic - 0.5) * g.dx, (ic - 0.5) * g.dy, indexing="ij")
    p[...] = 0.25 * (np.cos(4 * np.pi * XC) + np.cos(4 * np.pi * YC))
    for kind, a in (("u", u), ("v", v), ("cell", p), ("cell", c)):
        be.halo(kind, a)
    pr = be.properties(c)
    div = g.zeros("cell")
    be.divergence(u, v, div)
    div_err = float(np.max(np.abs(at(div, "cell", slice(1, 64), slice(1, 64)))))
    gu, gv = g.zeros("u"), g.zeros("v")
    be.grad_pressure(p, gu, gv)
    xf = np.arange(1, 64) * g.dx
    grad_err = float(np.max(np.abs(at(gu, "u", slice(1, 63), slice(1, 64)) - (-np.pi * np.sin(4 * np.pi * xf))[:, None])))
    vu, vv = g.zeros("u"), g.zeros("v")
    be.viscous_stress(u, v, pr["kappa"], pr["zeta"], pr["eta"], vu, vv)
    XF2, YN2 = np.meshgrid(xf, (np.arange(1, 65) - 0.5) * g.dy, indexing="ij")
    vex = 8 * np.pi ** 2 * np.sin(2 * np.pi * XF2) * np.cos(2 * np.pi * YN2)
    visc_err = float(np.max(np.abs(at(vu, "u", slice(1, 63), slice(1, 64)) - vex)))
    Y = [g.zeros(k) for k in ("u", "v", "cell")]
    be.matvec(u, v, p, *Y, u, v, pr, 1e-3)
    finite = all(np.isfinite(a).all() for a in Y)
    _close(be)
    return {"div_err": div_err, "grad_err": grad_err, "visc_err": visc_err, "matvec_finite": finite}


def lid_driven_cavity(be_cls, max_steps=350):
    """tests/test_lid_driven_cavity.f90:47-250 (32^2, Re = 100, BiCGStab
    tol 1e-4 called directly with a hand-assembled RHS)."""
    g = Grid(32, 32)
    prm = Params(rho1=1.0, rho2=1.0, mu1=0.01, mu2=0.01)
    be = make(be_cls, g, prm)
    st = new_state(be, g, g.full("cell", 1.0))
    pr = {k: st[k] for k in ("rho_c", "rho_u", "rho_v", "kappa", "zeta", "eta")}
    u, v, p = st["u_vel"], st["v_vel"], st["p_field"]
    from_oracle_bcs(be, g, prm, u, v, 1.0)
    dt = 0.01
    steps = 0
    for step in range(1, max_steps + 1):
        steps = step
        u_old, v_old = u.copy(order="F"), v.copy(order="F")
        Bu, Bv, Bp = g.zeros("u"), g.zeros("v"), g.zeros("cell")
        at(Bu, "u", slice(1, 31), slice(1, 32))[...] = at(pr["rho_u"], "u", slice(1, 31), slice(1, 32)) / dt * at(u_old, "u", slice(1, 31), slice(1, 32))
        lid = 2.0 * (at(pr["zeta"], "vert", slice(1, 31), 32) - at(pr["eta"], "vert", slice(1, 31), 32)) / (g.dy * g.dy) * 1.0
        at(Bu, "u", slice(1, 31), 32)[...] += lid
        at(Bv, "v", slice(1, 32), slice(1, 31))[...] = at(pr["rho_v"], "v", slice(1, 32), slice(1, 31)) / dt * at(v_old, "v", slice(1, 32), slice(1, 31))
        be.krylov(1, (u, v, p), (Bu, Bv, Bp), u_old, v_old, pr, dt, 1e-4, 100, 1.0)
        du = float(np.max(np.abs(at(u, "u", slice(1, 32), slice(1, 32)) - at(u_old, "u", slice(1, 32), slice(1, 32)))))
        if du / dt < 1e-4:
            break
    div = g.zeros("cell")
    be.divergence(u, v, div)
    div_max = float(np.max(np.abs(at(div, "cell", slice(1, 32), slice(1, 32)))))
    u_min = float(np.min(at(u, "u", 16, slice(1, 32))))
    vrow = at(v, "v", slice(1, 32), 16)
    _close(be)
    return {"u_min": u_min, "v_min": float(vrow.min()), "v_max": float(vrow.max()), "div": div_max, "steps": steps}


def from_oracle_bcs(be, g, prm, u, v, lid):
    if isinstance(be, GpuBackend):
        be.ctx.apply_velocity_bcs(u, v, lid)
    else:
        be.velocity_bcs(u, v, lid)


def static_droplet(be_cls):
    """tests/test_static_droplet.f90:33-143 (64^2, R = 0.25, SVOF + CSF)."""
    g = Grid(64, 64)
    prm = Params(sigma=1.0)
    be = make(be_cls, g, prm)
    c = cases.binary_circle(g, 0.5, 0.5, 0.25, 1.0)
    cs, kc = g.zeros("cell"), g.zeros("cell")
    be.svof(c, cs, 1.5 * g.dx, 150, 1e-7)
    be.curvature(cs, kc)
    fu, fv = g.zeros("u"), g.zeros("v")
    be.csf(c, kc, fu, fv)
    X, Y = cases.cell_centres_interior(g)
    r = np.sqrt((X - 0.5) ** 2 + (Y - 0.5) ** 2)
    band = np.abs(r - 0.25) <= 1.5 * g.dx
    kmean = float(at(kc, "cell", slice(1, 64), slice(1, 64))[band].mean())
    err = abs(kmean - 4.0) / 4.0 * 100
    fmax = max(float(np.max(np.abs(at(fu, "u", slice(1, 64), slice(1, 64))))),
               float(np.max(np.abs(at(fv, "v", slice(1, 64), slice(1, 64))))))
    _close(be)
    return {"kappa_err_pct": err, "f_max": fmax}


def laplace_coupled(be_cls):
    """tests/test_laplace_coupled.f90:40-196 (64^2, 20 adaptive steps)."""
    g = Grid(64, 64)
    prm = Params(rho1=1.0, rho2=1.0, mu1=0.1, mu2=0.1, sigma=1.0, gx=0.0, gy=0.0, cfl_target=0.25,
                 tol_bicgstab2=1e-5, max_iter_bicgstab2=150)
    be = make(be_cls, g, prm)
    st = new_state(be, g, cases.binary_circle(g, 0.5, 0.5, 0.25, 1.0))
    m0 = cases.fluid1_volume(g, st["c_field"])
    for step in range(1, 21):
        dt = be.adaptive_dt(st["u_vel"], st["v_vel"], 5e-4)
        be.step(st, dt, step, use_bicgstab2=False)
    m1 = cases.fluid1_volume(g, st["c_field"])
    dp = cases.laplace_jump(g, st["p_field"], 0.25)
    ui = at(st["u_vel"], "u", slice(1, 64), slice(1, 64))
    vi = at(st["v_vel"], "v", slice(1, 64), slice(1, 64))
    out = {"laplace_err_pct": abs(dp - 4.0) / 4.0 * 100, "mass_err": abs(m1 - m0) / m0,
           "div": cases.max_divergence(g, st["u_vel"], st["v_vel"]),
           "u_max": float(max(np.abs(ui).max(), np.abs(vi).max()))}
    _close(be)
    return out


def rising_bubble(be_cls):
    """tests/test_rising_bubble.f90:40-192 (32x64, <= 40 adaptive steps, t <= 0.5)."""
    g = Grid(32, 64, 1.0, 2.0)
    prm = Params(rho1=1000.0, rho2=100.0, mu1=10.0, mu2=1.0, sigma=24.5, gx=0.0, gy=-0.98, cfl_target=0.25,
                 tol_bicgstab2=1e-5, max_iter_bicgstab2=150)
    be = make(be_cls, g, prm)
    st = new_state(be, g, cases.initial_colour(g, "rising_bubble"))
    v0 = cases.bubble_volume(g, st["c_field"])
    t = 0.0
    for step in range(1, 41):
        if t >= 0.5:
            break
        dt = be.adaptive_dt(st["u_vel"], st["v_vel"], 2e-3)
        if t + dt > 0.5:
            dt = 0.5 - t
        be.step(st, dt, step, use_bicgstab2=False)
        t += dt
    ycm, vr = cases.bubble_centroid_velocity(g, st["c_field"], st["v_vel"])
    out = {"y_cm": ycm, "v_rise": vr, "mass_err": abs(cases.bubble_volume(g, st["c_field"]) - v0) / v0,
           "div": cases.max_divergence(g, st["u_vel"], st["v_vel"])}
    _close(be)
    return out


def poiseuille(be_cls):
    """tests/test_poiseuille_twophase.f90:36-149 (16x32, periodic x, BDF2)."""
    g = Grid(16, 32, periodic_x=True)
    prm = Params(rho1=1.0, rho2=1.0, mu1=1.0, mu2=0.25, sigma=0.0, gx=1.0, gy=0.0, time_order=2,
                 tol_bicgstab2=1e-7, max_iter_bicgstab2=200)
    be = make(be_cls, g, prm)
    st = new_state(be, g, cases.initial_colour(g, "poiseuille"))
    for step in range(1, 81):
        be.step(st, 0.05, step, use_bicgstab2=False)
    out = poiseuille_error(g, st["u_vel"], 1.0, 1.0, 0.25)
    _close(be)
    return out


def poiseuille_exact(y, G, mu1, mu2, Ly=1.0):
    """piecewise profile of tests/test_poiseuille_twophase.f90:307-323"""
    yi = 0.5 * Ly
    A1 = G * (yi ** 2 / (2 * mu1) + (Ly ** 2 - yi ** 2) / (2 * mu2)) / (yi + (mu1 / mu2) * (Ly - yi))
    A2 = (mu1 / mu2) * A1
    B2 = G * Ly ** 2 / (2 * mu2) - A2 * Ly
    return np.where(y <= yi, -(G / (2 * mu1)) * y ** 2 + A1 * y, -(G / (2 * mu2)) * y ** 2 + A2 * y + B2)


def poiseuille_error(g, u, G, mu1, mu2):
    y = (np.arange(1, g.ny + 1) - 0.5) * g.dy
    ue = poiseuille_exact(y, G, mu1, mu2, g.Ly)[None, :]
    ui = at(u, "u", slice(1, g.nx), slice(1, g.ny))
    err2 = float(np.sum((ui - ue) ** 2) * g.dx * g.dy)
    nrm2 = float(np.sum(np.broadcast_to(ue, ui.shape) ** 2) * g.dx * g.dy)
    return {"rel_l2": math.sqrt(err2 / max(nrm2, 1e-14)), "linf": float(np.max(np.abs(ui - ue)))}


def week6_darcy(be_cls):
    """tests/test_week6_advanced.f90:410-476 part A (Darcy cylinder + BDF2)."""
    g = Grid(32, 32, periodic_x=True)
    prm = Params(rho1=1.0, rho2=1.0, mu1=0.1, mu2=0.1, sigma=0.0, gx=1.0, gy=0.0, time_order=2,
                 alpha_penalty=1e12, tol_bicgstab2=1e-5, max_iter_bicgstab2=150)
    be = make(be_cls, g, prm)
    st = new_state(be, g, g.full("cell", 1.0))
    phi = be.cylinder_mask(0.5, 0.5, 0.15)
    for step in range(1, 11):
        be.step(st, 0.01, step, use_bicgstab2=False, phi_s=phi)
    pu = at(phi[0], "u", slice(1, 32), slice(1, 32)) > 0.5
    pv = at(phi[1], "v", slice(1, 32), slice(1, 32)) > 0.5
    us = max(float(np.max(np.abs(at(st["u_vel"], "u", slice(1, 32), slice(1, 32))[pu]), initial=0.0)),
             float(np.max(np.abs(at(st["v_vel"], "v", slice(1, 32), slice(1, 32))[pv]), initial=0.0)))
    out = {"u_solid": us, "div": cases.max_divergence(g, st["u_vel"], st["v_vel"]), "state": st, "phi": phi,
           "grid": g, "prm": prm}
    _close(be)
    return out


def week6_hysing2_amp(be_cls):
    """tests/test_week6_advanced.f90:518-592 part C (Hysing 2 + AMP + BDF2)."""
    g = Grid(32, 64, 1.0, 2.0)
    prm = Params(rho1=1000.0, rho2=1.0, mu1=10.0, mu2=0.1, sigma=1.96, gx=0.0, gy=-0.98, time_order=2,
                 alpha_penalty=1e12, tol_bicgstab2=1e-5, max_iter_bicgstab2=150)
    be = make(be_cls, g, prm)
    st = new_state(be, g, cases.initial_colour(g, "rising_bubble"))
    v0 = cases.bubble_volume(g, st["c_field"])
    for step in range(1, 21):
        be.step(st, 1e-3, step, use_bicgstab2=False, consistent_amp=True)
    ycm, _ = cases.bubble_centroid_velocity(g, st["c_field"], st["v_vel"])
    out = {"y_cm": ycm, "mass_err": abs(cases.bubble_volume(g, st["c_field"]) - v0) / v0}
    _close(be)
    return out


def _close(be):
    if hasattr(be, "close"):
        be.close()
