"""ctypes binding of the CPU oracle (``oracle/libfugu_oracle.so``).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU legs of ``bench.py`` as the checker.  The product never imports it.

Arrays are numpy float64 arrays in Fortran order with the padded shapes of
``coupled_codefort_2d_b200.layout``; they are passed by the address of their
first (lower-bound) element, exactly as the Fortran reference passes them.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfugu_oracle.so")


class FoModel(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("dx", C.c_double), ("dy", C.c_double),
        ("periodic_x", C.c_int), ("periodic_y", C.c_int),
        ("rho1", C.c_double), ("rho2", C.c_double), ("mu1", C.c_double), ("mu2", C.c_double),
        ("sigma", C.c_double), ("gx", C.c_double), ("gy", C.c_double),
        ("cfl_target", C.c_double), ("alpha_penalty", C.c_double),
        ("time_order", C.c_int), ("tol_bicgstab2", C.c_double), ("max_iter_bicgstab2", C.c_int),
        ("pcg_tol", C.c_double), ("pcg_max_iter", C.c_int), ("pcd_sweeps", C.c_int),
        ("jacobi_omega", C.c_double), ("svof_delta_h", C.c_double), ("svof_max_iter", C.c_int),
        ("svof_tol", C.c_double), ("limiter", C.c_int), ("free_slip_x", C.c_int),
        ("krylov_bc_fix", C.c_int), ("refine", C.c_int), ("refine_inner_tol", C.c_double),
        ("refine_max_inner", C.c_int), ("refine_max_outer", C.c_int), ("pcg_cap_start", C.c_int),
        ("pcd_sweeps_max", C.c_int), ("pcd_smoother", C.c_int), ("pcd_sor_omega", C.c_double),
        ("pcd_visc_scale", C.c_double),
    ]


class FoStepOpts(C.Structure):
    _fields_ = [
        ("use_bicgstab2", C.c_int), ("has_lid", C.c_int), ("u_top_lid", C.c_double),
        ("has_tol", C.c_int), ("tol", C.c_double), ("has_max_iter", C.c_int), ("max_iter", C.c_int),
        ("consistent_amp", C.c_int), ("phi_s_u", C.c_void_p), ("phi_s_v", C.c_void_p),
        ("has_u_solid", C.c_int), ("u_solid", C.c_double), ("has_v_solid", C.c_int),
        ("v_solid", C.c_double),
    ]


class FoStats(C.Structure):
    _fields_ = [
        ("iter", C.c_int), ("res", C.c_double), ("pcg_iters", C.c_long), ("pcg_calls", C.c_int),
        ("svof_iters", C.c_int), ("matvecs", C.c_int), ("outer", C.c_int), ("pcg_cap", C.c_int),
        ("pcd_sweeps", C.c_int),
    ]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = C.CDLL(LIB_PATH)
        _lib.fo_harmonic_viscosity.restype = C.c_double
        _lib.fo_coupled_dot.restype = C.c_double
        _lib.fo_compute_adaptive_dt.restype = C.c_double
        _lib.fo_svof_helmholtz_filter.restype = C.c_int
    return _lib


def P(a):
    """Address of a Fortran-ordered float64 array (None -> NULL)."""
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.f_contiguous, "oracle arrays must be F-ordered float64"
    return C.c_void_p(a.ctypes.data)


def model(g, prm) -> FoModel:
    m = FoModel()
    m.nx, m.ny, m.dx, m.dy = g.nx, g.ny, g.dx, g.dy
    m.periodic_x, m.periodic_y = int(g.periodic_x), int(g.periodic_y)
    for name, _ in FoModel._fields_[6:]:
        setattr(m, name, getattr(prm, name))
    return m


def D(x):
    return C.c_double(x)


# ------------------------------------------------------------------ wrappers
class Oracle:
    """Thin object mirror of the restated Fortran modules for one grid."""

    def __init__(self, g, prm):
        self.g, self.prm = g, prm
        self.m = model(g, prm)
        self.L = lib()
        self.pcg_cap = 0  # adaptive PCG cap carried from solve to solve (refine = 2)
        self.pcd_sweeps = 0  # adaptive PCD sweeps, likewise

    def halo(self, kind, a):
        fn = {"cell": self.L.fo_halo_scalar, "u": self.L.fo_halo_u, "v": self.L.fo_halo_v}[kind]
        fn(C.byref(self.m), P(a))

    def densities(self, c, rho_c, rho_u, rho_v):
        self.L.fo_compute_mixture_densities(C.byref(self.m), P(c), P(rho_c), P(rho_u), P(rho_v))

    def viscosities(self, c, kappa, zeta, eta):
        self.L.fo_compute_mixture_viscosities(C.byref(self.m), P(c), P(kappa), P(zeta), P(eta))

    def properties(self, c):
        g = self.g
        out = {k: g.zeros(kd) for k, kd in (("rho_c", "cell"), ("rho_u", "u"), ("rho_v", "v"),
                                             ("kappa", "cell"), ("zeta", "vert"), ("eta", "vert"))}
        self.densities(c, out["rho_c"], out["rho_u"], out["rho_v"])
        self.viscosities(c, out["kappa"], out["zeta"], out["eta"])
        return out

    def divergence(self, u, v, div):
        self.L.fo_op_divergence(C.byref(self.m), P(u), P(v), P(div))

    def grad_pressure(self, p, gu, gv):
        self.L.fo_op_grad_pressure(C.byref(self.m), P(p), P(gu), P(gv))

    def viscous_stress(self, u, v, kappa, zeta, eta, vu, vv):
        self.L.fo_op_viscous_stress(C.byref(self.m), P(u), P(v), P(kappa), P(zeta), P(eta), P(vu), P(vv))

    def advection(self, uadv, vadv, rho_c, rho_u, rho_v, u, v, au, av, mdu=None, mdv=None):
        self.L.fo_op_advection(C.byref(self.m), P(uadv), P(vadv), P(rho_c), P(rho_u), P(rho_v),
                               P(u), P(v), P(au), P(av), P(mdu), P(mdv))

    def velocity_bcs(self, u, v, u_lid=None):
        self.L.fo_apply_velocity_bcs(C.byref(self.m), P(u), P(v), int(u_lid is not None),
                                     D(0.0 if u_lid is None else u_lid))

    def matvec(self, Xu, Xv, Xp, Yu, Yv, Yp, uadv, vadv, pr, dt, include_adv=True,
               pen_u=None, pen_v=None, mdu=None, mdv=None):
        self.L.fo_matvec_coupled(C.byref(self.m), P(Xu), P(Xv), P(Xp), P(Yu), P(Yv), P(Yp),
                                 P(uadv), P(vadv), P(pr["rho_c"]), P(pr["rho_u"]), P(pr["rho_v"]),
                                 P(pr["kappa"]), P(pr["zeta"]), P(pr["eta"]), D(dt),
                                 int(include_adv), P(pen_u), P(pen_v), P(mdu), P(mdv))

    def poisson(self, phi, rhs, rho_u, rho_v, tol=1e-5, max_iter=150):
        it = C.c_int(0)
        res = C.c_double(0.0)
        self.L.fo_solve_poisson_pressure(C.byref(self.m), P(phi), P(rhs), P(rho_u), P(rho_v),
                                         D(tol), int(max_iter), C.byref(it), C.byref(res))
        return it.value, res.value

    def helmholtz_u(self, u_sol, rhs, pr, dt, n_sweeps=5, pen_u=None):
        self.L.fo_solve_helmholtz_u(C.byref(self.m), P(u_sol), P(rhs), P(pr["rho_u"]), P(pr["kappa"]),
                                    P(pr["zeta"]), P(pr["eta"]), D(dt), int(n_sweeps), P(pen_u))

    def helmholtz_v(self, v_sol, rhs, pr, dt, n_sweeps=5, pen_v=None):
        self.L.fo_solve_helmholtz_v(C.byref(self.m), P(v_sol), P(rhs), P(pr["rho_v"]), P(pr["kappa"]),
                                    P(pr["zeta"]), P(pr["eta"]), D(dt), int(n_sweeps), P(pen_v))

    def pcd(self, zu, zv, zp, ru, rv, rp, uadv, vadv, pr, dt, pen_u=None, pen_v=None):
        st = FoStats()
        self.L.fo_apply_pcd_precond(C.byref(self.m), P(zu), P(zv), P(zp), P(ru), P(rv), P(rp),
                                    P(uadv), P(vadv), P(pr["rho_u"]), P(pr["rho_v"]), P(pr["kappa"]),
                                    P(pr["zeta"]), P(pr["eta"]), D(dt), P(pen_u), P(pen_v), C.byref(st))
        return st

    def coupled_dot(self, a, b):
        return self.L.fo_coupled_dot(C.byref(self.m), P(a[0]), P(a[1]), P(a[2]), P(b[0]), P(b[1]), P(b[2]))

    def krylov(self, solver, X, B, uadv, vadv, pr, dt, tol, max_iter, u_lid=None,
               pen_u=None, pen_v=None, mdu=None, mdv=None):
        it = C.c_int(0)
        res = C.c_double(0.0)
        st = FoStats()
        st.pcg_cap = self.pcg_cap
        st.pcd_sweeps = self.pcd_sweeps
        self.L.fo_krylov_solve(C.byref(self.m), int(solver), P(X[0]), P(X[1]), P(X[2]),
                               P(B[0]), P(B[1]), P(B[2]), P(uadv), P(vadv), P(pr["rho_c"]),
                               P(pr["rho_u"]), P(pr["rho_v"]), P(pr["kappa"]), P(pr["zeta"]),
                               P(pr["eta"]), D(dt), D(tol), int(max_iter), int(u_lid is not None),
                               D(0.0 if u_lid is None else u_lid), P(pen_u), P(pen_v), P(mdu), P(mdv),
                               C.byref(it), C.byref(res), C.byref(st))
        self.pcg_cap = st.pcg_cap
        self.pcd_sweeps = st.pcd_sweeps
        return it.value, res.value, st

    def vof(self, c_in, c_out, u, v, dt, fx=None, fy=None):
        self.L.fo_vof_advection_tvd(C.byref(self.m), P(c_in), P(c_out), P(u), P(v), D(dt), P(fx), P(fy))

    def svof(self, c_raw, c_s, delta, max_iter=100, tol=1e-6):
        return self.L.fo_svof_helmholtz_filter(C.byref(self.m), P(c_raw), P(c_s), D(delta),
                                               int(max_iter), D(tol))

    def curvature(self, c_s, kc):
        self.L.fo_compute_interface_curvature(C.byref(self.m), P(c_s), P(kc))

    def csf(self, c, kc, fsu, fsv):
        self.L.fo_compute_csf_force(C.byref(self.m), P(c), P(kc), P(fsu), P(fsv))

    def adaptive_dt(self, u, v, dt_max):
        return self.L.fo_compute_adaptive_dt(C.byref(self.m), P(u), P(v), D(dt_max))

    def cylinder_mask(self, xc, yc, rad):
        pu, pv = self.g.zeros("u"), self.g.zeros("v")
        self.L.fo_build_cylinder_mask(C.byref(self.m), D(xc), D(yc), D(rad), P(pu), P(pv))
        return pu, pv

    def step(self, st, dt, step_idx, use_bicgstab2=True, u_top_lid=None, tol=None, max_iter=None,
             consistent_amp=False, phi_s=None, u_solid=None, v_solid=None):
        """advance_coupled_step on a state dict (keys as the Fortran dummies)."""
        o = FoStepOpts()
        o.use_bicgstab2 = int(use_bicgstab2)
        o.has_lid = int(u_top_lid is not None)
        o.u_top_lid = 0.0 if u_top_lid is None else u_top_lid
        o.has_tol = int(tol is not None)
        o.tol = 0.0 if tol is None else tol
        o.has_max_iter = int(max_iter is not None)
        o.max_iter = 0 if max_iter is None else max_iter
        o.consistent_amp = int(consistent_amp)
        if phi_s is not None:
            o.phi_s_u = phi_s[0].ctypes.data
            o.phi_s_v = phi_s[1].ctypes.data
        o.has_u_solid = int(u_solid is not None)
        o.u_solid = 0.0 if u_solid is None else u_solid
        o.has_v_solid = int(v_solid is not None)
        o.v_solid = 0.0 if v_solid is None else v_solid
        stats = FoStats()
        stats.pcg_cap = self.pcg_cap
        stats.pcd_sweeps = self.pcd_sweeps
        self.L.fo_advance_coupled_step(
            C.byref(self.m), P(st["u_vel"]), P(st["v_vel"]), P(st["p_field"]), P(st["c_field"]),
            P(st["u_prev"]), P(st["v_prev"]), P(st["rho_c"]), P(st["rho_u"]), P(st["rho_v"]),
            P(st["kappa"]), P(st["zeta"]), P(st["eta"]), P(st["kappa_curv"]), P(st["f_sigma_u"]),
            P(st["f_sigma_v"]), D(dt), int(step_idx), C.byref(o), C.byref(stats))
        self.pcg_cap = stats.pcg_cap
        self.pcd_sweeps = stats.pcd_sweeps
        return stats

    def write_checkpoint(self, path, step, t, st):
        return self.L.fo_write_checkpoint(C.byref(self.m), path.encode(), int(step), D(t),
                                          P(st["u_vel"]), P(st["v_vel"]), P(st["u_prev"]),
                                          P(st["v_prev"]), P(st["p_field"]), P(st["c_field"]))

    def read_checkpoint(self, path, st):
        step = C.c_int(0)
        t = C.c_double(0.0)
        rc = self.L.fo_read_checkpoint(C.byref(self.m), path.encode(), C.byref(step), C.byref(t),
                                       P(st["u_vel"]), P(st["v_vel"]), P(st["u_prev"]),
                                       P(st["v_prev"]), P(st["p_field"]), P(st["c_field"]))
        return rc, step.value, t.value


STATE_KINDS = {
    "u_vel": "u", "v_vel": "v", "p_field": "cell", "c_field": "cell", "u_prev": "u", "v_prev": "v",
    "rho_c": "cell", "rho_u": "u", "rho_v": "v", "kappa": "cell", "zeta": "vert", "eta": "vert",
    "kappa_curv": "cell", "f_sigma_u": "u", "f_sigma_v": "v",
}


def new_state(g, c_field, prm):
    """Zero velocity/pressure state with properties from C (the drivers'
    set-up, e.g. ``main.f90:105-111,185-186``)."""
    st = {k: g.zeros(kind) for k, kind in STATE_KINDS.items()}
    st["c_field"][...] = c_field
    o = Oracle(g, prm)
    o.densities(st["c_field"], st["rho_c"], st["rho_u"], st["rho_v"])
    o.viscosities(st["c_field"], st["kappa"], st["zeta"], st["eta"])
    return st
