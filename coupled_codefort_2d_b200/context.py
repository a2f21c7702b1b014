"""Host-side context of the B200 FUGU-2D hot path.

A :class:`Context` owns one CUDA context handle (``fugu_ctx``) for one grid:
the device-resident state, the Krylov work space and the stream.  Its methods
are the reference's module procedures with the same dummy arguments; the
module globals of the reference (``mod_params``, the grid of ``mod_mpi``) are
the context's :class:`~coupled_codefort_2d_b200.params.Params` and
:class:`~coupled_codefort_2d_b200.layout.Grid`.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import FIELD_ID, FIELD_KIND, FuguError, FuguParams, FuguStats, FuguStepOpts, ptr
from .layout import Grid, as_fortran
from .params import Params

# the state a step maps, in the order of fugu_step_vjp's arguments
VJP_STATE = (("u_vel", "u"), ("v_vel", "v"), ("c_field", "cell"), ("u_prev", "u"), ("v_prev", "v"))


def make_params(g: Grid, prm: Params, precision: int = _lib.FP64) -> FuguParams:
    p = FuguParams()
    _lib.lib().fugu_params_default(C.byref(p))
    p.nx, p.ny, p.dx, p.dy = g.nx, g.ny, g.dx, g.dy
    p.periodic_x, p.periodic_y = int(g.periodic_x), int(g.periodic_y)
    for name, _ in FuguParams._fields_[6:]:
        if name == "precision":
            continue
        setattr(p, name, getattr(prm, name))
    p.precision = precision
    return p


class Context:
    """One case on one GPU (``fugu_create`` / ``fugu_destroy``)."""

    def __init__(self, g: Grid, prm: Params, device: int = 0, precision: int = _lib.FP64):
        self.L = _lib.lib()
        self.g, self.prm, self.precision = g, prm, precision
        self._p = make_params(g, prm, precision)
        h = C.c_void_p()
        rc = self.L.fugu_create(C.byref(self._p), int(device), C.byref(h))
        if rc != 0:
            raise FuguError(rc, f"fugu_create failed for {g} (see stderr)")
        self.h = h

    @classmethod
    def view(cls, handle, g: Grid, prm: Params, precision: int = _lib.FP64) -> "Context":
        """A non-owning Context over a handle another object owns (a batch case)."""
        self = cls.__new__(cls)
        self.L = _lib.lib()
        self.g, self.prm, self.precision = g, prm, precision
        self._p = make_params(g, prm, precision)
        self.h = handle
        self._owned = False
        return self

    # -------------------------------------------------------------- plumbing
    def close(self):
        if getattr(self, "h", None):
            if getattr(self, "_owned", True):
                self.L.fugu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _ck(self, rc):
        if rc != 0:
            raise FuguError(rc, self.L.fugu_last_error(self.h).decode())

    def set_params(self, prm: Params, precision: int | None = None):
        self.prm = prm
        if precision is not None:
            self.precision = precision
        self._p = make_params(self.g, prm, self.precision)
        self._ck(self.L.fugu_set_params(self.h, C.byref(self._p)))

    def stream_handle(self) -> int:
        """cudaStream_t of the context (for torch.cuda.ExternalStream)."""
        s = C.c_void_p()
        self._ck(self.L.fugu_get_stream(self.h, C.byref(s)))
        return s.value or 0

    def profile(self, enable: int = -1) -> dict:
        """Read the measurement counters; enable >= 0 resets them and turns
        PCG event timing on (1) or off (0)."""
        out = _lib.FuguProfile()
        self._ck(self.L.fugu_profile(self.h, int(enable), C.byref(out)))
        return out.as_dict()

    def arm_barrier_timeout(self, spin_limit: int = 1000):
        """Failure-detection test hook: the next grid-wide PCG launch of this
        context waits for one CTA too many at its grid barriers and gives up
        after ``spin_limit`` polls, so the call that made it raises
        FUGU_ETIMEOUT (``fugu_test_arm_barrier_timeout``)."""
        self._ck(self.L.fugu_test_arm_barrier_timeout(self.h, int(spin_limit)))

    def _f(self, a, kind):
        return ptr(as_fortran(a, self.g, kind))

    def _o(self, a, kind):
        return None if a is None else self._f(a, kind)

    # -------------------------------------------------------- device state
    def upload(self, name: str, a: np.ndarray):
        self._ck(self.L.fugu_upload(self.h, FIELD_ID[name], self._f(a, FIELD_KIND[name])))

    def download(self, name: str, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = self.g.zeros(FIELD_KIND[name])
        self._ck(self.L.fugu_download(self.h, FIELD_ID[name], self._f(out, FIELD_KIND[name])))
        return out

    def upload_state(self, st: dict):
        for k, a in st.items():
            if k in FIELD_ID:
                self.upload(k, a)

    def download_state(self, names=None) -> dict:
        names = names or FIELD_ID.keys()
        return {k: self.download(k) for k in names}

    @staticmethod
    def step_opts(use_bicgstab2=True, u_top_lid=None, tol=None, max_iter=None, consistent_amp=False,
                  penalty=False, u_solid=None, v_solid=None) -> FuguStepOpts:
        o = FuguStepOpts()
        o.use_bicgstab2 = int(use_bicgstab2)
        o.has_lid = int(u_top_lid is not None)
        o.u_top_lid = 0.0 if u_top_lid is None else float(u_top_lid)
        o.has_tol = int(tol is not None)
        o.tol = 0.0 if tol is None else float(tol)
        o.has_max_iter = int(max_iter is not None)
        o.max_iter = 0 if max_iter is None else int(max_iter)
        o.consistent_amp = int(consistent_amp)
        o.has_penalty = int(penalty)
        o.has_u_solid = int(u_solid is not None)
        o.u_solid = 0.0 if u_solid is None else float(u_solid)
        o.has_v_solid = int(v_solid is not None)
        o.v_solid = 0.0 if v_solid is None else float(v_solid)
        return o

    def step(self, dt: float, step_idx: int, opts: FuguStepOpts) -> dict:
        """``advance_coupled_step`` on the device-resident state."""
        st = FuguStats()
        self._ck(self.L.fugu_step(self.h, float(dt), int(step_idx), C.byref(opts), C.byref(st)))
        return st.as_dict()

    def step_vjp(self, dt: float, step_idx: int, opts: FuguStepOpts, bar_out: dict):
        """Advance the device-resident state by one step, as ``step`` does, and
        return the adjoints of the state before it from those of the state
        after it (``fugu_step_vjp``; no counterpart in the reference).

        bar_out maps u_vel, v_vel, c_field, u_prev, v_prev to adjoint arrays in
        the reference layout (a missing key is zero).  Returns (bar_in with the
        same keys, d/d(sigma, mu1, mu2, rho1, rho2) of the step, statistics of
        the forward step with ``status`` the adjoint solve's)."""
        g = self.g
        bo = [g.zeros(kind) if bar_out.get(k) is None else as_fortran(bar_out[k], g, kind)
              for k, kind in VJP_STATE]
        bi = [g.zeros(kind) for _, kind in VJP_STATE]
        theta = np.zeros(5)
        st = FuguStats()
        self._ck(self.L.fugu_step_vjp(self.h, float(dt), int(step_idx), C.byref(opts), *[ptr(a) for a in bo],
                                      *[ptr(a) for a in bi], ptr(theta), C.byref(st)))
        return {k: a for (k, _), a in zip(VJP_STATE, bi)}, theta, st.as_dict()

    # --------------------------------------------- mod_solver_coupled mirror
    def advance_coupled_step(self, u_vel, v_vel, p_field, c_field, u_prev, v_prev, rho_c, rho_u, rho_v,
                             kappa, zeta, eta, kappa_curv, f_sigma_u, f_sigma_v, dt_step, step_idx,
                             use_bicgstab2=True, u_top_lid=None, tol_in=None, max_iter_in=None,
                             consistent_amp=False, phi_s_u=None, phi_s_v=None, u_solid_in=None,
                             v_solid_in=None) -> dict:
        """Drop-in of ``advance_coupled_step`` (mod_solver_coupled.f90:137-380)
        on host arrays; returns iter_out / res_out and statistics."""
        o = self.step_opts(use_bicgstab2, u_top_lid, tol_in, max_iter_in, consistent_amp,
                           phi_s_u is not None and phi_s_v is not None, u_solid_in, v_solid_in)
        st = FuguStats()
        g = self.g
        args = [self._f(a, k) for a, k in ((u_vel, "u"), (v_vel, "v"), (p_field, "cell"), (c_field, "cell"),
                                          (u_prev, "u"), (v_prev, "v"), (rho_c, "cell"), (rho_u, "u"),
                                          (rho_v, "v"), (kappa, "cell"), (zeta, "vert"), (eta, "vert"),
                                          (kappa_curv, "cell"), (f_sigma_u, "u"), (f_sigma_v, "v"))]
        args += [self._o(phi_s_u, "u"), self._o(phi_s_v, "v")]
        self._ck(self.L.fugu_advance_coupled_step(self.h, *args, float(dt_step), int(step_idx), C.byref(o),
                                                  C.byref(st)))
        del g
        return st.as_dict()

    def compute_adaptive_dt(self, u_vel, v_vel, dt_max) -> float:
        out = C.c_double()
        self._ck(self.L.fugu_compute_adaptive_dt(self.h, self._f(u_vel, "u"), self._f(v_vel, "v"),
                                                 float(dt_max), C.byref(out)))
        return out.value

    def build_cylinder_mask(self, xc, yc, rad):
        pu, pv = self.g.zeros("u"), self.g.zeros("v")
        self._ck(self.L.fugu_build_cylinder_mask(self.h, float(xc), float(yc), float(rad), ptr(pu), ptr(pv)))
        return pu, pv

    # ---------------------------------------------------------- mod_mpi mirror
    def halo(self, kind, a):
        fn = {"cell": self.L.fugu_halo_scalar, "u": self.L.fugu_halo_u, "v": self.L.fugu_halo_v}[kind]
        self._ck(fn(self.h, self._f(a, kind)))

    # ---------------------------------------------------- mod_viscosity mirror
    def compute_mixture_densities(self, c_field, rho_c, rho_u, rho_v):
        self._ck(self.L.fugu_compute_mixture_densities(self.h, self._f(c_field, "cell"), self._f(rho_c, "cell"),
                                                       self._f(rho_u, "u"), self._f(rho_v, "v")))

    def compute_mixture_viscosities(self, c_field, kappa, zeta, eta):
        self._ck(self.L.fugu_compute_mixture_viscosities(self.h, self._f(c_field, "cell"), self._f(kappa, "cell"),
                                                         self._f(zeta, "vert"), self._f(eta, "vert")))

    # ---------------------------------------------------- mod_operators mirror
    def op_divergence(self, u, v, div):
        self._ck(self.L.fugu_op_divergence(self.h, self._f(u, "u"), self._f(v, "v"), self._f(div, "cell")))

    def op_grad_pressure(self, p, gu, gv):
        self._ck(self.L.fugu_op_grad_pressure(self.h, self._f(p, "cell"), self._f(gu, "u"), self._f(gv, "v")))

    def op_viscous_stress(self, u, v, kappa, zeta, eta, visc_u, visc_v):
        self._ck(self.L.fugu_op_viscous_stress(self.h, self._f(u, "u"), self._f(v, "v"), self._f(kappa, "cell"),
                                               self._f(zeta, "vert"), self._f(eta, "vert"), self._f(visc_u, "u"),
                                               self._f(visc_v, "v")))

    def op_advection(self, u_adv, v_adv, rho_c, rho_u, rho_v, u, v, adv_u, adv_v, mdot_u_cons=None,
                     mdot_v_cons=None):
        self._ck(self.L.fugu_op_advection(self.h, self._f(u_adv, "u"), self._f(v_adv, "v"), self._f(rho_c, "cell"),
                                          self._f(rho_u, "u"), self._f(rho_v, "v"), self._f(u, "u"), self._f(v, "v"),
                                          self._f(adv_u, "u"), self._f(adv_v, "v"), self._o(mdot_u_cons, "u"),
                                          self._o(mdot_v_cons, "v")))

    def apply_velocity_bcs(self, u, v, u_top_lid=None):
        self._ck(self.L.fugu_apply_velocity_bcs(self.h, self._f(u, "u"), self._f(v, "v"), int(u_top_lid is not None),
                                                0.0 if u_top_lid is None else float(u_top_lid)))

    def matvec_coupled(self, X_u, X_v, X_p, Y_u, Y_v, Y_p, u_adv, v_adv, rho_c, rho_u, rho_v, kappa, zeta, eta,
                       dt_step, include_advection=True, penalty_u=None, penalty_v=None, mdot_u_cons=None,
                       mdot_v_cons=None):
        self._ck(self.L.fugu_matvec_coupled(
            self.h, self._f(X_u, "u"), self._f(X_v, "v"), self._f(X_p, "cell"), self._f(Y_u, "u"),
            self._f(Y_v, "v"), self._f(Y_p, "cell"), self._f(u_adv, "u"), self._f(v_adv, "v"),
            self._f(rho_c, "cell"), self._f(rho_u, "u"), self._f(rho_v, "v"), self._f(kappa, "cell"),
            self._f(zeta, "vert"), self._f(eta, "vert"), float(dt_step), int(include_advection),
            self._o(penalty_u, "u"), self._o(penalty_v, "v"), self._o(mdot_u_cons, "u"), self._o(mdot_v_cons, "v")))

    # --------------------------------------------------- mod_subsolvers mirror
    def solve_poisson_pressure(self, phi, rhs, rho_u, rho_v, tol_in=1.0e-5, max_iter_in=150):
        it, res = C.c_int(), C.c_double()
        self._ck(self.L.fugu_solve_poisson_pressure(self.h, self._f(phi, "cell"), self._f(rhs, "cell"),
                                                    self._f(rho_u, "u"), self._f(rho_v, "v"), float(tol_in),
                                                    int(max_iter_in), C.byref(it), C.byref(res)))
        return it.value, res.value

    def solve_helmholtz_u(self, u_sol, rhs_u, rho_u, kappa, zeta, eta, dt_step, n_sweeps_in=5, penalty_u=None):
        self._ck(self.L.fugu_solve_helmholtz_u(self.h, self._f(u_sol, "u"), self._f(rhs_u, "u"), self._f(rho_u, "u"),
                                               self._f(kappa, "cell"), self._f(zeta, "vert"), self._f(eta, "vert"),
                                               float(dt_step), int(n_sweeps_in), self._o(penalty_u, "u")))

    def solve_helmholtz_v(self, v_sol, rhs_v, rho_v, kappa, zeta, eta, dt_step, n_sweeps_in=5, penalty_v=None):
        self._ck(self.L.fugu_solve_helmholtz_v(self.h, self._f(v_sol, "v"), self._f(rhs_v, "v"), self._f(rho_v, "v"),
                                               self._f(kappa, "cell"), self._f(zeta, "vert"), self._f(eta, "vert"),
                                               float(dt_step), int(n_sweeps_in), self._o(penalty_v, "v")))

    # -------------------------------------------------- mod_pcd_precond mirror
    def apply_pcd_precond(self, z_u, z_v, z_p, r_u, r_v, r_p, u_adv, v_adv, rho_u, rho_v, kappa, zeta, eta,
                          dt_step, penalty_u=None, penalty_v=None):
        self._ck(self.L.fugu_apply_pcd_precond(
            self.h, self._f(z_u, "u"), self._f(z_v, "v"), self._f(z_p, "cell"), self._f(r_u, "u"),
            self._f(r_v, "v"), self._f(r_p, "cell"), self._f(u_adv, "u"), self._f(v_adv, "v"),
            self._f(rho_u, "u"), self._f(rho_v, "v"), self._f(kappa, "cell"), self._f(zeta, "vert"),
            self._f(eta, "vert"), float(dt_step), self._o(penalty_u, "u"), self._o(penalty_v, "v")))

    # ---------------------------------------------------- mod_bicgstab2 mirror
    def coupled_dot(self, u1, v1, p1, u2, v2, p2) -> float:
        out = C.c_double()
        self._ck(self.L.fugu_coupled_dot(self.h, self._f(u1, "u"), self._f(v1, "v"), self._f(p1, "cell"),
                                         self._f(u2, "u"), self._f(v2, "v"), self._f(p2, "cell"), C.byref(out)))
        return out.value

    def _krylov(self, solver, X_u, X_v, X_p, B_u, B_v, B_p, u_adv, v_adv, rho_c, rho_u, rho_v, kappa, zeta, eta,
                dt_step, tol_in=1.0e-5, max_iter_in=100, u_top_lid=None, penalty_u=None, penalty_v=None,
                mdot_u_cons=None, mdot_v_cons=None) -> dict:
        st = FuguStats()
        self._ck(self.L.fugu_krylov_solve(
            self.h, int(solver), self._f(X_u, "u"), self._f(X_v, "v"), self._f(X_p, "cell"), self._f(B_u, "u"),
            self._f(B_v, "v"), self._f(B_p, "cell"), self._f(u_adv, "u"), self._f(v_adv, "v"),
            self._f(rho_c, "cell"), self._f(rho_u, "u"), self._f(rho_v, "v"), self._f(kappa, "cell"),
            self._f(zeta, "vert"), self._f(eta, "vert"), float(dt_step), float(tol_in), int(max_iter_in),
            int(u_top_lid is not None), 0.0 if u_top_lid is None else float(u_top_lid),
            self._o(penalty_u, "u"), self._o(penalty_v, "v"), self._o(mdot_u_cons, "u"), self._o(mdot_v_cons, "v"),
            C.byref(st)))
        return st.as_dict()

    # ------------------------------------------------------ discrete adjoint
    def matvec_coupled_t(self, Y_u, Y_v, Y_p, X_u, X_v, X_p, u_adv, v_adv, rho_c, rho_u, rho_v, kappa, zeta, eta,
                         dt_step, penalty_u=None, penalty_v=None, mdot_u_cons=None, mdot_v_cons=None):
        """X = A^T Y for the solvers' operator A: x -> matvec_coupled(BC(x)) on
        the owned unknowns (no counterpart in the reference)."""
        self._ck(self.L.fugu_matvec_coupled_t(
            self.h, self._f(Y_u, "u"), self._f(Y_v, "v"), self._f(Y_p, "cell"), self._f(X_u, "u"),
            self._f(X_v, "v"), self._f(X_p, "cell"), self._f(u_adv, "u"), self._f(v_adv, "v"),
            self._f(rho_c, "cell"), self._f(rho_u, "u"), self._f(rho_v, "v"), self._f(kappa, "cell"),
            self._f(zeta, "vert"), self._f(eta, "vert"), float(dt_step), self._o(penalty_u, "u"),
            self._o(penalty_v, "v"), self._o(mdot_u_cons, "u"), self._o(mdot_v_cons, "v")))

    def adjoint_solve(self, g_u, g_v, g_p, lam_u, lam_v, lam_p, u_adv, v_adv, rho_c, rho_u, rho_v, kappa, zeta, eta,
                      dt_step, tol=1e-10, penalty_u=None, penalty_v=None, mdot_u_cons=None, mdot_v_cons=None) -> dict:
        """Solve A^T lambda = g (no counterpart in the reference)."""
        st = FuguStats()
        self._ck(self.L.fugu_adjoint_solve(
            self.h, self._f(g_u, "u"), self._f(g_v, "v"), self._f(g_p, "cell"), self._f(lam_u, "u"),
            self._f(lam_v, "v"), self._f(lam_p, "cell"), self._f(u_adv, "u"), self._f(v_adv, "v"),
            self._f(rho_c, "cell"), self._f(rho_u, "u"), self._f(rho_v, "v"), self._f(kappa, "cell"),
            self._f(zeta, "vert"), self._f(eta, "vert"), float(dt_step), float(tol), self._o(penalty_u, "u"),
            self._o(penalty_v, "v"), self._o(mdot_u_cons, "u"), self._o(mdot_v_cons, "v"), C.byref(st)))
        return st.as_dict()

    def bicgstab_solve(self, *a, **kw) -> dict:
        """``bicgstab_solve`` (mod_bicgstab2.f90:77-264); returns stats with
        iter (iter_out) and res (res_out)."""
        return self._krylov(1, *a, **kw)

    def bicgstab2_solve(self, *a, **kw) -> dict:
        """``bicgstab2_solve`` (mod_bicgstab2.f90:270-570)."""
        return self._krylov(2, *a, **kw)

    # ---------------------------------------------------------- mod_vof mirror
    def vof_advection_tvd(self, C_in, C_out, u_vel, v_vel, dt_step, flux_x_out=None, flux_y_out=None):
        self._ck(self.L.fugu_vof_advection_tvd(self.h, self._f(C_in, "cell"), self._f(C_out, "cell"),
                                               self._f(u_vel, "u"), self._f(v_vel, "v"), float(dt_step),
                                               self._o(flux_x_out, "u"), self._o(flux_y_out, "v")))

    def svof_helmholtz_filter(self, C_raw, C_smooth, delta_filter, max_iter=100, tol=1.0e-6) -> int:
        it = C.c_int()
        self._ck(self.L.fugu_svof_helmholtz_filter(self.h, self._f(C_raw, "cell"), self._f(C_smooth, "cell"),
                                                   float(delta_filter), int(max_iter), float(tol), C.byref(it)))
        return it.value

    # ---------------------------------------------- mod_surface_tension mirror
    def compute_interface_curvature(self, C_smooth, kappa_curv):
        self._ck(self.L.fugu_compute_interface_curvature(self.h, self._f(C_smooth, "cell"),
                                                         self._f(kappa_curv, "cell")))

    def compute_csf_force(self, C_raw, kappa_curv, f_sigma_u, f_sigma_v):
        self._ck(self.L.fugu_compute_csf_force(self.h, self._f(C_raw, "cell"), self._f(kappa_curv, "cell"),
                                               self._f(f_sigma_u, "u"), self._f(f_sigma_v, "v")))

    # ----------------------------------------------------------- mod_io mirror
    def write_checkpoint(self, path: str, step: int, t: float):
        self._ck(self.L.fugu_write_checkpoint(self.h, path.encode(), int(step), float(t)))

    def read_checkpoint(self, path: str):
        step, t = C.c_int(), C.c_double()
        self._ck(self.L.fugu_read_checkpoint(self.h, path.encode(), C.byref(step), C.byref(t)))
        return step.value, t.value
