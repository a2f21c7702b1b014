"""ctypes binding of ``libfugu_gpu.so`` (declarations in ``include/fugu_gpu.h``).

The product path has no CPU fallback: if the library is missing or cannot be
loaded this module raises, and every solver entry fails loudly.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfugu_gpu.so")

FUGU_OK = 0
ERRORS = {-1: "FUGU_EINVAL", -2: "FUGU_ECUDA", -3: "FUGU_ENOMEM", -4: "FUGU_EIO", -5: "FUGU_ETIMEOUT"}
CONVERGED, MAXITER, BREAKDOWN, NAN = 0, 1, 2, 3
FP64, MIXED = 0, 1

FIELDS = [
    "u_vel", "v_vel", "p_field", "c_field", "u_prev", "v_prev", "rho_c", "rho_u", "rho_v",
    "kappa", "zeta", "eta", "kappa_curv", "f_sigma_u", "f_sigma_v", "phi_s_u", "phi_s_v",
]
FIELD_ID = {name: i for i, name in enumerate(FIELDS)}
FIELD_KIND = {
    "u_vel": "u", "v_vel": "v", "p_field": "cell", "c_field": "cell", "u_prev": "u", "v_prev": "v",
    "rho_c": "cell", "rho_u": "u", "rho_v": "v", "kappa": "cell", "zeta": "vert", "eta": "vert",
    "kappa_curv": "cell", "f_sigma_u": "u", "f_sigma_v": "v", "phi_s_u": "u", "phi_s_v": "v",
}


class FuguParams(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("dx", C.c_double), ("dy", C.c_double),
        ("periodic_x", C.c_int), ("periodic_y", C.c_int),
        ("rho1", C.c_double), ("rho2", C.c_double), ("mu1", C.c_double), ("mu2", C.c_double),
        ("sigma", C.c_double), ("gx", C.c_double), ("gy", C.c_double),
        ("cfl_target", C.c_double), ("alpha_penalty", C.c_double), ("time_order", C.c_int),
        ("tol_bicgstab2", C.c_double), ("max_iter_bicgstab2", C.c_int),
        ("pcg_tol", C.c_double), ("pcg_max_iter", C.c_int), ("pcd_sweeps", C.c_int),
        ("jacobi_omega", C.c_double), ("svof_delta_h", C.c_double), ("svof_max_iter", C.c_int),
        ("svof_tol", C.c_double), ("limiter", C.c_int), ("free_slip_x", C.c_int),
        ("krylov_bc_fix", C.c_int), ("refine", C.c_int), ("refine_inner_tol", C.c_double),
        ("refine_max_inner", C.c_int), ("refine_max_outer", C.c_int), ("precision", C.c_int),
        ("pcg_cap_start", C.c_int), ("pcd_sweeps_max", C.c_int), ("pcd_smoother", C.c_int),
        ("pcd_sor_omega", C.c_double), ("graphs", C.c_int), ("pcd_visc_scale", C.c_double),
        ("vec_rows", C.c_int),
    ]


class FuguStepOpts(C.Structure):
    _fields_ = [
        ("use_bicgstab2", C.c_int), ("has_lid", C.c_int), ("u_top_lid", C.c_double),
        ("has_tol", C.c_int), ("tol", C.c_double), ("has_max_iter", C.c_int), ("max_iter", C.c_int),
        ("consistent_amp", C.c_int), ("has_penalty", C.c_int),
        ("has_u_solid", C.c_int), ("u_solid", C.c_double), ("has_v_solid", C.c_int), ("v_solid", C.c_double),
    ]


class FuguStats(C.Structure):
    _fields_ = [
        ("iter", C.c_int), ("res", C.c_double), ("pcg_iters", C.c_longlong), ("pcg_calls", C.c_int),
        ("svof_iters", C.c_int), ("matvecs", C.c_int), ("outer", C.c_int), ("status", C.c_int),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class FuguProfile(C.Structure):
    _fields_ = [
        ("kernel_launches", C.c_ulonglong), ("pcg_ms", C.c_double), ("pcg_launches", C.c_ulonglong),
        ("pcg_iters", C.c_ulonglong), ("pcg_cells", C.c_ulonglong), ("pcg_grid", C.c_int), ("svof_grid", C.c_int),
        ("pcg_cluster_fp64", C.c_int), ("pcg_cluster_fp32", C.c_int), ("pcg_iters_timed", C.c_ulonglong),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


# name -> (restype, argtypes); every pointer is c_void_p, NULL allowed
_vp, _i, _d = C.c_void_p, C.c_int, C.c_double
SIGNATURES = {
    "fugu_params_default": (None, [_vp]),
    "fugu_version": (C.c_char_p, []),
    "fugu_create": (_i, [_vp, _i, _vp]),
    "fugu_destroy": (None, [_vp]),
    "fugu_set_params": (_i, [_vp, _vp]),
    "fugu_last_error": (C.c_char_p, [_vp]),
    "fugu_get_stream": (_i, [_vp, _vp]),
    "fugu_profile": (_i, [_vp, _i, _vp]),
    "fugu_upload": (_i, [_vp, _i, _vp]),
    "fugu_download": (_i, [_vp, _i, _vp]),
    "fugu_step": (_i, [_vp, _d, _i, _vp, _vp]),
    "fugu_advance_coupled_step": (_i, [_vp] + [_vp] * 17 + [_d, _i, _vp, _vp]),
    "fugu_compute_adaptive_dt": (_i, [_vp, _vp, _vp, _d, _vp]),
    "fugu_build_cylinder_mask": (_i, [_vp, _d, _d, _d, _vp, _vp]),
    "fugu_halo_scalar": (_i, [_vp, _vp]),
    "fugu_halo_u": (_i, [_vp, _vp]),
    "fugu_halo_v": (_i, [_vp, _vp]),
    "fugu_compute_mixture_densities": (_i, [_vp] * 5),
    "fugu_compute_mixture_viscosities": (_i, [_vp] * 5),
    "fugu_op_divergence": (_i, [_vp] * 4),
    "fugu_op_grad_pressure": (_i, [_vp] * 4),
    "fugu_op_viscous_stress": (_i, [_vp] * 8),
    "fugu_op_advection": (_i, [_vp] * 12),
    "fugu_apply_velocity_bcs": (_i, [_vp, _vp, _vp, _i, _d]),
    "fugu_matvec_coupled": (_i, [_vp] * 15 + [_d, _i] + [_vp] * 4),
    "fugu_solve_poisson_pressure": (_i, [_vp] * 5 + [_d, _i, _vp, _vp]),
    "fugu_solve_helmholtz_u": (_i, [_vp] * 7 + [_d, _i, _vp]),
    "fugu_solve_helmholtz_v": (_i, [_vp] * 7 + [_d, _i, _vp]),
    "fugu_apply_pcd_precond": (_i, [_vp] * 14 + [_d, _vp, _vp]),
    "fugu_coupled_dot": (_i, [_vp] * 8),
    "fugu_krylov_solve": (_i, [_vp, _i] + [_vp] * 14 + [_d, _d, _i, _i, _d] + [_vp] * 5),
    "fugu_vof_advection_tvd": (_i, [_vp] * 5 + [_d, _vp, _vp]),
    "fugu_svof_helmholtz_filter": (_i, [_vp] * 3 + [_d, _i, _d, _vp]),
    "fugu_compute_interface_curvature": (_i, [_vp] * 3),
    "fugu_compute_csf_force": (_i, [_vp] * 5),
    "fugu_write_checkpoint": (_i, [_vp, C.c_char_p, _i, _d]),
    "fugu_read_checkpoint": (_i, [_vp, C.c_char_p, _vp, _vp]),
    "fugu_solve_poisson_pressure_noalloc": (_i, [_vp] * 6 + [_d, _i, _vp, _vp, _vp, _i]),
    "fugu_batch_create": (_i, [_vp, _i, _i, _vp, _vp]),
    "fugu_batch_destroy": (None, [_vp]),
    "fugu_batch_last_error": (C.c_char_p, [_vp]),
    "fugu_batch_size": (_i, [_vp]),
    "fugu_batch_case": (_i, [_vp, _i, _vp]),
    "fugu_batch_run": (_i, [_vp, _i] + [_vp] * 7),
    "fugu_batch_get_stream": (_i, [_vp, _vp]),
    "fugu_batch_launches": (C.c_ulonglong, [_vp]),
    "fugu_matvec_coupled_t": (_i, [_vp] * 15 + [_d] + [_vp] * 4),
    "fugu_adjoint_solve": (_i, [_vp] * 15 + [_d, _d] + [_vp] * 5),
    "fugu_step_vjp": (_i, [_vp, _d, _i, _vp] + [_vp] * 12),
    "fugu_test_arm_barrier_timeout": (_i, [_vp, C.c_uint]),
}


class FuguBatchOpts(C.Structure):
    _fields_ = [("nthreads", C.c_int), ("max_cluster", C.c_int), ("max_coop", C.c_int), ("lockstep", C.c_int),
                ("lockstep_group", C.c_int)]

_lib = None


def lib():
    """Load the CUDA library (raises if it is missing: no CPU fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m coupled_codefort_2d_b200.build` "
                "(the FUGU-2D GPU path has no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def ptr(a):
    """Address of a host array in the reference layout (None -> NULL)."""
    if a is None:
        return None
    if not isinstance(a, np.ndarray) or a.dtype != np.float64 or not a.flags.f_contiguous:
        raise TypeError("fields must be Fortran-ordered float64 numpy arrays")
    return a.ctypes.data


class FuguError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code
