"""Physics and solver parameters (the module globals of ``src/mod_params.f90``).

The reference keeps these as mutable module variables read by every routine
(``mod_params.f90:9-50``).  Here they are one explicit value object, passed
through the C ABI as ``fugu_params`` (``include/fugu_gpu.h``).  Defaults are
the reference's module defaults; knobs the reference hard-codes at call sites
are exposed with the reference's constants as defaults.
"""
from __future__ import annotations

from dataclasses import dataclass, replace


@dataclass(frozen=True)
class Params:
    # mod_params.f90:37-43
    rho1: float = 1000.0
    rho2: float = 1.0
    mu1: float = 1.0
    mu2: float = 0.01
    sigma: float = 0.0
    gx: float = 0.0
    gy: float = -9.81
    # mod_params.f90:48-54
    cfl_target: float = 0.5
    time_order: int = 1
    # mod_params.f90:59-68
    tol_bicgstab2: float = 1.0e-6
    max_iter_bicgstab2: int = 500
    alpha_penalty: float = 1.0e12
    # call-site constants of the reference
    pcg_tol: float = 1.0e-5  # mod_subsolvers.f90:53
    pcg_max_iter: int = 150  # mod_subsolvers.f90:55
    pcd_sweeps: int = 3  # mod_pcd_precond.f90:88,101
    jacobi_omega: float = 0.8  # mod_subsolvers.f90:272,334
    svof_delta_h: float = 1.5  # mod_solver_coupled.f90:243
    svof_max_iter: int = 150  # mod_solver_coupled.f90:245
    svof_tol: float = 1.0e-7  # mod_solver_coupled.f90:245
    # extensions; 0 keeps the reference behaviour
    limiter: int = 0  # 0 van Leer (mod_vof.f90:25-33), 1 Superbee
    free_slip_x: int = 0  # 1: side walls free-slip
    krylov_bc_fix: int = 0  # 1: BiCGStab(2) applies wall BCs to r before A*r
    # FP64 defect-correction outer loop (0 = reference Krylov stopping rule;
    # 1 = inner BiCGStab(l) of the step, 2 = inner flexible GMRES)
    refine: int = 0
    refine_inner_tol: float = 1.0e-2
    refine_max_inner: int = 20
    refine_max_outer: int = 30
    # refine = 2: PCD's PCG starts at this cap and doubles it up to pcg_max_iter
    # after an outer pass whose inner solve missed refine_inner_tol (0 = off)
    pcg_cap_start: int = 0
    # refine = 2: when the PCG cap cannot grow, a missed inner tolerance doubles
    # the PCD's Jacobi sweeps up to this many (<= pcd_sweeps: off)
    pcd_sweeps_max: int = 0
    # the PCD's velocity smoother: 0 damped Jacobi (jacobi_omega, the
    # reference), 1 red-black SOR with pcd_sor_omega (in place, two colour
    # passes per sweep)
    pcd_smoother: int = 0
    pcd_sor_omega: float = 1.0
    # 1: replay each flexible-GMRES Arnoldi step from a CUDA graph (execution
    # only; the results are the same)
    graphs: int = 0
    # > 0: the PCD's Schur step adds the viscous (Cahouet-Chabard) term
    # r_p -= pcd_visc_scale * mu_cell * z_p (0 = the reference's PCD)
    pcd_visc_scale: float = 0.0
    # 1: the damped-Jacobi sweeps and the PCD's Schur, residual and cross
    # steps take 16-byte vector accesses (same results); -1 never; 0 for
    # boxes of at least 2^20 points (the sweeps of wall-bounded cases 2^21)
    vec_rows: int = 0

    def with_(self, **kw) -> "Params":
        return replace(self, **kw)


VAN_LEER = 0
SUPERBEE = 1
