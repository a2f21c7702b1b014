/*
 * fugu_oracle.h -- CPU restatement of the FUGU-2D coupled-step hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the CUDA
 * product in coupled_codefort_2d_b200/.  Only tests/, __graft_entry__.smoke()
 * and the cpu_baseline / reference legs of bench.py may load it.  Nothing in
 * the product links, calls or falls back to it.
 *
 * What it restates: the Fortran 2008 modules of EL-I-Thiam/COUPLED_CODEFORT_2D
 * (mod_viscosity, mod_operators, mod_subsolvers, mod_pcd_precond,
 * mod_bicgstab2, mod_vof, mod_surface_tension, mod_solver_coupled) with the
 * single-rank semantics of mod_mpi (coords=(0,0), dims=(1,1); a periodic
 * direction wraps onto itself, a wall direction leaves ghosts untouched, as
 * MPI_PROC_NULL does).  Each function cites the reference file:line it
 * follows.  Loop order and summation order follow the reference.
 *
 * Pinning: the reference ships no golden vectors (its Fortran/MPI toolchain
 * is absent here, so it cannot be run).  The oracle is pinned against every
 * analytic acceptance criterion of the reference's own tests
 * (tests/test_*.f90) -- see tests/test_oracle_reference_criteria.py.  Parity
 * at the bit / 1e-8 level against the Fortran binary itself is unpinned.
 *
 * Array convention (identical to the Fortran callers, nh = 2): every field is
 * a column-major array passed by the address of its lower-bound element.
 *   cell   (1-nh:nx+nh, 1-nh:ny+nh)  leading dim nx+4
 *   u-face (0-nh:nx+nh, 1-nh:ny+nh)  leading dim nx+5
 *   v-face (1-nh:nx+nh, 0-nh:ny+nh)  leading dim nx+4
 *   vertex (0-nh:nx+nh, 0-nh:ny+nh)  leading dim nx+5
 */
#ifndef FUGU_ORACLE_H
#define FUGU_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Module globals of mod_params.f90:9-50 and the grid of mod_mpi.f90:10-26,
 * gathered in one struct; knobs the reference hard-codes at call sites are
 * exposed with the reference values as defaults (fo_model_defaults). */
typedef struct {
  int nx, ny;               /* Nx_global, Ny_global (= nx_loc, ny_loc)   */
  double dx, dy;            /* dx_grid, dy_grid                          */
  int periodic_x, periodic_y;
  double rho1, rho2, mu1, mu2, sigma, gx, gy;
  double cfl_target, alpha_penalty;
  int time_order;
  double tol_bicgstab2;
  int max_iter_bicgstab2;
  /* call-site constants of the reference, exposed */
  double pcg_tol;           /* 1e-5  mod_subsolvers.f90:53   */
  int pcg_max_iter;         /* 150   mod_subsolvers.f90:55   */
  int pcd_sweeps;           /* 3     mod_pcd_precond.f90:88,101 */
  double jacobi_omega;      /* 0.8   mod_subsolvers.f90:272,334 */
  double svof_delta_h;      /* 1.5   mod_solver_coupled.f90:243 */
  int svof_max_iter;        /* 150   mod_solver_coupled.f90:245 */
  double svof_tol;          /* 1e-7  mod_solver_coupled.f90:245 */
  /* extensions (flag-gated; 0 = reference behaviour) */
  int limiter;              /* 0 van Leer (mod_vof.f90:25-33), 1 Superbee */
  int free_slip_x;          /* 1: side walls free-slip (tangential v symmetric) */
  int krylov_bc_fix;        /* 1: BiCGStab(2) applies the wall BCs to r before
                               A*r (the reference does not, mod_bicgstab2.f90:430) */
  /* FP64 defect-correction outer loop (extension; refine = 0 is the reference):
   * X += inner_solve(B - A X) until |B - A X| / |B| < tol (coupled_dot norm);
   * the inner solve is the step's BiCGStab(l) when refine = 1, flexible GMRES
   * (right PCD preconditioning) when refine = 2 */
  int refine;
  double refine_inner_tol;
  int refine_max_inner;
  int refine_max_outer;
  /* refine = 2: the PCD's PCG starts each defect correction capped at
   * pcg_cap_start iterations and doubles the cap (up to pcg_max_iter) after
   * each outer pass whose flexible GMRES missed refine_inner_tol; 0 = off */
  int pcg_cap_start;
  /* refine = 2: once the cap cannot grow, a missed inner tolerance doubles
   * the PCD's Jacobi sweeps up to pcd_sweeps_max (<= pcd_sweeps: off) */
  int pcd_sweeps_max;
  /* velocity smoother of the PCD (extension): 0 damped Jacobi with
   * jacobi_omega (mod_subsolvers.f90:252-372), 1 red-black SOR with
   * pcd_sor_omega: each sweep updates the faces with (i + j) even, then
   * those with (i + j) odd, in place, refreshing the halo before each colour */
  int pcd_smoother;
  double pcd_sor_omega;
  /* Schur-complement step of the PCD (extension): > 0 adds the viscous
   * (Cahouet-Chabard) term, r_p -= pcd_visc_scale * mu_c * z_p with
   * mu_c = kappa / 2 the cell viscosity; 0 = the reference */
  double pcd_visc_scale;
} fo_model;

void fo_model_defaults(fo_model* m);
/* print the Krylov residual history to stderr (debugging aid) */
void fo_set_verbose(int v);

/* optional arguments of advance_coupled_step (mod_solver_coupled.f90:137-160) */
typedef struct {
  int use_bicgstab2;        /* present(use_bicgstab2) ? value : .true.      */
  int has_lid;              /* present(u_top_lid)                          */
  double u_top_lid;
  int has_tol;  double tol;
  int has_max_iter; int max_iter;
  int consistent_amp;
  const double* phi_s_u;    /* both non-NULL <=> Darcy penalty present     */
  const double* phi_s_v;
  int has_u_solid; double u_solid;
  int has_v_solid; double v_solid;
} fo_step_opts;

typedef struct {
  int iter;                 /* iter_out of the Krylov solve                */
  double res;               /* res_out (left-preconditioned rel. residual) */
  long pcg_iters;           /* total inner PCG iterations in the step      */
  int pcg_calls;            /* Poisson solves (= preconditioner applications) */
  int svof_iters;
  int matvecs;
  int outer;                /* defect-correction outer iterations (refine) */
  int pcg_cap;              /* in/out, adaptive PCG cap (refine = 2,
                               pcg_cap_start > 0): the cap a solve starts
                               from (0: pcg_cap_start) and ends with; the
                               caller carries it from step to step         */
  int pcd_sweeps;           /* in/out, adaptive PCD sweeps, as pcg_cap     */
} fo_stats;

/* --- mod_mpi single-rank halo semantics (mod_mpi.f90:113-245) ---------- */
void fo_halo_scalar(const fo_model* m, double* phi);
void fo_halo_u(const fo_model* m, double* u);
void fo_halo_v(const fo_model* m, double* v);

/* --- mod_viscosity (mod_viscosity.f90:28-151) --------------------------- */
double fo_harmonic_viscosity(const fo_model* m, double c);
void fo_compute_mixture_densities(const fo_model* m, const double* c,
                                  double* rho_c, double* rho_u, double* rho_v);
void fo_compute_mixture_viscosities(const fo_model* m, const double* c,
                                    double* kappa, double* zeta, double* eta);

/* --- mod_operators (mod_operators.f90:34-443) --------------------------- */
void fo_op_divergence(const fo_model* m, const double* u, const double* v, double* div);
void fo_op_grad_pressure(const fo_model* m, const double* p, double* gu, double* gv);
void fo_op_viscous_stress(const fo_model* m, const double* u, const double* v,
                          const double* kappa, const double* zeta, const double* eta,
                          double* visc_u, double* visc_v);
void fo_op_advection(const fo_model* m, const double* u_adv, const double* v_adv,
                     const double* rho_c, const double* rho_u, const double* rho_v,
                     const double* u, const double* v, double* adv_u, double* adv_v,
                     const double* mdot_u, const double* mdot_v);
void fo_apply_velocity_bcs(const fo_model* m, double* u, double* v,
                           int has_lid, double u_lid);
void fo_matvec_coupled(const fo_model* m, double* Xu, double* Xv, double* Xp,
                       double* Yu, double* Yv, double* Yp,
                       const double* u_adv, const double* v_adv,
                       const double* rho_c, const double* rho_u, const double* rho_v,
                       const double* kappa, const double* zeta, const double* eta,
                       double dt, int include_adv,
                       const double* pen_u, const double* pen_v,
                       const double* mdot_u, const double* mdot_v);

/* --- mod_subsolvers (mod_subsolvers.f90:32-416) ------------------------- */
void fo_solve_poisson_pressure(const fo_model* m, double* phi, const double* rhs,
                               const double* rho_u, const double* rho_v,
                               double tol, int max_iter, int* iter_out, double* res_out);
void fo_solve_helmholtz_u(const fo_model* m, double* u_sol, const double* rhs_u,
                          const double* rho_u, const double* kappa, const double* zeta,
                          const double* eta, double dt, int n_sweeps, const double* pen_u);
void fo_solve_helmholtz_v(const fo_model* m, double* v_sol, const double* rhs_v,
                          const double* rho_v, const double* kappa, const double* zeta,
                          const double* eta, double dt, int n_sweeps, const double* pen_v);

/* --- mod_pcd_precond (mod_pcd_precond.f90:14-104) ----------------------- */
void fo_apply_pcd_precond(const fo_model* m, const double* z_u, const double* z_v,
                          const double* z_p, double* r_u, double* r_v, double* r_p,
                          const double* u_adv, const double* v_adv,
                          const double* rho_u, const double* rho_v,
                          const double* kappa, const double* zeta, const double* eta,
                          double dt, const double* pen_u, const double* pen_v,
                          fo_stats* st);

/* --- mod_bicgstab2 (mod_bicgstab2.f90:32-570) --------------------------- */
double fo_coupled_dot(const fo_model* m, const double* u1, const double* v1, const double* p1,
                      const double* u2, const double* v2, const double* p2);
/* solver = 1: bicgstab_solve (:77-264), 2: bicgstab2_solve (:270-570) */
void fo_krylov_solve(const fo_model* m, int solver,
                     double* Xu, double* Xv, double* Xp,
                     const double* Bu, const double* Bv, const double* Bp,
                     const double* u_adv, const double* v_adv,
                     const double* rho_c, const double* rho_u, const double* rho_v,
                     const double* kappa, const double* zeta, const double* eta,
                     double dt, double tol, int max_iter,
                     int has_lid, double u_lid,
                     const double* pen_u, const double* pen_v,
                     const double* mdot_u, const double* mdot_v,
                     int* iter_out, double* res_out, fo_stats* st);

/* --- mod_vof (mod_vof.f90:25-237) --------------------------------------- */
void fo_vof_advection_tvd(const fo_model* m, const double* c_in, double* c_out,
                          const double* u, const double* v, double dt,
                          double* flux_x, double* flux_y);
int fo_svof_helmholtz_filter(const fo_model* m, const double* c_raw, double* c_smooth,
                             double delta, int max_iter, double tol);

/* --- mod_surface_tension (mod_surface_tension.f90:25-109) --------------- */
void fo_compute_interface_curvature(const fo_model* m, const double* c_s, double* kcurv);
void fo_compute_csf_force(const fo_model* m, const double* c_raw, const double* kcurv,
                          double* fsu, double* fsv);

/* --- mod_solver_coupled (mod_solver_coupled.f90:41-380) ----------------- */
double fo_compute_adaptive_dt(const fo_model* m, const double* u, const double* v, double dt_max);
void fo_build_cylinder_mask(const fo_model* m, double xc, double yc, double rad,
                            double* phi_u, double* phi_v);
void fo_advance_coupled_step(const fo_model* m,
                             double* u_vel, double* v_vel, double* p_field, double* c_field,
                             double* u_prev, double* v_prev,
                             double* rho_c, double* rho_u, double* rho_v,
                             double* kappa, double* zeta, double* eta,
                             double* kappa_curv, double* f_sigma_u, double* f_sigma_v,
                             double dt, int step_idx, const fo_step_opts* o, fo_stats* st);

/* --- mod_io checkpoint byte format (mod_io.f90:169-225) ------------------ */
int fo_write_checkpoint(const fo_model* m, const char* path, int step, double t,
                        const double* u, const double* v, const double* u_prev,
                        const double* v_prev, const double* p, const double* c);
int fo_read_checkpoint(const fo_model* m, const char* path, int* step, double* t,
                       double* u, double* v, double* u_prev, double* v_prev,
                       double* p, double* c);

#ifdef __cplusplus
}
#endif
#endif
