/*
 * fugu_gpu.h -- C ABI of the B200 (sm_100a) FUGU-2D coupled-step hot path.
 *
 * This is the boundary a Fortran caller binds with ISO_C_BINDING (see
 * INTEGRATION.md for the interface block).  Plain pointers and sizes only.
 *
 * Host arrays follow the reference's own convention (src/main.f90:97-103):
 * column-major, nh = 2 ghost layers, passed by the address of the lower-bound
 * element (c_loc(a(lbound(a,1), lbound(a,2)))).  Extents per kind:
 *   cell   (1-nh:nx+nh, 1-nh:ny+nh)   (nx+4) x (ny+4)
 *   u-face (0-nh:nx+nh, 1-nh:ny+nh)   (nx+5) x (ny+4)
 *   v-face (1-nh:nx+nh, 0-nh:ny+nh)   (nx+4) x (ny+5)
 *   vertex (0-nh:nx+nh, 0-nh:ny+nh)   (nx+5) x (ny+5)
 *
 * Every entry point returns an int status: FUGU_OK (0); a negative value for
 * misuse or a CUDA / device error (the message is in fugu_last_error()).
 * Numerical outcomes (converged, max-iter, breakdown, NaN) are reported in
 * fugu_stats.status, never as a failure of the call, because the reference
 * routines return silently in those cases.  Nothing aborts or throws across
 * the ABI.
 *
 * Threading: a context belongs to one host thread and owns one CUDA stream on
 * one device.  Several contexts (one per GPU) may run concurrently.
 */
#ifndef FUGU_GPU_H
#define FUGU_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define FUGU_ABI_VERSION 5  /* 5: fugu_params.vec_rows */

/* return codes */
#define FUGU_OK 0
#define FUGU_EINVAL (-1)   /* bad argument (NULL, size, option)          */
#define FUGU_ECUDA (-2)    /* CUDA runtime error                          */
#define FUGU_ENOMEM (-3)   /* device allocation failed                    */
#define FUGU_EIO (-4)      /* checkpoint file error                       */
#define FUGU_ETIMEOUT (-5) /* a device-side wait gave up (see message)    */

/* numerical status in fugu_stats.status */
#define FUGU_CONVERGED 0
#define FUGU_MAXITER 1
#define FUGU_BREAKDOWN 2
#define FUGU_NAN 3

/* precision of the Krylov solve */
#define FUGU_FP64 0  /* plain form: FP64 throughout                       */
#define FUGU_MIXED 1 /* FP32 inner Krylov+PCD inside FP64 defect correction */

/* Physics, grid and solver knobs: the module globals of src/mod_params.f90:9-50
 * and src/mod_mpi.f90:10-26 as one explicit struct.  fugu_params_default()
 * fills the reference's module defaults and call-site constants. */
typedef struct {
  int nx, ny;                 /* cells (Nx_global = nx_loc at one rank)     */
  double dx, dy;              /* dx_grid, dy_grid                           */
  int periodic_x, periodic_y; /* periods(1:2)                               */
  double rho1, rho2, mu1, mu2, sigma, gx, gy;
  double cfl_target, alpha_penalty;
  int time_order;             /* 1 = BDF1, 2 = BDF2                         */
  double tol_bicgstab2;
  int max_iter_bicgstab2;
  double pcg_tol;             /* 1e-5  (mod_subsolvers.f90:53)              */
  int pcg_max_iter;           /* 150   (mod_subsolvers.f90:55)              */
  int pcd_sweeps;             /* 3     (mod_pcd_precond.f90:88,101)         */
  double jacobi_omega;        /* 0.8   (mod_subsolvers.f90:272,334)         */
  double svof_delta_h;        /* 1.5   (mod_solver_coupled.f90:243)         */
  int svof_max_iter;          /* 150   (mod_solver_coupled.f90:245)         */
  double svof_tol;            /* 1e-7  (mod_solver_coupled.f90:245)         */
  /* extensions; 0 keeps the reference behaviour */
  int limiter;                /* 0 van Leer (mod_vof.f90:25-33), 1 Superbee */
  int free_slip_x;            /* 1: side walls free-slip                    */
  int krylov_bc_fix;          /* 1: BiCGStab(2) applies wall BCs to r before
                                 A*r (mod_bicgstab2.f90:430 does not)       */
  int refine;                 /* 1: FP64 defect-correction outer loop on the
                                 true residual |B-AX|/|B| < tol, inner solve
                                 the step's BiCGStab(l); 2: the same loop
                                 around flexible GMRES(refine_max_inner <= 127)
                                 with right PCD preconditioning              */
  double refine_inner_tol;
  int refine_max_inner;
  int refine_max_outer;
  int precision;              /* FUGU_FP64 or FUGU_MIXED (needs refine >= 1) */
  int pcg_cap_start;          /* refine = 2 only; 0 keeps the cap pcg_max_iter.
                                 > 0: each defect correction starts the PCD's
                                 PCG at this many iterations and doubles it (up
                                 to pcg_max_iter) after every outer pass whose
                                 flexible GMRES missed refine_inner_tol       */
  int pcd_sweeps_max;         /* refine = 2 only; > pcd_sweeps: once the PCG
                                 cap is at pcg_max_iter (or fixed), a missed
                                 refine_inner_tol doubles the PCD's Jacobi
                                 sweeps instead, up to this many; carried
                                 from step to step like the cap              */
  int pcd_smoother;           /* velocity smoother of the PCD: 0 the
                                 reference's damped Jacobi (jacobi_omega,
                                 mod_subsolvers.f90:252-372); 1 red-black SOR
                                 with pcd_sor_omega: each sweep updates the
                                 faces with (i + j) even, then the odd ones,
                                 in place, the halo refreshed before each     */
  double pcd_sor_omega;       /* 1.0 (Gauss-Seidel); 0 < omega < 2          */
  int graphs;                 /* 1: each flexible-GMRES Arnoldi step (refine
                                 = 2) is captured once as a CUDA graph and
                                 replayed (same kernels, same results); 0:
                                 launched kernel by kernel                   */
  double pcd_visc_scale;      /* > 0: the PCD's Schur step adds the viscous
                                 (Cahouet-Chabard) part of the Schur
                                 complement, r_p -= pcd_visc_scale * mu_c *
                                 z_p with mu_c = kappa / 2 at the cell; 0 =
                                 the reference (mod_pcd_precond.f90:49-64)   */
  int vec_rows;               /* damped-Jacobi sweeps and the PCD's Schur,
                                 residual and cross steps with 16-byte
                                 vector accesses, 16 / sizeof(real) elements
                                 of a row per thread (same results): 1 on,
                                 -1 off, 0 on for boxes of >= 2^20 points
                                 (large grids, where they stream HBM; the
                                 sweeps of wall-bounded cases from 2^21)    */
} fugu_params;

/* Optional arguments of advance_coupled_step (src/mod_solver_coupled.f90:137-160):
 * a has_* flag mirrors Fortran present(). */
typedef struct {
  int use_bicgstab2;          /* 1 = bicgstab2_solve, 0 = bicgstab_solve    */
  int has_lid;  double u_top_lid;
  int has_tol;  double tol;
  int has_max_iter; int max_iter;
  int consistent_amp;
  int has_penalty;            /* phi_s_u / phi_s_v uploaded (FUGU_F_PHI_S_*) */
  int has_u_solid; double u_solid;
  int has_v_solid; double v_solid;
} fugu_step_opts;

typedef struct {
  int iter;                   /* iter_out (refine: total inner iterations) */
  double res;                 /* res_out: left-preconditioned relative
                                 residual (refine: true relative residual)  */
  long long pcg_iters;        /* inner PCG iterations summed over the step  */
  int pcg_calls;              /* Poisson solves = preconditioner applications */
  int svof_iters;
  int matvecs;
  int outer;                  /* defect-correction outer iterations        */
  int status;                 /* FUGU_CONVERGED / MAXITER / BREAKDOWN / NAN */
} fugu_stats;

/* field identifiers of a context's device-resident state */
enum {
  FUGU_F_U_VEL = 0, FUGU_F_V_VEL, FUGU_F_P_FIELD, FUGU_F_C_FIELD,
  FUGU_F_U_PREV, FUGU_F_V_PREV,
  FUGU_F_RHO_C, FUGU_F_RHO_U, FUGU_F_RHO_V,
  FUGU_F_KAPPA, FUGU_F_ZETA, FUGU_F_ETA,
  FUGU_F_KAPPA_CURV, FUGU_F_F_SIGMA_U, FUGU_F_F_SIGMA_V,
  FUGU_F_PHI_S_U, FUGU_F_PHI_S_V,
  FUGU_NUM_FIELDS
};

typedef struct fugu_ctx fugu_ctx;

/* Measurement counters (no counterpart in the reference, which has none). */
typedef struct {
  unsigned long long kernel_launches; /* kernels launched since the last reset */
  double pcg_ms;                      /* CUDA-event time of the timed PCG
                                         launches: every launch, except that a
                                         flexible-GMRES cycle replayed from CUDA
                                         graphs times the PCG of its first
                                         Arnoldi step only                     */
  unsigned long long pcg_launches;    /* timed PCG launches                    */
  unsigned long long pcg_iters;       /* PCG iterations of all launches        */
  unsigned long long pcg_cells;       /* cells per PCG iteration (nx*ny)       */
  int pcg_grid, svof_grid;            /* CTAs of the persistent kernels        */
  int pcg_cluster_fp64;               /* CTAs of the cluster-resident PCG (0 =  */
  int pcg_cluster_fp32;               /*   grid-wide kernel used instead)       */
  unsigned long long pcg_iters_timed; /* PCG iterations of the timed launches  */
} fugu_profile_stats;

/* ---------------------------------------------------------------- context */
void fugu_params_default(fugu_params* p);
const char* fugu_version(void);
/* Create a context on CUDA device `device` for the grid in *p. */
int fugu_create(const fugu_params* p, int device, fugu_ctx** out);
void fugu_destroy(fugu_ctx* ctx);
/* Replace the module globals (grid size must not change). */
int fugu_set_params(fugu_ctx* ctx, const fugu_params* p);
const char* fugu_last_error(const fugu_ctx* ctx);
/* The context's CUDA stream (cudaStream_t), so a caller can time or order
 * work against it.  No counterpart in the reference. */
int fugu_get_stream(fugu_ctx* ctx, void** stream);
/* Read the counters into *out (may be NULL); enable >= 0 then resets them and
 * switches PCG event timing on (1) or off (0); enable < 0 only reads.
 * No counterpart in the reference. */
int fugu_profile(fugu_ctx* ctx, int enable, fugu_profile_stats* out);
/* Copy one device-resident field from / to a host array (reference layout). */
int fugu_upload(fugu_ctx* ctx, int field, const double* host);
int fugu_download(fugu_ctx* ctx, int field, double* host);

/* One coupled time step on the device-resident state (u_vel ... f_sigma_v,
 * phi_s_*).  Replaces advance_coupled_step, src/mod_solver_coupled.f90:137. */
int fugu_step(fugu_ctx* ctx, double dt, int step_idx, const fugu_step_opts* o, fugu_stats* st);

/* Drop-in for advance_coupled_step (src/mod_solver_coupled.f90:137-380) with
 * the reference's host arrays: uploads the state, steps, downloads it.
 * phi_s_u / phi_s_v may be NULL (no Darcy penalty). */
int fugu_advance_coupled_step(fugu_ctx* ctx,
                              double* u_vel, double* v_vel, double* p_field, double* c_field,
                              double* u_prev, double* v_prev,
                              double* rho_c, double* rho_u, double* rho_v,
                              double* kappa, double* zeta, double* eta,
                              double* kappa_curv, double* f_sigma_u, double* f_sigma_v,
                              const double* phi_s_u, const double* phi_s_v,
                              double dt, int step_idx, const fugu_step_opts* o, fugu_stats* st);

/* compute_adaptive_dt (src/mod_solver_coupled.f90:41-91) on host arrays */
int fugu_compute_adaptive_dt(fugu_ctx* ctx, const double* u_vel, const double* v_vel,
                             double dt_max, double* dt_out);
/* build_cylinder_mask (src/mod_solver_coupled.f90:96-132) */
int fugu_build_cylinder_mask(fugu_ctx* ctx, double xc, double yc, double rad,
                             double* phi_s_u, double* phi_s_v);

/* ------------------------------------------------ routine-level entries
 * Each takes the reference routine's dummy arguments as host arrays, runs the
 * device kernels the step uses, and writes the intent(out)/(inout) arrays
 * back.  NULL marks an absent optional argument. */

/* mod_mpi.f90:113-245 (single rank: periodic self-wrap, walls untouched) */
int fugu_halo_scalar(fugu_ctx* ctx, double* phi);
int fugu_halo_u(fugu_ctx* ctx, double* u);
int fugu_halo_v(fugu_ctx* ctx, double* v);

/* mod_viscosity.f90:54-93, :105-151 */
int fugu_compute_mixture_densities(fugu_ctx* ctx, const double* c_field,
                                   double* rho_c, double* rho_u, double* rho_v);
int fugu_compute_mixture_viscosities(fugu_ctx* ctx, const double* c_field,
                                     double* kappa, double* zeta, double* eta);

/* mod_operators.f90:34-53, :60-88, :99-162, :168-249, :254-333 */
int fugu_op_divergence(fugu_ctx* ctx, const double* u, const double* v, double* div);
int fugu_op_grad_pressure(fugu_ctx* ctx, const double* p, double* grad_u, double* grad_v);
int fugu_op_viscous_stress(fugu_ctx* ctx, const double* u, const double* v,
                           const double* kappa, const double* zeta, const double* eta,
                           double* visc_u, double* visc_v);
int fugu_op_advection(fugu_ctx* ctx, const double* u_adv, const double* v_adv,
                      const double* rho_c, const double* rho_u, const double* rho_v,
                      const double* u, const double* v, double* adv_u, double* adv_v,
                      const double* mdot_u, const double* mdot_v);
int fugu_apply_velocity_bcs(fugu_ctx* ctx, double* u, double* v, int has_lid, double u_lid);

/* matvec_coupled, mod_operators.f90:341-443 (X is intent(inout): its ghosts
 * receive the periodic halo, as in the reference) */
int fugu_matvec_coupled(fugu_ctx* ctx, double* X_u, double* X_v, double* X_p,
                        double* Y_u, double* Y_v, double* Y_p,
                        const double* u_adv, const double* v_adv,
                        const double* rho_c, const double* rho_u, const double* rho_v,
                        const double* kappa, const double* zeta, const double* eta,
                        double dt, int include_advection,
                        const double* penalty_u, const double* penalty_v,
                        const double* mdot_u, const double* mdot_v);

/* mod_subsolvers.f90:32-246, :252-309, :314-372 */
int fugu_solve_poisson_pressure(fugu_ctx* ctx, double* phi, const double* rhs,
                                const double* rho_u, const double* rho_v,
                                double tol, int max_iter, int* iter_out, double* res_out);
int fugu_solve_helmholtz_u(fugu_ctx* ctx, double* u_sol, const double* rhs_u,
                           const double* rho_u, const double* kappa, const double* zeta,
                           const double* eta, double dt, int n_sweeps, const double* penalty_u);
int fugu_solve_helmholtz_v(fugu_ctx* ctx, double* v_sol, const double* rhs_v,
                           const double* rho_v, const double* kappa, const double* zeta,
                           const double* eta, double dt, int n_sweeps, const double* penalty_v);

/* apply_pcd_precond, mod_pcd_precond.f90:14-104 */
int fugu_apply_pcd_precond(fugu_ctx* ctx, const double* z_u, const double* z_v, const double* z_p,
                           double* r_u, double* r_v, double* r_p,
                           const double* u_adv, const double* v_adv,
                           const double* rho_u, const double* rho_v,
                           const double* kappa, const double* zeta, const double* eta,
                           double dt, const double* penalty_u, const double* penalty_v);

/* coupled_dot, mod_bicgstab2.f90:32-72 */
int fugu_coupled_dot(fugu_ctx* ctx, const double* u1, const double* v1, const double* p1,
                     const double* u2, const double* v2, const double* p2, double* out);

/* bicgstab_solve (mod_bicgstab2.f90:77-264) when solver = 1,
 * bicgstab2_solve (:270-570) when solver = 2.  has_lid mirrors
 * present(u_top_lid).  With params.refine = 1 the solve is the FP64
 * defect-correction loop around the chosen inner solver. */
int fugu_krylov_solve(fugu_ctx* ctx, int solver,
                      double* X_u, double* X_v, double* X_p,
                      const double* B_u, const double* B_v, const double* B_p,
                      const double* u_adv, const double* v_adv,
                      const double* rho_c, const double* rho_u, const double* rho_v,
                      const double* kappa, const double* zeta, const double* eta,
                      double dt, double tol, int max_iter, int has_lid, double u_lid,
                      const double* penalty_u, const double* penalty_v,
                      const double* mdot_u, const double* mdot_v, fugu_stats* st);

/* ------------------------------------------------ discrete adjoint
 * No counterpart in the reference.  The linear map the Krylov solvers see is
 * A: x -> (matvec_coupled(BC(x)))_owned (mod_operators.f90:341-443 after the
 * homogeneous wall BCs, :254-333), on the owned unknowns (the coupled_dot set:
 * interior u faces, v faces and cells).  Its stencil is measured on the
 * device by probing with coloured unit vectors (about 75-200 products), then
 * applied transposed by a gather kernel.  Arrays are reference-layout host
 * arrays; entries outside the owned set are ignored on input and zero on
 * output.  The coefficient arguments are matvec_coupled's (advection always
 * included, as in the solvers). */
/* X = A^T Y */
int fugu_matvec_coupled_t(fugu_ctx* ctx, const double* Y_u, const double* Y_v, const double* Y_p,
                          double* X_u, double* X_v, double* X_p,
                          const double* u_adv, const double* v_adv,
                          const double* rho_c, const double* rho_u, const double* rho_v,
                          const double* kappa, const double* zeta, const double* eta, double dt,
                          const double* penalty_u, const double* penalty_v,
                          const double* mdot_u, const double* mdot_v);
/* Solve A^T lambda = g to true relative residual tol: the FP64 defect
 * correction around flexible GMRES on S A^T S (S flips the pressure block,
 * which turns A^T back into A's block structure with the velocity block
 * transposed) with the step's PCD as right preconditioner; when the
 * context's refine is 1, around BiCGStab(2) instead (the reference's solver,
 * mod_bicgstab2.f90:270-570, on the transposed system; it inherits that
 * solver's breakdowns on hard cases).  st reports the iterations; lambda's
 * pressure block is defined up to the null space of A^T (a constant in a
 * closed or periodic box). */
int fugu_adjoint_solve(fugu_ctx* ctx, const double* g_u, const double* g_v, const double* g_p,
                       double* lambda_u, double* lambda_v, double* lambda_p,
                       const double* u_adv, const double* v_adv,
                       const double* rho_c, const double* rho_u, const double* rho_v,
                       const double* kappa, const double* zeta, const double* eta, double dt, double tol,
                       const double* penalty_u, const double* penalty_v,
                       const double* mdot_u, const double* mdot_v, fugu_stats* st);

/* Vector-Jacobian product of one whole step (no counterpart in the
 * reference).  The step is the map of the state
 *   (u_vel, v_vel, c_field, u_prev, v_prev)
 *     -> (u_vel', v_vel', c_field', u_prev' = u_vel, v_prev' = v_vel)
 * that fugu_step computes (mod_solver_coupled.f90:137-380): VOF transport,
 * properties, SVOF, curvature, CSF, AB extrapolation, right-hand side and the
 * coupled solve, taken as exact.  The context must hold the state before
 * the step; the call runs the step (the context then holds the state after
 * it, as after fugu_step) and applies the transpose of the step's Jacobian,
 * for the branches the step took, to the adjoints of the state after it:
 *   bar_*_out (adjoints of u_vel', v_vel', c_field', u_prev', v_prev';
 *              reference-layout host arrays, every entry of the kind's extent)
 *   -> bar_*_in (adjoints of the state before the step, same layout).
 * p_field is only the solve's initial guess and has no adjoint.  bar_theta
 * (may be NULL) accumulates += the derivatives with respect to
 * {sigma, mu1, mu2, rho1, rho2}.  The step's own options apply (dt,
 * step_idx, BDF order, lid, tolerance, which the adjoint solve also uses);
 * wall-bounded boxes only, without consistent_amp or the Darcy penalty
 * (FUGU_EINVAL otherwise).  st holds the forward step's statistics, with
 * status the adjoint solve's when the forward step converged and outer its
 * outer iterations. */
int fugu_step_vjp(fugu_ctx* ctx, double dt, int step_idx, const fugu_step_opts* opts,
                  const double* bar_u_out, const double* bar_v_out, const double* bar_c_out,
                  const double* bar_uprev_out, const double* bar_vprev_out,
                  double* bar_u_in, double* bar_v_in, double* bar_c_in,
                  double* bar_uprev_in, double* bar_vprev_in, double* bar_theta, fugu_stats* st);

/* mod_vof.f90:38-140 (flux_x/flux_y may be NULL), :145-194 */
int fugu_vof_advection_tvd(fugu_ctx* ctx, const double* c_in, double* c_out,
                           const double* u, const double* v, double dt,
                           double* flux_x, double* flux_y);
int fugu_svof_helmholtz_filter(fugu_ctx* ctx, const double* c_raw, double* c_smooth,
                               double delta, int max_iter, double tol, int* iters_out);

/* mod_surface_tension.f90:25-72, :78-109 */
int fugu_compute_interface_curvature(fugu_ctx* ctx, const double* c_smooth, double* kappa_curv);
int fugu_compute_csf_force(fugu_ctx* ctx, const double* c_raw, const double* kappa_curv,
                           double* f_sigma_u, double* f_sigma_v);

/* mod_io.f90:169-225: checkpoint of the device-resident state in the
 * reference's stream-binary format (header step, t, nx, ny, nh; then
 * u, v, u_prev, v_prev, p, c with halos). */
int fugu_write_checkpoint(fugu_ctx* ctx, const char* path, int step, double t);
int fugu_read_checkpoint(fugu_ctx* ctx, const char* path, int* step, double* t);

/* ------------------------------------------------ batched form
 * Many independent cases (grids, physics and precision may differ) advanced
 * together on one GPU.  No counterpart in the reference, which runs one case
 * per mpirun.  Each case is a full context (fugu_batch_case gives it, for
 * fugu_upload / fugu_download / fugu_profile); a pool of host threads steps
 * the cases, largest grid first, so the device runs as many cases' kernels
 * at once as fit.  With max_cluster = 0 the CTAs of each case's
 * cluster-resident PCG are autotuned at creation: per distinct (grid,
 * boundaries, precision) every feasible size in {2, 4, 8, 16} is timed on
 * the device and the least CTAs x time per iteration wins. */
typedef struct fugu_batch fugu_batch;
typedef struct {
  int nthreads;     /* host threads stepping cases (0: hardware threads, <= ncases) */
  int max_cluster;  /* CTAs of each cluster-resident PCG, 1..16 (0: autotune)     */
  int max_coop;     /* CTAs of each grid-wide persistent kernel, launched as one  */
                    /* thread-block cluster so that it is scheduled whole (<= 8; 0: 8) */
  int lockstep;     /* 1: the coupled solves of all cases advance in lockstep,
                       one launch per kernel family serving every case still
                       running (work lists of (case, tile) items on the device,
                       per-case Krylov scalars and activity flags, each
                       flexible-GMRES cycle one CUDA graph whose Arnoldi steps
                       are conditional nodes armed on the device); needs every
                       case at refine = 2 with one precision, pcd_smoother and
                       refine_max_inner, and a PCG that fits a cluster; at most
                       1024 cases.  Within one fugu_batch_run of several
                       steps a case whose solve has ended takes its next
                       step while the others keep solving (continuous
                       batching).  Each case's results equal those of the
                       thread-pool form (0) bit for bit.                      */
  int lockstep_group; /* lockstep: the cases are grouped by their PCG's cluster
                       plan, at most this many per group (0: no limit); each
                       group runs in lockstep on its own stream and host
                       thread, and the groups do not wait for one another   */
} fugu_batch_opts;
int fugu_batch_create(const fugu_params* params, int ncases, int device, const fugu_batch_opts* opts,
                      fugu_batch** out);
void fugu_batch_destroy(fugu_batch* b);
const char* fugu_batch_last_error(const fugu_batch* b);
int fugu_batch_size(const fugu_batch* b);
int fugu_batch_case(fugu_batch* b, int i, fugu_ctx** ctx);
/* Advance case i by nsteps steps with dt[i], step indices step0[i] ..
 * step0[i]+nsteps-1 and options opts[i].  Per case (each output may be
 * NULL): last[i] = stats of its last step, max_res[i] = largest final
 * residual over its steps, status[i] = FUGU_OK or the error of the step
 * that stopped it, total[i] = its steps' stats summed (iter, outer,
 * pcg_iters, pcg_calls, matvecs, svof_iters; res the largest, status the
 * first that is not FUGU_CONVERGED).  Returns FUGU_OK, or the first failing
 * case's code. */
int fugu_batch_run(fugu_batch* b, int nsteps, const double* dt, const int* step0, const fugu_step_opts* opts,
                   fugu_stats* last, double* max_res, int* status, fugu_stats* total);
/* The batch stream (cudaStream_t): all device work of a fugu_batch_run
 * starts after the work queued on it before the call and ends before the
 * work queued on it after the call, so CUDA events recorded on it around a
 * run time the run on the device.  No counterpart in the reference. */
int fugu_batch_get_stream(fugu_batch* b, void** stream);
/* Kernel launches the batch has issued so far, replays of CUDA graphs
 * included (a measurement counter; no counterpart in the reference). */
unsigned long long fugu_batch_launches(const fugu_batch* b);

/* ------------------------------------------------ allocation-free entry
 * solve_poisson_pressure (mod_subsolvers.f90:32-246) with no context and no
 * allocation.  No counterpart in the reference, whose subroutine works on
 * arrays its caller already owns.  It serves callers that cannot call
 * cudaMalloc:
 *   - a host code whose own pool allocator already holds the device memory,
 *     where a cudaMalloc would fail or fragment that pool;
 *   - a time loop that cannot take the device-wide synchronisation that
 *     cudaFree implies.
 * Its working memory is one static device array of about 7.1 MB, present
 * on each device once the library's device code is loaded there.  The call
 * makes no cudaMalloc, cudaFree, cudaMallocHost or other allocating call.
 *
 * phi (in: initial guess; out: solution, ghosts as the reference), rhs,
 * rho_u and rho_v are reference-layout arrays (see the top of this file) in
 * host or device memory.  stream is a cudaStream_t (NULL: the default
 * stream).  The call returns once the stream has finished the solve.
 * iter_out and res_out are those of the reference routine (may be NULL).
 * A message goes to err (err_len bytes, may be NULL) when the call fails.
 *
 * Limit: round_up(nx+5, 16) * (ny+5) <= FUGU_NOALLOC_MAX_POINTS padded
 * points per field, which every grid up to 256 x 256 cells meets.  Larger
 * grids are rejected with FUGU_EINVAL.
 * Set-up: the first call on a device, with that device current, takes the
 * static array's device address (cudaGetSymbolAddress) and queries the
 * device; a later call redoes this when the device's current CUDA context
 * is no longer the one the address was taken in (after cudaDeviceReset).
 * Blocking: every call waits on `stream` (cudaStreamSynchronize) to read the
 * solve's result, so no call can be made while `stream` is being captured
 * into a CUDA graph.
 * A grid-barrier wait that gives up (see fugu_test_arm_barrier_timeout)
 * returns FUGU_ETIMEOUT with a message; phi then holds a partial result.
 * Zero state: the grid-barrier counters, the result record and the fields
 * must start at zero.  Every call clears them on `stream` before its
 * kernels run.
 * Concurrency: all calls on one device share the one static array.  Two
 * calls in flight at the same time on one device (from two host threads)
 * race, and both results are undefined.  Calls on different devices are
 * independent. */
#define FUGU_NOALLOC_MAX_POINTS 73728
int fugu_solve_poisson_pressure_noalloc(const fugu_params* p, void* stream, double* phi,
                                        const double* rhs, const double* rho_u, const double* rho_v,
                                        double tol, int max_iter, int* iter_out, double* res_out,
                                        char* err, int err_len);

/* ------------------------------------------------ failure-detection test hook
 * No counterpart in the reference, which has no device-side waits.  Arms the
 * next launch of the grid-wide persistent PCG kernel -- in ctx, or, with ctx
 * NULL, in the next fugu_solve_poisson_pressure_noalloc call of the process
 * -- so that each of its grid barriers waits for one CTA more than the launch
 * has and gives up after spin_limit polls (>= 1; about 40 ns each).  The
 * kernel then ends early, and the entry that made the launch returns
 * FUGU_ETIMEOUT with a message; the context stays usable.  In ctx, the armed
 * launch takes the grid-wide kernel even where the cluster-resident one
 * would run, and a launch inside a CUDA-graph capture is never armed.
 * One-shot: later launches run normally. */
int fugu_test_arm_barrier_timeout(fugu_ctx* ctx, unsigned int spin_limit);

#ifdef __cplusplus
}
#endif
#endif /* FUGU_GPU_H */
