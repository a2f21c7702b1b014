/*
 * fugu_oracle.c -- CPU restatement of the FUGU-2D coupled-step hot path.
 * TEST INFRASTRUCTURE ONLY (the checker, never the product); see fugu_oracle.h.
 *
 * Build: oracle/Makefile (gcc -O3 -ffp-contract=off, no -march=native, so
 * every a*b+c rounds twice, as the reference does on x86-64 gfortran).
 */
#include "fugu_oracle.h"

static int g_verbose = 0;
void fo_set_verbose(int v) { g_verbose = v; }

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------------- */
/* layout helpers                                                          */
/* ---------------------------------------------------------------------- */
#define NH 2
#define LDC(m) ((m)->nx + 4)
#define LDU(m) ((m)->nx + 5)
#define LDV(m) ((m)->nx + 4)
#define LDW(m) ((m)->nx + 5)
/* element (i,j) of a cell / u / v / vertex array (Fortran lower bounds) */
#define AC(a, i, j) (a)[(size_t)((i) + 1) + (size_t)((j) + 1) * LDC(m)]
#define AU(a, i, j) (a)[(size_t)((i) + 2) + (size_t)((j) + 1) * LDU(m)]
#define AV(a, i, j) (a)[(size_t)((i) + 1) + (size_t)((j) + 2) * LDV(m)]
#define AW(a, i, j) (a)[(size_t)((i) + 2) + (size_t)((j) + 2) * LDW(m)]

static size_t n_cell(const fo_model* m) { return (size_t)(m->nx + 4) * (m->ny + 4); }
static size_t n_u(const fo_model* m) { return (size_t)(m->nx + 5) * (m->ny + 4); }
static size_t n_v(const fo_model* m) { return (size_t)(m->nx + 4) * (m->ny + 5); }

static double* zalloc(size_t n) {
  double* p = (double*)calloc(n, sizeof(double));
  if (!p) { fprintf(stderr, "fugu_oracle: out of memory\n"); abort(); }
  return p;
}
/* Nearly order-independent sums: the reference accumulates each reduction
 * serially per MPI rank and then MPI_Allreduce-s the rank partials, so its
 * rounding depends on the rank count.  The oracle (and the CUDA path)
 * accumulate the same terms as an unevaluated pair hi + lo -- Knuth's TwoSum
 * on hi, the error terms added into lo with ordinary rounding -- and round
 * once.  When the terms' exponents span less than ~50 bits every lo addition
 * is exact and the result is the correctly rounded sum in any order; over a
 * wider span lo keeps an error near n * eps^2 * |partial sums|, and a sum that
 * cancels can then round its last bit differently from the CUDA path's tree
 * of short pairs. */
typedef struct { double hi, lo; } dsum;
static void ds_add(dsum* d, double x) {
  double s = d->hi + x;
  double bp = s - d->hi;
  double e = (d->hi - (s - bp)) + (x - bp);
  d->hi = s;
  d->lo = d->lo + e;
}
static double ds_val(dsum d) { return d.hi + d.lo; }

static double dmin(double a, double b) { return a < b ? a : b; }
static double dmax(double a, double b) { return a > b ? a : b; }
static double clip01(double x) { return dmax(0.0, dmin(1.0, x)); }

/* last (i) index of owned u / v unknowns: the east/north wall face is not an
 * unknown when the direction is a wall (mod_operators.f90:192-196) */
static int iu_max(const fo_model* m) { return m->periodic_x ? m->nx : m->nx - 1; }
static int jv_max(const fo_model* m) { return m->periodic_y ? m->ny : m->ny - 1; }

void fo_model_defaults(fo_model* m) {
  memset(m, 0, sizeof(*m));
  m->nx = 64; m->ny = 64; m->dx = 1.0 / 64; m->dy = 1.0 / 64;
  m->rho1 = 1000.0; m->rho2 = 1.0; m->mu1 = 1.0; m->mu2 = 0.01;
  m->sigma = 0.0; m->gx = 0.0; m->gy = -9.81;
  m->cfl_target = 0.5; m->alpha_penalty = 1.0e12;
  m->time_order = 1; m->tol_bicgstab2 = 1.0e-6; m->max_iter_bicgstab2 = 500;
  m->pcg_tol = 1.0e-5; m->pcg_max_iter = 150; m->pcd_sweeps = 3;
  m->jacobi_omega = 0.8; m->svof_delta_h = 1.5; m->svof_max_iter = 150;
  m->svof_tol = 1.0e-7; m->limiter = 0; m->free_slip_x = 0;
  m->pcd_smoother = 0; m->pcd_sor_omega = 1.0; m->pcd_visc_scale = 0.0;
}

/* ---------------------------------------------------------------------- */
/* mod_mpi.f90:113-245 at one rank: a periodic direction receives its own  */
/* opposite interior columns/rows (x pass first, over the full j range,    */
/* then y pass over the full i range, so corners come from the y pass);    */
/* a wall direction is a no-op (MPI_PROC_NULL).                            */
/* ---------------------------------------------------------------------- */
void fo_halo_scalar(const fo_model* m, double* phi) {
  const int nx = m->nx, ny = m->ny;
  if (m->periodic_x) {
    for (int j = 1 - NH; j <= ny + NH; ++j)
      for (int k = 0; k < NH; ++k) AC(phi, 1 - NH + k, j) = AC(phi, nx - NH + 1 + k, j);
    for (int j = 1 - NH; j <= ny + NH; ++j)
      for (int k = 0; k < NH; ++k) AC(phi, nx + 1 + k, j) = AC(phi, 1 + k, j);
  }
  if (m->periodic_y) {
    for (int k = 0; k < NH; ++k)
      for (int i = 1 - NH; i <= nx + NH; ++i) AC(phi, i, 1 - NH + k) = AC(phi, i, ny - NH + 1 + k);
    for (int k = 0; k < NH; ++k)
      for (int i = 1 - NH; i <= nx + NH; ++i) AC(phi, i, ny + 1 + k) = AC(phi, i, 1 + k);
  }
}

void fo_halo_u(const fo_model* m, double* u) {
  const int nx = m->nx, ny = m->ny;
  if (m->periodic_x) {
    for (int j = 1 - NH; j <= ny + NH; ++j)
      for (int k = 0; k < NH; ++k) AU(u, 1 - NH + k, j) = AU(u, nx - NH + 1 + k, j);
    for (int j = 1 - NH; j <= ny + NH; ++j)
      for (int k = 0; k < NH; ++k) AU(u, nx + 1 + k, j) = AU(u, 1 + k, j);
  }
  if (m->periodic_y) {
    for (int k = 0; k < NH; ++k)
      for (int i = 0 - NH; i <= nx + NH; ++i) AU(u, i, 1 - NH + k) = AU(u, i, ny - NH + 1 + k);
    for (int k = 0; k < NH; ++k)
      for (int i = 0 - NH; i <= nx + NH; ++i) AU(u, i, ny + 1 + k) = AU(u, i, 1 + k);
  }
}

void fo_halo_v(const fo_model* m, double* v) {
  const int nx = m->nx, ny = m->ny;
  if (m->periodic_x) {
    for (int j = 0 - NH; j <= ny + NH; ++j)
      for (int k = 0; k < NH; ++k) AV(v, 1 - NH + k, j) = AV(v, nx - NH + 1 + k, j);
    for (int j = 0 - NH; j <= ny + NH; ++j)
      for (int k = 0; k < NH; ++k) AV(v, nx + 1 + k, j) = AV(v, 1 + k, j);
  }
  if (m->periodic_y) {
    for (int k = 0; k < NH; ++k)
      for (int i = 1 - NH; i <= nx + NH; ++i) AV(v, i, 1 - NH + k) = AV(v, i, ny - NH + 1 + k);
    for (int k = 0; k < NH; ++k)
      for (int i = 1 - NH; i <= nx + NH; ++i) AV(v, i, ny + 1 + k) = AV(v, i, 1 + k);
  }
}

/* ---------------------------------------------------------------------- */
/* mod_viscosity.f90                                                       */
/* ---------------------------------------------------------------------- */
/* harmonic_viscosity, mod_viscosity.f90:28-46 */
double fo_harmonic_viscosity(const fo_model* m, double c) {
  double cc = clip01(c);
  if (fabs(m->mu1 - m->mu2) < 1.0e-14) return m->mu1;
  double denom = m->mu2 * cc + m->mu1 * (1.0 - cc);
  if (denom > 1.0e-15) return (m->mu1 * m->mu2) / denom;
  return dmin(m->mu1, m->mu2);
}

/* compute_mixture_densities, mod_viscosity.f90:54-93 */
void fo_compute_mixture_densities(const fo_model* m, const double* c,
                                  double* rho_c, double* rho_u, double* rho_v) {
  const int nx = m->nx, ny = m->ny;
  for (int j = 1 - NH; j <= ny + NH; ++j)
    for (int i = 1 - NH; i <= nx + NH; ++i) {
      double cv = clip01(AC(c, i, j));
      AC(rho_c, i, j) = m->rho1 * cv + m->rho2 * (1.0 - cv);
    }
  for (int j = 1 - NH; j <= ny + NH; ++j) {
    for (int i = 1 - NH; i <= nx + NH - 1; ++i)
      AU(rho_u, i, j) = 0.5 * (AC(rho_c, i, j) + AC(rho_c, i + 1, j));
    AU(rho_u, 0 - NH, j) = AU(rho_u, 1 - NH, j);
    AU(rho_u, nx + NH, j) = AU(rho_u, nx + NH - 1, j);
  }
  for (int i = 1 - NH; i <= nx + NH; ++i) {
    for (int j = 1 - NH; j <= ny + NH - 1; ++j)
      AV(rho_v, i, j) = 0.5 * (AC(rho_c, i, j) + AC(rho_c, i, j + 1));
    AV(rho_v, i, 0 - NH) = AV(rho_v, i, 1 - NH);
    AV(rho_v, i, ny + NH) = AV(rho_v, i, ny + NH - 1);
  }
}

/* compute_mixture_viscosities, mod_viscosity.f90:105-151 */
void fo_compute_mixture_viscosities(const fo_model* m, const double* c,
                                    double* kappa, double* zeta, double* eta) {
  const int nx = m->nx, ny = m->ny;
  for (int j = 1 - NH; j <= ny + NH; ++j)
    for (int i = 1 - NH; i <= nx + NH; ++i)
      AC(kappa, i, j) = 2.0 * fo_harmonic_viscosity(m, AC(c, i, j));
  for (int j = 1 - NH; j <= ny + NH - 1; ++j)
    for (int i = 1 - NH; i <= nx + NH - 1; ++i) {
      double cv = 0.25 * (AC(c, i, j) + AC(c, i + 1, j) + AC(c, i, j + 1) + AC(c, i + 1, j + 1));
      double mu = fo_harmonic_viscosity(m, cv);
      AW(zeta, i, j) = 2.0 * mu;
      AW(eta, i, j) = mu;
    }
  for (int j = 1 - NH; j <= ny + NH - 1; ++j) {
    AW(zeta, 0 - NH, j) = AW(zeta, 1 - NH, j);
    AW(zeta, nx + NH, j) = AW(zeta, nx + NH - 1, j);
    AW(eta, 0 - NH, j) = AW(eta, 1 - NH, j);
    AW(eta, nx + NH, j) = AW(eta, nx + NH - 1, j);
  }
  for (int i = 0 - NH; i <= nx + NH; ++i) {
    AW(zeta, i, 0 - NH) = AW(zeta, i, 1 - NH);
    AW(zeta, i, ny + NH) = AW(zeta, i, ny + NH - 1);
    AW(eta, i, 0 - NH) = AW(eta, i, 1 - NH);
    AW(eta, i, ny + NH) = AW(eta, i, ny + NH - 1);
  }
}

/* ---------------------------------------------------------------------- */
/* mod_operators.f90                                                       */
/* ---------------------------------------------------------------------- */
/* op_divergence, mod_operators.f90:34-53 (whole output zeroed first) */
void fo_op_divergence(const fo_model* m, const double* u, const double* v, double* div) {
  const int nx = m->nx, ny = m->ny;
  const double idx = 1.0 / m->dx, idy = 1.0 / m->dy;
  memset(div, 0, n_cell(m) * sizeof(double));
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i)
      AC(div, i, j) = (AU(u, i, j) - AU(u, i - 1, j)) * idx + (AV(v, i, j) - AV(v, i, j - 1)) * idy;
}

/* op_grad_pressure, mod_operators.f90:60-88 */
void fo_op_grad_pressure(const fo_model* m, const double* p, double* gu, double* gv) {
  const int nx = m->nx, ny = m->ny;
  const double idx = 1.0 / m->dx, idy = 1.0 / m->dy;
  memset(gu, 0, n_u(m) * sizeof(double));
  memset(gv, 0, n_v(m) * sizeof(double));
  for (int j = 1; j <= ny; ++j)
    for (int i = 0; i <= nx; ++i) AU(gu, i, j) = (AC(p, i + 1, j) - AC(p, i, j)) * idx;
  for (int j = 0; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i) AV(gv, i, j) = (AC(p, i, j + 1) - AC(p, i, j)) * idy;
}

/* op_viscous_stress, mod_operators.f90:99-162.  The vertex stresses use
 * (zeta - eta) exactly as written. */
void fo_op_viscous_stress(const fo_model* m, const double* u, const double* v,
                          const double* kappa, const double* zeta, const double* eta,
                          double* visc_u, double* visc_v) {
  const int nx = m->nx, ny = m->ny;
  const double idx = 1.0 / m->dx, idy = 1.0 / m->dy;
  /* local work arrays: T_xx(0:nx+1,1:ny), T_yy(1:nx,0:ny+1), T_xy/T_yx(0:nx,0:ny) */
  const int lxx = nx + 2, lyy = nx, lxy = nx + 1;
  double* txx = zalloc((size_t)lxx * ny);
  double* tyy = zalloc((size_t)lyy * (ny + 2));
  double* txy = zalloc((size_t)lxy * (ny + 1));
  double* tyx = zalloc((size_t)lxy * (ny + 1));
#define TXX(i, j) txx[(size_t)(i) + (size_t)((j)-1) * lxx]
#define TYY(i, j) tyy[(size_t)((i)-1) + (size_t)(j) * lyy]
#define TXY(i, j) txy[(size_t)(i) + (size_t)(j) * lxy]
#define TYX(i, j) tyx[(size_t)(i) + (size_t)(j) * lxy]
  for (int j = 1; j <= ny; ++j)
    for (int i = 0; i <= nx + 1; ++i)
      TXX(i, j) = AC(kappa, i, j) * (AU(u, i, j) - AU(u, i - 1, j)) * idx;
  for (int j = 0; j <= ny + 1; ++j)
    for (int i = 1; i <= nx; ++i)
      TYY(i, j) = AC(kappa, i, j) * (AV(v, i, j) - AV(v, i, j - 1)) * idy;
  for (int j = 0; j <= ny; ++j)
    for (int i = 0; i <= nx; ++i) {
      double du_dy = (AU(u, i, j + 1) - AU(u, i, j)) * idy;
      double dv_dx = (AV(v, i + 1, j) - AV(v, i, j)) * idx;
      TXY(i, j) = (AW(zeta, i, j) - AW(eta, i, j)) * du_dy + AW(eta, i, j) * dv_dx;
      TYX(i, j) = AW(eta, i, j) * du_dy + (AW(zeta, i, j) - AW(eta, i, j)) * dv_dx;
    }
  memset(visc_u, 0, n_u(m) * sizeof(double));
  for (int j = 1; j <= ny; ++j)
    for (int i = 0; i <= nx; ++i)
      AU(visc_u, i, j) = -((TXX(i + 1, j) - TXX(i, j)) * idx + (TXY(i, j) - TXY(i, j - 1)) * idy);
  memset(visc_v, 0, n_v(m) * sizeof(double));
  for (int j = 0; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i)
      AV(visc_v, i, j) = -((TYX(i, j) - TYX(i - 1, j)) * idx + (TYY(i, j + 1) - TYY(i, j)) * idy);
#undef TXX
#undef TYY
#undef TXY
#undef TYX
  free(txx); free(tyy); free(txy); free(tyx);
}

/* op_advection, mod_operators.f90:168-249 (centred, linearised about the
 * advecting field; AMP mass fluxes replace rho*u_adv when both are given) */
void fo_op_advection(const fo_model* m, const double* u_adv, const double* v_adv,
                     const double* rho_c, const double* rho_u, const double* rho_v,
                     const double* u, const double* v, double* adv_u, double* adv_v,
                     const double* mdot_u, const double* mdot_v) {
  const int nx = m->nx, ny = m->ny;
  const double idx = 1.0 / m->dx, idy = 1.0 / m->dy;
  const int cons = (mdot_u != NULL && mdot_v != NULL);
  const int imax = iu_max(m), jmax = jv_max(m);
  memset(adv_u, 0, n_u(m) * sizeof(double));
  memset(adv_v, 0, n_v(m) * sizeof(double));
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= imax; ++i) {
      double mE, mW, mN, mS;
      if (cons) {
        mE = 0.5 * (AU(mdot_u, i, j) + AU(mdot_u, i + 1, j));
        mW = 0.5 * (AU(mdot_u, i - 1, j) + AU(mdot_u, i, j));
        mN = 0.5 * (AV(mdot_v, i, j) + AV(mdot_v, i + 1, j));
        mS = 0.5 * (AV(mdot_v, i, j - 1) + AV(mdot_v, i + 1, j - 1));
      } else {
        mE = AC(rho_c, i + 1, j) * 0.5 * (AU(u_adv, i, j) + AU(u_adv, i + 1, j));
        mW = AC(rho_c, i, j) * 0.5 * (AU(u_adv, i - 1, j) + AU(u_adv, i, j));
        mN = 0.5 * (AV(rho_v, i, j) + AV(rho_v, i + 1, j)) * 0.5 * (AV(v_adv, i, j) + AV(v_adv, i + 1, j));
        mS = 0.5 * (AV(rho_v, i, j - 1) + AV(rho_v, i + 1, j - 1)) * 0.5 *
             (AV(v_adv, i, j - 1) + AV(v_adv, i + 1, j - 1));
      }
      double uE = 0.5 * (AU(u, i, j) + AU(u, i + 1, j));
      double uW = 0.5 * (AU(u, i - 1, j) + AU(u, i, j));
      double uN = 0.5 * (AU(u, i, j) + AU(u, i, j + 1));
      double uS = 0.5 * (AU(u, i, j - 1) + AU(u, i, j));
      AU(adv_u, i, j) = (mE * uE - mW * uW) * idx + (mN * uN - mS * uS) * idy;
    }
  for (int j = 1; j <= jmax; ++j)
    for (int i = 1; i <= nx; ++i) {
      double mE, mW, mN, mS;
      if (cons) {
        mE = 0.5 * (AU(mdot_u, i, j) + AU(mdot_u, i, j + 1));
        mW = 0.5 * (AU(mdot_u, i - 1, j) + AU(mdot_u, i - 1, j + 1));
        mN = 0.5 * (AV(mdot_v, i, j) + AV(mdot_v, i, j + 1));
        mS = 0.5 * (AV(mdot_v, i, j - 1) + AV(mdot_v, i, j));
      } else {
        mE = 0.5 * (AU(rho_u, i, j) + AU(rho_u, i, j + 1)) * 0.5 * (AU(u_adv, i, j) + AU(u_adv, i, j + 1));
        mW = 0.5 * (AU(rho_u, i - 1, j) + AU(rho_u, i - 1, j + 1)) * 0.5 *
             (AU(u_adv, i - 1, j) + AU(u_adv, i - 1, j + 1));
        mN = AC(rho_c, i, j + 1) * 0.5 * (AV(v_adv, i, j) + AV(v_adv, i, j + 1));
        mS = AC(rho_c, i, j) * 0.5 * (AV(v_adv, i, j - 1) + AV(v_adv, i, j));
      }
      double vE = 0.5 * (AV(v, i, j) + AV(v, i + 1, j));
      double vW = 0.5 * (AV(v, i - 1, j) + AV(v, i, j));
      double vN = 0.5 * (AV(v, i, j) + AV(v, i, j + 1));
      double vS = 0.5 * (AV(v, i, j - 1) + AV(v, i, j));
      AV(adv_v, i, j) = (mE * vE - mW * vW) * idx + (mN * vN - mS * vS) * idy;
    }
}

/* apply_velocity_bcs, mod_operators.f90:254-333.  West, east, south, north
 * in that order.  Extension: free_slip_x makes the tangential ghost of v at
 * the side walls symmetric (zero shear) instead of antisymmetric. */
void fo_apply_velocity_bcs(const fo_model* m, double* u, double* v, int has_lid, double u_lid_in) {
  const int nx = m->nx, ny = m->ny;
  const double u_lid = has_lid ? u_lid_in : 0.0;
  const double vs = m->free_slip_x ? 1.0 : -1.0;
  if (!m->periodic_x) {
    for (int j = 1 - NH; j <= ny + NH; ++j) {
      AU(u, 0, j) = 0.0;
      for (int i = 1; i <= NH; ++i) AU(u, -i, j) = -AU(u, i, j);
    }
    for (int j = 0 - NH; j <= ny + NH; ++j)
      for (int i = 1; i <= NH; ++i) AV(v, 1 - i, j) = vs * AV(v, i, j);
    for (int j = 1 - NH; j <= ny + NH; ++j) {
      AU(u, nx, j) = 0.0;
      for (int i = 1; i <= NH; ++i) AU(u, nx + i, j) = -AU(u, nx - i, j);
    }
    for (int j = 0 - NH; j <= ny + NH; ++j)
      for (int i = 1; i <= NH; ++i) AV(v, nx + i, j) = vs * AV(v, nx - i + 1, j);
  }
  if (!m->periodic_y) {
    for (int i = 1 - NH; i <= nx + NH; ++i) {
      AV(v, i, 0) = 0.0;
      for (int j = 1; j <= NH; ++j) AV(v, i, -j) = -AV(v, i, j);
    }
    for (int i = 0 - NH; i <= nx + NH; ++i)
      for (int j = 1; j <= NH; ++j) AU(u, i, 1 - j) = -AU(u, i, j);
    for (int i = 1 - NH; i <= nx + NH; ++i) {
      AV(v, i, ny) = 0.0;
      for (int j = 1; j <= NH; ++j) AV(v, i, ny + j) = -AV(v, i, ny - j);
    }
    for (int i = 0 - NH; i <= nx + NH; ++i)
      for (int j = 1; j <= NH; ++j) AU(u, i, ny + j) = 2.0 * u_lid - AU(u, i, ny - j + 1);
  }
}

/* matvec_coupled, mod_operators.f90:341-443 */
void fo_matvec_coupled(const fo_model* m, double* Xu, double* Xv, double* Xp,
                       double* Yu, double* Yv, double* Yp,
                       const double* u_adv, const double* v_adv,
                       const double* rho_c, const double* rho_u, const double* rho_v,
                       const double* kappa, const double* zeta, const double* eta,
                       double dt, int include_adv,
                       const double* pen_u, const double* pen_v,
                       const double* mdot_u, const double* mdot_v) {
  const int nx = m->nx, ny = m->ny;
  const int imax = iu_max(m), jmax = jv_max(m);
  double* visc_u = zalloc(n_u(m));
  double* adv_u = zalloc(n_u(m));
  double* gp_u = zalloc(n_u(m));
  double* visc_v = zalloc(n_v(m));
  double* adv_v = zalloc(n_v(m));
  double* gp_v = zalloc(n_v(m));

  fo_halo_u(m, Xu);
  fo_halo_v(m, Xv);
  fo_halo_scalar(m, Xp);
  fo_op_viscous_stress(m, Xu, Xv, kappa, zeta, eta, visc_u, visc_v);
  fo_op_grad_pressure(m, Xp, gp_u, gp_v);
  if (include_adv) {
    if (mdot_u && mdot_v)
      fo_op_advection(m, u_adv, v_adv, rho_c, rho_u, rho_v, Xu, Xv, adv_u, adv_v, mdot_u, mdot_v);
    else
      fo_op_advection(m, u_adv, v_adv, rho_c, rho_u, rho_v, Xu, Xv, adv_u, adv_v, NULL, NULL);
  }
  memset(Yu, 0, n_u(m) * sizeof(double));
  for (int j = 1; j <= ny; ++j) {
    for (int i = 1; i <= imax; ++i) {
      AU(Yu, i, j) = (AU(rho_u, i, j) / dt) * AU(Xu, i, j) + AU(adv_u, i, j) + AU(visc_u, i, j) +
                     AU(gp_u, i, j);
      if (pen_u) AU(Yu, i, j) = AU(Yu, i, j) + AU(pen_u, i, j) * AU(Xu, i, j);
    }
    if (!m->periodic_x) {
      AU(Yu, 0, j) = AU(Xu, 0, j);
      AU(Yu, nx, j) = AU(Xu, nx, j);
    }
  }
  memset(Yv, 0, n_v(m) * sizeof(double));
  for (int j = 1; j <= jmax; ++j)
    for (int i = 1; i <= nx; ++i) {
      AV(Yv, i, j) = (AV(rho_v, i, j) / dt) * AV(Xv, i, j) + AV(adv_v, i, j) + AV(visc_v, i, j) +
                     AV(gp_v, i, j);
      if (pen_v) AV(Yv, i, j) = AV(Yv, i, j) + AV(pen_v, i, j) * AV(Xv, i, j);
    }
  if (!m->periodic_y)
    for (int i = 1; i <= nx; ++i) {
      AV(Yv, i, 0) = AV(Xv, i, 0);
      AV(Yv, i, ny) = AV(Xv, i, ny);
    }
  fo_op_divergence(m, Xu, Xv, Yp);
  free(visc_u); free(adv_u); free(gp_u); free(visc_v); free(adv_v); free(gp_v);
}

/* ---------------------------------------------------------------------- */
/* mod_subsolvers.f90                                                      */
/* ---------------------------------------------------------------------- */
/* apply_neumann_bc_phi, mod_subsolvers.f90:378-416 (also mod_vof.f90:199-237) */
static void neumann_cell(const fo_model* m, double* phi) {
  const int nx = m->nx, ny = m->ny;
  if (!m->periodic_x) {
    for (int j = 1 - NH; j <= ny + NH; ++j)
      for (int i = 1; i <= NH; ++i) AC(phi, 1 - i, j) = AC(phi, i, j);
    for (int j = 1 - NH; j <= ny + NH; ++j)
      for (int i = 1; i <= NH; ++i) AC(phi, nx + i, j) = AC(phi, nx - i + 1, j);
  }
  if (!m->periodic_y) {
    for (int i = 1 - NH; i <= nx + NH; ++i)
      for (int j = 1; j <= NH; ++j) AC(phi, i, 1 - j) = AC(phi, i, j);
    for (int i = 1 - NH; i <= nx + NH; ++i)
      for (int j = 1; j <= NH; ++j) AC(phi, i, ny + j) = AC(phi, i, ny - j + 1);
  }
}

/* Poisson face coefficients of cell (i,j) with zero flux through walls
 * (mod_subsolvers.f90:65-78) */
static void poisson_coefs(const fo_model* m, const double* rho_u, const double* rho_v, int i,
                          int j, double idx2, double idy2, double* cE, double* cW, double* cN,
                          double* cS) {
  *cE = idx2 / AU(rho_u, i, j);
  *cW = idx2 / AU(rho_u, i - 1, j);
  *cN = idy2 / AV(rho_v, i, j);
  *cS = idy2 / AV(rho_v, i, j - 1);
  if (!m->periodic_x) {
    if (i == 1) *cW = 0.0;
    if (i == m->nx) *cE = 0.0;
  }
  if (!m->periodic_y) {
    if (j == 1) *cS = 0.0;
    if (j == m->ny) *cN = 0.0;
  }
}

/* solve_poisson_pressure, mod_subsolvers.f90:32-246 (Jacobi-PCG, zero-mean
 * projection when no direction is periodic) */
void fo_solve_poisson_pressure(const fo_model* m, double* phi, const double* rhs,
                               const double* rho_u, const double* rho_v,
                               double tol, int max_iter, int* iter_out, double* res_out) {
  const int nx = m->nx, ny = m->ny;
  const size_t nc = n_cell(m);
  const double idx2 = 1.0 / (m->dx * m->dx), idy2 = 1.0 / (m->dy * m->dy);
  const int closed = !m->periodic_x && !m->periodic_y;
  double* r = zalloc(nc);
  double* z = zalloc(nc);
  double* p = zalloc(nc);
  double* Ap = zalloc(nc);
  double* dinv = zalloc(nc);
  double* rw = zalloc(nc);
  double res_norm = 0.0, cE, cW, cN, cS;
  int iter;

  for (size_t k = 0; k < nc; ++k) dinv[k] = 1.0;
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i) {
      poisson_coefs(m, rho_u, rho_v, i, j, idx2, idy2, &cE, &cW, &cN, &cS);
      double d = cE + cW + cN + cS;
      AC(dinv, i, j) = d > 1.0e-14 ? 1.0 / d : 1.0;
    }

  memcpy(rw, rhs, nc * sizeof(double));
  if (closed) {
    dsum s = {0.0, 0.0};
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) ds_add(&s, AC(rhs, i, j));
    double mean = ds_val(s) / (double)(nx * ny);
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) AC(rw, i, j) = AC(rhs, i, j) - mean;
  }
  dsum dot = {0.0, 0.0};
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i) ds_add(&dot, AC(rw, i, j) * AC(rw, i, j));
  const double rhs_norm = sqrt(ds_val(dot));
  if (rhs_norm < 1.0e-14) {
    memset(phi, 0, nc * sizeof(double));
    if (iter_out) *iter_out = 0;
    if (res_out) *res_out = 0.0;
    goto done;
  }

  fo_halo_scalar(m, phi);
  neumann_cell(m, phi);
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i) {
      poisson_coefs(m, rho_u, rho_v, i, j, idx2, idy2, &cE, &cW, &cN, &cS);
      AC(Ap, i, j) = (cE + cW + cN + cS) * AC(phi, i, j) -
                     (cE * AC(phi, i + 1, j) + cW * AC(phi, i - 1, j) + cN * AC(phi, i, j + 1) +
                      cS * AC(phi, i, j - 1));
      AC(r, i, j) = AC(rw, i, j) - AC(Ap, i, j);
      AC(z, i, j) = AC(dinv, i, j) * AC(r, i, j);
      AC(p, i, j) = AC(z, i, j);
    }
  dsum rz0 = {0.0, 0.0};
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i) ds_add(&rz0, AC(r, i, j) * AC(z, i, j));
  double rz_old = ds_val(rz0);

  for (iter = 1; iter <= max_iter; ++iter) {
    fo_halo_scalar(m, p);
    neumann_cell(m, p);
    dsum pApd = {0.0, 0.0};
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        poisson_coefs(m, rho_u, rho_v, i, j, idx2, idy2, &cE, &cW, &cN, &cS);
        AC(Ap, i, j) = (cE + cW + cN + cS) * AC(p, i, j) -
                       (cE * AC(p, i + 1, j) + cW * AC(p, i - 1, j) + cN * AC(p, i, j + 1) +
                        cS * AC(p, i, j - 1));
        ds_add(&pApd, AC(p, i, j) * AC(Ap, i, j));
      }
    double pAp = ds_val(pApd);
    if (fabs(pAp) < 1.0e-30) break;
    double alpha = rz_old / pAp;
    dsum rrd = {0.0, 0.0};
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        AC(phi, i, j) = AC(phi, i, j) + alpha * AC(p, i, j);
        AC(r, i, j) = AC(r, i, j) - alpha * AC(Ap, i, j);
        AC(z, i, j) = AC(dinv, i, j) * AC(r, i, j);
        ds_add(&rrd, AC(r, i, j) * AC(r, i, j));
      }
    res_norm = sqrt(ds_val(rrd));
    if (res_norm / rhs_norm < tol) break;
    dsum rzn = {0.0, 0.0};
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) ds_add(&rzn, AC(r, i, j) * AC(z, i, j));
    double rz_new = ds_val(rzn);
    double beta = rz_new / rz_old;
    rz_old = rz_new;
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) AC(p, i, j) = AC(z, i, j) + beta * AC(p, i, j);
  }
  if (closed) {
    dsum s = {0.0, 0.0};
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) ds_add(&s, AC(phi, i, j));
    double mean = ds_val(s) / (double)(nx * ny);
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) AC(phi, i, j) = AC(phi, i, j) - mean;
  }
  if (iter_out) *iter_out = iter < max_iter ? iter : max_iter;
  if (res_out) *res_out = res_norm / rhs_norm;
done:
  free(r); free(z); free(p); free(Ap); free(dinv); free(rw);
}

/* solve_helmholtz_u, mod_subsolvers.f90:252-309 (damped Jacobi) */
void fo_solve_helmholtz_u(const fo_model* m, double* u_sol, const double* rhs_u,
                          const double* rho_u, const double* kappa, const double* zeta,
                          const double* eta, double dt, int n_sweeps, const double* pen_u) {
  const int nx = m->nx, ny = m->ny, imax = iu_max(m);
  const double om = m->jacobi_omega;
  const double idx2 = 1.0 / (m->dx * m->dx), idy2 = 1.0 / (m->dy * m->dy);
  if (m->pcd_smoother == 1) {
    /* red-black SOR (extension): in place, colour (i + j) & 1 per pass */
    const double w = m->pcd_sor_omega;
    for (int s = 0; s < n_sweeps; ++s)
      for (int col = 0; col < 2; ++col) {
        fo_halo_u(m, u_sol);
        for (int j = 1; j <= ny; ++j) {
          for (int i = 1; i <= imax; ++i) {
            if (((i + j) & 1) != col) continue;
            double cE = AC(kappa, i + 1, j) * idx2;
            double cW = AC(kappa, i, j) * idx2;
            double cN = (AW(zeta, i, j) - AW(eta, i, j)) * idy2;
            double cS = (AW(zeta, i, j - 1) - AW(eta, i, j - 1)) * idy2;
            double diag = (AU(rho_u, i, j) / dt) + cE + cW + cN + cS;
            if (pen_u) diag = diag + AU(pen_u, i, j);
            double off = cE * AU(u_sol, i + 1, j) + cW * AU(u_sol, i - 1, j) +
                         cN * AU(u_sol, i, j + 1) + cS * AU(u_sol, i, j - 1);
            if (diag > 1.0e-15)
              AU(u_sol, i, j) = (1.0 - w) * AU(u_sol, i, j) + w * ((AU(rhs_u, i, j) + off) / diag);
          }
          if (!m->periodic_x) {
            if ((j & 1) == col) AU(u_sol, 0, j) = AU(rhs_u, 0, j);
            if (((nx + j) & 1) == col) AU(u_sol, nx, j) = AU(rhs_u, nx, j);
          }
        }
      }
    return;
  }
  double* u_old = zalloc(n_u(m));
  for (int s = 0; s < n_sweeps; ++s) {
    fo_halo_u(m, u_sol);
    memcpy(u_old, u_sol, n_u(m) * sizeof(double));
    for (int j = 1; j <= ny; ++j) {
      for (int i = 1; i <= imax; ++i) {
        double cE = AC(kappa, i + 1, j) * idx2;
        double cW = AC(kappa, i, j) * idx2;
        double cN = (AW(zeta, i, j) - AW(eta, i, j)) * idy2;
        double cS = (AW(zeta, i, j - 1) - AW(eta, i, j - 1)) * idy2;
        double diag = (AU(rho_u, i, j) / dt) + cE + cW + cN + cS;
        if (pen_u) diag = diag + AU(pen_u, i, j);
        double off = cE * AU(u_old, i + 1, j) + cW * AU(u_old, i - 1, j) +
                     cN * AU(u_old, i, j + 1) + cS * AU(u_old, i, j - 1);
        if (diag > 1.0e-15)
          AU(u_sol, i, j) = (1.0 - om) * AU(u_old, i, j) + om * ((AU(rhs_u, i, j) + off) / diag);
      }
      if (!m->periodic_x) {
        AU(u_sol, 0, j) = AU(rhs_u, 0, j);
        AU(u_sol, nx, j) = AU(rhs_u, nx, j);
      }
    }
  }
  free(u_old);
}

/* solve_helmholtz_v, mod_subsolvers.f90:314-372 */
void fo_solve_helmholtz_v(const fo_model* m, double* v_sol, const double* rhs_v,
                          const double* rho_v, const double* kappa, const double* zeta,
                          const double* eta, double dt, int n_sweeps, const double* pen_v) {
  const int nx = m->nx, ny = m->ny, jmax = jv_max(m);
  const double om = m->jacobi_omega;
  const double idx2 = 1.0 / (m->dx * m->dx), idy2 = 1.0 / (m->dy * m->dy);
  if (m->pcd_smoother == 1) {
    /* red-black SOR (extension): in place, colour (i + j) & 1 per pass */
    const double w = m->pcd_sor_omega;
    for (int s = 0; s < n_sweeps; ++s)
      for (int col = 0; col < 2; ++col) {
        fo_halo_v(m, v_sol);
        for (int j = 1; j <= jmax; ++j)
          for (int i = 1; i <= nx; ++i) {
            if (((i + j) & 1) != col) continue;
            double cE = (AW(zeta, i, j) - AW(eta, i, j)) * idx2;
            double cW = (AW(zeta, i - 1, j) - AW(eta, i - 1, j)) * idx2;
            double cN = AC(kappa, i, j + 1) * idy2;
            double cS = AC(kappa, i, j) * idy2;
            double diag = (AV(rho_v, i, j) / dt) + cE + cW + cN + cS;
            if (pen_v) diag = diag + AV(pen_v, i, j);
            double off = cE * AV(v_sol, i + 1, j) + cW * AV(v_sol, i - 1, j) +
                         cN * AV(v_sol, i, j + 1) + cS * AV(v_sol, i, j - 1);
            if (diag > 1.0e-15)
              AV(v_sol, i, j) = (1.0 - w) * AV(v_sol, i, j) + w * ((AV(rhs_v, i, j) + off) / diag);
          }
        if (!m->periodic_y)
          for (int i = 1; i <= nx; ++i) {
            if ((i & 1) == col) AV(v_sol, i, 0) = AV(rhs_v, i, 0);
            if (((i + ny) & 1) == col) AV(v_sol, i, ny) = AV(rhs_v, i, ny);
          }
      }
    return;
  }
  double* v_old = zalloc(n_v(m));
  for (int s = 0; s < n_sweeps; ++s) {
    fo_halo_v(m, v_sol);
    memcpy(v_old, v_sol, n_v(m) * sizeof(double));
    for (int j = 1; j <= jmax; ++j)
      for (int i = 1; i <= nx; ++i) {
        double cE = (AW(zeta, i, j) - AW(eta, i, j)) * idx2;
        double cW = (AW(zeta, i - 1, j) - AW(eta, i - 1, j)) * idx2;
        double cN = AC(kappa, i, j + 1) * idy2;
        double cS = AC(kappa, i, j) * idy2;
        double diag = (AV(rho_v, i, j) / dt) + cE + cW + cN + cS;
        if (pen_v) diag = diag + AV(pen_v, i, j);
        double off = cE * AV(v_old, i + 1, j) + cW * AV(v_old, i - 1, j) +
                     cN * AV(v_old, i, j + 1) + cS * AV(v_old, i, j - 1);
        if (diag > 1.0e-15)
          AV(v_sol, i, j) = (1.0 - om) * AV(v_old, i, j) + om * ((AV(rhs_v, i, j) + off) / diag);
      }
    if (!m->periodic_y)
      for (int i = 1; i <= nx; ++i) {
        AV(v_sol, i, 0) = AV(rhs_v, i, 0);
        AV(v_sol, i, ny) = AV(rhs_v, i, ny);
      }
  }
  free(v_old);
}

/* ---------------------------------------------------------------------- */
/* mod_pcd_precond.f90:14-104                                              */
/* ---------------------------------------------------------------------- */
void fo_apply_pcd_precond(const fo_model* m, const double* z_u, const double* z_v,
                          const double* z_p, double* r_u, double* r_v, double* r_p,
                          const double* u_adv, const double* v_adv,
                          const double* rho_u, const double* rho_v,
                          const double* kappa, const double* zeta, const double* eta,
                          double dt, const double* pen_u, const double* pen_v,
                          fo_stats* st) {
  const int nx = m->nx, ny = m->ny;
  const double idx = 1.0 / m->dx, idy = 1.0 / m->dy;
  double* phi = zalloc(n_cell(m));
  double* zuw = zalloc(n_u(m));
  double* zvw = zalloc(n_v(m));
  int it = 0;
  double res = 0.0;
  memset(r_u, 0, n_u(m) * sizeof(double));
  memset(r_v, 0, n_v(m) * sizeof(double));
  memset(r_p, 0, n_cell(m) * sizeof(double));

  fo_solve_poisson_pressure(m, phi, z_p, rho_u, rho_v, m->pcg_tol, m->pcg_max_iter, &it, &res);
  if (st) { st->pcg_iters += it; st->pcg_calls += 1; }
  fo_halo_scalar(m, phi);
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i) {
      double ua = 0.5 * (AU(u_adv, i, j) + AU(u_adv, i - 1, j));
      double va = 0.5 * (AV(v_adv, i, j) + AV(v_adv, i, j - 1));
      double conv = ua * (AC(phi, i + 1, j) - AC(phi, i - 1, j)) * (0.5 * idx) +
                    va * (AC(phi, i, j + 1) - AC(phi, i, j - 1)) * (0.5 * idy);
      AC(r_p, i, j) = -((1.0 / dt) * AC(phi, i, j) + conv);
      /* extension: the viscous part of the Schur complement */
      if (m->pcd_visc_scale != 0.0) AC(r_p, i, j) -= m->pcd_visc_scale * 0.5 * AC(kappa, i, j) * AC(z_p, i, j);
    }
  fo_halo_scalar(m, r_p);

  for (int j = 1; j <= ny; ++j) {
    for (int i = 1; i <= nx - 1; ++i)
      AU(zuw, i, j) = AU(z_u, i, j) - (AC(r_p, i + 1, j) - AC(r_p, i, j)) * idx;
    AU(zuw, 0, j) = AU(z_u, 0, j);
    AU(zuw, nx, j) = AU(z_u, nx, j);
  }
  for (int j = 1; j <= ny - 1; ++j)
    for (int i = 1; i <= nx; ++i)
      AV(zvw, i, j) = AV(z_v, i, j) - (AC(r_p, i, j + 1) - AC(r_p, i, j)) * idy;
  for (int i = 1; i <= nx; ++i) {
    AV(zvw, i, 0) = AV(z_v, i, 0);
    AV(zvw, i, ny) = AV(z_v, i, ny);
  }

  fo_solve_helmholtz_v(m, r_v, zvw, rho_v, kappa, zeta, eta, dt, m->pcd_sweeps, pen_v);
  fo_halo_v(m, r_v);
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx - 1; ++i) {
      double cross = -idy * (AW(eta, i, j) * (AV(r_v, i + 1, j) - AV(r_v, i, j)) * idx -
                             AW(eta, i, j - 1) * (AV(r_v, i + 1, j - 1) - AV(r_v, i, j - 1)) * idx);
      AU(zuw, i, j) = AU(zuw, i, j) - cross;
    }
  fo_solve_helmholtz_u(m, r_u, zuw, rho_u, kappa, zeta, eta, dt, m->pcd_sweeps, pen_u);
  fo_halo_u(m, r_u);
  free(phi); free(zuw); free(zvw);
}

/* ---------------------------------------------------------------------- */
/* mod_bicgstab2.f90                                                       */
/* ---------------------------------------------------------------------- */
/* coupled_dot, mod_bicgstab2.f90:32-72 */
double fo_coupled_dot(const fo_model* m, const double* u1, const double* v1, const double* p1,
                      const double* u2, const double* v2, const double* p2) {
  const int nx = m->nx, ny = m->ny, imax = iu_max(m), jmax = jv_max(m);
  const double vol = m->dx * m->dy;
  dsum s = {0.0, 0.0};
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= imax; ++i) ds_add(&s, AU(u1, i, j) * AU(u2, i, j) * vol);
  for (int j = 1; j <= jmax; ++j)
    for (int i = 1; i <= nx; ++i) ds_add(&s, AV(v1, i, j) * AV(v2, i, j) * vol);
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i) ds_add(&s, AC(p1, i, j) * AC(p2, i, j) * vol);
  return ds_val(s);
}

/* a coupled (u,v,p) work triple allocated over the full padded extents */
typedef struct { double *u, *v, *p; } trip;
static trip trip_new(const fo_model* m) {
  trip t = {zalloc(n_u(m)), zalloc(n_v(m)), zalloc(n_cell(m))};
  return t;
}
static void trip_free(trip t) { free(t.u); free(t.v); free(t.p); }
/* whole-array y = a + s*b (Fortran array expressions over every element) */
static void lin2(const fo_model* m, trip y, trip a, double s, trip b) {
  for (size_t k = 0; k < n_u(m); ++k) y.u[k] = a.u[k] + s * b.u[k];
  for (size_t k = 0; k < n_v(m); ++k) y.v[k] = a.v[k] + s * b.v[k];
  for (size_t k = 0; k < n_cell(m); ++k) y.p[k] = a.p[k] + s * b.p[k];
}
static void copy3(const fo_model* m, trip y, trip a) {
  memcpy(y.u, a.u, n_u(m) * sizeof(double));
  memcpy(y.v, a.v, n_v(m) * sizeof(double));
  memcpy(y.p, a.p, n_cell(m) * sizeof(double));
}
static double cdot(const fo_model* m, trip a, trip b) { return fo_coupled_dot(m, a.u, a.v, a.p, b.u, b.v, b.p); }

typedef struct {
  const fo_model* m;
  const double *u_adv, *v_adv, *rho_c, *rho_u, *rho_v, *kappa, *zeta, *eta;
  const double *pen_u, *pen_v, *mdot_u, *mdot_v;
  double dt;
  fo_stats* st;
} kctx;

static void kc_matvec(const kctx* c, trip x, trip y) {
  fo_matvec_coupled(c->m, x.u, x.v, x.p, y.u, y.v, y.p, c->u_adv, c->v_adv, c->rho_c, c->rho_u,
                    c->rho_v, c->kappa, c->zeta, c->eta, c->dt, 1, c->pen_u, c->pen_v, c->mdot_u,
                    c->mdot_v);
  if (c->st) c->st->matvecs += 1;
}
static void kc_precond(const kctx* c, trip z, trip r) {
  fo_apply_pcd_precond(c->m, z.u, z.v, z.p, r.u, r.v, r.p, c->u_adv, c->v_adv, c->rho_u, c->rho_v,
                       c->kappa, c->zeta, c->eta, c->dt, c->pen_u, c->pen_v, c->st);
}

/* bicgstab_solve, mod_bicgstab2.f90:77-264 */
static void bicgstab1(const kctx* c, trip X, trip B, double tol, int max_iter, int has_lid,
                      double u_lid, int* iter_out, double* res_out) {
  const fo_model* m = c->m;
  trip bh = trip_new(m), r = trip_new(m), r0 = trip_new(m), p = trip_new(m), v = trip_new(m),
       s = trip_new(m), t = trip_new(m), z = trip_new(m);
  int k;
  fo_apply_velocity_bcs(m, X.u, X.v, 0, 0.0);
  kc_precond(c, B, bh);
  double norm_b = sqrt(cdot(m, bh, bh));
  if (norm_b < 1.0e-14) norm_b = 1.0;
  kc_matvec(c, X, z);
  kc_precond(c, z, v);
  lin2(m, r, bh, -1.0, v); /* r = b_hat - v  (a + (-1)*b == a - b exactly) */
  copy3(m, r0, r);
  copy3(m, p, r);
  double rho_old = cdot(m, r0, r);
  double rel = sqrt(cdot(m, r, r)) / norm_b;
  double alpha = 0.0, omega = 1.0;
  for (k = 1; k <= max_iter; ++k) {
    if (rel < tol) break;
    fo_apply_velocity_bcs(m, p.u, p.v, 0, 0.0);
    kc_matvec(c, p, z);
    kc_precond(c, z, v);
    fo_apply_velocity_bcs(m, v.u, v.v, 0, 0.0);
    double rv = cdot(m, r0, v);
    if (fabs(rv) < 1.0e-30) break;
    alpha = rho_old / rv;
    lin2(m, s, r, -alpha, v);
    fo_apply_velocity_bcs(m, s.u, s.v, 0, 0.0);
    kc_matvec(c, s, z);
    kc_precond(c, z, t);
    fo_apply_velocity_bcs(m, t.u, t.v, 0, 0.0);
    double tt = cdot(m, t, t), ts = cdot(m, t, s);
    omega = tt > 1.0e-30 ? ts / tt : 0.0;
    for (size_t q = 0; q < n_u(m); ++q) X.u[q] = X.u[q] + alpha * p.u[q] + omega * s.u[q];
    for (size_t q = 0; q < n_v(m); ++q) X.v[q] = X.v[q] + alpha * p.v[q] + omega * s.v[q];
    for (size_t q = 0; q < n_cell(m); ++q) X.p[q] = X.p[q] + alpha * p.p[q] + omega * s.p[q];
    lin2(m, r, s, -omega, t);
    rel = sqrt(cdot(m, r, r)) / norm_b;
    if (g_verbose) fprintf(stderr, "bicgstab k=%d rel=%.6e\n", k, rel);
    if (rel < tol) break;
    if (fabs(omega) < 1.0e-30) break;
    double rho_new = cdot(m, r0, r);
    if (fabs(rho_old) < 1.0e-30) break;
    double beta = (rho_new / rho_old) * (alpha / omega);
    rho_old = rho_new;
    for (size_t q = 0; q < n_u(m); ++q) p.u[q] = r.u[q] + beta * (p.u[q] - omega * v.u[q]);
    for (size_t q = 0; q < n_v(m); ++q) p.v[q] = r.v[q] + beta * (p.v[q] - omega * v.v[q]);
    for (size_t q = 0; q < n_cell(m); ++q) p.p[q] = r.p[q] + beta * (p.p[q] - omega * v.p[q]);
    fo_apply_velocity_bcs(m, X.u, X.v, 0, 0.0);
  }
  if (has_lid) fo_apply_velocity_bcs(m, X.u, X.v, 1, u_lid);
  if (iter_out) *iter_out = k < max_iter ? k : max_iter;
  if (res_out) *res_out = rel;
  trip_free(bh); trip_free(r); trip_free(r0); trip_free(p); trip_free(v); trip_free(s);
  trip_free(t); trip_free(z);
}

/* bicgstab2_solve, mod_bicgstab2.f90:270-570 */
static void bicgstab2(const kctx* c, trip X, trip B, double tol, int max_iter, int has_lid,
                      double u_lid, int* iter_out, double* res_out) {
  const fo_model* m = c->m;
  trip bh = trip_new(m), r = trip_new(m), rt = trip_new(m), uu = trip_new(m), vv = trip_new(m),
       ww = trip_new(m), ss = trip_new(m), tt = trip_new(m), z = trip_new(m), q = trip_new(m);
  int k;
  fo_apply_velocity_bcs(m, X.u, X.v, 0, 0.0);
  kc_precond(c, B, bh);
  double norm_b = sqrt(cdot(m, bh, bh));
  if (norm_b < 1.0e-14) norm_b = 1.0;
  kc_matvec(c, X, z);
  kc_precond(c, z, q);
  lin2(m, r, bh, -1.0, q);
  copy3(m, rt, r);
  /* uu, vv start at zero (trip_new) */
  double xi0 = 1.0, xi1, omega1 = 0.0, omega2 = 1.0, alpha = 0.0, beta, gamma;
  double rel = sqrt(cdot(m, r, r)) / norm_b;
  for (k = 1; k <= max_iter; ++k) {
    if (rel < tol) break;
    if (fabs(omega2) > 1.0e-14) xi0 = -omega2 * xi0;
    else if (fabs(omega1) > 1.0e-14) xi0 = -omega1 * xi0;
    else xi0 = -xi0;
    /* even half */
    xi1 = cdot(m, rt, r);
    if (fabs(xi0) < 1.0e-30) break;
    beta = alpha * (xi1 / xi0);
    xi0 = xi1;
    lin2(m, uu, r, -beta, uu);
    fo_apply_velocity_bcs(m, uu.u, uu.v, 0, 0.0);
    kc_matvec(c, uu, z);
    kc_precond(c, z, vv);
    fo_apply_velocity_bcs(m, vv.u, vv.v, 0, 0.0);
    gamma = cdot(m, rt, vv);
    if (fabs(gamma) < 1.0e-30) break;
    alpha = xi0 / gamma;
    lin2(m, r, r, -alpha, vv);
    if (m->krylov_bc_fix) fo_apply_velocity_bcs(m, r.u, r.v, 0, 0.0);
    kc_matvec(c, r, z);
    kc_precond(c, z, ss);
    fo_apply_velocity_bcs(m, ss.u, ss.v, 0, 0.0);
    lin2(m, X, X, alpha, uu);
    /* odd half */
    xi1 = cdot(m, rt, ss);
    if (fabs(xi0) < 1.0e-30) break;
    beta = alpha * (xi1 / xi0);
    xi0 = xi1;
    lin2(m, vv, ss, -beta, vv);
    fo_apply_velocity_bcs(m, vv.u, vv.v, 0, 0.0);
    kc_matvec(c, vv, z);
    kc_precond(c, z, ww);
    fo_apply_velocity_bcs(m, ww.u, ww.v, 0, 0.0);
    gamma = cdot(m, rt, ww);
    if (fabs(gamma) < 1.0e-30) break;
    alpha = xi0 / gamma;
    lin2(m, uu, r, -beta, uu);
    lin2(m, r, r, -alpha, vv);
    lin2(m, ss, ss, -alpha, ww);
    kc_matvec(c, ss, z);
    kc_precond(c, z, tt);
    fo_apply_velocity_bcs(m, tt.u, tt.v, 0, 0.0);
    /* GCR(2) */
    omega1 = cdot(m, r, ss);
    double lambda = cdot(m, ss, ss);
    double nu = cdot(m, ss, tt);
    double tau = cdot(m, tt, tt);
    omega2 = cdot(m, r, tt);
    if (lambda * tau > 1.0e-30) {
      double det = lambda * tau - nu * nu;
      if (det > 1.0e-14 * (lambda * tau)) {
        double c1 = omega1, c2 = omega2;
        omega1 = (c1 * tau - c2 * nu) / det;
        omega2 = (c2 * lambda - c1 * nu) / det;
      } else if (lambda > 1.0e-30) {
        omega1 = omega1 / lambda;
        omega2 = 0.0;
      } else {
        omega1 = 0.0;
        omega2 = 0.0;
      }
    } else if (lambda > 1.0e-30) {
      omega1 = omega1 / lambda;
      omega2 = 0.0;
    } else {
      omega1 = 0.0;
      omega2 = 0.0;
    }
    for (size_t qq = 0; qq < n_u(m); ++qq) X.u[qq] = X.u[qq] + omega1 * r.u[qq] + omega2 * ss.u[qq] + alpha * uu.u[qq];
    for (size_t qq = 0; qq < n_v(m); ++qq) X.v[qq] = X.v[qq] + omega1 * r.v[qq] + omega2 * ss.v[qq] + alpha * uu.v[qq];
    for (size_t qq = 0; qq < n_cell(m); ++qq) X.p[qq] = X.p[qq] + omega1 * r.p[qq] + omega2 * ss.p[qq] + alpha * uu.p[qq];
    for (size_t qq = 0; qq < n_u(m); ++qq) r.u[qq] = r.u[qq] - omega1 * ss.u[qq] - omega2 * tt.u[qq];
    for (size_t qq = 0; qq < n_v(m); ++qq) r.v[qq] = r.v[qq] - omega1 * ss.v[qq] - omega2 * tt.v[qq];
    for (size_t qq = 0; qq < n_cell(m); ++qq) r.p[qq] = r.p[qq] - omega1 * ss.p[qq] - omega2 * tt.p[qq];
    for (size_t qq = 0; qq < n_u(m); ++qq) uu.u[qq] = uu.u[qq] - omega1 * vv.u[qq] - omega2 * ww.u[qq];
    for (size_t qq = 0; qq < n_v(m); ++qq) uu.v[qq] = uu.v[qq] - omega1 * vv.v[qq] - omega2 * ww.v[qq];
    for (size_t qq = 0; qq < n_cell(m); ++qq) uu.p[qq] = uu.p[qq] - omega1 * vv.p[qq] - omega2 * ww.p[qq];
    rel = sqrt(cdot(m, r, r)) / norm_b;
    if (g_verbose) fprintf(stderr, "bicgstab2 k=%d rel=%.6e om1=%.3e om2=%.3e\n", k, rel, omega1, omega2);
    fo_apply_velocity_bcs(m, X.u, X.v, 0, 0.0);
  }
  if (has_lid) fo_apply_velocity_bcs(m, X.u, X.v, 1, u_lid);
  if (iter_out) *iter_out = k < max_iter ? k : max_iter;
  if (res_out) *res_out = rel;
  trip_free(bh); trip_free(r); trip_free(rt); trip_free(uu); trip_free(vv); trip_free(ww);
  trip_free(ss); trip_free(tt); trip_free(z); trip_free(q);
}

/* Flexible GMRES with right PCD preconditioning (extension, not in the
 * reference; the inner solve of refine_solve when refine == 2).  One cycle
 * of at most max_iter Arnoldi steps from X = 0: the outer defect correction
 * restarts it.  Z_j = M^{-1} V_j is kept because M (PCD around a truncated
 * PCG) differs from one application to the next; wall BCs are applied to
 * Z_j before A, as the Krylov solvers do.  Classical Gram-Schmidt applied
 * twice (all projections of a pass are independent dot products); Givens
 * rotations on the Hessenberg column.  Stops when |g_{j+1}| / |B| < tol,
 * which for right preconditioning is the residual of the unpreconditioned
 * system in exact arithmetic. */
static void fgmres(const kctx* c, trip X, trip B, double tol, int max_iter, int* iter_out, double* res_out) {
  const fo_model* m = c->m;
  const int mr = max_iter < 1 ? 1 : max_iter;
  trip* V = (trip*)calloc((size_t)mr + 1, sizeof(trip));
  trip* Z = (trip*)calloc((size_t)mr, sizeof(trip));
  double* H = (double*)calloc((size_t)(mr + 1) * mr, sizeof(double)); /* H[i + j*(mr+1)] */
  double *cs = (double*)calloc(mr, sizeof(double)), *sn = (double*)calloc(mr, sizeof(double));
  double *g = (double*)calloc((size_t)mr + 1, sizeof(double)), *y = (double*)calloc(mr, sizeof(double));
  double* h = (double*)calloc((size_t)mr + 1, sizeof(double));
  trip w = trip_new(m);
  int k = 0;
  const double beta = sqrt(cdot(m, B, B));
  double rel = 0.0;
  if (beta > 0.0) {
    V[0] = trip_new(m);
    lin2(m, V[0], V[0], 1.0 / beta, B); /* V0 = 0 + B/beta */
    g[0] = beta;
    rel = 1.0;
    for (int j = 0; j < mr; ++j) {
      Z[j] = trip_new(m);
      kc_precond(c, V[j], Z[j]);
      fo_apply_velocity_bcs(m, Z[j].u, Z[j].v, 0, 0.0);
      kc_matvec(c, Z[j], w);
      for (int i = 0; i <= j + 1; ++i) H[i + (size_t)j * (mr + 1)] = 0.0;
      for (int pass = 0; pass < 2; ++pass) {
        for (int i = 0; i <= j; ++i) h[i] = cdot(m, w, V[i]);
        for (int i = 0; i <= j; ++i) {
          lin2(m, w, w, -h[i], V[i]);
          H[i + (size_t)j * (mr + 1)] += h[i];
        }
      }
      const double hn = sqrt(cdot(m, w, w));
      H[j + 1 + (size_t)j * (mr + 1)] = hn;
      k = j + 1;
      /* apply the previous rotations, then a new one zeroing H[j+1, j] */
      double* col = &H[(size_t)j * (mr + 1)];
      for (int i = 0; i < j; ++i) {
        const double a = col[i], b = col[i + 1];
        col[i] = cs[i] * a + sn[i] * b;
        col[i + 1] = -sn[i] * a + cs[i] * b;
      }
      const double a = col[j], b = col[j + 1];
      const double rr = sqrt(a * a + b * b);
      cs[j] = rr > 0.0 ? a / rr : 1.0;
      sn[j] = rr > 0.0 ? b / rr : 0.0;
      col[j] = rr;
      col[j + 1] = 0.0;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs[j] * g[j];
      rel = fabs(g[j + 1]) / beta;
      if (g_verbose) fprintf(stderr, "fgmres k=%d rel=%.6e\n", k, rel);
      if (rel < tol || hn == 0.0 || j + 1 == mr) break;
      V[j + 1] = trip_new(m);
      lin2(m, V[j + 1], V[j + 1], 1.0 / hn, w);
    }
    /* back substitution R y = g, then X += sum_j y_j Z_j */
    for (int i = k - 1; i >= 0; --i) {
      double s = g[i];
      for (int q = i + 1; q < k; ++q) s -= H[i + (size_t)q * (mr + 1)] * y[q];
      y[i] = H[i + (size_t)i * (mr + 1)] != 0.0 ? s / H[i + (size_t)i * (mr + 1)] : 0.0;
    }
    for (int i = 0; i < k; ++i) lin2(m, X, X, y[i], Z[i]);
  }
  if (iter_out) *iter_out = k;
  if (res_out) *res_out = rel;
  for (int i = 0; i <= mr; ++i)
    if (V[i].u) trip_free(V[i]);
  for (int i = 0; i < mr; ++i)
    if (Z[i].u) trip_free(Z[i]);
  trip_free(w);
  free(V); free(Z); free(H); free(cs); free(sn); free(g); free(y); free(h);
}

/* FP64 defect correction around an inner BiCGStab(l)+PCD solve (extension,
 * not in the reference): the true residual B - A X is formed with the
 * homogeneous wall BCs applied to X, so the operator is the same linear map
 * in every product; the inner solve restarts from zero on each defect. */
static void refine_solve(const kctx* c, int solver, trip X, trip B, double tol, int has_lid,
                         double u_lid, int* iter_out, double* res_out) {
  const fo_model* m = c->m;
  trip r = trip_new(m), d = trip_new(m), ax = trip_new(m);
  int inner_total = 0, outer;
  double rel = 0.0;
  /* adaptive PCG cap of the PCD (refine = 2 with pcg_cap_start > 0) */
  const int adapt = m->refine == 2 && m->pcg_cap_start > 0;
  int cap = adapt && m->pcg_cap_start < m->pcg_max_iter ? m->pcg_cap_start : m->pcg_max_iter;
  if (adapt && c->st && c->st->pcg_cap > cap) cap = c->st->pcg_cap < m->pcg_max_iter ? c->st->pcg_cap : m->pcg_max_iter;
  /* adaptive PCD sweeps (refine = 2 with pcd_sweeps_max > pcd_sweeps) */
  const int adapt_sw = m->refine == 2 && m->pcd_sweeps_max > m->pcd_sweeps;
  int sweeps = m->pcd_sweeps;
  if (adapt_sw && c->st && c->st->pcd_sweeps > sweeps)
    sweeps = c->st->pcd_sweeps < m->pcd_sweeps_max ? c->st->pcd_sweeps : m->pcd_sweeps_max;
  fo_apply_velocity_bcs(m, X.u, X.v, 0, 0.0);
  double nb = sqrt(cdot(m, B, B));
  if (nb < 1.0e-300) nb = 1.0;
  for (outer = 0;; ++outer) {
    kc_matvec(c, X, ax);
    lin2(m, r, B, -1.0, ax);
    rel = sqrt(cdot(m, r, r)) / nb;
    if (g_verbose) fprintf(stderr, "refine outer=%d true_rel=%.6e inner_total=%d\n", outer, rel, inner_total);
    if (rel < tol || outer >= m->refine_max_outer) break;
    memset(d.u, 0, n_u(m) * sizeof(double));
    memset(d.v, 0, n_v(m) * sizeof(double));
    memset(d.p, 0, n_cell(m) * sizeof(double));
    int it = 0;
    double ires = 0.0;
    if (m->refine == 2) {
      /* the PCD of this pass runs its PCG at the current cap */
      fo_model mm = *m;
      mm.pcg_max_iter = cap;
      mm.pcd_sweeps = sweeps;
      kctx cc = *c;
      cc.m = &mm;
      fgmres(&cc, d, r, m->refine_inner_tol, m->refine_max_inner, &it, &ires);
      /* a pass whose inner solve missed its tolerance doubles the cap, or,
       * once the cap cannot grow, the PCD sweeps */
      if (!(ires < m->refine_inner_tol)) {
        if (adapt && cap < m->pcg_max_iter)
          cap = 2 * cap < m->pcg_max_iter ? 2 * cap : m->pcg_max_iter;
        else if (adapt_sw && sweeps < m->pcd_sweeps_max)
          sweeps = 2 * sweeps < m->pcd_sweeps_max ? 2 * sweeps : m->pcd_sweeps_max;
      }
    } else if (solver == 2) {
      bicgstab2(c, d, r, m->refine_inner_tol, m->refine_max_inner, 0, 0.0, &it, &ires);
    } else {
      bicgstab1(c, d, r, m->refine_inner_tol, m->refine_max_inner, 0, 0.0, &it, &ires);
    }
    inner_total += it;
    lin2(m, X, X, 1.0, d);
    fo_apply_velocity_bcs(m, X.u, X.v, 0, 0.0);
  }
  if (c->st) c->st->outer += outer;
  if (adapt && c->st) c->st->pcg_cap = cap;
  if (adapt_sw && c->st) c->st->pcd_sweeps = sweeps;
  if (has_lid) fo_apply_velocity_bcs(m, X.u, X.v, 1, u_lid);
  if (iter_out) *iter_out = inner_total;
  if (res_out) *res_out = rel;
  trip_free(r); trip_free(d); trip_free(ax);
}

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
                     int* iter_out, double* res_out, fo_stats* st) {
  kctx c = {m, u_adv, v_adv, rho_c, rho_u, rho_v, kappa, zeta, eta,
            pen_u, pen_v, mdot_u, mdot_v, dt, st};
  trip X = {Xu, Xv, Xp};
  trip B = {(double*)Bu, (double*)Bv, (double*)Bp};
  if (m->refine) refine_solve(&c, solver, X, B, tol, has_lid, u_lid, iter_out, res_out);
  else if (solver == 2) bicgstab2(&c, X, B, tol, max_iter, has_lid, u_lid, iter_out, res_out);
  else bicgstab1(&c, X, B, tol, max_iter, has_lid, u_lid, iter_out, res_out);
}

/* ---------------------------------------------------------------------- */
/* mod_vof.f90                                                             */
/* ---------------------------------------------------------------------- */
/* flux limiter: van_leer_limiter (mod_vof.f90:25-33); Superbee is the
 * flag-gated extension */
static double limiter(const fo_model* m, double r) {
  if (m->limiter == 1) {
    double a = dmin(2.0 * r, 1.0), b = dmin(r, 2.0);
    return dmax(0.0, dmax(a, b));
  }
  if (r <= 0.0) return 0.0;
  return (2.0 * r) / (1.0 + r);
}

/* vof_advection_tvd, mod_vof.f90:38-140 */
void fo_vof_advection_tvd(const fo_model* m, const double* c_in, double* c_out,
                          const double* u, const double* v, double dt,
                          double* flux_x, double* flux_y) {
  const int nx = m->nx, ny = m->ny;
  const double idx = 1.0 / m->dx, idy = 1.0 / m->dy;
  const int lfx = nx + 1, lfy = nx;
  double* fx = zalloc((size_t)lfx * ny);       /* Flux_x(0:nx, 1:ny) */
  double* fy = zalloc((size_t)lfy * (ny + 1)); /* Flux_y(1:nx, 0:ny) */
#define FX(i, j) fx[(size_t)(i) + (size_t)((j)-1) * lfx]
#define FY(i, j) fy[(size_t)((i)-1) + (size_t)(j) * lfy]
  for (int j = 1; j <= ny; ++j)
    for (int i = 0; i <= nx; ++i) {
      double uf = AU(u, i, j), num, den, r, cfl, cf;
      if (uf >= 0.0) {
        num = AC(c_in, i, j) - AC(c_in, i - 1, j);
        den = AC(c_in, i + 1, j) - AC(c_in, i, j);
        r = fabs(den) > 1.0e-12 ? num / den : 0.0;
        cfl = fabs(uf) * dt * idx;
        cf = AC(c_in, i, j) + 0.5 * (1.0 - cfl) * limiter(m, r) * den;
      } else {
        num = AC(c_in, i + 2, j) - AC(c_in, i + 1, j);
        den = AC(c_in, i + 1, j) - AC(c_in, i, j);
        r = fabs(den) > 1.0e-12 ? num / den : 0.0;
        cfl = fabs(uf) * dt * idx;
        cf = AC(c_in, i + 1, j) - 0.5 * (1.0 - cfl) * limiter(m, r) * den;
      }
      FX(i, j) = uf * clip01(cf);
    }
  for (int j = 0; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i) {
      double vf = AV(v, i, j), num, den, r, cfl, cf;
      if (vf >= 0.0) {
        num = AC(c_in, i, j) - AC(c_in, i, j - 1);
        den = AC(c_in, i, j + 1) - AC(c_in, i, j);
        r = fabs(den) > 1.0e-12 ? num / den : 0.0;
        cfl = fabs(vf) * dt * idy;
        cf = AC(c_in, i, j) + 0.5 * (1.0 - cfl) * limiter(m, r) * den;
      } else {
        num = AC(c_in, i, j + 2) - AC(c_in, i, j + 1);
        den = AC(c_in, i, j + 1) - AC(c_in, i, j);
        r = fabs(den) > 1.0e-12 ? num / den : 0.0;
        cfl = fabs(vf) * dt * idy;
        cf = AC(c_in, i, j + 1) - 0.5 * (1.0 - cfl) * limiter(m, r) * den;
      }
      FY(i, j) = vf * clip01(cf);
    }
  memcpy(c_out, c_in, n_cell(m) * sizeof(double));
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i) {
      double cnew = AC(c_in, i, j) - dt * ((FX(i, j) - FX(i - 1, j)) * idx + (FY(i, j) - FY(i, j - 1)) * idy);
      AC(c_out, i, j) = clip01(cnew);
    }
  if (flux_x) {
    memset(flux_x, 0, n_u(m) * sizeof(double));
    for (int j = 1; j <= ny; ++j)
      for (int i = 0; i <= nx; ++i) AU(flux_x, i, j) = FX(i, j);
    fo_halo_u(m, flux_x);
  }
  if (flux_y) {
    memset(flux_y, 0, n_v(m) * sizeof(double));
    for (int j = 0; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) AV(flux_y, i, j) = FY(i, j);
    fo_halo_v(m, flux_y);
  }
  fo_halo_scalar(m, c_out);
#undef FX
#undef FY
  free(fx); free(fy);
}

/* svof_helmholtz_filter, mod_vof.f90:145-194; returns the iteration count */
int fo_svof_helmholtz_filter(const fo_model* m, const double* c_raw, double* c_smooth,
                             double delta, int max_iter, double tol) {
  const int nx = m->nx, ny = m->ny;
  const double cx = (delta / m->dx) * (delta / m->dx);
  const double cy = (delta / m->dy) * (delta / m->dy);
  const double diag = 1.0 + 2.0 * (cx + cy);
  double* c_old = zalloc(n_cell(m));
  int it, used = 0;
  memcpy(c_smooth, c_raw, n_cell(m) * sizeof(double));
  for (it = 1; it <= max_iter; ++it) {
    used = it;
    fo_halo_scalar(m, c_smooth);
    neumann_cell(m, c_smooth);
    memcpy(c_old, c_smooth, n_cell(m) * sizeof(double));
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i)
        AC(c_smooth, i, j) = (AC(c_raw, i, j) + cx * (AC(c_old, i + 1, j) + AC(c_old, i - 1, j)) +
                              cy * (AC(c_old, i, j + 1) + AC(c_old, i, j - 1))) / diag;
    double res = 0.0;
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) res = dmax(res, fabs(AC(c_smooth, i, j) - AC(c_old, i, j)));
    if (res < tol) break;
  }
  fo_halo_scalar(m, c_smooth);
  neumann_cell(m, c_smooth);
  free(c_old);
  return used;
}

/* ---------------------------------------------------------------------- */
/* mod_surface_tension.f90                                                 */
/* ---------------------------------------------------------------------- */
/* compute_interface_curvature, mod_surface_tension.f90:25-72 */
void fo_compute_interface_curvature(const fo_model* m, const double* cs, double* kc) {
  const int nx = m->nx, ny = m->ny;
  const double idx = 1.0 / m->dx, idy = 1.0 / m->dy, eps = 1.0e-12;
  double* nxu = zalloc(n_u(m));
  double* nyv = zalloc(n_v(m));
  for (int j = 1; j <= ny; ++j)
    for (int i = 0; i <= nx; ++i) {
      double gx = (AC(cs, i + 1, j) - AC(cs, i, j)) * idx;
      double gy = 0.25 * (AC(cs, i, j + 1) + AC(cs, i + 1, j + 1) - AC(cs, i, j - 1) - AC(cs, i + 1, j - 1)) * idy;
      double nrm = sqrt(gx * gx + gy * gy + eps);
      AU(nxu, i, j) = gx / nrm;
    }
  for (int j = 0; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i) {
      double gx = 0.25 * (AC(cs, i + 1, j) + AC(cs, i + 1, j + 1) - AC(cs, i - 1, j) - AC(cs, i - 1, j + 1)) * idx;
      double gy = (AC(cs, i, j + 1) - AC(cs, i, j)) * idy;
      double nrm = sqrt(gx * gx + gy * gy + eps);
      AV(nyv, i, j) = gy / nrm;
    }
  memset(kc, 0, n_cell(m) * sizeof(double));
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i)
      AC(kc, i, j) = -((AU(nxu, i, j) - AU(nxu, i - 1, j)) * idx + (AV(nyv, i, j) - AV(nyv, i, j - 1)) * idy);
  fo_halo_scalar(m, kc);
  free(nxu); free(nyv);
}

/* compute_csf_force, mod_surface_tension.f90:78-109 */
void fo_compute_csf_force(const fo_model* m, const double* c, const double* kc,
                          double* fsu, double* fsv) {
  const int nx = m->nx, ny = m->ny;
  const double idx = 1.0 / m->dx, idy = 1.0 / m->dy;
  memset(fsu, 0, n_u(m) * sizeof(double));
  memset(fsv, 0, n_v(m) * sizeof(double));
  for (int j = 1; j <= ny; ++j)
    for (int i = 0; i <= nx; ++i) {
      double kf = 0.5 * (AC(kc, i, j) + AC(kc, i + 1, j));
      AU(fsu, i, j) = m->sigma * kf * (AC(c, i + 1, j) - AC(c, i, j)) * idx;
    }
  for (int j = 0; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i) {
      double kf = 0.5 * (AC(kc, i, j) + AC(kc, i, j + 1));
      AV(fsv, i, j) = m->sigma * kf * (AC(c, i, j + 1) - AC(c, i, j)) * idy;
    }
}

/* ---------------------------------------------------------------------- */
/* mod_solver_coupled.f90                                                  */
/* ---------------------------------------------------------------------- */
/* compute_adaptive_dt, mod_solver_coupled.f90:41-91 */
double fo_compute_adaptive_dt(const fo_model* m, const double* u, const double* v, double dt_max) {
  const int nx = m->nx, ny = m->ny;
  const double h = dmin(m->dx, m->dy);
  const double pi = 3.141592653589793238462643383279502884197;
  double um = 0.0, vm = 0.0, dtl, dcfl;
  for (int j = 1; j <= ny; ++j)
    for (int i = 0; i <= nx; ++i) um = dmax(um, fabs(AU(u, i, j)));
  for (int j = 0; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i) vm = dmax(vm, fabs(AV(v, i, j)));
  if (um / m->dx + vm / m->dy > 1.0e-12) dcfl = m->cfl_target / (um / m->dx + vm / m->dy);
  else dcfl = dt_max;
  dtl = dmin(dt_max, dcfl);
  if (m->sigma > 1.0e-14) {
    double dcap = 0.5 * sqrt((m->rho1 + m->rho2) * (h * h * h) / (4.0 * pi * m->sigma));
    dtl = dmin(dtl, dcap);
  }
  double g = sqrt(m->gx * m->gx + m->gy * m->gy);
  if (g > 1.0e-14) dtl = dmin(dtl, 0.5 * sqrt(h / g));
  return dtl;
}

/* build_cylinder_mask, mod_solver_coupled.f90:96-132 (i_start=j_start=1) */
void fo_build_cylinder_mask(const fo_model* m, double xc, double yc, double rad,
                            double* phi_u, double* phi_v) {
  const int nx = m->nx, ny = m->ny;
  memset(phi_u, 0, n_u(m) * sizeof(double));
  memset(phi_v, 0, n_v(m) * sizeof(double));
  for (int j = 1; j <= ny; ++j) {
    double y = ((double)j - 0.5) * m->dy;
    for (int i = 0; i <= nx; ++i) {
      double x = (double)i * m->dx;
      if (sqrt((x - xc) * (x - xc) + (y - yc) * (y - yc)) <= rad) AU(phi_u, i, j) = 1.0;
    }
  }
  for (int j = 0; j <= ny; ++j) {
    double y = (double)j * m->dy;
    for (int i = 1; i <= nx; ++i) {
      double x = ((double)i - 0.5) * m->dx;
      if (sqrt((x - xc) * (x - xc) + (y - yc) * (y - yc)) <= rad) AV(phi_v, i, j) = 1.0;
    }
  }
  fo_halo_u(m, phi_u);
  fo_halo_v(m, phi_v);
}

/* advance_coupled_step, mod_solver_coupled.f90:137-380 */
void fo_advance_coupled_step(const fo_model* m,
                             double* u_vel, double* v_vel, double* p_field, double* c_field,
                             double* u_prev, double* v_prev,
                             double* rho_c, double* rho_u, double* rho_v,
                             double* kappa, double* zeta, double* eta,
                             double* kappa_curv, double* f_sigma_u, double* f_sigma_v,
                             double dt, int step_idx, const fo_step_opts* o, fo_stats* st) {
  const int nx = m->nx, ny = m->ny, imax = iu_max(m), jmax = jv_max(m);
  const size_t NU = n_u(m), NV = n_v(m), NC = n_cell(m);
  const int has_pen = o->phi_s_u && o->phi_s_v;
  const double u_sol = o->has_u_solid ? o->u_solid : 0.0;
  const double v_sol = o->has_v_solid ? o->v_solid : 0.0;
  const double tol = o->has_tol ? o->tol : m->tol_bicgstab2;
  const int max_it = o->has_max_iter ? o->max_iter : m->max_iter_bicgstab2;
  const double u_lid = o->has_lid ? o->u_top_lid : 0.0;
  const int bdf2 = (m->time_order == 2 && step_idx >= 2);
  const double dt_eff = bdf2 ? dt / 1.5 : dt;

  double* u_n = zalloc(NU); double* v_n = zalloc(NV);
  double* u_nm1 = zalloc(NU); double* v_nm1 = zalloc(NV);
  double* u_adv = zalloc(NU); double* v_adv = zalloc(NV);
  double* c_new = zalloc(NC); double* c_s = zalloc(NC);
  double* Bu = zalloc(NU); double* Bv = zalloc(NV); double* Bp = zalloc(NC);
  double *fcx = NULL, *fcy = NULL, *mdu = NULL, *mdv = NULL, *pen_u = NULL, *pen_v = NULL;

  memcpy(u_n, u_vel, NU * sizeof(double));
  memcpy(v_n, v_vel, NV * sizeof(double));
  memcpy(u_nm1, u_prev, NU * sizeof(double));
  memcpy(v_nm1, v_prev, NV * sizeof(double));
  if (step_idx <= 1) {
    memcpy(u_adv, u_n, NU * sizeof(double));
    memcpy(v_adv, v_n, NV * sizeof(double));
  } else {
    for (size_t k = 0; k < NU; ++k) u_adv[k] = 2.0 * u_n[k] - u_nm1[k];
    for (size_t k = 0; k < NV; ++k) v_adv[k] = 2.0 * v_n[k] - v_nm1[k];
  }
  memcpy(u_prev, u_n, NU * sizeof(double));
  memcpy(v_prev, v_n, NV * sizeof(double));

  if (o->consistent_amp) {
    fcx = zalloc(NU); fcy = zalloc(NV); mdu = zalloc(NU); mdv = zalloc(NV);
    fo_vof_advection_tvd(m, c_field, c_new, u_n, v_n, dt, fcx, fcy);
    for (size_t k = 0; k < NU; ++k) mdu[k] = (m->rho1 - m->rho2) * fcx[k] + m->rho2 * u_adv[k];
    for (size_t k = 0; k < NV; ++k) mdv[k] = (m->rho1 - m->rho2) * fcy[k] + m->rho2 * v_adv[k];
  } else {
    fo_vof_advection_tvd(m, c_field, c_new, u_n, v_n, dt, NULL, NULL);
  }
  memcpy(c_field, c_new, NC * sizeof(double));

  fo_compute_mixture_densities(m, c_field, rho_c, rho_u, rho_v);
  fo_compute_mixture_viscosities(m, c_field, kappa, zeta, eta);

  if (m->sigma > 1.0e-14) {
    double delta = m->svof_delta_h * dmin(m->dx, m->dy);
    int its = fo_svof_helmholtz_filter(m, c_field, c_s, delta, m->svof_max_iter, m->svof_tol);
    if (st) st->svof_iters += its;
    fo_compute_interface_curvature(m, c_s, kappa_curv);
    fo_compute_csf_force(m, c_field, kappa_curv, f_sigma_u, f_sigma_v);
  } else {
    memset(kappa_curv, 0, NC * sizeof(double));
    memset(f_sigma_u, 0, NU * sizeof(double));
    memset(f_sigma_v, 0, NV * sizeof(double));
  }

  if (has_pen) {
    pen_u = zalloc(NU); pen_v = zalloc(NV);
    for (size_t k = 0; k < NU; ++k) pen_u[k] = m->alpha_penalty * o->phi_s_u[k];
    for (size_t k = 0; k < NV; ++k) pen_v[k] = m->alpha_penalty * o->phi_s_v[k];
  }

  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= imax; ++i) {
      double b;
      if (bdf2)
        b = (AU(rho_u, i, j) / dt) * (2.0 * AU(u_n, i, j) - 0.5 * AU(u_nm1, i, j)) +
            AU(rho_u, i, j) * m->gx + AU(f_sigma_u, i, j);
      else
        b = (AU(rho_u, i, j) / dt) * AU(u_n, i, j) + AU(rho_u, i, j) * m->gx + AU(f_sigma_u, i, j);
      if (has_pen) b = b + AU(pen_u, i, j) * u_sol;
      AU(Bu, i, j) = b;
    }
  if (o->has_lid && !m->periodic_y)
    for (int i = 1; i <= imax; ++i)
      AU(Bu, i, ny) = AU(Bu, i, ny) + (2.0 * (AW(zeta, i, ny) - AW(eta, i, ny)) / (m->dy * m->dy)) * u_lid;
  for (int j = 1; j <= jmax; ++j)
    for (int i = 1; i <= nx; ++i) {
      double b;
      if (bdf2)
        b = (AV(rho_v, i, j) / dt) * (2.0 * AV(v_n, i, j) - 0.5 * AV(v_nm1, i, j)) +
            AV(rho_v, i, j) * m->gy + AV(f_sigma_v, i, j);
      else
        b = (AV(rho_v, i, j) / dt) * AV(v_n, i, j) + AV(rho_v, i, j) * m->gy + AV(f_sigma_v, i, j);
      if (has_pen) b = b + AV(pen_v, i, j) * v_sol;
      AV(Bv, i, j) = b;
    }

  int it = 0;
  double res = 0.0;
  fo_krylov_solve(m, o->use_bicgstab2 ? 2 : 1, u_vel, v_vel, p_field, Bu, Bv, Bp, u_adv, v_adv,
                  rho_c, rho_u, rho_v, kappa, zeta, eta, dt_eff, tol, max_it, 1, u_lid, pen_u,
                  pen_v, o->consistent_amp ? mdu : NULL, o->consistent_amp ? mdv : NULL, &it,
                  &res, st);

  fo_halo_u(m, u_vel);
  fo_halo_v(m, v_vel);
  fo_halo_scalar(m, p_field);
  fo_apply_velocity_bcs(m, u_vel, v_vel, 1, u_lid);
  if (st) { st->iter = it; st->res = res; }

  free(u_n); free(v_n); free(u_nm1); free(v_nm1); free(u_adv); free(v_adv);
  free(c_new); free(c_s); free(Bu); free(Bv); free(Bp);
  free(fcx); free(fcy); free(mdu); free(mdv); free(pen_u); free(pen_v);
}

/* ---------------------------------------------------------------------- */
/* mod_io.f90:169-225 checkpoint: stream binary, header step(int32),       */
/* t(real64), nx, ny, nh (int32), then u, v, u_prev, v_prev, p, c whole    */
/* arrays including halos, column-major.                                   */
/* ---------------------------------------------------------------------- */
int fo_write_checkpoint(const fo_model* m, const char* path, int step, double t,
                        const double* u, const double* v, const double* u_prev,
                        const double* v_prev, const double* p, const double* c) {
  FILE* f = fopen(path, "wb");
  if (!f) return -1;
  int hdr[3] = {m->nx, m->ny, NH};
  fwrite(&step, sizeof(int), 1, f);
  fwrite(&t, sizeof(double), 1, f);
  fwrite(hdr, sizeof(int), 3, f);
  fwrite(u, sizeof(double), n_u(m), f);
  fwrite(v, sizeof(double), n_v(m), f);
  fwrite(u_prev, sizeof(double), n_u(m), f);
  fwrite(v_prev, sizeof(double), n_v(m), f);
  fwrite(p, sizeof(double), n_cell(m), f);
  fwrite(c, sizeof(double), n_cell(m), f);
  return fclose(f) == 0 ? 0 : -1;
}

int fo_read_checkpoint(const fo_model* m, const char* path, int* step, double* t,
                       double* u, double* v, double* u_prev, double* v_prev,
                       double* p, double* c) {
  FILE* f = fopen(path, "rb");
  if (!f) return -1;
  int hdr[3];
  if (fread(step, sizeof(int), 1, f) != 1 || fread(t, sizeof(double), 1, f) != 1 ||
      fread(hdr, sizeof(int), 3, f) != 3 || hdr[0] != m->nx || hdr[1] != m->ny || hdr[2] != NH) {
    fclose(f);
    return -2;
  }
  size_t ok = fread(u, sizeof(double), n_u(m), f) + fread(v, sizeof(double), n_v(m), f) +
              fread(u_prev, sizeof(double), n_u(m), f) + fread(v_prev, sizeof(double), n_v(m), f) +
              fread(p, sizeof(double), n_cell(m), f) + fread(c, sizeof(double), n_cell(m), f);
  fclose(f);
  return ok == 2 * n_u(m) + 2 * n_v(m) + 2 * n_cell(m) ? 0 : -3;
}
