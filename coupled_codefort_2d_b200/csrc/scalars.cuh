// scalars.cuh -- device-resident Krylov scalars and the fused dot + scalar
// recurrence kernel.  The recurrences of bicgstab_solve / bicgstab2_solve
// (mod_bicgstab2.f90:77-570) run on the GPU in the last CTA of each dot
// reduction, so an iteration needs no host round trip; an `exit` of the
// reference clears the `active` flag, which every later kernel of the
// iteration checks.
#pragma once

#include "fugu_internal.cuh"

namespace fugu {

enum Slot {
  S_ALPHA = 0, S_BETA, S_OMEGA, S_RHO, S_RHONEW, S_XI0, S_XI1, S_GAMMA, S_OM1, S_OM2,
  S_NORMB, S_REL, S_TT, S_TS, S_LAMBDA, S_NU, S_TAU,
  S_D0, S_D1, S_D2, S_D3, S_D4,
  S_ONE, S_RNORM, S_INVRNORM, S_REFNB, S_TRUEREL,
  NSLOTS = 32
};

enum Op {
  OP_STORE = 0,   // just store the dots
  OP_NORMB,       // norm_b = sqrt(d0), 1 if < 1e-14                      (:147-148, :345-346)
  OP_B1_INIT,     // rho_old = d0, rel = sqrt(d1)/norm_b, top check k=1     (:173-181)
  OP_B1_ALPHA,    // rv = d0, exit if |rv|<1e-30, alpha = rho_old/rv        (:196-198)
  OP_B1_OMEGA,    // omega = tt>1e-30 ? ts/tt : 0                           (:217-223)
  OP_B1_END,      // rel, exits, beta, rho_old                             (:233-242)
  OP_B2_INIT,     // rel = sqrt(d0)/norm_b, xi0=1, om1=0, om2=1, alpha=0    (:375-385)
  OP_B2_XI_EVEN,  // sign trick, xi1, beta, xi0                             (:387-401)
  OP_B2_XI_ODD,   // xi1, beta, xi0                                         (:449-452)
  OP_B2_GAMMA,    // gamma, alpha                                           (:421-423, :472-474)
  OP_B2_GCR,      // omega1, omega2 from the 2x2 normal equations           (:504-530)
  OP_B2_REL,      // rel = sqrt(d0)/norm_b                                  (:546-547)
  OP_TOPCHECK,    // exit at the top of iteration k if rel < tol            (:181, :385)
  OP_REF_NORMB,   // refine: |B|
  OP_REF_REL      // refine: |r|, 1/|r|, |r|/|B|
};

struct OpArgs {
  int op;
  int k;
  double tol;
};

struct KState {
  int active;
  int exit_iter;   // iteration at which the reference's loop exits (0 = ran out)
  int nan;
  unsigned int ticket;
  int kiter;       // iteration index of a BiCGStab(l) replayed from a CUDA graph
  unsigned long long matvecs;
};

__device__ __forceinline__ void kexit(KState* ks, int k) {
  ks->active = 0;
  ks->exit_iter = k;
}

// The iteration index an op reports on exit: o.k, or, when o.k < 0, the
// device counter ks->kiter, so that one captured BiCGStab(l) iteration serves
// every k.  OP_TOPCHECK tests the top of the next iteration (k + 1); it and
// OP_B1_END, the last op of an iteration, advance the counter.
__device__ __forceinline__ int op_k(const OpArgs& o, const KState* ks) {
  return o.k >= 0 ? o.k : ks->kiter + (o.op == OP_TOPCHECK ? 1 : 0);
}

__device__ inline void krylov_op_body(const OpArgs& o, double* sc, KState* ks);
__device__ inline void krylov_op(const OpArgs& o, double* sc, KState* ks) {
  krylov_op_body(o, sc, ks);
  if (o.k < 0 && (o.op == OP_TOPCHECK || o.op == OP_B1_END)) ks->kiter += 1;
}
__device__ inline void krylov_op_body(const OpArgs& o, double* sc, KState* ks) {
  const double d0 = sc[S_D0], d1 = sc[S_D1], d2 = sc[S_D2], d3 = sc[S_D3], d4 = sc[S_D4];
  switch (o.op) {
    case OP_STORE:
      break;
    case OP_NORMB: {
      double nb = sqrt(d0);
      if (nb < 1.0e-14) nb = 1.0;
      sc[S_NORMB] = nb;
      break;
    }
    case OP_B1_INIT:
      sc[S_RHO] = d0;
      sc[S_REL] = sqrt(d1) / sc[S_NORMB];
      sc[S_ALPHA] = 0.0;
      sc[S_OMEGA] = 1.0;
      if (sc[S_REL] < o.tol) kexit(ks, 1);
      break;
    case OP_B1_ALPHA:
      if (fabs(d0) < 1.0e-30) { kexit(ks, op_k(o, ks)); break; }
      sc[S_ALPHA] = sc[S_RHO] / d0;
      break;
    case OP_B1_OMEGA:
      sc[S_TT] = d0;
      sc[S_TS] = d1;
      sc[S_OMEGA] = d0 > 1.0e-30 ? d1 / d0 : 0.0;
      break;
    case OP_B1_END: {
      const double rel = sqrt(d0) / sc[S_NORMB];
      sc[S_REL] = rel;
      if (isnan(rel)) { ks->nan = 1; kexit(ks, op_k(o, ks)); break; }
      if (rel < o.tol) { kexit(ks, op_k(o, ks)); break; }
      if (fabs(sc[S_OMEGA]) < 1.0e-30) { kexit(ks, op_k(o, ks)); break; }
      const double rho_new = d1;
      if (fabs(sc[S_RHO]) < 1.0e-30) { kexit(ks, op_k(o, ks)); break; }
      sc[S_BETA] = (rho_new / sc[S_RHO]) * (sc[S_ALPHA] / sc[S_OMEGA]);
      sc[S_RHO] = rho_new;
      break;
    }
    case OP_B2_INIT:
      sc[S_XI0] = 1.0;
      sc[S_OM1] = 0.0;
      sc[S_OM2] = 1.0;
      sc[S_ALPHA] = 0.0;
      sc[S_REL] = sqrt(d0) / sc[S_NORMB];
      if (sc[S_REL] < o.tol) kexit(ks, 1);
      break;
    case OP_B2_XI_EVEN: {
      double xi0 = sc[S_XI0];
      if (fabs(sc[S_OM2]) > 1.0e-14) xi0 = -sc[S_OM2] * xi0;
      else if (fabs(sc[S_OM1]) > 1.0e-14) xi0 = -sc[S_OM1] * xi0;
      else xi0 = -xi0;
      sc[S_XI0] = xi0;
      sc[S_XI1] = d0;
      if (fabs(xi0) < 1.0e-30) { kexit(ks, op_k(o, ks)); break; }
      sc[S_BETA] = sc[S_ALPHA] * (d0 / xi0);
      sc[S_XI0] = d0;
      break;
    }
    case OP_B2_XI_ODD: {
      const double xi0 = sc[S_XI0];
      sc[S_XI1] = d0;
      if (fabs(xi0) < 1.0e-30) { kexit(ks, op_k(o, ks)); break; }
      sc[S_BETA] = sc[S_ALPHA] * (d0 / xi0);
      sc[S_XI0] = d0;
      break;
    }
    case OP_B2_GAMMA:
      sc[S_GAMMA] = d0;
      if (fabs(d0) < 1.0e-30) { kexit(ks, op_k(o, ks)); break; }
      sc[S_ALPHA] = sc[S_XI0] / d0;
      break;
    case OP_B2_GCR: {
      double om1 = d0, om2 = d4;
      const double lambda = d1, nu = d2, tau = d3;
      sc[S_LAMBDA] = lambda; sc[S_NU] = nu; sc[S_TAU] = tau;
      if (lambda * tau > 1.0e-30) {
        const double det = lambda * tau - nu * nu;
        if (det > 1.0e-14 * (lambda * tau)) {
          const double c1 = om1, c2 = om2;
          om1 = (c1 * tau - c2 * nu) / det;
          om2 = (c2 * lambda - c1 * nu) / det;
        } else if (lambda > 1.0e-30) {
          om1 = om1 / lambda;
          om2 = 0.0;
        } else {
          om1 = 0.0;
          om2 = 0.0;
        }
      } else if (lambda > 1.0e-30) {
        om1 = om1 / lambda;
        om2 = 0.0;
      } else {
        om1 = 0.0;
        om2 = 0.0;
      }
      sc[S_OM1] = om1;
      sc[S_OM2] = om2;
      break;
    }
    case OP_B2_REL: {
      const double rel = sqrt(d0) / sc[S_NORMB];
      sc[S_REL] = rel;
      if (isnan(rel)) { ks->nan = 1; kexit(ks, op_k(o, ks)); }
      break;
    }
    case OP_TOPCHECK:
      if (sc[S_REL] < o.tol) kexit(ks, op_k(o, ks));
      break;
    case OP_REF_NORMB: {
      double nb = sqrt(d0);
      if (nb < 1.0e-300) nb = 1.0;
      sc[S_REFNB] = nb;
      break;
    }
    case OP_REF_REL: {
      const double rn = sqrt(d0);
      sc[S_RNORM] = rn;
      sc[S_INVRNORM] = rn > 0.0 ? 1.0 / rn : 0.0;
      sc[S_TRUEREL] = rn / sc[S_REFNB];
      if (isnan(rn)) ks->nan = 1;
      break;
    }
  }
  (void)d2; (void)d3;
}

// coupled dots of up to 5 pairs + the scalar recurrence in the last CTA
template <typename T>
struct DotArgs {
  Geo g;
  long n;            // elements of one component buffer
  const T* a[5];
  const T* b[5];
  int npairs;
  double vol;
  double* part;      // >= 10 * gridDim.x (5 DD partials per CTA)
  double* sc;
  KState* ks;
  OpArgs op;
  int check_active;  // skip when the solve has exited
};

// one CTA's share (block b of G) of the coupled dots; the last CTA to finish
// runs the scalar op
template <typename T>
__device__ __forceinline__ void dot_op_body(const DotArgs<T>& d, int b, int G) {
  __shared__ DD sh[32];
  __shared__ bool last;
  const Geo g = d.g;
  DD acc[5];
#pragma unroll
  for (int p = 0; p < 5; ++p) acc[p] = DD{0.0, 0.0};
  const int nx = g.nx, ny = g.ny, imax = g.imax(), jmax = g.jmax();
  const long nu = (long)imax * ny, nv = (long)nx * jmax, np = (long)nx * ny;
  for (long q = b * (long)blockDim.x + threadIdx.x; q < nu + nv + np; q += (long)G * blockDim.x) {
    long e;
    if (q < nu) {
      e = g.at(1 + (int)(q % imax), 1 + (int)(q / imax));
    } else if (q < nu + nv) {
      const long r = q - nu;
      e = d.n + g.at(1 + (int)(r % nx), 1 + (int)(r / nx));
    } else {
      const long r = q - nu - nv;
      e = 2 * d.n + g.at(1 + (int)(r % nx), 1 + (int)(r / nx));
    }
#pragma unroll
    for (int p = 0; p < 5; ++p)
      if (p < d.npairs) dd_add(acc[p], (double(d.a[p][e]) * double(d.b[p][e])) * d.vol);
  }
  for (int p = 0; p < d.npairs; ++p) {
    const DD s = block_sum_dd(acc[p], sh);
    if (threadIdx.x == 0) put_partial(d.part + 2 * p * G, b, s);
  }
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned int t = atomicAdd(&d.ks->ticket, 1u);
    last = (t == (unsigned int)G - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int p = 0; p < d.npairs; ++p) {
    const double s = sum_partials_dd(d.part + 2 * p * G, G);
    if (threadIdx.x == 0) d.sc[S_D0 + p] = s;
  }
  if (threadIdx.x == 0) {
    d.ks->ticket = 0;
    krylov_op(d.op, d.sc, d.ks);
  }
}
template <typename T>
__global__ void __launch_bounds__(256) k_dot_op(DotArgs<T> d) {
  if (d.check_active && !d.ks->active) return;
  dot_op_body<T>(d, blockIdx.x, gridDim.x);
}

__global__ void k_scalar_op(OpArgs op, double* sc, KState* ks, int check_active) {
  if (check_active && !ks->active) return;
  krylov_op(op, sc, ks);
}

}  // namespace fugu
