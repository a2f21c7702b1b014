// step_vjp.cuh -- kernels of the vector-Jacobian product of one coupled step
// (extension, no counterpart in the reference).
//
// The explicit stages of advance_coupled_step (mod_solver_coupled.f90:137-380)
// are local stencils: an output entry depends only on input entries a few
// cells away.  Their transposes are taken without storing a Jacobian:
//   1. seed the tangent of one input field with 1 on the entries of one
//      colour (one point of a lattice of period s = 2R + 1 in padded
//      coordinates, R the stage's reach) and run the stage on ad::Dual;
//   2. every output within R of a seeded entry got its derivative from that
//      entry alone (the lattice has one point in any window of s entries), so
//      x_bar(q) = sum over outputs o within R of q of ydot(o) * y_bar(o).
// Over all colours this is exactly J^T y_bar for the branch the step took.
// The sums run in a fixed order, so the result is deterministic.
#pragma once

#include "adjoint.cuh"
#include "dual.cuh"
#include "kernels.cuh"

namespace fugu {

using ad::Dual;

// which entries of a padded field are inputs of a probe
enum VjpMask { VM_CELL = 0, VM_U = 1, VM_V = 2, VM_INTERIOR = 3, VM_OWNED_U = 4, VM_OWNED_V = 5 };

__device__ __forceinline__ bool vjp_in(const Geo& g, int mask, int i, int j) {
  switch (mask) {
    case VM_CELL: return in_kind(g, K_CELL, i, j);
    case VM_U: return in_kind(g, K_U, i, j);
    case VM_V: return in_kind(g, K_V, i, j);
    case VM_INTERIOR: return i >= 1 && i <= g.nx && j >= 1 && j <= g.ny;
    case VM_OWNED_U: return adj_owned(g, 0, i, j);
    case VM_OWNED_V: return adj_owned(g, 1, i, j);
    default: return false;
  }
}

// out = Dual(x, seed): seed 1 on the admitted entries of colour (a, b) of
// period s when `seeded`, else 0.  x may be null (values 0).
__global__ void k_dual_pack(Geo g, const double* x, Dual* out, int mask, int seeded, int s, int a, int b) {
  FUGU_BOX_IJ
  const double v = x ? x[k] : 0.0;
  const bool on = seeded && ii % s == a && jj % s == b && vjp_in(g, mask, i, j);
  out[k] = Dual(v, on ? 1.0 : 0.0);
}

constexpr int VJP_MAXOUT = 3;
struct VjpOut {
  const Dual* y[VJP_MAXOUT];     // tangent outputs (their .d)
  const Dual* ysub[VJP_MAXOUT];  // nullable: minus its .d (B - A X)
  const double* ybar[VJP_MAXOUT];
  int n;
};

// x_bar(q) += sum_{o: |o - q| <= R} sum_f ydot_f(o) * y_bar_f(o) for the admitted
// input entries q of colour (a, b); one thread per lattice point
__global__ void k_vjp_gather(Geo g, VjpOut o, int mask, int s, int a, int b, int R, double* xbar) {
  const int ii = a + s * (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int jj = b + s * (int)(blockIdx.y * blockDim.y + threadIdx.y);
  if (ii >= g.P || jj >= g.R) return;
  if (!vjp_in(g, mask, ii - 2, jj - 2)) return;
  double acc = 0.0;
  for (int dj = -R; dj <= R; ++dj) {
    const int oj = jj + dj;
    if (oj < 0 || oj >= g.R) continue;
    for (int di = -R; di <= R; ++di) {
      const int oi = ii + di;
      if (oi < 0 || oi >= g.P) continue;
      const long ko = oi + (long)oj * g.P;
      for (int f = 0; f < o.n; ++f) {
        double yd = o.y[f][ko].d;
        if (o.ysub[f]) yd = yd - o.ysub[f][ko].d;
        acc += yd * o.ybar[f][ko];
      }
    }
  }
  xbar[ii + (long)jj * g.P] += acc;
}

// u_adv of the AB extrapolation (k_extrapolate) on duals
__global__ void k_adv_dual(long n, const Dual* x, const Dual* prev, Dual* adv, int first) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x)
    adv[q] = first ? x[q] : 2.0 * x[q] - prev[q];
}

// zero every entry of a coupled triple that is not an owned unknown
__global__ void k_keep_owned(Geo g, double* t, long n) {
  FUGU_BOX_IJ
  for (int cc = 0; cc < 3; ++cc)
    if (!adj_owned(g, cc, i, j)) t[cc * n + k] = 0.0;
}

// dst += src on the interior cells
__global__ void k_add_interior(Geo g, const double* src, double* dst) {
  FUGU_BOX_IJ
  if (i >= 1 && i <= g.nx && j >= 1 && j <= g.ny) dst[k] += src[k];
}

// t = (B - Y).d on the owned unknowns, 0 elsewhere (the tangent of the
// solve's residual for a parameter seed)
__global__ void k_dual_resid(Geo g, const Dual* bu, const Dual* bv, const Dual* bp, const Dual* yu,
                             const Dual* yv, const Dual* yp, double* t, long n) {
  FUGU_BOX_IJ
  t[k] = adj_owned(g, 0, i, j) ? bu[k].d - yu[k].d : 0.0;
  t[n + k] = adj_owned(g, 1, i, j) ? bv[k].d - yv[k].d : 0.0;
  t[2 * n + k] = adj_owned(g, 2, i, j) ? bp[k].d - yp[k].d : 0.0;
}

}  // namespace fugu
