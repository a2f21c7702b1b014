// adjoint.cuh -- the transpose of the coupled operator (extension, no
// counterpart in the reference): the stencil of the linear map the Krylov
// solvers see, x_owned -> (A . BC(x))_owned (matvec_coupled,
// mod_operators.f90:341-443, after apply_velocity_bcs, :254-333), is measured
// by probing it with coloured unit vectors, then applied transposed by a
// gather kernel (a fixed summation order, no atomics).
//
// Every entry of a row couples unknowns at most 2 cells away in i and j
// (the 11-point coupling plus ghost values that mirror or wrap interior
// values); unit vectors of one colour are at least 5 cells apart (or the
// period divides the periodic extent), so each probe result entry belongs to
// exactly one column.  A probe entry that no column within reach can explain
// is counted as an error instead of being stored.
//
// Stencil storage: val[((cr * 3 + cc) * 25 + (di + 2) * 5 + (dj + 2)) * n + at(i, j)]
// = A[(cr, i, j), (cc, i + di, j + dj)] with component indices 0 = u, 1 = v,
// 2 = p and the column index wrapped in periodic directions.
#pragma once

#include "kernels.cuh"

namespace fugu {

constexpr int ADJ_SLOTS = 225;  // 3 row components x 3 column components x 5 x 5 offsets

// owned unknowns of a component (the coupled_dot index set)
__device__ __forceinline__ bool adj_owned(const Geo& g, int comp, int i, int j) {
  const int i1 = comp == 0 ? g.imax() : g.nx;
  const int j1 = comp == 1 ? g.jmax() : g.ny;
  return i >= 1 && i <= i1 && j >= 1 && j <= j1;
}
__device__ __forceinline__ int adj_wrap(int i, int len, int periodic) {
  if (!periodic) return i;
  return ((i - 1) % len + len) % len + 1;
}

// unit entries of component cc at owned (i, j) with colour ((i-1) % qx, (j-1) % qy) == (a, b)
__global__ void k_adj_probe_set(Geo g, double* X, long n, int cc, int qx, int qy, int a, int b) {
  FUGU_BOX_IJ
  if (adj_owned(g, cc, i, j) && (i - 1) % qx == a && (j - 1) % qy == b) X[cc * n + g.at(i, j)] = 1.0;
}

// store the probe result Y of colour (cc, a, b) into the stencil
__global__ void k_adj_probe_collect(Geo g, const double* Y, long n, int cc, int qx, int qy, int a, int b,
                                    double* val, unsigned int* err) {
  FUGU_BOX_IJ
  for (int cr = 0; cr < 3; ++cr) {
    if (!adj_owned(g, cr, i, j)) continue;
    const double y = Y[cr * n + g.at(i, j)];
    bool found = false;
    for (int di = -2; di <= 2 && !found; ++di) {
      const int ic = adj_wrap(i + di, g.nx, g.px);
      for (int dj = -2; dj <= 2; ++dj) {
        const int jc = adj_wrap(j + dj, g.ny, g.py);
        if (!adj_owned(g, cc, ic, jc) || (ic - 1) % qx != a || (jc - 1) % qy != b) continue;
        val[(long)((cr * 3 + cc) * 25 + (di + 2) * 5 + (dj + 2)) * n + g.at(i, j)] = y;
        found = true;
        break;
      }
    }
    if (!found && y != 0.0) atomicAdd(err, 1u);
  }
}

// y = S A^T S x over the owned unknowns (S = diag(1, 1, sp): sp = -1 flips the
// pressure block, 1 gives plain A^T); every other entry of y is set to zero
__global__ void k_adj_apply_t(Geo g, long n, const double* val, const double* x, double* y, double sp,
                              const int* active, unsigned long long* matvecs) {
  if (active && !*active) return;
  FUGU_BOX_IJ
  if (matvecs && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0 && threadIdx.y == 0) ++*matvecs;
  for (int cc = 0; cc < 3; ++cc) {
    const long e = cc * n + g.at(i, j);
    if (!adj_owned(g, cc, i, j)) {
      y[e] = 0.0;
      continue;
    }
    double s = 0.0;
    for (int cr = 0; cr < 3; ++cr) {
      const double sr = cr == 2 ? sp : 1.0;
      for (int di = -2; di <= 2; ++di) {
        const int ir = adj_wrap(i - di, g.nx, g.px);
        for (int dj = -2; dj <= 2; ++dj) {
          const int jr = adj_wrap(j - dj, g.ny, g.py);
          if (!adj_owned(g, cr, ir, jr)) continue;
          const long q = g.at(ir, jr);
          s += val[(long)((cr * 3 + cc) * 25 + (di + 2) * 5 + (dj + 2)) * n + q] * (sr * x[cr * n + q]);
        }
      }
    }
    y[e] = (cc == 2 ? sp : 1.0) * s;
  }
}

// negate the pressure block of a triple (applies S)
__global__ void k_adj_flip_p(long n, double* x) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x)
    x[2 * n + q] = -x[2 * n + q];
}

}  // namespace fugu
