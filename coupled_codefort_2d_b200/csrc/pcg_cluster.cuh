// pcg_cluster.cuh -- the PCG pressure Poisson solve of the PCD preconditioner
// (solve_poisson_pressure, mod_subsolvers.f90:32-246) resident in ONE
// thread-block cluster.
//
// The grid-wide persistent kernel (persistent.cuh) pays a global-memory
// barrier per reduction (~2.5-3 us on a B200 at 16-148 CTAs).  A cluster of
// up to 16 CTAs synchronises with the hardware cluster barrier and reduces
// through distributed shared memory (~0.4 us per barrier), so whenever a
// case fits, the whole solve lives in the cluster's shared memory:
//
//   CTA r owns cell rows [j0, j0+R) of all nx columns.  Shared memory holds z
//   and two p buffers with one halo row above and below, the face
//   coefficients cx (rows x (nx+1)), cy ((rows+1) x nx) and dinv; phi, r and
//   A p of the CTA's cells live in registers (CPT cells per thread).
//   After every update a CTA pushes its first and last rows of z and p into
//   the halo rows of its neighbours' shared memory (st.shared::cluster via
//   mapped pointers; periodic y wraps rank 0 <-> rank C-1).
//
// Arithmetic is identical to k_pcg and the oracle (same expressions, same
// error-free DD reductions, merged in rank order), so results are bit-exact.
// There is no software spin-wait: every wait is a hardware cluster barrier,
// and every CTA executes the same sequence of barriers because all branch
// decisions use cluster-reduced values.
#pragma once

#include <cooperative_groups.h>

#include "fugu_internal.cuh"
#include "persistent.cuh"

namespace fugu {

namespace cgc = cooperative_groups;

constexpr int PCGC_TPB = 512;

template <typename T>
struct PcgClusterArgs {
  Geo g;
  const T* rhs;
  const T* cx;
  const T* cy;
  const T* dinv;
  T* phi;
  PcgOut* out;
  const int* active;
  double tol;
  int max_iter;
  int phi_zero;
  int rows_per;  // rows of every CTA but possibly the last
};

// shared-memory footprint in elements of T for rows_per rows of nx cells
__host__ __device__ inline long pcgc_smem_elems(int nx, int rows_per) {
  return 3L * (rows_per + 2) * nx + (long)rows_per * (nx + 1) + (long)(rows_per + 1) * nx + (long)rows_per * nx;
}

template <typename T, int CPT>
__global__ void __launch_bounds__(PCGC_TPB, 1) k_pcg_cluster(PcgClusterArgs<T> a) {
  if (a.active && !*a.active) return;
  cgc::cluster_group cl = cgc::this_cluster();
  const int C = (int)cl.num_blocks();
  const int rank = (int)cl.block_rank();
  const Geo g = a.g;
  const int nx = g.nx, ny = g.ny, rp = a.rows_per;
  const int j0 = 1 + rank * rp;
  const int R = min(rp, ny - rank * rp);  // rows of this CTA (>= 1)
  const bool closed = !g.px && !g.py;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* zs = reinterpret_cast<T*>(smem_raw);
  T* ps0 = zs + (rp + 2) * nx;
  T* ps1 = ps0 + (rp + 2) * nx;
  T* cxs = ps1 + (rp + 2) * nx;
  T* cys = cxs + rp * (nx + 1);
  T* dis = cys + (rp + 1) * nx;
  __shared__ DD sh[32];
  __shared__ DD red[6];  // 0 pAp, 1 rr, 2 rz, 3 sum / mean, 4 rhs norm, 5 initial rz

  auto zi = [&](int lr, int i) { return (lr + 1) * nx + (i - 1); };  // lr in [-1, R]

  // cluster sum of one DD per thread: block sum -> own slot -> barrier ->
  // every CTA merges the C slots in rank order (identical everywhere)
  auto csum = [&](DD v, int slot) -> double {
    v = block_sum_dd(v, sh);
    if (threadIdx.x == 0) red[slot] = v;
    cl.sync();
    DD t{0.0, 0.0};
    for (int r = 0; r < C; ++r) t = dd_merge(t, *cl.map_shared_rank(&red[slot], r));
    return t.hi + t.lo;
  };
  // push first / last own row of buf (z or a p buffer) into the neighbours' halos
  auto push_halos = [&](T* buf) {
    if (rank > 0 || g.py) {
      const int dst = (rank - 1 + C) % C;
      const int Rd = min(rp, ny - dst * rp);
      T* rem = cl.map_shared_rank(buf, dst);
      for (int i = 1 + threadIdx.x; i <= nx; i += blockDim.x) rem[(Rd + 1) * nx + (i - 1)] = buf[zi(0, i)];
    }
    if (rank < C - 1 || g.py) {
      const int dst = (rank + 1) % C;
      T* rem = cl.map_shared_rank(buf, dst);
      for (int i = 1 + threadIdx.x; i <= nx; i += blockDim.x) rem[i - 1] = buf[zi(R - 1, i)];
    }
  };

  // ---- load coefficients of the own rows
  for (int q = threadIdx.x; q < R * (nx + 1); q += blockDim.x) {
    const int lr = q / (nx + 1), i = q % (nx + 1);
    cxs[lr * (nx + 1) + i] = a.cx[g.at(i, j0 + lr)];
  }
  for (int q = threadIdx.x; q < (R + 1) * nx; q += blockDim.x) {
    const int lf = q / nx - 1, i = q % nx + 1;  // face rows j0-1 .. j0+R-1
    cys[(lf + 1) * nx + (i - 1)] = a.cy[g.at(i, j0 + lf)];
  }
  for (int q = threadIdx.x; q < R * nx; q += blockDim.x) dis[q] = a.dinv[g.at(q % nx + 1, j0 + q / nx)];

  T phi_r[CPT], r_r[CPT], ap_r[CPT], p_r[CPT];
  const int ncell = R * nx;
#define PCGC_CELLS _Pragma("unroll") for (int c = 0; c < CPT; ++c)
#define PCGC_CELL                                        \
  const int q = threadIdx.x + c * PCGC_TPB;              \
  if (q >= ncell) continue;                              \
  const int lr = q / nx, i = q % nx + 1, j = j0 + lr;    \
  (void)j;

  // ---- (b) zero-mean projection and rhs norm
  double mean = 0.0;
  if (closed) {
    DD s{0.0, 0.0};
    PCGC_CELLS { PCGC_CELL dd_add(s, double(a.rhs[g.at(i, j)])); }
    mean = csum(s, 3) / (double)(nx * ny);
  }
  DD ss{0.0, 0.0};
  PCGC_CELLS {
    PCGC_CELL
    const T rw = closed ? T(double(a.rhs[g.at(i, j)]) - mean) : a.rhs[g.at(i, j)];
    r_r[c] = rw;
    dd_add(ss, double(rw) * double(rw));
  }
  const double rhs_norm = sqrt(csum(ss, 4));
  if (rhs_norm < 1.0e-14) {
    const long tot = g.n();
    for (long q = rank * (long)blockDim.x + threadIdx.x; q < tot; q += (long)C * blockDim.x) a.phi[q] = T(0);
    if (rank == 0 && threadIdx.x == 0) {
      a.out->iters = 0;
      a.out->res = 0.0;
      a.out->calls += 1;
    }
    cl.sync();
    return;
  }

  // ---- (c) phi ghosts (halo + Neumann), initial residual, z, p = z
  if (!a.phi_zero) {
    const long tot = g.n();
    for (long q = rank * (long)blockDim.x + threadIdx.x; q < tot; q += (long)C * blockDim.x) {
      const int gi = (int)(q % g.P) - 2, gj = (int)(q / g.P) - 2;
      if (gi < -1 || gj < -1 || gi > nx + 2 || gj > ny + 2) continue;
      if (gi >= 1 && gi <= nx && gj >= 1 && gj <= ny) continue;
      const int mi = (gi >= 1 && gi <= nx) ? gi : (g.px ? (gi < 1 ? gi + nx : gi - nx) : (gi < 1 ? 1 - gi : 2 * nx + 1 - gi));
      const int mj = (gj >= 1 && gj <= ny) ? gj : (g.py ? (gj < 1 ? gj + ny : gj - ny) : (gj < 1 ? 1 - gj : 2 * ny + 1 - gj));
      a.phi[q] = a.phi[g.at(mi, mj)];
    }
  }
  DD rz{0.0, 0.0};
  PCGC_CELLS {
    PCGC_CELL
    T rr = r_r[c];
    T ph = T(0);
    if (!a.phi_zero) {
      const T* gp = a.phi;
      ph = gp[g.at(i, j)];
      const T apv = poisson_ap<T>(g, a.cx, a.cy, i, j, [&](int x, int y) { return gp[g.at(x, y)]; });
      rr = rr - apv;
    }
    const T zz = dis[lr * nx + (i - 1)] * rr;
    phi_r[c] = ph;
    r_r[c] = rr;
    zs[zi(lr, i)] = zz;
    ps1[zi(lr, i)] = zz;  // p_1 = z lives in ps1 (odd iterations)
    dd_add(rz, double(rr) * double(zz));
  }
  __syncthreads();
  push_halos(zs);
  push_halos(ps1);
  double rz_old = csum(rz, 5);  // its barrier also publishes the halos

  // stencil at own cell (lr, i) on a field given by accessor f(lr', i')
  auto stencil = [&](int lr, int i, int j, auto f) -> T {
    const T cE = cxs[lr * (nx + 1) + i], cW = cxs[lr * (nx + 1) + i - 1];
    const T cN = cys[(lr + 1) * nx + (i - 1)], cS = cys[lr * nx + (i - 1)];
    const int ie = (i < nx) ? i + 1 : (g.px ? 1 : nx);
    const int iw = (i > 1) ? i - 1 : (g.px ? nx : 1);
    const int ln = (j == ny && !g.py) ? lr : lr + 1;
    const int ls = (j == 1 && !g.py) ? lr : lr - 1;
    return (cE + cW + cN + cS) * f(lr, i) - (cE * f(lr, ie) + cW * f(lr, iw) + cN * f(ln, i) + cS * f(ls, i));
  };

  double res_norm = 0.0, beta = 0.0;
  int iter;
  for (iter = 1; iter <= a.max_iter; ++iter) {
    T* pcur = (iter & 1) ? ps1 : ps0;
    const T* pprev = (iter & 1) ? ps0 : ps1;
    const T tb = T(beta);
    // phase A: p_k (on the fly) and A p_k
    DD papd{0.0, 0.0};
    PCGC_CELLS {
      PCGC_CELL
      T apv, pown;
      if (iter == 1) {
        pown = ps1[zi(lr, i)];
        apv = stencil(lr, i, j, [&](int l2, int i2) { return ps1[zi(l2, i2)]; });
      } else {
        auto pf = [&](int l2, int i2) {
          const int e = zi(l2, i2);
          return zs[e] + tb * pprev[e];
        };
        pown = pf(lr, i);
        apv = stencil(lr, i, j, pf);
      }
      p_r[c] = pown;
      ap_r[c] = apv;
      dd_add(papd, double(pown) * double(apv));
    }
    const double pap = csum(papd, 0);  // barrier: every CTA is done reading z / pprev
    if (fabs(pap) < 1.0e-30) break;
    const double alpha = rz_old / pap;
    const T ta = T(alpha);
    // phase B: phi, r, z updates; publish z and p_k rows
    DD rrd{0.0, 0.0}, rzd{0.0, 0.0};
    PCGC_CELLS {
      PCGC_CELL
      const T rv = r_r[c] - ta * ap_r[c];
      const T zv = dis[lr * nx + (i - 1)] * rv;
      phi_r[c] = phi_r[c] + ta * p_r[c];
      r_r[c] = rv;
      zs[zi(lr, i)] = zv;
      if (iter > 1) pcur[zi(lr, i)] = p_r[c];
      dd_add(rrd, double(rv) * double(rv));
      dd_add(rzd, double(rv) * double(zv));
    }
    __syncthreads();
    push_halos(zs);
    if (iter > 1) push_halos(pcur);
    rrd = block_sum_dd(rrd, sh);
    if (threadIdx.x == 0) red[1] = rrd;
    rzd = block_sum_dd(rzd, sh);
    if (threadIdx.x == 0) red[2] = rzd;
    cl.sync();
    DD trr{0.0, 0.0}, trz{0.0, 0.0};
    for (int r = 0; r < C; ++r) {
      trr = dd_merge(trr, *cl.map_shared_rank(&red[1], r));
      trz = dd_merge(trz, *cl.map_shared_rank(&red[2], r));
    }
    res_norm = sqrt(trr.hi + trr.lo);
    if (res_norm / rhs_norm < a.tol) break;
    const double rz_new = trz.hi + trz.lo;
    beta = rz_new / rz_old;
    rz_old = rz_new;
  }
  if (closed) {
    DD s{0.0, 0.0};
    PCGC_CELLS { PCGC_CELL dd_add(s, double(phi_r[c])); }
    const double m = csum(s, 3) / (double)(nx * ny);
    PCGC_CELLS { PCGC_CELL phi_r[c] = T(double(phi_r[c]) - m); }
  }
  PCGC_CELLS { PCGC_CELL a.phi[g.at(i, j)] = phi_r[c]; }
  if (rank == 0 && threadIdx.x == 0) {
    const int it = iter < a.max_iter ? iter : a.max_iter;
    a.out->iters = it;
    a.out->res = res_norm / rhs_norm;
    a.out->total_iters += (unsigned long long)it;
    a.out->calls += 1;
  }
  cl.sync();  // no CTA leaves while another may still read its shared memory
#undef PCGC_CELLS
#undef PCGC_CELL
}

}  // namespace fugu
