// pcg_cluster.cuh -- the PCG pressure Poisson solve of the PCD preconditioner
// (solve_poisson_pressure, mod_subsolvers.f90:32-246) resident in ONE
// thread-block cluster.
//
// The grid-wide persistent kernel (persistent.cuh) pays a global-memory
// barrier per reduction (~2.5-3 us on a B200 at 16-148 CTAs).  A cluster of
// up to 16 CTAs synchronises with the hardware cluster barrier and reduces
// through distributed shared memory (~0.4 us per barrier), so whenever a
// case fits, the whole solve lives in the cluster:
//
//   CTA r owns cell rows [j0, j0+R).  Thread t owns column i = t % nx + 1 and
//   a contiguous strip of CPT rows; its cells' phi, r, z, p and A p live in
//   registers.  Shared memory holds p_k of the CTA (for the east/west and
//   strip-end neighbours), the face coefficients cx (rows x (nx+1)),
//   cy ((rows+1) x nx) and dinv, and four halo rows: z and p of the row just
//   above and just below the CTA, pushed there by the neighbouring CTAs
//   (st.shared::cluster through mapped pointers; periodic y wraps rank 0 and
//   rank C-1).  p_k = z + beta p_{k-1} is formed once per cell; at a CTA
//   boundary it is formed from the halo z and p, which gives the same bits as
//   the owner's value.
//
// Lean variant (CPT = 32, FP32 only; grids of up to 16 x 512 cells per
// column strip, such as 320 x 640): five register arrays of 32 cells do not
// fit, so z is recomputed from r (z = dinv r, the same operation and bits)
// and p_k is read back from the shared-memory copy the CTA keeps anyway;
// phi, r and A p stay in registers.
//
// Arithmetic and reductions of the FP64 instantiation are those of k_pcg
// and the oracle (error-free DD sums merged in rank order), so results are
// bit-exact.  The FP32 instantiation (mixed-precision inner solve) sums its
// exact float products in double in a fixed order.  There is no software
// spin-wait: every wait is a hardware cluster barrier, and all CTAs execute
// the same sequence of barriers because every branch uses cluster-reduced
// values.
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
  int timed;     // the launch is timed: add its iterations to out->timed_iters
};

// the FP32 instantiations with strips of up to 16 cells run the
// single-reduction iteration (pcg_cluster_body_1r below)
template <typename T>
__host__ __device__ constexpr bool pcgc_one_reduction(int cpt) {
  return sizeof(T) == 4 && cpt <= 16;
}
// shared-memory footprint in elements of T for rows_per rows of nx cells:
// p_k (or u) of the CTA's cells, the halo rows (4 of them, or 12 halo rows
// and the inverse diagonal of the 2 halo rows in the single-reduction
// form), cx, cy and dinv
template <typename T>
__host__ __device__ inline long pcgc_smem_elems(int nx, int rows_per, int cpt) {
  const long halo = pcgc_one_reduction<T>(cpt) ? 14L * nx : 4L * nx;
  return (long)rows_per * nx + halo + (long)rows_per * (nx + 1) + (long)(rows_per + 1) * nx + (long)rows_per * nx;
}

// reduction accumulator: error-free DD for the FP64 parity path, plain
// double (exact float products, fixed order) for the FP32 inner solve
template <typename T>
struct RAcc {
  DD v{0.0, 0.0};
  __device__ __forceinline__ void add(double x) {
    if constexpr (sizeof(T) == 8) dd_add(v, x);
    else v.hi += x;
  }
};

template <typename T, int CPT>
__device__ __forceinline__ void pcg_cluster_body(const PcgClusterArgs<T>& a) {
  constexpr bool LEAN = CPT > 16;
  static_assert(!LEAN || sizeof(T) == 4, "the lean variant is FP32 only");
  cgc::cluster_group cl = cgc::this_cluster();
  const int C = (int)cl.num_blocks();
  const int rank = (int)cl.block_rank();
  const Geo g = a.g;
  const int nx = g.nx, ny = g.ny, rp = a.rows_per;
  const int j0 = 1 + rank * rp;
  const int R = min(rp, ny - rank * rp);  // rows of this CTA (>= 1)
  const bool closed = !g.px && !g.py;
  const int S = (R + CPT - 1) / CPT;       // strips per column
  const int t = threadIdx.x;
  const bool act = t < nx * S;
  const int i = act ? t % nx + 1 : 1;
  const int lr0 = act ? (t / nx) * CPT : 0;
  const int nr = act ? min(CPT, R - lr0) : 0;
  const int ie = (i < nx) ? i + 1 : (g.px ? 1 : nx);
  const int iw = (i > 1) ? i - 1 : (g.px ? nx : 1);

  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* pcs = reinterpret_cast<T*>(smem_raw);  // p_k of the CTA's cells, rp x nx
  T* zt = pcs + rp * nx;                     // z of the row above the CTA
  T* zb = zt + nx;                           // z of the row below
  T* pt = zb + nx;                           // p of the row above
  T* pb = pt + nx;                           // p of the row below
  T* cxs = pb + nx;
  T* cys = cxs + rp * (nx + 1);
  T* dis = cys + (rp + 1) * nx;
  __shared__ DD sh[32];
  __shared__ DD red[6];  // 0 pAp, 1 rr, 2 rz, 3 sum / mean, 4 rhs norm, 5 initial rz

  // cluster sum: block sum -> own slot -> barrier -> every CTA merges the C
  // slots in rank order (identical everywhere)
  auto bsum = [&](RAcc<T> acc) -> DD {
    if constexpr (sizeof(T) == 8) {
      return block_sum_dd(acc.v, sh);
    } else {
      DD r;
      r.hi = block_sum(acc.v.hi, reinterpret_cast<double*>(sh));
      r.lo = 0.0;
      return r;
    }
  };
  // two block sums in one interleaved pass (results into slots da, db)
  __shared__ DD sh2[32];
  auto bsum2 = [&](RAcc<T> a1, RAcc<T> a2, DD& da, DD& db) {
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
    DD v = a1.v, u = a2.v;
    if constexpr (sizeof(T) == 8) {
      for (int o = 16; o > 0; o >>= 1) {
        v = dd_merge(v, dd_shfl_down(v, o));
        u = dd_merge(u, dd_shfl_down(u, o));
      }
    } else {
      for (int o = 16; o > 0; o >>= 1) {
        v.hi += __shfl_down_sync(0xffffffffu, v.hi, o);
        u.hi += __shfl_down_sync(0xffffffffu, u.hi, o);
      }
    }
    __syncthreads();
    if (l == 0) {
      sh[w] = v;
      sh2[w] = u;
    }
    __syncthreads();
    if (w == 0) {
      v = l < nw ? sh[l] : DD{0.0, 0.0};
      u = l < nw ? sh2[l] : DD{0.0, 0.0};
      if constexpr (sizeof(T) == 8) {
        for (int o = 16; o > 0; o >>= 1) {
          v = dd_merge(v, dd_shfl_down(v, o));
          u = dd_merge(u, dd_shfl_down(u, o));
        }
      } else {
        for (int o = 16; o > 0; o >>= 1) {
          v.hi += __shfl_down_sync(0xffffffffu, v.hi, o);
          u.hi += __shfl_down_sync(0xffffffffu, u.hi, o);
        }
      }
      if (l == 0) {
        da = v;
        db = u;
      }
    }
  };
  // merge the C slots after a cluster barrier: lane r of warp 0 loads rank
  // r's slot (one DSMEM round trip for all ranks), a fixed shuffle tree sums
  // them, and the result is broadcast through shared memory.  Two slots can
  // be merged in the same pass (slot2 < 0: one).
  __shared__ double bcast[2];
  auto merge2 = [&](int slot, int slot2) {
    if (threadIdx.x < 32) {
      const int l = threadIdx.x;
      DD v{0.0, 0.0}, w{0.0, 0.0};
      if (l < C) {
        v = *cl.map_shared_rank(&red[slot], l);
        if (slot2 >= 0) w = *cl.map_shared_rank(&red[slot2], l);
      }
      if constexpr (sizeof(T) == 8) {
        for (int o = 16; o > 0; o >>= 1) {
          v = dd_merge(v, dd_shfl_down(v, o));
          if (slot2 >= 0) w = dd_merge(w, dd_shfl_down(w, o));
        }
        if (l == 0) {
          bcast[0] = v.hi + v.lo;
          bcast[1] = w.hi + w.lo;
        }
      } else {
        double a0 = v.hi, a1 = w.hi;
        for (int o = 16; o > 0; o >>= 1) {
          a0 += __shfl_down_sync(0xffffffffu, a0, o);
          a1 += __shfl_down_sync(0xffffffffu, a1, o);
        }
        if (l == 0) {
          bcast[0] = a0;
          bcast[1] = a1;
        }
      }
    }
    __syncthreads();
  };
  auto csum = [&](RAcc<T> acc, int slot) -> double {
    const DD v = bsum(acc);
    if (threadIdx.x == 0) red[slot] = v;
    cl.sync();
    merge2(slot, -1);
    return bcast[0];
  };
  // owners of the CTA's first / last row publish z and p into the halo rows
  // of the neighbouring CTAs (the row above CTA r-1 is my first row, the row
  // below CTA r+1 is my last row)
  auto push = [&](int c, T zv, T pv) {
    const int lr = lr0 + c;
    if (lr == 0 && (rank > 0 || g.py)) {
      const int dst = (rank - 1 + C) % C;
      cl.map_shared_rank(zt, dst)[i - 1] = zv;
      cl.map_shared_rank(pt, dst)[i - 1] = pv;
    }
    if (lr == R - 1 && (rank < C - 1 || g.py)) {
      const int dst = (rank + 1) % C;
      cl.map_shared_rank(zb, dst)[i - 1] = zv;
      cl.map_shared_rank(pb, dst)[i - 1] = pv;
    }
  };

  // ---- coefficients of the own rows
  for (int q = threadIdx.x; q < R * (nx + 1); q += blockDim.x) {
    const int lr = q / (nx + 1), ii = q % (nx + 1);
    cxs[lr * (nx + 1) + ii] = a.cx[g.at(ii, j0 + lr)];
  }
  for (int q = threadIdx.x; q < (R + 1) * nx; q += blockDim.x) {
    const int lf = q / nx - 1, ii = q % nx + 1;  // face rows j0-1 .. j0+R-1
    cys[(lf + 1) * nx + (ii - 1)] = a.cy[g.at(ii, j0 + lf)];
  }
  for (int q = threadIdx.x; q < R * nx; q += blockDim.x) dis[q] = a.dinv[g.at(q % nx + 1, j0 + q / nx)];

  T phi_r[CPT], r_r[CPT], ap_r[CPT];
  T z_r[LEAN ? 1 : CPT], p_r[LEAN ? 1 : CPT];  // (the lean variant does not use them)
  // z and p_k of own cell c (local row lr): registers, or (lean) recomputed / from pcs
#define PCGC_Z(c, lr) (LEAN ? dis[(lr) * nx + (i - 1)] * r_r[c] : z_r[LEAN ? 0 : (c)])
#define PCGC_P(c, lr) (LEAN ? pcs[(lr) * nx + (i - 1)] : p_r[LEAN ? 0 : (c)])
#define PCGC_CELLS _Pragma("unroll") for (int c = 0; c < CPT; ++c)
#define PCGC_CELL             \
  if (c >= nr) continue;      \
  const int lr = lr0 + c;     \
  const int j = j0 + lr;      \
  (void)j;

  // ---- (b) zero-mean projection and rhs norm
  double mean = 0.0;
  if (closed) {
    RAcc<T> s;
    PCGC_CELLS { PCGC_CELL s.add(double(a.rhs[g.at(i, j)])); }
    mean = csum(s, 3) / (double)(nx * ny);
  }
  RAcc<T> ss;
  PCGC_CELLS {
    PCGC_CELL
    const T rw = closed ? T(double(a.rhs[g.at(i, j)]) - mean) : a.rhs[g.at(i, j)];
    r_r[c] = rw;
    ss.add(double(rw) * double(rw));
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

  // ---- (c) phi ghosts (halo + Neumann), initial residual, z, p_1 = z
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
  __syncthreads();  // coefficients in shared memory
  RAcc<T> rz;
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
    if constexpr (!LEAN) {
      z_r[c] = zz;
      p_r[c] = zz;
    }
    push(c, zz, zz);
    rz.add(double(rr) * double(zz));
  }
  double rz_old = csum(rz, 5);  // its barrier also publishes the halos

  double res_norm = 0.0, beta = 0.0;
  int iter;
  for (iter = 1; iter <= a.max_iter; ++iter) {
    const T tb = T(beta);
    // phase A: p_k of the own cells, then A p_k
    PCGC_CELLS {
      PCGC_CELL
      const T zk = PCGC_Z(c, lr);
      const T pk = (iter == 1) ? zk : madd(tb, PCGC_P(c, lr), zk);
      if constexpr (!LEAN) p_r[c] = pk;
      pcs[lr * nx + (i - 1)] = pk;
    }
    __syncthreads();
    RAcc<T> papd;
    PCGC_CELLS {
      PCGC_CELL
      const T pk = PCGC_P(c, lr);
      const T cE = cxs[lr * (nx + 1) + i], cW = cxs[lr * (nx + 1) + i - 1];
      const T cN = cys[(lr + 1) * nx + (i - 1)], cS = cys[lr * nx + (i - 1)];
      const T pE = pcs[lr * nx + (ie - 1)], pW = pcs[lr * nx + (iw - 1)];
      T pN, pS;
      if (j == ny && !g.py) pN = pk;
      else if (c + 1 < nr) pN = PCGC_P(c + 1, lr + 1);
      else if (lr + 1 < R) pN = pcs[(lr + 1) * nx + (i - 1)];
      else pN = (iter == 1) ? zt[i - 1] : madd(tb, pt[i - 1], zt[i - 1]);
      if (j == 1 && !g.py) pS = pk;
      else if (c > 0) pS = PCGC_P(c - 1, lr - 1);
      else if (lr > 0) pS = pcs[(lr - 1) * nx + (i - 1)];
      else pS = (iter == 1) ? zb[i - 1] : madd(tb, pb[i - 1], zb[i - 1]);
      // (cE + cW + cN + cS) pk - (((cE pE + cW pW) + cN pN) + cS pS)
      const T off = madd(cS, pS, madd(cN, pN, madd(cW, pW, cE * pE)));
      const T apv = madd(cE + cW + cN + cS, pk, -off);
      ap_r[c] = apv;
      papd.add(double(pk) * double(apv));
    }
    const double pap = csum(papd, 0);  // barrier: every CTA is done reading pcs / halos
    if (fabs(pap) < 1.0e-30) break;
    const double alpha = rz_old / pap;
    const T ta = T(alpha);
    // phase B: phi, r, z updates; publish the boundary rows' z and p_k
    RAcc<T> rrd, rzd;
    PCGC_CELLS {
      PCGC_CELL
      const T rv = madd(-ta, ap_r[c], r_r[c]);
      const T zv = dis[lr * nx + (i - 1)] * rv;
      const T pk = PCGC_P(c, lr);
      phi_r[c] = madd(ta, pk, phi_r[c]);
      r_r[c] = rv;
      if constexpr (!LEAN) z_r[c] = zv;
      push(c, zv, pk);
      rrd.add(double(rv) * double(rv));
      rzd.add(double(rv) * double(zv));
    }
    bsum2(rrd, rzd, red[1], red[2]);
    cl.sync();
    merge2(1, 2);
    res_norm = sqrt(bcast[0]);
    if (res_norm / rhs_norm < a.tol) break;
    const double rz_new = bcast[1];
    beta = rz_new / rz_old;
    rz_old = rz_new;
  }
  if (closed) {
    RAcc<T> s;
    PCGC_CELLS { PCGC_CELL s.add(double(phi_r[c])); }
    const double m = csum(s, 3) / (double)(nx * ny);
    PCGC_CELLS { PCGC_CELL phi_r[c] = T(double(phi_r[c]) - m); }
  }
  PCGC_CELLS { PCGC_CELL a.phi[g.at(i, j)] = phi_r[c]; }
  if (rank == 0 && threadIdx.x == 0) {
    const int it = iter < a.max_iter ? iter : a.max_iter;
    a.out->iters = it;
    a.out->res = res_norm / rhs_norm;
    a.out->total_iters += (unsigned long long)it;
    if (a.timed) a.out->timed_iters += (unsigned long long)it;
    a.out->calls += 1;
  }
  cl.sync();  // no CTA leaves while another may still read its shared memory
#undef PCGC_CELLS
#undef PCGC_CELL
#undef PCGC_Z
#undef PCGC_P
}
// The FP32 inner solve's PCG with one cluster-wide reduction per iteration
// (the Chronopoulos-Gear arrangement of preconditioned CG; the FP64 parity
// path keeps the reference's recurrence above).  With u = M^-1 r, w = A u and
// s = A p carried as vectors, the three dot products an iteration needs,
// (r, u), (w, u) and (r, r), are formed in one pass and merged at one
// cluster barrier:
//   beta = gamma / gamma_old,  alpha = gamma / (delta - beta gamma / alpha_old)
//   p = u + beta p,  s = w + beta s,  phi += alpha p,  r -= alpha s,
//   u = M^-1 r,  w = A u,  gamma = (r, u),  delta = (w, u)
// The stencil of w = A u needs u of the rows just above and below the CTA.
// Instead of a second barrier to exchange them, the owners of a CTA's first
// and last rows push r, s and w of those rows into the neighbours' halo
// buffers before the barrier, and each neighbour forms the new s, r and u of
// the halo row itself with the owner's expressions (the same bits).  The
// halo buffers alternate between two sets by iteration, since a neighbour
// may push the next iteration's rows while this CTA still reads the
// current ones; so do the reduction slots.  Each iteration keeps phi, r, u,
// w, p and s of the thread's cells in registers and u of the CTA's cells in
// shared memory.  The same dot products and stopping test as the classic
// form: the solve stops when |r| / |rhs| < tol after an update.
template <int CPT>
__device__ __forceinline__ void pcg_cluster_body_1r(const PcgClusterArgs<float>& a) {
  using T = float;
  cgc::cluster_group cl = cgc::this_cluster();
  const int C = (int)cl.num_blocks();
  const int rank = (int)cl.block_rank();
  const Geo g = a.g;
  const int nx = g.nx, ny = g.ny, rp = a.rows_per;
  const int j0 = 1 + rank * rp;
  const int R = min(rp, ny - rank * rp);
  const bool closed = !g.px && !g.py;
  const int S = (R + CPT - 1) / CPT;
  const int t = threadIdx.x;
  const bool act = t < nx * S;
  const int i = act ? t % nx + 1 : 1;
  const int lr0 = act ? (t / nx) * CPT : 0;
  const int nr = act ? min(CPT, R - lr0) : 0;
  const int ie = (i < nx) ? i + 1 : (g.px ? 1 : nx);
  const int iw = (i > 1) ? i - 1 : (g.px ? nx : 1);
  const bool has_bot = rank > 0 || g.py, has_top = rank < C - 1 || g.py;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* uc = reinterpret_cast<T*>(smem_raw);  // u of own cells, rp x nx
  T* hb = uc + rp * nx;                      // [parity][r,s,w][bottom,top][nx]
  T* dh = hb + 12 * nx;                      // dinv of [bottom, top] halo rows
  T* cxs = dh + 2 * nx;
  T* cys = cxs + rp * (nx + 1);
  T* dis = cys + (rp + 1) * nx;
#define HB(par, f, side) (hb + (((par) * 3 + (f)) * 2 + (side)) * nx)
  __shared__ DD sh[32];
  __shared__ DD sh2[32];
  __shared__ DD sh3[32];
  __shared__ DD red[8];
  __shared__ double bcast[3];

  auto bsum = [&](RAcc<T> acc) -> DD {
    DD r;
    r.hi = block_sum(acc.v.hi, reinterpret_cast<double*>(sh));
    r.lo = 0.0;
    return r;
  };
  // three block sums in one pass, into red[s0..s0+2]
  auto bsum3 = [&](double x0, double x1, double x2, int s0) {
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int o = 16; o > 0; o >>= 1) {
      x0 += __shfl_down_sync(0xffffffffu, x0, o);
      x1 += __shfl_down_sync(0xffffffffu, x1, o);
      x2 += __shfl_down_sync(0xffffffffu, x2, o);
    }
    __syncthreads();
    if (l == 0) {
      sh[w].hi = x0;
      sh2[w].hi = x1;
      sh3[w].hi = x2;
    }
    __syncthreads();
    if (w == 0) {
      x0 = l < nw ? sh[l].hi : 0.0;
      x1 = l < nw ? sh2[l].hi : 0.0;
      x2 = l < nw ? sh3[l].hi : 0.0;
      for (int o = 16; o > 0; o >>= 1) {
        x0 += __shfl_down_sync(0xffffffffu, x0, o);
        x1 += __shfl_down_sync(0xffffffffu, x1, o);
        x2 += __shfl_down_sync(0xffffffffu, x2, o);
      }
      if (l == 0) {
        red[s0] = DD{x0, 0.0};
        red[s0 + 1] = DD{x1, 0.0};
        red[s0 + 2] = DD{x2, 0.0};
      }
    }
  };
  // merge the C ranks' slots s0..s0+n-1 (after a cluster barrier) into bcast
  auto merge = [&](int s0, int n) {
    if (threadIdx.x < 32) {
      const int l = threadIdx.x;
      double v[3] = {0.0, 0.0, 0.0};
      if (l < C)
        for (int q = 0; q < n; ++q) v[q] = cl.map_shared_rank(&red[s0 + q], l)->hi;
      for (int o = 16; o > 0; o >>= 1)
        for (int q = 0; q < 3; ++q) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
      if (l == 0)
        for (int q = 0; q < n; ++q) bcast[q] = v[q];
    }
    __syncthreads();
  };
  auto csum = [&](RAcc<T> acc, int slot) -> double {
    const DD v = bsum(acc);
    if (threadIdx.x == 0) red[slot] = v;
    cl.sync();
    merge(slot, 1);
    return bcast[0];
  };
  // push r, s, w of a boundary cell into the neighbours' halo buffers (parity par)
  auto push = [&](int c, int par, T rv, T sv, T wv) {
    const int lr = lr0 + c;
    if (lr == 0 && has_bot) {  // my first row is the row above CTA rank-1
      const int dst = (rank - 1 + C) % C;
      cl.map_shared_rank(HB(par, 0, 1), dst)[i - 1] = rv;
      cl.map_shared_rank(HB(par, 1, 1), dst)[i - 1] = sv;
      cl.map_shared_rank(HB(par, 2, 1), dst)[i - 1] = wv;
    }
    if (lr == R - 1 && has_top) {  // my last row is the row below CTA rank+1
      const int dst = (rank + 1) % C;
      cl.map_shared_rank(HB(par, 0, 0), dst)[i - 1] = rv;
      cl.map_shared_rank(HB(par, 1, 0), dst)[i - 1] = sv;
      cl.map_shared_rank(HB(par, 2, 0), dst)[i - 1] = wv;
    }
  };

  // ---- coefficients of the own rows and dinv of the halo rows
  for (int q = threadIdx.x; q < R * (nx + 1); q += blockDim.x) {
    const int lr = q / (nx + 1), ii = q % (nx + 1);
    cxs[lr * (nx + 1) + ii] = a.cx[g.at(ii, j0 + lr)];
  }
  for (int q = threadIdx.x; q < (R + 1) * nx; q += blockDim.x) {
    const int lf = q / nx - 1, ii = q % nx + 1;
    cys[(lf + 1) * nx + (ii - 1)] = a.cy[g.at(ii, j0 + lf)];
  }
  for (int q = threadIdx.x; q < R * nx; q += blockDim.x) dis[q] = a.dinv[g.at(q % nx + 1, j0 + q / nx)];
  for (int q = threadIdx.x; q < nx; q += blockDim.x) {
    const int jb = j0 - 1 >= 1 ? j0 - 1 : ny, jt = j0 + R <= ny ? j0 + R : 1;
    dh[q] = has_bot ? a.dinv[g.at(q + 1, jb)] : T(0);
    dh[nx + q] = has_top ? a.dinv[g.at(q + 1, jt)] : T(0);
  }

  T phi_r[CPT], r_r[CPT], u_r[CPT], w_r[CPT], p_r[CPT], s_r[CPT];
#define PCG1_CELLS _Pragma("unroll") for (int c = 0; c < CPT; ++c)
#define PCG1_CELL               \
  if (c >= nr) continue;      \
  const int lr = lr0 + c;     \
  const int j = j0 + lr;      \
  (void)j;

  double mean = 0.0;
  if (closed) {
    RAcc<T> s;
    PCG1_CELLS { PCG1_CELL s.add(double(a.rhs[g.at(i, j)])); }
    mean = csum(s, 3) / (double)(nx * ny);
  }
  RAcc<T> ss;
  PCG1_CELLS {
    PCG1_CELL
    const T rw = closed ? T(double(a.rhs[g.at(i, j)]) - mean) : a.rhs[g.at(i, j)];
    r_r[c] = rw;
    ss.add(double(rw) * double(rw));
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
  __syncthreads();
  // r0 = rhs_work - A phi0, u0 = dinv r0; p = s = 0
  PCG1_CELLS {
    PCG1_CELL
    T rr = r_r[c];
    T ph = T(0);
    if (!a.phi_zero) {
      const T* gp = a.phi;
      ph = gp[g.at(i, j)];
      const T apv = poisson_ap<T>(g, a.cx, a.cy, i, j, [&](int x, int y) { return gp[g.at(x, y)]; });
      rr = rr - apv;
    }
    phi_r[c] = ph;
    r_r[c] = rr;
    const T uu = dis[lr * nx + (i - 1)] * rr;
    u_r[c] = uu;
    uc[lr * nx + (i - 1)] = uu;
    p_r[c] = T(0);
    s_r[c] = T(0);
    push(c, 1, rr, T(0), T(0));  // r0 of the boundary rows (parity 1, read before barrier 0)
  }
  cl.sync();  // uc and the r0 halos are in place
  // halo u: u = dinv r (iteration 0: s and alpha are zero)
  auto halo_u = [&](int side, int par, T tb, T ta, bool first) -> T {
    const T* hr = HB(par, 0, side);
    const T* hs = HB(par, 1, side);
    const T* hw = HB(par, 2, side);
    if (first) return dh[side * nx + (i - 1)] * hr[i - 1];
    const T sv = madd(tb, hs[i - 1], hw[i - 1]);
    const T rv = madd(-ta, sv, hr[i - 1]);
    return dh[side * nx + (i - 1)] * rv;
  };
  // w = A u of own cell c, the south / north neighbours given
  auto apply = [&](int c, int lr, T us, T un) -> T {
    const T uk = u_r[c];
    const T cE = cxs[lr * (nx + 1) + i], cW = cxs[lr * (nx + 1) + i - 1];
    const T cN = cys[(lr + 1) * nx + (i - 1)], cS = cys[lr * nx + (i - 1)];
    const T uE = uc[lr * nx + (ie - 1)], uW = uc[lr * nx + (iw - 1)];
    const T off = madd(cS, us, madd(cN, un, madd(cW, uW, cE * uE)));
    return madd(cE + cW + cN + cS, uk, -off);
  };
  auto neighbours = [&](int c, int lr, int j, T hb_u, T ht_u, T& us, T& un) {
    const T uk = u_r[c];
    if (j == ny && !g.py) un = uk;
    else if (c + 1 < nr) un = u_r[c + 1];
    else if (lr + 1 < R) un = uc[(lr + 1) * nx + (i - 1)];
    else un = ht_u;
    if (j == 1 && !g.py) us = uk;
    else if (c > 0) us = u_r[c - 1];
    else if (lr > 0) us = uc[(lr - 1) * nx + (i - 1)];
    else us = hb_u;
  };
  double gam, del, rr;
  {
    const T hbu = (lr0 == 0 && has_bot) ? halo_u(0, 1, T(0), T(0), true) : T(0);
    const T htu = (act && lr0 + nr == R && has_top) ? halo_u(1, 1, T(0), T(0), true) : T(0);
    double x0 = 0.0, x1 = 0.0, x2 = 0.0;
    PCG1_CELLS {
      PCG1_CELL
      T us, un;
      neighbours(c, lr, j, hbu, htu, us, un);
      const T wv = apply(c, lr, us, un);
      w_r[c] = wv;
      x0 += double(r_r[c]) * double(u_r[c]);
      x1 += double(wv) * double(u_r[c]);
      x2 += double(r_r[c]) * double(r_r[c]);
      push(c, 0, r_r[c], s_r[c], wv);
    }
    bsum3(x0, x1, x2, 0);
    cl.sync();
    merge(0, 3);
    gam = bcast[0];
    del = bcast[1];
    rr = bcast[2];
  }
  double res_norm = sqrt(rr), alpha = 0.0, beta = 0.0, gam_old = 0.0;
  int iter;
  for (iter = 1; iter <= a.max_iter; ++iter) {
    if (iter == 1) {
      beta = 0.0;
      if (fabs(del) < 1.0e-30) break;
      alpha = gam / del;
    } else {
      beta = gam / gam_old;
      const double den = del - beta * gam / alpha;
      if (fabs(den) < 1.0e-30) break;
      alpha = gam / den;
    }
    const T tb = T(beta), ta = T(alpha);
    const int par = (iter - 1) & 1;  // buffers written at the end of the previous step
    PCG1_CELLS {
      PCG1_CELL
      const T pk = madd(tb, p_r[c], u_r[c]);
      const T sk = madd(tb, s_r[c], w_r[c]);
      phi_r[c] = madd(ta, pk, phi_r[c]);
      const T rv = madd(-ta, sk, r_r[c]);
      const T uv = dis[lr * nx + (i - 1)] * rv;
      p_r[c] = pk;
      s_r[c] = sk;
      r_r[c] = rv;
      u_r[c] = uv;
      uc[lr * nx + (i - 1)] = uv;
    }
    const T hbu = (lr0 == 0 && has_bot) ? halo_u(0, par, tb, ta, false) : T(0);
    const T htu = (act && lr0 + nr == R && has_top) ? halo_u(1, par, tb, ta, false) : T(0);
    __syncthreads();
    double x0 = 0.0, x1 = 0.0, x2 = 0.0;
    PCG1_CELLS {
      PCG1_CELL
      T us, un;
      neighbours(c, lr, j, hbu, htu, us, un);
      const T wv = apply(c, lr, us, un);
      w_r[c] = wv;
      x0 += double(r_r[c]) * double(u_r[c]);
      x1 += double(wv) * double(u_r[c]);
      x2 += double(r_r[c]) * double(r_r[c]);
      push(c, iter & 1, r_r[c], s_r[c], wv);
    }
    bsum3(x0, x1, x2, (iter & 1) ? 3 : 0);
    cl.sync();
    merge((iter & 1) ? 3 : 0, 3);
    gam_old = gam;
    gam = bcast[0];
    del = bcast[1];
    res_norm = sqrt(bcast[2]);
    if (res_norm / rhs_norm < a.tol) break;
  }
  if (closed) {
    RAcc<T> s;
    PCG1_CELLS { PCG1_CELL s.add(double(phi_r[c])); }
    const double m = csum(s, 6) / (double)(nx * ny);
    PCG1_CELLS { PCG1_CELL phi_r[c] = T(double(phi_r[c]) - m); }
  }
  PCG1_CELLS { PCG1_CELL a.phi[g.at(i, j)] = phi_r[c]; }
  if (rank == 0 && threadIdx.x == 0) {
    const int it = iter < a.max_iter ? iter : a.max_iter;
    a.out->iters = it;
    a.out->res = res_norm / rhs_norm;
    a.out->total_iters += (unsigned long long)it;
    if (a.timed) a.out->timed_iters += (unsigned long long)it;
    a.out->calls += 1;
  }
  cl.sync();
#undef PCG1_CELLS
#undef PCG1_CELL
#undef HB
}
template <typename T, int CPT>
__global__ void __launch_bounds__(PCGC_TPB, 1) k_pcg_cluster(PcgClusterArgs<T> a) {
  if (a.active && !*a.active) return;
  if constexpr (pcgc_one_reduction<T>(CPT)) pcg_cluster_body_1r<CPT>(a);
  else pcg_cluster_body<T, CPT>(a);
}

}  // namespace fugu
