// persistent.cuh -- persistent (cooperative) kernels: the Jacobi-PCG pressure
// Poisson solve and the SVOF Helmholtz filter.  One launch runs every
// iteration; CTAs meet at bounded grid barriers (fugu_internal.cuh), the
// convergence tests are evaluated identically by every CTA from the same
// deterministic reductions, so no host round trip is needed per iteration.
#pragma once

#include "fugu_internal.cuh"

namespace fugu {

struct PcgOut {
  int iters;            // iter_out of the last solve
  int status;           // 0 ok, 1 barrier timeout
  double res;           // res_out of the last solve
  unsigned long long total_iters;  // accumulated over solves (statistics)
  unsigned long long calls;
  unsigned long long timed_iters;  // accumulated over the launches with timed = 1
};

// A thread's walk over the interior cells q = tid, tid + nthr, ... with
// q = (i - 1) + (j - 1) * nx, as (i, j) from the thread's first cell and
// the stride's (di, dj), advanced by carry: a cell costs two adds and a
// compare instead of a 64-bit division and remainder, and the cells and
// their order are those of the plain strided loop (q < nx * ny is j <= ny).
struct CellWalk {
  int i0, j0, di, dj;
  __device__ __forceinline__ CellWalk(long tid, long nthr, int nx)
      : i0(1 + (int)(tid % nx)), j0(1 + (int)(tid / nx)), di((int)(nthr % nx)), dj((int)(nthr / nx)) {}
  __device__ __forceinline__ void next(int& i, int& j, int nx) const {
    i += di;
    j += dj;
    if (i > nx) {
      i -= nx;
      ++j;
    }
  }
};

template <typename T>
struct PcgArgs {
  Geo g;
  const T* rhs;        // right-hand side (cell layout)
  const T* cx;         // u-face coefficients idx2/rho_u, zero on wall faces
  const T* cy;         // v-face coefficients idy2/rho_v, zero on wall faces
  const T* dinv;       // Jacobi inverse diagonal at cells
  T* phi;              // in: initial guess; out: solution (ghosts as the reference)
  T* r;                // work (interior)
  T* z;
  T* pb0;
  T* pb1;
  T* ap;
  double* part;        // 12 * gridDim.x partial sums (6 DD slots)
  GridSync* gs;
  PcgOut* out;
  const int* active;   // skip when *active == 0 (nullable)
  double tol;
  int max_iter;
  int phi_zero;        // phi is identically zero on entry (preconditioner use)
  int timed;           // the launch is timed: add its iterations to out->timed_iters
  // failure-detection test: each grid barrier waits for gridDim.x +
  // extra_arrivals CTAs (1 makes every wait run out) and gives up after
  // spin_limit polls (0: FUGU_SPIN_LIMIT).  Both 0 in normal use.
  unsigned int spin_limit;
  int extra_arrivals;
  T* w1;               // k_pcg1 only: the second w buffer and p (work)
  T* pv;
};

// the arrival count and poll limit of one grid-wide launch's barriers
struct Barrier {
  GridSync* gs;
  unsigned int nb;
  unsigned int lim;
  unsigned int gen;
};

// Grid-wide order-independent sum of one (or two) DD values per thread: CTA
// partials, one bounded grid barrier, then every CTA sums the partials in
// the same order.  Returns false when the barrier gave up.
__device__ __forceinline__ bool grid_allreduce(Barrier& bar, double* part, DD v, DD* sh, double& out) {
  v = block_sum_dd(v, sh);
  if (threadIdx.x == 0) put_partial(part, blockIdx.x, v);
  if (!grid_sync(bar.gs, bar.nb, bar.gen, bar.lim)) return false;
  out = sum_partials_dd(part, gridDim.x);
  return true;
}
__device__ __forceinline__ bool grid_allreduce2(Barrier& bar, double* pa, double* pb, DD a, DD b, DD* sh,
                                                double& oa, double& ob) {
  a = block_sum_dd(a, sh);
  if (threadIdx.x == 0) put_partial(pa, blockIdx.x, a);
  b = block_sum_dd(b, sh);
  if (threadIdx.x == 0) put_partial(pb, blockIdx.x, b);
  if (!grid_sync(bar.gs, bar.nb, bar.gen, bar.lim)) return false;
  sum_partials_dd2(pa, pb, gridDim.x, oa, ob);
  return true;
}

// three sums at one barrier (the single-reduction PCG)
__device__ __forceinline__ bool grid_allreduce3(Barrier& bar, double* pa, double* pb, double* pc, DD a, DD b, DD c,
                                                DD* sh, double* out) {
  a = block_sum_dd(a, sh);
  if (threadIdx.x == 0) put_partial(pa, blockIdx.x, a);
  b = block_sum_dd(b, sh);
  if (threadIdx.x == 0) put_partial(pb, blockIdx.x, b);
  c = block_sum_dd(c, sh);
  if (threadIdx.x == 0) put_partial(pc, blockIdx.x, c);
  if (!grid_sync(bar.gs, bar.nb, bar.gen, bar.lim)) return false;
  __shared__ double s_res3[3];
  if (threadIdx.x < 32) {
    const double* parts[3] = {pa, pb, pc};
    double r[3];
    merge_partials_dd<3>(parts, gridDim.x, r);
    if (threadIdx.x == 0) {
      s_res3[0] = r[0];
      s_res3[1] = r[1];
      s_res3[2] = r[2];
    }
  }
  __syncthreads();
  out[0] = s_res3[0];
  out[1] = s_res3[1];
  out[2] = s_res3[2];
  __syncthreads();
  return true;
}

// stencil of the variable-density Poisson operator at cell (i,j) applied to
// a field given by accessor f (mod_subsolvers.f90:142-144, :182-184)
template <typename T, typename F>
__device__ __forceinline__ T poisson_ap(const Geo& g, const T* cx, const T* cy, int i, int j, F f) {
  const T cE = __ldg(cx + g.at(i, j)), cW = __ldg(cx + g.at(i - 1, j));
  const T cN = __ldg(cy + g.at(i, j)), cS = __ldg(cy + g.at(i, j - 1));
  const int ie = (i < g.nx) ? i + 1 : (g.px ? 1 : g.nx);
  const int iw = (i > 1) ? i - 1 : (g.px ? g.nx : 1);
  const int jn = (j < g.ny) ? j + 1 : (g.py ? 1 : g.ny);
  const int js = (j > 1) ? j - 1 : (g.py ? g.ny : 1);
  return (cE + cW + cN + cS) * f(i, j) - (cE * f(ie, j) + cW * f(iw, j) + cN * f(i, jn) + cS * f(i, js));
}

// solve_poisson_pressure, mod_subsolvers.f90:32-246.
template <typename T>
__global__ void __launch_bounds__(512) k_pcg(PcgArgs<T> a) {
  if (a.active && !*a.active) return;
  __shared__ DD sh[32];
  const Geo g = a.g;
  const int G = gridDim.x;
  const long tid = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long nthr = (long)G * blockDim.x;
  const bool closed = !g.px && !g.py;
  Barrier bar{a.gs, (unsigned int)(G + a.extra_arrivals), a.spin_limit ? a.spin_limit : FUGU_SPIN_LIMIT, 0u};
  // a barrier that gave up: record it in the result (the host reads it as
  // FUGU_ETIMEOUT) and unwind; every CTA writes the same value
  auto gave_up = [&]() {
    if (threadIdx.x == 0) a.out->status = 1;
  };
  double* P0 = a.part;           // setup sum / final mean
  double* P1 = a.part + 2 * G;   // rhs norm
  double* P2 = a.part + 4 * G;   // initial r.z
  double* PA = a.part + 6 * G;   // p.Ap
  double* PB = a.part + 8 * G;   // r.r
  double* PC = a.part + 10 * G;  // r.z
  const CellWalk cw(tid, nthr, g.nx);
#define CELL_LOOP for (int i = cw.i0, j = cw.j0; j <= g.ny; cw.next(i, j, g.nx))
#define CELL_IJ const int c = g.at(i, j);

  // (b) zero-mean projection of the right-hand side when no direction is periodic
  double mean = 0.0;
  if (closed) {
    DD s{0.0, 0.0};
    CELL_LOOP { CELL_IJ dd_add(s, double(a.rhs[c])); }
    double tot;
    if (!grid_allreduce(bar, P0, s, sh, tot)) { gave_up(); return; }
    mean = tot / (double)(g.nx * g.ny);
  }
  DD ss{0.0, 0.0};
  CELL_LOOP {
    CELL_IJ
    const T rw = closed ? T(double(a.rhs[c]) - mean) : a.rhs[c];
    a.r[c] = rw;  // r holds rhs_work until the initial residual is formed
    dd_add(ss, double(rw) * double(rw));
  }
  double ssum;
  if (!grid_allreduce(bar, P1, ss, sh, ssum)) { gave_up(); return; }
  const double rhs_norm = sqrt(ssum);
  if (rhs_norm < 1.0e-14) {
    for (long q = tid; q < g.n(); q += nthr) a.phi[q] = T(0);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      a.out->iters = 0;
      a.out->res = 0.0;
      a.out->calls += 1;
    }
    return;
  }
  // (c) ghosts of phi from halo exchange + Neumann BC, then r = rhs_work - A phi
  if (!a.phi_zero) {
    for (long q = tid; q < g.n(); q += nthr) {
      const int i = (int)(q % g.P) - 2, j = (int)(q / g.P) - 2;
      if (i < -1 || j < -1 || i > g.nx + 2 || j > g.ny + 2) continue;
      if (i >= 1 && i <= g.nx && j >= 1 && j <= g.ny) continue;
      const int mi = (i >= 1 && i <= g.nx) ? i : (g.px ? (i < 1 ? i + g.nx : i - g.nx) : (i < 1 ? 1 - i : 2 * g.nx + 1 - i));
      const int mj = (j >= 1 && j <= g.ny) ? j : (g.py ? (j < 1 ? j + g.ny : j - g.ny) : (j < 1 ? 1 - j : 2 * g.ny + 1 - j));
      a.phi[q] = a.phi[g.at(mi, mj)];
    }
  }
  DD rz{0.0, 0.0};
  CELL_LOOP {
    CELL_IJ
    T rr = a.r[c];
    if (!a.phi_zero) {
      const T* ph = a.phi;
      const T apv = poisson_ap<T>(g, a.cx, a.cy, i, j, [&](int x, int y) { return ph[g.at(x, y)]; });
      rr = rr - apv;
    }
    const T zz = a.dinv[c] * rr;
    a.r[c] = rr;
    a.z[c] = zz;
    a.pb0[c] = zz;
    dd_add(rz, double(rr) * double(zz));
  }
  double rz_old;
  if (!grid_allreduce(bar, P2, rz, sh, rz_old)) { gave_up(); return; }

  // (d) PCG iterations; the direction update p = z + beta p of iteration k-1
  // is evaluated where iteration k needs it (own cell and stencil
  // neighbours, identical arithmetic), double-buffered in pb0 / pb1.
  double res_norm = 0.0, beta = 0.0;
  int iter;
  for (iter = 1; iter <= a.max_iter; ++iter) {
    T* pcur = (iter & 1) ? a.pb0 : a.pb1;        // p of this iteration
    const T* pprev = (iter & 1) ? a.pb1 : a.pb0; // p of the previous one
    const T tb = T(beta);
    DD papd{0.0, 0.0};
    CELL_LOOP {
      CELL_IJ
      T apv, pown;
      if (iter == 1) {
        const T* p0 = a.pb0;
        pown = __ldcg(p0 + c);
        apv = poisson_ap<T>(g, a.cx, a.cy, i, j, [&](int x, int y) { return __ldcg(p0 + g.at(x, y)); });
      } else {
        const T* zz = a.z;
        auto pf = [&](int x, int y) {
          const int e = g.at(x, y);
          return __ldcg(zz + e) + tb * __ldcg(pprev + e);
        };
        pown = pf(i, j);
        apv = poisson_ap<T>(g, a.cx, a.cy, i, j, pf);
        pcur[c] = pown;
      }
      a.ap[c] = apv;
      dd_add(papd, double(pown) * double(apv));
    }
    double pap;
    if (!grid_allreduce(bar, PA, papd, sh, pap)) { gave_up(); return; }
    if (fabs(pap) < 1.0e-30) break;
    const double alpha = rz_old / pap;
    const T ta = T(alpha);
    DD rrd{0.0, 0.0}, rzd{0.0, 0.0};
    CELL_LOOP {
      CELL_IJ
      const T pown = pcur[c];
      const T rv = a.r[c] - ta * a.ap[c];
      const T zv = a.dinv[c] * rv;
      a.phi[c] = a.phi[c] + ta * pown;
      a.r[c] = rv;
      a.z[c] = zv;
      dd_add(rrd, double(rv) * double(rv));
      dd_add(rzd, double(rv) * double(zv));
    }
    double rr, rz_new;
    if (!grid_allreduce2(bar, PB, PC, rrd, rzd, sh, rr, rz_new)) { gave_up(); return; }
    res_norm = sqrt(rr);
    if (res_norm / rhs_norm < a.tol) break;
    beta = rz_new / rz_old;
    rz_old = rz_new;
  }
  if (closed) {
    DD s{0.0, 0.0};
    CELL_LOOP { CELL_IJ dd_add(s, double(a.phi[c])); }
    double tot;
    if (!grid_allreduce(bar, P0, s, sh, tot)) { gave_up(); return; }
    const double m = tot / (double)(g.nx * g.ny);
    CELL_LOOP { CELL_IJ a.phi[c] = T(double(a.phi[c]) - m); }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const int it = iter < a.max_iter ? iter : a.max_iter;
    a.out->iters = it;
    a.out->res = res_norm / rhs_norm;
    a.out->total_iters += (unsigned long long)it;
    if (a.timed) a.out->timed_iters += (unsigned long long)it;
    a.out->calls += 1;
  }
#undef CELL_LOOP
#undef CELL_IJ
}

// The mean subtraction above uses (phi - mean) in double for both T; for T =
// double it is exactly phi(i,j) - mean_val of mod_subsolvers.f90:238.

// The FP32 inner solve's grid-wide PCG with one grid barrier per iteration:
// the single-reduction (Chronopoulos-Gear) arrangement of
// pcg_cluster_body_1r, for the grids that do not fit one cluster.  With
// u = M^-1 r, w = A u and s = A p, an iteration is one pass over the cells,
//   s = w + beta s,  p = u + beta p,  phi += alpha p,  r -= alpha s,
//   u = M^-1 r,  w = A u,  and the sums (r, u), (w, u), (r, r),
// then one barrier.  w = A u needs the new u of the neighbouring cells; a
// thread forms it from the neighbour's previous r, s and w with the owner's
// expressions (the same bits), so r, s and w are double-buffered by
// iteration parity (read one set, write the other), and so are the partial
// sums' slots (a fast CTA may write the next iteration's partial while a
// slow one still reads this one's).  Buffers: r in r / z, s in pb0 / pb1,
// w in ap / w1, p in pv.  Stopping test and outputs as k_pcg.
template <typename T>
__global__ void __launch_bounds__(512) k_pcg1(PcgArgs<T> a) {
  if (a.active && !*a.active) return;
  __shared__ DD sh[32];
  const Geo g = a.g;
  const int G = gridDim.x;
  const long tid = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long nthr = (long)G * blockDim.x;
  const bool closed = !g.px && !g.py;
  Barrier bar{a.gs, (unsigned int)(G + a.extra_arrivals), a.spin_limit ? a.spin_limit : FUGU_SPIN_LIMIT, 0u};
  auto gave_up = [&]() {
    if (threadIdx.x == 0) a.out->status = 1;
  };
  // the two sets of r, s and w, picked by parity with selects (an array of
  // pointers indexed at run time would live in local memory)
  auto rb = [&](int q) { return q ? a.z : a.r; };
  auto sb = [&](int q) { return q ? a.pb1 : a.pb0; };
  auto wb = [&](int q) { return q ? a.w1 : a.ap; };
  T* pv = a.pv;
  double* P0 = a.part;           // setup sum / final mean
  double* P1 = a.part + 2 * G;   // rhs norm
  double* PS = a.part + 4 * G;   // two sets of three slots: (r, u), (w, u), (r, r)
  const CellWalk cw(tid, nthr, g.nx);
#define CELL_LOOP1 for (int i = cw.i0, j = cw.j0; j <= g.ny; cw.next(i, j, g.nx))
#define CELL_IJ1 const int c = g.at(i, j);

  double mean = 0.0;
  if (closed) {
    DD s{0.0, 0.0};
    CELL_LOOP1 { CELL_IJ1 dd_add(s, double(a.rhs[c])); }
    double tot;
    if (!grid_allreduce(bar, P0, s, sh, tot)) { gave_up(); return; }
    mean = tot / (double)(g.nx * g.ny);
  }
  DD ss{0.0, 0.0};
  CELL_LOOP1 {
    CELL_IJ1
    const T rw = closed ? T(double(a.rhs[c]) - mean) : a.rhs[c];
    rb(0)[c] = rw;
    dd_add(ss, double(rw) * double(rw));
  }
  double ssum;
  if (!grid_allreduce(bar, P1, ss, sh, ssum)) { gave_up(); return; }
  const double rhs_norm = sqrt(ssum);
  if (rhs_norm < 1.0e-14) {
    for (long q = tid; q < g.n(); q += nthr) a.phi[q] = T(0);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      a.out->iters = 0;
      a.out->res = 0.0;
      a.out->calls += 1;
    }
    return;
  }
  if (!a.phi_zero) {
    for (long q = tid; q < g.n(); q += nthr) {
      const int i = (int)(q % g.P) - 2, j = (int)(q / g.P) - 2;
      if (i < -1 || j < -1 || i > g.nx + 2 || j > g.ny + 2) continue;
      if (i >= 1 && i <= g.nx && j >= 1 && j <= g.ny) continue;
      const int mi = (i >= 1 && i <= g.nx) ? i : (g.px ? (i < 1 ? i + g.nx : i - g.nx) : (i < 1 ? 1 - i : 2 * g.nx + 1 - i));
      const int mj = (j >= 1 && j <= g.ny) ? j : (g.py ? (j < 1 ? j + g.ny : j - g.ny) : (j < 1 ? 1 - j : 2 * g.ny + 1 - j));
      a.phi[q] = a.phi[g.at(mi, mj)];
    }
  }
  // r0 = rhs_work - A phi0 (poisson_ap reads interior cells only); s = p = 0
  CELL_LOOP1 {
    CELL_IJ1
    T rr = rb(0)[c];
    if (!a.phi_zero) {
      const T* ph = a.phi;
      rr = rr - poisson_ap<T>(g, a.cx, a.cy, i, j, [&](int x, int y) { return ph[g.at(x, y)]; });
    }
    rb(0)[c] = rr;
    sb(0)[c] = T(0);
    pv[c] = T(0);
  }
  if (!grid_sync(bar.gs, bar.nb, bar.gen, bar.lim)) { gave_up(); return; }
  // w0 = A u0 and the first sums
  double red[3];
  {
    DD d0{0.0, 0.0}, d1{0.0, 0.0}, d2{0.0, 0.0};
    CELL_LOOP1 {
      CELL_IJ1
      const T* r0 = rb(0);
      const T uv = a.dinv[c] * r0[c];
      const T wv = poisson_ap<T>(g, a.cx, a.cy, i, j, [&](int x, int y) {
        const int e = g.at(x, y);
        return a.dinv[e] * __ldcg(r0 + e);
      });
      wb(0)[c] = wv;
      const T rv = r0[c];
      dd_add(d0, double(rv) * double(uv));
      dd_add(d1, double(wv) * double(uv));
      dd_add(d2, double(rv) * double(rv));
    }
    if (!grid_allreduce3(bar, PS, PS + 2 * G, PS + 4 * G, d0, d1, d2, sh, red)) { gave_up(); return; }
  }
  double gam = red[0], del = red[1], res_norm = sqrt(red[2]), alpha = 0.0, beta = 0.0, gam_old = 0.0;
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
    const int rd = (iter - 1) & 1, wr = iter & 1;
    const T* ro = rb(rd);
    const T* so = sb(rd);
    const T* wo = wb(rd);
    // u_k of a cell from its previous r, s and w (the owner's expressions)
    auto unew = [&](int e) {
      const T sv = madd(tb, __ldcg(so + e), __ldcg(wo + e));
      const T rv = madd(-ta, sv, __ldcg(ro + e));
      return a.dinv[e] * rv;
    };
    DD d0{0.0, 0.0}, d1{0.0, 0.0}, d2{0.0, 0.0};
    CELL_LOOP1 {
      CELL_IJ1
      // every load of the cell (its own values and the stencil's) comes
      // before its first store, so they are issued together: one memory
      // round trip per cell (a store in between would hold back the loads
      // after it, since the compiler cannot rule out aliasing)
      const T sk = madd(tb, __ldcg(so + c), __ldcg(wo + c));
      const T uo = a.dinv[c] * __ldcg(ro + c);
      const T pk = madd(tb, pv[c], uo);
      const T ph = madd(ta, pk, a.phi[c]);
      const T rv = madd(-ta, sk, __ldcg(ro + c));
      const T uv = a.dinv[c] * rv;
      const T wv = poisson_ap<T>(g, a.cx, a.cy, i, j, [&](int x, int y) { return unew(g.at(x, y)); });
      a.phi[c] = ph;
      pv[c] = pk;
      sb(wr)[c] = sk;
      rb(wr)[c] = rv;
      wb(wr)[c] = wv;
      dd_add(d0, double(rv) * double(uv));
      dd_add(d1, double(wv) * double(uv));
      dd_add(d2, double(rv) * double(rv));
    }
    double* slot = PS + (iter & 1) * 6 * G;
    if (!grid_allreduce3(bar, slot, slot + 2 * G, slot + 4 * G, d0, d1, d2, sh, red)) { gave_up(); return; }
    gam_old = gam;
    gam = red[0];
    del = red[1];
    res_norm = sqrt(red[2]);
    if (res_norm / rhs_norm < a.tol) break;
  }
  if (closed) {
    DD s{0.0, 0.0};
    CELL_LOOP1 { CELL_IJ1 dd_add(s, double(a.phi[c])); }
    double tot;
    if (!grid_allreduce(bar, P0, s, sh, tot)) { gave_up(); return; }
    const double m = tot / (double)(g.nx * g.ny);
    CELL_LOOP1 { CELL_IJ1 a.phi[c] = T(double(a.phi[c]) - m); }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const int it = iter < a.max_iter ? iter : a.max_iter;
    a.out->iters = it;
    a.out->res = res_norm / rhs_norm;
    a.out->total_iters += (unsigned long long)it;
    if (a.timed) a.out->timed_iters += (unsigned long long)it;
    a.out->calls += 1;
  }
#undef CELL_LOOP1
#undef CELL_IJ1
}

struct SvofArgs {
  Geo g;
  const double* craw;
  double* out;    // C_smooth
  double* work;   // second Jacobi buffer
  double cx, cy, diag;
  int max_iter;
  double tol;
  double* part;
  GridSync* gs;
  int* iters;     // accumulated iteration count
  int* status;
};

// svof_helmholtz_filter, mod_vof.f90:145-194.  Ghost reads go through the
// halo + Neumann index maps, which reproduce the ghosts the reference
// refreshes before every sweep.
__global__ void __launch_bounds__(512) k_svof(SvofArgs a) {
  __shared__ double sh[32];  // max reduction (exact in any order)
  const Geo g = a.g;
  const int G = gridDim.x;
  const long tid = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long nthr = (long)G * blockDim.x;
  const CellWalk cw(tid, nthr, g.nx);
  unsigned int gen = 0;
  for (long q = tid; q < g.n(); q += nthr) a.out[q] = a.craw[q];
  if (!grid_sync(a.gs, G, gen)) { if (threadIdx.x == 0) *a.status = 1; return; }
  auto mx = [&](int i) { return (i >= 1 && i <= g.nx) ? i : (g.px ? (i < 1 ? i + g.nx : i - g.nx) : (i < 1 ? 1 - i : 2 * g.nx + 1 - i)); };
  auto my = [&](int j) { return (j >= 1 && j <= g.ny) ? j : (g.py ? (j < 1 ? j + g.ny : j - g.ny) : (j < 1 ? 1 - j : 2 * g.ny + 1 - j)); };
  int it, used = 0;
  const double* fin = a.out;
  for (it = 1; it <= a.max_iter; ++it) {
    used = it;
    const double* src = (it & 1) ? a.out : a.work;
    double* dst = (it & 1) ? a.work : a.out;
    double res = 0.0;
    // four cells of the walk at a time: every load of the four before the
    // first store, so they go out together (a store in between would hold
    // back the loads after it, since src and dst may alias for all the
    // compiler knows); each cell's expression is unchanged, and the max-norm
    // is exact in any order
    for (int i = cw.i0, j = cw.j0; j <= g.ny;) {
      constexpr int U = 4;
      int cc[U];
      bool on[U];
      double o[U], cr[U], e[U], w[U], n[U], so[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        on[u] = j <= g.ny;
        if (on[u]) {
          const int c = g.at(i, j);
          cc[u] = c;
          o[u] = __ldcg(src + c);
          cr[u] = a.craw[c];
          e[u] = __ldcg(src + g.at(mx(i + 1), j));
          w[u] = __ldcg(src + g.at(mx(i - 1), j));
          n[u] = __ldcg(src + g.at(i, my(j + 1)));
          so[u] = __ldcg(src + g.at(i, my(j - 1)));
          cw.next(i, j, g.nx);
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (on[u]) {
          const double val = (cr[u] + a.cx * (e[u] + w[u]) + a.cy * (n[u] + so[u])) / a.diag;
          dst[cc[u]] = val;
          res = fmax(res, fabs(val - o[u]));
        }
    }
    res = block_max(res, sh);
    if (threadIdx.x == 0) a.part[blockIdx.x] = res;
    if (!grid_sync(a.gs, G, gen)) { if (threadIdx.x == 0) *a.status = 1; return; }
    fin = dst;
    if (max_partials(a.part, G) < a.tol) break;
  }
  // final halo + Neumann: every ghost of C_smooth from its interior
  for (long q = tid; q < g.n(); q += nthr) {
    const int i = (int)(q % g.P) - 2, j = (int)(q / g.P) - 2;
    if (i < -1 || j < -1 || i > g.nx + 2 || j > g.ny + 2) continue;
    const bool inner = (i >= 1 && i <= g.nx && j >= 1 && j <= g.ny);
    if (inner) {
      if (fin != a.out) a.out[q] = __ldcg(fin + q);
    } else {
      a.out[q] = __ldcg(fin + g.at(mx(i), my(j)));
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *a.iters += used;
}

}  // namespace fugu
