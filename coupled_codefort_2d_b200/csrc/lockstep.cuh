// lockstep.cuh -- the fused batched form: many independent cases of uneven
// grid sizes advance their coupled solves in lockstep, and one launch of each
// kernel family serves every case that is still active.
//
// Work lists.  A family kernel runs a fixed persistent grid whose CTAs loop
// over virtual blocks.  A plan kernel maps the active cases to contiguous
// ranges of virtual blocks (one prefix table per family) and a virtual block
// finds its case by binary search in that table.  No launch shape depends on
// which cases are active, so a phase is captured into a CUDA graph once and
// replayed while cases drop out; a finished case costs nothing.
//
// Per case, a virtual block does exactly what one CTA of the single-case
// kernel does -- the same element functions, and for the reductions the same
// partition of the unknowns over CTAs and the same merge order -- so every
// case's results equal those of a context that runs it alone, bit for bit.
//
// Families (virtual blocks of LS_TPB threads):
//   box   32 x 8 tiles of the case's padded box (the stencil kernels)
//   tile  RB_TX x RB_TY tiles (the fused red-black SOR sweeps, the staged matvec)
//   e1    element-wise over a coupled triple, four elements per thread
//   dot   the coupled dot + Krylov scalar op (dot_grid blocks per case)
//   mdot  the FGMRES multi-vector dots (G(nvec) x nvec blocks per case)
//   one   one block per case (ghost cells, wall BCs, small scalar steps)
// and the cluster-resident PCG, launched per grid class with one cluster per
// case of the class.
#pragma once

#include "fgmres.cuh"
#include "kernels.cuh"
#include "pcg_cluster.cuh"
#include "scalars.cuh"

namespace fugu {

constexpr int LS_MAX = 1024;  // cases of one lockstep batch
constexpr int LS_TPB = 256;   // threads of a virtual block

// One case's buffers: pointers into its own context, fixed for the batch.
template <typename T>
struct LsCase {
  Geo g;
  long n;          // elements of one component buffer
  int dot_grid;    // CTAs of the single-case k_dot_op
  int nsm;         // SM count the single-case k_mdot partition uses
  long mdot_gmax;  // ceil(mdot_items / warps per CTA)
  // outer FP64 defect correction
  double *X, *B, *r64, *ax;
  Coefs<double> c64;  // with pen_* / mdot_* set (the step decides whether they are used)
  double *sc, *part;
  KState* ks;
  PcgOut* pcg_out;
  // inner solve in T
  T *ri, *di;        // inner right-hand side and correction triples
  T *V, *Z, *w;      // FGMRES basis V_0..V_m, Z_0..Z_{m-1}, work triple
  double* st;        // FgLayout scalars
  Coefs<T> cf;       // coefficients in T (the FP64 fields themselves when T = double)
  T *cx, *cy, *dinv; // Poisson coefficients of the PCD's PCG
  T *phi, *zuw, *zvw, *tmp;
  // solver settings of the case
  double pcg_tol, inner_tol;
  double jac_omega, sor_omega, visc;
};

// What the host sets per pass / step for each case.
struct LsDyn {
  int run;       // the case takes part in this pass
  int pcg_cap;   // PCG iterations of the PCD
  int sweeps;    // velocity sweeps of the PCD
  int pen, amp;  // the step uses the Darcy penalty / AMP mass fluxes
  int has_lid;
  double dt;     // dt_eff of the step
  double lid;
};

// Active cases and the prefix tables of virtual blocks per family.
struct LsPlan {
  int n;
  int slot[LS_MAX];
  int box[LS_MAX + 1];
  int e1[LS_MAX + 1];
  int dot[LS_MAX + 1];
  int mdot[LS_MAX + 1];   // nvec vectors
  int mdot1[LS_MAX + 1];  // one vector (the norms)
  int tile[LS_MAX + 1];   // RB_TX x RB_TY tiles (the fused red-black sweeps, the matvec)
};

// per-case values the host reads after a phase
struct LsRead {
  double true_rel;  // |B - AX| / |B| of the defect correction
  double inner_rel; // FGMRES relative residual of the cycle
  int nan, active, exit_iter, pad;
};

__host__ __device__ inline int ls_box_blocks(const Geo& g) { return ((g.P + 31) / 32) * ((g.R + 7) / 8); }
__host__ __device__ inline int ls_tile_blocks(const Geo& g) {
  return ((g.P + RB_TX - 1) / RB_TX) * ((g.R + RB_TY - 1) / RB_TY);
}
__host__ __device__ inline int ls_e1_blocks(long n3) { return (int)((n3 + 4L * LS_TPB - 1) / (4L * LS_TPB)); }
// the single-case k_mdot grid width for nvec vectors (mdot() in fugu_gpu.cu)
__host__ __device__ inline int ls_mdot_g(int nsm, long gmax, int nvec) {
  long G = (4L * nsm + nvec - 1) / nvec;
  if (G > gmax) G = gmax;
  if (G < 1) G = 1;
  return (int)G;
}

// largest k in [0, n) with tab[k] <= b (tab ascending, tab[0] = 0)
__device__ __forceinline__ int ls_find(const int* tab, int n, int b) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(tab + mid) <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// ------------------------------------------------------------------ plan
// src 0: the cases with dyn.run; src 1: those whose inner solve is still
// active as well.  One CTA of LS_MAX threads; scans in shared memory.
template <typename T>
__global__ void __launch_bounds__(LS_MAX) k_ls_plan(const LsCase<T>* cs, const LsDyn* dyn, int ncase, int src,
                                                     int nvec, LsPlan* P) {
  constexpr int NT = 6;  // tables
  __shared__ int sc[NT + 1][LS_MAX];
  const int t = threadIdx.x;
  int f = 0, nb[NT] = {0, 0, 0, 0, 0, 0};
  if (t < ncase) {
    const LsCase<T>& c = cs[t];
    f = dyn[t].run && (src == 0 || c.ks->active);
    if (f) {
      nb[0] = ls_box_blocks(c.g);
      nb[1] = ls_e1_blocks(3 * c.n);
      nb[2] = c.dot_grid;
      nb[3] = ls_mdot_g(c.nsm, c.mdot_gmax, nvec) * nvec;
      nb[4] = ls_mdot_g(c.nsm, c.mdot_gmax, 1);
      nb[5] = ls_tile_blocks(c.g);
    }
  }
  sc[0][t] = f;
  for (int q = 0; q < NT; ++q) sc[q + 1][t] = nb[q];
  __syncthreads();
  // Hillis-Steele inclusive scans of the columns
  for (int o = 1; o < LS_MAX; o <<= 1) {
    int v[NT + 1];
    for (int q = 0; q <= NT; ++q) v[q] = t >= o ? sc[q][t - o] : 0;
    __syncthreads();
    for (int q = 0; q <= NT; ++q) sc[q][t] += v[q];
    __syncthreads();
  }
  int* tabs[NT] = {P->box, P->e1, P->dot, P->mdot, P->mdot1, P->tile};
  const int pos = sc[0][t] - f;  // exclusive position among the active cases
  if (f) {
    P->slot[pos] = t;
    for (int q = 0; q < NT; ++q) tabs[q][pos] = sc[q + 1][t] - nb[q];
  }
  if (t == LS_MAX - 1) {
    const int na = sc[0][t];
    P->n = na;
    for (int q = 0; q < NT; ++q) tabs[q][na] = sc[q + 1][t];
  }
}

// ----------------------------------------------------------- family loops
// box: f(c, d, s, k, i, j) at every element of the case's padded box
template <typename T, class F>
__global__ void __launch_bounds__(LS_TPB) k_ls_box(const LsCase<T>* cs, const LsDyn* dyn, const LsPlan* P, F f) {
  const int na = P->n, total = P->box[na];
  for (int vb = blockIdx.x; vb < total; vb += gridDim.x) {
    const int kk = ls_find(P->box, na, vb);
    const int s = P->slot[kk], lb = vb - P->box[kk];
    const LsCase<T>& c = cs[s];
    const int P_ = c.g.P, tx = (P_ + 31) >> 5;
    const int ii = (lb % tx) * 32 + (threadIdx.x & 31), jj = (lb / tx) * 8 + (threadIdx.x >> 5);
    if (ii < P_ && jj < c.g.R) f(c, dyn[s], s, ii + jj * P_, ii - 2, jj - 2);
  }
}
// e1: f(c, d, s, lb, nb) runs virtual block lb of the case's nb
template <typename T, class F>
__global__ void __launch_bounds__(LS_TPB) k_ls_e1(const LsCase<T>* cs, const LsDyn* dyn, const LsPlan* P, F f) {
  const int na = P->n, total = P->e1[na];
  for (int vb = blockIdx.x; vb < total; vb += gridDim.x) {
    const int kk = ls_find(P->e1, na, vb);
    const int s = P->slot[kk];
    f(cs[s], dyn[s], s, vb - P->e1[kk], P->e1[kk + 1] - P->e1[kk]);
  }
}
// one: f(c, d, s) by one block per active case
template <typename T, class F>
__global__ void k_ls_one(const LsCase<T>* cs, const LsDyn* dyn, const LsPlan* P, F f) {
  for (int k = blockIdx.x; k < P->n; k += gridDim.x) {
    const int s = P->slot[k];
    f(cs[s], dyn[s], s);
  }
}
// one block per case of the batch, whether active or not (resets, readback)
template <typename T, class F>
__global__ void k_ls_all(const LsCase<T>* cs, const LsDyn* dyn, int ncase, F f) {
  for (int s = blockIdx.x; s < ncase; s += gridDim.x) f(cs[s], dyn[s], s);
}

// grid-stride pass of virtual block lb of nb over [0, len), four elements per
// thread, loads before stores (the element-wise kernels of kernels.cuh)
#define LS_E1_LOOP(len, body_load, body_store)                                              \
  {                                                                                         \
    const long S_ = (long)nb * LS_TPB;                                                      \
    for (long q0 = (long)lb * LS_TPB + threadIdx.x; q0 < (len); q0 += 4 * S_) {             \
      _Pragma("unroll") for (int u = 0; u < 4; ++u) {                                       \
        const long q = q0 + u * S_;                                                         \
        if (q < (len)) { body_load }                                                        \
      }                                                                                     \
      _Pragma("unroll") for (int u = 0; u < 4; ++u) {                                       \
        const long q = q0 + u * S_;                                                         \
        if (q < (len)) { body_store }                                                       \
      }                                                                                     \
    }                                                                                       \
  }

// ------------------------------------------------------------ functors
// Krylov state of a pass (reset_ks in fugu_gpu.cu) for the cases in it
struct LsResetKs {
  template <typename C>
  __device__ void operator()(const C& c, const LsDyn& d, int) const {
    // a case outside the pass keeps its flags: it may be between steps, its
    // own stream working on its context (nothing reads its flags without
    // checking d.run first)
    if (threadIdx.x == 0 && d.run) {
      c.ks->active = 1;
      c.ks->exit_iter = 0;
      c.ks->nan = 0;
      c.ks->ticket = 0;
      c.ks->kiter = 1;
    }
  }
};

// which buffer a functor works on
enum LsBuf {
  LB_X = 0,   // the state triple (FP64)
  LB_ZJ,      // Z_j
  LB_PHI,     // the PCD's Poisson solution
  LB_JTMP,    // Z_j component or the PCD's tmp, by the parity of a Jacobi sweep
};

// ghost cells of one field (k_halo) when the case is periodic (sweep >= 0:
// the halo before that smoother sweep, skipped by a case that has fewer)
template <typename T>
struct LsHalo {
  int buf, comp, j, sweep;
  __device__ void operator()(const LsCase<T>& c, const LsDyn& d, int) const {
    const Geo& g = c.g;
    if (!g.px && !g.py) return;
    if (sweep >= 0 && sweep >= d.sweeps) return;
    const int kind = comp == 0 ? K_U : (comp == 1 ? K_V : K_CELL);
    if (buf == LB_X) {
      halo_body<double>(g, c.X + comp * c.n, kind);
      return;
    }
    if (!c.ks->active) return;
    T* a;
    if (buf == LB_ZJ) a = c.Z + (long)j * 3 * c.n + comp * c.n;
    else if (buf == LB_PHI) a = c.phi;
    else a = (sweep & 1) ? c.tmp : c.Z + (long)j * 3 * c.n + comp * c.n;
    halo_body<T>(g, a, kind);
  }
};

// wall BCs (k_velocity_bcs): of the state (lid: the step's, when final) or of Z_j
template <typename T>
struct LsVbcs {
  int buf, j, final_lid;
  __device__ void operator()(const LsCase<T>& c, const LsDyn& d, int) const {
    const Geo& g = c.g;
    if (g.px && g.py) return;
    if (buf == LB_X) {
      if (final_lid && !d.has_lid) return;
      vbcs_body<double>(g, c.X, c.X + c.n, final_lid ? d.lid : 0.0);
      return;
    }
    if (!c.ks->active) return;
    T* z = c.Z + (long)j * 3 * c.n;
    vbcs_body<T>(g, z, z + c.n, T(0));
  }
};

template <typename U>
__device__ __forceinline__ Coefs<U> ls_coefs(Coefs<U> cf, const LsDyn& d) {
  if (!d.pen) { cf.pen_u = nullptr; cf.pen_v = nullptr; }
  if (!d.amp) { cf.mdot_u = nullptr; cf.mdot_v = nullptr; }
  return cf;
}

// A X of the defect correction (FP64, every running case)
template <typename T>
struct LsMatvecOuter {
  __device__ void operator()(const LsCase<T>& c, const LsDyn& d, int, int k, int i, int j) const {
    if (k == 0) atomicAdd(&c.ks->matvecs, 1ull);
    const double* X = c.X;
    double* Y = c.ax;
    matvec_at<double>(c.g, ls_coefs(c.c64, d), X, X + c.n, X + 2 * c.n, Y, Y + c.n, Y + 2 * c.n, d.dt, 1, k, i, j);
  }
};

// Poisson coefficients of the PCD's PCG in T (k_poisson_coefs)
template <typename T>
struct LsPoissonCoefs {
  __device__ void operator()(const LsCase<T>& c, const LsDyn&, int, int k, int i, int j) const {
    poisson_coefs_at<T>(c.g, c.c64.rho_u, c.c64.rho_v, c.cx, c.cy, c.dinv, k, i, j);
  }
};

// the step's coefficient fields converted to T (k_convert with scale 1)
template <typename T>
struct LsCvtCoefs {
  __device__ void operator()(const LsCase<T>& c, const LsDyn& d, int, int lb, int nb) const {
    const long n = c.n;
    const double* src[12] = {c.c64.u_adv, c.c64.v_adv, c.c64.rho_c, c.c64.rho_u, c.c64.rho_v, c.c64.kappa,
                             c.c64.zeta, c.c64.eta, c.c64.pen_u, c.c64.pen_v, c.c64.mdot_u, c.c64.mdot_v};
    T* dst[12] = {(T*)c.cf.u_adv, (T*)c.cf.v_adv, (T*)c.cf.rho_c, (T*)c.cf.rho_u, (T*)c.cf.rho_v,
                  (T*)c.cf.kappa, (T*)c.cf.zeta, (T*)c.cf.eta, (T*)c.cf.pen_u, (T*)c.cf.pen_v,
                  (T*)c.cf.mdot_u, (T*)c.cf.mdot_v};
    for (int f = 0; f < 12; ++f) {
      if (f >= 8 && f < 10 && !d.pen) continue;
      if (f >= 10 && !d.amp) continue;
      double a[4];
      LS_E1_LOOP(n, a[u] = src[f][q];, dst[f][q] = T(a[u] * 1.0);)
    }
  }
};

// r = B - A X  (lin: y = x + (s1 * c1) z1 with s1 = -1, c1 = sc[S_ONE])
template <typename T>
struct LsDefect {
  __device__ void operator()(const LsCase<T>& c, const LsDyn&, int, int lb, int nb) const {
    const double c1 = -1.0 * c.sc[S_ONE];
    const long n3 = 3 * c.n;
    double a[4];
    LS_E1_LOOP(n3, a[u] = c.B[q] + c1 * c.ax[q];, c.r64[q] = a[u];)
  }
};
// X = X + (1 * sc[S_ONE]) d  (the FP64 inner form's update)
template <typename T>
struct LsUpdate64 {
  __device__ void operator()(const LsCase<T>& c, const LsDyn&, int, int lb, int nb) const {
    const double c1 = 1.0 * c.sc[S_ONE];
    const long n3 = 3 * c.n;
    const double* dd = (const double*)c.di;
    double a[4];
    LS_E1_LOOP(n3, a[u] = c.X[q] + c1 * dd[q];, c.X[q] = a[u];)
  }
};
// inner right-hand side r / |r| in T (k_convert_scaled) and a zero correction
template <typename T>
struct LsScaleDefect {
  __device__ void operator()(const LsCase<T>& c, const LsDyn&, int, int lb, int nb) const {
    const double sc = c.sc[S_INVRNORM];
    const long n3 = 3 * c.n;
    double a[4];
    LS_E1_LOOP(n3, a[u] = c.r64[q];, c.ri[q] = T(a[u] * sc); c.di[q] = T(0);)
  }
};
// the FP64 inner form starts from a zero correction
template <typename T>
struct LsZeroCorrection {
  __device__ void operator()(const LsCase<T>& c, const LsDyn&, int, int lb, int nb) const {
    const long n3 = 3 * c.n;
    int a[4];
    LS_E1_LOOP(n3, a[u] = 0;, c.di[q] = T(a[u]);)
  }
};
// X += |r| d  (k_accumulate)
template <typename T>
struct LsAccumulate {
  __device__ void operator()(const LsCase<T>& c, const LsDyn&, int, int lb, int nb) const {
    const double s = c.sc[S_RNORM];
    const long n3 = 3 * c.n;
    double a[4];
    LS_E1_LOOP(n3, a[u] = c.X[q] + s * double(c.di[q]);, c.X[q] = a[u];)
  }
};

// the FGMRES scalars of a cycle start at zero
template <typename T>
struct LsZeroSt {
  int size;
  __device__ void operator()(const LsCase<T>& c, const LsDyn&, int) const {
    for (int q = threadIdx.x; q < size; q += blockDim.x) c.st[q] = 0.0;
  }
};

// a new basis vector V_dst = 0 + inv * src (k_fg_scale); src: the inner
// right-hand side (dst 0) or the work vector
template <typename T>
struct LsFgScale {
  int dst;
  int inv_slot;
  __device__ void operator()(const LsCase<T>& c, const LsDyn&, int, int lb, int nb) const {
    if (!c.ks->active) return;
    const T f = T(c.st[inv_slot]);
    const T* src = dst == 0 ? c.ri : c.w;
    T* out = c.V + (long)dst * 3 * c.n;
    const long n3 = 3 * c.n;
    T a[4];
    LS_E1_LOOP(n3, a[u] = src[q];, out[q] = T(0) + f * a[u];)
  }
};

// PCD output Z_j and the Poisson solution start at zero
template <typename T>
struct LsZeroPcd {
  int j;
  __device__ void operator()(const LsCase<T>& c, const LsDyn&, int, int lb, int nb) const {
    if (!c.ks->active) return;
    T* z = c.Z + (long)j * 3 * c.n;
    const long n3 = 3 * c.n;
    int a[4];
    LS_E1_LOOP(n3, a[u] = 0;, z[q] = T(a[u]);)
    LS_E1_LOOP(c.n, a[u] = 0;, c.phi[q] = T(a[u]);)
  }
};

// PCD steps on V_j -> Z_j (apply_pcd_precond, mod_pcd_precond.f90:14-104)
template <typename T>
struct LsSchur {
  int jj;
  __device__ void operator()(const LsCase<T>& c, const LsDyn& d, int, int k, int i, int j) const {
    if (!c.ks->active) return;
    const T* zp = c.V + (long)jj * 3 * c.n + 2 * c.n;
    T* rp = c.Z + (long)jj * 3 * c.n + 2 * c.n;
    rp[k] = pcd_schur_at<T>(c.g, k, i, j, c.phi, c.cf.u_adv, c.cf.v_adv, T(1.0 / d.dt), c.cf.kappa, zp, T(c.visc));
  }
};
template <typename T>
struct LsZwork {
  int jj;
  __device__ void operator()(const LsCase<T>& c, const LsDyn&, int, int k, int i, int j) const {
    if (!c.ks->active) return;
    const T* z = c.V + (long)jj * 3 * c.n;
    const T* rp = c.Z + (long)jj * 3 * c.n + 2 * c.n;
    pcd_zwork_at<T>(c.g, k, i, j, z, z + c.n, rp, c.zuw, c.zvw);
  }
};
template <typename T>
struct LsCross {
  int jj;
  __device__ void operator()(const LsCase<T>& c, const LsDyn&, int, int k, int i, int j) const {
    if (!c.ks->active) return;
    const T* rv = c.Z + (long)jj * 3 * c.n + c.n;
    pcd_cross_at<T>(c.g, k, i, j, c.cf.eta, rv, c.zuw);
  }
};
// one colour pass of red-black SOR on component comp of Z_j (sweep s; a
// case with fewer sweeps skips it) -- the periodic batches
template <typename T>
struct LsRbsor {
  int jj, comp, sweep, col;
  __device__ void operator()(const LsCase<T>& c, const LsDyn& d, int, int k, int i, int j) const {
    if (!c.ks->active || sweep >= d.sweeps) return;
    T* z = c.Z + (long)jj * 3 * c.n + comp * c.n;
    const T* pen = d.pen ? (comp == 0 ? c.cf.pen_u : c.cf.pen_v) : nullptr;
    if (comp == 0) {
      if (!rbsor_u_face(c.g, i, j, col)) return;
      z[k] = jacobi_u_at<T>(c.g, k, i, j, z, c.zuw, c.cf.rho_u, c.cf.kappa, c.cf.zeta, c.cf.eta, pen, T(d.dt),
                            T(c.sor_omega));
    } else {
      if (!rbsor_v_face(c.g, i, j, col)) return;
      z[k] = jacobi_v_at<T>(c.g, k, i, j, z, c.zvw, c.cf.rho_v, c.cf.kappa, c.cf.zeta, c.cf.eta, pen, T(d.dt),
                            T(c.sor_omega));
    }
  }
};
// one damped-Jacobi sweep s on component comp of Z_j: even sweeps read Z_j
// and write tmp, odd ones the reverse (the single-case cur / nxt swap)
template <typename T>
struct LsJacobi {
  int jj, comp, sweep;
  __device__ void operator()(const LsCase<T>& c, const LsDyn& d, int, int k, int i, int j) const {
    if (!c.ks->active || sweep >= d.sweeps) return;
    T* z = c.Z + (long)jj * 3 * c.n + comp * c.n;
    const T* src = (sweep & 1) ? c.tmp : z;
    T* dst = (sweep & 1) ? z : c.tmp;
    const T* pen = d.pen ? (comp == 0 ? c.cf.pen_u : c.cf.pen_v) : nullptr;
    if (comp == 0)
      dst[k] = jacobi_u_at<T>(c.g, k, i, j, src, c.zuw, c.cf.rho_u, c.cf.kappa, c.cf.zeta, c.cf.eta, pen, T(d.dt),
                              T(c.jac_omega));
    else
      dst[k] = jacobi_v_at<T>(c.g, k, i, j, src, c.zvw, c.cf.rho_v, c.cf.kappa, c.cf.zeta, c.cf.eta, pen, T(d.dt),
                              T(c.jac_omega));
  }
};
// after an odd number of Jacobi sweeps the result is in tmp: copy it back
template <typename T>
struct LsJacobiCopy {
  int jj, comp;
  __device__ void operator()(const LsCase<T>& c, const LsDyn& d, int, int lb, int nb) const {
    if (!c.ks->active || !(d.sweeps & 1)) return;
    T* z = c.Z + (long)jj * 3 * c.n + comp * c.n;
    T a[4];
    LS_E1_LOOP(c.n, a[u] = c.tmp[q];, z[q] = a[u];)
  }
};

// back substitution of the cycle (k_fg_solve) over the k columns used
template <typename T>
struct LsFgSolve {
  int m;
  __device__ void operator()(const LsCase<T>& c, const LsDyn&, int) const {
    if (threadIdx.x != 0) return;
    const int k = c.ks->active ? m : c.ks->exit_iter;
    if (k > 0) fg_solve_body(c.st, FgLayout{m}, k);
  }
};

// what the host reads after a phase
template <typename T>
struct LsReadback {
  LsRead* out;
  int m;
  __device__ void operator()(const LsCase<T>& c, const LsDyn&, int s) const {
    if (threadIdx.x != 0) return;
    LsRead r;
    r.true_rel = c.sc[S_TRUEREL];
    r.inner_rel = c.st[FgLayout{m}.rel()];
    r.nan = c.ks->nan;
    r.active = c.ks->active;
    r.exit_iter = c.ks->exit_iter;
    r.pad = 0;
    out[s] = r;
  }
};

// arm the conditional node of the next Arnoldi step: some case still active
__global__ void k_ls_cond(const LsPlan* P, cudaGraphConditionalHandle h) {
  if (threadIdx.x == 0) cudaGraphSetConditional(h, P->n > 0 ? 1u : 0u);
}

// ------------------------------------------------------ reduction families
// coupled dots + Krylov scalar op of the defect correction (k_dot_op)
// which: 0 (B, B), 1 (r, r)
template <typename T>
__global__ void __launch_bounds__(256) k_ls_dot(const LsCase<T>* cs, const LsPlan* P, int which, OpArgs op) {
  const int na = P->n, total = P->dot[na];
  for (int vb = blockIdx.x; vb < total; vb += gridDim.x) {
    const int kk = ls_find(P->dot, na, vb);
    const int s = P->slot[kk];
    const LsCase<T>& c = cs[s];
    DotArgs<double> d;
    d.g = c.g;
    d.n = c.n;
    const double* v = which == 0 ? c.B : c.r64;
    d.a[0] = v;
    d.b[0] = v;
    for (int q = 1; q < 5; ++q) { d.a[q] = nullptr; d.b[q] = nullptr; }
    d.npairs = 1;
    d.vol = c.g.dx * c.g.dy;
    d.part = c.part;
    d.sc = c.sc;
    d.ks = c.ks;
    d.op = op;
    d.check_active = 0;
    __syncthreads();  // the previous virtual block is done with shared memory
    dot_op_body<double>(d, vb - P->dot[kk], c.dot_grid);
  }
}

// FGMRES multi-vector dots (k_mdot): which 0: (ri; ri) FG_BETA, 1: (w; V_0..V_j)
// Gram-Schmidt passes, 2: (w; w) FG_ROTATE
template <typename T>
__global__ void __launch_bounds__(MDOT_TPB) k_ls_mdot(const LsCase<T>* cs, const LsPlan* P, int which, int nvec,
                                                      int op, int j, int m) {
  const int* tab = which == 1 ? P->mdot : P->mdot1;
  const int na = P->n, total = tab[na];
  for (int vb = blockIdx.x; vb < total; vb += gridDim.x) {
    const int kk = ls_find(tab, na, vb);
    const int s = P->slot[kk];
    const LsCase<T>& c = cs[s];
    __syncthreads();  // the previous virtual block is done with shared memory
    if (!c.ks->active) continue;
    const int G = ls_mdot_g(c.nsm, c.mdot_gmax, nvec);
    const int local = vb - tab[kk];
    MdotArgs<T> a;
    a.g = c.g;
    a.n = c.n;
    a.w = which == 0 ? c.ri : c.w;
    a.V0 = which == 0 ? c.ri : (which == 1 ? c.V : c.w);
    a.stride = 3 * c.n;
    a.nvec = nvec;
    a.vol = c.g.dx * c.g.dy;
    a.part = c.part;
    a.st = c.st;
    a.ks = c.ks;
    a.L = FgLayout{m};
    a.op = op;
    a.j = j;
    a.tol = c.inner_tol;
    mdot_body<T>(a, local % G, local / G, G, nvec);
  }
}

// w += sign * sum coef[i] V_i (k_maxpy): which 0: w -= V_0..V_j h (nvec
// j + 1), 1: d += Z_0..Z_{k-1} y with k the cycle's steps (every running case)
template <typename T>
__global__ void __launch_bounds__(LS_TPB) k_ls_maxpy(const LsCase<T>* cs, const LsPlan* P, int which, int nvec,
                                                     int m) {
  const int na = P->n, total = P->e1[na];
  const FgLayout L{m};
  for (int vb = blockIdx.x; vb < total; vb += gridDim.x) {
    const int kk = ls_find(P->e1, na, vb);
    const int s = P->slot[kk];
    const LsCase<T>& c = cs[s];
    const long n3 = 3 * c.n;
    int nv;
    T* w;
    const T* V0;
    const double* coef;
    double sign;
    if (which == 0) {
      if (!c.ks->active) continue;
      nv = nvec;
      w = c.w;
      V0 = c.V;
      coef = c.st + L.h();
      sign = -1.0;
    } else {
      nv = c.ks->active ? m : c.ks->exit_iter;
      if (nv <= 0) continue;
      w = c.di;
      V0 = c.Z;
      coef = c.st + L.y();
      sign = 1.0;
    }
    __syncthreads();  // the previous virtual block is done with shared memory
    maxpy_body<T>(n3, w, V0, n3, coef, nv, sign, vb - P->e1[kk], P->e1[kk + 1] - P->e1[kk]);
  }
}

// one fused red-black SOR sweep (both colours, kernels.cuh) of component comp
// of Z_j for every active case with more than `sweep` sweeps; every case of
// the batch is wall-bounded
template <typename T>
__global__ void __launch_bounds__(RB_TPB) k_ls_rbsor(const LsCase<T>* cs, const LsDyn* dyn, const LsPlan* P,
                                                     int jj, int comp, int sweep) {
  __shared__ RbSmem<T> sm;
  const int na = P->n, total = P->tile[na];
  for (int vb = blockIdx.x; vb < total; vb += gridDim.x) {
    const int kk = ls_find(P->tile, na, vb);
    const int s = P->slot[kk];
    const LsCase<T>& c = cs[s];
    const LsDyn& d = dyn[s];
    __syncthreads();  // the previous tile is done with shared memory
    if (!c.ks->active || sweep >= d.sweeps) continue;
    const int lb = vb - P->tile[kk], ntx = (c.g.P + RB_TX - 1) / RB_TX;
    // even sweeps from Z_j into tmp, odd ones back (LsJacobiCopy after an odd count)
    T* z = c.Z + (long)jj * 3 * c.n + comp * c.n;
    const T* src = (sweep & 1) ? c.tmp : z;
    T* dst = (sweep & 1) ? z : c.tmp;
    const T* pen = d.pen ? (comp == 0 ? c.cf.pen_u : c.cf.pen_v) : nullptr;
    rbsor_sweep_tile<T>(c.g, comp, lb % ntx, lb / ntx, src, dst, comp == 0 ? c.zuw : c.zvw,
                        comp == 0 ? c.cf.rho_u : c.cf.rho_v, c.cf.kappa, c.cf.zeta, c.cf.eta, pen, T(d.dt),
                        T(c.sor_omega), sm);
  }
}

// w = A Z_j of Arnoldi step j, on the staged tiles of k_matvec_tile (the tile
// family: its RB_TX x RB_TY tiles are MT_TX x RB_TY matvec tiles)
static_assert(MT_TX == RB_TX && RB_TY % 8 == 0, "the matvec tiles are the tile family's tiles");
template <typename T>
__global__ void __launch_bounds__(MT_TPB) k_ls_matvec(const LsCase<T>* cs, const LsDyn* dyn, const LsPlan* P,
                                                      int jj) {
  extern __shared__ __align__(16) unsigned char mt_smem[];
  const int na = P->n, total = P->tile[na];
  for (int vb = blockIdx.x; vb < total; vb += gridDim.x) {
    const int kk = ls_find(P->tile, na, vb);
    const int s = P->slot[kk];
    const LsCase<T>& c = cs[s];
    const LsDyn& d = dyn[s];
    __syncthreads();  // the previous tile is done with shared memory
    if (!c.ks->active) continue;
    const int lb = vb - P->tile[kk], ntx = (c.g.P + MT_TX - 1) / MT_TX;
    if (lb == 0 && threadIdx.x == 0) atomicAdd(&c.ks->matvecs, 1ull);
    const T* X = c.Z + (long)jj * 3 * c.n;
    matvec_tile<T, RB_TY>(c.g, ls_coefs(c.cf, d), X, X + c.n, X + 2 * c.n, c.w, c.w + c.n, c.w + 2 * c.n, T(d.dt), 1,
                          lb % ntx, lb / ntx, (T*)mt_smem);
  }
}

// cluster-resident PCG of the PCD on V_j's pressure block for the cases of
// one grid class: cluster q solves case cls[q] (k_pcg_cluster)
template <typename T, int CPT>
__global__ void __launch_bounds__(PCGC_TPB, 1) k_ls_pcg(const LsCase<T>* cs, const LsDyn* dyn, const int* cls,
                                                       int rows_per, int j) {
  const int C = (int)cgc::this_cluster().num_blocks();
  const int s = cls[blockIdx.x / C];
  const LsCase<T>& c = cs[s];
  const LsDyn& d = dyn[s];
  if (!d.run || !c.ks->active) return;  // the same for every CTA of the cluster
  PcgClusterArgs<T> a;
  a.g = c.g;
  a.rhs = c.V + (long)j * 3 * c.n + 2 * c.n;
  a.cx = c.cx;
  a.cy = c.cy;
  a.dinv = c.dinv;
  a.phi = c.phi;
  a.out = c.pcg_out;
  a.active = nullptr;
  a.tol = c.pcg_tol;
  a.max_iter = d.pcg_cap;
  a.phi_zero = 1;
  a.rows_per = rows_per;
  a.timed = 0;
  if constexpr (pcgc_one_reduction<T>(CPT)) pcg_cluster_body_1r<CPT>(a);
  else pcg_cluster_body<T, CPT>(a);
}

}  // namespace fugu
