// kernels.cuh -- hand-written sm_100a kernels of the FUGU-2D coupled step.
//
// Each kernel restates one loop nest of the Fortran reference (file:line in
// the comment above it) in the uniform device layout of fugu_internal.cuh.
// Expressions keep the reference's operand order; the FP64 instantiation is
// compiled with --fmad=false, so element-wise results match the CPU oracle
// bit for bit.  Templates on T let the mixed-precision inner solve reuse the
// same code in FP32.
#pragma once

#include "fugu_internal.cuh"

namespace fugu {

// --------------------------------------------------------------- helpers
template <typename T>
__device__ __forceinline__ T clip01(T x) { return fmax(T(0), fmin(T(1), x)); }

#define FUGU_BOX_IJ                                          \
  const int ii = blockIdx.x * blockDim.x + threadIdx.x;      \
  const int jj = blockIdx.y * blockDim.y + threadIdx.y;      \
  if (ii >= g.P || jj >= g.R) return;                        \
  const int i = ii - 2, j = jj - 2;                          \
  const int k = ii + jj * g.P;                               \
  (void)k;

__device__ __forceinline__ bool in_kind(const Geo& g, int kind, int i, int j) {
  int i0, i1, j0, j1;
  g.extent(kind, i0, i1, j0, j1);
  return i >= i0 && i <= i1 && j >= j0 && j <= j1;
}

// ------------------------------------------------------------ halos
// mpi_exchange_halos_{scalar,u,v} at one rank (mod_mpi.f90:113-245): a
// periodic direction copies its own opposite interior layers (x pass over the
// full j range first, then y pass over the full i range); a wall direction is
// untouched.  One CTA; phases separated by __syncthreads.
template <typename T>
__device__ __forceinline__ void halo_body(const Geo& g, T* a, int kind) {
  int i0, i1, j0, j1;
  g.extent(kind, i0, i1, j0, j1);
  const int nx = g.nx, ny = g.ny;
  if (g.px) {
    const int nj = j1 - j0 + 1;
    for (int t = threadIdx.x; t < 2 * nj; t += blockDim.x) {
      const int kk = t & 1, j = j0 + (t >> 1);
      a[g.at(-1 + kk, j)] = a[g.at(nx - 1 + kk, j)];
    }
    __syncthreads();
    for (int t = threadIdx.x; t < 2 * nj; t += blockDim.x) {
      const int kk = t & 1, j = j0 + (t >> 1);
      a[g.at(nx + 1 + kk, j)] = a[g.at(1 + kk, j)];
    }
    __syncthreads();
  }
  if (g.py) {
    const int ni = i1 - i0 + 1;
    for (int t = threadIdx.x; t < 2 * ni; t += blockDim.x) {
      const int kk = t / ni, i = i0 + t % ni;
      a[g.at(i, -1 + kk)] = a[g.at(i, ny - 1 + kk)];
    }
    __syncthreads();
    for (int t = threadIdx.x; t < 2 * ni; t += blockDim.x) {
      const int kk = t / ni, i = i0 + t % ni;
      a[g.at(i, ny + 1 + kk)] = a[g.at(i, 1 + kk)];
    }
  }
}
template <typename T>
__global__ void k_halo(Geo g, T* a, int kind, const int* active) {
  if (active && !*active) return;
  halo_body<T>(g, a, kind);
}

// ------------------------------------------------------------ velocity BCs
// apply_velocity_bcs, mod_operators.f90:254-333: west, east, south, north in
// that order (each phase reads what the previous one wrote at the corners).
// Extension fsx: symmetric (free-slip) tangential ghosts at the side walls.
template <typename T>
__device__ __forceinline__ void vbcs_body(const Geo& g, T* u, T* v, T u_lid) {
  const int nx = g.nx, ny = g.ny;
  const T vs = g.fsx ? T(1) : T(-1);
  if (!g.px) {
    for (int t = threadIdx.x; t < ny + 5; t += blockDim.x) {  // west
      const int j = -2 + t;
      if (j >= -1) {
        u[g.at(0, j)] = T(0);
        u[g.at(-1, j)] = -u[g.at(1, j)];
        u[g.at(-2, j)] = -u[g.at(2, j)];
      }
      v[g.at(0, j)] = vs * v[g.at(1, j)];
      v[g.at(-1, j)] = vs * v[g.at(2, j)];
    }
    __syncthreads();
    for (int t = threadIdx.x; t < ny + 5; t += blockDim.x) {  // east
      const int j = -2 + t;
      if (j >= -1) {
        u[g.at(nx, j)] = T(0);
        u[g.at(nx + 1, j)] = -u[g.at(nx - 1, j)];
        u[g.at(nx + 2, j)] = -u[g.at(nx - 2, j)];
      }
      v[g.at(nx + 1, j)] = vs * v[g.at(nx, j)];
      v[g.at(nx + 2, j)] = vs * v[g.at(nx - 1, j)];
    }
    __syncthreads();
  }
  if (!g.py) {
    for (int t = threadIdx.x; t < nx + 5; t += blockDim.x) {  // south
      const int i = -2 + t;
      if (i >= -1) {
        v[g.at(i, 0)] = T(0);
        v[g.at(i, -1)] = -v[g.at(i, 1)];
        v[g.at(i, -2)] = -v[g.at(i, 2)];
      }
      u[g.at(i, 0)] = -u[g.at(i, 1)];
      u[g.at(i, -1)] = -u[g.at(i, 2)];
    }
    __syncthreads();
    const T two_lid = T(2) * u_lid;
    for (int t = threadIdx.x; t < nx + 5; t += blockDim.x) {  // north
      const int i = -2 + t;
      if (i >= -1) {
        v[g.at(i, ny)] = T(0);
        v[g.at(i, ny + 1)] = -v[g.at(i, ny - 1)];
        v[g.at(i, ny + 2)] = -v[g.at(i, ny - 2)];
      }
      u[g.at(i, ny + 1)] = two_lid - u[g.at(i, ny)];
      u[g.at(i, ny + 2)] = two_lid - u[g.at(i, ny - 1)];
    }
  }
}
template <typename T>
__global__ void k_velocity_bcs(Geo g, T* u, T* v, T u_lid, const int* active) {
  if (active && !*active) return;
  vbcs_body<T>(g, u, v, u_lid);
}

// ------------------------------------------------------------ properties
// The explicit stages of the step (properties, VOF transport, curvature,
// CSF, right-hand side) are templates on their scalar type S: double for the
// step itself, ad::Dual for its tangent (the discrete adjoint).
template <typename S>
struct MixT {
  S rho1, rho2, mu1, mu2;
};
using Mix = MixT<double>;

// harmonic_viscosity, mod_viscosity.f90:28-46
template <typename S>
__device__ __forceinline__ S harmonic_mu(const MixT<S>& m, S c) {
  const S cc = clip01(c);
  if (fabs(m.mu1 - m.mu2) < 1.0e-14) return m.mu1;
  const S den = m.mu2 * cc + m.mu1 * (1.0 - cc);
  if (den > 1.0e-15) return (m.mu1 * m.mu2) / den;
  return fmin(m.mu1, m.mu2);
}
template <typename S>
__device__ __forceinline__ S rho_of(const MixT<S>& m, S c) {
  const S cv = clip01(c);
  return m.rho1 * cv + m.rho2 * (1.0 - cv);
}

// compute_mixture_densities + compute_mixture_viscosities
// (mod_viscosity.f90:54-151) in one pass: every output element is computed
// from C directly; the border copies of the reference become index clamps.
template <typename S>
__global__ void k_properties(Geo g, MixT<S> m, const S* __restrict__ c, S* rho_c, S* rho_u, S* rho_v, S* kappa,
                             S* zeta, S* eta) {
  FUGU_BOX_IJ
  const int nx = g.nx, ny = g.ny;
  if (in_kind(g, K_CELL, i, j)) {
    rho_c[k] = rho_of(m, c[k]);
    kappa[k] = 2.0 * harmonic_mu(m, c[k]);
  }
  if (in_kind(g, K_U, i, j)) {
    const int ie = min(max(i, -1), nx + 1);
    rho_u[k] = 0.5 * (rho_of(m, c[g.at(ie, j)]) + rho_of(m, c[g.at(ie + 1, j)]));
  }
  if (in_kind(g, K_V, i, j)) {
    const int je = min(max(j, -1), ny + 1);
    rho_v[k] = 0.5 * (rho_of(m, c[g.at(i, je)]) + rho_of(m, c[g.at(i, je + 1)]));
  }
  {  // vertex extent is the whole box's kind range
    if (in_kind(g, K_VERT, i, j)) {
      const int ie = min(max(i, -1), nx + 1), je = min(max(j, -1), ny + 1);
      const S cv = 0.25 * (c[g.at(ie, je)] + c[g.at(ie + 1, je)] + c[g.at(ie, je + 1)] + c[g.at(ie + 1, je + 1)]);
      const S mu = harmonic_mu(m, cv);
      zeta[k] = 2.0 * mu;
      eta[k] = mu;
    }
  }
}

// ------------------------------------------------------------ operators
// Field views.  The operator formulas read a field at Fortran (i, j) through
// a view, so one expression (and one operand order) serves a field in global
// memory and a tile of it staged in shared memory; the two give the same bits.
template <typename T>
struct GView {  // a whole padded box in global memory
  const T* p;
  int P;
  __device__ __forceinline__ T operator()(int i, int j) const { return p[(i + 2) + (j + 2) * P]; }
};
template <typename T>
__device__ __forceinline__ GView<T> gview(const Geo& g, const T* p) { return GView<T>{p, g.P}; }
template <typename T, int W>
struct SView {  // a staged tile of W elements per row; (i0, j0) is the Fortran index of s[0]
  const T* s;
  int i0, j0;
  __device__ __forceinline__ T operator()(int i, int j) const { return s[(j - j0) * W + (i - i0)]; }
};

// T_xx, T_yy at cells and T_xy, T_yx at vertices (mod_operators.f90:119-140)
template <typename T, typename V>
__device__ __forceinline__ T txx(const V& u, const V& kap, int i, int j, T idx) {
  return kap(i, j) * (u(i, j) - u(i - 1, j)) * idx;
}
template <typename T, typename V>
__device__ __forceinline__ T tyy(const V& v, const V& kap, int i, int j, T idy) {
  return kap(i, j) * (v(i, j) - v(i, j - 1)) * idy;
}
template <typename T, typename V>
__device__ __forceinline__ void txy_tyx(const V& u, const V& v, const V& zeta, const V& eta, int i, int j, T idx,
                                        T idy, T& txy, T& tyx) {
  const T du_dy = (u(i, j + 1) - u(i, j)) * idy;
  const T dv_dx = (v(i + 1, j) - v(i, j)) * idx;
  const T z = zeta(i, j), e = eta(i, j);
  txy = (z - e) * du_dy + e * dv_dx;
  tyx = e * du_dy + (z - e) * dv_dx;
}
// -div(T) on a u face (mod_operators.f90:145-150)
template <typename T, typename V>
__device__ __forceinline__ T visc_u_at(const V& u, const V& v, const V& kap, const V& zeta, const V& eta, int i,
                                       int j, T idx, T idy) {
  T a0, b0, a1, b1;
  txy_tyx<T>(u, v, zeta, eta, i, j, idx, idy, a0, b0);
  txy_tyx<T>(u, v, zeta, eta, i, j - 1, idx, idy, a1, b1);
  return -((txx<T>(u, kap, i + 1, j, idx) - txx<T>(u, kap, i, j, idx)) * idx + (a0 - a1) * idy);
}
// -div(T) on a v face (mod_operators.f90:155-160)
template <typename T, typename V>
__device__ __forceinline__ T visc_v_at(const V& u, const V& v, const V& kap, const V& zeta, const V& eta, int i,
                                       int j, T idx, T idy) {
  T a0, b0, a1, b1;
  txy_tyx<T>(u, v, zeta, eta, i, j, idx, idy, a0, b0);
  txy_tyx<T>(u, v, zeta, eta, i - 1, j, idx, idy, a1, b1);
  return -((b0 - b1) * idx + (tyy<T>(v, kap, i, j + 1, idy) - tyy<T>(v, kap, i, j, idy)) * idy);
}

// op_advection, mod_operators.f90:201-222 (u component); amp: the mass fluxes
// mdu / mdv replace rho * velocity (consistent AMP)
template <typename T, typename V>
__device__ __forceinline__ T adv_u_at(const V& ua, const V& va, const V& rc, const V& rv, const V& u,
                                      const GView<T>& mdu, const GView<T>& mdv, bool amp, int i, int j, T idx,
                                      T idy) {
  const T h = T(0.5);
  T mE, mW, mN, mS;
  if (amp) {
    mE = h * (mdu(i, j) + mdu(i + 1, j));
    mW = h * (mdu(i - 1, j) + mdu(i, j));
    mN = h * (mdv(i, j) + mdv(i + 1, j));
    mS = h * (mdv(i, j - 1) + mdv(i + 1, j - 1));
  } else {
    mE = rc(i + 1, j) * h * (ua(i, j) + ua(i + 1, j));
    mW = rc(i, j) * h * (ua(i - 1, j) + ua(i, j));
    mN = h * (rv(i, j) + rv(i + 1, j)) * h * (va(i, j) + va(i + 1, j));
    mS = h * (rv(i, j - 1) + rv(i + 1, j - 1)) * h * (va(i, j - 1) + va(i + 1, j - 1));
  }
  const T uE = h * (u(i, j) + u(i + 1, j));
  const T uW = h * (u(i - 1, j) + u(i, j));
  const T uN = h * (u(i, j) + u(i, j + 1));
  const T uS = h * (u(i, j - 1) + u(i, j));
  return (mE * uE - mW * uW) * idx + (mN * uN - mS * uS) * idy;
}
// op_advection, mod_operators.f90:225-247 (v component)
template <typename T, typename V>
__device__ __forceinline__ T adv_v_at(const V& ua, const V& va, const V& rc, const V& ru, const V& v,
                                      const GView<T>& mdu, const GView<T>& mdv, bool amp, int i, int j, T idx,
                                      T idy) {
  const T h = T(0.5);
  T mE, mW, mN, mS;
  if (amp) {
    mE = h * (mdu(i, j) + mdu(i, j + 1));
    mW = h * (mdu(i - 1, j) + mdu(i - 1, j + 1));
    mN = h * (mdv(i, j) + mdv(i, j + 1));
    mS = h * (mdv(i, j - 1) + mdv(i, j));
  } else {
    mE = h * (ru(i, j) + ru(i, j + 1)) * h * (ua(i, j) + ua(i, j + 1));
    mW = h * (ru(i - 1, j) + ru(i - 1, j + 1)) * h * (ua(i - 1, j) + ua(i - 1, j + 1));
    mN = rc(i, j + 1) * h * (va(i, j) + va(i, j + 1));
    mS = rc(i, j) * h * (va(i, j - 1) + va(i, j));
  }
  const T vE = h * (v(i, j) + v(i + 1, j));
  const T vW = h * (v(i - 1, j) + v(i, j));
  const T vN = h * (v(i, j) + v(i, j + 1));
  const T vS = h * (v(i, j - 1) + v(i, j));
  return (mE * vE - mW * vW) * idx + (mN * vN - mS * vS) * idy;
}

// Coefficient fields of the coupled operator for one precision.
template <typename T>
struct Coefs {
  const T *u_adv, *v_adv, *rho_c, *rho_u, *rho_v, *kappa, *zeta, *eta;
  const T *pen_u, *pen_v;   // nullable
  const T *mdot_u, *mdot_v; // nullable (AMP)
};

// The eleven fields the coupled operator reads with a stencil, as views.
enum { MV_XU, MV_XV, MV_XP, MV_UA, MV_VA, MV_RC, MV_RU, MV_RV, MV_KA, MV_ZE, MV_ET, MV_N };

// matvec_coupled, mod_operators.f90:341-443, at one (i, j): Y_u(i,j),
// Y_v(i,j) and Y_p(i,j) of the whole padded box (zero where the reference
// zeroes), computing the viscous stresses, the pressure gradient, the
// advection and the divergence from X on the fly.  X must already hold its
// periodic halo (k_halo).  f: the stencil fields as views; the penalty (one
// value per face) and the AMP mass fluxes are read from global memory.
template <typename T, typename V>
__device__ __forceinline__ void matvec_vals(const Geo& g, const V* f, const Coefs<T>& c, T dt, int with_adv, int k,
                                            int i, int j, T& yu, T& yv, T& yp) {
  const int nx = g.nx, ny = g.ny;
  const T idx = T(g.idx), idy = T(g.idy);
  const V& Xu = f[MV_XU];
  const V& Xv = f[MV_XV];
  const V& Xp = f[MV_XP];
  const bool amp = c.mdot_u != nullptr;
  const GView<T> mdu = gview(g, c.mdot_u), mdv = gview(g, c.mdot_v);
  // u row
  yu = T(0);
  if (j >= 1 && j <= ny) {
    if (i >= 1 && i <= g.imax()) {
      const T adv = with_adv ? adv_u_at<T>(f[MV_UA], f[MV_VA], f[MV_RC], f[MV_RV], Xu, mdu, mdv, amp, i, j, idx, idy)
                             : T(0);
      const T vis = visc_u_at<T>(Xu, Xv, f[MV_KA], f[MV_ZE], f[MV_ET], i, j, idx, idy);
      const T gp = (Xp(i + 1, j) - Xp(i, j)) * idx;
      yu = (f[MV_RU](i, j) / dt) * Xu(i, j) + adv + vis + gp;
      if (c.pen_u) yu = yu + c.pen_u[k] * Xu(i, j);
    } else if (!g.px && (i == 0 || i == nx)) {
      yu = Xu(i, j);
    }
  }
  // v row
  yv = T(0);
  if (i >= 1 && i <= nx) {
    if (j >= 1 && j <= g.jmax()) {
      const T adv = with_adv ? adv_v_at<T>(f[MV_UA], f[MV_VA], f[MV_RC], f[MV_RU], Xv, mdu, mdv, amp, i, j, idx, idy)
                             : T(0);
      const T vis = visc_v_at<T>(Xu, Xv, f[MV_KA], f[MV_ZE], f[MV_ET], i, j, idx, idy);
      const T gp = (Xp(i, j + 1) - Xp(i, j)) * idy;
      yv = (f[MV_RV](i, j) / dt) * Xv(i, j) + adv + vis + gp;
      if (c.pen_v) yv = yv + c.pen_v[k] * Xv(i, j);
    } else if (!g.py && (j == 0 || j == ny)) {
      yv = Xv(i, j);
    }
  }
  // p row: op_divergence (mod_operators.f90:34-53)
  yp = T(0);
  if (i >= 1 && i <= nx && j >= 1 && j <= ny) yp = (Xu(i, j) - Xu(i - 1, j)) * idx + (Xv(i, j) - Xv(i, j - 1)) * idy;
}
template <typename T>
__device__ __forceinline__ void mv_gviews(const Geo& g, const Coefs<T>& c, const T* Xu, const T* Xv, const T* Xp,
                                          GView<T>* f) {
  f[MV_XU] = gview(g, Xu); f[MV_XV] = gview(g, Xv); f[MV_XP] = gview(g, Xp);
  f[MV_UA] = gview(g, c.u_adv); f[MV_VA] = gview(g, c.v_adv); f[MV_RC] = gview(g, c.rho_c);
  f[MV_RU] = gview(g, c.rho_u); f[MV_RV] = gview(g, c.rho_v); f[MV_KA] = gview(g, c.kappa);
  f[MV_ZE] = gview(g, c.zeta); f[MV_ET] = gview(g, c.eta);
}
// the operator at (i, j) with every field read from global memory
template <typename T>
__device__ __forceinline__ void matvec_at(const Geo& g, const Coefs<T>& c, const T* __restrict__ Xu,
                                          const T* __restrict__ Xv, const T* __restrict__ Xp, T* __restrict__ Yu,
                                          T* __restrict__ Yv, T* __restrict__ Yp, T dt, int with_adv, int k, int i,
                                          int j) {
  GView<T> f[MV_N];
  mv_gviews(g, c, Xu, Xv, Xp, f);
  T yu, yv, yp;
  matvec_vals<T>(g, f, c, dt, with_adv, k, i, j, yu, yv, yp);
  Yu[k] = yu;
  Yv[k] = yv;
  Yp[k] = yp;
}
template <typename T>
__global__ void k_matvec(Geo g, Coefs<T> c, const T* __restrict__ Xu, const T* __restrict__ Xv,
                         const T* __restrict__ Xp, T* __restrict__ Yu, T* __restrict__ Yv,
                         T* __restrict__ Yp, T dt, int with_adv, const int* active,
                         unsigned long long* count) {
  if (active && !*active) return;
  if (count && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0 && threadIdx.y == 0) atomicAdd(count, 1ull);
  FUGU_BOX_IJ
  matvec_at<T>(g, c, Xu, Xv, Xp, Yu, Yv, Yp, dt, with_adv, k, i, j);
}

// ----------------------------------------------- staged stencil tiles
// A CTA of 256 threads stages a tile of MT_TX x TY outputs of the padded box
// plus a ring of one (widened to four columns either side, so that every
// row segment starts on a 16-byte boundary) for each field it reads with a
// stencil, by 16-byte asynchronous copies (cp.async) straight into shared
// memory, then computes the tile from there: each field element is read
// from HBM once and the stencil's neighbour reads hit shared memory.  Parts
// of a staged segment outside the padded box are zero-filled (no global
// read); the formulas never use them.  Each thread computes TY / 8
// consecutive rows of one column, so a row's neighbours above and below come
// from the same thread's reads.  Needs 16-byte aligned field bases and
// P * sizeof(T) a multiple of 16 (every buffer of the uniform layout).
constexpr int MT_TX = 32;
constexpr int MT_TPB = 256;
template <int TY>
struct MtShape {
  static constexpr int W = MT_TX + 8;  // staged columns: ii0 - 4 .. ii0 + MT_TX + 3
  static constexpr int H = TY + 2;     // staged rows: jj0 - 1 .. jj0 + TY
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool ok) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(ok ? 16 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// stage rows jj0 - 1 .. jj0 + TY and columns ii0 - 4 .. ii0 + MT_TX + 3 of
// field src into dst (H x W elements)
template <typename T, int TY>
__device__ __forceinline__ void mt_stage(const Geo& g, const T* src, T* dst, int ii0, int jj0) {
  constexpr int W = MtShape<TY>::W, H = MtShape<TY>::H, VPC = 16 / sizeof(T), CPR = W / VPC;
  for (int q = threadIdx.x; q < H * CPR; q += MT_TPB) {
    const int r = q / CPR, cc = q % CPR;
    const int ii = ii0 - 4 + cc * VPC, jj = jj0 - 1 + r;
    const bool ok = ii >= 0 && ii < g.P && jj >= 0 && jj < g.R;
    cp_async16(dst + r * W + cc * VPC, ok ? src + ii + (long)jj * g.P : src, ok);
  }
}
template <typename T, int TY>
constexpr int mt_matvec_smem() { return MV_N * MtShape<TY>::H * MtShape<TY>::W * (int)sizeof(T); }

// the coupled operator on the tile (bx, by) of the box (see k_matvec)
template <typename T, int TY>
__device__ __forceinline__ void matvec_tile(const Geo& g, const Coefs<T>& c, const T* Xu, const T* Xv, const T* Xp,
                                            T* __restrict__ Yu, T* __restrict__ Yv, T* __restrict__ Yp, T dt,
                                            int with_adv, int bx, int by, T* sm) {
  constexpr int W = MtShape<TY>::W, H = MtShape<TY>::H, RPT = TY / 8;
  static_assert(TY % 8 == 0 && 16 % sizeof(T) == 0, "tile shape");
  const int ii0 = bx * MT_TX, jj0 = by * TY;
  const T* src[MV_N] = {Xu, Xv, Xp, c.u_adv, c.v_adv, c.rho_c, c.rho_u, c.rho_v, c.kappa, c.zeta, c.eta};
#pragma unroll
  for (int q = 0; q < MV_N; ++q) mt_stage<T, TY>(g, src[q], sm + q * H * W, ii0, jj0);
  cp_async_wait_all();
  __syncthreads();
  SView<T, W> f[MV_N];
#pragma unroll
  for (int q = 0; q < MV_N; ++q) f[q] = SView<T, W>{sm + q * H * W, ii0 - 6, jj0 - 3};
  const int ii = ii0 + threadIdx.x % MT_TX;
#pragma unroll
  for (int r = 0; r < RPT; ++r) {
    const int jj = jj0 + (threadIdx.x / MT_TX) * RPT + r;
    if (ii < g.P && jj < g.R) {
      const int k = ii + jj * g.P;
      T yu, yv, yp;
      matvec_vals<T>(g, f, c, dt, with_adv, k, ii - 2, jj - 2, yu, yv, yp);
      Yu[k] = yu;
      Yv[k] = yv;
      Yp[k] = yp;
    }
  }
}
template <typename T, int TY>
__global__ void __launch_bounds__(MT_TPB) k_matvec_tile(Geo g, Coefs<T> c, const T* Xu, const T* Xv, const T* Xp,
                                                        T* __restrict__ Yu, T* __restrict__ Yv, T* __restrict__ Yp,
                                                        T dt, int with_adv, const int* active,
                                                        unsigned long long* count) {
  if (active && !*active) return;
  if (count && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) atomicAdd(count, 1ull);
  extern __shared__ __align__(16) unsigned char mt_smem[];
  matvec_tile<T, TY>(g, c, Xu, Xv, Xp, Yu, Yv, Yp, dt, with_adv, blockIdx.x, blockIdx.y, (T*)mt_smem);
}

// The individual operators of mod_operators.f90 (routine-level entries).
__global__ void k_op_divergence(Geo g, const double* u, const double* v, double* div) {
  FUGU_BOX_IJ
  double d = 0.0;
  if (i >= 1 && i <= g.nx && j >= 1 && j <= g.ny)
    d = (u[k] - u[g.at(i - 1, j)]) * g.idx + (v[k] - v[g.at(i, j - 1)]) * g.idy;
  div[k] = d;
}
__global__ void k_op_grad(Geo g, const double* p, double* gu, double* gv) {
  FUGU_BOX_IJ
  gu[k] = (j >= 1 && j <= g.ny && i >= 0 && i <= g.nx) ? (p[g.at(i + 1, j)] - p[k]) * g.idx : 0.0;
  gv[k] = (i >= 1 && i <= g.nx && j >= 0 && j <= g.ny) ? (p[g.at(i, j + 1)] - p[k]) * g.idy : 0.0;
}
__global__ void k_op_visc(Geo g, const double* u, const double* v, const double* kap,
                          const double* zeta, const double* eta, double* vu, double* vv) {
  FUGU_BOX_IJ
  const GView<double> U = gview(g, u), Vv = gview(g, v), K = gview(g, kap), Z = gview(g, zeta), E = gview(g, eta);
  vu[k] = (j >= 1 && j <= g.ny && i >= 0 && i <= g.nx) ? visc_u_at<double>(U, Vv, K, Z, E, i, j, g.idx, g.idy) : 0.0;
  vv[k] = (i >= 1 && i <= g.nx && j >= 0 && j <= g.ny) ? visc_v_at<double>(U, Vv, K, Z, E, i, j, g.idx, g.idy) : 0.0;
}
__global__ void k_op_adv(Geo g, Coefs<double> c, const double* u, const double* v, double* au, double* av) {
  FUGU_BOX_IJ
  const GView<double> ua = gview(g, c.u_adv), va = gview(g, c.v_adv), rc = gview(g, c.rho_c);
  const GView<double> ru = gview(g, c.rho_u), rv = gview(g, c.rho_v), md_u = gview(g, c.mdot_u), md_v = gview(g, c.mdot_v);
  const bool amp = c.mdot_u != nullptr;
  au[k] = (j >= 1 && j <= g.ny && i >= 1 && i <= g.imax())
              ? adv_u_at<double>(ua, va, rc, rv, gview(g, u), md_u, md_v, amp, i, j, g.idx, g.idy) : 0.0;
  av[k] = (i >= 1 && i <= g.nx && j >= 1 && j <= g.jmax())
              ? adv_v_at<double>(ua, va, rc, ru, gview(g, v), md_u, md_v, amp, i, j, g.idx, g.idy) : 0.0;
}

// ------------------------------------------------------------ PCD pieces
// Poisson face coefficients with zero flux through walls
// (mod_subsolvers.f90:61-87): cx on u faces (i = 0..nx), cy on v faces
// (j = 0..ny), and the Jacobi inverse diagonal at cells.
template <typename T>
__device__ __forceinline__ void poisson_coefs_at(const Geo& g, const double* rho_u, const double* rho_v, T* cx,
                                                 T* cy, T* dinv, int k, int i, int j) {
  const int nx = g.nx, ny = g.ny;
  T vx = T(0), vy = T(0), di = T(1);
  if (j >= 1 && j <= ny && i >= 0 && i <= nx) {
    double cxv = g.idx2 / rho_u[k];
    if (!g.px && (i == 0 || i == nx)) cxv = 0.0;
    vx = T(cxv);
  }
  if (i >= 1 && i <= nx && j >= 0 && j <= ny) {
    double cyv = g.idy2 / rho_v[k];
    if (!g.py && (j == 0 || j == ny)) cyv = 0.0;
    vy = T(cyv);
  }
  if (i >= 1 && i <= nx && j >= 1 && j <= ny) {
    double cE = g.idx2 / rho_u[k], cW = g.idx2 / rho_u[g.at(i - 1, j)];
    double cN = g.idy2 / rho_v[k], cS = g.idy2 / rho_v[g.at(i, j - 1)];
    if (!g.px) { if (i == 1) cW = 0.0; if (i == nx) cE = 0.0; }
    if (!g.py) { if (j == 1) cS = 0.0; if (j == ny) cN = 0.0; }
    const double d = cE + cW + cN + cS;
    di = T(d > 1.0e-14 ? 1.0 / d : 1.0);
  }
  cx[k] = vx;
  cy[k] = vy;
  dinv[k] = di;
}
template <typename T>
__global__ void k_poisson_coefs(Geo g, const double* rho_u, const double* rho_v, T* cx, T* cy, T* dinv) {
  FUGU_BOX_IJ
  poisson_coefs_at<T>(g, rho_u, rho_v, cx, cy, dinv, k, i, j);
}

// PCD Schur step r_p = -((1/dt) phi + u.grad phi) (mod_pcd_precond.f90:54-62);
// r_p is zero outside the interior (as after r_p = zero).
// Each PCD step is an element function plus a thin whole-box kernel around it.
template <typename T, typename V>
__device__ __forceinline__ T pcd_schur_vals(const Geo& g, int i, int j, const V& phi, const V& ua, const V& va,
                                            T inv_dt, const V& kap, const V& zp, T visc) {
  T r = T(0);
  if (i >= 1 && i <= g.nx && j >= 1 && j <= g.ny) {
    const T h = T(0.5);
    const T uavg = h * (ua(i, j) + ua(i - 1, j));
    const T vavg = h * (va(i, j) + va(i, j - 1));
    const T conv = uavg * (phi(i + 1, j) - phi(i - 1, j)) * (h * T(g.idx)) +
                   vavg * (phi(i, j + 1) - phi(i, j - 1)) * (h * T(g.idy));
    r = -(inv_dt * phi(i, j) + conv);
    // extension (visc > 0): the viscous Cahouet-Chabard part, visc * mu_c * z_p
    if (visc != T(0)) r = r - ((visc * T(0.5)) * kap(i, j)) * zp(i, j);
  }
  return r;
}
template <typename T>
__device__ __forceinline__ T pcd_schur_at(const Geo& g, int k, int i, int j, const T* phi, const T* ua,
                                          const T* va, T inv_dt, const T* kap, const T* zp, T visc) {
  (void)k;
  return pcd_schur_vals<T>(g, i, j, gview(g, phi), gview(g, ua), gview(g, va), inv_dt, gview(g, kap), gview(g, zp),
                           visc);
}
template <typename T>
__global__ void k_pcd_schur(Geo g, const T* phi, const T* ua, const T* va, T* rp, T inv_dt, const T* kap,
                            const T* zp, T visc, const int* active) {
  if (active && !*active) return;
  FUGU_BOX_IJ
  rp[k] = pcd_schur_at<T>(g, k, i, j, phi, ua, va, inv_dt, kap, zp, visc);
}

// velocity residual update z - B_p^T r_p (mod_pcd_precond.f90:66-84)
template <typename T, typename V>
__device__ __forceinline__ void pcd_zwork_vals(const Geo& g, int i, int j, T zu, T zv, const V& rp, T& a, T& b) {
  const int nx = g.nx, ny = g.ny;
  a = T(0);
  b = T(0);
  if (j >= 1 && j <= ny) {
    if (i >= 1 && i <= nx - 1) a = zu - (rp(i + 1, j) - rp(i, j)) * T(g.idx);
    else if (i == 0 || i == nx) a = zu;
  }
  if (i >= 1 && i <= nx) {
    if (j >= 1 && j <= ny - 1) b = zv - (rp(i, j + 1) - rp(i, j)) * T(g.idy);
    else if (j == 0 || j == ny) b = zv;
  }
}
template <typename T>
__device__ __forceinline__ void pcd_zwork_at(const Geo& g, int k, int i, int j, const T* zu, const T* zv,
                                             const T* rp, T* zuw, T* zvw) {
  T a, b;
  pcd_zwork_vals<T>(g, i, j, zu[k], zv[k], gview(g, rp), a, b);
  zuw[k] = a;
  zvw[k] = b;
}
template <typename T>
__global__ void k_pcd_zwork(Geo g, const T* zu, const T* zv, const T* rp, T* zuw, T* zvw, const int* active) {
  if (active && !*active) return;
  FUGU_BOX_IJ
  pcd_zwork_at<T>(g, k, i, j, zu, zv, rp, zuw, zvw);
}

// cross term from r_v into the u residual (mod_pcd_precond.f90:91-98)
template <typename T, typename V>
__device__ __forceinline__ T pcd_cross_vals(const Geo& g, int i, int j, const V& eta, const V& rv, T zuw) {
  if (j >= 1 && j <= g.ny && i >= 1 && i <= g.nx - 1) {
    const T idx = T(g.idx), idy = T(g.idy);
    const T cross = -idy * (eta(i, j) * (rv(i + 1, j) - rv(i, j)) * idx -
                            eta(i, j - 1) * (rv(i + 1, j - 1) - rv(i, j - 1)) * idx);
    return zuw - cross;
  }
  return zuw;
}
template <typename T>
__device__ __forceinline__ void pcd_cross_at(const Geo& g, int k, int i, int j, const T* eta, const T* rv,
                                             T* zuw) {
  if (j >= 1 && j <= g.ny && i >= 1 && i <= g.nx - 1)
    zuw[k] = pcd_cross_vals<T>(g, i, j, gview(g, eta), gview(g, rv), zuw[k]);
}
template <typename T>
__global__ void k_pcd_cross(Geo g, const T* eta, const T* rv, T* zuw, const int* active) {
  if (active && !*active) return;
  FUGU_BOX_IJ
  pcd_cross_at<T>(g, k, i, j, eta, rv, zuw);
}

// One damped-Jacobi sweep of solve_helmholtz_u (mod_subsolvers.f90:284-306):
// un = Jacobi(uo) on owned faces, rhs on wall faces, uo elsewhere (the
// reference's u_old = u_sol copy).  uo, kap, zeta and eta (read with a
// stencil) through views; rhs, rho_u and pen (one value per face) at k.
template <typename T, typename V>
__device__ __forceinline__ T jacobi_u_vals(const Geo& g, int k, int i, int j, const V& uo, const V& kap,
                                           const V& zeta, const V& eta, const T* rhs, const T* rho_u, const T* pen,
                                           T dt, T om) {
  const int nx = g.nx, ny = g.ny;
  T val = uo(i, j);
  if (j >= 1 && j <= ny) {
    if (i >= 1 && i <= g.imax()) {
      const T ix2 = T(g.idx2), iy2 = T(g.idy2);
      const T cE = kap(i + 1, j) * ix2;
      const T cW = kap(i, j) * ix2;
      const T cN = (zeta(i, j) - eta(i, j)) * iy2;
      const T cS = (zeta(i, j - 1) - eta(i, j - 1)) * iy2;
      T diag = (rho_u[k] / dt) + cE + cW + cN + cS;
      if (pen) diag = diag + pen[k];
      const T off = madd(cS, uo(i, j - 1), madd(cN, uo(i, j + 1), madd(cW, uo(i - 1, j), cE * uo(i + 1, j))));
      if (diag > T(1.0e-15)) val = madd(T(1) - om, uo(i, j), om * ((rhs[k] + off) / diag));
    } else if (!g.px && (i == 0 || i == nx)) {
      val = rhs[k];
    }
  }
  return val;
}
template <typename T>
__device__ __forceinline__ T jacobi_u_at(const Geo& g, int k, int i, int j, const T* uo, const T* rhs,
                                         const T* rho_u, const T* kap, const T* zeta, const T* eta, const T* pen,
                                         T dt, T om) {
  return jacobi_u_vals<T>(g, k, i, j, gview(g, uo), gview(g, kap), gview(g, zeta), gview(g, eta), rhs, rho_u, pen, dt,
                          om);
}
template <typename T>
__global__ void k_jacobi_u(Geo g, const T* uo, T* un, const T* rhs, const T* rho_u, const T* kap,
                           const T* zeta, const T* eta, const T* pen, T dt, T om, const int* active) {
  if (active && !*active) return;
  FUGU_BOX_IJ
  un[k] = jacobi_u_at<T>(g, k, i, j, uo, rhs, rho_u, kap, zeta, eta, pen, dt, om);
}

// One damped-Jacobi sweep of solve_helmholtz_v (mod_subsolvers.f90:346-369)
template <typename T, typename V>
__device__ __forceinline__ T jacobi_v_vals(const Geo& g, int k, int i, int j, const V& vo, const V& kap,
                                           const V& zeta, const V& eta, const T* rhs, const T* rho_v, const T* pen,
                                           T dt, T om) {
  const int nx = g.nx, ny = g.ny;
  T val = vo(i, j);
  if (i >= 1 && i <= nx) {
    if (j >= 1 && j <= g.jmax()) {
      const T ix2 = T(g.idx2), iy2 = T(g.idy2);
      const T cE = (zeta(i, j) - eta(i, j)) * ix2;
      const T cW = (zeta(i - 1, j) - eta(i - 1, j)) * ix2;
      const T cN = kap(i, j + 1) * iy2;
      const T cS = kap(i, j) * iy2;
      T diag = (rho_v[k] / dt) + cE + cW + cN + cS;
      if (pen) diag = diag + pen[k];
      const T off = madd(cS, vo(i, j - 1), madd(cN, vo(i, j + 1), madd(cW, vo(i - 1, j), cE * vo(i + 1, j))));
      if (diag > T(1.0e-15)) val = madd(T(1) - om, vo(i, j), om * ((rhs[k] + off) / diag));
    } else if (!g.py && (j == 0 || j == ny)) {
      val = rhs[k];
    }
  }
  return val;
}
template <typename T>
__device__ __forceinline__ T jacobi_v_at(const Geo& g, int k, int i, int j, const T* vo, const T* rhs,
                                         const T* rho_v, const T* kap, const T* zeta, const T* eta, const T* pen,
                                         T dt, T om) {
  return jacobi_v_vals<T>(g, k, i, j, gview(g, vo), gview(g, kap), gview(g, zeta), gview(g, eta), rhs, rho_v, pen, dt,
                          om);
}
template <typename T>
__global__ void k_jacobi_v(Geo g, const T* vo, T* vn, const T* rhs, const T* rho_v, const T* kap,
                           const T* zeta, const T* eta, const T* pen, T dt, T om, const int* active) {
  if (active && !*active) return;
  FUGU_BOX_IJ
  vn[k] = jacobi_v_at<T>(g, k, i, j, vo, rhs, rho_v, kap, zeta, eta, pen, dt, om);
}

// One colour pass of the red-black SOR smoother (extension, pcd_smoother = 1):
// the faces with (i + j) & 1 == col take the damped-Jacobi formula above with
// omega = pcd_sor_omega, reading u in place.  Every neighbour of such a face
// has the other colour (ghosts were refreshed before the pass and are not
// written), so the pass is race-free and order-independent.
// the faces one colour pass of the u / v smoother updates
__device__ __forceinline__ bool rbsor_u_face(const Geo& g, int i, int j, int col) {
  if (j < 1 || j > g.ny || ((i + j) & 1) != col) return false;
  return (i >= 1 && i <= g.imax()) || (!g.px && (i == 0 || i == g.nx));
}
__device__ __forceinline__ bool rbsor_v_face(const Geo& g, int i, int j, int col) {
  if (i < 1 || i > g.nx || ((i + j) & 1) != col) return false;
  return (j >= 1 && j <= g.jmax()) || (!g.py && (j == 0 || j == g.ny));
}
template <typename T>
__global__ void k_rbsor_u(Geo g, T* u, const T* rhs, const T* rho_u, const T* kap, const T* zeta, const T* eta,
                          const T* pen, T dt, T om, int col, const int* active) {
  if (active && !*active) return;
  FUGU_BOX_IJ
  if (!rbsor_u_face(g, i, j, col)) return;
  u[k] = jacobi_u_at<T>(g, k, i, j, u, rhs, rho_u, kap, zeta, eta, pen, dt, om);
}
template <typename T>
__global__ void k_rbsor_v(Geo g, T* v, const T* rhs, const T* rho_v, const T* kap, const T* zeta, const T* eta,
                          const T* pen, T dt, T om, int col, const int* active) {
  if (active && !*active) return;
  FUGU_BOX_IJ
  if (!rbsor_v_face(g, i, j, col)) return;
  v[k] = jacobi_v_at<T>(g, k, i, j, v, rhs, rho_v, kap, zeta, eta, pen, dt, om);
}

// ------------------------------------------------- vectorised row kernels
// The damped-Jacobi sweep and the PCD's Schur, residual and cross steps with
// VW = 16 / sizeof(T) consecutive elements of one box row per thread (four
// floats or two doubles): each array is read and written with 16-byte vector
// accesses, the rows above and below with vector loads too, and the one
// neighbour either side of the segment with a scalar load.  The values go to
// a window of registers (RView) that the element functions above read
// through, so every face gets the bits of the one-thread-per-face kernels
// with a quarter (FP32) or half (FP64) of the load instructions.  P is a
// multiple of 16, so a segment starting at a multiple of VW is 16-byte
// aligned when the array is (the host checks every pointer before taking
// these kernels).  Block VEC_TX x VEC_TY threads covers VEC_TX * VW columns.
constexpr int VEC_TX = 32, VEC_TY = 8;
// rows j0 - 1, j0, j0 + 1 (slots 0..2) of the columns i0 - 1 .. i0 + W
template <typename T, int W>
struct RView {
  T v[3][W + 2];
  int i0, j0;
  __device__ __forceinline__ T operator()(int i, int j) const { return v[j - j0 + 1][i - i0 + 1]; }
};
// slot r of the window from the row segment starting at box index k, with
// the left / right neighbours when asked (and only then read)
template <typename T, int W>
__device__ __forceinline__ void rv_row(RView<T, W>& w, int r, const T* p, long k, bool left, bool right) {
  ldv(p + k, &w.v[r][1]);
  w.v[r][0] = left ? p[k - 1] : T(0);
  w.v[r][W + 1] = right ? p[k + W] : T(0);
}
#define FUGU_VEC_SEG                                                        \
  constexpr int W = VecW<T>::value;                                         \
  const int ii0 = (blockIdx.x * blockDim.x + threadIdx.x) * W;             \
  const int jj = blockIdx.y * blockDim.y + threadIdx.y;                    \
  if (ii0 >= g.P || jj >= g.R) return;                                      \
  const int i0 = ii0 - 2, j = jj - 2;                                       \
  const long P = g.P;                                                       \
  const long k0 = ii0 + jj * P;                                             \
  const bool lft = ii0 > 0, rgt = ii0 + W < g.P;                            \
  (void)lft; (void)rgt;

// one damped-Jacobi sweep (k_jacobi_u for comp 0, k_jacobi_v for comp 1)
template <typename T>
__global__ void __launch_bounds__(VEC_TX * VEC_TY)
    k_jacobi_vec(Geo g, int comp, const T* __restrict__ uo, T* __restrict__ un, const T* __restrict__ rhs,
                 const T* __restrict__ rho, const T* __restrict__ kap, const T* __restrict__ zeta,
                 const T* __restrict__ eta, const T* __restrict__ pen, T dt, T om, const int* active) {
  if (active && !*active) return;
  FUGU_VEC_SEG
  RView<T, W> U, K, Z, E;
  U.i0 = K.i0 = Z.i0 = E.i0 = i0;
  U.j0 = K.j0 = Z.j0 = E.j0 = j;
  T rv[W], bv[W], pv[W];
  rv_row(U, 1, uo, k0, lft, rgt);
  ldv(rhs + k0, rv);
  ldv(rho + k0, bv);
  if (pen) ldv(pen + k0, pv);
  // the stencil is read only on owned rows (j in 1..ny for u, 1..jmax for v)
  if (j >= 1 && j <= (comp == 0 ? g.ny : g.jmax())) {
    rv_row(U, 0, uo, k0 - P, lft, rgt);
    rv_row(U, 2, uo, k0 + P, lft, rgt);
    if (comp == 0) {  // kap(i, j), kap(i + 1, j); zeta, eta at rows j and j - 1
      rv_row(K, 1, kap, k0, false, rgt);
      ldv(zeta + k0, &Z.v[1][1]);
      ldv(zeta + k0 - P, &Z.v[0][1]);
      ldv(eta + k0, &E.v[1][1]);
      ldv(eta + k0 - P, &E.v[0][1]);
    } else {  // kap at rows j and j + 1; zeta, eta at (i, j) and (i - 1, j)
      ldv(kap + k0, &K.v[1][1]);
      ldv(kap + k0 + P, &K.v[2][1]);
      rv_row(Z, 1, zeta, k0, lft, false);
      rv_row(E, 1, eta, k0, lft, false);
    }
  }
  T out[W];
#pragma unroll
  for (int e = 0; e < W; ++e)
    out[e] = comp == 0 ? jacobi_u_vals<T>(g, e, i0 + e, j, U, K, Z, E, rv, bv, pen ? pv : nullptr, dt, om)
                       : jacobi_v_vals<T>(g, e, i0 + e, j, U, K, Z, E, rv, bv, pen ? pv : nullptr, dt, om);
  stv(un + k0, out);
}

// the PCD's Schur step (k_pcd_schur)
template <typename T>
__global__ void __launch_bounds__(VEC_TX * VEC_TY)
    k_pcd_schur_vec(Geo g, const T* __restrict__ phi, const T* __restrict__ ua, const T* __restrict__ va,
                    T* __restrict__ rp, T inv_dt, const T* __restrict__ kap, const T* __restrict__ zp, T visc,
                    const int* active) {
  if (active && !*active) return;
  FUGU_VEC_SEG
  RView<T, W> F, A, B, K, Z;
  F.i0 = A.i0 = B.i0 = K.i0 = Z.i0 = i0;
  F.j0 = A.j0 = B.j0 = K.j0 = Z.j0 = j;
  T out[W];
  if (j >= 1 && j <= g.ny) {
    rv_row(F, 0, phi, k0 - P, false, false);
    rv_row(F, 1, phi, k0, lft, rgt);
    rv_row(F, 2, phi, k0 + P, false, false);
    rv_row(A, 1, ua, k0, lft, false);
    ldv(va + k0, &B.v[1][1]);
    ldv(va + k0 - P, &B.v[0][1]);
    if (visc != T(0)) {
      ldv(kap + k0, &K.v[1][1]);
      ldv(zp + k0, &Z.v[1][1]);
    }
#pragma unroll
    for (int e = 0; e < W; ++e) out[e] = pcd_schur_vals<T>(g, i0 + e, j, F, A, B, inv_dt, K, Z, visc);
  } else {
#pragma unroll
    for (int e = 0; e < W; ++e) out[e] = T(0);
  }
  stv(rp + k0, out);
}

// the PCD's velocity residual update (k_pcd_zwork)
template <typename T>
__global__ void __launch_bounds__(VEC_TX * VEC_TY)
    k_pcd_zwork_vec(Geo g, const T* __restrict__ zu, const T* __restrict__ zv, const T* __restrict__ rp,
                    T* __restrict__ zuw, T* __restrict__ zvw, const int* active) {
  if (active && !*active) return;
  FUGU_VEC_SEG
  RView<T, W> R;
  R.i0 = i0;
  R.j0 = j;
  T a[W], b[W], zuv[W], zvv[W];
  ldv(zu + k0, zuv);
  ldv(zv + k0, zvv);
  // rp(i, j), rp(i + 1, j) on the rows j in 1..ny; rp(i, j + 1) on 1..ny-1
  if (j >= 1 && j <= g.ny) {
    rv_row(R, 1, rp, k0, false, rgt);
    if (j <= g.ny - 1) ldv(rp + k0 + P, &R.v[2][1]);
  }
#pragma unroll
  for (int e = 0; e < W; ++e) pcd_zwork_vals<T>(g, i0 + e, j, zuv[e], zvv[e], R, a[e], b[e]);
  stv(zuw + k0, a);
  stv(zvw + k0, b);
}

// the PCD's cross term from r_v into the u residual (k_pcd_cross)
template <typename T>
__global__ void __launch_bounds__(VEC_TX * VEC_TY)
    k_pcd_cross_vec(Geo g, const T* __restrict__ eta, const T* __restrict__ rv, T* __restrict__ zuw,
                    const int* active) {
  if (active && !*active) return;
  FUGU_VEC_SEG
  if (j < 1 || j > g.ny) return;  // zuw is left as it is outside the rows 1..ny
  RView<T, W> E, V;
  E.i0 = V.i0 = i0;
  E.j0 = V.j0 = j;
  ldv(eta + k0, &E.v[1][1]);
  ldv(eta + k0 - P, &E.v[0][1]);
  rv_row(V, 1, rv, k0, false, rgt);
  rv_row(V, 0, rv, k0 - P, false, rgt);
  T z[W];
  ldv(zuw + k0, z);
#pragma unroll
  for (int e = 0; e < W; ++e) z[e] = pcd_cross_vals<T>(g, i0 + e, j, E, V, z[e]);
  stv(zuw + k0, z);
}
#undef FUGU_VEC_SEG

// ------------------------------------------------- fused red-black SOR sweep
// One whole red-black SOR sweep (both colour passes) of one velocity
// component of a wall-bounded case, per tile of RB_TX x RB_TY faces, from
// the buffer uin into the buffer uout.  The tile and a ring of two faces of
// uin are staged in shared memory; the coefficients of the tile and a ring of
// one (cE, cW, cN, cS, the diagonal and the right-hand side of jacobi_u_at /
// jacobi_v_at) are formed once per face.  The red faces (i + j even) of the
// tile and of its ring are updated there, then the black faces of the tile
// from those red values, and every element of the tile goes to uout.  Each
// update is jacobi_u_at / jacobi_v_at's formula with its operand order, so a
// sweep gives the bits of the two in-place colour-pass launches (k_rbsor_u /
// k_rbsor_v) it replaces while it reads and writes each array once instead
// of twice.  Two buffers, because a tile reads its ring while the
// neighbouring tiles of the same launch write theirs: in place, it could read
// a value its neighbour has already updated.  Callers alternate the buffers
// and copy back after an odd number of sweeps.  A periodic case refreshes its
// ghosts between the two colours, so it keeps the two launches.
constexpr int RB_TX = 32, RB_TY = 16;
constexpr int RB_SX = RB_TX + 4, RB_SY = RB_TY + 4;  // with the ring of two
constexpr int RB_CX = RB_TX + 2, RB_CY = RB_TY + 2;  // with the ring of one
constexpr int RB_TPB = 256;

template <typename T>
struct RbSmem {
  T u[RB_SY][RB_SX];
  T cE[RB_CY][RB_CX], cW[RB_CY][RB_CX], cN[RB_CY][RB_CX], cS[RB_CY][RB_CX], dg[RB_CY][RB_CX], rh[RB_CY][RB_CX];
  unsigned char kind[RB_CY][RB_CX];  // 0 not updated, 1 owned face (Jacobi formula), 2 wall face (= rhs)
};

// tile (tx, ty) of component comp (0 u, 1 v); needs !g.px && !g.py
template <typename T>
__device__ __forceinline__ void rbsor_sweep_tile(const Geo& g, int comp, int tx, int ty, const T* uin, T* uout,
                                                 const T* rhs, const T* rho, const T* kap, const T* zeta,
                                                 const T* eta, const T* pen, T dt, T om, RbSmem<T>& sm) {
  const int ii0 = tx * RB_TX - 2, jj0 = ty * RB_TY - 2;  // padded-box coordinates of sm.u[0][0]
  const int nx = g.nx, ny = g.ny;
  const T ix2 = T(g.idx2), iy2 = T(g.idy2);
  for (int q = threadIdx.x; q < RB_SX * RB_SY; q += blockDim.x) {
    const int a = q % RB_SX, b = q / RB_SX;
    const int ii = ii0 + a, jj = jj0 + b;
    sm.u[b][a] = (ii >= 0 && ii < g.P && jj >= 0 && jj < g.R) ? uin[ii + jj * g.P] : T(0);
  }
  for (int q = threadIdx.x; q < RB_CX * RB_CY; q += blockDim.x) {
    const int a = q % RB_CX, b = q / RB_CX;
    const int ii = ii0 + 1 + a, jj = jj0 + 1 + b;
    const int i = ii - 2, j = jj - 2;
    unsigned char kd = 0;
    if (ii >= 0 && ii < g.P && jj >= 0 && jj < g.R) {
      const int k = ii + jj * g.P;
      if (comp == 0 && j >= 1 && j <= ny) {
        if (i >= 1 && i <= nx - 1) {
          kd = 1;
          const T e = kap[g.at(i + 1, j)] * ix2, w = kap[k] * ix2;
          const T nn = (zeta[k] - eta[k]) * iy2, ss = (zeta[g.at(i, j - 1)] - eta[g.at(i, j - 1)]) * iy2;
          T d = (rho[k] / dt) + e + w + nn + ss;
          if (pen) d = d + pen[k];
          sm.cE[b][a] = e; sm.cW[b][a] = w; sm.cN[b][a] = nn; sm.cS[b][a] = ss; sm.dg[b][a] = d;
        } else if (i == 0 || i == nx) {
          kd = 2;
        }
      } else if (comp == 1 && i >= 1 && i <= nx) {
        if (j >= 1 && j <= ny - 1) {
          kd = 1;
          const T e = (zeta[k] - eta[k]) * ix2, w = (zeta[g.at(i - 1, j)] - eta[g.at(i - 1, j)]) * ix2;
          const T nn = kap[g.at(i, j + 1)] * iy2, ss = kap[k] * iy2;
          T d = (rho[k] / dt) + e + w + nn + ss;
          if (pen) d = d + pen[k];
          sm.cE[b][a] = e; sm.cW[b][a] = w; sm.cN[b][a] = nn; sm.cS[b][a] = ss; sm.dg[b][a] = d;
        } else if (j == 0 || j == ny) {
          kd = 2;
        }
      }
      if (kd) sm.rh[b][a] = rhs[k];
    }
    sm.kind[b][a] = kd;
  }
  __syncthreads();
  // red on the tile and its ring, then black on the tile
  for (int col = 0; col < 2; ++col) {
    const int lo = col == 0 ? 0 : 1, cx = col == 0 ? RB_CX : RB_TX, cy = col == 0 ? RB_CY : RB_TY;
    for (int q = threadIdx.x; q < cx * cy; q += blockDim.x) {
      const int a = lo + q % cx, b = lo + q / cx;  // coefficient-array indices
      const unsigned char kd = sm.kind[b][a];
      const int i = ii0 + a - 1, j = jj0 + b - 1;
      if (!kd || ((i + j) & 1) != col) continue;
      const int ua = a + 1, ub = b + 1;  // the same face in sm.u
      if (kd == 2) {
        sm.u[ub][ua] = sm.rh[b][a];
        continue;
      }
      const T d = sm.dg[b][a];
      if (d > T(1.0e-15)) {
        const T off = madd(sm.cS[b][a], sm.u[ub - 1][ua],
                           madd(sm.cN[b][a], sm.u[ub + 1][ua], madd(sm.cW[b][a], sm.u[ub][ua - 1],
                                                                  sm.cE[b][a] * sm.u[ub][ua + 1])));
        sm.u[ub][ua] = madd(T(1) - om, sm.u[ub][ua], om * ((sm.rh[b][a] + off) / d));
      }
    }
    __syncthreads();
  }
  for (int q = threadIdx.x; q < RB_TX * RB_TY; q += blockDim.x) {
    const int a = 1 + q % RB_TX, b = 1 + q / RB_TX;
    const int ii = ii0 + 1 + a, jj = jj0 + 1 + b;
    if (ii < g.P && jj < g.R) uout[ii + jj * g.P] = sm.u[b + 1][a + 1];
  }
}
template <typename T>
__global__ void __launch_bounds__(RB_TPB) k_rbsor_sweep(Geo g, int comp, const T* uin, T* uout, const T* rhs,
                                                        const T* rho, const T* kap, const T* zeta, const T* eta,
                                                        const T* pen, T dt, T om, const int* active) {
  if (active && !*active) return;
  __shared__ RbSmem<T> sm;
  rbsor_sweep_tile<T>(g, comp, blockIdx.x, blockIdx.y, uin, uout, rhs, rho, kap, zeta, eta, pen, dt, om, sm);
}

// ------------------------------------------------ several Jacobi sweeps at once
// Up to JM_K damped-Jacobi sweeps (solve_helmholtz_u/v's, jacobi_u_vals /
// jacobi_v_vals) of one velocity component of a wall-bounded case in one
// launch, per tile of JM_TX x JM_TY faces, from uin into uout.  The tile and
// a ring of JM_K faces of uin go to shared memory (the ring widened to eight
// columns either side so that rows start on 16-byte boundaries), the
// coefficients of the tile and a ring of JM_K - 1 are formed once, and sweep
// s of nsw updates the tile and a ring of nsw - s faces from the previous
// sweep's values, alternating between two shared-memory buffers; each face
// takes the formula with its operand order (owned faces), the right-hand side
// (wall faces) or keeps its value (other elements), as in k_jacobi_u/v.  So
// nsw sweeps give the bits of nsw k_jacobi_u/v launches, reading and writing
// each array once.  Periodic cases refresh their halo between sweeps and
// keep the one-sweep launches.
constexpr int JM_TX = 32, JM_TY = 16, JM_K = 6, JM_TPB = 256;
constexpr int JM_SX = JM_TX + 16, JM_SY = JM_TY + 2 * JM_K;            // staged values
constexpr int JM_CX = JM_TX + 2 * (JM_K - 1), JM_CY = JM_TY + 2 * (JM_K - 1);  // coefficients
template <typename T>
struct JmSmem {
  T u[2][JM_SY][JM_SX];
  T cE[JM_CY][JM_CX], cW[JM_CY][JM_CX], cN[JM_CY][JM_CX], cS[JM_CY][JM_CX], dg[JM_CY][JM_CX], rh[JM_CY][JM_CX];
  unsigned char kind[JM_CY][JM_CX];  // 0 keeps its value, 1 owned face (formula), 2 wall face (= rhs)
};
template <typename T>
__device__ __forceinline__ void jacobi_multi_tile(const Geo& g, int comp, int nsw, int tx, int ty, const T* uin,
                                                  T* __restrict__ uout, const T* rhs, const T* rho, const T* kap,
                                                  const T* zeta, const T* eta, const T* pen, T dt, T om,
                                                  JmSmem<T>& sm) {
  const int ii0 = tx * JM_TX, jj0 = ty * JM_TY;  // padded coordinates of the tile's first face
  const int sx0 = ii0 - 8, sy0 = jj0 - JM_K;     // of sm.u[.][0][0]
  const int cx0 = ii0 - (JM_K - 1), cy0 = jj0 - (JM_K - 1);  // of the coefficient arrays' [0][0]
  const int nx = g.nx, ny = g.ny;
  const T ix2 = T(g.idx2), iy2 = T(g.idy2);
  for (int q = threadIdx.x; q < JM_SX * JM_SY; q += blockDim.x) {
    const int a = q % JM_SX, b = q / JM_SX;
    const int ii = sx0 + a, jj = sy0 + b;
    sm.u[0][b][a] = (ii >= 0 && ii < g.P && jj >= 0 && jj < g.R) ? uin[ii + jj * g.P] : T(0);
  }
  for (int q = threadIdx.x; q < JM_CX * JM_CY; q += blockDim.x) {
    const int a = q % JM_CX, b = q / JM_CX;
    const int ii = cx0 + a, jj = cy0 + b;
    const int i = ii - 2, j = jj - 2;
    unsigned char kd = 0;
    if (ii >= 0 && ii < g.P && jj >= 0 && jj < g.R) {
      const int k = ii + jj * g.P;
      if (comp == 0 && j >= 1 && j <= ny) {
        if (i >= 1 && i <= nx - 1) {
          kd = 1;
          const T e = kap[g.at(i + 1, j)] * ix2, w = kap[k] * ix2;
          const T nn = (zeta[k] - eta[k]) * iy2, ss = (zeta[g.at(i, j - 1)] - eta[g.at(i, j - 1)]) * iy2;
          T d = (rho[k] / dt) + e + w + nn + ss;
          if (pen) d = d + pen[k];
          sm.cE[b][a] = e; sm.cW[b][a] = w; sm.cN[b][a] = nn; sm.cS[b][a] = ss; sm.dg[b][a] = d;
        } else if (i == 0 || i == nx) {
          kd = 2;
        }
      } else if (comp == 1 && i >= 1 && i <= nx) {
        if (j >= 1 && j <= ny - 1) {
          kd = 1;
          const T e = (zeta[k] - eta[k]) * ix2, w = (zeta[g.at(i - 1, j)] - eta[g.at(i - 1, j)]) * ix2;
          const T nn = kap[g.at(i, j + 1)] * iy2, ss = kap[k] * iy2;
          T d = (rho[k] / dt) + e + w + nn + ss;
          if (pen) d = d + pen[k];
          sm.cE[b][a] = e; sm.cW[b][a] = w; sm.cN[b][a] = nn; sm.cS[b][a] = ss; sm.dg[b][a] = d;
        } else if (j == 0 || j == ny) {
          kd = 2;
        }
      }
      if (kd) sm.rh[b][a] = rhs[k];
    }
    sm.kind[b][a] = kd;
  }
  __syncthreads();
  int cur = 0;
  for (int sweep = 1; sweep <= nsw; ++sweep) {
    const int ring = nsw - sweep;  // faces updated around the tile in this sweep
    const int wx = JM_TX + 2 * ring, wy = JM_TY + 2 * ring;
    for (int q = threadIdx.x; q < wx * wy; q += blockDim.x) {
      const int ii = ii0 - ring + q % wx, jj = jj0 - ring + q / wx;  // padded coordinates
      const int a = ii - cx0, b = jj - cy0;                           // coefficient indices
      const int ua = ii - sx0, ub = jj - sy0;                         // value indices
      const unsigned char kd = sm.kind[b][a];
      const T uo = sm.u[cur][ub][ua];
      T val = uo;
      if (kd == 2) {
        val = sm.rh[b][a];
      } else if (kd == 1) {
        const T d = sm.dg[b][a];
        const T off = madd(sm.cS[b][a], sm.u[cur][ub - 1][ua],
                           madd(sm.cN[b][a], sm.u[cur][ub + 1][ua],
                                madd(sm.cW[b][a], sm.u[cur][ub][ua - 1], sm.cE[b][a] * sm.u[cur][ub][ua + 1])));
        if (d > T(1.0e-15)) val = madd(T(1) - om, uo, om * ((sm.rh[b][a] + off) / d));
      }
      sm.u[cur ^ 1][ub][ua] = val;
    }
    __syncthreads();
    cur ^= 1;
  }
  for (int q = threadIdx.x; q < JM_TX * JM_TY; q += blockDim.x) {
    const int ii = ii0 + q % JM_TX, jj = jj0 + q / JM_TX;
    if (ii < g.P && jj < g.R) uout[ii + jj * g.P] = sm.u[cur][jj - sy0][ii - sx0];
  }
}
template <typename T>
__global__ void __launch_bounds__(JM_TPB) k_jacobi_multi(Geo g, int comp, int nsw, const T* uin, T* __restrict__ uout,
                                                         const T* rhs, const T* rho, const T* kap, const T* zeta,
                                                         const T* eta, const T* pen, T dt, T om, const int* active) {
  if (active && !*active) return;
  extern __shared__ __align__(16) unsigned char jm_smem[];
  jacobi_multi_tile<T>(g, comp, nsw, blockIdx.x, blockIdx.y, uin, uout, rhs, rho, kap, zeta, eta, pen, dt, om,
                       *reinterpret_cast<JmSmem<T>*>(jm_smem));
}

// ------------------------------------------------------------ Krylov vectors
// Whole-buffer linear combinations over a coupled triple (u, v, p buffers of
// n elements each, contiguous in one allocation of 3n).  Coefficients are
// read from device scalars so the sequence can run without host round trips;
// sgn flips the sign exactly.  Evaluation order is the reference's
// left-to-right: y = ((x + c1 z1) + c2 z2) + c3 z3.
template <typename T>
struct Lin {
  const T* x;
  const T* z1;
  const T* z2;
  const T* z3;
  const double* c1;
  const double* c2;
  const double* c3;
  double s1, s2, s3;
};
//
// The element-wise kernels below take four elements per thread per pass of
// their grid-stride loop (q, q + S, q + 2S, q + 3S; S = the grid's thread
// count): all four elements' loads come before any store (the output may be
// one of the inputs, element by element), so they are in flight together and
// a pass over buffers larger than L2 runs at HBM bandwidth instead of at the
// latency of one load per thread.
template <typename T>
__global__ void k_lin(long n3, T* y, Lin<T> L, const int* active) {
  if (active && !*active) return;
  const T c1 = L.c1 ? T(L.s1 * *L.c1) : T(0);
  const T c2 = L.c2 ? T(L.s2 * *L.c2) : T(0);
  const T c3 = L.c3 ? T(L.s3 * *L.c3) : T(0);
  const long S = (long)gridDim.x * blockDim.x;
  for (long q0 = blockIdx.x * (long)blockDim.x + threadIdx.x; q0 < n3; q0 += 4 * S) {
    T a[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const long q = q0 + u * S;
      if (q < n3) {
        T t = L.x[q];
        if (L.z1) t = t + c1 * L.z1[q];
        if (L.z2) t = t + c2 * L.z2[q];
        if (L.z3) t = t + c3 * L.z3[q];
        a[u] = t;
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (q0 + u * S < n3) y[q0 + u * S] = a[u];
  }
}
// bicgstab_solve direction update p = r + beta (p - omega v) (mod_bicgstab2.f90:244-246)
template <typename T>
__global__ void k_pupdate(long n3, T* p, const T* r, const T* v, const double* beta,
                          const double* omega, const int* active) {
  if (active && !*active) return;
  const T b = T(*beta), w = T(*omega);
  const long S = (long)gridDim.x * blockDim.x;
  for (long q0 = blockIdx.x * (long)blockDim.x + threadIdx.x; q0 < n3; q0 += 4 * S) {
    T a[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const long q = q0 + u * S;
      if (q < n3) a[u] = r[q] + b * (p[q] - w * v[q]);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (q0 + u * S < n3) p[q0 + u * S] = a[u];
  }
}

// ------------------------------------------------------------ VOF transport
template <typename S>
__device__ __forceinline__ S limiter_psi(int lim, S r) {
  if (lim == 1) {  // Superbee (extension)
    const S a = fmin(2.0 * r, 1.0), b = fmin(r, 2.0);
    return fmax(0.0, fmax(a, b));
  }
  if (r <= 0.0) return S(0.0);  // van_leer_limiter, mod_vof.f90:25-33
  return (2.0 * r) / (1.0 + r);
}
// face fluxes of vof_advection_tvd (mod_vof.f90:59-114)
template <typename S>
__device__ __forceinline__ S flux_x_at(const Geo& g, int lim, const S* c, const S* u, int i, int j, double dt) {
  const S uf = u[g.at(i, j)];
  S num, den, r, cfl, cf;
  if (uf >= 0.0) {
    num = c[g.at(i, j)] - c[g.at(i - 1, j)];
    den = c[g.at(i + 1, j)] - c[g.at(i, j)];
    r = fabs(den) > 1.0e-12 ? num / den : S(0.0);
    cfl = fabs(uf) * dt * g.idx;
    cf = c[g.at(i, j)] + 0.5 * (1.0 - cfl) * limiter_psi(lim, r) * den;
  } else {
    num = c[g.at(i + 2, j)] - c[g.at(i + 1, j)];
    den = c[g.at(i + 1, j)] - c[g.at(i, j)];
    r = fabs(den) > 1.0e-12 ? num / den : S(0.0);
    cfl = fabs(uf) * dt * g.idx;
    cf = c[g.at(i + 1, j)] - 0.5 * (1.0 - cfl) * limiter_psi(lim, r) * den;
  }
  return uf * clip01(cf);
}
template <typename S>
__device__ __forceinline__ S flux_y_at(const Geo& g, int lim, const S* c, const S* v, int i, int j, double dt) {
  const S vf = v[g.at(i, j)];
  S num, den, r, cfl, cf;
  if (vf >= 0.0) {
    num = c[g.at(i, j)] - c[g.at(i, j - 1)];
    den = c[g.at(i, j + 1)] - c[g.at(i, j)];
    r = fabs(den) > 1.0e-12 ? num / den : S(0.0);
    cfl = fabs(vf) * dt * g.idy;
    cf = c[g.at(i, j)] + 0.5 * (1.0 - cfl) * limiter_psi(lim, r) * den;
  } else {
    num = c[g.at(i, j + 2)] - c[g.at(i, j + 1)];
    den = c[g.at(i, j + 1)] - c[g.at(i, j)];
    r = fabs(den) > 1.0e-12 ? num / den : S(0.0);
    cfl = fabs(vf) * dt * g.idy;
    cf = c[g.at(i, j + 1)] - 0.5 * (1.0 - cfl) * limiter_psi(lim, r) * den;
  }
  return vf * clip01(cf);
}
// conservative update + clipping (mod_vof.f90:117-126); ghosts copied from C_in
template <typename S>
__global__ void k_vof_update(Geo g, int lim, const S* c, const S* u, const S* v, double dt, S* cout) {
  FUGU_BOX_IJ
  S val = c[k];
  if (i >= 1 && i <= g.nx && j >= 1 && j <= g.ny) {
    const S fe = flux_x_at(g, lim, c, u, i, j, dt), fw = flux_x_at(g, lim, c, u, i - 1, j, dt);
    const S fn = flux_y_at(g, lim, c, v, i, j, dt), fs = flux_y_at(g, lim, c, v, i, j - 1, dt);
    val = clip01(c[k] - dt * ((fe - fw) * g.idx + (fn - fs) * g.idy));
  }
  cout[k] = val;
}
// optional flux outputs for the AMP mass fluxes (mod_vof.f90:128-137)
__global__ void k_vof_fluxes(Geo g, int lim, const double* c, const double* u, const double* v,
                             double dt, double* fx, double* fy) {
  FUGU_BOX_IJ
  fx[k] = (j >= 1 && j <= g.ny && i >= 0 && i <= g.nx) ? flux_x_at(g, lim, c, u, i, j, dt) : 0.0;
  fy[k] = (i >= 1 && i <= g.nx && j >= 0 && j <= g.ny) ? flux_y_at(g, lim, c, v, i, j, dt) : 0.0;
}

// ------------------------------------------------------------ SVOF, curvature, CSF
// Index maps of a ghost onto the interior after halo exchange + Neumann BC
// (mod_vof.f90:169-170, :199-237): periodic wraps, a wall mirrors.
__device__ __forceinline__ int map_x(const Geo& g, int i) {
  if (i >= 1 && i <= g.nx) return i;
  if (g.px) return i < 1 ? i + g.nx : i - g.nx;
  return i < 1 ? 1 - i : 2 * g.nx + 1 - i;
}
__device__ __forceinline__ int map_y(const Geo& g, int j) {
  if (j >= 1 && j <= g.ny) return j;
  if (g.py) return j < 1 ? j + g.ny : j - g.ny;
  return j < 1 ? 1 - j : 2 * g.ny + 1 - j;
}
// fill every ghost cell of a cell array from its interior (halo + Neumann)
template <typename S>
__global__ void k_fill_ghost_neumann(Geo g, S* a) {
  FUGU_BOX_IJ
  if (!in_kind(g, K_CELL, i, j)) return;
  if (i >= 1 && i <= g.nx && j >= 1 && j <= g.ny) return;
  a[k] = a[g.at(map_x(g, i), map_y(g, j))];
}

// compute_interface_curvature (mod_surface_tension.f90:25-72): face normals
// on the fly, kappa = -div n at cells; ghosts 0 at walls or wrapped (halo).
template <typename S>
__device__ __forceinline__ S nx_face(const Geo& g, const S* cs, int i, int j) {
  const S gx = (cs[g.at(i + 1, j)] - cs[g.at(i, j)]) * g.idx;
  const S gy = 0.25 * (cs[g.at(i, j + 1)] + cs[g.at(i + 1, j + 1)] - cs[g.at(i, j - 1)] -
                            cs[g.at(i + 1, j - 1)]) * g.idy;
  return gx / sqrt(gx * gx + gy * gy + 1.0e-12);
}
template <typename S>
__device__ __forceinline__ S ny_face(const Geo& g, const S* cs, int i, int j) {
  const S gx = 0.25 * (cs[g.at(i + 1, j)] + cs[g.at(i + 1, j + 1)] - cs[g.at(i - 1, j)] -
                            cs[g.at(i - 1, j + 1)]) * g.idx;
  const S gy = (cs[g.at(i, j + 1)] - cs[g.at(i, j)]) * g.idy;
  return gy / sqrt(gx * gx + gy * gy + 1.0e-12);
}
template <typename S>
__global__ void k_curvature(Geo g, const S* cs, S* kc) {
  FUGU_BOX_IJ
  if (!in_kind(g, K_CELL, i, j)) { kc[k] = S(0.0); return; }
  int ci = i, cj = j;
  const bool gi = (i < 1 || i > g.nx), gj = (j < 1 || j > g.ny);
  if ((gi && !g.px) || (gj && !g.py)) { kc[k] = S(0.0); return; }
  if (gi) ci = map_x(g, i);
  if (gj) cj = map_y(g, j);
  kc[k] = -((nx_face(g, cs, ci, cj) - nx_face(g, cs, ci - 1, cj)) * g.idx +
            (ny_face(g, cs, ci, cj) - ny_face(g, cs, ci, cj - 1)) * g.idy);
}
// compute_csf_force (mod_surface_tension.f90:78-109)
template <typename S>
__global__ void k_csf(Geo g, S sigma, const S* c, const S* kc, S* fu, S* fv) {
  FUGU_BOX_IJ
  S a = S(0.0), b = S(0.0);
  if (j >= 1 && j <= g.ny && i >= 0 && i <= g.nx) {
    const S kf = 0.5 * (kc[k] + kc[g.at(i + 1, j)]);
    a = sigma * kf * (c[g.at(i + 1, j)] - c[k]) * g.idx;
  }
  if (i >= 1 && i <= g.nx && j >= 0 && j <= g.ny) {
    const S kf = 0.5 * (kc[k] + kc[g.at(i, j + 1)]);
    b = sigma * kf * (c[g.at(i, j + 1)] - c[k]) * g.idy;
  }
  fu[k] = a;
  fv[k] = b;
}

// ------------------------------------------------------------ step pieces
// AB extrapolation + history shift (mod_solver_coupled.f90:209-222):
// adv = step<=1 ? x : 2x - prev; nm1 = prev; prev = x.
__global__ void k_extrapolate(long n, const double* x, double* prev, double* nm1, double* adv, int first) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    const double xv = x[q], pv = prev[q];
    adv[q] = first ? xv : 2.0 * xv - pv;
    nm1[q] = pv;
    prev[q] = xv;
  }
}
// a = s1 * x + s2 * y (AMP mass flux, penalty scaling; whole buffers)
__global__ void k_axpby(long n, double* a, double s1, const double* x, double s2, const double* y) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x)
    a[q] = y ? s1 * x[q] + s2 * y[q] : s1 * x[q];
}
// dst = T(src * s), four elements per thread per pass (loads first)
template <typename T>
__device__ __forceinline__ void convert4(long n, T* dst, const double* src, double s) {
  const long S = (long)gridDim.x * blockDim.x;
  for (long q0 = blockIdx.x * (long)blockDim.x + threadIdx.x; q0 < n; q0 += 4 * S) {
    double a[4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (q0 + u * S < n) a[u] = src[q0 + u * S];
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (q0 + u * S < n) dst[q0 + u * S] = T(a[u] * s);
  }
}
template <typename T>
__global__ void k_convert(long n, T* dst, const double* src, double scale) {
  convert4<T>(n, dst, src, scale);
}
template <typename T>
__global__ void k_convert_scaled(long n, T* dst, const double* src, const double* scale) {
  convert4<T>(n, dst, src, *scale);
}
template <typename T>
__global__ void k_accumulate(long n, double* x, const T* d, const double* scale) {
  const double s = *scale;
  const long S = (long)gridDim.x * blockDim.x;
  for (long q0 = blockIdx.x * (long)blockDim.x + threadIdx.x; q0 < n; q0 += 4 * S) {
    double a[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const long q = q0 + u * S;
      if (q < n) a[u] = x[q] + s * double(d[q]);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (q0 + u * S < n) x[q0 + u * S] = a[u];
  }
}

// monolithic right-hand side (mod_solver_coupled.f90:261-303)
template <typename S>
struct RhsArgsT {
  const S *rho_u, *rho_v, *u_n, *u_nm1, *v_n, *v_nm1, *fsu, *fsv, *pen_u, *pen_v, *zeta, *eta;
  double dt, gx, gy, u_sol, v_sol, u_lid;
  int bdf2, has_lid;
};
using RhsArgs = RhsArgsT<double>;
template <typename S>
__global__ void k_rhs(Geo g, RhsArgsT<S> a, S* Bu, S* Bv, S* Bp) {
  FUGU_BOX_IJ
  S bu = S(0.0), bv = S(0.0);
  if (j >= 1 && j <= g.ny && i >= 1 && i <= g.imax()) {
    if (a.bdf2)
      bu = (a.rho_u[k] / a.dt) * (2.0 * a.u_n[k] - 0.5 * a.u_nm1[k]) + a.rho_u[k] * a.gx + a.fsu[k];
    else
      bu = (a.rho_u[k] / a.dt) * a.u_n[k] + a.rho_u[k] * a.gx + a.fsu[k];
    if (a.pen_u) bu = bu + a.pen_u[k] * a.u_sol;
    if (a.has_lid && !g.py && j == g.ny)
      bu = bu + (2.0 * (a.zeta[k] - a.eta[k]) / (g.dy * g.dy)) * a.u_lid;
  }
  if (i >= 1 && i <= g.nx && j >= 1 && j <= g.jmax()) {
    if (a.bdf2)
      bv = (a.rho_v[k] / a.dt) * (2.0 * a.v_n[k] - 0.5 * a.v_nm1[k]) + a.rho_v[k] * a.gy + a.fsv[k];
    else
      bv = (a.rho_v[k] / a.dt) * a.v_n[k] + a.rho_v[k] * a.gy + a.fsv[k];
    if (a.pen_v) bv = bv + a.pen_v[k] * a.v_sol;
  }
  Bu[k] = bu;
  Bv[k] = bv;
  Bp[k] = S(0.0);
}

// max |u| over faces 0..nx x 1..ny and |v| over 1..nx x 0..ny
// (compute_adaptive_dt, mod_solver_coupled.f90:54-66); part[2*blk]
__global__ void k_maxvel(Geo g, const double* u, const double* v, double* part) {
  __shared__ double sh[32];
  double mu = 0.0, mv = 0.0;
  const long nu = (long)(g.nx + 1) * g.ny, nv = (long)g.nx * (g.ny + 1);
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < nu + nv; q += (long)gridDim.x * blockDim.x) {
    if (q < nu) mu = fmax(mu, fabs(u[g.at((int)(q % (g.nx + 1)), 1 + (int)(q / (g.nx + 1)))]));
    else {
      const long r = q - nu;
      mv = fmax(mv, fabs(v[g.at(1 + (int)(r % g.nx), (int)(r / g.nx))]));
    }
  }
  mu = block_max(mu, sh);
  if (threadIdx.x == 0) part[2 * blockIdx.x] = mu;
  mv = block_max(mv, sh);
  if (threadIdx.x == 0) part[2 * blockIdx.x + 1] = mv;
}

// build_cylinder_mask (mod_solver_coupled.f90:96-132), i_start = j_start = 1
__global__ void k_cylinder(Geo g, double xc, double yc, double rad, double* pu, double* pv) {
  FUGU_BOX_IJ
  double a = 0.0, b = 0.0;
  if (j >= 1 && j <= g.ny && i >= 0 && i <= g.nx) {
    const double x = (double)i * g.dx, y = ((double)j - 0.5) * g.dy;
    if (sqrt((x - xc) * (x - xc) + (y - yc) * (y - yc)) <= rad) a = 1.0;
  }
  if (i >= 1 && i <= g.nx && j >= 0 && j <= g.ny) {
    const double x = ((double)i - 0.5) * g.dx, y = (double)j * g.dy;
    if (sqrt((x - xc) * (x - xc) + (y - yc) * (y - yc)) <= rad) b = 1.0;
  }
  pu[k] = a;
  pv[k] = b;
}

}  // namespace fugu
