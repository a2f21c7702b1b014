// fgmres.cuh -- flexible GMRES(m) with right PCD preconditioning (extension,
// not in the reference): the inner solve of the FP64 defect correction when
// refine = 2.  The reference's BiCGStab(l) needs a fixed preconditioner; PCD
// around a truncated PCG is not one, and BiCGStab(2) diverges on high
// density-ratio bubbles, while flexible GMRES keeps Z_j = M^{-1} V_j and
// minimises the true residual over span(Z).
//
// Device pieces: a multi-vector coupled dot (all projections of one
// Gram-Schmidt pass in one launch), a multi-vector axpy, the scale of a new
// basis vector, and the scalar steps (projections into H, Givens rotations,
// the small triangular solve), which run in the last CTA of the reductions
// like the BiCGStab recurrences do.
#pragma once

#include "scalars.cuh"

namespace fugu {

// device-resident scalars of one FGMRES cycle (doubles)
struct FgLayout {
  int m;  // Arnoldi steps of the cycle
  __host__ __device__ int H(int i, int j) const { return i + j * (m + 1); }  // (m+1) x m, column-major
  __host__ __device__ int cs() const { return (m + 1) * m; }
  __host__ __device__ int sn() const { return cs() + m; }
  __host__ __device__ int g() const { return sn() + m; }
  __host__ __device__ int y() const { return g() + m + 1; }
  __host__ __device__ int h() const { return y() + m; }  // projections of the current pass
  __host__ __device__ int beta() const { return h() + m + 1; }
  __host__ __device__ int inv() const { return beta() + 1; }  // scale of the next basis vector
  __host__ __device__ int rel() const { return beta() + 2; }
  __host__ __device__ int size() const { return beta() + 3; }
};

enum FgOp {
  FG_BETA = 0,  // beta = |B|; V_0 scale; g[0] = beta; exit when beta == 0
  FG_PROJ1,     // first Gram-Schmidt pass: h = d, H[0..j, j] = 0 + d
  FG_PROJ2,     // second pass: h = d, H[0..j, j] += d
  FG_ROTATE,    // H[j+1, j] = |w|, Givens rotations, g, rel, exit test
};

__device__ inline void fg_op(int op, const double* d, int j, double tol, const FgLayout L, double* st, KState* ks) {
  switch (op) {
    case FG_BETA: {
      const double beta = sqrt(d[0]);
      st[L.beta()] = beta;
      st[L.g()] = beta;
      st[L.inv()] = beta > 0.0 ? 1.0 / beta : 0.0;
      st[L.rel()] = beta > 0.0 ? 1.0 : 0.0;
      if (isnan(beta)) ks->nan = 1;
      if (!(beta > 0.0)) kexit(ks, 0);
      break;
    }
    case FG_PROJ1:
    case FG_PROJ2:
      for (int i = 0; i <= j; ++i) {
        st[L.h() + i] = d[i];
        if (op == FG_PROJ1) st[L.H(i, j)] = 0.0;
        st[L.H(i, j)] += d[i];
      }
      break;
    case FG_ROTATE: {
      const double hn = sqrt(d[0]);
      double* col = st + L.H(0, j);
      double* cs = st + L.cs();
      double* sn = st + L.sn();
      double* g = st + L.g();
      col[j + 1] = hn;
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
      const double rel = fabs(g[j + 1]) / st[L.beta()];
      st[L.rel()] = rel;
      st[L.inv()] = hn > 0.0 ? 1.0 / hn : 0.0;
      if (isnan(rel)) ks->nan = 1;
      if (rel < tol || hn == 0.0 || j + 1 == L.m || isnan(rel)) kexit(ks, j + 1);
      break;
    }
  }
}

// coupled dots of w with nvec vectors V_i = V0 + i * stride.  The work items
// are chunks of MDOT_CHUNK consecutive unknowns of one grid row of one
// component (u, v or p rows of the owned interior), so a warp reads contiguous
// memory and maps an item to its row once.  Each CTA keeps one DD partial for
// its vector; the last CTA merges the partials of each vector with one warp per
// vector and runs fg_op.  Launch: grid (Gx, nvec) of MDOT_TPB threads, grid
// row y computing the dot with V_y.
constexpr int MDOT_TPB = 256;
constexpr int MDOT_CHUNK = 128;
constexpr int MDOT_MAXV = 128;

template <typename T>
struct MdotArgs {
  Geo g;
  long n;  // elements of one component buffer
  const T* w;
  const T* V0;
  long stride;
  int nvec;      // <= MDOT_MAXV
  double vol;
  double* part;  // >= 2 * nvec * gridDim.x
  double* st;
  KState* ks;
  FgLayout L;
  int op, j;
  double tol;
};

// number of work items of a grid (u rows, v rows, p rows in MDOT_CHUNK pieces)
__host__ __device__ inline long mdot_items(const Geo& g) {
  const long cu = (g.imax() + MDOT_CHUNK - 1) / MDOT_CHUNK, cv = (g.nx + MDOT_CHUNK - 1) / MDOT_CHUNK;
  return (long)g.ny * cu + (long)g.jmax() * cv + (long)g.ny * cv;
}

// CTA (bx, by) of a (Gx, Gy = nvec) grid
// a lane's running sum of its products: error-free (double-double) for the
// FP64 parity path; the FP32 inner solve needs only a fixed order, so a plain
// double sum of its (exact) float products serves there at a fraction of the
// dependent FP64 work
template <typename T>
__device__ __forceinline__ void mdot_acc(DD& acc, double x) {
  if constexpr (sizeof(T) == 8) dd_add(acc, x);
  else acc.hi += x;
}
template <typename T>
__device__ __forceinline__ void mdot_body(const MdotArgs<T>& a, int bx, int by, int Gx, int Gy) {
  constexpr int NW = MDOT_TPB / 32;
  __shared__ DD wsum[NW];
  __shared__ double dsum[MDOT_MAXV];
  __shared__ bool last;
  const Geo g = a.g;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nx = g.nx, ny = g.ny, imax = g.imax(), jmax = g.jmax();
  const int cu = (imax + MDOT_CHUNK - 1) / MDOT_CHUNK, cv = (nx + MDOT_CHUNK - 1) / MDOT_CHUNK;
  const long iu = (long)ny * cu, iv = (long)jmax * cv, ip = (long)ny * cv;
  const long items = iu + iv + ip;
  const T* V = a.V0 + by * a.stride;  // this grid row's vector
  DD acc{0.0, 0.0};
  for (long it = (long)bx * NW + warp; it < items; it += (long)Gx * NW) {
    long base;
    int len, c;
    if (it < iu) {
      c = (int)(it % cu);
      base = g.at(1, 1 + (int)(it / cu));
      len = imax;
    } else if (it < iu + iv) {
      const long r = it - iu;
      c = (int)(r % cv);
      base = a.n + g.at(1, 1 + (int)(r / cv));
      len = nx;
    } else {
      const long r = it - iu - iv;
      c = (int)(r % cv);
      base = 2 * a.n + g.at(1, 1 + (int)(r / cv));
      len = nx;
    }
    const int i0 = c * MDOT_CHUNK + lane, i1 = min(len, (c + 1) * MDOT_CHUNK);
    if (i1 - c * MDOT_CHUNK == MDOT_CHUNK) {
      // a full chunk: issue the lane's 2 x 4 loads before the dependent
      // double-double chain (same accumulation order as the loop below)
      constexpr int U = MDOT_CHUNK / 32;
      T wv[U], vv[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        wv[u] = a.w[base + i0 + 32 * u];
        vv[u] = V[base + i0 + 32 * u];
      }
#pragma unroll
      for (int u = 0; u < U; ++u) mdot_acc<T>(acc, (double(wv[u]) * double(vv[u])) * a.vol);
    } else {
      for (int i = i0; i < i1; i += 32) {
        const long e = base + i;
        mdot_acc<T>(acc, (double(a.w[e]) * double(V[e])) * a.vol);
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) acc = dd_merge(acc, dd_shfl_down(acc, o));
  if (lane == 0) wsum[warp] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    DD s = wsum[0];
    for (int k = 1; k < NW; ++k) s = dd_merge(s, wsum[k]);
    put_partial(a.part + 2L * by * Gx, bx, s);
    __threadfence();
    const unsigned int t = atomicAdd(&a.ks->ticket, 1u);
    last = (t == (unsigned int)(Gx * Gy) - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int v = warp; v < a.nvec; v += NW) {
    const double* pv = a.part + 2L * v * Gx;
    DD s{0.0, 0.0};
    for (int k = lane; k < Gx; k += 32) {
      DD q;
      q.hi = __ldcg(pv + 2 * k);
      q.lo = __ldcg(pv + 2 * k + 1);
      s = dd_merge(s, q);
    }
    for (int o = 16; o > 0; o >>= 1) s = dd_merge(s, dd_shfl_down(s, o));
    if (lane == 0) dsum[v] = s.hi + s.lo;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    a.ks->ticket = 0;
    fg_op(a.op, dsum, a.j, a.tol, a.L, a.st, a.ks);
  }
}
template <typename T>
__global__ void __launch_bounds__(MDOT_TPB) k_mdot(MdotArgs<T> a) {
  if (!a.ks->active) return;
  mdot_body<T>(a, blockIdx.x, blockIdx.y, gridDim.x, gridDim.y);
}

// w = (...((w + s_0 V_0) + s_1 V_1) ...) + s_{nvec-1} V_{nvec-1}, s_i = sign * coef[i],
// over every element of the triple (whole-array, as the reference's array
// expressions).  Each element takes the same updates in the same order
// however the elements are spread over threads, so the two paths below give
// the same bits.
template <typename T>
__device__ __forceinline__ void maxpy_body(long n3, T* w, const T* V0, long stride, const double* coef, int nvec,
                                           double sign, int b, int G) {
  __shared__ T s[MDOT_MAXV];  // the coefficients, converted once per CTA
  for (int i = threadIdx.x; i < nvec; i += blockDim.x) s[i] = T(sign * coef[i]);
  __syncthreads();
  constexpr int W = VecW<T>::value;
  const long S = (long)G * blockDim.x;
  const bool aligned = ((reinterpret_cast<uintptr_t>(w) | reinterpret_cast<uintptr_t>(V0)) & 15u) == 0;
  if (n3 % W == 0 && stride % W == 0 && aligned) {
    // W consecutive elements per thread with 16-byte loads and stores, the
    // loads of up to eight vectors in flight before their updates: a
    // thread's elements are a few long, wide round trips rather than many
    // short ones (at 2048^2 a one-element-per-thread pass was latency-bound)
    for (long q = (b * (long)blockDim.x + threadIdx.x) * W; q < n3; q += S * W) {
      T x[W];
      ldv(w + q, x);
      for (int i = 0; i < nvec; i += 8) {
        T v[8][W];
#pragma unroll
        for (int u = 0; u < 8; ++u)
          if (i + u < nvec) ldv(V0 + (i + u) * stride + q, v[u]);
#pragma unroll
        for (int u = 0; u < 8; ++u)
          if (i + u < nvec) {
#pragma unroll
            for (int e = 0; e < W; ++e) x[e] = madd(s[i + u], v[u][e], x[e]);
          }
      }
      stv(w + q, x);
    }
    return;
  }
  for (long q = b * (long)blockDim.x + threadIdx.x; q < n3; q += S) {
    T x = w[q];
    // the loads of up to 16 vectors in flight together before the (ordered)
    // dependent updates: each group of loads costs one memory round trip,
    // so a projection on up to 16 vectors is one round trip per element
    for (int i = 0; i < nvec; i += 16) {
      T v[16];
#pragma unroll
      for (int u = 0; u < 16; ++u) v[u] = i + u < nvec ? V0[(i + u) * stride + q] : T(0);
#pragma unroll
      for (int u = 0; u < 16; ++u)
        if (i + u < nvec) x = madd(s[i + u], v[u], x);
    }
    w[q] = x;
  }
}
template <typename T>
__global__ void k_maxpy(long n3, T* w, const T* V0, long stride, const double* coef, int nvec, double sign,
                        const int* active) {
  if (active && !*active) return;
  maxpy_body<T>(n3, w, V0, stride, coef, nvec, sign, blockIdx.x, gridDim.x);
}

// dst = 0 + s * src (the reference-style array expression of a fresh vector)
template <typename T>
__global__ void k_fg_scale(long n3, T* dst, const T* src, const double* s, const int* active) {
  if (active && !*active) return;
  const T f = T(*s);
  const long S = (long)gridDim.x * blockDim.x;
  for (long q0 = blockIdx.x * (long)blockDim.x + threadIdx.x; q0 < n3; q0 += 4 * S) {
    T a[4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (q0 + u * S < n3) a[u] = src[q0 + u * S];
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (q0 + u * S < n3) dst[q0 + u * S] = T(0) + f * a[u];
  }
}

// back substitution R y = g over the k columns used
__device__ __forceinline__ void fg_solve_body(double* st, FgLayout L, int k) {
  const double* g = st + L.g();
  double* y = st + L.y();
  for (int i = k - 1; i >= 0; --i) {
    double s = g[i];
    for (int q = i + 1; q < k; ++q) s -= st[L.H(i, q)] * y[q];
    const double hii = st[L.H(i, i)];
    y[i] = hii != 0.0 ? s / hii : 0.0;
  }
}
__global__ void k_fg_solve(double* st, FgLayout L, int k) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  fg_solve_body(st, L, k);
}

}  // namespace fugu
