// fugu_internal.cuh -- device layout, launch helpers and the bounded grid
// barrier shared by the B200 kernels of the FUGU-2D coupled-step path.
//
// Device layout.  Every field kind (cell, u-face, v-face, vertex) is stored in
// one uniform padded box: element (i, j) lives at (i + 2) + (j + 2) * P with
// P >= nx + 5 a multiple of 16 (128-byte rows) and R = ny + 5 rows.  A u-face
// (i, j), the cell (i, j) and the vertex (i, j) therefore share one linear
// index, so every stencil offset is +-1 / +-P whatever the kinds involved, and
// one thread per (i, j) can produce the u, v and p rows of the coupled
// operator together.  The Fortran extents of each kind are sub-boxes of it:
//   cell (-1..nx+2, -1..ny+2)  u (-2..nx+2, -1..ny+2)
//   v    (-1..nx+2, -2..ny+2)  vertex (-2..nx+2, -2..ny+2)
// Elements outside a kind's extent are padding; they are zero at allocation
// and every whole-buffer operation keeps them zero.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace fugu {

enum Kind { K_CELL = 0, K_U = 1, K_V = 2, K_VERT = 3 };

struct Geo {
  int nx, ny;
  int P, R;            // pitch (elements) and rows of the padded box
  double dx, dy;
  double idx, idy;     // 1/dx, 1/dy  (computed as one / dx_grid, as the reference)
  double idx2, idy2;   // 1/(dx*dx), 1/(dy*dy)
  int px, py;          // periodic flags
  int fsx;             // free-slip side walls (extension)
  __host__ __device__ __forceinline__ int at(int i, int j) const { return (i + 2) + (j + 2) * P; }
  __host__ __device__ __forceinline__ long n() const { return (long)P * R; }
  __host__ __device__ __forceinline__ int imax() const { return px ? nx : nx - 1; }  // owned u faces
  __host__ __device__ __forceinline__ int jmax() const { return py ? ny : ny - 1; }  // owned v faces
  // extent of a kind in Fortran indices (inclusive)
  __host__ __device__ __forceinline__ void extent(int kind, int& i0, int& i1, int& j0, int& j1) const {
    i0 = (kind == K_U || kind == K_VERT) ? -2 : -1;
    j0 = (kind == K_V || kind == K_VERT) ? -2 : -1;
    i1 = nx + 2;
    j1 = ny + 2;
  }
};

// 2-D launch over the whole padded box: ii = 0..P-1, jj = 0..R-1 (i = ii - 2)
struct Box {
  dim3 grid, block;
};
inline Box box_launch(const Geo& g) {
  Box b;
  b.block = dim3(32, 8, 1);
  b.grid = dim3((g.P + 31) / 32, (g.R + 7) / 8, 1);
  return b;
}

// 16-byte vector access: VecW<T>::value elements (four floats or two
// doubles) from / to an address that is a multiple of 16 bytes
template <typename T>
struct VecW {
  static constexpr int value = 16 / (int)sizeof(T);
};
__device__ __forceinline__ void ldv(const float* p, float* o) {
  const float4 x = *reinterpret_cast<const float4*>(p);
  o[0] = x.x; o[1] = x.y; o[2] = x.z; o[3] = x.w;
}
__device__ __forceinline__ void ldv(const double* p, double* o) {
  const double2 x = *reinterpret_cast<const double2*>(p);
  o[0] = x.x; o[1] = x.y;
}
__device__ __forceinline__ void stv(float* p, const float* o) {
  *reinterpret_cast<float4*>(p) = make_float4(o[0], o[1], o[2], o[3]);
}
__device__ __forceinline__ void stv(double* p, const double* o) {
  *reinterpret_cast<double2*>(p) = make_double2(o[0], o[1]);
}

// a * b + c.  FP32 (the mixed form's inner solve, which needs no bit parity
// with the oracle): one fused multiply-add, one rounding and one issue slot.
// Every other type: the product and the sum rounded separately -- the library
// is compiled without contraction, so the FP64 plain form stays bit-exact
// with the CPU oracle.  Callers write a * b + c as madd(a, b, c) only where
// the sum's operands are the same two values either way (IEEE addition is
// commutative and x + (-y) equals x - y), so the FP64 bits do not change.
template <typename T>
__device__ __forceinline__ T madd(T a, T b, T c) {
  return a * b + c;
}
template <>
__device__ __forceinline__ float madd<float>(float a, float b, float c) {
  return __fmaf_rn(a, b, c);
}

// --------------------------------------------------------------------------
// Bounded grid barrier for persistent kernels launched cooperatively (all
// CTAs co-resident).  One thread per CTA arrives on a counter; the last one
// resets it and bumps the generation.  Every wait polls at most
// FUGU_SPIN_LIMIT times (about a second); on timeout, or when another CTA
// has already flagged an error, the CTA records the error and returns false
// so the kernel can unwind instead of hanging the GPU.
// --------------------------------------------------------------------------
#ifndef FUGU_SPIN_LIMIT
#define FUGU_SPIN_LIMIT (1u << 24)
#endif

struct GridSync {
  unsigned int count;  // arrivals since the launch began (zeroed before every launch)
  unsigned int gen;    // not used by the barrier below; keeps the 16-byte layout
  int error;           // 0 ok, 1 barrier timeout
  int pad;
};

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int ld_relaxed_i32(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Returns true when every CTA arrived; false on timeout / error.  nblocks is
// the arrival count the barrier waits for (gridDim.x, or one more in the
// failure-detection test, which makes every wait run out); spin_limit bounds
// each wait in polls.  gen counts the launch's barriers so far.
//
// The arrival counter only grows within a launch (the host zeroes it before
// every launch), so barrier gen is complete once it reaches
// (gen + 1) * nblocks: the last CTA's arrival is itself the release, and no
// CTA has to reset a counter and publish a new generation after it (two
// more dependent global operations on the critical path).  A CTA can only
// arrive at barrier gen + 1 after every CTA arrived at barrier gen, so an
// early arrival never completes a barrier that is still missing one.
__device__ __forceinline__ bool grid_sync(GridSync* gs, unsigned int nblocks, unsigned int& gen,
                                          unsigned int spin_limit = FUGU_SPIN_LIMIT) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned int target = (gen + 1u) * nblocks;
    __threadfence();
    atomicAdd(&gs->count, 1u);
    unsigned int spins = 0;
    while (ld_acquire_u32(&gs->count) < target) {
      if (++spins > spin_limit || ld_relaxed_i32(&gs->error) != 0) {
        atomicExch(&gs->error, 1);
        ok = 0;
        break;
      }
      __nanosleep(40);
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  gen += 1;
  return s_ok != 0;
}

// --------------------------------------------------------------------------
// Nearly order-independent sums.  Every sum of the hot path (coupled_dot, the
// PCG scalars, the zero-mean projections) is accumulated as an unevaluated
// pair hi + lo: Knuth's TwoSum makes each hi addition error-free, lo adds the
// error terms with ordinary rounding, and the pair is rounded once.  While the
// terms' exponents span less than ~50 bits the lo additions are exact and the
// result is the correctly rounded sum in any order.  Wider spans (~2e5 terms
// of a Krylov vector at 256^2) leave lo an error near n * eps^2 * |partial
// sums|, so the GPU's short per-thread pairs merged in a tree and the oracle's
// one serial pair can round the last bit differently when the sum cancels.
// The reference's own sums depend on its MPI rank count.  Needs IEEE add
// without contraction or reassociation
// (the FP64 build uses --fmad=false).
// --------------------------------------------------------------------------
struct DD {
  double hi, lo;
};
__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  const double bp = s - a;
  e = (a - (s - bp)) + (b - bp);
}
__device__ __forceinline__ void dd_add(DD& d, double x) {
  double s, e;
  two_sum(d.hi, x, s, e);
  d.hi = s;
  d.lo = d.lo + e;
}
__device__ __forceinline__ DD dd_merge(DD a, DD b) {
  double s, e;
  two_sum(a.hi, b.hi, s, e);
  e = e + (a.lo + b.lo);
  DD r;
  r.hi = s + e;
  r.lo = e - (r.hi - s);
  return r;
}
__device__ __forceinline__ DD dd_shfl_down(DD v, int o) {
  DD r;
  r.hi = __shfl_down_sync(0xffffffffu, v.hi, o);
  r.lo = __shfl_down_sync(0xffffffffu, v.lo, o);
  return r;
}
// block reduction of one DD per thread; result valid in thread 0
__device__ __forceinline__ DD block_sum_dd(DD v, DD* sh /* >= 32 */) {
  for (int o = 16; o > 0; o >>= 1) v = dd_merge(v, dd_shfl_down(v, o));
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  const int nw = blockDim.x >> 5;
  if (w == 0) {
    if (l < nw) v = sh[l];
    else { v.hi = 0.0; v.lo = 0.0; }
    for (int o = 16; o > 0; o >>= 1) v = dd_merge(v, dd_shfl_down(v, o));
  }
  return v;
}
// store a CTA's DD partial as two doubles: part[2b], part[2b+1]
__device__ __forceinline__ void put_partial(double* part, int b, DD v) {
  part[2 * b] = v.hi;
  part[2 * b + 1] = v.lo;
}
// rounded sum of n DD partials, identical in every CTA (fixed order).  Lane
// l of warp 0 merges partials l, l + 32, l + 64, ... in that order, then a
// fixed shuffle tree merges the lanes.  The loads of up to eight of a lane's
// partials are issued together before they are merged (one round trip to
// L2 per eight instead of one per partial); the order of the merges is the
// same either way.
template <int NA>
__device__ __forceinline__ void merge_partials_dd(const double* const* parts, int n, double* res) {
  DD v[NA];
#pragma unroll
  for (int a = 0; a < NA; ++a) v[a] = DD{0.0, 0.0};
  for (int k0 = threadIdx.x; k0 < n; k0 += 32 * 8) {
    DD p[NA][8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int k = k0 + 32 * u;
#pragma unroll
      for (int a = 0; a < NA; ++a) {
        p[a][u] = DD{0.0, 0.0};
        if (k < n) {
          p[a][u].hi = __ldcg(parts[a] + 2 * k);
          p[a][u].lo = __ldcg(parts[a] + 2 * k + 1);
        }
      }
    }
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (k0 + 32 * u < n) {
#pragma unroll
        for (int a = 0; a < NA; ++a) v[a] = dd_merge(v[a], p[a][u]);
      }
  }
#pragma unroll
  for (int a = 0; a < NA; ++a) {
    for (int o = 16; o > 0; o >>= 1) v[a] = dd_merge(v[a], dd_shfl_down(v[a], o));
    res[a] = v[a].hi + v[a].lo;
  }
}
__device__ __forceinline__ double sum_partials_dd(const double* part, int n) {
  __shared__ double s_res;
  if (threadIdx.x < 32) {
    const double* parts[1] = {part};
    double r[1];
    merge_partials_dd<1>(parts, n, r);
    if (threadIdx.x == 0) s_res = r[0];
  }
  __syncthreads();
  const double r = s_res;
  __syncthreads();
  return r;
}
// the rounded sums of two arrays of n DD partials in one pass
__device__ __forceinline__ void sum_partials_dd2(const double* pa, const double* pb, int n, double& oa,
                                                 double& ob) {
  __shared__ double s_res2[2];
  if (threadIdx.x < 32) {
    const double* parts[2] = {pa, pb};
    double r[2];
    merge_partials_dd<2>(parts, n, r);
    if (threadIdx.x == 0) {
      s_res2[0] = r[0];
      s_res2[1] = r[1];
    }
  }
  __syncthreads();
  oa = s_res2[0];
  ob = s_res2[1];
  __syncthreads();
}

// deterministic block reduction (sum) of one double per thread; result valid
// in thread 0.  blockDim.x must be a multiple of 32 and <= 1024.
__device__ __forceinline__ double block_sum(double v, double* sh /* >= 32 */) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  const int nw = blockDim.x >> 5;
  if (w == 0) {
    v = l < nw ? sh[l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  return v;
}
__device__ __forceinline__ double block_max(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  const int nw = blockDim.x >> 5;
  if (w == 0) {
    v = l < nw ? sh[l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  }
  return v;
}

// Sum of n per-CTA partials, identical in every CTA (fixed order): warp 0
// reads lane-strided and tree-reduces.  Result broadcast through shared.
__device__ __forceinline__ double sum_partials(const double* part, int n, double* sh) {
  __shared__ double s_res;
  if (threadIdx.x < 32) {
    double v = 0.0;
    for (int k = threadIdx.x; k < n; k += 32) v += __ldcg(part + k);
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) s_res = v;
  }
  __syncthreads();
  double r = s_res;
  __syncthreads();
  (void)sh;
  return r;
}
__device__ __forceinline__ double max_partials(const double* part, int n) {
  __shared__ double s_res;
  if (threadIdx.x < 32) {
    // loads eight at a time (the maximum does not depend on the order)
    double v = 0.0;
    for (int k0 = threadIdx.x; k0 < n; k0 += 32 * 8) {
      double x[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) x[u] = k0 + 32 * u < n ? __ldcg(part + k0 + 32 * u) : 0.0;
#pragma unroll
      for (int u = 0; u < 8; ++u) v = fmax(v, x[u]);
    }
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    if (threadIdx.x == 0) s_res = v;
  }
  __syncthreads();
  double r = s_res;
  __syncthreads();
  return r;
}

}  // namespace fugu
