// dual.cuh -- forward-mode dual numbers for the tangent of a coupled step
// (extension, no counterpart in the reference).
//
// A Dual carries a value v and one directional derivative d.  The kernels of
// the step's explicit stages are templates on their scalar type; instantiated
// on Dual they compute, next to the same values, the exact derivative of the
// branch the values take (limiter, clip and upwind choices are decided on v).
// The overloads live in their own namespace so that, inside namespace fugu,
// an unqualified fmin/fmax/fabs/sqrt on doubles still names the CUDA math
// function; argument-dependent lookup finds these for Dual arguments.
#pragma once

namespace fugu {
namespace ad {

struct Dual {
  double v, d;
  Dual() = default;
  __host__ __device__ constexpr Dual(double x) : v(x), d(0.0) {}
  __host__ __device__ constexpr Dual(double x, double dx) : v(x), d(dx) {}
};

__host__ __device__ __forceinline__ Dual operator-(Dual a) { return {-a.v, -a.d}; }
__host__ __device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__host__ __device__ __forceinline__ Dual operator+(Dual a, double b) { return {a.v + b, a.d}; }
__host__ __device__ __forceinline__ Dual operator+(double a, Dual b) { return {a + b.v, b.d}; }
__host__ __device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__host__ __device__ __forceinline__ Dual operator-(Dual a, double b) { return {a.v - b, a.d}; }
__host__ __device__ __forceinline__ Dual operator-(double a, Dual b) { return {a - b.v, -b.d}; }
__host__ __device__ __forceinline__ Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__host__ __device__ __forceinline__ Dual operator*(Dual a, double b) { return {a.v * b, a.d * b}; }
__host__ __device__ __forceinline__ Dual operator*(double a, Dual b) { return {a * b.v, a * b.d}; }
__host__ __device__ __forceinline__ Dual operator/(Dual a, Dual b) {
  const double q = a.v / b.v;
  return {q, (a.d - q * b.d) / b.v};
}
__host__ __device__ __forceinline__ Dual operator/(Dual a, double b) { return {a.v / b, a.d / b}; }
__host__ __device__ __forceinline__ Dual operator/(double a, Dual b) {
  const double q = a / b.v;
  return {q, -q * b.d / b.v};
}

#define FUGU_DUAL_CMP(op)                                                                             \
  __host__ __device__ __forceinline__ bool operator op(Dual a, Dual b) { return a.v op b.v; }      \
  __host__ __device__ __forceinline__ bool operator op(Dual a, double b) { return a.v op b; }      \
  __host__ __device__ __forceinline__ bool operator op(double a, Dual b) { return a op b.v; }
FUGU_DUAL_CMP(<)
FUGU_DUAL_CMP(>)
FUGU_DUAL_CMP(<=)
FUGU_DUAL_CMP(>=)
#undef FUGU_DUAL_CMP

__device__ __forceinline__ Dual fabs(Dual a) { return a.v < 0.0 ? -a : a; }
__device__ __forceinline__ Dual sqrt(Dual a) {
  const double s = ::sqrt(a.v);
  return {s, a.d / (2.0 * s)};
}
// the CUDA fmin / fmax return the other operand for a NaN; the values here
// are never NaN, and on a tie the first operand is returned
__device__ __forceinline__ Dual fmin(Dual a, Dual b) { return b.v < a.v ? b : a; }
__device__ __forceinline__ Dual fmin(Dual a, double b) { return fmin(a, Dual(b)); }
__device__ __forceinline__ Dual fmin(double a, Dual b) { return fmin(Dual(a), b); }
__device__ __forceinline__ Dual fmax(Dual a, Dual b) { return b.v > a.v ? b : a; }
__device__ __forceinline__ Dual fmax(Dual a, double b) { return fmax(a, Dual(b)); }
__device__ __forceinline__ Dual fmax(double a, Dual b) { return fmax(Dual(a), b); }

}  // namespace ad
}  // namespace fugu
