/*
 * gp_dual.cuh -- forward-mode dual numbers for the adjoint.
 *
 * Dual<W> carries a value and its derivatives along W seeded directions.
 * Arithmetic follows the value exactly as double arithmetic does (same
 * operations in the same order on .v), so a cell function evaluated on Dual
 * returns the double result bit for bit plus the exact partial derivatives of
 * that result with respect to the seeded inputs.  Comparisons look at values
 * only, so branches follow the forward trajectory (the derivative of a
 * piecewise function is the derivative of the piece the forward step took).
 */
#pragma once
#include <cmath>

namespace gpd {

template <int W>
struct Dual {
  double v;
  double d[W];
  __host__ __device__ Dual() {}
  __host__ __device__ Dual(double x) : v(x) {
#pragma unroll
    for (int i = 0; i < W; i++) d[i] = 0.0;
  }
};

template <typename T>
struct is_dual { static constexpr bool value = false; };
template <int W>
struct is_dual<Dual<W>> { static constexpr bool value = true; };

__host__ __device__ __forceinline__ double val(double x) { return x; }
template <int W>
__host__ __device__ __forceinline__ double val(const Dual<W> &x) { return x.v; }

#define GPD_BIN(op, dv, dd)                                                                       \
  template <int W>                                                                               \
  __host__ __device__ __forceinline__ Dual<W> operator op(const Dual<W> &a, const Dual<W> &b) {  \
    Dual<W> r;                                                                                   \
    r.v = dv;                                                                                    \
    _Pragma("unroll") for (int i = 0; i < W; i++) r.d[i] = dd;                                   \
    return r;                                                                                    \
  }
GPD_BIN(+, a.v + b.v, a.d[i] + b.d[i])
GPD_BIN(-, a.v - b.v, a.d[i] - b.d[i])
GPD_BIN(*, a.v * b.v, a.d[i] * b.v + a.v * b.d[i])
#undef GPD_BIN

template <int W>
__host__ __device__ __forceinline__ Dual<W> operator/(const Dual<W> &a, const Dual<W> &b) {
  Dual<W> r;
  r.v = a.v / b.v;
  const double ib = 1.0 / b.v;
#pragma unroll
  for (int i = 0; i < W; i++) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
  return r;
}
template <int W>
__host__ __device__ __forceinline__ Dual<W> operator-(const Dual<W> &a) {
  Dual<W> r;
  r.v = -a.v;
#pragma unroll
  for (int i = 0; i < W; i++) r.d[i] = -a.d[i];
  return r;
}
/* mixed forms: the double operand is a constant */
template <int W> __host__ __device__ __forceinline__ Dual<W> operator+(const Dual<W> &a, double b) { return a + Dual<W>(b); }
template <int W> __host__ __device__ __forceinline__ Dual<W> operator+(double a, const Dual<W> &b) { return Dual<W>(a) + b; }
template <int W> __host__ __device__ __forceinline__ Dual<W> operator-(const Dual<W> &a, double b) { return a - Dual<W>(b); }
template <int W> __host__ __device__ __forceinline__ Dual<W> operator-(double a, const Dual<W> &b) { return Dual<W>(a) - b; }
template <int W> __host__ __device__ __forceinline__ Dual<W> operator*(const Dual<W> &a, double b) { return a * Dual<W>(b); }
template <int W> __host__ __device__ __forceinline__ Dual<W> operator*(double a, const Dual<W> &b) { return Dual<W>(a) * b; }
template <int W> __host__ __device__ __forceinline__ Dual<W> operator/(const Dual<W> &a, double b) { return a / Dual<W>(b); }
template <int W> __host__ __device__ __forceinline__ Dual<W> operator/(double a, const Dual<W> &b) { return Dual<W>(a) / b; }
template <int W, typename U> __host__ __device__ __forceinline__ Dual<W> &operator+=(Dual<W> &a, const U &b) { return a = a + b; }
template <int W, typename U> __host__ __device__ __forceinline__ Dual<W> &operator-=(Dual<W> &a, const U &b) { return a = a - b; }
template <int W, typename U> __host__ __device__ __forceinline__ Dual<W> &operator*=(Dual<W> &a, const U &b) { return a = a * b; }
template <int W, typename U> __host__ __device__ __forceinline__ Dual<W> &operator/=(Dual<W> &a, const U &b) { return a = a / b; }

#define GPD_CMP(op)                                                                                                  \
  template <int W> __host__ __device__ __forceinline__ bool operator op(const Dual<W> &a, const Dual<W> &b) { return a.v op b.v; } \
  template <int W> __host__ __device__ __forceinline__ bool operator op(const Dual<W> &a, double b) { return a.v op b; }          \
  template <int W> __host__ __device__ __forceinline__ bool operator op(double a, const Dual<W> &b) { return a op b.v; }
GPD_CMP(<)
GPD_CMP(>)
GPD_CMP(<=)
GPD_CMP(>=)
GPD_CMP(==)
GPD_CMP(!=)
#undef GPD_CMP

template <int W>
__host__ __device__ __forceinline__ Dual<W> sqrt(const Dual<W> &a) {
  Dual<W> r;
  r.v = ::sqrt(a.v);
  const double s = 0.5 / r.v;
#pragma unroll
  for (int i = 0; i < W; i++) r.d[i] = a.d[i] * s;
  return r;
}
/* |x|: the derivative of the branch taken; at x = 0 (either sign) the
 * derivative is taken as that of +x, as in the value (fabs(-0) = +0) */
template <int W>
__host__ __device__ __forceinline__ Dual<W> fabs(const Dual<W> &a) {
  Dual<W> r;
  r.v = ::fabs(a.v);
  const double s = a.v < 0.0 ? -1.0 : 1.0;
#pragma unroll
  for (int i = 0; i < W; i++) r.d[i] = a.d[i] * s;
  return r;
}

/* the double forms stay visible next to the Dual ones inside this namespace */
using ::fabs;
using ::sqrt;

}  // namespace gpd
