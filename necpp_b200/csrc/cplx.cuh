// Device complex arithmetic for the FP64 kernels.
//
// The reference does its complex arithmetic with std::complex<double>
// (libstdc++ / libgcc).  To track it to a few ulps the operations here use
// the same textbook forms: (ac-bd, ad+bc) products, Smith's division
// (libgcc __divdc3 for finite operands), the principal square root in the
// hypot-based form, exp(x)(cos y, sin y).
#pragma once
#include <cuda_runtime.h>

namespace necb {

struct cplx {
  double re, im;
};

__host__ __device__ __forceinline__ cplx mk(double r, double i) { return cplx{r, i}; }
__host__ __device__ __forceinline__ cplx operator+(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
__host__ __device__ __forceinline__ cplx operator-(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
__host__ __device__ __forceinline__ cplx operator-(cplx a) { return {-a.re, -a.im}; }
__host__ __device__ __forceinline__ cplx operator*(cplx a, cplx b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__host__ __device__ __forceinline__ cplx operator*(cplx a, double s) { return {a.re * s, a.im * s}; }
__host__ __device__ __forceinline__ cplx operator*(double s, cplx a) { return {s * a.re, s * a.im}; }
__host__ __device__ __forceinline__ cplx operator/(cplx a, double s) { return {a.re / s, a.im / s}; }
__host__ __device__ __forceinline__ cplx operator+(cplx a, double s) { return {a.re + s, a.im}; }
__host__ __device__ __forceinline__ cplx operator+(double s, cplx a) { return {s + a.re, a.im}; }
__host__ __device__ __forceinline__ cplx operator-(double s, cplx a) { return {s - a.re, -a.im}; }
__host__ __device__ __forceinline__ cplx operator-(cplx a, double s) { return {a.re - s, a.im}; }
__host__ __device__ __forceinline__ cplx& operator+=(cplx& a, cplx b) {
  a.re += b.re;
  a.im += b.im;
  return a;
}
__host__ __device__ __forceinline__ cplx& operator-=(cplx& a, cplx b) {
  a.re -= b.re;
  a.im -= b.im;
  return a;
}

// Smith's algorithm (R. L. Smith, CACM 5(8), 1962), the finite-operand path
// of libgcc's __divdc3.
__host__ __device__ __forceinline__ cplx operator/(cplx a, cplx b) {
  double c = b.re, d = b.im;
  if (fabs(c) < fabs(d)) {
    double ratio = c / d;
    double denom = (c * ratio) + d;
    return {((a.re * ratio) + a.im) / denom, ((a.im * ratio) - a.re) / denom};
  }
  double ratio = d / c;
  double denom = (d * ratio) + c;
  return {((a.im * ratio) + a.re) / denom, (a.im - (a.re * ratio)) / denom};
}
__host__ __device__ __forceinline__ cplx operator/(double s, cplx b) { return cplx{s, 0.0} / b; }

__host__ __device__ __forceinline__ double cnorm(cplx a) { return a.re * a.re + a.im * a.im; }
__host__ __device__ __forceinline__ double cabs_(cplx a) { return hypot(a.re, a.im); }

// Principal square root (branch cut on the negative real axis, sign of the
// imaginary part follows the argument's), W. Kahan's formulation.
__host__ __device__ __forceinline__ cplx csqrt_(cplx z) {
  double x = z.re, y = z.im;
  if (y == 0.0) {
    if (x >= 0.0) return {sqrt(x), y};
    return {0.0, copysign(sqrt(-x), y)};
  }
  if (x == 0.0) {
    double r = sqrt(0.5 * fabs(y));
    return {r, copysign(r, y)};
  }
  double d = hypot(x, y);
  if (x > 0.0) {
    double r = sqrt(0.5 * (d + x));
    double s = 0.5 * (y / r);
    return {r, s};
  }
  double s = sqrt(0.5 * (d - x));
  double r = fabs(0.5 * (y / s));
  return {r, copysign(s, y)};
}

__host__ __device__ __forceinline__ cplx cexp_(cplx z) {
  double e = exp(z.re);
  double s, c;
  sincos(z.im, &s, &c);
  return {e * c, e * s};
}

}  // namespace necb
