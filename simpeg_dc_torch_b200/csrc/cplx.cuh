// Double-precision complex numbers for the complex-symmetric factor and solve
// (plans of dtype DCT_C128): the same multifrontal kernels as the float64
// path, instantiated with this type.  A complex-symmetric matrix (A^T = A,
// not Hermitian) factors as A = L L^T without conjugation, so every real
// kernel carries over with complex arithmetic; the pivot test becomes
// "finite and non-zero" and the square root is the principal one.
// Layout: two doubles (re, im), 16-byte aligned, the layout of torch's
// complex128 and of C's double _Complex.
#pragma once
#include <cuda_runtime.h>

#include <cmath>

namespace dct {

// the overloads below must not hide the real ones inside this namespace
using ::atomicAdd;
using ::sqrt;
using ::__shfl_sync;

struct __align__(16) cplx {
  double re, im;
  __host__ __device__ constexpr cplx() : re(0.0), im(0.0) {}
  __host__ __device__ constexpr cplx(double r) : re(r), im(0.0) {}
  __host__ __device__ constexpr cplx(double r, double i) : re(r), im(i) {}
  __host__ __device__ cplx& operator+=(const cplx& o) {
    re += o.re;
    im += o.im;
    return *this;
  }
  __host__ __device__ cplx& operator-=(const cplx& o) {
    re -= o.re;
    im -= o.im;
    return *this;
  }
  __host__ __device__ cplx& operator*=(const cplx& o) {
    const double r = re * o.re - im * o.im;
    im = re * o.im + im * o.re;
    re = r;
    return *this;
  }
};

__host__ __device__ inline cplx operator+(cplx a, const cplx& b) { return a += b; }
__host__ __device__ inline cplx operator-(cplx a, const cplx& b) { return a -= b; }
__host__ __device__ inline cplx operator*(cplx a, const cplx& b) { return a *= b; }
__host__ __device__ inline cplx operator-(const cplx& a) { return cplx(-a.re, -a.im); }

// a / b by Smith's method (scaled by the larger of |Re b|, |Im b|, so that
// neither overflows nor underflows on the way)
__host__ __device__ inline cplx operator/(const cplx& a, const cplx& b) {
  if (fabs(b.re) >= fabs(b.im)) {
    const double r = b.im / b.re, d = b.re + b.im * r;
    return cplx((a.re + a.im * r) / d, (a.im - a.re * r) / d);
  }
  const double r = b.re / b.im, d = b.re * r + b.im;
  return cplx((a.re * r + a.im) / d, (a.im * r - a.re) / d);
}

// principal square root: |z| from hypot, then the half-angle formulas
__host__ __device__ inline cplx sqrt(const cplx& z) {
  if (z.re == 0.0 && z.im == 0.0) return cplx(0.0, 0.0);
  const double m = hypot(z.re, z.im);
  double a = ::sqrt(0.5 * (m + fabs(z.re)));
  double b = z.im / (2.0 * a);
  if (z.re >= 0.0) return cplx(a, b);
  return cplx(fabs(b), z.im >= 0.0 ? a : -a);
}

// a usable pivot of the complex-symmetric LL^T: finite and not zero
__device__ __forceinline__ bool good_pivot(const cplx& v) {
  const double m = fabs(v.re) + fabs(v.im);
  return m > 0.0 && m < INFINITY;
}

__device__ __forceinline__ cplx inv_sqrt(const cplx& x) { return cplx(1.0) / sqrt(x); }

__device__ __forceinline__ cplx __shfl_sync(unsigned mask, const cplx& v, int src,
                                            int width = 32) {
  return cplx(::__shfl_sync(mask, v.re, src, width), ::__shfl_sync(mask, v.im, src, width));
}

__device__ __forceinline__ void atomicAdd(cplx* p, const cplx& v) {
  ::atomicAdd(&p->re, v.re);
  ::atomicAdd(&p->im, v.im);
}

}  // namespace dct
