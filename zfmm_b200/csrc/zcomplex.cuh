// Complex double arithmetic for host and device.
//
// The elementary complex functions are built from their definitions on the
// principal branch (arg in (-pi, pi]), calling the real sqrt/log/exp/atan2
// /hypot/sincos of the CUDA math library:
//   sqrt(z): t = sqrt((|x| + |z|)/2);  x >= 0 -> (t, y/(2t)),
//            x < 0 -> (|y|/(2t), copysign(t, y))       (no cancellation)
//   log(z):  (log|z|, atan2(y, x))
//   exp(z):  e^x (cos y, sin y)
// These match the signed-zero conventions of the C99 / Fortran intrinsics the
// reference relies on (sqrt(-1-0i) = -i, log(-1-0i) = -i pi).
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#define ZF_HD __host__ __device__ __forceinline__

struct __align__(16) zdc {
  double re, im;
};

ZF_HD zdc mkz(double r, double i = 0.0) { return zdc{r, i}; }
ZF_HD zdc operator+(zdc a, zdc b) { return zdc{a.re + b.re, a.im + b.im}; }
ZF_HD zdc operator-(zdc a, zdc b) { return zdc{a.re - b.re, a.im - b.im}; }
ZF_HD zdc operator-(zdc a) { return zdc{-a.re, -a.im}; }
ZF_HD zdc operator*(zdc a, zdc b) {
  return zdc{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
ZF_HD zdc operator*(double s, zdc a) { return zdc{s * a.re, s * a.im}; }
ZF_HD zdc operator*(zdc a, double s) { return zdc{s * a.re, s * a.im}; }
ZF_HD zdc operator/(zdc a, double s) { return zdc{a.re / s, a.im / s}; }
ZF_HD zdc& operator+=(zdc& a, zdc b) { a.re += b.re; a.im += b.im; return a; }
ZF_HD zdc& operator-=(zdc& a, zdc b) { a.re -= b.re; a.im -= b.im; return a; }
ZF_HD zdc zconj(zdc a) { return zdc{a.re, -a.im}; }
ZF_HD zdc zmul_i(zdc a) { return zdc{-a.im, a.re}; }  // i*a
ZF_HD double zabs(zdc a) { return hypot(a.re, a.im); }

// a / b with Smith's scaling (avoids overflow of |b|^2)
ZF_HD zdc zdiv_smith(zdc a, zdc b) {
  if (fabs(b.re) >= fabs(b.im)) {
    double r = b.im / b.re, d = b.re + b.im * r;
    return zdc{(a.re + a.im * r) / d, (a.im - a.re * r) / d};
  } else {
    double r = b.re / b.im, d = b.re * r + b.im;
    return zdc{(a.re * r + a.im) / d, (a.im * r - a.re) / d};
  }
}
// a / b = a conj(b) / |b|^2 with one real division where neither |b|^2 nor
// the products can overflow or underflow (|b|^2 in [1e-290, 1e290], parts of
// a below 1e150); Smith's form otherwise (and for NaN / Inf operands)
ZF_HD zdc operator/(zdc a, zdc b) {
  const double d = b.re * b.re + b.im * b.im;
  if (d > 1e-290 && d < 1e290 && fabs(a.re) < 1e150 && fabs(a.im) < 1e150) {
    const double r = 1.0 / d;
    return zdc{(a.re * b.re + a.im * b.im) * r, (a.im * b.re - a.re * b.im) * r};
  }
  return zdiv_smith(a, b);
}
ZF_HD zdc zinv(zdc b) {
  const double d = b.re * b.re + b.im * b.im;
  if (d > 1e-290 && d < 1e290) {
    const double r = 1.0 / d;
    return zdc{b.re * r, -b.im * r};
  }
  return zdiv_smith(mkz(1.0), b);
}
ZF_HD zdc operator/(double a, zdc b) { return a * zinv(b); }
// max(|Re a|, |Im a|) > t: the overflow guard of the recurrences (within a
// factor sqrt(2) of |a| > t, without the square root)
ZF_HD bool zbig(zdc a, double t) { return fabs(a.re) > t || fabs(a.im) > t; }

ZF_HD zdc zsqrt_p(zdc z) {
  double x = z.re, y = z.im;
  if (x == 0.0 && y == 0.0) return zdc{0.0, y};
  double t = sqrt((fabs(x) + hypot(x, y)) * 0.5);
  if (x >= 0.0) return zdc{t, y / (2.0 * t)};
  return zdc{fabs(y) / (2.0 * t), copysign(t, y)};
}
ZF_HD zdc zlog_p(zdc z) { return zdc{log(hypot(z.re, z.im)), atan2(z.im, z.re)}; }
ZF_HD zdc zexp_p(zdc z) {
  double e = exp(z.re), s, c;
#ifdef __CUDA_ARCH__
  sincos(z.im, &s, &c);
#else
  s = sin(z.im);
  c = cos(z.im);
#endif
  return zdc{e * c, e * s};
}
// z^n, n >= 0, by binary powering
ZF_HD zdc zpown(zdc z, int n) {
  zdc r = mkz(1.0);
  while (n > 0) {
    if (n & 1) r = r * z;
    z = z * z;
    n >>= 1;
  }
  return r;
}

#ifdef __CUDACC__
__device__ __forceinline__ zdc shfl_xor_z(zdc v, int m) {
  return zdc{__shfl_xor_sync(0xffffffffu, v.re, m), __shfl_xor_sync(0xffffffffu, v.im, m)};
}
__device__ __forceinline__ zdc ldz(const zdc* p) {
  double2 v = __ldg(reinterpret_cast<const double2*>(p));
  return zdc{v.x, v.y};
}
#endif
