// Spherical Hankel and Bessel functions of complex argument, scaled as the
// reference's h3dall (zfmm3d/src/helmholtz/h3dcommon.f:59-140):
//   h[n] = h_n(z) scale^n,   hd[n] = h_n'(z) scale^n
// and besseljs3d (zfmm3d/src/helmholtz/besseljs3d.f:5-169):
//   f[n] = j_n(z) / scale^n,  fd[n] = d/dz of f[n]
// restated for host and device.  besseljs3d_z runs the reference's upward
// search for the start order (|f|^2 > 1e40), the downward Miller recurrence
// with rescaling by 1e-40, and normalisation against j_0 or j_1 (whichever
// is larger), keeping only the orders 0..n+1 it needs (n <= 126).
#pragma once
#include "zcomplex.cuh"

namespace zf {

ZF_HD zdc zsin_c(zdc z) {
  double s, c;
#ifdef __CUDA_ARCH__
  sincos(z.re, &s, &c);
#else
  s = sin(z.re);
  c = cos(z.re);
#endif
  return mkz(s * cosh(z.im), c * sinh(z.im));
}
ZF_HD zdc zcos_c(zdc z) {
  double s, c;
#ifdef __CUDA_ARCH__
  sincos(z.re, &s, &c);
#else
  s = sin(z.re);
  c = cos(z.re);
#endif
  return mkz(c * cosh(z.im), -(s * sinh(z.im)));
}

// h3d01 (h3dcommon.f:16-55) and h3dall; h and hd hold n+2 entries (hd may be
// null when no derivative is wanted)
ZF_HD void h3dall_z(int n, zdc z, double scale, zdc* h, zdc* hd) {
  if (zabs(z) < 1.0e-15) {
    for (int i = 0; i <= n; i++) {
      h[i] = mkz(0.0);
      if (hd) hd[i] = mkz(0.0);
    }
    return;
  }
  zdc cd = zmul_i(z);
  zdc h0 = zexp_p(cd) / cd;
  h[0] = h0;
  h[1] = (h0 * (zinv(z) - mkz(0.0, 1.0))) * scale;
  double scal2 = scale * scale;
  zdc zi = scale / z;
  for (int i = 1; i <= n - 1; i++) h[i + 1] = (zi * (2 * i + 1.0)) * h[i] - scal2 * h[i - 1];
  if (hd) {
    hd[0] = -(h[1] / scale);
    zdc zi1 = zinv(z);
    for (int i = 1; i <= n; i++) hd[i] = scale * h[i - 1] - (zi1 * (i + 1.0)) * h[i];
  }
}

// besseljs3d, n <= 126; f holds n+2 entries, fd n+1 (fd may be null)
ZF_HD void besseljs3d_z(int n, zdc z, double scale, zdc* f, zdc* fd) {
  const double up2 = 1.0e40, up2inv = 1.0e-40;
  if (zabs(z) < 1.0e-200) {
    f[0] = mkz(1.0);
    for (int i = 1; i <= n; i++) f[i] = mkz(0.0);
    if (fd) {
      for (int i = 0; i <= n; i++) fd[i] = mkz(0.0);
      if (n >= 1) fd[1] = mkz(1.0 / (3 * scale));
    }
    return;
  }
  zdc zi = zinv(z);
  // step 1: start order
  zdc fm1 = mkz(0.0), f0 = mkz(1.0);
  int ntop = n + 100000;
  for (int i = n; i <= n + 100000; i++) {
    zdc f1 = ((2 * i + 1.0) * zi) * f0 - fm1;
    double a = zabs(f1);
    if (a * a > up2) {
      ntop = i + 1;
      break;
    }
    fm1 = f0;
    f0 = f1;
  }
  // step 2: downward recurrence; orders <= n+1 are kept in f, rescale events
  // at orders <= n in two bit masks (later events do not reach these orders)
  unsigned long long sc0 = 0, sc1 = 0;
  zdc a = mkz(0.0), b = mkz(1.0);  // orders i+1, i
  if (ntop <= n + 1) f[ntop] = mkz(0.0);
  for (int i = ntop - 1; i >= 1; i--) {
    zdc c = ((2 * i + 1.0) * zi) * b - a;  // order i-1
    double ac = zabs(c);
    if (ac * ac > up2) {
      b = b * up2inv;
      c = c * up2inv;
      if (i <= n) {
        if (i < 64) sc0 |= 1ull << i;
        else sc1 |= 1ull << (i - 64);
      }
    }
    if (i <= n + 1) f[i] = b;
    a = b;
    b = c;
  }
  f[0] = b;
  // step 3: common scaling
  double sinv = 1.0 / scale, sct = 1.0;
  for (int i = 1; i <= n + 1; i++) {
    sct = sct * sinv;
    int k = i - 1;
    bool ev = k < 64 ? ((sc0 >> k) & 1ull) : ((sc1 >> (k - 64)) & 1ull);
    if (ev) sct = sct * up2inv;
    f[i] = f[i] * sct;
  }
  // normalisation
  zdc j0 = zsin_c(z) * zi;
  zdc j1 = j0 * zi - zcos_c(z) * zi;
  zdc zs = (zabs(j1) > zabs(j0)) ? j1 / (f[1] * scale) : j0 / f[0];
  if (fd) {
    fd[0] = -((f[1] * zs) * scale);
    for (int i = 1; i <= n; i++) {
      double dc1 = i / (2 * i + 1.0), dc2 = 1.0 - dc1;
      dc1 = dc1 * sinv;
      dc2 = dc2 * scale;
      fd[i] = (dc1 * f[i - 1] - dc2 * f[i + 1]) * zs;
    }
  }
  for (int i = 0; i <= n; i++) f[i] = f[i] * zs;
}

}  // namespace zf
