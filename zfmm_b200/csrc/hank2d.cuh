// Bessel and Hankel functions of complex argument for the 2D Helmholtz FMM
// (host and device).
//
// hank01(z) -> H0^(1)(z), H1^(1)(z) on the principal branch
// (-pi < arg z <= pi, cut along the negative real axis).  A zero imaginary
// part is taken as +0, so the negative real axis belongs to the upper side,
// as in the reference's hank101/hank103 (zfmm2d/src/helmholtz/hank103.f:131-263:
// "if(rea(2) .lt. 0)" selects the lower half-plane, and -0 is not < 0).
// Methods (all from the mathematics, see DLMF chapter 10):
//   |z| < 2:          ascending series of J0, J1 and of the regular parts
//                     S_nu = Y_nu - (2/pi) log(z) J_nu  (DLMF 10.8.1-2);
//   Im z >= 0:        Hankel's integral
//                     H_nu(z) = sqrt(2/(pi z)) e^{i(z - nu pi/2 - pi/4)} / Gamma(nu+1/2)
//                               * int_0^inf e^{-t} t^{nu-1/2} (1 + i t/(2z))^{nu-1/2} dt
//                     (DLMF 10.9.E? Laplace-type form, valid for -pi/2 < arg z < 3pi/2),
//                     with t = s^2 and the trapezoidal rule in s (step 0.2, 32 nodes;
//                     the integrand is analytic in a strip of half-width >= 1.4 for
//                     |z| >= 2 in the closed upper half-plane, so the rule converges
//                     geometrically);
//   Im z < 0:         J_n by Miller's backward recurrence normalised with
//                     e^{iz} = J0 + 2 sum_n i^n J_n (|e^{iz}| >= 1 here, no
//                     cancellation), Neumann series for S0, S1 (DLMF 10.23.E?, A&S
//                     9.1.88-89 differentiated), and for Re z < 0 the reflection
//                     z -> -conj(z) of these entire functions with real Taylor
//                     coefficients; then H = J + i((2/pi) log z J + S).
// Accuracy against 160-digit mpmath: <= 2.5e-14 relative except within 1e-3 rad
// of the cut from below at |z| >~ 100 (1.4e-12), see tests/test_hankel.py.
#pragma once
#include "zcomplex.cuh"

namespace zf {

constexpr double ZF_PI = 3.14159265358979323846;
constexpr double ZF_2_PI = 0.63661977236758134308;      // 2/pi
constexpr double ZF_EULER = 0.57721566490153286061;
constexpr double ZF_LN2 = 0.69314718055994530942;
constexpr double ZF_SQRT_2_PI = 0.79788456080286535588;  // sqrt(2/pi)
constexpr double ZF_INV_SQRT_PI = 0.56418958354775628695;
constexpr int ZF_HQ_NODES = 32;
constexpr double ZF_HQ_STEP = 0.2;

// ascending series: J0, J1, S0, S1 (S = Y - (2/pi) log(z) J)
ZF_HD void bessel01_series(zdc z, zdc& J0, zdc& J1, zdc& S0, zdc& S1) {
  zdc q = 0.25 * (z * z), mq = -q;
  zdc t0 = mkz(1.0), t1 = mkz(1.0);
  zdc sj0 = t0, sj1 = t1, s0 = mkz(0.0), s1 = t1;  // s1 starts with (H_0 + H_1) t1 = t1
  double H = 0.0;
  for (int k = 1; k < 40; k++) {
    t0 = (mq * t0) / (double)(k * k);
    t1 = (mq * t1) / (double)(k * (k + 1));
    H += 1.0 / k;
    sj0 += t0;
    sj1 += t1;
    s0 += H * t0;
    s1 += (2.0 * H + 1.0 / (k + 1)) * t1;
    double a0 = t0.re * t0.re + t0.im * t0.im, b0 = sj0.re * sj0.re + sj0.im * sj0.im;
    double a1 = t1.re * t1.re + t1.im * t1.im, b1 = sj1.re * sj1.re + sj1.im * sj1.im;
    if (a0 < 1e-36 * b0 && a1 < 1e-36 * b1) break;  // |t| < 1e-18 |s|, squared
  }
  zdc zh = 0.5 * z;
  J0 = sj0;
  J1 = zh * sj1;
  double c = ZF_2_PI * (ZF_EULER - ZF_LN2);
  S0 = c * J0 - ZF_2_PI * s0;
  S1 = c * J1 - ZF_2_PI * zinv(z) - (1.0 / ZF_PI) * (zh * s1);
}

// Miller backward recurrence at w (Im w <= 0): J0, J1, S0, S1
ZF_HD void bessel01_miller(zdc w, zdc& J0, zdc& J1, zdc& S0, zdc& S1) {
  double aw = zabs(w);
  int N = (int)(aw + 30.0 + 3.0 * cbrt(aw));
  N += N & 1;
  zdc iw2 = 2.0 * zinv(w);
  zdc fp1 = mkz(0.0), f = mkz(1e-30);  // f_{n+1}, f_n at n = N
  // accumulators (unnormalised): norm = f0 + 2 sum i^n f_n, a0 = sum_k (-1)^k f_2k / k,
  // a1 = sum over odd n of c(n) f_n (see header), f0, f1
  zdc norm = mkz(0.0), a0 = mkz(0.0), a1 = mkz(0.0), f0 = mkz(0.0), f1 = mkz(0.0);
  for (int n = N; n >= 0; n--) {
    // f holds f_n
    if (n == 0) {
      norm += f;
      f0 = f;
    } else {
      int r = n & 3;  // i^n
      zdc in_f = r == 0 ? f : (r == 1 ? zmul_i(f) : (r == 2 ? -f : -zmul_i(f)));
      norm += 2.0 * in_f;
      if ((n & 1) == 0) {
        int k = n / 2;
        a0 += ((k & 1) ? -1.0 : 1.0) / k * f;
      } else {
        int kp = (n + 1) / 2;
        double c = ((kp & 1) ? -1.0 : 1.0) / kp;
        if (n >= 3) {
          int km = (n - 1) / 2;
          c -= ((km & 1) ? -1.0 : 1.0) / km;
        }
        a1 += c * f;
        if (n == 1) f1 = f;
      }
      zdc fm1 = ((double)n * iw2) * f - fp1;
      fp1 = f;
      f = fm1;
      if (zbig(f, 1e250)) {
        const double sc = 1e-250;
        f = sc * f; fp1 = sc * fp1; norm = sc * norm; a0 = sc * a0; a1 = sc * a1; f1 = sc * f1;
      }
    }
  }
  zdc scale = zexp_p(zmul_i(w)) / norm;
  J0 = scale * f0;
  J1 = scale * f1;
  double c = ZF_2_PI * (ZF_EULER - ZF_LN2);
  S0 = c * J0 - (2.0 * ZF_2_PI) * (scale * a0);
  S1 = c * J1 - ZF_2_PI * (zinv(w) * J0) + ZF_2_PI * (scale * a1);
}

// Hankel's integral, Im z >= 0, |z| >= 2
ZF_HD void hank01_integral(zdc z, zdc& h0, zdc& h1) {
  zdc c = zmul_i(zinv(2.0 * z));  // i/(2z)
  zdc f0 = mkz(0.0), f1 = mkz(0.0);
  for (int k = 0; k < ZF_HQ_NODES; k++) {
    double s = ZF_HQ_STEP * k, s2 = s * s;
    double w = ZF_HQ_STEP * exp(-s2) * (k == 0 ? 0.5 : 1.0);
    zdc g = mkz(1.0) + s2 * c;
    zdc r = zsqrt_p(g);
    f0 += w * zinv(r);
    f1 += (w * s2) * r;
  }
  zdc pre = ZF_SQRT_2_PI * zinv(zsqrt_p(z));
  zdc e = zexp_p(zmul_i(z));
  // e^{-i pi/4} and e^{-i 3pi/4}
  const double r2 = 0.70710678118654752440;
  zdc p0 = pre * (e * zdc{r2, -r2}), p1 = pre * (e * zdc{-r2, -r2});
  h0 = (2.0 * ZF_INV_SQRT_PI) * (p0 * f0);
  h1 = (4.0 * ZF_INV_SQRT_PI) * (p1 * f1);
}

ZF_HD void hank01(zdc z, zdc& h0, zdc& h1) {
  if (z.im == 0.0) z.im = 0.0;  // -0 -> +0
  double az = zabs(z);
  zdc J0, J1, S0, S1;
  if (az < 2.0) {
    bessel01_series(z, J0, J1, S0, S1);
  } else if (z.im >= 0.0) {
    hank01_integral(z, h0, h1);
    return;
  } else if (z.re >= 0.0) {
    bessel01_miller(z, J0, J1, S0, S1);
  } else {
    zdc w = zdc{-z.re, z.im};  // -conj(z), lower-right quadrant
    bessel01_miller(w, J0, J1, S0, S1);
    J0 = zconj(J0);
    J1 = -zconj(J1);
    S0 = zconj(S0);
    S1 = -zconj(S1);
  }
  zdc L = ZF_2_PI * zlog_p(z);
  h0 = J0 + zmul_i(L * J0 + S0);
  h1 = J1 + zmul_i(L * J1 + S1);
}

// Scaled Hankel functions hvec(n) = H_n(z) rscale^n, n = 0..nterms, and
// derivatives hder(n) = H_n'(z) rscale^n (h2dall, zfmm2d/src/helmholtz/h2dcommon.f:71-173:
// forward recurrence H_{n+1} = (2n/z) H_n - H_{n-1}, zero output for |z| < 1e-200).
ZF_HD void h2dall(int nterms, zdc z, double rscale, zdc* hvec, int ifder, zdc* hder) {
  if (zabs(z) < 1e-200) {
    for (int i = 0; i <= nterms; i++) {
      hvec[i] = mkz(0.0);
      if (ifder == 1) hder[i] = mkz(0.0);
    }
    return;
  }
  zdc h0, h1;
  hank01(z, h0, h1);
  hvec[0] = h0;
  if (nterms >= 1) hvec[1] = h1 * rscale;
  double sc2 = rscale * rscale;
  zdc zi = rscale * zinv(z);
  for (int i = 1; i < nterms; i++) hvec[i + 1] = ((2.0 * i) * zi) * hvec[i] - sc2 * hvec[i - 1];
  if (ifder == 1) {
    hder[0] = -hvec[1] / rscale;
    zdc zi1 = zinv(z);
    for (int i = 1; i <= nterms; i++) hder[i] = rscale * hvec[i - 1] - ((double)i * zi1) * hvec[i];
  }
}

// Start index of the backward recurrence for J_n, n <= nterms: the first n >=
// nterms where the forward recurrence from (J_{nterms-1}, J_nterms) ~ (0, 1)
// has grown past 1e20 (the same criterion as the reference's jbessel2d,
// cdjseval2d.f:23-221), plus one.
ZF_HD int jbessel_top(int nterms, zdc z) {
  zdc zi = zinv(z), fm1 = mkz(0.0), f = mkz(1.0);
  for (int i = nterms; i < nterms + 100000; i++) {
    zdc fp = ((2.0 * i) * zi) * f - fm1;
    if (fp.re * fp.re + fp.im * fp.im > 1e40) return i + 1;
    fm1 = f;
    f = fp;
  }
  return nterms + 100000;
}

// Scaled Bessel functions fjs(n) = J_n(z) / rscale^n, n = 0..nterms, and
// derivatives fjder(n) = d fjs(n)/dz (jbessel2d, cdjseval2d.f:23-221): Miller's
// backward recurrence normalised by e^{-iz} = J0 + 2 sum (-i)^n J_n for Im z >= 0
// and e^{iz} = J0 + 2 sum i^n J_n for Im z < 0.  fjs and fjder need nterms+2
// entries (fjs(nterms+1) is used for the derivatives).  `tmp` needs
// jbessel_top(nterms, z) + 1 entries.
ZF_HD void jbessel2d(int nterms, zdc z, double rscale, zdc* fjs, int ifder, zdc* fjder,
                     zdc* tmp, int ntop) {
  if (zabs(z) < 1e-200) {
    fjs[0] = mkz(1.0);
    for (int i = 1; i <= nterms + 1; i++) fjs[i] = mkz(0.0);
    if (ifder == 1) {
      for (int i = 0; i <= nterms; i++) fjder[i] = mkz(0.0);
      if (nterms >= 1) fjder[1] = mkz(1.0 / (2.0 * rscale));
    }
    return;
  }
  zdc zi = zinv(z);
  // backward recurrence for g_n = f_n / rscale^n:
  //   g_{n-1} = (2n/z) rscale g_n - rscale^2 g_{n+1};
  // on overflow every value computed so far is scaled down by 1e-200 (rare:
  // the start index keeps the growth between ntop and nterms near 1e20).
  tmp[ntop] = mkz(0.0);
  tmp[ntop - 1] = mkz(1.0);
  double sc2 = rscale * rscale;
  zdc zr = rscale * zi;
  for (int n = ntop - 1; n >= 1; n--) {
    tmp[n - 1] = ((2.0 * n) * zr) * tmp[n] - sc2 * tmp[n + 1];
    if (zbig(tmp[n - 1], 1e200))
      for (int k = n - 1; k <= ntop; k++) tmp[k] = 1e-200 * tmp[k];
  }
  // normalisation: psi = g_0 + 2 sum_n (zmul)^n rscale^n g_n
  zdc zmul = z.im < 0.0 ? mkz(0.0, 1.0) : mkz(0.0, -1.0);
  zdc psi = mkz(0.0);
  for (int n = ntop; n >= 1; n--) {
    int r = n & 3;
    zdc zn = r == 0 ? mkz(1.0) : (r == 1 ? zmul : (r == 2 ? mkz(-1.0) : -zmul));
    psi = rscale * psi + zn * tmp[n];
  }
  psi = 2.0 * rscale * psi + tmp[0];
  zdc e = z.im < 0.0 ? zexp_p(zmul_i(z)) : zexp_p(-zmul_i(z));
  zdc sc = e / psi;
  for (int i = 0; i <= nterms + 1 && i <= ntop; i++) fjs[i] = tmp[i] * sc;
  if (ifder == 1) {
    fjder[0] = -fjs[1] * rscale;
    double d1 = 0.5 / rscale, d2 = 0.5 * rscale;
    for (int i = 1; i <= nterms; i++) fjder[i] = d1 * fjs[i - 1] - d2 * fjs[i + 1];
  }
}

}  // namespace zf
