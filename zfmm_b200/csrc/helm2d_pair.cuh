// One source-target interaction of zh2devaldirect
// (zfmm2d/src/helmholtz/zhfmm2d.f:773-838), unscaled (the driver applies i/4):
//   pot  += q H0(zk R) + ds (v . (y - x)) zk H1(zk R) / R
//   grad += -q zk H1 (x - y)/R + dipole terms through H1' = (H0 - H2)/2
// with R = sqrt((y1-x1)^2 + (y2-x2)^2) on the principal branch.  The pair is
// skipped unless |zk R| > 1E-16 (a REAL*4 literal in the reference) and
// Im(zk R) > -32, as in the reference.
//
// Near pairs (|z| < 2, z = zk R: the ascending-series region of hank01) are
// evaluated without forming R.  Every quantity the pair needs is a function
// of w = R^2: with the series of J0, J1/z and of the regular parts S0, S1 in
// q = z^2/4 = zk^2 w/4 (hank2d.cuh),
//   H0      = J0 + i (L J0 + S0),      L = (2/pi) log z
//   H1 / R  = (zk/2) sJ1 (1 + i (L + c)) - i ((2/pi)/(zk w) + (zk/(2 pi)) sS1)
//   zk H1' / R^2 - H1 / R^3 = (zk H0 - 2 H1/R) / w
// (J1 = (z/2) sJ1, S1 = c J1 - (2/pi)/z - (z/(2 pi)) sS1, z/R = zk), and
// log z = log zk + log(w)/2, which is the principal logarithm of zk sqrt(w)
// when |arg zk| < pi/2 (arg sqrt(w) lies in (-pi/2, pi/2]).  The identities
// are exact; the results differ from the R-based evaluation by rounding only.
// Other pairs, or Re zk <= 0, take the R-based evaluation with hank01.
#pragma once
#include "hank2d.cuh"

namespace zf {

// per-wavenumber constants of the pair evaluation
struct HelmK {
  zdc zk, zk2, izk, lzk;  // zk, zk^2, 1/zk, log zk
  double azk4;            // |zk|^4
  bool near_ok;           // Re zk > 0: the R-free near-pair form applies
};

ZF_HD HelmK helm_k(zdc zk) {
  HelmK K;
  K.zk = zk;
  K.zk2 = zk * zk;
  K.izk = zinv(zk);
  K.lzk = zlog_p(zk);
  double a2 = zk.re * zk.re + zk.im * zk.im;
  K.azk4 = a2 * a2;
  K.near_ok = zk.re > 0.0;
  return K;
}

// Coefficients of the ascending series as power series in x = -z^2/4:
//   J0      = sum_k a_k x^k,  a_k = 1/(k!)^2
//   2 J1/z  = sum_k b_k x^k,  b_k = 1/(k! (k+1)!)
//   s0      = sum_k H_k a_k x^k                       (H_k = 1 + 1/2 + ... + 1/k)
//   s1      = sum_k (2 H_k + 1/(k+1)) b_k x^k
// (DLMF 10.8.1-2 with the harmonic sums of the regular parts), and
// r4_k = 1/k^4 for the choice of the number of terms, k = 0..40.
struct SeriesCoef {
  double a[41], b[41], c[41], d[41], r4[41];
};
constexpr SeriesCoef make_series_coef() {
  SeriesCoef r{};
  double a = 1.0, b = 1.0, H = 0.0;
  for (int k = 0; k <= 40; k++) {
    if (k >= 1) {
      a /= (double)k * (double)k;
      b /= (double)k * (double)(k + 1);
      H += 1.0 / (double)k;
      r.r4[k] = 1.0 / ((double)k * k * k * k);
    }
    r.a[k] = a;
    r.b[k] = b;
    r.c[k] = H * a;
    r.d[k] = (2.0 * H + 1.0 / (double)(k + 1)) * b;
  }
  return r;
}
static __constant__ SeriesCoef c_series = make_series_coef();

template <bool GRAD>
__device__ __forceinline__ void helm_pair(const HelmK& K, zdc x1, zdc x2, zdc y1, zdc y2, zdc q,
                                          zdc ds, zdc d1, zdc d2, int ifcharge, int ifdipole,
                                          zdc& pot, zdc& g1, zdc& g2) {
  const zdc zk = K.zk;
  zdc y1mx1 = y1 - x1, y2mx2 = y2 - x2;
  zdc w = y1mx1 * y1mx1 + y2mx2 * y2mx2;
  double az4 = K.azk4 * (w.re * w.re + w.im * w.im);  // |z|^4
  if (K.near_ok && az4 < 16.0) {
    const double thr = (double)1e-16f;  // REAL*4 literal of the exclusion test
    if (!(az4 > (thr * thr) * (thr * thr))) return;
    // ascending series in x = -z^2/4 with the terms k = 0..nk, nk the last k
    // with |x|^k / (k!)^2 >= 1e-20 (the terms fall monotonically for
    // |x| < 4), |J0| > 0.2 and |2 J1/z| > 0.5 for |z| < 2, so the first term
    // left out is below 1e-19 of the sums
    const zdc x = -(0.25 * (K.zk2 * w));
    const double ax2 = x.re * x.re + x.im * x.im;
    int nk = 0;
    for (double tt = 1.0; nk < 39;) {  // tt = (|x|^k / (k!)^2)^2 of k = nk + 1
      tt *= ax2 * c_series.r4[nk + 1];
      if (tt < 1e-40) break;
      nk++;
    }
    zdc sj0 = mkz(1.0), sj1 = mkz(1.0), s0 = mkz(0.0), s1 = mkz(1.0), xp = x;
    for (int k = 1; k <= nk; k++) {
      sj0 += c_series.a[k] * xp;
      sj1 += c_series.b[k] * xp;
      s0 += c_series.c[k] * xp;
      s1 += c_series.d[k] * xp;
      xp = xp * x;
    }
    const double c = ZF_2_PI * (ZF_EULER - ZF_LN2);
    zdc L = ZF_2_PI * (K.lzk + 0.5 * zlog_p(w));
    zdc J0 = sj0;
    zdc S0 = c * J0 - ZF_2_PI * s0;
    zdc h0 = J0 + zmul_i(L * J0 + S0);
    zdc iw = zinv(w);
    zdc hz = (0.5 * sj1) * zk;  // J1 / R
    zdc G = hz + zmul_i((L + mkz(c)) * hz - ZF_2_PI * (K.izk * iw) - (0.5 / ZF_PI) * (zk * s1));
    zdc zh1r = zk * G;  // zk H1 / R
    if (ifcharge) {
      pot += q * h0;
      if (GRAD) {
        zdc f = q * zh1r;
        g1 += f * y1mx1;
        g2 += f * y2mx2;
      }
    }
    if (ifdipole) {
      zdc tmp = d1 * y1mx1 + d2 * y2mx2;
      pot += ds * (tmp * zh1r);
      if (GRAD) {
        zdc a = (zk * h0 - 2.0 * G) * iw;  // multiplies x - y = -(y - x)
        zdc dsz = ds * zk;
        g1 += dsz * ((-a * y1mx1) * tmp) - ds * zh1r * d1;
        g2 += dsz * ((-a * y2mx2) * tmp) - ds * zh1r * d2;
      }
    }
    return;
  }
  zdc rz = zsqrt_p(w);
  zdc z = rz * zk;
  if (!(zabs(z) > (double)1e-16f && z.im > -32.0)) return;  // REAL*4 literal 1E-16
  zdc h0, h1;
  hank01(z, h0, h1);
  zdc irz = zinv(rz);
  zdc zh1 = zk * h1;
  if (ifcharge) {
    pot += q * h0;
    if (GRAD) {
      zdc f = q * (zh1 * irz);
      g1 += f * y1mx1;  // -q zk h1 (x - y)/rz
      g2 += f * y2mx2;
    }
  }
  if (ifdipole) {
    zdc tmp = d1 * y1mx1 + d2 * y2mx2;
    pot += ds * (tmp * (zh1 * irz));
    if (GRAD) {
      zdc h2 = (2.0 * zinv(z)) * h1 - h0;
      zdc dh1 = 0.5 * (h0 - h2);
      zdc irz2 = irz * irz, irz3 = irz2 * irz;
      zdc a = zk * dh1 * irz2 - h1 * irz3;  // multiplies x - y = -(y - x)
      zdc dsz = ds * zk;
      g1 += dsz * ((-a * y1mx1) * tmp) - ds * (zh1 * irz) * d1;
      g2 += dsz * ((-a * y2mx2) * tmp) - ds * (zh1 * irz) * d2;
    }
  }
}

}  // namespace zf
