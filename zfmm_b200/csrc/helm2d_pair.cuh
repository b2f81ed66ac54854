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

// reciprocals of k^2, k (k+1) and k for the ascending series, k = 0..40
struct SeriesRecip {
  double k2[41], kk1[41], k1[42];
};
constexpr SeriesRecip make_series_recip() {
  SeriesRecip r{};
  for (int k = 1; k <= 40; k++) {
    r.k2[k] = 1.0 / (double)(k * k);
    r.kk1[k] = 1.0 / (double)(k * (k + 1));
  }
  for (int k = 1; k <= 41; k++) r.k1[k] = 1.0 / (double)k;
  return r;
}
static __constant__ SeriesRecip c_series = make_series_recip();

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
    // ascending series in q = z^2/4 (bessel01_series with the convergence
    // test on squared moduli)
    zdc mq = -(0.25 * (K.zk2 * w));
    zdc t0 = mkz(1.0), t1 = mkz(1.0);
    zdc sj0 = t0, sj1 = t1, s0 = mkz(0.0), s1 = t1;
    double H = 0.0;
    for (int k = 1; k < 40; k++) {
      t0 = (mq * t0) * c_series.k2[k];
      t1 = (mq * t1) * c_series.kk1[k];
      H += c_series.k1[k];
      sj0 += t0;
      sj1 += t1;
      s0 += H * t0;
      s1 += (2.0 * H + c_series.k1[k + 1]) * t1;
      double a0 = t0.re * t0.re + t0.im * t0.im, b0 = sj0.re * sj0.re + sj0.im * sj0.im;
      double a1 = t1.re * t1.re + t1.im * t1.im, b1 = sj1.re * sj1.re + sj1.im * sj1.im;
      if (a0 < 1e-36 * b0 && a1 < 1e-36 * b1) break;
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
