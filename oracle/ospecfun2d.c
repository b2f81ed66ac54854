/*
 * Oracle (TEST INFRASTRUCTURE ONLY): Bessel/Hankel functions of complex
 * argument for the 2D Helmholtz oracle.
 *
 * The reference evaluates H0, H1 with Rokhlin's piecewise approximations
 * (zfmm2d/src/helmholtz/hank103.f:131-1015, hank101.f:18-977), whose
 * coefficient tables are not restated here.  The oracle computes the same
 * functions on the same (principal) branch from the mathematics instead:
 * ascending series for |z| < 2, Hankel's Laplace-type integral by the
 * trapezoidal rule (32 nodes, step 0.2) in the closed upper
 * half-plane, and Miller's algorithm with Neumann series below the real axis
 * (reflection z -> -conj z on the left).  Values are pinned against 160-digit
 * mpmath in tests/test_hankel.py.  A zero imaginary part counts as +0, as in
 * hank103 ("rea(2) .lt. 0" selects the lower half-plane).
 *
 * jbessel2d (cdjseval2d.f:23-221) and h2dall (h2dcommon.f:71-173) follow the
 * reference's recurrences (Miller backward recurrence with the e^{-+iz}
 * normalisation, forward recurrence for H_n).
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "oracle.h"

typedef double complex lcplx;
static const double LPI = 3.141592653589793238462643383279503;
static const double LEULER = 0.577215664901532860606512090082402;
static const double LLN2 = 0.693147180559945309417232121458177;

static void series01(lcplx z, lcplx *J0, lcplx *J1, lcplx *S0, lcplx *S1) {
  lcplx q = z * z / 4, t0 = 1, t1 = 1, sj0 = 1, sj1 = 1, s0 = 0, s1 = 1;
  double H = 0;
  for (int k = 1; k < 60; k++) {
    t0 = -q * t0 / ((double)k * k);
    t1 = -q * t1 / ((double)k * (k + 1));
    H += 1.0 / k;
    sj0 += t0;
    sj1 += t1;
    s0 += H * t0;
    s1 += (2 * H + 1.0 / (k + 1)) * t1;
    if (cabs(t0) < 1e-18 * cabs(sj0) && cabs(t1) < 1e-18 * cabs(sj1)) break;
  }
  double c = 2 / LPI * (LEULER - LLN2);
  *J0 = sj0;
  *J1 = z / 2 * sj1;
  *S0 = c * *J0 - 2 / LPI * s0;
  *S1 = c * *J1 - 2 / (LPI * z) - 1 / LPI * (z / 2) * s1;
}

static void miller01(lcplx w, lcplx *J0, lcplx *J1, lcplx *S0, lcplx *S1) {
  double aw = cabs(w);
  int N = (int)(aw + 30 + 3 * cbrt(aw));
  N += N & 1;
  lcplx fbuf[512];
  lcplx *f = N + 2 <= 512 ? fbuf : (lcplx *)malloc((N + 2) * sizeof(lcplx));
  memset(f, 0, (N + 2) * sizeof(lcplx));
  f[N] = 1e-30;
  for (int n = N; n >= 1; n--) {
    f[n - 1] = (2.0 * n / w) * f[n] - f[n + 1];
    if (cabs(f[n - 1]) > 1e300)
      for (int k = n - 1; k <= N; k++) f[k] *= 1e-300;
  }
  lcplx norm = f[0];
  lcplx ipow = 1;
  for (int n = 1; n <= N; n++) {
    ipow *= I;
    norm += 2 * ipow * f[n];
  }
  lcplx sc = cexp(I * w) / norm;
  lcplx a0 = 0, a1 = 0;
  for (int k = 1; 2 * k + 1 <= N; k++) {
    double sg = (k & 1) ? -1.0 : 1.0;
    a0 += sg * f[2 * k] / k;
    a1 += sg * (f[2 * k - 1] - f[2 * k + 1]) / k;
  }
  double c = 2 / LPI * (LEULER - LLN2);
  *J0 = sc * f[0];
  *J1 = sc * f[1];
  *S0 = c * *J0 - 4 / LPI * sc * a0;
  *S1 = c * *J1 - 2 / (LPI * w) * *J0 + 2 / LPI * sc * a1;
  if (f != fbuf) free(f);
}

static void integral01(lcplx z, lcplx *h0, lcplx *h1) {
  const int nn = 32;
  const double hs = 0.2;
  lcplx c = I / (2 * z), f0 = 0, f1 = 0;
  for (int k = 0; k < nn; k++) {
    double s = hs * k, s2 = s * s;
    double w = hs * exp(-s2) * (k == 0 ? 0.5 : 1.0);
    lcplx r = csqrt(1 + s2 * c);
    f0 += w / r;
    f1 += w * s2 * r;
  }
  lcplx pre = sqrt(2 / LPI) / csqrt(z) * cexp(I * z);
  *h0 = pre * cexp(-I * LPI / 4) * 2 / sqrt(LPI) * f0;
  *h1 = pre * cexp(-I * 3 * LPI / 4) * 4 / sqrt(LPI) * f1;
}

void o_hank103(double zr, double zi, double *h0, double *h1) {
  if (zi == 0.0) zi = 0.0;
  lcplx z = (double)zr + I * (double)zi;
  lcplx J0, J1, S0, S1, H0, H1;
  double az = cabs(z);
  if (az < 2) {
    series01(z, &J0, &J1, &S0, &S1);
  } else if (zi >= 0) {
    integral01(z, &H0, &H1);
    h0[0] = creal(H0); h0[1] = cimag(H0);
    h1[0] = creal(H1); h1[1] = cimag(H1);
    return;
  } else if (zr >= 0) {
    miller01(z, &J0, &J1, &S0, &S1);
  } else {
    lcplx w = -conj(z);
    miller01(w, &J0, &J1, &S0, &S1);
    J0 = conj(J0); J1 = -conj(J1); S0 = conj(S0); S1 = -conj(S1);
  }
  lcplx L = 2 / LPI * clog(z);
  H0 = J0 + I * (L * J0 + S0);
  H1 = J1 + I * (L * J1 + S1);
  h0[0] = creal(H0); h0[1] = cimag(H0);
  h1[0] = creal(H1); h1[1] = cimag(H1);
}

void o_h2dall(int nterms, double zr, double zi, double rscale, double *hvec_, int ifder,
              double *hder_) {
  double complex *hvec = (double complex *)hvec_, *hder = (double complex *)hder_;
  double complex z = zr + I * zi;
  if (cabs(z) < 1e-200) {
    for (int i = 0; i <= nterms; i++) {
      hvec[i] = 0;
      if (ifder == 1) hder[i] = 0;
    }
    return;
  }
  double a[2], b[2];
  o_hank103(zr, zi, a, b);
  hvec[0] = a[0] + I * a[1];
  hvec[1] = (b[0] + I * b[1]) * rscale;
  double scal2 = rscale * rscale;
  double complex zinv = rscale / z;
  for (int i = 1; i <= nterms - 1; i++) hvec[i + 1] = (zinv * (2.0 * i)) * hvec[i] - scal2 * hvec[i - 1];
  if (ifder == 1) {
    hder[0] = -hvec[1] / rscale;
    zinv = 1.0 / z;
    for (int i = 1; i <= nterms; i++) hder[i] = rscale * hvec[i - 1] - (zinv * (double)i) * hvec[i];
  }
}

/* jbessel2d: fjs(n) = J_n(z)/rscale^n, n = 0..nterms (fjs needs nterms+2) */
void o_jbessel2d(int nterms, double zr, double zi, double rscale, double *fjs_, int ifder,
                 double *fjder_) {
  double complex *fjs = (double complex *)fjs_, *fjder = (double complex *)fjder_;
  double complex z = zr + I * zi;
  if (cabs(z) < 1e-200) {
    fjs[0] = 1;
    for (int i = 1; i <= nterms + 1; i++) fjs[i] = 0;
    if (ifder == 1) {
      for (int i = 0; i <= nterms; i++) fjder[i] = 0;
      fjder[1] = 1.0 / (2 * rscale);
    }
    return;
  }
  double complex zinv = 1.0 / z, ffn = 1, ffnm1 = 0;
  int ntop = nterms + 100000;
  for (int i = nterms; i <= nterms + 100000; i++) {
    double complex t = (2.0 * i) * zinv * ffn - ffnm1;
    double dd = creal(t) * creal(t) + cimag(t) * cimag(t);
    if (dd > 1e40) {
      ntop = i + 1;
      break;
    }
    ffnm1 = ffn;
    ffn = t;
  }
  /* backward recurrence in double on unscaled J; on overflow the two
     newest values are scaled down and the event is recorded, and the values
     above are brought to the same scale in one upward pass */
  lcplx *f = (lcplx *)calloc(ntop + 2, sizeof(lcplx));
  char *mark = (char *)calloc(ntop + 2, 1);
  lcplx lz = (double)zr + I * (double)zi;
  f[ntop] = 0;
  f[ntop - 1] = 1;
  for (int n = ntop - 1; n >= 1; n--) {
    f[n - 1] = (2.0 * n / lz) * f[n] - f[n + 1];
    if (cabs(f[n - 1]) > 1e300) {
      f[n - 1] *= 1e-300;
      f[n] *= 1e-300;
      mark[n] = 1;
    }
  }
  {
    double sct = 1;
    for (int i = 1; i <= ntop; i++) {
      if (mark[i - 1]) sct *= 1e-300;
      f[i] *= sct;
    }
  }
  free(mark);
  lcplx zm = zi < 0 ? I : -I, p = 1, psi = f[0];
  for (int n = 1; n <= ntop; n++) {
    p *= zm;
    psi += 2 * p * f[n];
  }
  lcplx sc = (zi < 0 ? cexp(I * lz) : cexp(-I * lz)) / psi;
  double rs = 1;
  for (int n = 0; n <= nterms + 1 && n <= ntop; n++) {
    fjs[n] = (double complex)(sc * f[n] / rs);
    rs *= rscale;
  }
  free(f);
  if (ifder == 1) {
    fjder[0] = -fjs[1] * rscale;
    double dc1 = 0.5 / rscale, dc2 = 0.5 * rscale;
    for (int i = 1; i <= nterms; i++) fjder[i] = dc1 * fjs[i - 1] - dc2 * fjs[i + 1];
  }
}

/* h2dterms (zfmm2d/src/helmholtz/h2dterms.f:35-97) */
int o_h2dterms(double bsize, double zkr, double zki, double eps, int isep) {
  const int ntmax = 50000;
  double complex zk = zkr + I * zki;
  double complex z1 = (zk * bsize) * (0.5 + isep * 1.0);
  double rscale = 1.0;
  double pi2 = 8 * atan(1.0);
  if (cabs(zk * bsize) < pi2) rscale = cabs(zk * bsize);
  double complex *hfun = (double complex *)malloc(sizeof(double complex) * (ntmax + 102));
  double complex *jfun = (double complex *)malloc(sizeof(double complex) * (ntmax + 102));
  o_h2dall(ntmax, creal(z1), cimag(z1), rscale, (double *)hfun, 0, NULL);
  double complex z2 = (zk * bsize) * sqrt(2.0) / 2.0;
  o_jbessel2d(ntmax, creal(z2), cimag(z2), rscale, (double *)jfun, 0, NULL);
  double xtemp0 = cabs(jfun[0] * hfun[0]) + cabs(jfun[1] * hfun[1]);
  int nterms = 10001;
  for (int j = 2; j <= ntmax; j++) {
    double xtemp = (cabs(jfun[j] * hfun[j]) + cabs(jfun[j - 1] * hfun[j - 1])) * cabs(hfun[0]);
    if (xtemp < eps * xtemp0) {
      nterms = j + 1;
      break;
    }
  }
  free(hfun);
  free(jfun);
  return nterms;
}
