/*
 * Oracle (TEST INFRASTRUCTURE ONLY): pieces shared by the 3D Laplace and
 * Helmholtz restatements (header-only, static): the complex square root and
 * spherical coordinates of ztoolbox.f, the Legendre recurrences of
 * yrecursion.f (ylgndrini :694, zylgndrf :1220, zylgndr2sf :1330, and
 * myzylgndr2sf of ztoolbox.f:273-327) and the rotations of zrotate.f
 * (z3dzrot :1-27, z3dyrot :94-239; the FFT of length 2p+1 between ifftshift
 * and fftshift is a plain DFT here: the same sums).
 *
 * Expansions mp(n, m), 0 <= n <= p, -n <= m <= n, are stored row-major as
 * mp[n*(2p+1) + m + p].
 */
#ifndef ZFMM_O3DCOMMON_H
#define ZFMM_O3DCOMMON_H
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "ocommon.h"

#define F16 ((double)1e-16f) /* REAL*4 literal 1E-16 */
static const double PI = 3.14159265358979323846;
#define MPI(p, n, m) ((n) * (2 * (p) + 1) + (m) + (p))

/* zsqrt (ztoolbox.f:110-124): phase atan2 in (-pi, pi] with -pi mapped to pi */
static cplx zsqrt_r(cplx z2) {
  double r = sqrt(cabs(z2));
  double ph = atan2(cimag(z2), creal(z2));
  if (ph == -PI) ph = PI;
  ph = ph * 0.5;
  return r * cos(ph) + I * (r * sin(ph));
}

static void zcart2sph(const cplx *xyz, const cplx *c0, cplx *rz, cplx *ct, cplx *st, cplx *cp,
                      cplx *sp, cplx *eip) {
  cplx z1 = xyz[0] - c0[0], z2 = xyz[1] - c0[1], z3 = xyz[2] - c0[2];
  cplx r2 = z1 * z1 + z2 * z2 + z3 * z3;
  *rz = zsqrt_r(r2);
  *ct = z3 / *rz;
  cplx s2 = z1 * z1 + z2 * z2;
  *st = zsqrt_r(s2) / *rz;
  cplx zrxy = zsqrt_r(s2);
  if (cabs(zrxy) <= F16) {
    *cp = 1; *sp = 0; *eip = 1;
  } else {
    *cp = z1 / zrxy; *sp = z2 / zrxy; *eip = *cp + I * *sp;
  }
}

typedef struct { int n; double *r1, *r2; } rats;
static rats rats_new(int n) {
  rats R;
  R.n = n;
  R.r1 = (double *)calloc((size_t)(n + 1) * (n + 1), sizeof(double));
  R.r2 = (double *)calloc((size_t)(n + 1) * (n + 1), sizeof(double));
  /* ylgndrini: rat(n,m) at [n*(N+1)+m] */
  int N = n;
#define R1(a, b) R.r1[(a) * (N + 1) + (b)]
#define R2(a, b) R.r2[(a) * (N + 1) + (b)]
  R1(0, 0) = 1;
  R2(0, 0) = 1;
  for (int m = 0; m <= N; m++) {
    if (m > 0) { R1(m, m) = sqrt((2 * m - 1.0) / (2 * m)); R2(m, m) = 1; }
    if (m < N) { R1(m + 1, m) = sqrt(2 * m + 1.0); R2(m + 1, m) = 1; }
    for (int k = m + 2; k <= N; k++) {
      R1(k, m) = (2 * k - 1);
      R2(k, m) = sqrt((k + m - 1.0) * (k - m - 1.0));
      R1(k, m) = R1(k, m) / sqrt((double)(k - m) * (k + m));
      R2(k, m) = R2(k, m) / sqrt((double)(k - m) * (k + m));
    }
  }
  return R;
}
static void rats_free(rats *R) { free(R->r1); free(R->r2); }

/* Y(n,m) at y[n*(N+1)+m] */
static void zylgndrf(int N, cplx z, cplx *y, const rats *R) {
  cplx u = -zsqrt_r(1 - z * z);
  y[0] = 1;
  for (int m = 0; m <= N; m++) {
    if (m > 0) y[m * (N + 1) + m] = y[(m - 1) * (N + 1) + m - 1] * u * R->r1[m * (R->n + 1) + m];
    if (m < N) y[(m + 1) * (N + 1) + m] = z * y[m * (N + 1) + m] * R->r1[(m + 1) * (R->n + 1) + m];
    for (int n = m + 2; n <= N; n++)
      y[n * (N + 1) + m] = R->r1[n * (R->n + 1) + m] * z * y[(n - 1) * (N + 1) + m] -
                           R->r2[n * (R->n + 1) + m] * y[(n - 2) * (N + 1) + m];
  }
  for (int n = 0; n <= N; n++)
    for (int m = 0; m <= n; m++) y[n * (N + 1) + m] *= sqrt(2 * n + 1.0);
}

/* zylgndr2sf (mode 0) / myzylgndr2sf (mode 1, with stheta) */
static void zylgndr2s(int N, cplx z, cplx stheta, int mode, cplx *y, cplx *d, const rats *R) {
  cplx u;
  cplx u2 = 1 - z * z;
  if (mode == 0) {
    u = -zsqrt_r(u2);
  } else {
    if (cabs(u2) >= (double)1e-12f) u = -zsqrt_r(u2);
    else u = -stheta;
  }
  int L = R->n + 1;
#define Y(a, b) y[(a) * (N + 1) + (b)]
#define D(a, b) d[(a) * (N + 1) + (b)]
  Y(0, 0) = 1;
  D(0, 0) = 0;
  if (0 < N) {
    Y(1, 0) = z * Y(0, 0) * R->r1[1 * L + 0];
    D(1, 0) = (z * D(0, 0) + Y(0, 0)) * R->r1[1 * L + 0];
  }
  for (int n = 2; n <= N; n++) {
    Y(n, 0) = R->r1[n * L] * z * Y(n - 1, 0) - R->r2[n * L] * Y(n - 2, 0);
    D(n, 0) = R->r1[n * L] * (z * D(n - 1, 0) + Y(n - 1, 0)) - R->r2[n * L] * D(n - 2, 0);
  }
  for (int m = 1; m <= N; m++) {
    if (m == 1) Y(m, m) = Y(m - 1, m - 1) * (-1.0) * R->r1[m * L + m];
    else Y(m, m) = Y(m - 1, m - 1) * u * R->r1[m * L + m];
    D(m, m) = Y(m, m) * (double)(-m) * z;
    if (m < N) {
      Y(m + 1, m) = z * Y(m, m) * R->r1[(m + 1) * L + m];
      D(m + 1, m) = (z * D(m, m) + (1 - z * z) * Y(m, m)) * R->r1[(m + 1) * L + m];
    }
    for (int n = m + 2; n <= N; n++) {
      Y(n, m) = R->r1[n * L + m] * z * Y(n - 1, m) - R->r2[n * L + m] * Y(n - 2, m);
      D(n, m) = R->r1[n * L + m] * (z * D(n - 1, m) + (1 - z * z) * Y(n - 1, m)) -
                R->r2[n * L + m] * D(n - 2, m);
    }
  }
  for (int n = 0; n <= N; n++)
    for (int m = 0; m <= n; m++) {
      Y(n, m) *= sqrt(2 * n + 1.0);
      D(n, m) *= sqrt(2 * n + 1.0);
    }
#undef Y
#undef D
}

/* ---- rotations ---------------------------------------------------------- */
static void zrot(int p, const cplx *a, cplx *b, cplx cb, cplx sb) {
  cplx eb = cb + I * sb;
  cplx *E = (cplx *)malloc(sizeof(cplx) * (2 * p + 1)), *e = E + p;
  e[0] = 1;
  for (int m = 1; m <= p; m++) e[m] = e[m - 1] * eb;
  for (int m = 1; m <= p; m++) e[-m] = 1.0 / e[m];
  for (int n = 0; n <= p; n++)
    for (int m = -n; m <= n; m++) b[MPI(p, n, m)] = a[MPI(p, n, m)] * e[m];
  free(E);
}

static void yrot(int p, const cplx *a, cplx *b, cplx ca, cplx sa, const rats *R) {
  int N = p, NS = 2 * p + 1;
  double s4 = sqrt(4 * PI), s4i = 1.0 / s4;
  cplx *f = (cplx *)calloc((size_t)(N + 1) * NS, sizeof(cplx)); /* fdat+dfdat [n][j] */
  cplx *yls = (cplx *)calloc((size_t)(N + 1) * (N + 1), sizeof(cplx));
  cplx *dyls = (cplx *)calloc((size_t)(N + 1) * (N + 1), sizeof(cplx));
  cplx *E = (cplx *)malloc(sizeof(cplx) * (2 * N + 1)), *e = E + N;
  memset(b, 0, sizeof(cplx) * (size_t)(N + 1) * NS);
  for (int j = -N; j <= N; j++) {
    double ph = j * 2 * PI / (2 * N + 1);
    cplx x1 = cos(ph) * ca, x2 = sin(ph);
    cplx zrxy = zsqrt_r(x1 * x1 + x2 * x2);
    cplx ct = -cos(ph) * sa;
    cplx st = zsqrt_r(1 - (cos(ph) * cos(ph)) * (1 - ca * ca));
    if (ph == 0) st = (cabs(st + ca) <= cabs(st - ca)) ? -ca : ca;
    cplx cp, sp, eip;
    if (cabs(zrxy) >= F16) { cp = x1 / zrxy; sp = x2 / zrxy; eip = cp + I * sp; }
    else { cp = 1; sp = 0; eip = 1; }
    e[0] = 1;
    for (int m = 1; m <= N; m++) e[m] = e[m - 1] * eip;
    for (int m = 1; m <= N; m++) e[-m] = 1.0 / e[m];
    zylgndr2s(N, ct, st, 1, yls, dyls, R);
    cplx z1 = s4i * st, z2 = (st * ca - ct * cp * sa) * s4i, z3 = sp * sa * s4i * I;
    for (int n = 0; n <= N; n++) {
      cplx fd = a[MPI(p, n, 0)] * yls[n * (N + 1)] * s4i;
      cplx dfd = -a[MPI(p, n, 0)] * dyls[n * (N + 1)] * z2 * st;
      for (int m = 1; m <= n; m++) {
        cplx z4 = a[MPI(p, n, m)] * e[m], z5 = a[MPI(p, n, -m)] * e[-m], z6 = z4 + z5;
        double sg = (m & 1) ? -1.0 : 1.0;
        fd += z1 * z6 * sg * yls[n * (N + 1) + m];
        dfd += sg * (-dyls[n * (N + 1) + m] * z2 * z6 + yls[n * (N + 1) + m] * z3 * (double)m * z4 -
                     yls[n * (N + 1) + m] * z3 * (double)m * z5);
      }
      f[n * NS + (j + N)] = fd + dfd;
    }
  }
  zylgndr2s(N, 0, 0, 0, yls, dyls, R);
  double factor = s4 / (2 * N + 1);
  for (int n = 0; n <= N; n++) {
    for (int m = -n; m <= n; m++) {
      cplx c = 0;
      for (int j = -N; j <= N; j++) {
        double ang = -(double)m * j * 2 * PI / (2 * N + 1);
        c += f[n * NS + (j + N)] * (cos(ang) + I * sin(ang));
      }
      int am = m < 0 ? -m : m;
      if (m == 0) {
        b[MPI(p, n, 0)] = c / (yls[n * (N + 1)] - dyls[n * (N + 1)]) * factor;
      } else {
        double sg = (am & 1) ? -1.0 : 1.0;
        cplx zz = sg * (yls[n * (N + 1) + am] - dyls[n * (N + 1) + am]) / factor;
        b[MPI(p, n, m)] = c / zz;
      }
    }
  }
  free(f); free(yls); free(dyls); free(E);
}


#endif
