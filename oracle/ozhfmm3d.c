/*
 * Oracle (TEST INFRASTRUCTURE ONLY): 3D Helmholtz complex-coordinate FMM.
 *
 * Restates zfmm3d/src/helmholtz/zhfmm3d.f (driver :1-249 with the rescaling by
 * 1/boxsize(0) and zk*boxsize(0), zhfmm3dmain :256-600, zh3devaldirect
 * :626-693, zh3dformmp :699-851, zh3dformloc :857-1009, zh3devalmp
 * :1015-1158, zh3devalloc :1164-1309), the translations of
 * zfmm3d/src/helmholtz/zh3dtrans.f (zh3dmploc :1-98, zh3dmpmp :105-200,
 * zh3dlocloc :207-312, and the quadrature z-shifts :319-780), the special
 * functions of h3dcommon.f (h3d01 :16-55, h3dall :59-140), besseljs3d.f:5-169,
 * h3dterms.f:16-75, hndiv_fast.f:1-37, zylgndr of yrecursion.f:1009-1060, and
 * the 3D pieces shared with the Laplace oracle (o3dcommon.h).
 *
 * The Gauss-Legendre rule of the z-shifts (legeexps with itype = 1) is
 * generated here by Newton's method on P_n: the same nodes and weights to
 * rounding.  The reference leaves n0 (zhfmm3d.f:223) uninitialised; it is 0
 * here.  Expansions of level l have order nterms(l) and are stored as in
 * o3dcommon.h with p = nterms(l).
 */
#include <stdio.h>
#include "o3dcommon.h"

static int o_hndiv3d(double eps, int ns, int nt) {
  /* hndiv_fast.f:16-34 (idivflag = 0) */
  if (eps >= 0.5e-3) return 300;
  if (eps >= 0.5e-15) return 1000;
  return ns + nt;
}

/* h3d01 (h3dcommon.f:16-55) */
static void h3d01(cplx z, cplx *h0, cplx *h1) {
  if (cabs(z) < 1.0e-15) { *h0 = 0; *h1 = 0; return; }
  cplx cd = I * z;
  *h0 = cexp(cd) / cd;
  *h1 = *h0 * (1.0 / z - I);
}

/* h3dall (h3dcommon.f:59-140): hvec(n) = h_n(z) scale^n; arrays of nterms+2 */
static void h3dall(int nterms, cplx z, double scale, cplx *hvec, int ifder, cplx *hder) {
  if (cabs(z) < 1.0e-15) {
    for (int i = 0; i <= nterms; i++) {
      hvec[i] = 0;
      if (hder) hder[i] = 0;
    }
    return;
  }
  h3d01(z, &hvec[0], &hvec[1]);
  hvec[1] = hvec[1] * scale;
  double scal2 = scale * scale;
  cplx zinv = scale / z;
  for (int i = 1; i <= nterms - 1; i++) {
    double dtmp = 2 * i + 1.0;
    cplx ztmp = zinv * dtmp;
    hvec[i + 1] = ztmp * hvec[i] - scal2 * hvec[i - 1];
  }
  if (ifder == 1) {
    hder[0] = -hvec[1] / scale;
    zinv = 1.0 / z;
    for (int i = 1; i <= nterms; i++) {
      double dtmp = i + 1.0;
      cplx ztmp = zinv * dtmp;
      hder[i] = scale * hvec[i - 1] - ztmp * hvec[i];
    }
  }
}

/* besseljs3d (besseljs3d.f:5-169): fjs(n) = j_n(z) / scale^n, fjs[0..nterms] */
static void besseljs3d(int nterms, cplx z, double scale, cplx *fjs, int ifder, cplx *fjder) {
  const double upbound2 = 1.0e40, upbound2inv = 1.0e-40, tiny = 1.0e-200;
  if (cabs(z) < tiny) {
    fjs[0] = 1;
    for (int i = 1; i <= nterms; i++) fjs[i] = 0;
    if (ifder == 1) {
      for (int i = 0; i <= nterms; i++) fjder[i] = 0;
      if (nterms >= 1) fjder[1] = 1.0 / (3 * scale);
    }
    return;
  }
  cplx zinv = 1.0 / z;
  cplx fjm1 = 0, fj0 = 1, fj1;
  int lwfjs = nterms + 100000, ntop = lwfjs;
  for (int i = nterms; i <= lwfjs; i++) {
    double dcoef = 2 * i + 1.0;
    fj1 = dcoef * zinv * fj0 - fjm1;
    double a = cabs(fj1), dd = a * a;
    if (dd > upbound2) { ntop = i + 1; break; }
    fjm1 = fj0;
    fj0 = fj1;
  }
  int *iscale = (int *)calloc((size_t)ntop + 1, sizeof(int));
  cplx *fjtmp = (cplx *)calloc((size_t)ntop + 1, sizeof(cplx));
  fjtmp[ntop] = 0;
  fjtmp[ntop - 1] = 1;
  for (int i = ntop - 1; i >= 1; i--) {
    double dcoef = 2 * i + 1.0;
    fjtmp[i - 1] = dcoef * zinv * fjtmp[i] - fjtmp[i + 1];
    double a = cabs(fjtmp[i - 1]), dd = a * a;
    if (dd > upbound2) {
      fjtmp[i] = fjtmp[i] * upbound2inv;
      fjtmp[i - 1] = fjtmp[i - 1] * upbound2inv;
      iscale[i] = 1;
    }
  }
  double scalinv = 1.0 / scale, sctot = 1.0;
  for (int i = 1; i <= ntop; i++) {
    sctot = sctot * scalinv;
    if (iscale[i - 1] == 1) sctot = sctot * upbound2inv;
    fjtmp[i] = fjtmp[i] * sctot;
  }
  fj0 = csin(z) * zinv;
  fj1 = fj0 * zinv - ccos(z) * zinv;
  double d0 = cabs(fj0), d1 = cabs(fj1);
  cplx zscale = (d1 > d0) ? fj1 / (fjtmp[1] * scale) : fj0 / fjtmp[0];
  for (int i = 0; i <= nterms; i++) fjs[i] = fjtmp[i] * zscale;
  if (ifder == 1) {
    fjder[0] = -fjs[1] * scale;
    for (int i = 1; i <= nterms; i++) {
      double dc1 = i / (2 * i + 1.0), dc2 = 1.0 - dc1;
      dc1 = dc1 * scalinv;
      dc2 = dc2 * scale;
      fjder[i] = (dc1 * fjtmp[i - 1] - dc2 * fjtmp[i + 1]) * zscale;
    }
  }
  free(iscale);
  free(fjtmp);
}

/* h3dterms (h3dterms.f:16-75) */
int o_h3dterms(double size, double zkr, double zki, double eps, int isep) {
  cplx zk = zkr + I * zki;
  enum { NT = 5000 };
  cplx *hfun = (cplx *)malloc(sizeof(cplx) * (NT + 2));
  cplx *jfun = (cplx *)malloc(sizeof(cplx) * (NT + 2));
  cplx z1 = (zk * size) * (0.5 + isep * 1.0);
  double rscale = 1.0;
  if (cabs(zk * size) < 1.0) rscale = cabs(zk * size);
  h3dall(NT, z1, rscale, hfun, 0, NULL);
  cplx z2 = (zk * size) * sqrt(3.0) / 2.0;
  besseljs3d(NT, z2, rscale, jfun, 0, NULL);
  double xtemp0 = cabs(jfun[0] * hfun[0]) + cabs(jfun[1] * hfun[1]);
  int nterms = 5000;
  for (int j = 2; j <= NT; j++) {
    double xtemp = (cabs(jfun[j] * hfun[j]) + cabs(jfun[j - 1] * hfun[j - 1])) * cabs(hfun[0]) *
                   cabs(zk);
    if (xtemp < eps * xtemp0) { nterms = j + 1; break; }
  }
  free(hfun);
  free(jfun);
  return nterms;
}

/* zylgndr (yrecursion.f:1009-1060): coefficients evaluated inline */
static void zylgndr_plain(int N, cplx z, cplx *y) {
  cplx u = -zsqrt_r(1 - z * z);
#define YP(a, b) y[(a) * (N + 1) + (b)]
  YP(0, 0) = 1;
  for (int m = 0; m <= N; m++) {
    if (m > 0) YP(m, m) = YP(m - 1, m - 1) * u * sqrt((2 * m - 1.0) / (2 * m));
    if (m < N) YP(m + 1, m) = z * YP(m, m) * sqrt(2 * m + 1.0);
    for (int n = m + 2; n <= N; n++)
      YP(n, m) = ((double)(2 * n - 1) * z * YP(n - 1, m) -
                  sqrt((n + m - 1.0) * (n - m - 1.0)) * YP(n - 2, m)) /
                 sqrt((n - m + 0.0) * (n + m));
  }
  for (int n = 0; n <= N; n++)
    for (int m = 0; m <= n; m++) YP(n, m) *= sqrt(2 * n + 1.0);
#undef YP
}

/* Gauss-Legendre nodes (ascending) and weights on [-1, 1] */
static void gauss_legendre(int n, double *x, double *w) {
  for (int i = 0; i < n; i++) {
    double t = cos(PI * (i + 0.75) / (n + 0.5)), dp = 1.0;
    for (int it = 0; it < 100; it++) {
      double p0 = 1.0, p1 = t;
      for (int k = 2; k <= n; k++) {
        double p2 = ((2 * k - 1) * t * p1 - (k - 1) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      if (n == 1) p0 = 1.0;
      dp = n * (t * p1 - p0) / (t * t - 1.0);
      double dt = p1 / dp;
      t -= dt;
      if (fabs(dt) < 1e-16) break;
    }
    {
      double p0 = 1.0, p1 = t;
      for (int k = 2; k <= n; k++) {
        double p2 = ((2 * k - 1) * t * p1 - (k - 1) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      dp = n * (t * p1 - p0) / (t * t - 1.0);
    }
    x[n - 1 - i] = t;
    w[n - 1 - i] = 2.0 / ((1.0 - t * t) * dp * dp);
  }
}

void o_gauss_legendre(int n, double *x, double *w) { gauss_legendre(n, x, w); }

/* ---- direct sum --------------------------------------------------------- */
void o_zh3devaldirect(const double *zk_, int nt, const double *ztarg, int ns, const double *zsrc,
                      const double *charge, const double *dipstr, const double *dipvec,
                      int ifcharge, double *pot, double *grad, int ifdipole, int ifpgh) {
  cplx zk = zk_[0] + I * zk_[1];
  const cplx *zt = (const cplx *)ztarg, *zs = (const cplx *)zsrc;
  const cplx *q = (const cplx *)charge, *ds = (const cplx *)dipstr, *dv = (const cplx *)dipvec;
  cplx *P_ = (cplx *)pot, *G_ = (cplx *)grad;
  double pi4 = 4 * PI;
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < nt; i++) {
    cplx p = 0, g[3] = {0, 0, 0};
    for (int j = 0; j < ns; j++) {
      cplx x[3];
      for (int d = 0; d < 3; d++) x[d] = zt[3 * i + d] - zs[3 * j + d];
      cplx rz = csqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
      cplx z = I * zk * rz;
      if (!(cabs(rz) > F16)) continue;
      if (ifcharge == 1) {
        cplx h0 = cexp(z) / (pi4 * rz);
        p += q[j] * h0;
        if (ifpgh >= 2) {
          cplx r3 = 1.0 / (pi4 * (rz * rz * rz));
          cplx h1 = cexp(z) * (1.0 - z) * r3;
          for (int d = 0; d < 3; d++) g[d] += q[j] * (-x[d]) * h1;
        }
      }
      if (ifdipole == 1) {
        cplx dot = x[0] * dv[3 * j] + x[1] * dv[3 * j + 1] + x[2] * dv[3 * j + 2];
        cplx t3 = cexp(z), t4 = 1.0 - z;
        cplx r3 = 1.0 / (pi4 * (rz * rz * rz));
        p -= ds[j] * t3 * dot * t4 * r3;
        if (ifpgh >= 2) {
          cplx t1 = dot * t3 * r3;
          t1 = t1 * (zk * zk - 3.0 * t4 / (rz * rz));
          cplx t2 = t4 * t3 * r3;
          for (int d = 0; d < 3; d++) g[d] -= ds[j] * (dv[3 * j + d] * t2 + x[d] * t1);
        }
      }
    }
    P_[i] += p;
    if (ifpgh >= 2)
      for (int d = 0; d < 3; d++) G_[3 * i + d] += g[d];
  }
}

/* ---- form / eval ---------------------------------------------------------- */
/* zh3dformmp (local = 0) / zh3dformloc (local = 1) */
static void hform3(cplx zk, double rscale, const cplx *zs, int npts, const cplx *q, const cplx *ds,
                   const cplx *dv, const cplx *zc, int p, cplx *mp, int ifcharge, int ifdipole,
                   int local, const rats *R) {
  int N = p;
  cplx *yl = (cplx *)calloc((size_t)(N + 1) * (N + 1), sizeof(cplx));
  cplx *dyl = (cplx *)calloc((size_t)(N + 1) * (N + 1), sizeof(cplx));
  cplx *f = (cplx *)calloc((size_t)N + 3, sizeof(cplx)), *fd = (cplx *)calloc((size_t)N + 3, sizeof(cplx));
  cplx *eia = (cplx *)malloc(sizeof(cplx) * (2 * N + 1)), *E = eia + N;
  cplx c4 = (1.0 / (4 * PI)) * I * zk;
  for (int i = 0; i < npts; i++) {
    cplx zr, ct, st, cp, sp, eip;
    zcart2sph(&zs[3 * i], zc, &zr, &ct, &st, &cp, &sp, &eip);
    E[0] = 1;
    for (int m = 1; m <= N; m++) E[m] = E[m - 1] * eip;
    for (int m = 1; m <= N; m++) E[-m] = 1.0 / E[m];
    cplx dzr_ = 0, dth_ = 0, dph_ = 0;
    if (ifdipole == 1) {
      cplx ezr[3] = {st * cp, st * sp, ct}, eth[3] = {ct * cp, ct * sp, -st}, eph[3] = {-sp, cp, 0};
      for (int d = 0; d < 3; d++) {
        dzr_ += dv[3 * i + d] * ezr[d];
        dth_ += dv[3 * i + d] * eth[d];
        dph_ += dv[3 * i + d] * eph[d];
      }
    }
    cplx zrk = zr * zk;
    if (!local) besseljs3d(N, zrk, rscale, f, ifdipole, fd);
    else h3dall(N, zrk, rscale, f, ifdipole, fd);
    if (ifdipole == 0) {
      if (!local) zylgndr_plain(N, ct, yl);
      else zylgndrf(N, ct, yl, R);
    } else {
      zylgndr2s(N, ct, 0, 0, yl, dyl, R);
    }
    for (int n = 0; n <= N; n++)
      for (int m = 0; m <= n; m++) {
        double sg = (m & 1) ? -1.0 : 1.0;
        yl[n * (N + 1) + m] = yl[n * (N + 1) + m] * c4 * sg;
        if (ifdipole == 1) dyl[n * (N + 1) + m] = dyl[n * (N + 1) + m] * c4 * sg;
      }
    if (ifcharge == 1) {
      for (int n = 0; n <= N; n++) {
        mp[MPI(p, n, 0)] += q[i] * f[n] * yl[n * (N + 1)];
        for (int m = 1; m <= n; m++) {
          cplx z1 = q[i] * f[n] * yl[n * (N + 1) + m];
          if (ifdipole == 1) z1 = z1 * st;
          mp[MPI(p, n, m)] += z1 * E[-m];
          mp[MPI(p, n, -m)] += z1 * E[m];
        }
      }
    }
    if (ifdipole == 1) {
      cplx dthz = dth_ / zr, dphz = dph_ / zr;
      for (int n = 0; n <= N; n++) {
        mp[MPI(p, n, 0)] -= ds[i] * zk * fd[n] * yl[n * (N + 1)] * dzr_;
        mp[MPI(p, n, 0)] += ds[i] * f[n] * dyl[n * (N + 1)] * st * dthz;
        for (int m = 1; m <= n; m++) {
          cplx y = yl[n * (N + 1) + m], dy = dyl[n * (N + 1) + m];
          cplx z1 = ds[i] * zk * fd[n] * y * st * dzr_;
          mp[MPI(p, n, m)] -= z1 * E[-m];
          mp[MPI(p, n, -m)] -= z1 * E[m];
          z1 = ds[i] * f[n] * dy * dthz;
          mp[MPI(p, n, m)] += z1 * E[-m];
          mp[MPI(p, n, -m)] += z1 * E[m];
          z1 = ds[i] * (double)m * I * f[n] * y * dphz;
          mp[MPI(p, n, m)] += z1 * E[-m];
          mp[MPI(p, n, -m)] -= z1 * E[m];
        }
      }
    }
  }
  free(yl); free(dyl); free(f); free(fd); free(eia);
}

/* zh3devalmp (local = 0) / zh3devalloc (local = 1) */
static void heval3(cplx zk, int nt, const cplx *zt, double rscale, int p, const cplx *zc,
                   const cplx *mp, cplx *pot, cplx *grad, int ifpgh, int local, const rats *R) {
  int N = p;
  cplx *yl = (cplx *)calloc((size_t)(N + 1) * (N + 1), sizeof(cplx));
  cplx *dyl = (cplx *)calloc((size_t)(N + 1) * (N + 1), sizeof(cplx));
  cplx *f = (cplx *)calloc((size_t)N + 3, sizeof(cplx)), *fd = (cplx *)calloc((size_t)N + 3, sizeof(cplx));
  cplx *eia = (cplx *)malloc(sizeof(cplx) * (2 * N + 1)), *E = eia + N;
  int ifder = ifpgh >= 2;
  for (int i = 0; i < nt; i++) {
    cplx zr, ct, st, cp, sp, eip;
    zcart2sph(&zt[3 * i], zc, &zr, &ct, &st, &cp, &sp, &eip);
    E[0] = 1;
    for (int m = 1; m <= N; m++) E[m] = E[m - 1] * eip;
    for (int m = 1; m <= N; m++) E[-m] = 1.0 / E[m];
    cplx ezr[3] = {0, 0, 0}, ethz[3] = {0, 0, 0}, ephz[3] = {0, 0, 0};
    if (ifpgh == 2) {
      ezr[0] = st * cp; ezr[1] = st * sp; ezr[2] = ct;
      ethz[0] = ct * cp / zr; ethz[1] = ct * sp / zr; ethz[2] = -st / zr;
      ephz[0] = -sp / zr; ephz[1] = cp / zr; ephz[2] = 0.0 / zr;
    }
    cplx zrk = zr * zk;
    if (!local) h3dall(N, zrk, rscale, f, ifder, fd);
    else besseljs3d(N, zrk, rscale, f, ifder, fd);
    if (ifpgh == 1) zylgndrf(N, ct, yl, R);
    else zylgndr2s(N, ct, 0, 0, yl, dyl, R);
    for (int n = 0; n <= N; n++)
      for (int m = 0; m <= n; m++) {
        double sg = (m & 1) ? -1.0 : 1.0;
        yl[n * (N + 1) + m] *= sg;
        if (ifpgh >= 2) dyl[n * (N + 1) + m] *= sg;
      }
    for (int n = 0; n <= N; n++) {
      pot[i] += mp[MPI(p, n, 0)] * f[n] * yl[n * (N + 1)];
      for (int m = 1; m <= n; m++) {
        cplx z1 = f[n] * yl[n * (N + 1) + m];
        if (ifpgh != 1) z1 = z1 * st;
        pot[i] += z1 * (mp[MPI(p, n, m)] * E[m] + mp[MPI(p, n, -m)] * E[-m]);
      }
    }
    if (ifpgh >= 2) {
      for (int n = 0; n <= N; n++) {
        cplx a0 = mp[MPI(p, n, 0)];
        for (int d = 0; d < 3; d++)
          grad[3 * i + d] += a0 * (zk * fd[n] * yl[n * (N + 1)] * ezr[d] -
                                   f[n] * dyl[n * (N + 1)] * st * ethz[d]);
        for (int m = 1; m <= n; m++) {
          cplx z1 = mp[MPI(p, n, m)] * E[m], z2 = mp[MPI(p, n, -m)] * E[-m];
          cplx y = yl[n * (N + 1) + m], dy = dyl[n * (N + 1) + m];
          for (int d = 0; d < 3; d++) {
            grad[3 * i + d] += zk * fd[n] * y * st * ezr[d] * (z1 + z2);
            grad[3 * i + d] -= f[n] * dy * ethz[d] * (z1 + z2);
            grad[3 * i + d] += (double)m * I * f[n] * y * ephz[d] * (z1 - z2);
          }
        }
      }
    }
  }
  free(yl); free(dyl); free(f); free(fd); free(eia);
}

/* ---- quadrature z-shifts (zh3dtrans.f:319-780) ------------------------------
 * kind 0 mpmp (evaluate with h, project with h), 1 mploc (h, then j),
 * 2 locloc (j, then j).  a1 has order p1, a2 (overwritten) order p2. */
static void hzshift(int kind, double r, int nquad, cplx zshift, int p1, int p2, double rs1,
                    double rs2, cplx kwave, const cplx *a1, cplx *a2, const rats *R) {
  int nterm = p1 > p2 ? p1 : p2, W = 2 * nterm + 1;
  int ne = kind == 0 ? nterm : p1;  /* order of the evaluation Legendre / radial tables */
  double *x = (double *)malloc(sizeof(double) * nquad), *w = (double *)malloc(sizeof(double) * nquad);
  gauss_legendre(nquad, x, w);
  cplx *fdat = (cplx *)calloc((size_t)nquad * W, sizeof(cplx));
  cplx *dfdat = (cplx *)calloc((size_t)nquad * W, sizeof(cplx));
  cplx *yls = (cplx *)calloc((size_t)(nterm + 1) * (nterm + 1), sizeof(cplx));
  cplx *dyls = (cplx *)calloc((size_t)(nterm + 1) * (nterm + 1), sizeof(cplx));
  cplx *f = (cplx *)calloc((size_t)nterm + 3, sizeof(cplx)), *fd = (cplx *)calloc((size_t)nterm + 3, sizeof(cplx));
  double s4i = 1.0 / sqrt(4 * PI), pi2i = 1.0 / (2 * PI);
  for (int i = 0; i < nquad; i++) {
    double yi = sqrt(1 - x[i] * x[i]);
    cplx zi = zshift + r * x[i];
    cplx ri2 = (r * yi) * (r * yi) + zi * zi;
    cplx ri = zsqrt_r(ri2);
    cplx cthi = zi / ri;
    cplx sthi = zsqrt_r(1 - cthi * cthi);
    cplx cthi_ri = cthi / ri, sthi_ri = sthi / ri;
    cplx zk = ri * kwave;
    int L = ne + 1;
    zylgndr2s(ne, cthi, 0, 0, yls, dyls, R);
    for (int n = 0; n <= p1; n++)
      for (int m = 0; m <= n; m++) {
        double sg = (m & 1) ? -1.0 : 1.0;
        yls[n * L + m] = yls[n * L + m] * sg * s4i;
        dyls[n * L + m] = dyls[n * L + m] * sg * s4i;
      }
    if (kind == 2) besseljs3d(p1, zk, rs1, f, 1, fd);
    else h3dall(ne, zk, rs1, f, 1, fd);
    for (int n = 0; n <= ne; n++) fd[n] = kwave * fd[n];
    cplx *F = fdat + (size_t)i * W + nterm, *DF = dfdat + (size_t)i * W + nterm;
    for (int n = 0; n <= p1; n++) {
      cplx a0 = a1[MPI(p1, n, 0)];
      F[0] += a0 * f[n] * yls[n * L];
      cplx df_r = fd[n] * yls[n * L];
      cplx df_th = -f[n] * dyls[n * L] * sthi;
      cplx df_x = df_r * sthi + df_th * cthi_ri;
      cplx df_y = df_r * cthi - df_th * sthi_ri;
      cplx df = df_x * yi + df_y * x[i];
      DF[0] += a0 * df;
      for (int m = 1; m <= n; m++) {
        cplx z1 = f[n] * yls[n * L + m] * sthi;
        F[m] += a1[MPI(p1, n, m)] * z1;
        F[-m] += a1[MPI(p1, n, -m)] * z1;
        df_r = fd[n] * yls[n * L + m] * sthi;
        df_th = -f[n] * dyls[n * L + m];
        df_x = df_r * sthi + df_th * cthi_ri;
        df_y = df_r * cthi - df_th * sthi_ri;
        df = df_x * yi + df_y * x[i];
        DF[m] += a1[MPI(p1, n, m)] * df;
        DF[-m] += a1[MPI(p1, n, -m)] * df;
      }
    }
  }
  cplx zk = kwave * r;
  if (kind == 0) h3dall(p2, zk, rs2, f, 1, fd);
  else besseljs3d(p2, zk, rs2, f, 1, fd);
  cplx *gsum = (cplx *)calloc((size_t)p2 + 1, sizeof(cplx));
  for (int n = 0; n <= p2; n++) {
    fd[n] = kwave * fd[n];
    gsum[n] = (f[n] * f[n] + fd[n] * fd[n]) * pi2i;
  }
  memset(a2, 0, sizeof(cplx) * (size_t)(p2 + 1) * (2 * p2 + 1));
  for (int i = 0; i < nquad; i++) {
    int L = p2 + 1;
    zylgndrf(p2, x[i], yls, R);
    for (int n = 0; n <= p2; n++)
      for (int m = 0; m <= n; m++) yls[n * L + m] = yls[n * L + m] * ((m & 1) ? -1.0 : 1.0) * s4i;
    const cplx *F = fdat + (size_t)i * W + nterm, *DF = dfdat + (size_t)i * W + nterm;
    for (int n = 0; n <= p2; n++) {
      a2[MPI(p2, n, 0)] += w[i] * yls[n * L] * (f[n] * F[0] + fd[n] * DF[0]) / gsum[n];
      for (int m = 1; m <= n; m++) {
        cplx z1 = yls[n * L + m] * f[n] / gsum[n];
        cplx z2 = yls[n * L + m] * fd[n] / gsum[n];
        a2[MPI(p2, n, m)] += w[i] * (z1 * F[m] + z2 * DF[m]);
        a2[MPI(p2, n, -m)] += w[i] * (z1 * F[-m] + z2 * DF[-m]);
      }
    }
  }
  free(x); free(w); free(fdat); free(dfdat); free(yls); free(dyls); free(f); free(fd);
  free(gsum);
}

/* zh3dmpmp / zh3dmploc / zh3dlocloc: rotate, shift along z, rotate back, add */
static void htranslate3(int kind, const cplx *c0, int p1, const cplx *a0, double rs1, double w1,
                        const cplx *c, int p2, cplx *out, double rs2, double w2, cplx zk,
                        const rats *R) {
  size_t n1 = (size_t)(p1 + 1) * (2 * p1 + 1), n2 = (size_t)(p2 + 1) * (2 * p2 + 1);
  cplx *az = (cplx *)calloc(n1, sizeof(cplx)), *azy = (cplx *)calloc(n1, sizeof(cplx));
  cplx *bzy = (cplx *)calloc(n2, sizeof(cplx)), *bz = (cplx *)calloc(n2, sizeof(cplx));
  cplx *bn = (cplx *)calloc(n2, sizeof(cplx));
  cplx xc1[3], xc2[3], cb = 1, sb = 0, ca = 1, sa = 0;
  double e2 = cabs(c[1] - c0[1]);
  for (int d = 0; d < 3; d++) xc1[d] = c[d] - c0[d];
  if (e2 <= F16) {
    memcpy(az, a0, n1 * sizeof(cplx));
  } else {
    cplx rxy = zsqrt_r(xc1[0] * xc1[0] + xc1[1] * xc1[1]);
    cb = -xc1[0] / rxy;
    sb = -xc1[1] / rxy;
    xc1[0] = -rxy;
    xc1[1] = 0;
    zrot(p1, a0, az, cb, sb);
  }
  double e1 = cabs(xc1[0]);
  if (e1 <= F16) {
    for (int d = 0; d < 3; d++) xc2[d] = xc1[d];
    memcpy(azy, az, n1 * sizeof(cplx));
  } else {
    cplx rxz = zsqrt_r(xc1[0] * xc1[0] + xc1[2] * xc1[2]);
    xc2[0] = 0; xc2[1] = 0; xc2[2] = rxz;
    ca = xc1[2] / rxz;
    sa = xc1[0] / rxz;
    yrot(p1, az, azy, ca, sa, R);
  }
  cplx zshift = xc2[2];
  int nquad = (int)(p2 * 2.5);
  double r = kind == 1 ? w1 / 2 * sqrt(3.0) : (kind == 0 ? w1 * sqrt(3.0) : w2 * sqrt(3.0));
  hzshift(kind, r, nquad, zshift, p1, p2, rs1, rs2, zk, azy, bzy, R);
  if (e1 <= F16) memcpy(bz, bzy, n2 * sizeof(cplx));
  else yrot(p2, bzy, bz, ca, -sa, R);
  if (e2 <= F16) memcpy(bn, bz, n2 * sizeof(cplx));
  else zrot(p2, bz, bn, cb, -sb);
  for (size_t i = 0; i < n2; i++) out[i] += bn[i];
  free(az); free(azy); free(bzy); free(bz); free(bn);
}

int o_zhfmm3d(double eps, const double *zk_, int ns, const double *zsrc_, int ifcharge,
              const double *charge_, int ifdipole, const double *dipstr_, const double *dipvec_,
              double *pot_, double *grad_, int nt, const double *ztarg_, int ifpgh, int isep,
              int ifprint) {
  (void)ifprint;
  cplx zk = zk_[0] + I * zk_[1];
  if (ifcharge < 0 || ifcharge > 1) ifcharge = 1;
  if (ifdipole < 0 || ifdipole > 1) ifdipole = 0;
  if (ifpgh < 0 || ifpgh > 2) ifpgh = 1;
  memset(pot_, 0, sizeof(double) * 2 * nt);
  memset(grad_, 0, sizeof(double) * 6 * nt);
  const cplx *zsrc = (const cplx *)zsrc_, *ztarg = (const cplx *)ztarg_;
  double *src = (double *)malloc(sizeof(double) * 3 * ns), *targ = (double *)malloc(sizeof(double) * 3 * nt);
  for (int i = 0; i < 3 * ns; i++) src[i] = creal(zsrc[i]);
  for (int i = 0; i < 3 * nt; i++) targ[i] = creal(ztarg[i]);
  int ndiv = o_hndiv3d(eps, ns, nt);
  otree t;
  if (otree_build(3, src, ns, targ, nt, 0, ndiv, 0, 51, isep, 1, &t)) return -1;
  int nb = t.nboxes, nlev = t.nlevels;
  int *isrc = (int *)malloc(sizeof(int) * ns), *itarg = (int *)malloc(sizeof(int) * nt);
  int *isrcse = (int *)malloc(sizeof(int) * 2 * nb), *itargse = (int *)malloc(sizeof(int) * 2 * nb);
  otree_sort(&t, nt, targ, itarg, itargse);
  otree_sort(&t, ns, src, isrc, isrcse);
  free(src); free(targ);
  cplx *zs = (cplx *)calloc(3 * (size_t)ns, sizeof(cplx)), *zt = (cplx *)calloc(3 * (size_t)nt, sizeof(cplx));
  cplx *q = (cplx *)calloc(ns, sizeof(cplx)), *dsv = (cplx *)calloc(ns, sizeof(cplx));
  cplx *dv = (cplx *)calloc(3 * (size_t)ns, sizeof(cplx));
  for (int i = 0; i < ns; i++) {
    int j = isrc[i];
    for (int d = 0; d < 3; d++) zs[3 * i + d] = zsrc[3 * j + d];
    if (ifcharge == 1) q[i] = ((const cplx *)charge_)[j];
    if (ifdipole == 1) {
      dsv[i] = ((const cplx *)dipstr_)[j];
      for (int d = 0; d < 3; d++) dv[3 * i + d] = ((const cplx *)dipvec_)[3 * j + d];
    }
  }
  for (int i = 0; i < nt; i++)
    for (int d = 0; d < 3; d++) zt[3 * i + d] = ztarg[3 * itarg[i] + d];
  cplx *zcs = (cplx *)calloc(3 * (size_t)nb, sizeof(cplx)), *zct = (cplx *)calloc(3 * (size_t)nb, sizeof(cplx));
  for (int b = 0; b < nb; b++)
    for (int pass = 0; pass < 2; pass++) {
      const int *se = pass ? itargse : isrcse;
      const cplx *pts = pass ? zt : zs;
      cplx *zc = pass ? zct : zcs;
      int s0 = se[2 * b], s1 = se[2 * b + 1];
      if (s0 <= s1) {
        double a[3] = {0, 0, 0};
        for (int i = s0; i <= s1; i++)
          for (int d = 0; d < 3; d++) a[d] += cimag(pts[3 * i + d]);
        for (int d = 0; d < 3; d++) zc[3 * b + d] = t.centers[3 * b + d] + I * (a[d] / (s1 - s0 + 1));
      }
    }
  /* rescale to the unit root box (zhfmm3d.f:183-205) */
  double b0 = t.boxsize[0], b0inv = 1.0 / b0, b0inv2 = b0inv * b0inv;
  for (int i = 0; i < 3 * ns; i++) zs[i] *= b0inv;
  for (int i = 0; i < 3 * nt; i++) zt[i] *= b0inv;
  if (ifcharge == 1) for (int i = 0; i < ns; i++) q[i] *= b0inv;
  if (ifdipole == 1) for (int i = 0; i < 3 * ns; i++) dv[i] *= b0inv2;
  for (int i = 0; i < 3 * nb; i++) { zcs[i] *= b0inv; zct[i] *= b0inv; }
  cplx zkf = zk * b0;
  double *bsz = (double *)malloc(sizeof(double) * (nlev + 1)), *rsc = (double *)malloc(sizeof(double) * (nlev + 1));
  int *pl = (int *)malloc(sizeof(int) * (nlev + 1));
  int pmax = 0;
  for (int l = 0; l <= nlev; l++) {
    bsz[l] = t.boxsize[l] * b0inv;
    rsc[l] = bsz[l] * cabs(zkf);
    if (rsc[l] > 1) rsc[l] = 1;
  }
  for (int l = 0; l <= nlev; l++) {
    pl[l] = o_h3dterms(bsz[l], creal(zkf), cimag(zkf), eps, isep) + 0; /* n0 = 0 */
    if (pl[l] > pmax) pmax = pl[l];
    if (l > 0 && pl[l] > pl[l - 1]) pl[l] = pl[l - 1];
  }
  olists L;
  olists_build(&t, &L);
  rats R = rats_new(pmax);
  size_t *off = (size_t *)malloc(sizeof(size_t) * (nb + 1));
  off[0] = 0;
  for (int b = 0; b < nb; b++) {
    int p = pl[t.ilevel[b]];
    off[b + 1] = off[b] + (size_t)(p + 1) * (2 * p + 1);
  }
  cplx *mp = (cplx *)calloc(off[nb], sizeof(cplx)), *loc = (cplx *)calloc(off[nb], sizeof(cplx));
  cplx *ps = (cplx *)calloc(nt, sizeof(cplx)), *gs = (cplx *)calloc(3 * (size_t)nt, sizeof(cplx));
#define NS3(b) (isrcse[2 * (b) + 1] - isrcse[2 * (b)] + 1)
#define NT3(b) (itargse[2 * (b) + 1] - itargse[2 * (b)] + 1)
  /* step 1: P2M */
  for (int l = 1; l <= nlev; l++)
#pragma omp parallel for schedule(dynamic)
    for (int b = t.laddr[2 * l]; b <= t.laddr[2 * l + 1]; b++) {
      int s0 = isrcse[2 * b];
      if (t.nchild[b] == 0 && NS3(b) > 0)
        hform3(zkf, rsc[l], &zs[3 * s0], NS3(b), &q[s0], &dsv[s0], &dv[3 * s0], &zcs[3 * b], pl[l],
               mp + off[b], ifcharge, ifdipole, 0, &R);
    }
  /* step 2: M2M */
  for (int l = nlev - 1; l >= 1; l--)
#pragma omp parallel for schedule(dynamic)
    for (int b = t.laddr[2 * l]; b <= t.laddr[2 * l + 1]; b++)
      if (t.nchild[b] > 0 && NS3(b) > 0)
        for (int c = 0; c < t.nchild[b]; c++) {
          int jb = t.ichild[8 * b + c];
          if (NS3(jb) > 0)
            htranslate3(0, &zcs[3 * jb], pl[l + 1], mp + off[jb], rsc[l + 1], bsz[l + 1],
                        &zcs[3 * b], pl[l], mp + off[b], rsc[l], bsz[l], zkf, &R);
        }
  /* step 3: P2P */
#pragma omp parallel for schedule(dynamic)
  for (int b = 0; b < nb; b++) {
    int s0 = itargse[2 * b];
    if (NT3(b) > 0 && L.nlist[0][b] > 0 && t.nchild[b] == 0)
      for (int i = 0; i < L.nlist[0][b]; i++) {
        int jb = L.list[0][(size_t)b * L.mnlist[0] + i];
        int j0 = isrcse[2 * jb];
        if (NS3(jb) > 0) {
          double zkd[2] = {creal(zkf), cimag(zkf)};
          o_zh3devaldirect(zkd, NT3(b), (const double *)&zt[3 * s0], NS3(jb),
                           (const double *)&zs[3 * j0], (const double *)&q[j0],
                           (const double *)&dsv[j0], (const double *)&dv[3 * j0], ifcharge,
                           (double *)&ps[s0], (double *)&gs[3 * s0], ifdipole, ifpgh);
        }
      }
  }
  /* step 4: M2L */
#pragma omp parallel for schedule(dynamic)
  for (int b = 0; b < nb; b++) {
    int l = t.ilevel[b];
    if (NT3(b) > 0 && L.nlist[1][b] > 0)
      for (int i = 0; i < L.nlist[1][b]; i++) {
        int jb = L.list[1][(size_t)b * L.mnlist[1] + i];
        if (NS3(jb) > 0)
          htranslate3(1, &zcs[3 * jb], pl[l], mp + off[jb], rsc[l], bsz[l], &zct[3 * b], pl[l],
                      loc + off[b], rsc[l], bsz[l], zkf, &R);
      }
  }
  /* step 5: M2T (list 3) */
#pragma omp parallel for schedule(dynamic)
  for (int b = 0; b < nb; b++) {
    int s0 = itargse[2 * b];
    if (NT3(b) > 0 && t.nchild[b] == 0 && L.nlist[2][b] > 0)
      for (int i = 0; i < L.nlist[2][b]; i++) {
        int jb = L.list[2][(size_t)b * L.mnlist[2] + i];
        if (NS3(jb) > 0) {
          int lj = t.ilevel[jb];
          heval3(zkf, NT3(b), &zt[3 * s0], rsc[lj], pl[lj], &zcs[3 * jb], mp + off[jb], &ps[s0],
                 &gs[3 * s0], ifpgh, 0, &R);
        }
      }
  }
  /* step 6: P2L (list 4) */
#pragma omp parallel for schedule(dynamic)
  for (int b = 0; b < nb; b++) {
    int l = t.ilevel[b];
    if (NT3(b) > 0 && L.nlist[3][b] > 0)
      for (int i = 0; i < L.nlist[3][b]; i++) {
        int jb = L.list[3][(size_t)b * L.mnlist[3] + i];
        int j0 = isrcse[2 * jb];
        if (NS3(jb) > 0)
          hform3(zkf, rsc[l], &zs[3 * j0], NS3(jb), &q[j0], &dsv[j0], &dv[3 * j0], &zct[3 * b],
                 pl[l], loc + off[b], ifcharge, ifdipole, 1, &R);
      }
  }
  /* step 7: L2L; the test is (A and B) or C as written (zhfmm3d.f:572-573) */
  for (int l = 1; l <= nlev - 1; l++)
#pragma omp parallel for schedule(dynamic)
    for (int b = t.laddr[2 * l]; b <= t.laddr[2 * l + 1]; b++)
      if ((NT3(b) > 0 && L.nlist[1][b] > 0) || L.nlist[3][b] > 0)
        for (int c = 0; c < t.nchild[b]; c++) {
          int jb = t.ichild[8 * b + c];
          if (NT3(jb) > 0)
            htranslate3(2, &zct[3 * b], pl[l], loc + off[b], rsc[l], bsz[l], &zct[3 * jb],
                        pl[l + 1], loc + off[jb], rsc[l + 1], bsz[l + 1], zkf, &R);
        }
  /* step 8: L2T */
#pragma omp parallel for schedule(dynamic)
  for (int b = 0; b < nb; b++) {
    int s0 = itargse[2 * b];
    if (t.nchild[b] == 0 && NT3(b) > 0) {
      int l = t.ilevel[b];
      heval3(zkf, NT3(b), &zt[3 * s0], rsc[l], pl[l], &zct[3 * b], loc + off[b], &ps[s0],
             &gs[3 * s0], ifpgh, 1, &R);
    }
  }
  cplx *P_ = (cplx *)pot_, *G_ = (cplx *)grad_;
  for (int i = 0; i < nt; i++) {
    int j = itarg[i];
    P_[j] = ps[i];
    if (ifpgh >= 2)
      for (int d = 0; d < 3; d++) G_[3 * j + d] = gs[3 * i + d] * b0inv;
  }
  rats_free(&R);
  free(mp); free(loc); free(off); free(ps); free(gs); free(bsz); free(rsc); free(pl);
  free(zs); free(zt); free(q); free(dsv); free(dv); free(zcs); free(zct);
  free(isrc); free(itarg); free(isrcse); free(itargse);
  olists_free(&L);
  otree_free(&t);
  return 0;
}
