/*
 * Oracle (TEST INFRASTRUCTURE ONLY): 2D Laplace complex-coordinate FMM.
 *
 * Restates zfmm2d/src/laplace/zlfmm2d.f (driver :14-234, zlfmm2dmain
 * :240-594, zl2devaldirect :600-654, zl2dformmp :660-724, zl2dformloc
 * :730-798, zl2devalmp :804-857, zl2devalloc :863-915), the translations in
 * zfmm2d/src/laplace/zl2dtrans.f (zl2dlocloc :8-75, zl2dmploc :81-150,
 * zl2dmpmp :156-229), lndiv2d.f:1-39, l2dterms.f:38-82 and init_carray
 * (zfmm2d/src/common/fmmcommon2d.f:150-165).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "ocommon.h"

void o_lndiv2d(double eps, int ns, int nt, int *ndiv, int *idivflag) {
  *idivflag = 0;
  if (eps >= 0.5e-0) *ndiv = 3;
  else if (eps >= 0.5e-1) *ndiv = 5;
  else if (eps >= 0.5e-2) *ndiv = 8;
  else if (eps >= 0.5e-3) *ndiv = 10;
  else if (eps >= 0.5e-6) *ndiv = 15;
  else if (eps >= 0.5e-9) *ndiv = 20;
  else if (eps >= 0.5e-12) *ndiv = 25;
  else if (eps >= 0.5e-15) *ndiv = 45;
  else *ndiv = ns + nt;
}

int o_l2dterms(double eps) {
  /* decay of (sqrt(2)/2)^j / 1.5^(j+1); first j in 2..100 below eps */
  double z2 = sqrt(2.0) / 2.0;
  for (int j = 2; j <= 100; j++) {
    double x = pow(z2, j) / pow(1.5, j + 1);
    if (x < eps) return j;
  }
  return 1;
}

void o_init_carray(double *c, int ldc) {
  int n = ldc + 1;
  for (int l = 0; l <= ldc; l++) c[l * n + 0] = 1.0;
  for (int m = 1; m <= ldc; m++) {
    c[m * n + m] = 1.0;
    for (int l = m + 1; l <= ldc; l++) c[l * n + m] = c[(l - 1) * n + m] + c[(l - 1) * n + m - 1];
  }
}
#define CARR(l, m) carray[(l) * (ldc + 1) + (m)]

void o_zl2devaldirect(int nt, const double *ztarg, int ns, const double *zsrc,
                      const double *charge, const double *dipstr, const double *dipvec,
                      int ifcharge, double *pot, double *grad, int ifdipole, int ifpgh) {
  const cplx *zt = (const cplx *)ztarg, *zs = (const cplx *)zsrc;
  const cplx *q = (const cplx *)charge, *ds = (const cplx *)dipstr, *dv = (const cplx *)dipvec;
  cplx *p = (cplx *)pot, *g = (cplx *)grad;
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < nt; i++) {
    cplx pi = 0, g1 = 0, g2 = 0;
    for (int j = 0; j < ns; j++) {
      cplx y1mx1 = zs[2 * j] - zt[2 * i], y2mx2 = zs[2 * j + 1] - zt[2 * i + 1];
      cplx x1my1 = -y1mx1, x2my2 = -y2mx2;
      cplx rsq = y1mx1 * y1mx1 + y2mx2 * y2mx2;
      cplx rz = csqrt(rsq);
      if (cabs(rz) > (double)1e-16f) {  /* REAL*4 literal 1E-16 */
        if (ifcharge == 1) pi += q[j] * clog(rz);
        if (ifdipole == 1) pi -= ds[j] * (dv[2 * j] * y1mx1 + dv[2 * j + 1] * y2mx2) / rsq;
        if (ifpgh > 1) {
          if (ifcharge == 1) {
            g1 += q[j] * x1my1 / rsq;
            g2 += q[j] * x2my2 / rsq;
          }
          if (ifdipole == 1) {
            cplx r4 = rsq * rsq;
            g1 -= ds[j] * (dv[2 * j] * (x1my1 * x1my1 - x2my2 * x2my2) +
                           dv[2 * j + 1] * 2.0 * x1my1 * x2my2) / r4;
            g2 -= ds[j] * (dv[2 * j] * 2.0 * x1my1 * x2my2 +
                           dv[2 * j + 1] * (x2my2 * x2my2 - x1my1 * x1my1)) / r4;
          }
        }
      }
    }
    p[i] += pi;
    if (ifpgh > 1) { g[2 * i] += g1; g[2 * i + 1] += g2; }
  }
}

static void formmp(double rscale, const cplx *zs, int npts, const cplx *q, const cplx *ds,
                   const cplx *dv, const cplx *zc, int nterm, cplx *mp, int ifcharge,
                   int ifdipole, int local) {
  /* mp indexed -nterm..nterm via mp[nterm + m] */
  cplx *zall = (cplx *)malloc(sizeof(cplx) * (nterm + 1));
  cplx *ezall = (cplx *)malloc(sizeof(cplx) * (nterm + 1));
  zall[0] = 1; ezall[0] = 1;
  cplx *M = mp + nterm;
  for (int i = 0; i < npts; i++) {
    cplx rz, ez;
    o_zcart2polar(&zs[2 * i], zc, &rz, &ez);
    cplx z = rz / rscale;
    for (int m = 1; m <= nterm; m++) { zall[m] = zall[m - 1] * z; ezall[m] = ezall[m - 1] * ez; }
    cplx pr = 0, pe = 0;
    if (ifdipole == 1) {
      cplx vr1 = (zs[2 * i] - zc[0]) / rz, vr2 = (zs[2 * i + 1] - zc[1]) / rz;
      cplx ve1 = -vr2, ve2 = vr1;
      pr = vr1 * dv[2 * i] + vr2 * dv[2 * i + 1];
      pe = ve1 * dv[2 * i] + ve2 * dv[2 * i + 1];
    }
    if (!local) {
      if (ifcharge == 1) M[0] += q[i];
      for (int m = 1; m <= nterm; m++) {
        if (ifcharge == 1) {
          M[m] -= zall[m] / ezall[m] * q[i] / (double)m / 2.0;
          M[-m] -= zall[m] * ezall[m] * q[i] / (double)m / 2.0;
        }
        if (ifdipole == 1) {
          cplx dr = -zall[m - 1] / ezall[m] / 2.0 / rscale;
          cplx dth = I * zall[m] / ezall[m] / 2.0;
          M[m] -= ds[i] * (dr * pr + dth * pe / rz);
          dr = -zall[m - 1] * ezall[m] / 2.0 / rscale;
          dth = -I * zall[m] * ezall[m] / 2.0;
          M[-m] -= ds[i] * (dr * pr + dth * pe / rz);
        }
      }
    } else {
      if (ifdipole == 1) M[0] -= ds[i] * pr / rz;
      if (ifcharge == 1) M[0] += q[i] * clog(rz);
      for (int m = 1; m <= nterm; m++) {
        if (ifcharge == 1) {
          M[m] -= 1.0 / zall[m] / ezall[m] * q[i] / (double)m / 2.0;
          M[-m] -= 1.0 / zall[m] * ezall[m] * q[i] / (double)m / 2.0;
        }
        if (ifdipole == 1) {
          cplx dr = 1.0 / zall[m] / rz / ezall[m] / 2.0;
          cplx dth = I / zall[m] / ezall[m] / 2.0;
          M[m] -= ds[i] * (dr * pr + dth * pe / rz);
          dr = 1.0 / zall[m] / rz * ezall[m] / 2.0;
          dth = -I / zall[m] * ezall[m] / 2.0;
          M[-m] -= ds[i] * (dr * pr + dth * pe / rz);
        }
      }
    }
  }
  free(zall); free(ezall);
}

static void evalexp(int nt, const cplx *zt, double rscale, int nterm, const cplx *zc,
                    const cplx *mp, cplx *pot, cplx *grad, int ifpgh, int local) {
  cplx *zall = (cplx *)malloc(sizeof(cplx) * (nterm + 1));
  cplx *ezall = (cplx *)malloc(sizeof(cplx) * (nterm + 1));
  zall[0] = 1; ezall[0] = 1;
  const cplx *M = mp + nterm;
  for (int i = 0; i < nt; i++) {
    cplx zr, ez;
    o_zcart2polar(&zt[2 * i], zc, &zr, &ez);
    cplx z = zr / rscale;
    for (int m = 1; m <= nterm; m++) { zall[m] = zall[m - 1] * z; ezall[m] = ezall[m - 1] * ez; }
    cplx vr1 = 0, vr2 = 0, ve1 = 0, ve2 = 0;
    if (ifpgh > 1) {
      vr1 = (zt[2 * i] - zc[0]) / zr; vr2 = (zt[2 * i + 1] - zc[1]) / zr;
      ve1 = -vr2; ve2 = vr1;
    }
    if (!local) {
      pot[i] += M[0] * clog(zr);
      if (ifpgh > 1) {
        cplx dr = 1.0 / zr;
        grad[2 * i] += M[0] * dr * vr1;
        grad[2 * i + 1] += M[0] * dr * vr2;
      }
      for (int m = 1; m <= nterm; m++) {
        pot[i] += M[m] / zall[m] * ezall[m];
        pot[i] += M[-m] / zall[m] / ezall[m];
        if (ifpgh > 1) {
          cplx dr = -(double)m / zall[m] * ezall[m] / zr;
          cplx dth = I * (double)m / zall[m] * ezall[m];
          grad[2 * i] += M[m] * (dr * vr1 + dth * ve1 / zr);
          grad[2 * i + 1] += M[m] * (dr * vr2 + dth * ve2 / zr);
          dr = -(double)m / zall[m] / ezall[m] / zr;
          dth = -I * (double)m / zall[m] / ezall[m];
          grad[2 * i] += M[-m] * (dr * vr1 + dth * ve1 / zr);
          grad[2 * i + 1] += M[-m] * (dr * vr2 + dth * ve2 / zr);
        }
      }
    } else {
      pot[i] += M[0];
      for (int m = 1; m <= nterm; m++) {
        pot[i] += M[m] * zall[m] * ezall[m];
        pot[i] += M[-m] * zall[m] / ezall[m];
        if (ifpgh > 1) {
          cplx dr = (double)m * zall[m - 1] * ezall[m] / rscale;
          cplx dth = I * (double)m * zall[m] * ezall[m];
          grad[2 * i] += M[m] * (dr * vr1 + dth * ve1 / zr);
          grad[2 * i + 1] += M[m] * (dr * vr2 + dth * ve2 / zr);
          dr = (double)m * zall[m - 1] / ezall[m] / rscale;
          dth = -I * (double)m * zall[m] / ezall[m];
          grad[2 * i] += M[-m] * (dr * vr1 + dth * ve1 / zr);
          grad[2 * i + 1] += M[-m] * (dr * vr2 + dth * ve2 / zr);
        }
      }
    }
  }
  free(zall); free(ezall);
}

static double isgn(int n) { return (n & 1) ? -1.0 : 1.0; }

/* zl2dlocloc: loc2 at zc2 -> loc1 at zc1 */
static void locloc(const cplx *zc1, const cplx *zc2, double rs1, double rs2, int n1, int n2,
                   cplx *loc1, const cplx *loc2, const double *carray, int ldc) {
  double *r1 = (double *)malloc(sizeof(double) * (n1 + 1)), *r2 = (double *)malloc(sizeof(double) * (n2 + 1));
  r1[0] = 1; for (int n = 1; n <= n1; n++) r1[n] = r1[n - 1] * rs1;
  r2[0] = 1; for (int n = 1; n <= n2; n++) r2[n] = r2[n - 1] * rs2;
  cplx r0, e0;
  o_zcart2polar(zc2, zc1, &r0, &e0);
  int nt = n1 > n2 ? n1 : n2;
  cplx *ra = (cplx *)malloc(sizeof(cplx) * (n1 + n2 + 1)), *ea = (cplx *)malloc(sizeof(cplx) * (n1 + n2 + 1));
  for (int n = 0; n <= n1 + n2; n++) { ra[n] = 1; ea[n] = 1; }
  for (int n = 1; n <= nt; n++) { ra[n] = ra[n - 1] * r0; ea[n] = ea[n - 1] * e0; }
  cplx *L1 = loc1 + n1;
  const cplx *L2 = loc2 + n2;
  L1[0] += L2[0];
  for (int n = 1; n <= n2; n++) {
    L1[0] += isgn(n) * ra[n] * ea[n] * L2[n] / r2[n];
    L1[0] += isgn(n) * ra[n] / ea[n] * L2[-n] / r2[n];
  }
  for (int k = 1; k <= n1; k++)
    for (int n = k; n <= n2; n++) {
      L1[k] += isgn(n - k) * CARR(n, k) * ra[n - k] * ea[n - k] * L2[n] * r1[k] / r2[n];
      L1[-k] += isgn(n - k) * CARR(n, k) * ra[n - k] / ea[n - k] * L2[-n] * r1[k] / r2[n];
    }
  free(r1); free(r2); free(ra); free(ea);
}

/* zl2dmploc: mp at zc2 -> loc at zc1 */
static void mploc(const cplx *zc1, const cplx *zc2, double rs1, double rs2, int n1, int n2,
                  cplx *loc, const cplx *mp, const double *carray, int ldc) {
  double *r1 = (double *)malloc(sizeof(double) * (n1 + 1)), *r2 = (double *)malloc(sizeof(double) * (n2 + 1));
  r1[0] = 1; for (int n = 1; n <= n1; n++) r1[n] = r1[n - 1] * rs1;
  r2[0] = 1; for (int n = 1; n <= n2; n++) r2[n] = r2[n - 1] * rs2;
  cplx r0, e0;
  o_zcart2polar(zc2, zc1, &r0, &e0);
  int nt = n1 + n2;
  cplx *ra = (cplx *)malloc(sizeof(cplx) * (nt + 1)), *ea = (cplx *)malloc(sizeof(cplx) * (nt + 1));
  ra[0] = 1; ea[0] = 1;
  for (int m = 1; m <= nt; m++) { ra[m] = ra[m - 1] * r0; ea[m] = ea[m - 1] * e0; }
  cplx *L = loc + n1;
  const cplx *M = mp + n2;
  L[0] += M[0] * clog(r0);
  for (int n = 1; n <= n2; n++) {
    L[0] += r2[n] * isgn(n) * M[n] * ea[n] / ra[n];
    L[0] += r2[n] * isgn(n) * M[-n] / ea[n] / ra[n];
  }
  for (int k = 1; k <= n1; k++) {
    L[k] -= r1[k] * M[0] * ((1.0 / 2) / k) / ea[k] / ra[k];
    L[-k] -= r1[k] * M[0] * ((1.0 / 2) / k) * ea[k] / ra[k];
    for (int n = 1; n <= n2; n++) {
      L[k] += isgn(n) * M[-n] * r1[k] * r2[n] * CARR(n + k - 1, k) / ea[n + k] / ra[n + k];
      L[-k] += isgn(n) * M[n] * r1[k] * r2[n] * CARR(n + k - 1, k) * ea[n + k] / ra[n + k];
    }
  }
  free(r1); free(r2); free(ra); free(ea);
}

/* zl2dmpmp: mp2 at zc2 -> mp1 at zc1 */
static void mpmp(const cplx *zc1, const cplx *zc2, double rs1, double rs2, int n1, int n2,
                 cplx *mp1, const cplx *mp2, const double *carray, int ldc) {
  double *r1 = (double *)malloc(sizeof(double) * (n1 + 1)), *r2 = (double *)malloc(sizeof(double) * (n2 + 1));
  r1[0] = 1; for (int n = 1; n <= n1; n++) r1[n] = r1[n - 1] * rs1;
  r2[0] = 1; for (int n = 1; n <= n2; n++) r2[n] = r2[n - 1] * rs2;
  cplx r0, e0;
  o_zcart2polar(zc2, zc1, &r0, &e0);
  int nt = n1 > n2 ? n1 : n2;
  cplx *ra = (cplx *)malloc(sizeof(cplx) * (n1 + n2 + 1)), *ea = (cplx *)malloc(sizeof(cplx) * (n1 + n2 + 1));
  ra[0] = 1; ea[0] = 1;
  for (int n = 1; n <= nt; n++) { ra[n] = ra[n - 1] * r0; ea[n] = ea[n - 1] * e0; }
  cplx *A = mp1 + n1;
  const cplx *Bm = mp2 + n2;
  A[0] += Bm[0];
  for (int k = 1; k <= n1; k++) {
    A[k] -= ((1.0 / 2) / k) * ra[k] / ea[k] * Bm[0] / r1[k];
    A[-k] -= ((1.0 / 2) / k) * ra[k] * ea[k] * Bm[0] / r1[k];
    for (int n = 1; n <= k; n++) {
      if (n <= n2) {
        double rfrac = r2[n] / r1[k];
        A[k] += rfrac * CARR(k - 1, k - n) * ra[k - n] / ea[k - n] * Bm[n];
        A[-k] += rfrac * CARR(k - 1, k - n) * ra[k - n] * ea[k - n] * Bm[-n];
      }
    }
  }
  free(r1); free(r2); free(ra); free(ea);
}

int o_zlfmm2d(double eps, int ns, const double *zsrc, int ifcharge, const double *charge,
              int ifdipole, const double *dipstr, const double *dipvec, double *pot,
              double *grad, int nt, const double *ztarg, int ifpgh, int isep, int ifprint) {
  (void)ifprint;
  if (ifcharge < 0 || ifcharge > 1) ifcharge = 1;
  if (ifdipole < 0 || ifdipole > 1) ifdipole = 0;
  if (ifpgh < 0 || ifpgh > 2) ifpgh = 1;
  memset(pot, 0, sizeof(double) * 2 * nt);
  memset(grad, 0, sizeof(double) * 4 * nt);
  int ndiv, idivflag;
  o_lndiv2d(eps, ns, nt, &ndiv, &idivflag);
  o2d_state S;
  if (o2d_setup(ns, zsrc, ifcharge, charge, ifdipole, dipstr, dipvec, nt, ztarg, idivflag, ndiv,
                isep, &S))
    return -1;
  otree *t = &S.t;
  olists *L = &S.L;
  int nb = t->nboxes, nlev = t->nlevels;
  double *rscales = (double *)malloc(sizeof(double) * (nlev + 1));
  int *nterms = (int *)malloc(sizeof(int) * (nlev + 1));
  int nmax = 0;
  for (int i = 0; i <= nlev; i++) {
    rscales[i] = t->boxsize[i];
    nterms[i] = o_l2dterms(eps);
    if (nterms[i] > nmax) nmax = nterms[i];
  }
  int P = 2 * nmax + 1;
  cplx *mp = (cplx *)calloc((size_t)P * nb, sizeof(cplx));
  cplx *loc = (cplx *)calloc((size_t)P * nb, sizeof(cplx));
  int ldc = 2 * nmax;
  double *carray = (double *)malloc(sizeof(double) * (ldc + 1) * (ldc + 1));
  o_init_carray(carray, ldc);
  cplx *potsort = (cplx *)calloc(nt, sizeof(cplx));
  cplx *gradsort = (cplx *)calloc(2 * (size_t)nt, sizeof(cplx));
  const int *se_s = S.isrcse, *se_t = S.itargse;
#define MP(b, nterm) (mp + (size_t)(b) * P + (nmax - (nterm)))
#define LOC(b, nterm) (loc + (size_t)(b) * P + (nmax - (nterm)))
#define NS(b) (se_s[2 * (b) + 1] - se_s[2 * (b)] + 1)
#define NT(b) (se_t[2 * (b) + 1] - se_t[2 * (b)] + 1)
  /* step 1: P2M */
  for (int ilev = 1; ilev <= nlev; ilev++) {
    int nterm = nterms[ilev];
#pragma omp parallel for schedule(dynamic)
    for (int ib = t->laddr[2 * ilev]; ib <= t->laddr[2 * ilev + 1]; ib++) {
      int s = se_s[2 * ib];
      if (t->nchild[ib] == 0 && NS(ib) > 0)
        formmp(rscales[ilev], &S.zsrcsort[2 * s], NS(ib), &S.chargesort[s], &S.dipstrsort[s],
               &S.dipvecsort[2 * s], &S.zcsrc[2 * ib], nterm, MP(ib, nterm), ifcharge, ifdipole, 0);
    }
  }
  /* step 2: M2M */
  for (int ilev = nlev - 1; ilev >= 1; ilev--) {
    int nterm = nterms[ilev], nterm1 = nterms[ilev + 1];
#pragma omp parallel for schedule(dynamic)
    for (int ib = t->laddr[2 * ilev]; ib <= t->laddr[2 * ilev + 1]; ib++) {
      if (t->nchild[ib] > 0 && NS(ib) > 0)
        for (int j = 0; j < t->nchild[ib]; j++) {
          int jb = t->ichild[ib * 4 + j];
          if (NS(jb) > 0)
            mpmp(&S.zcsrc[2 * ib], &S.zcsrc[2 * jb], rscales[ilev], rscales[ilev + 1], nterm,
                 nterm1, MP(ib, nterm), MP(jb, nterm1), carray, ldc);
        }
    }
  }
  /* step 3: P2P over list1 */
#pragma omp parallel for schedule(dynamic)
  for (int ib = 0; ib < nb; ib++) {
    int s = se_t[2 * ib];
    if (NT(ib) > 0 && L->nlist[0][ib] > 0 && t->nchild[ib] == 0)
      for (int il = 0; il < L->nlist[0][ib]; il++) {
        int jb = L->list[0][(size_t)ib * L->mnlist[0] + il];
        int js = se_s[2 * jb];
        if (NS(jb) > 0)
          o_zl2devaldirect(NT(ib), (const double *)&S.ztargsort[2 * s], NS(jb),
                           (const double *)&S.zsrcsort[2 * js], (const double *)&S.chargesort[js],
                           (const double *)&S.dipstrsort[js], (const double *)&S.dipvecsort[2 * js],
                           ifcharge, (double *)&potsort[s], (double *)&gradsort[2 * s], ifdipole,
                           ifpgh);
      }
  }
  /* step 4: M2L over list2 */
#pragma omp parallel for schedule(dynamic)
  for (int ib = 0; ib < nb; ib++) {
    int lev = t->ilevel[ib], nterm = nterms[lev];
    if (NT(ib) > 0 && L->nlist[1][ib] > 0)
      for (int il = 0; il < L->nlist[1][ib]; il++) {
        int jb = L->list[1][(size_t)ib * L->mnlist[1] + il];
        if (NS(jb) > 0)
          mploc(&S.zctarg[2 * ib], &S.zcsrc[2 * jb], rscales[lev], rscales[lev], nterm, nterm,
                LOC(ib, nterm), MP(jb, nterm), carray, ldc);
      }
  }
  /* step 5: M2T over list3 */
#pragma omp parallel for schedule(dynamic)
  for (int ib = 0; ib < nb; ib++) {
    int s = se_t[2 * ib];
    if (NT(ib) > 0 && t->nchild[ib] == 0 && L->nlist[2][ib] > 0)
      for (int il = 0; il < L->nlist[2][ib]; il++) {
        int jb = L->list[2][(size_t)ib * L->mnlist[2] + il];
        if (NS(jb) > 0) {
          int lev = t->ilevel[jb], nterm = nterms[lev];
          evalexp(NT(ib), &S.ztargsort[2 * s], rscales[lev], nterm, &S.zcsrc[2 * jb],
                  MP(jb, nterm), &potsort[s], &gradsort[2 * s], ifpgh, 0);
        }
      }
  }
  /* step 6: P2L over list4 */
#pragma omp parallel for schedule(dynamic)
  for (int ib = 0; ib < nb; ib++) {
    int lev = t->ilevel[ib], nterm = nterms[lev];
    if (NT(ib) > 0 && L->nlist[3][ib] > 0)
      for (int il = 0; il < L->nlist[3][ib]; il++) {
        int jb = L->list[3][(size_t)ib * L->mnlist[3] + il];
        int js = se_s[2 * jb];
        if (NS(jb) > 0)
          formmp(rscales[lev], &S.zsrcsort[2 * js], NS(jb), &S.chargesort[js], &S.dipstrsort[js],
                 &S.dipvecsort[2 * js], &S.zctarg[2 * ib], nterm, LOC(ib, nterm), ifcharge,
                 ifdipole, 1);
      }
  }
  /* step 7: L2L */
  for (int ilev = 1; ilev <= nlev - 1; ilev++) {
    int nterm = nterms[ilev], nterm1 = nterms[ilev + 1];
#pragma omp parallel for schedule(dynamic)
    for (int ib = t->laddr[2 * ilev]; ib <= t->laddr[2 * ilev + 1]; ib++) {
      if (NT(ib) > 0 && (L->nlist[1][ib] > 0 || L->nlist[3][ib] > 0))
        for (int j = 0; j < t->nchild[ib]; j++) {
          int jb = t->ichild[ib * 4 + j];
          if (NT(jb) > 0)
            locloc(&S.zctarg[2 * jb], &S.zctarg[2 * ib], rscales[ilev + 1], rscales[ilev], nterm1,
                   nterm, LOC(jb, nterm1), LOC(ib, nterm), carray, ldc);
        }
    }
  }
  /* step 8: L2T */
#pragma omp parallel for schedule(dynamic)
  for (int ib = 0; ib < nb; ib++) {
    int s = se_t[2 * ib];
    if (t->nchild[ib] == 0 && NT(ib) > 0) {
      int lev = t->ilevel[ib], nterm = nterms[lev];
      evalexp(NT(ib), &S.ztargsort[2 * s], rscales[lev], nterm, &S.zctarg[2 * ib],
              LOC(ib, nterm), &potsort[s], &gradsort[2 * s], ifpgh, 1);
    }
  }
  cplx *P_ = (cplx *)pot, *G_ = (cplx *)grad;
  const double scale = 1.0 / (2.0 * M_PI);
  for (int i = 0; i < nt; i++) {
    int j = S.itarg[i];
    P_[j] = potsort[i] / 2.0 / M_PI;
    if (ifpgh > 1) { G_[2 * j] = gradsort[2 * i] / 2.0 / M_PI; G_[2 * j + 1] = gradsort[2 * i + 1] / 2.0 / M_PI; }
  }
  (void)scale;
  free(rscales); free(nterms); free(mp); free(loc); free(carray); free(potsort); free(gradsort);
  o2d_free(&S);
  return 0;
}
