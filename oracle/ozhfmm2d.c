/*
 * Oracle (TEST INFRASTRUCTURE ONLY): 2D Helmholtz complex-coordinate FMM.
 *
 * Restates zfmm2d/src/helmholtz/zhfmm2d.f (driver :14-227, zhfmm2dmain
 * :233-604, zh2dformmp :610-686, zh2dformloc :692-766, zh2devaldirect
 * :773-838, zh2devalmp :844-901, zh2devalloc :907-964), the Graf translations
 * of zfmm2d/src/helmholtz/zh2dtrans.f (zh2dlocloc :6-78, zh2dmploc :84-142,
 * zh2dmpmp :225-303) and hndiv2d.f (same table as lndiv2d).  Special functions
 * come from ospecfun2d.c.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "ocommon.h"

static void hank(cplx z, cplx *h0, cplx *h1) {
  double a[2], b[2];
  o_hank103(creal(z), cimag(z), a, b);
  *h0 = a[0] + I * a[1];
  *h1 = b[0] + I * b[1];
}
static void h2dall_c(int n, cplx z, double rs, cplx *hv, int ifder, cplx *hd) {
  o_h2dall(n, creal(z), cimag(z), rs, (double *)hv, ifder, (double *)hd);
}
static void jbes_c(int n, cplx z, double rs, cplx *fj, int ifder, cplx *fd) {
  o_jbessel2d(n, creal(z), cimag(z), rs, (double *)fj, ifder, (double *)fd);
}
static double isg(int n) { return (n & 1) ? -1.0 : 1.0; }

void o_zh2devaldirect(const double *zk_, int nt, const double *ztarg, int ns, const double *zsrc,
                      const double *charge, const double *dipstr, const double *dipvec,
                      int ifcharge, double *pot, double *grad, int ifdipole, int ifpgh) {
  cplx zk = zk_[0] + I * zk_[1];
  const cplx *zt = (const cplx *)ztarg, *zs = (const cplx *)zsrc;
  const cplx *q = (const cplx *)charge, *ds = (const cplx *)dipstr, *dv = (const cplx *)dipvec;
  cplx *p = (cplx *)pot, *g = (cplx *)grad;
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < nt; i++) {
    cplx pi = 0, g1 = 0, g2 = 0;
    for (int j = 0; j < ns; j++) {
      cplx y1mx1 = zs[2 * j] - zt[2 * i], y2mx2 = zs[2 * j + 1] - zt[2 * i + 1];
      cplx x1my1 = -y1mx1, x2my2 = -y2mx2;
      cplx rz = csqrt(y1mx1 * y1mx1 + y2mx2 * y2mx2);
      cplx z = rz * zk, h0, h1;
      if (!(cabs(z) > (double)1e-16f && cimag(z) > -32)) continue; /* REAL*4 literal 1E-16 */
      hank(z, &h0, &h1);
      if (ifcharge == 1) pi += q[j] * h0;
      if (ifdipole == 1) {
        pi += ds[j] * dv[2 * j] * h1 * zk * y1mx1 / rz;
        pi += ds[j] * dv[2 * j + 1] * h1 * zk * y2mx2 / rz;
      }
      if (ifpgh > 1) {
        if (ifcharge == 1) {
          g1 -= q[j] * zk * h1 * (zt[2 * i] - zs[2 * j]) / rz;
          g2 -= q[j] * zk * h1 * (zt[2 * i + 1] - zs[2 * j + 1]) / rz;
        }
        if (ifdipole == 1) {
          cplx h2 = (2.0 / z) * h1 - h0;
          cplx dh1 = (h0 - h2) / 2.0;
          cplx tmp = dv[2 * j] * y1mx1 + dv[2 * j + 1] * y2mx2;
          cplx tmp1 = zk * dh1 * x1my1 / (rz * rz) - h1 * x1my1 / (rz * rz * rz);
          cplx tmp2 = zk * dh1 * x2my2 / (rz * rz) - h1 * x2my2 / (rz * rz * rz);
          g1 += ds[j] * zk * tmp1 * tmp - ds[j] * (zk * h1 / rz) * dv[2 * j];
          g2 += ds[j] * zk * tmp2 * tmp - ds[j] * (zk * h1 / rz) * dv[2 * j + 1];
        }
      }
    }
    p[i] += pi;
    if (ifpgh > 1) { g[2 * i] += g1; g[2 * i + 1] += g2; }
  }
}

/* zh2dformmp (local=0) and zh2dformloc (local=1) */
static void hform(cplx zk, double rscale, const cplx *zs, int npts, const cplx *q, const cplx *ds,
                  const cplx *dv, const cplx *zc, int nterm, cplx *mp, int ifcharge, int ifdipole,
                  int local) {
  int ifder = ifdipole == 1;
  cplx *f = (cplx *)calloc(nterm + 2, sizeof(cplx)), *fd = (cplx *)calloc(nterm + 2, sizeof(cplx));
  cplx *ezs = (cplx *)malloc(sizeof(cplx) * (2 * nterm + 1));
  cplx *E = ezs + nterm;
  cplx *M = mp + nterm;
  E[0] = 1;
  for (int i = 0; i < npts; i++) {
    cplx rz, ez;
    o_zcart2polar(&zs[2 * i], zc, &rz, &ez);
    cplx z = rz * zk;
    for (int m = 1; m <= nterm; m++) E[m] = E[m - 1] * ez;
    for (int m = 1; m <= nterm; m++) E[-m] = 1.0 / E[m];
    if (local) h2dall_c(nterm, z, rscale, f, ifder, fd);
    else jbes_c(nterm, z, rscale, f, ifder, fd);
    cplx pr = 0, pe = 0;
    if (ifdipole == 1) {
      cplx vr1 = (zs[2 * i] - zc[0]) / rz, vr2 = (zs[2 * i + 1] - zc[1]) / rz;
      cplx ve1 = -vr2, ve2 = vr1;
      pr = vr1 * dv[2 * i] + vr2 * dv[2 * i + 1];
      pe = ve1 * dv[2 * i] + ve2 * dv[2 * i + 1];
    }
    for (int m = 0; m <= nterm; m++) {
      if (ifcharge == 1) M[m] += f[m] * E[-m] * q[i];
      if (ifdipole == 1) {
        cplx dr = E[-m] * fd[m] * zk, dth = f[m] * (I * (double)(-m)) * E[-m];
        M[m] -= ds[i] * (dr * pr + dth * pe / rz);
      }
    }
    for (int m = -nterm; m <= -1; m++) {
      if (ifcharge == 1) M[m] += isg(m) * f[-m] * E[-m] * q[i];
      if (ifdipole == 1) {
        cplx dr = E[-m] * fd[-m] * zk, dth = f[-m] * (I * (double)(-m)) * E[-m];
        M[m] -= ds[i] * isg(m) * (dr * pr + dth * pe / rz);
      }
    }
  }
  free(f); free(fd); free(ezs);
}

/* zh2devalmp (local=0, Hankel) and zh2devalloc (local=1, Bessel) */
static void heval(cplx zk, int nt, const cplx *zt, double rscale, int nterm, const cplx *zc,
                  const cplx *mp, cplx *pot, cplx *grad, int ifpgh, int local) {
  int ifder = ifpgh > 1;
  cplx *f = (cplx *)calloc(nterm + 2, sizeof(cplx)), *fd = (cplx *)calloc(nterm + 2, sizeof(cplx));
  cplx *eis = (cplx *)malloc(sizeof(cplx) * (2 * nterm + 1));
  cplx *E = eis + nterm;
  const cplx *M = mp + nterm;
  E[0] = 1;
  for (int i = 0; i < nt; i++) {
    cplx zr, ei;
    o_zcart2polar(&zt[2 * i], zc, &zr, &ei);
    for (int m = 1; m <= nterm; m++) E[m] = E[m - 1] * ei;
    for (int m = 1; m <= nterm; m++) E[-m] = 1.0 / E[m];
    cplx z = zr * zk;
    if (local) jbes_c(nterm, z, rscale, f, ifder, fd);
    else h2dall_c(nterm, z, rscale, f, ifder, fd);
    cplx vr1 = 0, vr2 = 0, ve1 = 0, ve2 = 0;
    if (ifpgh > 1) {
      vr1 = (zt[2 * i] - zc[0]) / zr; vr2 = (zt[2 * i + 1] - zc[1]) / zr;
      ve1 = -vr2; ve2 = vr1;
    }
    for (int m = 0; m <= nterm; m++) {
      pot[i] += M[m] * f[m] * E[m];
      if (ifpgh > 1) {
        cplx dr = E[m] * fd[m] * zk, dth = f[m] * (I * (double)m) * E[m];
        grad[2 * i] += M[m] * (dr * vr1 + dth * ve1 / zr);
        grad[2 * i + 1] += M[m] * (dr * vr2 + dth * ve2 / zr);
      }
    }
    for (int m = -nterm; m <= -1; m++) {
      pot[i] += M[m] * isg(m) * f[-m] * E[m];
      if (ifpgh > 1) {
        cplx dr = E[m] * fd[-m] * zk, dth = f[-m] * (I * (double)m) * E[m];
        grad[2 * i] += isg(m) * M[m] * (dr * vr1 + dth * ve1 / zr);
        grad[2 * i + 1] += isg(m) * M[m] * (dr * vr2 + dth * ve2 / zr);
      }
    }
  }
  free(f); free(fd); free(eis);
}

/* zh2dmploc: mp at zc2 -> loc at zc1, same rscale/nterm */
static void hmploc(cplx zk, const cplx *zc1, const cplx *zc2, double rscale, int nterm, cplx *loc,
                   const cplx *mp) {
  cplx rz, ez;
  o_zcart2polar(zc1, zc2, &rz, &ez);
  int n2 = 2 * nterm;
  cplx *ezs = (cplx *)malloc(sizeof(cplx) * (2 * n2 + 1)), *E = ezs + n2;
  E[0] = 1;
  for (int m = 1; m <= n2; m++) E[m] = E[m - 1] * ez;
  for (int m = 1; m <= n2; m++) E[-m] = 1.0 / E[m];
  cplx *fh = (cplx *)calloc(n2 + 2, sizeof(cplx));
  h2dall_c(n2, rz * zk, rscale, fh, 0, NULL);
  double *rs = (double *)malloc(sizeof(double) * (n2 + 1));
  rs[0] = 1;
  for (int m = 1; m <= n2; m++) rs[m] = rs[m - 1] * rscale;
  cplx *L = loc + nterm;
  const cplx *M = mp + nterm;
  for (int m = -nterm; m <= nterm; m++)
    for (int n = -nterm; n <= nterm; n++) {
      cplx t = (n - m >= 0) ? fh[n - m] : fh[m - n] * isg(m - n);
      t = t * M[n] * E[n - m];
      t = t * rs[abs(m)] * rs[abs(n)] / rs[abs(m - n)];
      L[m] += t;
    }
  free(ezs); free(fh); free(rs);
}

/* zh2dlocloc: loc2 at zc2 -> loc1 at zc1 */
static void hlocloc(cplx zk, const cplx *zc1, const cplx *zc2, double rs1, double rs2, int n1,
                    int n2, cplx *loc1, const cplx *loc2) {
  int nt = n1 + n2;
  cplx rz, ez;
  o_zcart2polar(zc1, zc2, &rz, &ez);
  cplx *ezs = (cplx *)malloc(sizeof(cplx) * (2 * nt + 1)), *E = ezs + nt;
  E[0] = 1;
  for (int m = 1; m <= nt; m++) E[m] = E[m - 1] * ez;
  for (int m = 1; m <= nt; m++) E[-m] = 1.0 / E[m];
  cplx *fj = (cplx *)calloc(nt + 2, sizeof(cplx));
  jbes_c(nt, rz * zk, rs1, fj, 0, NULL);
  double *r1 = (double *)malloc(sizeof(double) * (nt + 1)), *r2 = (double *)malloc(sizeof(double) * (nt + 1));
  r1[0] = 1; r2[0] = 1;
  for (int m = 1; m <= nt; m++) { r1[m] = r1[m - 1] * rs1; r2[m] = r2[m - 1] * rs2; }
  cplx *A = loc1 + n1;
  const cplx *B = loc2 + n2;
  for (int m = -n1; m <= n1; m++)
    for (int n = -n2; n <= n2; n++) {
      double rfrac = r1[abs(m)] * r1[abs(m - n)] / r2[abs(n)];
      cplx t = (n - m >= 0) ? fj[n - m] * rfrac : isg(n - m) * fj[m - n] * rfrac;
      A[m] += B[n] * t * E[n - m];
    }
  free(ezs); free(fj); free(r1); free(r2);
}

/* zh2dmpmp: mp2 at zc2 -> mp1 at zc1 */
static void hmpmp(cplx zk, const cplx *zc1, const cplx *zc2, double rs1, double rs2, int n1,
                  int n2, cplx *mp1, const cplx *mp2) {
  int nt = n1 + n2;
  cplx rz, ez;
  o_zcart2polar(zc1, zc2, &rz, &ez);
  cplx *ezs = (cplx *)malloc(sizeof(cplx) * (2 * nt + 1)), *E = ezs + nt;
  E[0] = 1;
  for (int m = 1; m <= nt; m++) E[m] = E[m - 1] * ez;
  for (int m = 1; m <= nt; m++) E[-m] = 1.0 / E[m];
  cplx *fj = (cplx *)calloc(nt + 2, sizeof(cplx));
  jbes_c(nt, rz * zk, rs1, fj, 0, NULL);
  double *r1 = (double *)malloc(sizeof(double) * (nt + 1)), *r2 = (double *)malloc(sizeof(double) * (nt + 1));
  r1[0] = 1; r2[0] = 1;
  for (int m = 1; m <= nt; m++) { r1[m] = r1[m - 1] * rs1; r2[m] = r2[m - 1] * rs2; }
  cplx *A = mp1 + n1;
  const cplx *B = mp2 + n2;
  for (int m = -n1; m <= n1; m++)
    for (int n = -n2; n <= n2; n++) {
      double rfrac = r2[abs(n)] * r1[abs(m - n)] / r1[abs(m)];
      cplx t = (m - n >= 0) ? fj[m - n] * rfrac : isg(n - m) * fj[n - m] * rfrac;
      A[m] += t * B[n] * E[n - m] * isg(m + n);
    }
  free(ezs); free(fj); free(r1); free(r2);
}

int o_zhfmm2d(double eps, const double *zk_, int ns, const double *zsrc, int ifcharge,
              const double *charge, int ifdipole, const double *dipstr, const double *dipvec,
              double *pot, double *grad, int nt, const double *ztarg, int ifpgh, int isep,
              int ifprint) {
  (void)ifprint;
  cplx zk = zk_[0] + I * zk_[1];
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
  double pi = 4 * atan(1.0);
  double *rscales = (double *)malloc(sizeof(double) * (nlev + 1));
  int *nterms = (int *)malloc(sizeof(int) * (nlev + 1));
  for (int i = 0; i <= nlev; i++) {
    double a = cabs(zk * t->boxsize[i] / (2.0 * pi));
    rscales[i] = a < 1.0 ? a : 1.0;
    nterms[i] = o_h2dterms(t->boxsize[i], creal(zk), cimag(zk), eps, isep);
  }
  /* expansion storage per box, sized by its level */
  size_t *off = (size_t *)malloc(sizeof(size_t) * nb);
  size_t tot = 0;
  for (int l = 0; l <= nlev; l++)
    for (int b = t->laddr[2 * l]; b <= t->laddr[2 * l + 1]; b++) {
      off[b] = tot;
      tot += 2 * nterms[l] + 1;
    }
  cplx *mp = (cplx *)calloc(tot, sizeof(cplx)), *loc = (cplx *)calloc(tot, sizeof(cplx));
  cplx *potsort = (cplx *)calloc(nt, sizeof(cplx)), *gradsort = (cplx *)calloc(2 * (size_t)nt, sizeof(cplx));
  const int *se_s = S.isrcse, *se_t = S.itargse;
#define NS(b) (se_s[2 * (b) + 1] - se_s[2 * (b)] + 1)
#define NT(b) (se_t[2 * (b) + 1] - se_t[2 * (b)] + 1)
  for (int ilev = 1; ilev <= nlev; ilev++) {
#pragma omp parallel for schedule(dynamic)
    for (int ib = t->laddr[2 * ilev]; ib <= t->laddr[2 * ilev + 1]; ib++) {
      int s = se_s[2 * ib];
      if (t->nchild[ib] == 0 && NS(ib) > 0)
        hform(zk, rscales[ilev], &S.zsrcsort[2 * s], NS(ib), &S.chargesort[s], &S.dipstrsort[s],
              &S.dipvecsort[2 * s], &S.zcsrc[2 * ib], nterms[ilev], mp + off[ib], ifcharge,
              ifdipole, 0);
    }
  }
  for (int ilev = nlev - 1; ilev >= 1; ilev--) {
#pragma omp parallel for schedule(dynamic)
    for (int ib = t->laddr[2 * ilev]; ib <= t->laddr[2 * ilev + 1]; ib++)
      if (t->nchild[ib] > 0 && NS(ib) > 0)
        for (int j = 0; j < t->nchild[ib]; j++) {
          int jb = t->ichild[ib * 4 + j];
          if (NS(jb) > 0)
            hmpmp(zk, &S.zcsrc[2 * ib], &S.zcsrc[2 * jb], rscales[ilev], rscales[ilev + 1],
                  nterms[ilev], nterms[ilev + 1], mp + off[ib], mp + off[jb]);
        }
  }
#pragma omp parallel for schedule(dynamic)
  for (int ib = 0; ib < nb; ib++) {
    int s = se_t[2 * ib];
    if (NT(ib) > 0 && L->nlist[0][ib] > 0 && t->nchild[ib] == 0)
      for (int il = 0; il < L->nlist[0][ib]; il++) {
        int jb = L->list[0][(size_t)ib * L->mnlist[0] + il];
        int js = se_s[2 * jb];
        if (NS(jb) > 0)
          o_zh2devaldirect(zk_, NT(ib), (const double *)&S.ztargsort[2 * s], NS(jb),
                           (const double *)&S.zsrcsort[2 * js], (const double *)&S.chargesort[js],
                           (const double *)&S.dipstrsort[js], (const double *)&S.dipvecsort[2 * js],
                           ifcharge, (double *)&potsort[s], (double *)&gradsort[2 * s], ifdipole,
                           ifpgh);
      }
  }
#pragma omp parallel for schedule(dynamic)
  for (int ib = 0; ib < nb; ib++) {
    int lev = t->ilevel[ib];
    if (NT(ib) > 0 && L->nlist[1][ib] > 0)
      for (int il = 0; il < L->nlist[1][ib]; il++) {
        int jb = L->list[1][(size_t)ib * L->mnlist[1] + il];
        if (NS(jb) > 0)
          hmploc(zk, &S.zctarg[2 * ib], &S.zcsrc[2 * jb], rscales[lev], nterms[lev],
                 loc + off[ib], mp + off[jb]);
      }
  }
#pragma omp parallel for schedule(dynamic)
  for (int ib = 0; ib < nb; ib++) {
    int s = se_t[2 * ib];
    if (NT(ib) > 0 && t->nchild[ib] == 0 && L->nlist[2][ib] > 0)
      for (int il = 0; il < L->nlist[2][ib]; il++) {
        int jb = L->list[2][(size_t)ib * L->mnlist[2] + il];
        if (NS(jb) > 0) {
          int lev = t->ilevel[jb];
          heval(zk, NT(ib), &S.ztargsort[2 * s], rscales[lev], nterms[lev], &S.zcsrc[2 * jb],
                mp + off[jb], &potsort[s], &gradsort[2 * s], ifpgh, 0);
        }
      }
  }
#pragma omp parallel for schedule(dynamic)
  for (int ib = 0; ib < nb; ib++) {
    int lev = t->ilevel[ib];
    if (NT(ib) > 0 && L->nlist[3][ib] > 0)
      for (int il = 0; il < L->nlist[3][ib]; il++) {
        int jb = L->list[3][(size_t)ib * L->mnlist[3] + il];
        int js = se_s[2 * jb];
        if (NS(jb) > 0)
          hform(zk, rscales[lev], &S.zsrcsort[2 * js], NS(jb), &S.chargesort[js],
                &S.dipstrsort[js], &S.dipvecsort[2 * js], &S.zctarg[2 * ib], nterms[lev],
                loc + off[ib], ifcharge, ifdipole, 1);
      }
  }
  for (int ilev = 1; ilev <= nlev - 1; ilev++) {
#pragma omp parallel for schedule(dynamic)
    for (int ib = t->laddr[2 * ilev]; ib <= t->laddr[2 * ilev + 1]; ib++)
      if (NT(ib) > 0 && (L->nlist[1][ib] > 0 || L->nlist[3][ib] > 0))
        for (int j = 0; j < t->nchild[ib]; j++) {
          int jb = t->ichild[ib * 4 + j];
          if (NT(jb) > 0)
            hlocloc(zk, &S.zctarg[2 * jb], &S.zctarg[2 * ib], rscales[ilev + 1], rscales[ilev],
                    nterms[ilev + 1], nterms[ilev], loc + off[jb], loc + off[ib]);
        }
  }
#pragma omp parallel for schedule(dynamic)
  for (int ib = 0; ib < nb; ib++) {
    int s = se_t[2 * ib];
    if (t->nchild[ib] == 0 && NT(ib) > 0) {
      int lev = t->ilevel[ib];
      heval(zk, NT(ib), &S.ztargsort[2 * s], rscales[lev], nterms[lev], &S.zctarg[2 * ib],
            loc + off[ib], &potsort[s], &gradsort[2 * s], ifpgh, 1);
    }
  }
  cplx *P_ = (cplx *)pot, *G_ = (cplx *)grad;
  for (int i = 0; i < nt; i++) {
    int j = S.itarg[i];
    P_[j] = potsort[i] * I / 4.0;
    if (ifpgh > 1) { G_[2 * j] = gradsort[2 * i] * I / 4.0; G_[2 * j + 1] = gradsort[2 * i + 1] * I / 4.0; }
  }
  free(rscales); free(nterms); free(off); free(mp); free(loc); free(potsort); free(gradsort);
  o2d_free(&S);
  return 0;
}
