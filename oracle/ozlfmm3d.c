/*
 * Oracle (TEST INFRASTRUCTURE ONLY): 3D Laplace complex-coordinate FMM.
 *
 * Restates zfmm3d/src/laplace/zlfmm3d.f (driver :14-245 with the rescaling by
 * 1/boxsize(0), zlfmm3dmain :252-622, zl3devaldirect :628-683, zl3dformmp
 * :689-851, zl3dformloc :857-1005, zl3devalmp :1011-1131, zl3devalloc
 * :1137-1277, zl3dterms :1283-1321), the point-and-shoot translations of
 * zfmm3d/src/laplace/zl3dtrans.f (zl3dmpmp :1-101, zl3dmploc :107-216,
 * zl3dlocloc :222-321, the z-shifts :327-540, get_amat :546-570), the rotations
 * of zfmm3d/src/common/zrotate.f (z3dzrot :1-27, z3dzrotini :32-49, z3dyrotini
 * :55-88, z3dyrot :94-239), the Legendre recurrences of
 * zfmm3d/src/common/yrecursion.f (ylgndrini :694, zylgndrf :1220, zylgndr2sf
 * :1330) and ztoolbox.f (zsqrt :110-124, zcart2sph :132-160, myzylgndr2sf
 * :273-327).  The FFT of length 2p+1 in z3dyrot (FFTPACK zfftf between
 * ifftshift and fftshift) is a plain DFT here: the same sums.
 *
 * Expansions mp(n, m), 0 <= n <= p, -n <= m <= n, stored row-major as
 * mp[n*(2p+1) + m + p].
 */
#include "o3dcommon.h"

static int o_lndiv3d(double eps, int ns, int nt) {
  /* lndiv_fast.f:17-35 */
  if (eps >= 0.5e-0) return 300;
  if (eps >= 0.5e-1) return 300;
  if (eps >= 0.5e-2) return 300;
  if (eps >= 0.5e-3) return 300;
  if (eps >= 0.5e-6) return 1000;
  if (eps >= 0.5e-9) return 1000;
  if (eps >= 0.5e-12) return 1000;
  if (eps >= 0.5e-15) return 1000;
  return ns + nt;
}

int o_zl3dterms(double eps) {
  double z1 = 1.5, z2 = sqrt(3.0) / 2.0, jfun = z2, hfun = 1.0 / (z1 * z1);
  for (int j = 2; j <= 1000; j++) {
    hfun = hfun / z1;
    jfun = jfun * z2;
    if (jfun * hfun < eps) return j;
  }
  return 1;
}


void o_zl3devaldirect(int nt, const double *ztarg, int ns, const double *zsrc,
                      const double *charge, const double *dipstr, const double *dipvec,
                      int ifcharge, double *pot, double *grad, int ifdipole, int ifpgh) {
  const cplx *zt = (const cplx *)ztarg, *zs = (const cplx *)zsrc;
  const cplx *q = (const cplx *)charge, *ds = (const cplx *)dipstr, *dv = (const cplx *)dipvec;
  cplx *P_ = (cplx *)pot, *G_ = (cplx *)grad;
  double pi4 = 4 * PI;
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < nt; i++) {
    cplx p = 0, g[3] = {0, 0, 0};
    for (int j = 0; j < ns; j++) {
      cplx y[3];
      for (int d = 0; d < 3; d++) y[d] = zs[3 * j + d] - zt[3 * i + d];
      cplx rz = csqrt(y[0] * y[0] + y[1] * y[1] + y[2] * y[2]);
      if (!(cabs(rz) > F16)) continue;
      cplx r1 = 1.0 / (pi4 * rz), r3 = 1.0 / (pi4 * rz * rz * rz);
      if (ifcharge == 1) {
        p += q[j] * r1;
        if (ifpgh >= 2)
          for (int d = 0; d < 3; d++) g[d] += q[j] * y[d] * r3;
      }
      if (ifdipole == 1) {
        cplx dot = -(y[0] * dv[3 * j] + y[1] * dv[3 * j + 1] + y[2] * dv[3 * j + 2]);
        p -= ds[j] * dot * r3;
        if (ifpgh >= 2) {
          cplx r5 = rz * rz * rz * rz * rz;
          cplx dd = dot * 3.0 / (pi4 * r5);
          for (int d = 0; d < 3; d++) g[d] -= ds[j] * (dv[3 * j + d] * r3 + dd * y[d]);
        }
      }
    }
    P_[i] += p;
    if (ifpgh >= 2)
      for (int d = 0; d < 3; d++) G_[3 * i + d] += g[d];
  }
}

/* zl3dformmp (local = 0) / zl3dformloc (local = 1) */
static void form3(const cplx *zs, int npts, const cplx *q, const cplx *ds, const cplx *dv,
                  const cplx *zc, double rscale, int p, cplx *mp, int ifdipole, int local,
                  const rats *R) {
  int N = p;
  cplx *yl = (cplx *)calloc((size_t)(N + 1) * (N + 1), sizeof(cplx));
  cplx *dyl = (cplx *)calloc((size_t)(N + 1) * (N + 1), sizeof(cplx));
  cplx *rza = (cplx *)malloc(sizeof(cplx) * (2 * N + 4)), *RZ = rza + N + 1;
  cplx *eia = (cplx *)malloc(sizeof(cplx) * (2 * N + 1)), *E = eia + N;
  double s4 = 1.0 / sqrt(4 * PI);
  for (int i = 0; i < npts; i++) {
    cplx zr, ct, st, cp, sp, eip;
    zcart2sph(&zs[3 * i], zc, &zr, &ct, &st, &cp, &sp, &eip);
    cplx rz = zr / rscale;
    RZ[0] = 1;
    E[0] = 1;
    for (int n = 1; n <= N; n++) {
      RZ[n] = RZ[n - 1] * rz;
      E[n] = E[n - 1] * eip;
      E[-n] = 1.0 / E[n];
      if (local) RZ[-n] = 1.0 / RZ[n];
    }
    if (local) { RZ[N + 1] = RZ[N] * rz; RZ[-N - 1] = 1.0 / RZ[N + 1]; }
    if (ifdipole == 0) zylgndrf(N, ct, yl, R);
    else zylgndr2s(N, ct, 0, 0, yl, dyl, R);
    for (int n = 0; n <= N; n++)
      for (int m = 0; m <= n; m++) {
        double f = s4 * ((m & 1) ? -1.0 : 1.0) / (2 * n + 1.0);
        yl[n * (N + 1) + m] *= f;
        if (ifdipole == 1) dyl[n * (N + 1) + m] *= f;
      }
    for (int n = 0; n <= N; n++) {
      cplx rp = local ? RZ[-n - 1] : RZ[n];
      mp[MPI(p, n, 0)] += q[i] * rp * yl[n * (N + 1)];
      for (int m = 1; m <= n; m++) {
        cplx y = yl[n * (N + 1) + m];
        if (ifdipole == 1) y = st * y;
        mp[MPI(p, n, m)] += q[i] * rp * y * E[-m];
        mp[MPI(p, n, -m)] += q[i] * rp * y * E[m];
      }
    }
    if (ifdipole == 1) {
      cplx ezr[3] = {st * cp, st * sp, ct}, eth[3] = {ct * cp, ct * sp, -st}, eph[3] = {-sp, cp, 0};
      cplx dzr_ = 0, dth_ = 0, dph_ = 0;
      for (int d = 0; d < 3; d++) {
        dzr_ += dv[3 * i + d] * ezr[d];
        dth_ += dv[3 * i + d] * eth[d];
        dph_ += dv[3 * i + d] * eph[d];
      }
      cplx dthz = dth_ / zr, dphz = dph_ / zr;
      for (int n = 0; n <= N; n++) {
        cplx y0 = yl[n * (N + 1)], d0 = dyl[n * (N + 1)];
        cplx dzr, dth;
        if (!local) {
          dzr = n == 0 ? 0 : (double)n * RZ[n - 1] / rscale * y0;
          dth = -RZ[n] * d0 * st;
        } else {
          dzr = -(double)(n + 1) * y0 * RZ[-n - 1] / zr;
          dth = -d0 * st * RZ[-n - 1];
        }
        mp[MPI(p, n, 0)] -= ds[i] * (dzr_ * dzr + dthz * dth);
        for (int m = 1; m <= n; m++) {
          cplx y = yl[n * (N + 1) + m], dy = dyl[n * (N + 1) + m];
          for (int s = 0; s < 2; s++) {
            int mm = s ? -m : m;
            cplx e = E[-mm];
            cplx dz, dt, dp;
            if (!local) {
              dz = (double)n * RZ[n - 1] / rscale * y * st * e;
              dt = -RZ[n] * dy * e;
              dp = -I * (double)mm * RZ[n] * y * e;
            } else {
              dz = -(double)(n + 1) * y * st * e * RZ[-n - 1] / zr;
              dt = -dy * e * RZ[-n - 1];
              dp = -(double)mm * I * y * e * RZ[-n - 1];
            }
            mp[MPI(p, n, mm)] -= ds[i] * (dzr_ * dz + dthz * dt + dphz * dp);
          }
        }
      }
    }
  }
  free(yl); free(dyl); free(rza); free(eia);
}

/* zl3devalmp (local = 0) / zl3devalloc (local = 1) */
static void eval3(int nt, const cplx *zt, int p, const cplx *zc, double rscale, const cplx *mp,
                  cplx *pot, cplx *grad, int ifpgh, int local, const rats *R) {
  int N = p;
  cplx *yl = (cplx *)calloc((size_t)(N + 1) * (N + 1), sizeof(cplx));
  cplx *dyl = (cplx *)calloc((size_t)(N + 1) * (N + 1), sizeof(cplx));
  cplx *RZ = (cplx *)malloc(sizeof(cplx) * (N + 2));
  cplx *eia = (cplx *)malloc(sizeof(cplx) * (2 * N + 1)), *E = eia + N;
  double s4 = 1.0 / sqrt(4 * PI);
  for (int i = 0; i < nt; i++) {
    cplx zr, ct, st, cp, sp, eip;
    zcart2sph(&zt[3 * i], zc, &zr, &ct, &st, &cp, &sp, &eip);
    cplx rz = zr / rscale;
    RZ[0] = 1;
    E[0] = 1;
    for (int n = 1; n <= N; n++) {
      RZ[n] = RZ[n - 1] * rz;
      E[n] = E[n - 1] * eip;
      E[-n] = 1.0 / E[n];
    }
    RZ[N + 1] = RZ[N] * rz;
    cplx ezr[3], ethz[3], ephz[3];
    if (ifpgh == 1) {
      zylgndrf(N, ct, yl, R);
    } else {
      zylgndr2s(N, ct, 0, 0, yl, dyl, R);
      ezr[0] = st * cp; ezr[1] = st * sp; ezr[2] = ct;
      ethz[0] = ct * cp / zr; ethz[1] = ct * sp / zr; ethz[2] = -st / zr;
      ephz[0] = -sp / zr; ephz[1] = cp / zr; ephz[2] = 0;
    }
    for (int n = 0; n <= N; n++)
      for (int m = 0; m <= n; m++) {
        double f = s4 * ((m & 1) ? -1.0 : 1.0) / rscale;
        yl[n * (N + 1) + m] *= f;
        if (ifpgh >= 2) dyl[n * (N + 1) + m] *= f;
      }
    for (int n = 0; n <= N; n++) {
      cplx rfac = local ? RZ[n] : 1.0 / RZ[n + 1];
      pot[i] += mp[MPI(p, n, 0)] * yl[n * (N + 1)] * rfac;
      for (int m = 1; m <= n; m++) {
        cplx y = yl[n * (N + 1) + m];
        if (ifpgh >= 2) y = y * st;
        pot[i] += y * (mp[MPI(p, n, m)] * E[m] + mp[MPI(p, n, -m)] * E[-m]) * rfac;
      }
    }
    if (ifpgh >= 2) {
      for (int n = 0; n <= N; n++) {
        cplx y0 = yl[n * (N + 1)], d0 = dyl[n * (N + 1)];
        cplx dzr, dth;
        if (!local) {
          dzr = -(double)(n + 1) * y0 / RZ[n + 1] / zr;
          dth = -d0 * st / RZ[n + 1];
        } else {
          dzr = n == 0 ? 0 : (double)n * RZ[n - 1] / rscale * y0;
          dth = -RZ[n] * d0 * st;
        }
        for (int d = 0; d < 3; d++) grad[3 * i + d] += mp[MPI(p, n, 0)] * (dzr * ezr[d] + dth * ethz[d]);
        for (int m = 1; m <= n; m++) {
          cplx y = yl[n * (N + 1) + m], dy = dyl[n * (N + 1) + m];
          for (int s = 0; s < 2; s++) {
            int mm = s ? -m : m;
            cplx e = E[mm];
            cplx dz, dt, dp;
            if (!local) {
              dz = -(double)(n + 1) * y * st * e / RZ[n + 1] / zr;
              dt = -dy * e / RZ[n + 1];
              dp = (double)mm * I * y * e / RZ[n + 1];
            } else {
              dz = (double)n * RZ[n - 1] / rscale * y * st * e;
              dt = -RZ[n] * dy * e;
              dp = (double)mm * I * RZ[n] * y * e;
            }
            for (int d = 0; d < 3; d++)
              grad[3 * i + d] += mp[MPI(p, n, mm)] * (dz * ezr[d] + dt * ethz[d] + dp * ephz[d]);
          }
        }
      }
    }
  }
  free(yl); free(dyl); free(RZ); free(eia);
}

/* ---- axial shifts --------------------------------------------------------- */
#define AM(n, m) amat[(n) * (2 * nmax + 1) + (m) + nmax]
static void shift_sign(cplx zshift, int nmx, cplx *rz, double *yl) {
  if (cabs(csqrt(zshift * zshift) - zshift) > F16) {
    *rz = -zshift;
    for (int n = 0; n <= nmx; n++) yl[n] = sqrt(2 * n + 1.0) * ((n & 1) ? -1.0 : 1.0);
  } else {
    *rz = zshift;
    for (int n = 0; n <= nmx; n++) yl[n] = sqrt(2 * n + 1.0);
  }
}

static void mpmp_zshift(cplx zshift, int p0, const cplx *mp0, double rs0, int p, cplx *mp,
                        double rs, int nmax, const double *amat) {
  double s4 = sqrt(4 * PI);
  double *yl = (double *)malloc(sizeof(double) * (p + 1));
  cplx rz;
  shift_sign(zshift, p, &rz, yl);
  rz = rz / rs0;
  cplx *ra = (cplx *)malloc(sizeof(cplx) * (p + 1));
  ra[0] = 1;
  for (int n = 1; n <= p; n++) ra[n] = ra[n - 1] * rz;
  for (int j = 0; j <= p; j++) {
    double tj = s4 * (pow(rs0, j) / pow(rs, j));
    for (int k = -j; k <= j; k++)
      for (int n = 0; n <= j; n++) {
        int ak = k < 0 ? -k : k;
        if (ak <= j - n && j - n <= p0) {
          cplx t = mp0[MPI(p0, j - n, k)] * AM(n, 0) * AM(j - n, k) / AM(j, k);
          t = t * ra[n] * yl[n] / (2 * n + 1.0);
          mp[MPI(p, j, k)] += t * tj;
        }
      }
  }
  free(yl); free(ra);
}

static void mploc_zshift(cplx zshift, int p0, const cplx *mp0, double rs0, int p, cplx *loc,
                         double rs, int nmax, const double *amat) {
  (void)rs;
  double s4 = sqrt(4 * PI);
  int nn = p + p0;
  double *yl = (double *)malloc(sizeof(double) * (nn + 1));
  cplx rz;
  shift_sign(zshift, nn, &rz, yl);
  rz = rz / rs0;
  cplx *ra = (cplx *)malloc(sizeof(cplx) * (nn + 1));
  ra[0] = 1;
  for (int n = 1; n <= nn; n++) ra[n] = ra[n - 1] * rz;
  for (int j = 0; j <= p; j++) {
    cplx tj = s4 / rz / (2 * j + 1.0);
    for (int k = -j; k <= j; k++)
      for (int n = 0; n <= p0; n++) {
        int ak = k < 0 ? -k : k;
        if (ak <= n) {
          cplx t = mp0[MPI(p0, n, k)] * AM(n, k) * AM(j, k) / AM(j + n, 0);
          int e = n + k < 0 ? -(n + k) : n + k;
          t = t * ((e & 1) ? -1.0 : 1.0) / ra[n + j];
          loc[MPI(p, j, k)] += t * yl[n + j] * tj;
        }
      }
  }
  free(yl); free(ra);
}

static void locloc_zshift(cplx zshift, int p0, const cplx *loc0, double rs0, int p, cplx *loc,
                          double rs, int nmax, const double *amat) {
  double s4 = sqrt(4 * PI);
  double *yl = (double *)malloc(sizeof(double) * (p0 + 1));
  cplx rz;
  shift_sign(zshift, p0, &rz, yl);
  rz = rz / rs;
  cplx *ra = (cplx *)malloc(sizeof(cplx) * (p + p0 + 1));
  ra[0] = 1;
  for (int n = 1; n <= p + p0; n++) ra[n] = ra[n - 1] * rz;
  for (int j = 0; j <= p; j++) {
    double tj = s4 / (2 * j + 1.0);
    for (int k = -j; k <= j; k++)
      for (int n = j; n <= p0; n++) {
        cplx t = loc0[MPI(p0, n, k)] * (AM(n - j, 0) * AM(j, k) / AM(n, k));
        t = t * (((n + j) & 1) ? -1.0 : 1.0) * ra[n - j] * yl[n - j];
        t = t * (2 * n + 1.0) / (2 * (n - j) + 1.0);
        t = t * pow(rs, n + 1) / pow(rs0, n + 1);
        loc[MPI(p, j, k)] += t * tj;
      }
  }
  free(yl); free(ra);
}

/* kind 0 mpmp, 1 mploc, 2 locloc: point-and-shoot (zl3dtrans.f:1-321) */
static void translate3(int kind, const cplx *c0, int p0, const cplx *a0, double rs0,
                       const cplx *c, int p, cplx *out, double rs, int nmax, const double *amat,
                       const rats *R0, const rats *R) {
  size_t n0 = (size_t)(p0 + 1) * (2 * p0 + 1), n1 = (size_t)(p + 1) * (2 * p + 1);
  cplx *az = (cplx *)calloc(n0, sizeof(cplx)), *azy = (cplx *)calloc(n0, sizeof(cplx));
  cplx *bzy = (cplx *)calloc(n1, sizeof(cplx)), *bz = (cplx *)calloc(n1, sizeof(cplx));
  cplx *bn = (cplx *)calloc(n1, sizeof(cplx));
  cplx xc1[3], xc2[3], cb = 1, sb = 0, ca = 1, sa = 0;
  double e2 = cabs(c[1] - c0[1]);
  if (e2 <= F16) {
    for (int d = 0; d < 3; d++) xc1[d] = c[d] - c0[d];
    memcpy(az, a0, n0 * sizeof(cplx));
  } else {
    for (int d = 0; d < 3; d++) xc1[d] = c[d] - c0[d];
    cplx rxy = zsqrt_r(xc1[0] * xc1[0] + xc1[1] * xc1[1]);
    cb = -xc1[0] / rxy;
    sb = -xc1[1] / rxy;
    xc1[0] = -rxy;
    xc1[1] = 0;
    zrot(p0, a0, az, cb, sb);
  }
  double e1 = cabs(xc1[0]);
  if (e1 <= F16) {
    for (int d = 0; d < 3; d++) xc2[d] = xc1[d];
    memcpy(azy, az, n0 * sizeof(cplx));
  } else {
    cplx rxz = zsqrt_r(xc1[0] * xc1[0] + xc1[2] * xc1[2]);
    xc2[0] = 0; xc2[1] = 0; xc2[2] = rxz;
    ca = xc1[2] / rxz;
    sa = xc1[0] / rxz;
    yrot(p0, az, azy, ca, sa, R0);
  }
  cplx zshift = -xc2[2];
  if (kind == 0) mpmp_zshift(zshift, p0, azy, rs0, p, bzy, rs, nmax, amat);
  else if (kind == 1) mploc_zshift(zshift, p0, azy, rs0, p, bzy, rs, nmax, amat);
  else locloc_zshift(zshift, p0, azy, rs0, p, bzy, rs, nmax, amat);
  if (e1 <= F16) memcpy(bz, bzy, n1 * sizeof(cplx));
  else yrot(p, bzy, bz, ca, -sa, R);
  if (e2 <= F16) memcpy(bn, bz, n1 * sizeof(cplx));
  else zrot(p, bz, bn, cb, -sb);
  for (size_t i = 0; i < n1; i++) out[i] += bn[i];
  free(az); free(azy); free(bzy); free(bz); free(bn);
}

int o_zlfmm3d(double eps, int ns, const double *zsrc_, int ifcharge, const double *charge_,
              int ifdipole, const double *dipstr_, const double *dipvec_, double *pot_,
              double *grad_, int nt, const double *ztarg_, int ifpgh, int isep, int ifprint) {
  (void)ifprint;
  if (ifcharge < 0 || ifcharge > 1) ifcharge = 1;
  if (ifdipole < 0 || ifdipole > 1) ifdipole = 0;
  if (ifpgh < 0 || ifpgh > 2) ifpgh = 1;
  memset(pot_, 0, sizeof(double) * 2 * nt);
  memset(grad_, 0, sizeof(double) * 6 * nt);
  const cplx *zsrc = (const cplx *)zsrc_, *ztarg = (const cplx *)ztarg_;
  double *src = (double *)malloc(sizeof(double) * 3 * ns), *targ = (double *)malloc(sizeof(double) * 3 * nt);
  for (int i = 0; i < 3 * ns; i++) src[i] = creal(zsrc[i]);
  for (int i = 0; i < 3 * nt; i++) targ[i] = creal(ztarg[i]);
  int ndiv = o_lndiv3d(eps, ns, nt);
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
  /* rescale to the unit root box (zlfmm3d.f:187-200) */
  double b0 = t.boxsize[0], b0inv = 1.0 / b0, b0inv2 = b0inv * b0inv;
  for (int i = 0; i < 3 * ns; i++) zs[i] *= b0inv;
  for (int i = 0; i < 3 * nt; i++) zt[i] *= b0inv;
  if (ifcharge == 1) for (int i = 0; i < ns; i++) q[i] *= b0inv;
  if (ifdipole == 1) for (int i = 0; i < 3 * ns; i++) dv[i] *= b0inv2;
  for (int i = 0; i < 3 * nb; i++) { zcs[i] *= b0inv; zct[i] *= b0inv; }
  double *bsz = (double *)malloc(sizeof(double) * (nlev + 1)), *rsc = (double *)malloc(sizeof(double) * (nlev + 1));
  for (int l = 0; l <= nlev; l++) {
    bsz[l] = t.boxsize[l] * b0inv;
    rsc[l] = bsz[l] > 1 ? 1 : bsz[l];
  }
  int p = o_zl3dterms(eps);
  olists L;
  olists_build(&t, &L);
  int nmax = nlev > 0 ? 2 * p : p;
  double *amat = (double *)calloc((size_t)(nmax + 1) * (2 * nmax + 1), sizeof(double));
  {
    double *facts = (double *)malloc(sizeof(double) * (2 * nmax + 1));
    facts[0] = 1;
    for (int i = 1; i <= 2 * nmax; i++) facts[i] = sqrt(i + 0.0) * facts[i - 1];
    for (int n = 0; n <= nmax; n++) {
      double cst = ((n & 1) ? -1.0 : 1.0) * sqrt((2 * n + 1) * (1.0 / (4 * PI)));
      for (int m = -n; m <= n; m++) AM(n, m) = cst / facts[n - m] / facts[n + m];
    }
    free(facts);
  }
  rats R = rats_new(p);
  size_t ne = (size_t)(p + 1) * (2 * p + 1);
  cplx *mp = (cplx *)calloc(ne * nb, sizeof(cplx)), *loc = (cplx *)calloc(ne * nb, sizeof(cplx));
  cplx *ps = (cplx *)calloc(nt, sizeof(cplx)), *gs = (cplx *)calloc(3 * (size_t)nt, sizeof(cplx));
#define NS3(b) (isrcse[2 * (b) + 1] - isrcse[2 * (b)] + 1)
#define NT3(b) (itargse[2 * (b) + 1] - itargse[2 * (b)] + 1)
  for (int l = 1; l <= nlev; l++)
#pragma omp parallel for schedule(dynamic)
    for (int b = t.laddr[2 * l]; b <= t.laddr[2 * l + 1]; b++) {
      int s0 = isrcse[2 * b];
      if (t.nchild[b] == 0 && NS3(b) > 0)
        form3(&zs[3 * s0], NS3(b), &q[s0], &dsv[s0], &dv[3 * s0], &zcs[3 * b], rsc[l], p,
              mp + ne * b, ifdipole, 0, &R);
    }
  for (int l = nlev - 1; l >= 1; l--)
#pragma omp parallel for schedule(dynamic)
    for (int b = t.laddr[2 * l]; b <= t.laddr[2 * l + 1]; b++)
      if (t.nchild[b] > 0 && NS3(b) > 0)
        for (int c = 0; c < t.nchild[b]; c++) {
          int jb = t.ichild[8 * b + c];
          if (NS3(jb) > 0)
            translate3(0, &zcs[3 * jb], p, mp + ne * jb, rsc[l + 1], &zcs[3 * b], p, mp + ne * b,
                       rsc[l], nmax, amat, &R, &R);
        }
#pragma omp parallel for schedule(dynamic)
  for (int b = 0; b < nb; b++) {
    int s0 = itargse[2 * b];
    if (NT3(b) > 0 && L.nlist[0][b] > 0 && t.nchild[b] == 0)
      for (int i = 0; i < L.nlist[0][b]; i++) {
        int jb = L.list[0][(size_t)b * L.mnlist[0] + i];
        int j0 = isrcse[2 * jb];
        if (NS3(jb) > 0)
          o_zl3devaldirect(NT3(b), (const double *)&zt[3 * s0], NS3(jb), (const double *)&zs[3 * j0],
                           (const double *)&q[j0], (const double *)&dsv[j0],
                           (const double *)&dv[3 * j0], ifcharge, (double *)&ps[s0],
                           (double *)&gs[3 * s0], ifdipole, ifpgh);
      }
  }
#pragma omp parallel for schedule(dynamic)
  for (int b = 0; b < nb; b++) {
    int l = t.ilevel[b];
    if (NT3(b) > 0 && L.nlist[1][b] > 0)
      for (int i = 0; i < L.nlist[1][b]; i++) {
        int jb = L.list[1][(size_t)b * L.mnlist[1] + i];
        if (NS3(jb) > 0)
          translate3(1, &zcs[3 * jb], p, mp + ne * jb, rsc[l], &zct[3 * b], p, loc + ne * b, rsc[l],
                     nmax, amat, &R, &R);
      }
  }
#pragma omp parallel for schedule(dynamic)
  for (int b = 0; b < nb; b++) {
    int s0 = itargse[2 * b];
    if (NT3(b) > 0 && t.nchild[b] == 0 && L.nlist[2][b] > 0)
      for (int i = 0; i < L.nlist[2][b]; i++) {
        int jb = L.list[2][(size_t)b * L.mnlist[2] + i];
        if (NS3(jb) > 0)
          eval3(NT3(b), &zt[3 * s0], p, &zcs[3 * jb], rsc[t.ilevel[jb]], mp + ne * jb, &ps[s0],
                &gs[3 * s0], ifpgh, 0, &R);
      }
  }
#pragma omp parallel for schedule(dynamic)
  for (int b = 0; b < nb; b++) {
    int l = t.ilevel[b];
    if (NT3(b) > 0 && L.nlist[3][b] > 0)
      for (int i = 0; i < L.nlist[3][b]; i++) {
        int jb = L.list[3][(size_t)b * L.mnlist[3] + i];
        int j0 = isrcse[2 * jb];
        if (NS3(jb) > 0)
          form3(&zs[3 * j0], NS3(jb), &q[j0], &dsv[j0], &dv[3 * j0], &zct[3 * b], rsc[l], p,
                loc + ne * b, ifdipole, 1, &R);
      }
  }
  for (int l = 1; l <= nlev - 1; l++)
#pragma omp parallel for schedule(dynamic)
    for (int b = t.laddr[2 * l]; b <= t.laddr[2 * l + 1]; b++)
      if (NT3(b) > 0 && (L.nlist[1][b] > 0 || L.nlist[3][b] > 0))
        for (int c = 0; c < t.nchild[b]; c++) {
          int jb = t.ichild[8 * b + c];
          if (NT3(jb) > 0)
            translate3(2, &zct[3 * b], p, loc + ne * b, rsc[l], &zct[3 * jb], p, loc + ne * jb,
                       rsc[l + 1], nmax, amat, &R, &R);
        }
#pragma omp parallel for schedule(dynamic)
  for (int b = 0; b < nb; b++) {
    int s0 = itargse[2 * b];
    if (t.nchild[b] == 0 && NT3(b) > 0)
      eval3(NT3(b), &zt[3 * s0], p, &zct[3 * b], rsc[t.ilevel[b]], loc + ne * b, &ps[s0],
            &gs[3 * s0], ifpgh, 1, &R);
  }
  cplx *P_ = (cplx *)pot_, *G_ = (cplx *)grad_;
  for (int i = 0; i < nt; i++) {
    int j = itarg[i];
    P_[j] = ps[i];
    if (ifpgh >= 2)
      for (int d = 0; d < 3; d++) G_[3 * j + d] = gs[3 * i + d] * b0inv;
  }
  rats_free(&R);
  free(amat); free(mp); free(loc); free(ps); free(gs); free(bsz); free(rsc);
  free(zs); free(zt); free(q); free(dsv); free(dv); free(zcs); free(zct);
  free(isrc); free(itarg); free(isrcse); free(itargse);
  olists_free(&L);
  otree_free(&t);
  return 0;
}
