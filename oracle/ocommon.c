/*
 * Oracle (TEST INFRASTRUCTURE ONLY): driver set-up shared by the 2D FMMs.
 * Follows zlfmm2d.f:70-200 (identical in zhfmm2d.f:73-195): real parts ->
 * tree -> pts_tree_sort of targets and sources -> reorder -> complex box
 * centres (real centre + i * mean of the imaginary parts of the box's points).
 */
#include <stdlib.h>
#include <string.h>
#include "ocommon.h"

int o2d_setup(int ns, const double *zsrc, int ifcharge, const double *charge, int ifdipole,
              const double *dipstr, const double *dipvec, int nt, const double *ztarg,
              int idivflag, int ndiv, int isep, o2d_state *S) {
  memset(S, 0, sizeof(*S));
  const cplx *zs = (const cplx *)zsrc, *zt = (const cplx *)ztarg;
  double *src = (double *)malloc(sizeof(double) * 2 * ns);
  double *targ = (double *)malloc(sizeof(double) * 2 * nt);
  for (int i = 0; i < 2 * ns; i++) src[i] = creal(zs[i]);
  for (int i = 0; i < 2 * nt; i++) targ[i] = creal(zt[i]);
  int rc = otree_build(2, src, ns, targ, nt, idivflag, ndiv, 0, 51, isep, 0, &S->t);
  if (rc) { free(src); free(targ); return rc; }
  int nb = S->t.nboxes;
  S->ns = ns; S->nt = nt;
  S->isrc = (int *)malloc(sizeof(int) * ns);
  S->itarg = (int *)malloc(sizeof(int) * nt);
  S->isrcse = (int *)malloc(sizeof(int) * 2 * nb);
  S->itargse = (int *)malloc(sizeof(int) * 2 * nb);
  otree_sort(&S->t, nt, targ, S->itarg, S->itargse);
  otree_sort(&S->t, ns, src, S->isrc, S->isrcse);
  free(src); free(targ);
  S->zsrcsort = (cplx *)malloc(sizeof(cplx) * 2 * ns);
  S->ztargsort = (cplx *)malloc(sizeof(cplx) * 2 * nt);
  S->chargesort = (cplx *)calloc(ns, sizeof(cplx));
  S->dipstrsort = (cplx *)calloc(ns, sizeof(cplx));
  S->dipvecsort = (cplx *)calloc(2 * (size_t)ns, sizeof(cplx));
  for (int i = 0; i < ns; i++) {
    int j = S->isrc[i];
    S->zsrcsort[2 * i] = zs[2 * j];
    S->zsrcsort[2 * i + 1] = zs[2 * j + 1];
    if (ifcharge == 1) S->chargesort[i] = ((const cplx *)charge)[j];
    if (ifdipole == 1) {
      S->dipstrsort[i] = ((const cplx *)dipstr)[j];
      S->dipvecsort[2 * i] = ((const cplx *)dipvec)[2 * j];
      S->dipvecsort[2 * i + 1] = ((const cplx *)dipvec)[2 * j + 1];
    }
  }
  for (int i = 0; i < nt; i++) {
    int j = S->itarg[i];
    S->ztargsort[2 * i] = zt[2 * j];
    S->ztargsort[2 * i + 1] = zt[2 * j + 1];
  }
  S->zcsrc = (cplx *)calloc(2 * (size_t)nb, sizeof(cplx));
  S->zctarg = (cplx *)calloc(2 * (size_t)nb, sizeof(cplx));
  for (int ib = 0; ib < nb; ib++) {
    for (int pass = 0; pass < 2; pass++) {
      const int *se = pass ? S->itargse : S->isrcse;
      const cplx *pts = pass ? S->ztargsort : S->zsrcsort;
      cplx *zc = pass ? S->zctarg : S->zcsrc;
      int s = se[2 * ib], e = se[2 * ib + 1];
      if (s <= e) {
        double a0 = 0, a1 = 0;
        for (int i = s; i <= e; i++) { a0 += cimag(pts[2 * i]); a1 += cimag(pts[2 * i + 1]); }
        int npts = e - s + 1;
        a0 = a0 / npts;
        a1 = a1 / npts;
        zc[2 * ib] = S->t.centers[2 * ib] + I * a0;
        zc[2 * ib + 1] = S->t.centers[2 * ib + 1] + I * a1;
      }
    }
  }
  olists_build(&S->t, &S->L);
  return 0;
}

void o2d_free(o2d_state *S) {
  otree_free(&S->t);
  olists_free(&S->L);
  free(S->isrc); free(S->itarg); free(S->isrcse); free(S->itargse);
  free(S->zsrcsort); free(S->ztargsort); free(S->chargesort); free(S->dipstrsort);
  free(S->dipvecsort); free(S->zcsrc); free(S->zctarg);
  memset(S, 0, sizeof(*S));
}

/* ---- test helpers: tree summaries ---- */
int o_tree_info(int D, double eps_unused, int ndiv, const double *zsrc, int ns,
                const double *ztarg, int nt, int isep, int *nlevels, int *laddr_out,
                int laddr_cap, int *mnlist_out) {
  (void)eps_unused;
  double *src = (double *)malloc(sizeof(double) * D * ns);
  double *targ = (double *)malloc(sizeof(double) * D * nt);
  for (int i = 0; i < D * ns; i++) src[i] = zsrc[2 * i];
  for (int i = 0; i < D * nt; i++) targ[i] = ztarg[2 * i];
  otree t;
  int rc = otree_build(D, src, ns, targ, nt, 0, ndiv, 0, 51, isep, D == 3, &t);
  free(src); free(targ);
  if (rc) return -1;
  *nlevels = t.nlevels;
  for (int i = 0; i < 2 * (t.nlevels + 1) && i < laddr_cap; i++) laddr_out[i] = t.laddr[i];
  olists L;
  olists_build(&t, &L);
  for (int k = 0; k < 4; k++) mnlist_out[k] = L.mnlist[k];
  olists_free(&L);
  int nb = t.nboxes;
  otree_free(&t);
  return nb;
}

int o_tree_dump(int D, int ndiv, const double *zsrc, int ns, const double *ztarg, int nt,
                int isep, int *ilevel, int *iparent, int *nchild, int *ichild,
                double *centers, int *isrc, int *isrcse, int *itarg, int *itargse,
                int *nlist, int *list_flat, int list_cap) {
  double *src = (double *)malloc(sizeof(double) * D * ns);
  double *targ = (double *)malloc(sizeof(double) * D * nt);
  for (int i = 0; i < D * ns; i++) src[i] = zsrc[2 * i];
  for (int i = 0; i < D * nt; i++) targ[i] = ztarg[2 * i];
  otree t;
  int rc = otree_build(D, src, ns, targ, nt, 0, ndiv, 0, 51, isep, D == 3, &t);
  if (rc) { free(src); free(targ); return -1; }
  int nb = t.nboxes, NC = t.NC;
  memcpy(ilevel, t.ilevel, sizeof(int) * nb);
  memcpy(iparent, t.iparent, sizeof(int) * nb);
  memcpy(nchild, t.nchild, sizeof(int) * nb);
  memcpy(ichild, t.ichild, sizeof(int) * nb * NC);
  memcpy(centers, t.centers, sizeof(double) * nb * D);
  otree_sort(&t, ns, src, isrc, isrcse);
  otree_sort(&t, nt, targ, itarg, itargse);
  free(src); free(targ);
  olists L;
  olists_build(&t, &L);
  /* nlist: [4*nb]; list_flat: concatenation per list k, per box, of entries */
  size_t pos = 0;
  for (int k = 0; k < 4; k++)
    for (int b = 0; b < nb; b++) {
      nlist[k * nb + b] = L.nlist[k][b];
      for (int i = 0; i < L.nlist[k][b]; i++) {
        if ((int)pos < list_cap) list_flat[pos] = L.list[k][(size_t)b * L.mnlist[k] + i];
        pos++;
      }
    }
  olists_free(&L);
  otree_free(&t);
  return (int)pos;
}
