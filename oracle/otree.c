/*
 * Oracle (TEST INFRASTRUCTURE ONLY): adaptive level-restricted quad/oct tree
 * on the real parts of the coordinates, and the U/V/W/X interaction lists.
 *
 * Restates, for D = 2 and D = 3 in one code:
 *   pts_tree_mem / pts_tree_build   zfmm2d/src/common/pts_tree2d.f:34-665
 *                                   zfmm3d/src/common/pts_tree3d.f:41-907
 *   sort_pts_to_children            pts_tree2d.f:669-764, pts_tree3d.f:913-1102
 *   pts_tree_fix_lr                 pts_tree2d.f:768-1078
 *   pts_tree_reorg                  pts_tree2d.f:1083-1232
 *   pts_tree_sort                   pts_tree2d.f:1239-1264
 *   tree_refine_boxes(_flag)        zfmm2d/src/common/tree_routs2d.f:9-56, 337-391
 *   computecoll                     tree_routs2d.f:100-212
 *   updateflags                     tree_routs2d.f:218-329
 *   computemnlists / computelists   tree_routs2d.f:463-746 (3D: tree_routs3d.f:414-712)
 *
 * Child c (0-based) of a box has bit 0 set when x >= centre_x, bit 1 for y,
 * bit 2 for z (the reference's 1..4 / 1..8 numbering minus one).  The
 * reference's partition (y then x; z, y then x) is stable in each pass, so the
 * net effect is a stable partition by child index, which is what
 * sort_children below does.
 *
 * Floating-point literals follow the Fortran source: "1.05" without d0 is a
 * REAL*4 constant (computecoll, and the colleague update inside fix_lr, where
 * "isep*1.05" is even evaluated in single precision).
 */
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include "oracle.h"

typedef struct {
  int D, NC, cap, n;
  int *ilevel, *iparent, *nchild, *ichild, *iflag;
  double *centers;
} boxes_t;

static void bx_reserve(boxes_t *B, int need) {
  if (need <= B->cap) return;
  int nc = B->cap ? B->cap : 64;
  while (nc < need) nc *= 2;
  B->ilevel = (int *)realloc(B->ilevel, sizeof(int) * nc);
  B->iparent = (int *)realloc(B->iparent, sizeof(int) * nc);
  B->nchild = (int *)realloc(B->nchild, sizeof(int) * nc);
  B->iflag = (int *)realloc(B->iflag, sizeof(int) * nc);
  B->ichild = (int *)realloc(B->ichild, sizeof(int) * nc * B->NC);
  B->centers = (double *)realloc(B->centers, sizeof(double) * nc * B->D);
  B->cap = nc;
}

/* children of box ib: centre offsets of +-bs/2 per axis (tree_routs2d.f:30-45) */
static void make_children(boxes_t *B, int ib, int first, double bs, int lev, int flagmode) {
  int D = B->D, NC = B->NC;
  B->nchild[ib] = NC;
  for (int c = 0; c < NC; c++) {
    int jb = first + c;
    for (int d = 0; d < D; d++) {
      double s = ((c >> d) & 1) ? 1.0 : -1.0;
      B->centers[jb * D + d] = B->centers[ib * D + d] + (s * bs) / 2;
    }
    B->iparent[jb] = ib;
    B->nchild[jb] = 0;
    for (int l = 0; l < NC; l++) B->ichild[jb * NC + l] = -1;
    B->ichild[ib * NC + c] = jb;
    B->ilevel[jb] = lev;
    if (flagmode) {
      if (B->iflag[ib] == 1) B->iflag[jb] = 3;
      else if (B->iflag[ib] == 2) B->iflag[jb] = 0;
    } else {
      B->iflag[jb] = 0;
    }
  }
}

/* stable partition of the box's point segment into its children */
static void sort_children(const boxes_t *B, int ib, const double *xs, int *idx, int *se,
                          int *tmp) {
  int D = B->D, NC = B->NC;
  int s = se[2 * ib], e = se[2 * ib + 1];
  int cnt[8] = {0};
  int n = e - s + 1;
  for (int k = 0; k < n; k++) {
    int p = idx[s + k], c = 0;
    for (int d = 0; d < D; d++)
      if (!(xs[(size_t)p * D + d] - B->centers[ib * D + d] < 0)) c |= 1 << d;
    cnt[c]++;
  }
  int off[8];
  off[0] = 0;
  for (int c = 1; c < NC; c++) off[c] = off[c - 1] + cnt[c - 1];
  int pos[8];
  memcpy(pos, off, sizeof(pos));
  for (int k = 0; k < n; k++) {
    int p = idx[s + k], c = 0;
    for (int d = 0; d < D; d++)
      if (!(xs[(size_t)p * D + d] - B->centers[ib * D + d] < 0)) c |= 1 << d;
    tmp[pos[c]++] = p;
  }
  for (int k = 0; k < n; k++) idx[s + k] = tmp[k];
  for (int c = 0; c < NC; c++) {
    int jb = B->ichild[ib * NC + c];
    se[2 * jb] = s + off[c];
    se[2 * jb + 1] = s + off[c] + cnt[c] - 1;
  }
}

static int within(const double *a, const double *b, int D, double tol) {
  for (int d = 0; d < D; d++)
    if (!(fabs(a[d] - b[d]) <= tol)) return 0;
  return 1;
}

static void computecoll(const boxes_t *B, int nlevels, const int *laddr, const double *bsz,
                        int isep, int mnbors, int *ncoll, int *coll) {
  int D = B->D, NC = B->NC;
  for (int i = 0; i < B->n; i++) {
    ncoll[i] = 0;
    for (int j = 0; j < mnbors; j++) coll[(size_t)i * mnbors + j] = -1;
  }
  ncoll[0] = 1;
  coll[0] = 0;
  for (int ilev = 1; ilev <= nlevels; ilev++) {
    double tol = (double)1.05f * bsz[ilev] * (double)isep;
#pragma omp parallel for schedule(static)
    for (int ib = laddr[2 * ilev]; ib <= laddr[2 * ilev + 1]; ib++) {
      int dad = B->iparent[ib];
      for (int i = 0; i < ncoll[dad]; i++) {
        int jb = coll[(size_t)dad * mnbors + i];
        for (int c = 0; c < NC; c++) {
          int kb = B->ichild[jb * NC + c];
          if (kb >= 0 && within(&B->centers[kb * D], &B->centers[ib * D], D, tol)) {
            coll[(size_t)ib * mnbors + ncoll[ib]] = kb;
            ncoll[ib]++;
          }
        }
      }
    }
  }
}

/* tree_refine_boxes_flag over boxes [lo,hi]: subdivide iflag>0 boxes, children appended */
static void refine_flag_range(boxes_t *B, int lo, int hi, double bs, int ilev) {
  int nref = 0;
  for (int ib = lo; ib <= hi; ib++)
    if (B->iflag[ib] > 0) nref++;
  if (nref == 0) return;
  bx_reserve(B, B->n + nref * B->NC);
  int r = 0;
  for (int ib = lo; ib <= hi; ib++)
    if (B->iflag[ib] > 0) {
      make_children(B, ib, B->n + r * B->NC, bs, ilev + 1, 1);
      r++;
    }
  B->n += nref * B->NC;
}

static void reorg(boxes_t *B, int nlevels, int *laddr, const int *laddrtail) {
  int n = B->n, D = B->D, NC = B->NC;
  boxes_t T = {0};
  T.D = D;
  T.NC = NC;
  bx_reserve(&T, n);
  memcpy(T.ilevel, B->ilevel, sizeof(int) * n);
  memcpy(T.iparent, B->iparent, sizeof(int) * n);
  memcpy(T.nchild, B->nchild, sizeof(int) * n);
  memcpy(T.iflag, B->iflag, sizeof(int) * n);
  memcpy(T.ichild, B->ichild, sizeof(int) * n * NC);
  memcpy(T.centers, B->centers, sizeof(double) * n * D);
  int *map = (int *)malloc(sizeof(int) * n);
  for (int ilev = 0; ilev <= 1 && ilev <= nlevels; ilev++)
    for (int ib = laddr[2 * ilev]; ib <= laddr[2 * ilev + 1]; ib++) map[ib] = ib;
  int cur = laddr[4];
  for (int ilev = 2; ilev <= nlevels; ilev++) {
    int lo_old = laddr[2 * ilev], hi_old = laddr[2 * ilev + 1];
    laddr[2 * ilev] = cur;
    for (int pass = 0; pass < 2; pass++) {
      int lo = pass ? laddrtail[2 * ilev] : lo_old;
      int hi = pass ? laddrtail[2 * ilev + 1] : hi_old;
      for (int ib = lo; ib <= hi; ib++) {
        B->ilevel[cur] = T.ilevel[ib];
        B->nchild[cur] = T.nchild[ib];
        for (int d = 0; d < D; d++) B->centers[cur * D + d] = T.centers[ib * D + d];
        B->iflag[cur] = T.iflag[ib];
        map[ib] = cur;
        cur++;
      }
    }
    laddr[2 * ilev + 1] = cur - 1;
  }
  for (int ib = 0; ib < n; ib++) {
    int nb = map[ib];
    B->iparent[nb] = T.iparent[ib] < 0 ? -1 : map[T.iparent[ib]];
    for (int c = 0; c < NC; c++) {
      int ch = T.ichild[ib * NC + c];
      B->ichild[nb * NC + c] = ch < 0 ? -1 : map[ch];
    }
  }
  free(map);
  free(T.ilevel); free(T.iparent); free(T.nchild); free(T.iflag);
  free(T.ichild); free(T.centers);
}

static void updateflags(boxes_t *B, int curlev, int lo, int hi, const double *bsz, int isep,
                        int mnbors, const int *ncoll, const int *coll) {
  int D = B->D, NC = B->NC;
  double distest = 1.05 * (bsz[curlev] + bsz[curlev + 1]) / 2.0;
  distest = distest * isep;
  for (int ib = lo; ib <= hi; ib++) {
    if (B->iflag[ib] != 3) continue;
    B->iflag[ib] = 0;
    for (int i = 0; i < ncoll[ib] && B->iflag[ib] == 0; i++) {
      int jb = coll[(size_t)ib * mnbors + i];
      for (int c = 0; c < NC; c++) {
        int kb = B->ichild[jb * NC + c];
        if (kb >= 0 && B->nchild[kb] > 0 &&
            within(&B->centers[kb * D], &B->centers[ib * D], D, distest)) {
          B->iflag[ib] = 1;
          break;
        }
      }
    }
  }
}

static void fix_lr(boxes_t *B, int nlevels, int *laddr, const double *bsz, int isep,
                   int quirk, int mnbors, int **ncollp, int **collp) {
  int D = B->D, NC = B->NC;
  int *ncoll = *ncollp, *coll = *collp;
  for (int i = 0; i < B->n; i++) B->iflag[i] = 0;
  for (int ilev = nlevels; ilev >= 2; ilev--) {
    double distest = 1.05 * (bsz[ilev - 1] + bsz[ilev - 2]) / 2.0;
    distest = distest * isep;
    for (int ib = laddr[2 * ilev]; ib <= laddr[2 * ilev + 1]; ib++) {
      int idad = B->iparent[ib], igd = B->iparent[idad];
      for (int i = 0; i < ncoll[igd]; i++) {
        int jb = coll[(size_t)igd * mnbors + i];
        if (B->nchild[jb] == 0 && B->iflag[jb] == 0 &&
            within(&B->centers[jb * D], &B->centers[idad * D], D, distest))
          B->iflag[jb] = 1;
      }
    }
  }
  for (int ilev = nlevels; ilev >= 1; ilev--) {
    double distest = 1.05 * (bsz[ilev] + bsz[ilev - 1]) / 2.0;
    if (!quirk) distest = distest * isep;
    for (int ib = laddr[2 * ilev]; ib <= laddr[2 * ilev + 1]; ib++) {
      if (B->iflag[ib] != 1 && B->iflag[ib] != 2) continue;
      int idad = B->iparent[ib];
      for (int i = 0; i < ncoll[idad]; i++) {
        int jb = coll[(size_t)idad * mnbors + i];
        if (B->nchild[jb] == 0 && B->iflag[jb] == 0 &&
            within(&B->centers[jb * D], &B->centers[ib * D], D, distest))
          B->iflag[jb] = 2;
      }
    }
  }
  int *tail = (int *)malloc(sizeof(int) * 2 * (nlevels + 1));
  for (int l = 0; l <= nlevels; l++) { tail[2 * l] = 0; tail[2 * l + 1] = -1; }
  for (int ilev = 1; ilev <= nlevels - 2; ilev++) {
    tail[2 * (ilev + 1)] = B->n;
    refine_flag_range(B, laddr[2 * ilev], laddr[2 * ilev + 1], bsz[ilev + 1], ilev);
    tail[2 * (ilev + 1) + 1] = B->n - 1;
  }
  reorg(B, nlevels, laddr, tail);
  ncoll = (int *)realloc(ncoll, sizeof(int) * B->n);
  coll = (int *)realloc(coll, sizeof(int) * (size_t)B->n * mnbors);
  computecoll(B, nlevels, laddr, bsz, isep, mnbors, ncoll, coll);

  for (int ib = 0; ib < B->n; ib++)
    if (B->iflag[ib] != 3) B->iflag[ib] = 0;
  for (int l = 0; l <= nlevels; l++) { tail[2 * l] = 0; tail[2 * l + 1] = -1; }
  for (int ilev = 2; ilev <= nlevels - 2; ilev++) {
    updateflags(B, ilev, laddr[2 * ilev], laddr[2 * ilev + 1], bsz, isep, mnbors, ncoll, coll);
    updateflags(B, ilev, tail[2 * ilev], tail[2 * ilev + 1], bsz, isep, mnbors, ncoll, coll);
    tail[2 * (ilev + 1)] = B->n;
    refine_flag_range(B, laddr[2 * ilev], laddr[2 * ilev + 1], bsz[ilev + 1], ilev);
    refine_flag_range(B, tail[2 * ilev], tail[2 * ilev + 1], bsz[ilev + 1], ilev);
    tail[2 * (ilev + 1) + 1] = B->n - 1;
    ncoll = (int *)realloc(ncoll, sizeof(int) * B->n);
    coll = (int *)realloc(coll, sizeof(int) * (size_t)B->n * mnbors);
    /* colleague list of the new boxes: "isep*1.05" is a single-precision product */
    double tol = (double)((float)isep * 1.05f) * bsz[ilev + 1];
    for (int ib = tail[2 * (ilev + 1)]; ib <= tail[2 * (ilev + 1) + 1]; ib++) {
      ncoll[ib] = 0;
      for (int j = 0; j < mnbors; j++) coll[(size_t)ib * mnbors + j] = -1;
      int dad = B->iparent[ib];
      for (int i = 0; i < ncoll[dad]; i++) {
        int jb = coll[(size_t)dad * mnbors + i];
        for (int c = 0; c < NC; c++) {
          int kb = B->ichild[jb * NC + c];
          if (kb >= 0 && within(&B->centers[kb * D], &B->centers[ib * D], D, tol)) {
            coll[(size_t)ib * mnbors + ncoll[ib]] = kb;
            ncoll[ib]++;
          }
        }
      }
    }
  }
  reorg(B, nlevels, laddr, tail);
  computecoll(B, nlevels, laddr, bsz, isep, mnbors, ncoll, coll);
  free(tail);
  *ncollp = ncoll;
  *collp = coll;
}

int otree_build(int D, const double *src, int ns, const double *targ, int nt, int idivflag,
                int ndiv, int nlmin, int nlmax, int isep, int lr_isep_quirk, otree *t) {
  memset(t, 0, sizeof(*t));
  if (ns < 1 || nt < 1 || (D != 2 && D != 3)) return -1;
  int NC = 1 << D;
  int mnbors = 1;
  for (int d = 0; d < D; d++) mnbors *= (2 * isep + 1);
  double mn[3], mx[3];
  for (int d = 0; d < D; d++) mn[d] = mx[d] = src[d];
  for (int i = 0; i < ns; i++)
    for (int d = 0; d < D; d++) {
      double v = src[(size_t)i * D + d];
      if (v < mn[d]) mn[d] = v;
      if (v > mx[d]) mx[d] = v;
    }
  for (int i = 0; i < nt; i++)
    for (int d = 0; d < D; d++) {
      double v = targ[(size_t)i * D + d];
      if (v < mn[d]) mn[d] = v;
      if (v > mx[d]) mx[d] = v;
    }
  double *bsz = (double *)calloc(nlmax + 1, sizeof(double));
  bsz[0] = mx[0] - mn[0];
  for (int d = 1; d < D; d++)
    if (mx[d] - mn[d] > bsz[0]) bsz[0] = mx[d] - mn[d];

  boxes_t B = {0};
  B.D = D;
  B.NC = NC;
  bx_reserve(&B, 1);
  B.n = 1;
  for (int d = 0; d < D; d++) B.centers[d] = (mn[d] + mx[d]) / 2;
  B.ilevel[0] = 0;
  B.iparent[0] = -1;
  B.nchild[0] = 0;
  B.iflag[0] = 0;
  for (int c = 0; c < NC; c++) B.ichild[c] = -1;

  int *laddr = (int *)malloc(sizeof(int) * 2 * (nlmax + 1));
  laddr[0] = 0;
  laddr[1] = 0;
  int *isrc = (int *)malloc(sizeof(int) * ns), *itarg = (int *)malloc(sizeof(int) * nt);
  int *tmp = (int *)malloc(sizeof(int) * (ns > nt ? ns : nt));
  for (int i = 0; i < ns; i++) isrc[i] = i;
  for (int i = 0; i < nt; i++) itarg[i] = i;
  int secap = 64;
  int *isrcse = (int *)malloc(sizeof(int) * 2 * secap), *itargse = (int *)malloc(sizeof(int) * 2 * secap);
  isrcse[0] = 0; isrcse[1] = ns - 1;
  itargse[0] = 0; itargse[1] = nt - 1;

  int ilev;
  for (ilev = 0; ilev < nlmax; ilev++) {
    int lo = laddr[2 * ilev], hi = laddr[2 * ilev + 1];
    int nref = 0;
    for (int ib = lo; ib <= hi; ib++) {
      int refine;
      if (ilev >= nlmin) {
        int nss = isrcse[2 * ib + 1] - isrcse[2 * ib] + 1;
        int ntt = itargse[2 * ib + 1] - itargse[2 * ib] + 1;
        int nn = idivflag == 0 ? nss : (idivflag == 1 ? ntt : (ntt > nss ? ntt : nss));
        refine = nn > ndiv;
      } else {
        refine = 1;
      }
      B.iflag[ib] = refine;
      nref += refine;
    }
    if (nref == 0) break;
    bsz[ilev + 1] = bsz[ilev] / 2;
    laddr[2 * (ilev + 1)] = B.n;
    bx_reserve(&B, B.n + nref * NC);
    if (B.cap > secap) {
      secap = B.cap;
      isrcse = (int *)realloc(isrcse, sizeof(int) * 2 * secap);
      itargse = (int *)realloc(itargse, sizeof(int) * 2 * secap);
    }
    int r = 0;
    for (int ib = lo; ib <= hi; ib++)
      if (B.iflag[ib]) {
        make_children(&B, ib, B.n + r * NC, bsz[ilev + 1], ilev + 1, 0);
        r++;
      }
    B.n += nref * NC;
    for (int ib = lo; ib <= hi; ib++)
      if (B.iflag[ib]) {
        sort_children(&B, ib, src, isrc, isrcse, tmp);
        sort_children(&B, ib, targ, itarg, itargse, tmp);
      }
    laddr[2 * (ilev + 1) + 1] = B.n - 1;
  }
  int nlevels = ilev;
  for (int i = 0; i < B.n; i++) B.iflag[i] = 0;
  free(isrc); free(itarg); free(tmp); free(isrcse); free(itargse);

  int *ncoll = (int *)malloc(sizeof(int) * B.n);
  int *coll = (int *)malloc(sizeof(int) * (size_t)B.n * mnbors);
  computecoll(&B, nlevels, laddr, bsz, isep, mnbors, ncoll, coll);
  if (nlevels >= 2) fix_lr(&B, nlevels, laddr, bsz, isep, lr_isep_quirk, mnbors, &ncoll, &coll);

  t->D = D; t->NC = NC; t->isep = isep; t->mnbors = mnbors;
  t->nlevels = nlevels; t->nboxes = B.n;
  t->laddr = laddr; t->ilevel = B.ilevel; t->iparent = B.iparent; t->nchild = B.nchild;
  t->ichild = B.ichild; t->centers = B.centers; t->ncoll = ncoll; t->coll = coll;
  t->boxsize = bsz;
  free(B.iflag);
  return 0;
}

void otree_free(otree *t) {
  free(t->laddr); free(t->ilevel); free(t->iparent); free(t->nchild); free(t->ichild);
  free(t->ncoll); free(t->coll); free(t->centers); free(t->boxsize);
  memset(t, 0, sizeof(*t));
}

void otree_sort(const otree *t, int n, const double *xys, int *ixy, int *ixyse) {
  boxes_t B = {0};
  B.D = t->D; B.NC = t->NC; B.n = t->nboxes;
  B.centers = t->centers; B.ichild = t->ichild;
  int *tmp = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
  for (int i = 0; i < n; i++) ixy[i] = i;
  ixyse[0] = 0;
  ixyse[1] = n - 1;
  for (int ilev = 0; ilev < t->nlevels; ilev++)
    for (int ib = t->laddr[2 * ilev]; ib <= t->laddr[2 * ilev + 1]; ib++)
      if (t->nchild[ib] > 0) sort_children(&B, ib, xys, ixy, ixyse, tmp);
  free(tmp);
}

/* computemnlists + computelists (tree_routs2d.f:463-746) */
int olists_build(const otree *t, olists *L) {
  int D = t->D, NC = t->NC, nb = t->nboxes, isep = t->isep, mn = t->mnbors;
  const double *bsz = t->boxsize, *C = t->centers;
  memset(L, 0, sizeof(*L));
  for (int k = 0; k < 4; k++) L->nlist[k] = (int *)calloc(nb, sizeof(int));
  for (int pass = 0; pass < 2; pass++) {
    for (int k = 0; k < 4; k++) memset(L->nlist[k], 0, sizeof(int) * nb);
    int *n1 = L->nlist[0], *n2 = L->nlist[1], *n3 = L->nlist[2], *n4 = L->nlist[3];
#define PUSH(k, ib, v)                                              \
  do {                                                              \
    if (pass) L->list[k][(size_t)(ib) * L->mnlist[k] + L->nlist[k][ib]] = (v); \
    L->nlist[k][ib]++;                                              \
  } while (0)
    if (t->nchild[0] == 0) PUSH(0, 0, 0);
    for (int ilev = 1; ilev <= t->nlevels; ilev++) {
      for (int ib = t->laddr[2 * ilev]; ib <= t->laddr[2 * ilev + 1]; ib++) {
        int dad = t->iparent[ib];
        double sep = 1.05 * isep * bsz[ilev];
        for (int i = 0; i < t->ncoll[dad]; i++) {
          int jb = t->coll[(size_t)dad * mn + i];
          for (int c = 0; c < NC; c++) {
            int kb = t->ichild[jb * NC + c];
            if (kb < 0) continue;
            int far = 0;
            for (int d = 0; d < D; d++)
              if (fabs(C[kb * D + d] - C[ib * D + d]) >= sep) far = 1;
            if (far) PUSH(1, ib, kb);
          }
        }
        if (t->nchild[ib] == 0) {
          for (int i = 0; i < t->ncoll[ib]; i++) {
            int jb = t->coll[(size_t)ib * mn + i];
            if (t->nchild[jb] == 0) {
              PUSH(0, ib, jb);
            } else {
              double distest = 1.05 * (bsz[ilev] + bsz[ilev + 1]) / 2.0 * isep;
              for (int c = 0; c < NC; c++) {
                int kb = t->ichild[jb * NC + c];
                if (kb < 0) continue;
                int near = 1;
                for (int d = 0; d < D; d++)
                  if (!(fabs(C[kb * D + d] - C[ib * D + d]) < distest)) near = 0;
                if (near) PUSH(0, ib, kb);
                else PUSH(2, ib, kb);
              }
            }
          }
          for (int i = 0; i < t->ncoll[dad]; i++) {
            int jb = t->coll[(size_t)dad * mn + i];
            if (t->nchild[jb] == 0) {
              double distest = 1.05 * (bsz[ilev] + bsz[ilev - 1]) / 2.0 * isep;
              int near = 1;
              for (int d = 0; d < D; d++)
                if (!(fabs(C[jb * D + d] - C[ib * D + d]) < distest)) near = 0;
              if (near) PUSH(0, ib, jb);
            }
          }
        }
        for (int i = 0; i < t->ncoll[dad]; i++) {
          int jb = t->coll[(size_t)dad * mn + i];
          if (t->nchild[jb] == 0) {
            double distest = 1.05 * (bsz[ilev] + bsz[ilev - 1]) / 2.0 * isep;
            int far = 0;
            for (int d = 0; d < D; d++)
              if (fabs(C[jb * D + d] - C[ib * D + d]) > distest) far = 1;
            if (far) PUSH(3, ib, jb);
          }
        }
      }
    }
#undef PUSH
    (void)n1; (void)n2; (void)n3; (void)n4;
    if (!pass) {
      for (int k = 0; k < 4; k++) {
        int m = 0;
        for (int i = 0; i < nb; i++)
          if (L->nlist[k][i] > m) m = L->nlist[k][i];
        L->mnlist[k] = m;
        L->list[k] = (int *)malloc(sizeof(int) * ((size_t)(m > 0 ? m : 1) * nb));
        for (size_t i = 0; i < (size_t)(m > 0 ? m : 1) * nb; i++) L->list[k][i] = -1;
      }
    }
  }
  return 0;
}

void olists_free(olists *L) {
  for (int k = 0; k < 4; k++) { free(L->nlist[k]); free(L->list[k]); }
  memset(L, 0, sizeof(*L));
}
