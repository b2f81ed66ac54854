/*
 * CPU oracle for the complex-coordinate FMM hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is a plain-C restatement of the
 * reference Fortran (wangyuguan/zfmm) used to check the CUDA product path.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
 * arm may load it.  The product library (zfmm_b200) never links or calls it.
 *
 * Conventions: boxes are numbered from 0 (the reference numbers from 1);
 * "none" is -1 as in the reference.  Complex arrays are interleaved
 * (re, im) doubles in Fortran column-major order, e.g. zsrc(d, ns).
 */
#ifndef ZFMM_ORACLE_H
#define ZFMM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int D;         /* 2 or 3 */
  int NC;        /* 4 or 8 children */
  int isep;
  int mnbors;    /* (2*isep+1)^D */
  int nlevels;
  int nboxes;
  int *laddr;    /* [2*(nlevels+1)] first,last box of each level */
  int *ilevel;   /* [nboxes] */
  int *iparent;  /* [nboxes] */
  int *nchild;   /* [nboxes] */
  int *ichild;   /* [NC*nboxes], child c of box b at ichild[b*NC+c] */
  int *ncoll;    /* [nboxes] */
  int *coll;     /* [mnbors*nboxes] */
  double *centers; /* [D*nboxes] */
  double *boxsize; /* [nlevels+1] */
} otree;

typedef struct {
  int mnlist[4];
  int *nlist[4];  /* [nboxes] */
  int *list[4];   /* [mnlist_k * nboxes], entry i of box b at list[k][b*mnlist_k+i] */
} olists;

/* tree build (pts_tree_mem + pts_tree_build + fix_lr), real coordinates
 * src(D,ns), targ(D,nt).  bbox_mode 0 = 2D pts_tree_mem, 1 = 3D estimate_bounding_box
 * (identical arithmetic).  lr_isep_quirk=1 drops isep from the flag+ distance
 * (pts_tree3d.f:1209). */
int otree_build(int D, const double *src, int ns, const double *targ, int nt,
                int idivflag, int ndiv, int nlmin, int nlmax, int isep,
                int lr_isep_quirk, otree *t);
void otree_free(otree *t);
/* pts_tree_sort: permutation ixy[n] (0-based original indices) and ranges
 * ixyse[2*nboxes] (0-based first,last; empty when last<first). */
void otree_sort(const otree *t, int n, const double *xys, int *ixy, int *ixyse);
int olists_build(const otree *t, olists *L);
void olists_free(olists *L);

/* sizing tables */
void o_lndiv2d(double eps, int ns, int nt, int *ndiv, int *idivflag);
int o_l2dterms(double eps);
void o_init_carray(double *carray, int ldc);

/* 2D Laplace: direct sum (unscaled, zlfmm2d.f:600-654) and FMM (scaled by 1/2pi) */
void o_zl2devaldirect(int nt, const double *ztarg, int ns, const double *zsrc,
                      const double *charge, const double *dipstr, const double *dipvec,
                      int ifcharge, double *pot, double *grad, int ifdipole, int ifpgh);
int o_zlfmm2d(double eps, int ns, const double *zsrc, int ifcharge, const double *charge,
              int ifdipole, const double *dipstr, const double *dipvec, double *pot,
              double *grad, int nt, const double *ztarg, int ifpgh, int isep, int ifprint);

/* 2D Helmholtz */
void o_hank103(double zr, double zi, double *h0, double *h1);
void o_jbessel2d(int nterms, double zr, double zi, double rscale, double *fjs,
                 int ifder, double *fjder);
void o_h2dall(int nterms, double zr, double zi, double rscale, double *hvec,
              int ifder, double *hder);
int o_h2dterms(double bsize, double zkr, double zki, double eps, int isep);
void o_zh2devaldirect(const double *zk, int nt, const double *ztarg, int ns,
                      const double *zsrc, const double *charge, const double *dipstr,
                      const double *dipvec, int ifcharge, double *pot, double *grad,
                      int ifdipole, int ifpgh);
int o_zhfmm2d(double eps, const double *zk, int ns, const double *zsrc, int ifcharge,
              const double *charge, int ifdipole, const double *dipstr, const double *dipvec,
              double *pot, double *grad, int nt, const double *ztarg, int ifpgh, int isep,
              int ifprint);

/* 3D Laplace: direct sum (with 1/(4 pi), zlfmm3d.f:628-683) and FMM */
int o_zl3dterms(double eps);
void o_zl3devaldirect(int nt, const double *ztarg, int ns, const double *zsrc,
                      const double *charge, const double *dipstr, const double *dipvec,
                      int ifcharge, double *pot, double *grad, int ifdipole, int ifpgh);
int o_zlfmm3d(double eps, int ns, const double *zsrc, int ifcharge, const double *charge,
              int ifdipole, const double *dipstr, const double *dipvec, double *pot,
              double *grad, int nt, const double *ztarg, int ifpgh, int isep, int ifprint);

/* 3D Helmholtz: direct sum (with 1/(4 pi), zhfmm3d.f:626-693) and FMM; zk = (re, im) */
int o_h3dterms(double size, double zkr, double zki, double eps, int isep);
void o_gauss_legendre(int n, double *x, double *w);
void o_zh3devaldirect(const double *zk, int nt, const double *ztarg, int ns, const double *zsrc,
                      const double *charge, const double *dipstr, const double *dipvec,
                      int ifcharge, double *pot, double *grad, int ifdipole, int ifpgh);
int o_zhfmm3d(double eps, const double *zk, int ns, const double *zsrc, int ifcharge,
              const double *charge, int ifdipole, const double *dipstr, const double *dipvec,
              double *pot, double *grad, int nt, const double *ztarg, int ifpgh, int isep,
              int ifprint);

/* tree inspection helpers for tests: build the tree exactly as the 2D/3D drivers
 * do and copy out summary arrays.  Returns nboxes; fills nlevels. */
int o_tree_info(int D, double eps_ndiv, int ndiv_override, const double *zsrc, int ns,
                const double *ztarg, int nt, int isep, int *nlevels, int *laddr_out,
                int laddr_cap, int *mnlist_out);
/* full dump: arrays sized by the caller from o_tree_info's nboxes */
int o_tree_dump(int D, int ndiv, const double *zsrc, int ns, const double *ztarg, int nt,
                int isep, int *ilevel, int *iparent, int *nchild, int *ichild,
                double *centers, int *isrc, int *isrcse, int *itarg, int *itargse,
                int *nlist, int *list_flat, int list_cap);

#ifdef __cplusplus
}
#endif
#endif
