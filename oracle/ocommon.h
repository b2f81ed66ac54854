/*
 * Oracle (TEST INFRASTRUCTURE ONLY): shared driver pieces of the 2D FMMs.
 */
#ifndef ZFMM_OCOMMON_H
#define ZFMM_OCOMMON_H
#include <complex.h>
#include "oracle.h"

typedef double complex cplx;

/* state shared by zlfmm2d / zhfmm2d after tree, sort, reorder and complex centres
 * (zlfmm2d.f:70-200, zhfmm2d.f:73-195) */
typedef struct {
  otree t;
  olists L;
  int ns, nt;
  int *isrc, *isrcse, *itarg, *itargse;
  cplx *zsrcsort, *ztargsort, *chargesort, *dipstrsort, *dipvecsort;
  cplx *zcsrc, *zctarg; /* [2*nboxes] complex centres */
} o2d_state;

int o2d_setup(int ns, const double *zsrc, int ifcharge, const double *charge, int ifdipole,
              const double *dipstr, const double *dipvec, int nt, const double *ztarg,
              int idivflag, int ndiv, int isep, o2d_state *S);
void o2d_free(o2d_state *S);

/* zcart2polar (toolbox.f:73-82): rz = sqrt(z1^2+z2^2), ez = z1/rz + i*z2/rz */
static inline void o_zcart2polar(const cplx *xy, const cplx *x0y0, cplx *rz, cplx *ez) {
  cplx z1 = xy[0] - x0y0[0], z2 = xy[1] - x0y0[1];
  *rz = csqrt(z1 * z1 + z2 * z2);
  *ez = z1 / *rz + I * (z2 / *rz);
}

#endif
