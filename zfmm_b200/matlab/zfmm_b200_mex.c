/*
 * MATLAB gateway of libzfmm_b200 (hand-written; no counterpart file in the
 * reference, whose gateways are generated by mwrap from the .mw specs,
 * e.g. zfmm3d/matlab_linux/zhfmm3dmex.c:1094-1425).
 *
 * Calling protocol: the one mwrap generates from a .mw file
 * (zfmm2d/matlab_linux/zlfmm2d.mw:7 and siblings), so the .m wrappers that
 * mwrap writes for the reference call this gateway unchanged:
 *
 *     [pot, grad] = zlfmm2dmex(mex_id_, arg_1, ..., arg_N, dims...)
 *
 *   mex_id_  'name(i double[x], i int[x], i dcomplex[xx], ...)': the routine
 *            name before '(' selects the call; the list must have the
 *            routine's N arguments (the FORTRAN line of its .mw spec)
 *   arg_k    the FORTRAN arguments in .mw order (scalars, vectors, d x n
 *            matrices; integers as MATLAB doubles)
 *   dims     one size per [x] argument and two per [xx] argument, in order;
 *            every argument is checked against them ("Bad argument size")
 *   outputs  the inout arrays, pot (nt x 1) and grad (d x nt)
 *
 * Unlike an mwrap gateway, this one calls the status-returning C entry points
 * (zfmm_zlfmm2d ... of include/zfmm.h) and turns a non-zero status into a
 * MATLAB error carrying zfmm_last_error(); flags are clamped like the
 * reference (zlfmm2d.f:58-68) by the library.  Complex arrays use MATLAB's
 * interleaved complex storage (mxGetComplexDoubles, MATLAB R2018a and later,
 * build with -R2018a); a real array where a complex one is expected is
 * promoted.  One source serves all eight routines: build it once per MEX name
 * (zlfmm2dmex, zhfmm2dmex, ...), see build_mex.sh.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mex.h"
#include "zfmm.h"

/* argument kinds */
enum { A_DBL, A_INT, A_ZSC, A_ZVEC, A_ZMAT, A_IOVEC, A_IOMAT };

typedef struct {
  const char *name;   /* routine name */
  int d;              /* dimension (2 or 3) */
  int helm;           /* 1: zk is the first complex scalar */
  int fmm;            /* 1: FMM (eps, ... isep, ifprint), 0: direct sum */
  int nargs;
  int kind[16];       /* argument kinds in .mw FORTRAN order */
  const char *argname[16];
} Routine;

/* the FORTRAN argument lists of the .mw specs (zfmm2d/matlab_linux/zlfmm2d.mw:7 and
 * siblings in zfmm2d/matlab_linux and zfmm3d/matlab_linux) */
#define FMM_L(nm, D)                                                                             \
  {nm, D, 0, 1, 15,                                                                              \
   {A_DBL, A_INT, A_ZMAT, A_INT, A_ZVEC, A_INT, A_ZVEC, A_ZMAT, A_IOVEC, A_IOMAT, A_INT, A_ZMAT, \
    A_INT, A_INT, A_INT},                                                                        \
   {"eps", "ns", "zsrc", "ifcharge", "charge", "ifdipole", "dipstr", "dipvec", "pot", "grad",    \
    "nt", "ztarg", "ifpgh", "isep", "ifprint"}}
#define FMM_H(nm, D)                                                                             \
  {nm, D, 1, 1, 16,                                                                              \
   {A_DBL, A_ZSC, A_INT, A_ZMAT, A_INT, A_ZVEC, A_INT, A_ZVEC, A_ZMAT, A_IOVEC, A_IOMAT, A_INT,  \
    A_ZMAT, A_INT, A_INT, A_INT},                                                                \
   {"eps", "zk", "ns", "zsrc", "ifcharge", "charge", "ifdipole", "dipstr", "dipvec", "pot",      \
    "grad", "nt", "ztarg", "ifpgh", "isep", "ifprint"}}
#define DIR_L(nm, D)                                                                             \
  {nm, D, 0, 0, 12,                                                                              \
   {A_INT, A_ZMAT, A_INT, A_ZMAT, A_ZVEC, A_ZVEC, A_ZMAT, A_INT, A_IOVEC, A_IOMAT, A_INT, A_INT}, \
   {"nt", "ztarg", "ns", "zsrc", "charge", "dipstr", "dipvec", "ifcharge", "pot", "grad",        \
    "ifdipole", "ifpgh"}}
#define DIR_H(nm, D)                                                                             \
  {nm, D, 1, 0, 13,                                                                              \
   {A_ZSC, A_INT, A_ZMAT, A_INT, A_ZMAT, A_ZVEC, A_ZVEC, A_ZMAT, A_INT, A_IOVEC, A_IOMAT, A_INT, \
    A_INT},                                                                                      \
   {"zk", "nt", "ztarg", "ns", "zsrc", "charge", "dipstr", "dipvec", "ifcharge", "pot", "grad",  \
    "ifdipole", "ifpgh"}}

static const Routine kRoutines[] = {
    FMM_L("zlfmm2d", 2), FMM_H("zhfmm2d", 2), FMM_L("zlfmm3d", 3), FMM_H("zhfmm3d", 3),
    DIR_L("zl2devaldirect", 2), DIR_H("zh2devaldirect", 2), DIR_L("zl3devaldirect", 3),
    DIR_H("zh3devaldirect", 3),
};

static int ndims_of(int kind) { return (kind == A_ZMAT || kind == A_IOMAT) ? 2 : 1; }

/* complex data of a MATLAB array as interleaved doubles; a real array is
 * promoted into `tmp` (freed by the caller) */
static double *complex_data(const mxArray *a, double **tmp) {
  size_t n = mxGetM(a) * mxGetN(a), i;
  if (mxIsComplex(a)) return (double *)mxGetComplexDoubles(a);
  *tmp = (double *)mxMalloc(2 * (n ? n : 1) * sizeof(double));
  const double *r = mxGetDoubles(a);
  for (i = 0; i < n; i++) {
    (*tmp)[2 * i] = r ? r[i] : 0.0;
    (*tmp)[2 * i + 1] = 0.0;
  }
  return *tmp;
}

static void run(const Routine *R, int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
  char msg[512];
  int k, ndim = 0, ntmp = 0;
  double *tmp[16] = {0};
  double *z[16] = {0};   /* complex arrays, interleaved */
  int iv[16] = {0};      /* integer scalars */
  double dv[16] = {0};   /* double scalars */
  mxArray *out[2] = {0, 0};
  int nout = 0, st = 0;
  for (k = 0; k < R->nargs; k++) ndim += ndims_of(R->kind[k]);
  if (nrhs != R->nargs + ndim) {
    snprintf(msg, sizeof msg, "%s: expected %d arguments and %d sizes, got %d inputs", R->name,
             R->nargs, ndim, nrhs);
    mexErrMsgTxt(msg);
  }
  /* sizes, in mwrap's order after the arguments */
  {
    const mxArray **dims = prhs + R->nargs;
    int j = 0;
    for (k = 0; k < R->nargs; k++) {
      const mxArray *a = prhs[k];
      if (ndims_of(R->kind[k]) == 1) {
        size_t want = (size_t)mxGetScalar(dims[j++]);
        if (mxGetM(a) * mxGetN(a) != want) {
          snprintf(msg, sizeof msg, "Bad argument size: %s", R->argname[k]);
          mexErrMsgTxt(msg);
        }
      } else {
        size_t m = (size_t)mxGetScalar(dims[j]), n = (size_t)mxGetScalar(dims[j + 1]);
        j += 2;
        if (mxGetM(a) != m || mxGetN(a) != n) {
          snprintf(msg, sizeof msg, "Bad argument size: %s", R->argname[k]);
          mexErrMsgTxt(msg);
        }
      }
    }
  }
  for (k = 0; k < R->nargs; k++) {
    const mxArray *a = prhs[k];
    switch (R->kind[k]) {
      case A_DBL: dv[k] = mxGetScalar(a); break;
      case A_INT: iv[k] = (int)mxGetScalar(a); break;
      case A_ZSC:
      case A_ZVEC:
      case A_ZMAT: z[k] = complex_data(a, &tmp[ntmp]); if (tmp[ntmp]) ntmp++; break;
      case A_IOVEC:
      case A_IOMAT: {
        /* inout: a fresh complex copy of the input is updated and returned */
        double *tin = 0, *src = complex_data(a, &tin);
        mxArray *o = mxCreateDoubleMatrix(mxGetM(a), mxGetN(a), mxCOMPLEX);
        memcpy(mxGetComplexDoubles(o), src, 2 * mxGetM(a) * mxGetN(a) * sizeof(double));
        if (tin) mxFree(tin);
        z[k] = (double *)mxGetComplexDoubles(o);
        out[nout++] = o;
        break;
      }
    }
  }
  if (R->fmm) {
    /* FMM: [eps, (zk), ns, zsrc, ifcharge, charge, ifdipole, dipstr, dipvec, pot, grad, nt,
     *       ztarg, ifpgh, isep, ifprint] */
    int o = R->helm;
    double eps = dv[0];
    int ns = iv[1 + o], ifc = iv[3 + o], ifd = iv[5 + o], nt = iv[10 + o], ifpgh = iv[12 + o];
    int isep = iv[13 + o], ifprint = iv[14 + o];
    const double *zs = z[2 + o], *q = z[4 + o], *ds = z[6 + o], *dvv = z[7 + o];
    double *pot = z[8 + o], *grad = z[9 + o];
    const double *zt = z[11 + o];
    if (!R->helm && R->d == 2)
      st = zfmm_zlfmm2d(eps, ns, zs, ifc, q, ifd, ds, dvv, pot, grad, nt, zt, ifpgh, isep, ifprint);
    else if (R->d == 2)
      st = zfmm_zhfmm2d(eps, z[1], ns, zs, ifc, q, ifd, ds, dvv, pot, grad, nt, zt, ifpgh, isep,
                        ifprint);
    else if (!R->helm)
      st = zfmm_zlfmm3d(eps, ns, zs, ifc, q, ifd, ds, dvv, pot, grad, nt, zt, ifpgh, isep, ifprint);
    else
      st = zfmm_zhfmm3d(eps, z[1], ns, zs, ifc, q, ifd, ds, dvv, pot, grad, nt, zt, ifpgh, isep,
                        ifprint);
  } else {
    /* direct sum: [(zk), nt, ztarg, ns, zsrc, charge, dipstr, dipvec, ifcharge, pot, grad,
     *              ifdipole, ifpgh] */
    int o = R->helm;
    int nt = iv[0 + o], ns = iv[2 + o], ifc = iv[7 + o], ifd = iv[10 + o], ifpgh = iv[11 + o];
    const double *zt = z[1 + o], *zs = z[3 + o], *q = z[4 + o], *ds = z[5 + o], *dvv = z[6 + o];
    double *pot = z[8 + o], *grad = z[9 + o];
    if (!R->helm && R->d == 2)
      st = zfmm_zl2devaldirect(nt, zt, ns, zs, q, ds, dvv, ifc, pot, grad, ifd, ifpgh);
    else if (R->d == 2)
      st = zfmm_zh2devaldirect(z[0], nt, zt, ns, zs, q, ds, dvv, ifc, pot, grad, ifd, ifpgh);
    else if (!R->helm)
      st = zfmm_zl3devaldirect(nt, zt, ns, zs, q, ds, dvv, ifc, pot, grad, ifd, ifpgh);
    else
      st = zfmm_zh3devaldirect(z[0], nt, zt, ns, zs, q, ds, dvv, ifc, pot, grad, ifd, ifpgh);
  }
  for (k = 0; k < ntmp; k++) mxFree(tmp[k]);
  if (st != 0) {
    for (k = 0; k < nout; k++) mxDestroyArray(out[k]);
    snprintf(msg, sizeof msg, "%s: status %d: %s", R->name, st, zfmm_last_error());
    mexErrMsgTxt(msg);
  }
  for (k = 0; k < nout; k++) {
    if (k < nlhs || (k == 0 && nlhs == 0)) plhs[k] = out[k];
    else mxDestroyArray(out[k]);
  }
}

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
  char id[1024];
  size_t i, n;
  if (nrhs == 0) {
    mexPrintf("zfmm_b200 MEX gateway (%s)\n", zfmm_version());
    return;
  }
  if (mxGetString(prhs[0], id, sizeof(id)) != 0) mexErrMsgTxt("Identifier should be a string");
  for (i = 0; i < sizeof(kRoutines) / sizeof(kRoutines[0]); i++) {
    const Routine *R = &kRoutines[i];
    n = strlen(R->name);
    if (strncmp(id, R->name, n) == 0 && id[n] == '(') {
      /* the identifier's argument list must have the routine's length */
      int nargs = 1;
      const char *p;
      for (p = id + n + 1; *p && *p != ')'; p++)
        if (*p == ',') nargs++;
      if (nargs != R->nargs) mexErrMsgTxt("Identifier does not match the routine's arguments");
      run(R, nlhs, plhs, nrhs - 1, prhs + 1);
      return;
    }
  }
  mexErrMsgTxt("Unknown identifier");
}
