/* Implementation of the test stand-in for MATLAB's MEX API (mex.h here) and
 * the handful of helpers the tests call through ctypes to build arguments,
 * run mexFunction and read the outputs. */
#include <setjmp.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mex.h"

struct mxArray_tag {
  mwSize m, n;
  int complex_, is_string;
  double *data; /* m*n doubles, or 2*m*n interleaved (re, im) */
  char *str;
};

static jmp_buf g_jmp;
static char g_err[1024];

mwSize mxGetM(const mxArray *a) { return a->m; }
mwSize mxGetN(const mxArray *a) { return a->n; }
int mxIsComplex(const mxArray *a) { return a->complex_; }
double *mxGetDoubles(const mxArray *a) { return a->complex_ ? NULL : a->data; }
mxComplexDouble *mxGetComplexDoubles(const mxArray *a) {
  return a->complex_ ? (mxComplexDouble *)a->data : NULL;
}
double mxGetScalar(const mxArray *a) { return (a->data && a->m * a->n) ? a->data[0] : 0.0; }
int mxGetString(const mxArray *a, char *buf, mwSize buflen) {
  if (!a->is_string || strlen(a->str) + 1 > buflen) return 1;
  strcpy(buf, a->str);
  return 0;
}
mxArray *mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity c) {
  mxArray *a = (mxArray *)calloc(1, sizeof(mxArray));
  a->m = m;
  a->n = n;
  a->complex_ = c == mxCOMPLEX;
  a->data = (double *)calloc((a->complex_ ? 2 : 1) * (m * n ? m * n : 1), sizeof(double));
  return a;
}
void mxDestroyArray(mxArray *a) {
  if (!a) return;
  free(a->data);
  free(a->str);
  free(a);
}
void *mxMalloc(size_t n) { return malloc(n); }
void mxFree(void *p) { free(p); }
void mexErrMsgTxt(const char *msg) {
  snprintf(g_err, sizeof g_err, "%s", msg);
  longjmp(g_jmp, 1);
}
int mexPrintf(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  int r = vprintf(fmt, ap);
  va_end(ap);
  return r;
}

/* ---- helpers for the tests ---- */
mxArray *shim_real(mwSize m, mwSize n, const double *v) {
  mxArray *a = mxCreateDoubleMatrix(m, n, mxREAL);
  if (v) memcpy(a->data, v, m * n * sizeof(double));
  return a;
}
mxArray *shim_complex(mwSize m, mwSize n, const double *interleaved) {
  mxArray *a = mxCreateDoubleMatrix(m, n, mxCOMPLEX);
  if (interleaved) memcpy(a->data, interleaved, 2 * m * n * sizeof(double));
  return a;
}
mxArray *shim_string(const char *s) {
  mxArray *a = (mxArray *)calloc(1, sizeof(mxArray));
  a->m = 1;
  a->n = strlen(s);
  a->is_string = 1;
  a->str = strdup(s);
  return a;
}
double *shim_data(mxArray *a) { return a->data; }
int shim_is_complex(mxArray *a) { return a->complex_; }
mwSize shim_m(mxArray *a) { return a->m; }
mwSize shim_n(mxArray *a) { return a->n; }
void shim_free(mxArray *a) { mxDestroyArray(a); }
const char *shim_error(void) { return g_err; }

/* runs mexFunction; 0 on success, 1 if it raised a MATLAB error */
int shim_call(int nlhs, mxArray **plhs, int nrhs, const mxArray **prhs) {
  g_err[0] = 0;
  if (setjmp(g_jmp)) return 1;
  mexFunction(nlhs, plhs, nrhs, prhs);
  return 0;
}
