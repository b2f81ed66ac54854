/* Minimal stand-in for MATLAB's mex.h / matrix.h (interleaved-complex API of
 * R2018a), enough to compile and drive zfmm_b200/matlab/zfmm_b200_mex.c in the
 * tests without MATLAB.  Arrays are double, real or complex, m x n;
 * mexErrMsgTxt returns to shim_call() through longjmp. */
#ifndef ZFMM_TEST_MEX_H
#define ZFMM_TEST_MEX_H
#include <stddef.h>

typedef size_t mwSize;
typedef struct mxArray_tag mxArray;
typedef struct {
  double real, imag;
} mxComplexDouble;
typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;

mwSize mxGetM(const mxArray *a);
mwSize mxGetN(const mxArray *a);
int mxIsComplex(const mxArray *a);
double *mxGetDoubles(const mxArray *a);
mxComplexDouble *mxGetComplexDoubles(const mxArray *a);
double mxGetScalar(const mxArray *a);
int mxGetString(const mxArray *a, char *buf, mwSize buflen);
mxArray *mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity c);
void mxDestroyArray(mxArray *a);
void *mxMalloc(size_t n);
void mxFree(void *p);
void mexErrMsgTxt(const char *msg);
int mexPrintf(const char *fmt, ...);

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]);
#endif
