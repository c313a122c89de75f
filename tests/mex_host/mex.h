/*
 * The part of MATLAB's MEX API (R2017b, 64-bit indices) that the gateways in
 * magpackage_b200/mex/ use, so that tests can compile them and run them
 * end to end without MATLAB: mx_runtime.cpp implements it. A MATLAB build
 * uses MATLAB's own <mex.h> instead.
 */
#ifndef MAG_TEST_MEX_H
#define MAG_TEST_MEX_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef size_t mwSize;
typedef size_t mwIndex;
typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;
typedef struct mxArray_tag mxArray;

double *mxGetPr(const mxArray *a);
size_t mxGetM(const mxArray *a);
size_t mxGetN(const mxArray *a);
size_t mxGetNumberOfElements(const mxArray *a);
double mxGetScalar(const mxArray *a);
int mxIsEmpty(const mxArray *a);
int mxIsSparse(const mxArray *a);
mwIndex *mxGetJc(const mxArray *a);
mwIndex *mxGetIr(const mxArray *a);
mxArray *mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity c);
mxArray *mxCreateSparse(mwSize m, mwSize n, mwSize nzmax, mxComplexity c);
void mxDestroyArray(mxArray *a);
void *mxMalloc(size_t n);
void mxFree(void *p);
void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...);

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]);

#ifdef __cplusplus
}
#endif

#endif
