/*
 * Minimal stand-in for MATLAB's <mex.h>: test infrastructure for the oracle only.
 *
 * MATLAB is not installed here, so the reference's MEX element kernels
 * (src/mex/assemble_*_kernel_mex.cpp) are compiled unchanged against this
 * header. It models an mxArray as a column-major real double matrix with its
 * own storage, which is all those kernels use:
 *   mxGetPr / mxGetM / mxGetN / mxGetNumberOfElements / mxGetScalar / mxIsEmpty
 *   mxCreateDoubleMatrix (zero-filled, like MATLAB) and mexErrMsgIdAndTxt.
 * Error reporting: mexErrMsgIdAndTxt records the message and longjmps back to
 * the glue layer (oracle/ref_glue.cpp), mirroring MATLAB's non-local exit.
 */
#ifndef ORACLE_MEX_SHIM_H
#define ORACLE_MEX_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;

typedef struct mxArray_tag {
    double *pr;
    size_t m;
    size_t n;
    int owns;
} mxArray;

double *mxGetPr(const mxArray *a);
size_t mxGetM(const mxArray *a);
size_t mxGetN(const mxArray *a);
size_t mxGetNumberOfElements(const mxArray *a);
double mxGetScalar(const mxArray *a);
int mxIsEmpty(const mxArray *a);
mxArray *mxCreateDoubleMatrix(size_t m, size_t n, mxComplexity c);
void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...);

/* Gateway entry point; C linkage as in MATLAB's own header. */
void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]);

#ifdef __cplusplus
}
#endif

#endif
