/*
 * MEX gateway: [I,V] = assemble_source_kernel_mex(P,T,Dofs,Signs,Js,Qw,ValRef)
 * Drop-in for src/mex/assemble_source_kernel_mex.cpp:16-114 (Assembler.m:87-89):
 * Js is [3 x NumElems]; the element loop runs on the GPU.
 */
#include "magasm.h"
#include "mex.h"

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    (void)nlhs;
    if (nrhs != 7) mexErrMsgIdAndTxt("MagPackage:Args", "Expected 7 inputs.");
    int64_t Nn = (int64_t)mxGetN(prhs[0]), Ne = (int64_t)mxGetN(prhs[1]);
    if (mxGetM(prhs[4]) != 3 || (int64_t)mxGetN(prhs[4]) != Ne)
        mexErrMsgIdAndTxt("MagPackage:Dim", "Js must be [3 x NumElems]");
    int nq = (int)mxGetNumberOfElements(prhs[5]);
    plhs[0] = mxCreateDoubleMatrix((size_t)Ne * 6, 1, mxREAL);
    plhs[1] = mxCreateDoubleMatrix((size_t)Ne * 6, 1, mxREAL);
    int rc = mag_mex_source(mxGetPr(prhs[0]), Nn, mxGetPr(prhs[1]), Ne, mxGetPr(prhs[2]), mxGetPr(prhs[3]),
                            mxGetPr(prhs[4]), mxGetPr(prhs[5]), nq, mxGetPr(prhs[6]), mxGetPr(plhs[0]),
                            mxGetPr(plhs[1]));
    if (rc != MAG_OK) mexErrMsgIdAndTxt("MagPackage:GPU", "%s", mag_last_error());
}
