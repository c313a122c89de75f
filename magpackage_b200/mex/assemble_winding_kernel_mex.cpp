/*
 * MEX gateway: [I,V] = assemble_winding_kernel_mex(P,T,Dofs,Signs,Tags,CoilID,DirField,
 *     UniDir,Scale,Qw,ValRef)
 * Drop-in for src/mex/assemble_winding_kernel_mex.cpp:13-127 (Assembler.m:157-166):
 * DirField [3 x NumElems] or the empty [] (UniDir for every element); the element
 * loop runs on the GPU.
 */
#include "magasm.h"
#include "mex.h"

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    (void)nlhs;
    if (nrhs != 11) mexErrMsgIdAndTxt("MagPackage:Args", "Expected 11 inputs.");
    int64_t Nn = (int64_t)mxGetN(prhs[0]), Ne = (int64_t)mxGetN(prhs[1]);
    const double *field = mxIsEmpty(prhs[6]) ? 0 : mxGetPr(prhs[6]);
    if (field && (int64_t)mxGetNumberOfElements(prhs[6]) != 3 * Ne)
        mexErrMsgIdAndTxt("MagPackage:Dim", "DirField must be [3 x NumElems] or empty");
    if (!field && mxGetNumberOfElements(prhs[7]) < 3)
        mexErrMsgIdAndTxt("MagPackage:Dim", "UniformDir must be [3 x 1]");
    int nq = (int)mxGetNumberOfElements(prhs[9]);
    plhs[0] = mxCreateDoubleMatrix((size_t)Ne * 6, 1, mxREAL);
    plhs[1] = mxCreateDoubleMatrix((size_t)Ne * 6, 1, mxREAL);
    int rc = mag_mex_winding(mxGetPr(prhs[0]), Nn, mxGetPr(prhs[1]), Ne, mxGetPr(prhs[2]), mxGetPr(prhs[3]),
                             mxGetPr(prhs[4]), mxGetScalar(prhs[5]), field, mxGetPr(prhs[7]),
                             mxGetScalar(prhs[8]), mxGetPr(prhs[9]), nq, mxGetPr(prhs[10]), mxGetPr(plhs[0]),
                             mxGetPr(plhs[1]));
    if (rc != MAG_OK) mexErrMsgIdAndTxt("MagPackage:GPU", "%s", mag_last_error());
}
