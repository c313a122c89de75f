/*
 * MEX gateway: [I,J,V] = assemble_curl_curl_kernel_mex(P,T,Dofs,Signs,Nu,Qw,CurlRef)
 * Drop-in for src/mex/assemble_curl_curl_kernel_mex.cpp:18-121 (Assembler.m:33,
 * tests/test_mex_assembly.m:60); the element loop runs on the GPU.
 */
#include "mex.h"
#include "magasm.h"

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    (void)nlhs;
    if (nrhs != 7) mexErrMsgIdAndTxt("MagPackage:Args", "Expected 7 inputs.");
    int64_t Nn = (int64_t)mxGetN(prhs[0]), Ne = (int64_t)mxGetN(prhs[1]);
    int nq = (int)mxGetNumberOfElements(prhs[5]);
    size_t n = (size_t)Ne * 36;
    for (int k = 0; k < 3; k++) plhs[k] = mxCreateDoubleMatrix(n, 1, mxREAL);
    int rc = mag_mex_curl_curl(mxGetPr(prhs[0]), Nn, mxGetPr(prhs[1]), Ne, mxGetPr(prhs[2]),
                               mxGetPr(prhs[3]), mxGetPr(prhs[4]), mxGetPr(prhs[5]), nq,
                               mxGetPr(prhs[6]), mxGetPr(plhs[0]), mxGetPr(plhs[1]), mxGetPr(plhs[2]));
    if (rc != MAG_OK) mexErrMsgIdAndTxt("MagPackage:GPU", "%s", mag_last_error());
}
