/*
 * MEX gateway: [I,J,V] = assemble_curl_curl_kernel_mex(P,T,Dofs,Signs,Nu,Qw,CurlRef)
 * Drop-in for src/mex/assemble_curl_curl_kernel_mex.cpp:18-121 (Assembler.m:33,
 * tests/test_mex_assembly.m:60); the element loop runs on the GPU.
 *
 * Optional 8th input Ndof: when positive the gateway returns
 * K = sparse(I,J,V,Ndof,Ndof) (Assembler.m:37-38), summed on the GPU.
 */
#include "mag_mex_sparse.h"

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    (void)nlhs;
    if (nrhs != 7 && nrhs != 8) mexErrMsgIdAndTxt("MagPackage:Args", "Expected 7 inputs (8 with Ndof).");
    int64_t Nn = (int64_t)mxGetN(prhs[0]), Ne = (int64_t)mxGetN(prhs[1]);
    int nq = (int)mxGetNumberOfElements(prhs[5]);
    const double ndof = nrhs == 8 ? mxGetScalar(prhs[7]) : 0.0;
    if (ndof > 0.0) {
        mag_sparse *K = NULL;
        int rc = mag_mex_curl_curl_sparse(mxGetPr(prhs[0]), Nn, mxGetPr(prhs[1]), Ne, mxGetPr(prhs[2]),
                                          mxGetPr(prhs[3]), mxGetPr(prhs[4]), mxGetPr(prhs[5]), nq,
                                          mxGetPr(prhs[6]), (int64_t)ndof, &K);
        if (rc != MAG_OK) mexErrMsgIdAndTxt("MagPackage:GPU", "%s", mag_last_error());
        plhs[0] = mag_to_matlab_sparse(K);
        return;
    }
    size_t n = (size_t)Ne * 36;
    for (int k = 0; k < 3; k++) plhs[k] = mxCreateDoubleMatrix(n, 1, mxREAL);
    int rc = mag_mex_curl_curl(mxGetPr(prhs[0]), Nn, mxGetPr(prhs[1]), Ne, mxGetPr(prhs[2]),
                               mxGetPr(prhs[3]), mxGetPr(prhs[4]), mxGetPr(prhs[5]), nq,
                               mxGetPr(prhs[6]), mxGetPr(plhs[0]), mxGetPr(plhs[1]), mxGetPr(plhs[2]));
    if (rc != MAG_OK) mexErrMsgIdAndTxt("MagPackage:GPU", "%s", mag_last_error());
}
