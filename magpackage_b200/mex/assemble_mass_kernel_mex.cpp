/*
 * MEX gateway: [I,J,V] = assemble_mass_kernel_mex(P,T,Dofs,Signs,Coeffs,Qw,ValRef)
 * Drop-in for src/mex/assemble_mass_kernel_mex.cpp:17-127 (Assembler.m:48,67).
 * An empty Coeffs (or one whose length differs from the element count) means
 * sigma = 1, as in the reference (:155,:187).
 *
 * Optional 8th input Ndof: when positive the gateway returns
 * M = sparse(I,J,V,Ndof,Ndof) (Assembler.m:52-53,71-72), summed on the GPU.
 */
#include "mag_mex_sparse.h"

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    (void)nlhs;
    if (nrhs != 7 && nrhs != 8) mexErrMsgIdAndTxt("MagPackage:Args", "Expected 7 inputs (8 with Ndof).");
    int64_t Nn = (int64_t)mxGetN(prhs[0]), Ne = (int64_t)mxGetN(prhs[1]);
    int64_t nc = (int64_t)mxGetNumberOfElements(prhs[4]);
    int nq = (int)mxGetNumberOfElements(prhs[5]);
    const double ndof = nrhs == 8 ? mxGetScalar(prhs[7]) : 0.0;
    if (ndof > 0.0) {
        mag_sparse *M = NULL;
        int rc = mag_mex_mass_sparse(mxGetPr(prhs[0]), Nn, mxGetPr(prhs[1]), Ne, mxGetPr(prhs[2]),
                                     mxGetPr(prhs[3]), nc ? mxGetPr(prhs[4]) : 0, nc, mxGetPr(prhs[5]), nq,
                                     mxGetPr(prhs[6]), (int64_t)ndof, &M);
        if (rc != MAG_OK) mexErrMsgIdAndTxt("MagPackage:GPU", "%s", mag_last_error());
        plhs[0] = mag_to_matlab_sparse(M);
        return;
    }
    size_t n = (size_t)Ne * 36;
    for (int k = 0; k < 3; k++) plhs[k] = mxCreateDoubleMatrix(n, 1, mxREAL);
    int rc = mag_mex_mass(mxGetPr(prhs[0]), Nn, mxGetPr(prhs[1]), Ne, mxGetPr(prhs[2]),
                          mxGetPr(prhs[3]), nc ? mxGetPr(prhs[4]) : 0, nc, mxGetPr(prhs[5]), nq,
                          mxGetPr(prhs[6]), mxGetPr(plhs[0]), mxGetPr(plhs[1]), mxGetPr(plhs[2]));
    if (rc != MAG_OK) mexErrMsgIdAndTxt("MagPackage:GPU", "%s", mag_last_error());
}
