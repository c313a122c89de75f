/*
 * MEX gateway: [I,J,V,R_idx,R_val] = assemble_jacobian_kernel_mex(P,T,Dofs,Signs,Tags,SolA,
 *     Qw,CurlRef,lin,isNon,maxB,brk,coe,start,cnt,coeStart,calcJ)
 *
 * Same name, 17 inputs and outputs as the reference gateway
 * (src/mex/assemble_jacobian_kernel_mex.cpp:8-153), so Assembler.m:199-202 calls
 * it unchanged; the element loop runs on the GPU through libmagasm.
 *
 * Optional 18th input asSparse: when nonzero the gateway returns what
 * Assembler.m:204-216 builds from the triplets instead,
 *     [J_mat, R_mat] = assemble_jacobian_kernel_mex(..., calcJ, 1)
 * J_mat = sparse(I,J,V,Ndof,Ndof) ([] when calcJ is false) and
 * R_mat = sparse(R_idx,1,R_val,Ndof,1), Ndof = numel(SolA), summed on the GPU.
 * Build: mex -R2017b -I<repo>/include assemble_jacobian_kernel_mex.cpp -L<repo>/magpackage_b200 -lmagasm
 */
#include "mag_mex_sparse.h"

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    (void)nlhs;
    if (nrhs != 17 && nrhs != 18)
        mexErrMsgIdAndTxt("MagPackage:Args", "Expected 17 inputs (18 with the sparse-output flag).");
    int64_t Nn = (int64_t)mxGetN(prhs[0]), Ne = (int64_t)mxGetN(prhs[1]);
    int64_t Ndof = (int64_t)mxGetNumberOfElements(prhs[5]);
    int nq = (int)(mxGetM(prhs[6]) * mxGetN(prhs[6]));
    int nmat = (int)mxGetNumberOfElements(prhs[8]);
    int nbrk = (int)mxGetNumberOfElements(prhs[11]), ncoe = (int)mxGetNumberOfElements(prhs[12]);
    int calcj = mxGetScalar(prhs[16]) != 0.0;
    if (nrhs == 18 && mxGetScalar(prhs[17]) != 0.0) {
        double *R = (double *)mxMalloc((size_t)(Ndof > 0 ? Ndof : 1) * sizeof(double));
        mag_sparse *Jm = NULL;
        int rc = mag_mex_jacobian_sparse(mxGetPr(prhs[0]), Nn, mxGetPr(prhs[1]), Ne, mxGetPr(prhs[2]),
                                         mxGetPr(prhs[3]), mxGetPr(prhs[4]), mxGetPr(prhs[5]), Ndof,
                                         mxGetPr(prhs[6]), nq, mxGetPr(prhs[7]), mxGetPr(prhs[8]),
                                         mxGetPr(prhs[9]), mxGetPr(prhs[10]), nmat, mxGetPr(prhs[11]), nbrk,
                                         mxGetPr(prhs[12]), ncoe, mxGetPr(prhs[13]), mxGetPr(prhs[14]),
                                         mxGetPr(prhs[15]), calcj, &Jm, R);
        if (rc != MAG_OK) {
            mxFree(R);
            mexErrMsgIdAndTxt("MagPackage:GPU", "%s", mag_last_error());
        }
        plhs[0] = calcj ? mag_to_matlab_sparse(Jm) : mxCreateDoubleMatrix(0, 0, mxREAL);
        plhs[1] = mag_sparse_column(R, Ndof);
        mxFree(R);
        return;
    }
    size_t nk = calcj ? (size_t)Ne * 36 : 0;
    plhs[0] = mxCreateDoubleMatrix(nk, 1, mxREAL);
    plhs[1] = mxCreateDoubleMatrix(nk, 1, mxREAL);
    plhs[2] = mxCreateDoubleMatrix(nk, 1, mxREAL);
    plhs[3] = mxCreateDoubleMatrix((size_t)Ne * 6, 1, mxREAL);
    plhs[4] = mxCreateDoubleMatrix((size_t)Ne * 6, 1, mxREAL);
    int rc = mag_mex_jacobian(mxGetPr(prhs[0]), Nn, mxGetPr(prhs[1]), Ne, mxGetPr(prhs[2]),
                              mxGetPr(prhs[3]), mxGetPr(prhs[4]), mxGetPr(prhs[5]), Ndof,
                              mxGetPr(prhs[6]), nq, mxGetPr(prhs[7]), mxGetPr(prhs[8]),
                              mxGetPr(prhs[9]), mxGetPr(prhs[10]), nmat, mxGetPr(prhs[11]), nbrk,
                              mxGetPr(prhs[12]), ncoe, mxGetPr(prhs[13]), mxGetPr(prhs[14]),
                              mxGetPr(prhs[15]), calcj, mxGetPr(plhs[0]), mxGetPr(plhs[1]),
                              mxGetPr(plhs[2]), mxGetPr(plhs[3]), mxGetPr(plhs[4]));
    if (rc != MAG_OK) mexErrMsgIdAndTxt("MagPackage:GPU", "%s", mag_last_error());
}
