/*
 * MATLAB sparse outputs of the gateways (their optional trailing argument):
 * the library's compressed-column result copied straight into
 * mxCreateSparse's jc / ir / pr, and a residual vector stored as the sparse
 * column that sparse(R_idx, 1, R_val, Ndof, 1) gives (Assembler.m:215).
 */
#ifndef MAG_MEX_SPARSE_H
#define MAG_MEX_SPARSE_H

#include <stdint.h>

#include "magasm.h"
#include "mex.h"

static_assert(sizeof(mwIndex) == sizeof(uint64_t), "the gateways need 64-bit mwIndex (mex -R2017b)");

/* n x n MATLAB sparse from a library result; the handle is destroyed. */
static inline mxArray *mag_to_matlab_sparse(mag_sparse *sp) {
    int64_t n = 0, nnz = 0;
    mag_sparse_info(sp, &n, &nnz);
    mxArray *a = mxCreateSparse((mwSize)n, (mwSize)n, (mwSize)(nnz > 0 ? nnz : 1), mxREAL);
    int rc = mag_sparse_copy(sp, (uint64_t *)mxGetJc(a), (uint64_t *)mxGetIr(a), mxGetPr(a));
    mag_sparse_destroy(sp);
    if (rc != MAG_OK) mexErrMsgIdAndTxt("MagPackage:GPU", "%s", mag_last_error());
    return a;
}

/* n x 1 MATLAB sparse holding the nonzeros of a dense column. */
static inline mxArray *mag_sparse_column(const double *r, int64_t n) {
    int64_t nnz = 0;
    for (int64_t i = 0; i < n; i++) nnz += r[i] != 0.0;
    mxArray *a = mxCreateSparse((mwSize)n, 1, (mwSize)(nnz > 0 ? nnz : 1), mxREAL);
    mwIndex *jc = mxGetJc(a), *ir = mxGetIr(a);
    double *pr = mxGetPr(a);
    int64_t k = 0;
    for (int64_t i = 0; i < n; i++)
        if (r[i] != 0.0) {
            ir[k] = (mwIndex)i;
            pr[k] = r[i];
            k++;
        }
    jc[0] = 0;
    jc[1] = (mwIndex)k;
    return a;
}

#endif
