/*
 * CPU restatement of MagPackage's Nedelec element-assembly path.
 *
 * TEST INFRASTRUCTURE ONLY: the CUDA path is compared with this library.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
 * it. Parity is pinned: tests/test_oracle.py checks every function here against
 * the reference's own MEX kernels compiled unchanged (oracle/_ref) and against
 * the golden vectors in tests/golden/ that those kernels produced.
 *
 * Conventions follow the reference's MATLAB/MEX boundary: arrays are
 * column-major doubles, node/dof indices 1-based stored as doubles, exactly as
 * Assembler.m hands them to the MEX gateways.
 */
#ifndef MAG_ORACLE_H
#define MAG_ORACLE_H

#include <stddef.h>
#include <stdint.h>

/* Mesh.generateEdges (src/Mesh.m:114-138). T: int32 [4 x Ne] 1-based.
 * Outputs: edges [2 x E] 1-based (lexicographic by (min,max) node),
 * t2e [6 x Ne] 1-based edge ids, sign [6 x Ne] (+1/-1). Returns E. */
int64_t oracle_generate_edges(const int32_t *T, int64_t Ne, int32_t *edges_out, int64_t edges_cap,
                              int32_t *t2e, int8_t *sign);

/* Jacobian + residual element kernel, restating
 * src/mex/assemble_jacobian_kernel_mex.cpp:8-153 and
 * src/mex/MexMaterialUtils.hpp:24-87. Output layout as the MEX (:135-152). */
void oracle_jacobian(const double *P, const double *T, int64_t Ne, const double *Dofs,
                     const double *Signs, const double *Tags, const double *SolA, const double *Qw,
                     int nq, const double *CurlRef, const double *lin, const double *isNon,
                     const double *maxB, const double *brk, const double *coe, const double *start,
                     const double *cnt, const double *coeStart, int calcJ, double *I, double *J,
                     double *V, double *Ridx, double *Rval);

/* evaluate_nu_derivative (MexMaterialUtils.hpp:24-87) at n values s = |B|^2 with
 * 1-based tags; the packed tables as for oracle_jacobian. */
void oracle_material_eval(const double *s, const double *Tags, int64_t n, const double *lin,
                          const double *isNon, const double *maxB, const double *brk,
                          const double *coe, const double *start, const double *cnt,
                          const double *coeStart, double *nu, double *dnu);

/* Curl-curl element kernel, src/mex/assemble_curl_curl_kernel_mex.cpp:18-121. */
void oracle_curl_curl(const double *P, const double *T, int64_t Ne, const double *Dofs,
                      const double *Signs, const double *Nu, const double *Qw, int nq,
                      const double *CurlRef, double *I, double *J, double *V);

/* Sigma-weighted mass element kernel, src/mex/assemble_mass_kernel_mex.cpp:17-127.
 * Coeffs == NULL (or ncoeff != Ne) means sigma = 1 (:155,:187). */
void oracle_mass(const double *P, const double *T, int64_t Ne, const double *Dofs,
                 const double *Signs, const double *Coeffs, int64_t ncoeff, const double *Qw, int nq,
                 const double *ValRef, double *I, double *J, double *V);

/* Winding vector element kernel, src/mex/assemble_winding_kernel_mex.cpp:13-127.
 * DirField [3 x Ne] or NULL (then UniDir [3]). */
void oracle_winding(const double *P, const double *T, int64_t Ne, const double *Dofs,
                    const double *Signs, const double *Tags, double CoilID, const double *DirField,
                    const double *UniDir, double Scale, const double *Qw, int nq, const double *ValRef,
                    double *I, double *V);
/* Source vector element kernel, src/mex/assemble_source_kernel_mex.cpp:16-114. */
void oracle_source(const double *P, const double *T, int64_t Ne, const double *Dofs,
                   const double *Signs, const double *Js, const double *Qw, int nq,
                   const double *ValRef, double *I, double *V);

/* Harmonic-balance element kernel, src/mex/assemble_hbfem_kernel_mex.cpp:26-258, with the
 * spline coefficient offsets coeStart passed (the gateway leaves them unset). SolR/SolI
 * [Ndof x K], DR/DI [N x K], PR/PI [K x N] column-major; SolI, DI, PI may be NULL.
 * Outputs as the gateway: I,J,V [36 K Ne] (when calcJ), R rows/cols/re/im [6 K Ne]. */
void oracle_hbfem(const double *P, const double *T, int64_t Ne, const double *Dofs,
                  const double *Signs, const double *Tags, const double *SolR, const double *SolI,
                  int64_t Ndof, int K, const double *DR, const double *DI, const double *PR,
                  const double *PI, int N, const double *Qw, int nq, const double *CurlRef,
                  const double *lin, const double *isNon, const double *maxB, const double *brk,
                  const double *coe, const double *start, const double *cnt, const double *coeStart,
                  int calcJ, const double *Scalings, double *I, double *J, double *V, double *Rrows,
                  double *Rcols, double *Rre, double *Rim);

/* MATLAB sparse(I(valid),J(valid),V(valid),N,N) as used at Assembler.m:37-38,
 * 205-206: valid = I>0 & J>0; duplicates summed in order of appearance;
 * drop_zeros != 0 removes entries whose sum is exactly zero (MATLAB stores no
 * explicit zeros). Result in CSR (rows = I). Two-call protocol: call with
 * col_idx == NULL to get nnz, then again with buffers of that size.
 * Returns nnz, or -1 on bad index. */
int64_t oracle_sparse_csr(const double *I, const double *J, const double *V, int64_t n, int64_t N,
                          int drop_zeros, int64_t *row_ptr, int32_t *col_idx, double *vals);

/* Same for a vector: sparse(R_idx(valid),1,R_val(valid),N,1) (Assembler.m:214-215),
 * densified: out[N] = sum over valid entries in order of appearance. */
int oracle_sparse_vec(const double *Ridx, const double *Rval, int64_t n, int64_t N, double *out);

/* MATLAB pchip(x, y) piecewise cubic Hermite coefficients (Fritsch-Carlson
 * slopes with the shape-preserving three-point end rule), as called at
 * src/MaterialLib.m:117. coefs: [n-1 x 4] row-major, highest power first,
 * matching pp.coefs. Returns 0 on success. */
int oracle_pchip(const double *x, const double *y, int64_t n, double *coefs);

#endif
