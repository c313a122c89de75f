// Sparse linear algebra on the assembled CSR (sparse.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace mag {

struct PcgSolver;

int csr_spmv(int64_t n, const int64_t *rp, const int32_t *ci, const double *v, const double *x, double *y,
             cudaStream_t s);
int csr_dirichlet(int64_t n, const int64_t *rp, const int32_t *ci, double *v, const uint8_t *fixed, double *rhs,
                  cudaStream_t s);
int pcg_create(int64_t n, PcgSolver **out);
void pcg_destroy(PcgSolver *p);
int pcg_set_aux(PcgSolver *p, int64_t ni, const int64_t *g_rp, const int32_t *g_ci, const double *g_v,
                const int64_t *gt_rp, const int32_t *gt_ci, const double *gt_v, const double *dn_inv);
int pcg_solve(PcgSolver *p, const int64_t *rp, const int32_t *ci, const double *v, const double *b, double *x,
              double rtol, int max_iter, int *iters, double *relres, int *status, cudaStream_t caller);

}  // namespace mag
