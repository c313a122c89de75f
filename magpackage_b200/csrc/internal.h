// Internal (C++) interfaces between the library's translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace mag {

// CSR pattern + incidence plan produced by build_pattern (device memory).
struct PatternBuffers {
    int32_t *row_ptr = nullptr;   // [ndof+1]
    int32_t *col_idx = nullptr;   // [nnz]
    int32_t *inc_ptr = nullptr;   // [ndof+1]
    uint32_t *inc_elem = nullptr; // [ninc]
    uint32_t *inc_pos = nullptr;  // [ninc] or [ninc][2] (wide)
    int64_t nnz = 0;
    int64_t ninc = 0;
    int max_row = 0;
    int wide = 0;
};

int generate_edges(const int32_t *d_T, int64_t ne, int64_t nn, int32_t *d_edges, int32_t *d_t2e,
                   int8_t *d_sign, int64_t *E_out, cudaStream_t s);
int build_pattern(const int32_t *d_dofs, int64_t ne, int64_t ndof, PatternBuffers *out,
                  cudaStream_t s);
void free_pattern(PatternBuffers *p, cudaStream_t s);
int csr_drop_zeros(const int64_t *rp, const int32_t *ci, const double *v, int64_t nrows,
                   int64_t *rp_out, int32_t *ci_out, double *v_out, int64_t *nnz_out,
                   cudaStream_t s);

}  // namespace mag
