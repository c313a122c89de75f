// Launchers for the assembly kernels (defined in assemble.cu).
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"

namespace mag {

int launch_jacobian_elems(const ElemData &m, const double *sol, const QuadParams &qp,
                          const MaterialParams &mp, int calcj, double *scratch, cudaStream_t s);
int launch_jacobian_seeded_elems(const ElemData &m, const double *sol, const double *bscale, const QuadParams &qp,
                                 const MaterialParams &mp, double *scratch, cudaStream_t s);
int launch_seed_midpoint(const ElemData &m, const double *sol, const double *nu_hat, const MaterialParams &mp,
                         double max_scale, double *bscale, cudaStream_t s);
int launch_stiffness_elems(const ElemData &m, const double *nu, const QuadParams &qp,
                           double *scratch, cudaStream_t s);
int launch_mass_elems(const ElemData &m, const double *sigma, const QuadParams &qp, double *scratch,
                      cudaStream_t s);
int launch_source_elems(const ElemData &m, const double *js, const QuadParams &qp, double *scratch,
                        cudaStream_t s);
// Winding vector (coil region `coil`, direction field [Ne][3] or uniform dir, times scale):
// residual slot of `scratch` and/or the reference's (I, V) pairs (either may be NULL).
int launch_winding_elems(const ElemData &m, int coil, const double *field, const double dir[3], double scale,
                         const QuadParams &qp, double *scratch, double *I, double *V, cudaStream_t s);
int launch_element_b(const ElemData &m, const double *sol, double *b, double *bsq, cudaStream_t s,
                     const MaterialParams *mp = nullptr, double *nu = nullptr, double *dnu = nullptr);
int launch_rows_reduce(const RowPlan &rp, int max_row, const double *scratch, double *vals,
                       double *vec, cudaStream_t s);
int launch_to_triplets(const double *scratch, const int32_t *dofs, int64_t ne, int calcj, double *I,
                       double *J, double *V, double *Ridx, double *Rval, cudaStream_t s);

}  // namespace mag
