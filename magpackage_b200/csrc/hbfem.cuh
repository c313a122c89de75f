// Harmonic-balance assembly (hbfem.cu).
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"

namespace mag {

constexpr int kMaxHarm = 16;  // harmonics per call

int launch_hbfem(const ElemData &m, const RowPlan &rp, int max_row, const double *sr, const double *si, int K,
                 const double *dr, const double *di, const double *pr, const double *pi, int N,
                 const QuadParams &qp, const MaterialParams &mp, double *scratch, double *rscr, double *vals,
                 double *out_re, double *out_im, cudaStream_t s);

}  // namespace mag
