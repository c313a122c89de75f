// Row-block assembly schedule: plan and launcher (see rowblock.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "common.cuh"

namespace mag {

constexpr int kBlockInc = 256;  // incidences per CTA == threads per CTA

struct RowBlockPlan {
    int32_t *block_row = nullptr;  // [nblocks+1]
    int32_t nblocks = 0;
    int64_t bytes = 0;
    int ok = 0;
};

int build_rowblock_plan(const RowPlan &rp, RowBlockPlan *out, cudaStream_t s, int block_inc = kBlockInc);
void free_rowblock_plan(RowBlockPlan *p);
int launch_rowblock_jacobian(const RowBlockPlan &bp, const ElemData &m, const RowPlan &rp, const double *sol,
                             const QuadParams &qp, const MaterialParams &mp, int calcj, double *vals,
                             double *res, cudaStream_t s);

}  // namespace mag
