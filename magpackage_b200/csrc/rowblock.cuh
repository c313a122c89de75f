// Row-block assembly schedule: plan and launcher (see rowblock.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "common.cuh"

namespace mag {

constexpr int kBlockInc = 256;  // incidences per CTA == threads per CTA

constexpr int kMaxBlockElems = 224;  // distinct elements per 256-incidence block the shared kernel holds
constexpr int kSharedBlockInc = 256; // block size of the shared-element schedule (4 CTAs per SM)
constexpr int kSharedMaxElems = 192; // distinct elements per block (larger blocks are split)
constexpr int kNzMaxSpan = 1024;     // CSR nonzeros per block of the nonzero-pass kernel (larger blocks are split)

struct RowBlockPlan {
    int32_t *block_row = nullptr;  // [nblocks+1]
    int32_t nblocks = 0;
    int64_t bytes = 0;
    int ok = 0;
    int block_inc = 0;
    // shared-element variant: each block's distinct elements, ascending, stored at the
    // block's first incidence offset; per incidence its slot in that list and local row
    int32_t *blk_nelem = nullptr;  // [nblocks]
    int32_t *blk_k0 = nullptr;     // [nblocks+1] first incidence of each block
    int32_t *blk_elem = nullptr;   // [ninc] (first blk_nelem[b] entries after the block's offset)
    uint16_t *inc_slot = nullptr;  // [ninc] slot | local row << 8
    uint32_t *inc_sorted = nullptr; // [ninc] per block in element order: slot | local row << 8 | incidence << 16
                                    // | second-contributor bits << 24 (when nz_ok)
    int shared_ok = 0;
    // nonzero-pass kernel: every off-diagonal CSR entry has at most two contributions and
    // inc_sorted carries, per incidence and local column, whether it is the second of them
    int nz_ok = 0;
};


// Per incidence (row order) bit j: the incidence is the second of the (at most two)
// contributions to its column j's off-diagonal entry. *out = NULL when some row breaks
// that bound (a repeated dof): the nonzero-pass kernels are then unavailable. The
// caller owns and frees the array (ninc bytes).
int build_second_masks(const RowPlan &rp, int64_t ninc, uint8_t **out, cudaStream_t s);
// `second`: the masks above, or NULL (no nonzero-pass plan).
int build_rowblock_plan(const RowPlan &rp, RowBlockPlan *out, cudaStream_t s, int block_inc = kBlockInc,
                        bool with_shared = false, const uint8_t *second = nullptr);
void free_rowblock_plan(RowBlockPlan *p);
int launch_rowblock_jacobian(const RowBlockPlan &bp, const ElemData &m, const RowPlan &rp, const double *sol,
                             const QuadParams &qp, const MaterialParams &mp, int calcj, double *vals,
                             double *res, cudaStream_t s);
// Same result, bit for bit, with each block's distinct elements evaluated once
// (standard curl table only; needs bp.shared_ok).
int launch_rowblock_shared_jacobian(const RowBlockPlan &bp, const ElemData &m, const RowPlan &rp,
                                    const double *sol, const QuadParams &qp, const MaterialParams &mp, int calcj,
                                    double *vals, double *res, cudaStream_t s);
// Same result, bit for bit: shared-element blocks whose off-diagonal entries are placed
// by the incidences themselves and stored by one pass over the block's nonzeros; only
// the diagonal and the residual are summed per row (needs bp.nz_ok).
int launch_rowblock_nz_jacobian(const RowBlockPlan &bp, const ElemData &m, const RowPlan &rp, const double *sol,
                                const QuadParams &qp, const MaterialParams &mp, int calcj, double *vals,
                                double *res, cudaStream_t s);
// The curl-curl matrix K(nu) (per-element reluctivity nu [Ne]) with the same kernel: bit for
// bit the two-pass stiffness assembly, one launch, no scratch (needs bp.nz_ok).
int launch_rowblock_nz_stiffness(const RowBlockPlan &bp, const ElemData &m, const RowPlan &rp, const double *nu,
                                 const QuadParams &qp, double *vals, cudaStream_t s);

}  // namespace mag
