// Fused single-launch assembly: plan and launcher.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "common.cuh"

namespace mag {

// Static schedule for one persistent cooperative launch. Items are processed
// by CTA b in the order b, b+G, b+2G, ... Item codes: >= 0 an element tile,
// < 0 a CSR row chunk (-1 - chunk). Every wait points at earlier items only.
struct FusedPlan {
    int32_t *sched = nullptr;      // [nitems] item codes in schedule order
    int32_t *need = nullptr;       // [nitems] every item before this position must be done first
    int32_t *ctrl = nullptr;       // error word + per-CTA progress counters
    double *ring = nullptr;        // [ring * kTileElems * kScratchPerElem]
    int32_t nitems = 0, ntiles = 0, nchunks = 0, ring_tiles = 0, grid = 0;
    size_t ctrl_bytes = 0;
    int64_t bytes = 0;
    int ok = 0;
};

constexpr int kTileElems = 256;     // elements per tile == threads per CTA
constexpr int kChunkRows = 32;      // CSR rows per chunk
constexpr int kCtrlHeader = 32;     // ints before the progress counters
constexpr double kLagWaves = 4.0;   // dependency distance, in waves of one item per CTA
constexpr long long kSpinLimit = 1LL << 20;  // polls (each >= ~1 us) before a wait gives up

int build_fused_plan(const ElemData &m, const RowPlan &rp, int max_row, FusedPlan *fp, cudaStream_t s);
void free_fused_plan(FusedPlan *fp);
// op: 0 Jacobian+residual, 1 residual only
int launch_fused_jacobian(const FusedPlan &fp, const ElemData &m, const RowPlan &rp, const double *sol,
                          const QuadParams &qp, const MaterialParams &mp, int calcj, double *vals,
                          double *res, cudaStream_t s);
// reads the error word (synchronises s)
int fused_status(const FusedPlan &fp, cudaStream_t s);

}  // namespace mag
