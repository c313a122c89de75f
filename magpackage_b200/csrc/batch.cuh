// Batched complex assembly: per-instance parameters and launch plumbing (batch.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "common.cuh"
#include "tile.cuh"

namespace mag {

struct BatchInstance {
    ElemData m;
    RowPlan rp;
    const int32_t *block_row;  // row blocks of the variant in use
    const double *nu;          // [Ne]
    const double *sigma;       // [Ne] or NULL (sigma = 1)
    const double *val_ref;     // [18 * nq] reference basis values
    const uint8_t *second;     // per incidence: second-contributor bits, or NULL (row phase only)
    double qw[kMaxQuad];
    int nq;
    int nq4;                   // 4 equal weights
    double omega;
    double *vals;              // complex128 [nnz] as (re, im) pairs
};

struct BatchVariantData {
    void *items = nullptr;
    void *inst = nullptr;
    int nitems = 0;
    int grid = 0;
};

struct BatchState {
    std::vector<BatchInstance> inst_host;
    std::vector<int64_t> inst_ne;
    std::vector<const int32_t *> block_row256, block_row128;
    std::vector<int32_t> nblocks256, nblocks128;
    std::vector<int32_t *> owned;  // block_row128 arrays built for the batch
    BatchVariantData var[4];
    std::vector<TileComplexInput> tile_in;  // the meshes' tile plans (variants 4, 5)
    TileComplexBatch tile;
};

int batch_build(BatchState *b, cudaStream_t s);
int batch_launch(const BatchState &b, int variant, cudaStream_t s);
int batch_num_variants();
bool batch_variant_available(const BatchState &b, int v);
const char *batch_variant_name(int v);
void batch_free_variants(BatchState *b);

}  // namespace mag
