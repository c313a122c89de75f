// Tile-block assembly schedule: plan and launcher (see tile.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "common.cuh"

namespace mag {

constexpr int kTileMaxNnz = 8191;   // CSR nonzeros per block (13-bit offsets in the row table)
constexpr int kTileMaxInc = 4095;   // (row, element) incidences per block (12-bit offsets)
constexpr int kTileMaxColors = 8;   // element colour classes per block
constexpr int kTileChunk = 256;     // nonzeros per store chunk (one warp stores a chunk)
constexpr int kTileSlotPad = 32;    // doubles of slack after a block's values in shared memory (even):
                                    // a row's first nonzero plus any 5-bit position stays inside
constexpr int kTileVariants = 4;    // launch shapes of the Jacobian kernel (tile_variant_name)
constexpr int kTileDepths = 3;      // L2 staging depths, in waves of resident CTAs (0, 1, 2)
constexpr uint32_t kTileAbsent = 0xFFFFFFFFu;

// One CTA's work: whole CSR rows whose edges start in one spatial tile of nodes, and
// every element incident to those rows, in colour classes.
struct TileBlock {
    int32_t row0, nrows;        // entries of TilePlan::rows
    int32_t rec0, nrec;         // records (elements of the block, sorted by colour then id)
    int32_t chunk0, nchunks;    // store chunks
    int32_t nnz, ninc;          // shared-memory extents
    int32_t ncolors;
    int32_t col_end[kTileMaxColors];  // record count at the end of each colour class
    int32_t pad[3];
};
static_assert(sizeof(TileBlock) == 80, "TileBlock layout");

// Device plan. Records are 96 bytes in six 16-byte planes (plane k of record i at
// recs[k * nrec_total + i]) so that a warp's loads of one plane are contiguous:
//   plane 0: tet (4 node ids)
//   plane 1: dofs 0..3
//   plane 2: dofs 4, 5, element id, tag | sign bits << 8
//   plane 3: per local row 0..3 its six 5-bit in-row column positions (a column without a
//            dof holds the row's diagonal position: the value added there is overwritten)
//   plane 4: positions of local rows 4, 5; slots of local rows 0, 1
//   plane 5: slots of local rows 2..5
// where a slot is (row's first nonzero in the block) | (incidence slot << 16), or
// kTileAbsent when the row is not one of the block's.
// rows: per block row (ascending ids) x = global row, y = nonzero base (13 bits) |
// incidence base (12 bits) << 13 | diagonal position (5 bits) << 25.
// chunks: x = block nonzero base | length << 16, y = global nonzero base.
struct TilePlan {
    TileBlock *blocks = nullptr;
    uint2 *rows = nullptr;
    uint2 *chunks = nullptr;
    uint4 *recs = nullptr;
    int32_t nblocks = 0;
    int64_t nrows = 0, nchunks = 0, nrec = 0, nnz = 0;
    int32_t max_nnz = 0, max_inc = 0, max_colors = 0, max_rows = 0, max_chunks = 0;
    double evals_per_elem = 0.0;  // records / elements
    double build_ms = 0.0;
    int64_t bytes = 0;
    int ok = 0;
    int variant = 0;  // launch shape of the Newton Jacobian (0 .. kTileVariants-1)
    int prefetch_waves = 1;  // staging depth: a CTA prefetches the block this many waves ahead (0: none)
};

struct TilePlanInput {
    const double4 *xyz;      // device [Nn]
    const int4 *tet;         // device [Ne]
    const int32_t *dofs;     // device [Ne][6]
    const uint8_t *tags;     // device [Ne]
    const uint8_t *signbits; // device [Ne] or NULL (derived from tet)
    const int32_t *row_ptr, *inc_ptr;
    const uint32_t *inc_elem, *inc_pos;
    int64_t nn, ne, ndof, nnz, ninc;
    int wide;
};

// Host copies of what the planner reads (the device mesh and incidence plan).
struct TileHostMesh {
    std::vector<double4> xyz;
    std::vector<int4> tet;
    std::vector<int32_t> dofs, row_ptr, inc_ptr;
    std::vector<uint8_t> tags, sbits;  // sbits empty: signs derived from tet
    std::vector<uint32_t> inc_elem, inc_pos;
    int64_t nnz = 0;
};

// The plan's arrays on the host, in the device layout.
struct TileHostPlan {
    std::vector<TileBlock> blocks;
    std::vector<uint2> rows, chunks;
    std::vector<uint4> planes;  // 6 * nrec
    int64_t nrec = 0;
    int32_t max_nnz = 0, max_inc = 0, max_colors = 0, max_rows = 0, max_chunks = 0;
};

// The planner itself (host only): false when the mesh does not suit the schedule.
bool plan_tiles_host(const TileHostMesh &hm, TileHostPlan *out);

// Builds the plan on the host from the mesh's incidence plan (copied down once).
// Leaves plan->ok = 0 (and returns MAG_OK) when the mesh does not suit the schedule:
// wide rows (> 31 entries), an off-diagonal entry with more than two contributions
// (repeated dofs), or a block needing more than kTileMaxColors colours.
int build_tile_plan(const TilePlanInput &in, TilePlan *plan, cudaStream_t s);
void free_tile_plan(TilePlan *plan);

// Jacobian (calc_j) and residual; vals may be NULL when !calc_j.
int launch_tile_jacobian(const TilePlan &tp, const ElemData &m, const double *sol, const QuadParams &qp,
                         const MaterialParams &mp, int calc_j, double *vals, double *res, int *err,
                         cudaStream_t s);
// Jacobian with a seeded tangent (mag_assemble_jacobian_seeded): residual at the state,
// tangent at the flux density scaled by bscale [Ne].
int launch_tile_seeded(const TilePlan &tp, const ElemData &m, const double *sol, const double *bscale,
                       const QuadParams &qp, const MaterialParams &mp, double *vals, double *res, int *err,
                       cudaStream_t s);
const char *tile_variant_name(int v);

// Batched complex assembly A_i = K_i(nu_i) + j omega_i M_i(sigma_i) over the tile blocks of
// many meshes: one CTA per (mesh, block) item; K pass then, where the block holds a
// conducting element, M pass over the same shared-memory slots.
struct TileComplexInput {
    const TilePlan *tp;
    ElemData m;
    QuadParams qp;
    const double *nu;     // [Ne]
    const double *sigma;  // [Ne] or NULL (sigma = 1 everywhere)
    double omega;
    double *vals;         // complex128 [nnz] as (re, im) pairs
    int *err;             // the mesh's status word
};

constexpr int kTileComplexVariants = 2;

struct TileComplexBatch {
    void *inst = nullptr;   // device array of the per-mesh launch arguments
    int2 *items = nullptr;  // device (mesh, block), larger meshes first
    int nitems = 0, q4 = 0;
    int smem_nnz = 0, smem_inc = 0, smem_rows = 0, smem_chunks = 0;
    size_t smem = 0;
    int ahead[kTileComplexVariants] = {0, 0};  // CTAs resident at once per launch shape
    int ok = 0;
};

// Builds the work queue; leaves b->ok = 0 (and returns MAG_OK) when some mesh has no tile
// plan or a non-standard curl table.
int build_tile_complex(const std::vector<TileComplexInput> &in, TileComplexBatch *b, cudaStream_t s);
int launch_tile_complex(const TileComplexBatch &b, int variant, cudaStream_t s);
const char *tile_complex_variant_name(int v);
void free_tile_complex(TileComplexBatch *b);
// K(nu) with per-element reluctivity nu [Ne].
int launch_tile_stiffness(const TilePlan &tp, const ElemData &m, const double *nu, const QuadParams &qp,
                          double *vals, int *err, cudaStream_t s);

}  // namespace mag
