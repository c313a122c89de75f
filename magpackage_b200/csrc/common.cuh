// Shared definitions for the sm_100a assembly library (libmagasm).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>

#include "magasm.h"

namespace mag {

// Thread-local error text behind mag_last_error().
void set_error(const char *fmt, ...);

#define MAG_CUDA_TRY(expr)                                                              \
    do {                                                                                \
        cudaError_t e__ = (expr);                                                       \
        if (e__ != cudaSuccess) {                                                       \
            ::mag::set_error("%s:%d: %s: %s", __FILE__, __LINE__, #expr,                \
                             cudaGetErrorString(e__));                                  \
            return MAG_E_CUDA;                                                          \
        }                                                                               \
    } while (0)

#define MAG_TRY(expr)               \
    do {                            \
        int r__ = (expr);           \
        if (r__ != MAG_OK) return r__; \
    } while (0)

constexpr int kMaxQuad = 16;
constexpr int kMaxMaterials = 255;   // tags are stored as uint8
constexpr int kScratchStride = 8;    // doubles per (element, local row): K row (6), R, pad
constexpr int kScratchPerElem = 6 * kScratchStride;
constexpr int kCompactMaxRow = 31;   // 5-bit in-row positions; 31 marks "no dof"
constexpr int kWideMaxRow = 255;     // 8-bit positions; 255 marks "no dof"

// Local edges (1,2),(1,3),(1,4),(2,3),(2,4),(3,4) of src/Mesh.m:118.
__host__ __device__ constexpr int edge_a(int k) { return k < 3 ? 0 : (k < 5 ? 1 : 2); }
__host__ __device__ constexpr int edge_b(int k) { return k == 0 ? 1 : (k == 1 || k == 3) ? 2 : 3; }

// Quadrature / reference basis, passed by value to kernels.
struct QuadParams {
    int nq;
    int uniform_w;      // all Qw equal
    int standard_curl;  // CurlRef equals the nedelec_tet_p1 table at every point
    double qw[kMaxQuad];
    const double *curl_ref;  // device [18 * nq], entry (i, c, q) at i + 6c + 18q
    const double *val_ref;   // device [18 * nq]
};

// Material tables in device memory (layout of Assembler.packMaterialData).
struct MaterialParams {
    int nmat;
    int nbreaks;
    int ncoefs;
    const double *lin;
    const double *is_non;
    const double *max_bsq;
    const double *breaks;
    const double *coefs;
    const int *start;
    const int *count;
    const int *coef_start;
    // Optional windows of the spline search (NULL: binary search over the whole table): per
    // material kMatBuckets buckets uniform in s = |B|^2 from origin = the first break to
    // MaxBSq; bucket[2 kMatBuckets m + i] and bucket[2 kMatBuckets m + kMatBuckets + i] are the
    // window of bucket i; bucket_geom[2m], [2m + 1] = origin, scale (buckets per unit of s;
    // 0 = this material has no buckets).
    const int *bucket;
    const double *bucket_geom;
};

constexpr int kMatBuckets = 256;

// Element-side mesh data in the handle's layout.
struct ElemData {
    const double4 *xyz;       // [Nn] (x, y, z, 0)
    const int4 *tet;          // [Ne] 0-based nodes
    const int32_t *dofs;      // [Ne][6] 0-based, -1 = none
    const uint8_t *tags;      // [Ne] 1-based material tags
    const uint8_t *signbits;  // [Ne] bit k set = sign -1; NULL = derive from tet
    int64_t ne;
};

// Row-side (CSR) plan.
struct RowPlan {
    const int32_t *row_ptr;   // [ndof+1]
    const int32_t *inc_ptr;   // [ndof+1]
    const uint32_t *inc_elem; // [ninc] element | local row << 29
    const uint32_t *inc_pos;  // [ninc] compact: 6 x 5-bit positions; wide: [ninc][2] 6 x 8-bit
    int64_t ndof;
    int wide;
};

}  // namespace mag
