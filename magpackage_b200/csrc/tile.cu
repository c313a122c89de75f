// Tile-block Newton-Jacobian assembly (FP64, sm_100a): one launch, no scratch in HBM,
// each element evaluated by one thread, about 1.5 times per assembly.
//
// Rows (edges) are grouped by the spatial tile of their lower node: nodes are binned
// into coordinate layers along x, y and z, and 4 x 4 x 4 layers make a tile (a CTA
// block holds at most kTileMaxNnz nonzeros and kTileMaxInc incidences; larger tiles
// are cut). A CTA takes one block: its CSR rows, and every element incident to them.
//   colour phases -- one thread per element evaluates geometry, the six curls, B and
//              nu(|B|^2) once (the reference's arithmetic), then, for each of its local
//              rows that belongs to the block, the row of the 6x6 tangent and the
//              residual entry. Off-diagonal entries go straight into the block's
//              shared-memory copy of its CSR values as slot = slot + v. An
//              off-diagonal entry has at most two contributions (the two tetrahedra
//              that share a face) and (0 + a) + b equals (0 + b) + a bit for bit, so
//              the order does not matter, only that the two updates never overlap:
//              the plan colours the block's elements so that no two elements of a
//              colour share an entry (the face-adjacency graph of a Kuhn mesh is
//              bipartite: two colours), and the colours run one after another.
//              Diagonal entries and residual entries go to per-incidence slots.
//   row phase -- one thread per row sums its diagonal and residual contributions in
//              ascending element order (the reference's sparse() order).
//   store phase -- the block's rows form runs of consecutive rows, contiguous in the
//              CSR; warps store them in chunks, coalesced.
// No floating-point atomics; results equal the reference's MEX + sparse() bit for bit.
#include <omp.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "element.cuh"
#include "tile.cuh"

// Node layers per tile along z (x and y: 4); a build option (-DMAG_TILE_LAYERS_Z=n).
#ifndef MAG_TILE_LAYERS_Z
#define MAG_TILE_LAYERS_Z 4
#endif
// Order a colour's records by the rows they hold in the block (build option).
#ifndef MAG_TILE_SORT_ROWS
#define MAG_TILE_SORT_ROWS 0
#endif

namespace mag {

namespace {

using namespace elem;

struct TileArgs {
    const TileBlock *blocks;
    const uint2 *rows;
    const uint2 *chunks;
    const uint4 *recs;
    int64_t nrec;
    const double4 *xyz;
    const double *sol;
    const double *nu_e;    // K(nu): per-element reluctivity
    const double *bscale;  // seeded Jacobian: per-element flux-density scale of the tangent
    QuadParams qp;
    MaterialParams mp;
    double *vals;
    double *res;
    int *err;
    int64_t nnz_total, ndof;
    int smem_nnz;  // doubles reserved for the block's values (even)
    int smem_inc, smem_rows, smem_chunks;  // incidence slots, row-table and chunk entries reserved
};

// Sum over the quadrature points of v * w_q (w_q = qw_q |det J|) from zero, in point
// order. Q4: four equal weights, u = v w_0; the reference's ((u + u) + u) + u equals
// (3 u) + u because u + u is exact, so 3 u rounds like (u + u) + u.
template <bool Q4>
__device__ __forceinline__ double qsum4(double v, const QuadParams &qp, double w0, double adet) {
    const double u = v * w0;
    if (Q4) {
        const double t = 3.0 * u;
        return t + u;
    }
    double acc = u;
    if (qp.uniform_w) {
        for (int q = 1; q < qp.nq; q++) acc = acc + u;
    } else {
        for (int q = 1; q < qp.nq; q++) acc = acc + v * (qp.qw[q] * adet);
    }
    return acc;
}

__device__ __forceinline__ void flag(int *err) { atomicOr(err, 1); }

enum TileMode { kJacobian = 0, kStiffness = 1, kSeeded = 2 };

// One element of the block: record i.
//   kJacobian: residual and tangent at the element's state (assemble_jacobian_kernel_mex.cpp:92-131);
//   kStiffness: K(nu) with the element's given nu (assemble_curl_curl_kernel_mex.cpp:94-101), no residual;
//   kSeeded: residual at B, tangent at the seeded state beta B:
//            nu(|beta B|^2) Ci.Cj + 2 nu'(|beta B|^2) (beta B.Ci)(beta B.Cj), the operation order of
//            the two-pass seeded kernel.
// FIRST: the block's first colour class. Its slots are all still +0 (no element of the
// class shares one), so an entry is stored rather than added: slot = v instead of
// slot = 0 + v, the same value up to the sign of an exact zero, which the store phase
// normalises (x + 0 turns -0 into +0 and leaves every other value unchanged).
template <bool CALCJ, bool Q4, int MODE, bool FIRST = false>
__device__ __forceinline__ void tile_element(const TileArgs &A, int64_t i, double *__restrict__ slot,
                                             double2 *__restrict__ incv, int bnnz, int binc) {
    const int64_t n = A.nrec;
    const uint4 p0 = __ldg(A.recs + i), p1 = __ldg(A.recs + n + i), p2 = __ldg(A.recs + 2 * n + i);
    const uint4 p3 = __ldg(A.recs + 3 * n + i), p4 = __ldg(A.recs + 4 * n + i), p5 = __ldg(A.recs + 5 * n + i);
    const int4 tt = make_int4((int)p0.x, (int)p0.y, (int)p0.z, (int)p0.w);
    const unsigned sb = (p2.w >> 8) & 0x3Fu;
    const unsigned pos[6] = {p3.x, p3.y, p3.z, p3.w, p4.x, p4.y};
    const unsigned sl[6] = {p4.z, p4.w, p5.x, p5.y, p5.z, p5.w};
    Geo g;
    geometry(A.xyz, tt, g);
    double C[6][3];
    curls_standard(g, C);
    // Orientation signs folded into the curls (C_j s_j): negation is exact and commutes with
    // rounding to nearest, so B = sum a_j C_j is the same bits with unsigned edge values, and
    // every entry below comes out as s_l s_j times the unsigned one, which is how the
    // reference signs its finished entries. Only the sign of an exact zero can differ, and
    // every sum these entries enter starts from +0, which absorbs it.
#pragma unroll
    for (int j = 0; j < 6; j++)
        if ((sb >> j) & 1u) {
            C[j][0] = -C[j][0];
            C[j][1] = -C[j][1];
            C[j][2] = -C[j][2];
        }
    constexpr bool STIFF = MODE == kStiffness;
    double nu, g2 = 0.0, b[6];
    double nut = 0.0, be = 1.0;  // seeded tangent: nu(|beta B|^2), beta
    if (STIFF) {
        nu = __ldg(A.nu_e + p2.z);
#pragma unroll
        for (int j = 0; j < 6; j++) b[j] = 0.0;
    } else {
        const int d[6] = {(int)p1.x, (int)p1.y, (int)p1.z, (int)p1.w, (int)p2.x, (int)p2.y};
        double a[6];
#pragma unroll
        for (int k = 0; k < 6; k++) a[k] = d[k] >= 0 ? __ldg(A.sol + d[k]) : 0.0;  // signs in C
        double B[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            double v = a[0] * C[0][c];
#pragma unroll
            for (int k = 1; k < 6; k++) v = v + a[k] * C[k][c];
            B[c] = v;
        }
        double dnu;
        material_eval(A.mp, (int)(p2.w & 0xFFu), dot3(B, B), nu, dnu);
#pragma unroll
        for (int j = 0; j < 6; j++) b[j] = dot3(B, C[j]);
        g2 = 2.0 * dnu;
        if (MODE == kSeeded && CALCJ) {
            be = __ldg(A.bscale + p2.z);
            double dnut;
            material_eval(A.mp, (int)(p2.w & 0xFFu), (be * be) * dot3(B, B), nut, dnut);
            g2 = 2.0 * dnut;
        }
    }
    const double adet = g.adet, w0 = A.qp.qw[0] * adet;
#pragma unroll
    for (int l = 0; l < 6; l++) {
        const unsigned s = sl[l];
        if (s == kTileAbsent) continue;
        const int nzb = (int)(s & 0xFFFFu), is = (int)(s >> 16);
        // One check per row: the slot region has kTileSlotPad doubles beyond the largest
        // block, so nzb < bnnz keeps every nzb + p (p <= 30) inside it.
        if (nzb >= bnnz) {
            flag(A.err);
            continue;
        }
        const double rv = STIFF ? 0.0 : qsum4<Q4>(nu * b[l], A.qp, w0, adet);  // signed through C
        double dv = 0.0;
        if (CALCJ) {
            // the row's six entries first, then its five off-diagonal updates (the six
            // independent chains of arithmetic overlap; placing each entry as it is formed
            // measured slower)
            double v[6];
            if (MODE == kSeeded) {
                const double gl = g2 * (be * b[l]);
#pragma unroll
                for (int j = 0; j < 6; j++)
                    v[j] = qsum4<Q4>(nut * dot3(C[l], C[j]) + gl * (be * b[j]), A.qp, w0, adet);
            } else if (g2 == 0.0) {
#pragma unroll
                for (int j = 0; j < 6; j++) v[j] = qsum4<Q4>(nu * dot3(C[l], C[j]), A.qp, w0, adet);
            } else {
                const double gl = g2 * b[l];
#pragma unroll
                for (int j = 0; j < 6; j++) v[j] = qsum4<Q4>(nu * dot3(C[l], C[j]) + gl * b[j], A.qp, w0, adet);
            }
            dv = v[l];
#pragma unroll
            for (int j = 0; j < 6; j++) {
                if (j == l) continue;
                const int k = nzb + (int)((pos[l] >> (5 * j)) & 31u);  // absent column: the diagonal
                if (FIRST) slot[k] = v[j];
                else slot[k] = slot[k] + v[j];
            }
        }
        if (is < binc) {
            incv[is] = make_double2(rv, dv);
        } else {
            flag(A.err);
        }
    }
}

// L2 prefetch of [p, p + bytes) (16-byte aligned start and length; the plan's arrays are
// padded so that the rounded range stays inside them).
__device__ __forceinline__ void l2_prefetch(const void *p, size_t bytes) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    const uintptr_t lo = a & ~uintptr_t(15), hi = (a + bytes + 15) & ~uintptr_t(15);
    if (hi > lo)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(lo), "r"((uint32_t)(hi - lo)) : "memory");
}

// What a block's next CTA visit will read first: its descriptor, records (six planes), rows
// and chunks.
__device__ __forceinline__ void prefetch_block(const TileArgs &A, int b) {
    const TileBlock *Bp = A.blocks + b;
    l2_prefetch(Bp, sizeof(TileBlock));
    const int rec0 = Bp->rec0, nrec = Bp->nrec;
    for (int k = 0; k < 6; k++) l2_prefetch(A.recs + (int64_t)k * A.nrec + rec0, (size_t)nrec * sizeof(uint4));
    l2_prefetch(A.rows + Bp->row0, (size_t)Bp->nrows * sizeof(uint2));
    l2_prefetch(A.chunks + Bp->chunk0, (size_t)Bp->nchunks * sizeof(uint2));
}

// 8-byte asynchronous global -> shared copies (both addresses 8-byte aligned).
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// One CTA per block. The CTA of block b prefetches into L2 the records of block b + ahead
// (ahead = the CTAs resident at once), the block the hardware starts about when b ends.
// The block's row table and store chunks are copied into shared memory while its
// elements run, so the row and store phases start without a global round trip.
template <int BT, int MINB, bool CALCJ, bool Q4, int MODE>
__global__ void __launch_bounds__(BT, MINB) k_tile(TileArgs A, int nblocks, int ahead) {
    constexpr bool STIFF = MODE == kStiffness;
    extern __shared__ __align__(16) double tile_smem[];
    double *slot = tile_smem;
    double2 *incv = reinterpret_cast<double2 *>(tile_smem + A.smem_nnz);
    uint2 *srows = reinterpret_cast<uint2 *>(incv + A.smem_inc);
    uint2 *schunks = srows + A.smem_rows;
    const int tid = threadIdx.x;
    {
        const int blk = blockIdx.x;
        if (tid == 0 && blk + ahead < nblocks) prefetch_block(A, blk + ahead);
        const TileBlock *Bp = A.blocks + blk;
        const int nrows = Bp->nrows, row0 = Bp->row0, rec0 = Bp->rec0, nrec = Bp->nrec;
        const int nnz = Bp->nnz, ninc = Bp->ninc, ncolors = Bp->ncolors;
        const int chunk0 = Bp->chunk0, nchunks = Bp->nchunks;
        if (nrows > A.smem_rows || nchunks > A.smem_chunks || nnz > A.smem_nnz - kTileSlotPad || ninc > A.smem_inc) {
            if (tid == 0) flag(A.err);  // the whole CTA leaves before its first barrier
            return;
        }
        for (int i = tid; i < nrows; i += BT) cp_async8(srows + i, A.rows + row0 + i);
        if (CALCJ)
            for (int i = tid; i < nchunks; i += BT) cp_async8(schunks + i, A.chunks + chunk0 + i);
        cp_async_commit();
        if (CALCJ) {
            for (int i = tid; i < (nnz + 1) / 2; i += BT)  // 16-byte stores; an odd tail's pair ends in the pad
        reinterpret_cast<double2 *>(slot)[i] = make_double2(0.0, 0.0);
            __syncthreads();
            int c0 = 0;
            for (int c = 0; c < ncolors; c++) {
                const int c1 = Bp->col_end[c];
                if (c == 0)
                    for (int i = c0 + tid; i < c1; i += BT)
                        tile_element<CALCJ, Q4, MODE, true>(A, (int64_t)rec0 + i, slot, incv, nnz, ninc);
                else
                    for (int i = c0 + tid; i < c1; i += BT)
                        tile_element<CALCJ, Q4, MODE>(A, (int64_t)rec0 + i, slot, incv, nnz, ninc);
                c0 = c1;
                if (c + 1 == ncolors) cp_async_wait_all();
                __syncthreads();
            }
            if (ncolors == 0) {
                cp_async_wait_all();
                __syncthreads();
            }
        } else {
            for (int i = tid; i < nrec; i += BT)
                tile_element<CALCJ, Q4, MODE>(A, (int64_t)rec0 + i, slot, incv, nnz, ninc);
            cp_async_wait_all();
            __syncthreads();
        }
        // rows: diagonal and residual in ascending element order
        for (int r = tid; r < nrows; r += BT) {
            const uint2 rw = srows[r];
            const int nzb = (int)(rw.y & 0x1FFFu), incb = (int)((rw.y >> 13) & 0xFFFu);
            const int diag = (int)((rw.y >> 25) & 31u);
            int ince = r + 1 < nrows ? (int)((srows[r + 1].y >> 13) & 0xFFFu) : ninc;
            if (ince > ninc) ince = ninc;
            double racc = 0.0, dacc = 0.0;
            for (int k = incb; k < ince; k++) {
                const double2 v = incv[k];
                racc = racc + v.x;
                if (CALCJ) dacc = dacc + v.y;
            }
            if (!STIFF) {
                if ((int64_t)rw.x < A.ndof) A.res[rw.x] = racc;
                else flag(A.err);
            }
            if (CALCJ && ince > incb) {
                if (nzb + diag < nnz) slot[nzb + diag] = dacc;
                else flag(A.err);
            }
        }
        __syncthreads();
        if (CALCJ) {
            const int warp = tid >> 5, lane = tid & 31;
            for (int c = warp; c < nchunks; c += BT / 32) {
                const uint2 ch = schunks[c];
                const int sb0 = (int)(ch.x & 0xFFFFu), len = (int)(ch.x >> 16);
                const int64_t g = (int64_t)ch.y;
                if (sb0 + len > nnz || g + len > A.nnz_total) {
                    if (lane == 0) flag(A.err);
                    continue;
                }
                for (int i = lane; i < len; i += 32) A.vals[g + i] = slot[sb0 + i] + 0.0;  // -0 -> +0
            }
        }
    }
}

// ---- batched complex assembly: K(nu) + j omega M(sigma) over many meshes ------------

struct TileComplexInstance {
    TileArgs a;              // the mesh's plan, coordinates, nu (nu_e), quadrature, error word
    const double *sigma;     // [Ne] or NULL (sigma = 1)
    const double *val_ref;   // [18 * nq] reference basis values, entry (i, c, q) at i + 6c + 18q
    double omega;
    double *cvals;           // complex128 [nnz] as (re, im)
};

// The sigma-mass rows of one element of the block (assemble_mass_kernel_mex.cpp:186-230):
// per local row l, m_j = sum_q ((N_l . N_j) sigma) w_q with N = J^{-T} N_ref at each point,
// signed; off-diagonal entries into their nonzeros' slots, the diagonal into the
// incidence slot's x. Elements with |sigma| <= 1e-12 add nothing (the reference skips
// them; a skipped contribution and a +0 one give the same sums).
__device__ __forceinline__ void tile_mass_element(const TileComplexInstance &I, int64_t i, double *__restrict__ slot,
                                                  double2 *__restrict__ incv, int bnnz, int binc,
                                                  const double *__restrict__ sval) {
    const TileArgs &A = I.a;
    const int64_t n = A.nrec;
    const uint4 p2 = __ldg(A.recs + 2 * n + i);
    const double sigma = I.sigma ? __ldg(I.sigma + p2.z) : 1.0;
    if (!(fabs(sigma) > 1e-12)) return;
    const uint4 p0 = __ldg(A.recs + i), p3 = __ldg(A.recs + 3 * n + i), p4 = __ldg(A.recs + 4 * n + i),
                p5 = __ldg(A.recs + 5 * n + i);
    const int4 tt = make_int4((int)p0.x, (int)p0.y, (int)p0.z, (int)p0.w);
    const unsigned sb = (p2.w >> 8) & 0x3Fu;
    const unsigned pos[6] = {p3.x, p3.y, p3.z, p3.w, p4.x, p4.y};
    const unsigned sl[6] = {p4.z, p4.w, p5.x, p5.y, p5.z, p5.w};
    Geo g;
    geometry(A.xyz, tt, g);
    double iv[3][3];
    inverse3(g, iv);
    const int nq = A.qp.nq;
#pragma unroll
    for (int l = 0; l < 6; l++) {
        const unsigned s = sl[l];
        if (s == kTileAbsent) continue;
        const int nzb = (int)(s & 0xFFFFu), is = (int)(s >> 16);
        if (nzb >= bnnz) {  // one check per row (kTileSlotPad)
            flag(A.err);
            continue;
        }
        const unsigned si = (sb >> l) & 1u;
        double m[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll 1
        for (int q = 0; q < nq; q++) {
            const double w = A.qp.qw[q] * g.adet;
            const double *r = sval + 18 * q;
            double Nl[3];
#pragma unroll
            for (int c = 0; c < 3; c++) Nl[c] = iv[0][c] * r[l] + iv[1][c] * r[l + 6] + iv[2][c] * r[l + 12];
#pragma unroll
            for (int j = 0; j < 6; j++) {
                double Nj[3];
#pragma unroll
                for (int c = 0; c < 3; c++) Nj[c] = iv[0][c] * r[j] + iv[1][c] * r[j + 6] + iv[2][c] * r[j + 12];
                m[j] = m[j] + dot3(Nl, Nj) * sigma * w;
            }
        }
#pragma unroll
        for (int j = 0; j < 6; j++) {
            if (j == l) continue;
            const int k = nzb + (int)((pos[l] >> (5 * j)) & 31u);  // absent column: the diagonal
            slot[k] = slot[k] + flip(m[j], si ^ ((sb >> j) & 1u));
        }
        if (is < binc) incv[is].x = m[l];  // the diagonal: si ^ si = 0, no flip
        else flag(A.err);
    }
}

// Sums each row's diagonal contributions (incidence slots, component x or y) in ascending
// element order into the row's diagonal nonzero.
template <int BT, bool COMP_Y>
__device__ __forceinline__ void tile_rows_diag(const uint2 *srows, int nrows, const double2 *incv, int ninc,
                                               double *slot, int nnz, int *err) {
    for (int r = threadIdx.x; r < nrows; r += BT) {
        const uint2 rw = srows[r];
        const int nzb = (int)(rw.y & 0x1FFFu), incb = (int)((rw.y >> 13) & 0xFFFu);
        const int diag = (int)((rw.y >> 25) & 31u);
        int ince = r + 1 < nrows ? (int)((srows[r + 1].y >> 13) & 0xFFFu) : ninc;
        if (ince > ninc) ince = ninc;
        double dacc = 0.0;
        for (int k = incb; k < ince; k++) dacc = dacc + (COMP_Y ? incv[k].y : incv[k].x);
        if (ince > incb) {
            if (nzb + diag < nnz) slot[nzb + diag] = dacc;
            else flag(err);
        }
    }
}

// One CTA per (mesh, block) item. K pass: the tile kernel's K(nu) elements (incidence
// slots get (0, K diagonal)), row sums, real parts stored. M pass, only when some element
// of the block conducts: slots zeroed again, the conducting elements' M rows, row sums,
// imaginary parts stored as omega * M; otherwise the imaginary parts are omega * 0.
// Values equal (K_ab, omega * M_ab) of MATLAB's K + 1j*omega*M (FrequencySolver.m:131).
template <int BT, int MINB, bool Q4>
__global__ void __launch_bounds__(BT, MINB)
    k_tile_complex(const TileComplexInstance *__restrict__ inst, const int2 *__restrict__ items, int nitems,
                   int ahead, int smem_nnz, int smem_inc, int smem_rows, int smem_chunks) {
    extern __shared__ __align__(16) double tile_smem[];
    double *slot = tile_smem;
    double2 *incv = reinterpret_cast<double2 *>(tile_smem + smem_nnz);
    uint2 *srows = reinterpret_cast<uint2 *>(incv + smem_inc);
    uint2 *schunks = srows + smem_rows;
    double *sval = reinterpret_cast<double *>(schunks + smem_chunks);
    const int tid = threadIdx.x;
    const int it = blockIdx.x;
    if (tid == 0 && it + ahead < nitems) {
        const int2 nx = items[it + ahead];
        prefetch_block(inst[nx.x].a, nx.y);
    }
    const int2 w = items[it];
    const TileComplexInstance &I = inst[w.x];
    const TileArgs &A = I.a;
    const TileBlock *Bp = A.blocks + w.y;
    const int nrows = Bp->nrows, row0 = Bp->row0, rec0 = Bp->rec0;
    const int nnz = Bp->nnz, ninc = Bp->ninc, ncolors = Bp->ncolors;
    const int chunk0 = Bp->chunk0, nchunks = Bp->nchunks;
    const int nq = A.qp.nq;
    if (nrows > smem_rows || nchunks > smem_chunks || nnz > smem_nnz - kTileSlotPad || ninc > smem_inc ||
        nq > kMaxQuad) {
        if (tid == 0) flag(A.err);  // the whole CTA leaves before its first barrier
        return;
    }
    for (int i = tid; i < nrows; i += BT) cp_async8(srows + i, A.rows + row0 + i);
    for (int i = tid; i < nchunks; i += BT) cp_async8(schunks + i, A.chunks + chunk0 + i);
    cp_async_commit();
    for (int i = tid; i < 18 * nq; i += BT) sval[i] = __ldg(I.val_ref + i);
    for (int i = tid; i < (nnz + 1) / 2; i += BT)  // 16-byte stores; an odd tail's pair ends in the pad
        reinterpret_cast<double2 *>(slot)[i] = make_double2(0.0, 0.0);
    __syncthreads();
    // K pass; the barrier after its last colour also tells every thread whether any element
    // of the block conducts
    int conducting = 0;
    int c0 = 0;
    bool any_m = false;
    for (int c = 0; c < ncolors; c++) {
        const int c1 = Bp->col_end[c];
        for (int i = c0 + tid; i < c1; i += BT) {
            const int64_t r = (int64_t)rec0 + i;
            if (c == 0) tile_element<true, Q4, kStiffness, true>(A, r, slot, incv, nnz, ninc);
            else tile_element<true, Q4, kStiffness>(A, r, slot, incv, nnz, ninc);
            if (!conducting) {
                const double sg = I.sigma ? __ldg(I.sigma + __ldg(A.recs + 2 * A.nrec + r).z) : 1.0;
                conducting = fabs(sg) > 1e-12;
            }
        }
        c0 = c1;
        if (c + 1 == ncolors) {
            cp_async_wait_all();
            any_m = __syncthreads_or(conducting) != 0;
        } else {
            __syncthreads();
        }
    }
    if (ncolors == 0) {
        cp_async_wait_all();
        __syncthreads();
    }
    tile_rows_diag<BT, true>(srows, nrows, incv, ninc, slot, nnz, A.err);
    __syncthreads();
    // real parts; a block without a conductor stores (K, omega * 0) pairs in this one pass
    const int warp = tid >> 5, lane = tid & 31;
    double2 *cv2 = reinterpret_cast<double2 *>(I.cvals);
    for (int c = warp; c < nchunks; c += BT / 32) {
        const uint2 ch = schunks[c];
        const int sb0 = (int)(ch.x & 0xFFFFu), len = (int)(ch.x >> 16);
        const int64_t g = (int64_t)ch.y;
        if (sb0 + len > nnz || g + len > A.nnz_total) {
            if (lane == 0) flag(A.err);
            continue;
        }
        if (any_m)  // (+ 0.0: -0 -> +0, the first colour stores its entries)
            for (int i = lane; i < len; i += 32) I.cvals[2 * (g + i)] = slot[sb0 + i] + 0.0;
        else
            for (int i = lane; i < len; i += 32) cv2[g + i] = make_double2(slot[sb0 + i] + 0.0, I.omega * 0.0);
    }
    if (!any_m) return;
    // M pass over the same slots
    __syncthreads();  // the real parts are read out of the slots
    for (int i = tid; i < (nnz + 1) / 2; i += BT)  // 16-byte stores; an odd tail's pair ends in the pad
        reinterpret_cast<double2 *>(slot)[i] = make_double2(0.0, 0.0);
    __syncthreads();
    c0 = 0;
    for (int c = 0; c < ncolors; c++) {
        const int c1 = Bp->col_end[c];
        for (int i = c0 + tid; i < c1; i += BT) tile_mass_element(I, (int64_t)rec0 + i, slot, incv, nnz, ninc, sval);
        c0 = c1;
        __syncthreads();
    }
    tile_rows_diag<BT, false>(srows, nrows, incv, ninc, slot, nnz, A.err);
    __syncthreads();
    for (int c = warp; c < nchunks; c += BT / 32) {
        const uint2 ch = schunks[c];
        const int sb0 = (int)(ch.x & 0xFFFFu), len = (int)(ch.x >> 16);
        const int64_t g = (int64_t)ch.y;
        if (sb0 + len > nnz || g + len > A.nnz_total) continue;  // flagged in the K pass
        for (int i = lane; i < len; i += 32) I.cvals[2 * (g + i) + 1] = I.omega * slot[sb0 + i];
    }
}

// 320 threads: a colour class of an interior 4x4x4 tile holds about 288 elements, so each
// colour phase runs in one pass (256 threads left a second pass with one warp busy).
constexpr int kTileBT = 320;
constexpr int kTileMinB = 2;

// ---- host plan builder --------------------------------------------------------------

struct HostRec {
    uint32_t w[24];  // the six 16-byte planes of one record, plane-major
};

// Layer index of every node along one axis: sorted coordinates split where
// consecutive values are more than 0.3 h apart or a layer would span more than h.
void axis_layers(const std::vector<double4> &xyz, int axis, double h, std::vector<int32_t> &layer) {
    const int64_t n = (int64_t)xyz.size();
    std::vector<std::pair<double, int32_t>> v((size_t)n);
    for (int64_t i = 0; i < n; i++) {
        const double c = axis == 0 ? xyz[i].x : axis == 1 ? xyz[i].y : xyz[i].z;
        v[i] = {c, (int32_t)i};
    }
    std::sort(v.begin(), v.end());
    layer.assign((size_t)n, 0);
    int32_t L = 0;
    double start = n ? v[0].first : 0.0;
    for (int64_t i = 1; i < n; i++) {
        const double x = v[i].first;
        if (x - v[i - 1].first > 0.3 * h || x - start > h) {
            L++;
            start = x;
        }
        layer[v[i].second] = L;
    }
}

template <typename T>
int download(std::vector<T> &dst, const T *src, int64_t count, cudaStream_t s) {
    dst.resize((size_t)count);
    if (count == 0) return MAG_OK;
    MAG_CUDA_TRY(cudaMemcpyAsync(dst.data(), src, (size_t)count * sizeof(T), cudaMemcpyDeviceToHost, s));
    return MAG_OK;
}

}  // namespace

void free_tile_plan(TilePlan *p) {
    void *q[] = {p->blocks, p->rows, p->chunks, p->recs};
    for (void *x : q)
        if (x) cudaFree(x);
    *p = TilePlan{};
}

bool plan_tiles_host(const TileHostMesh &hm, TileHostPlan *out) {
    *out = TileHostPlan{};
    const std::vector<double4> &xyz = hm.xyz;
    const std::vector<int4> &tet = hm.tet;
    const std::vector<int32_t> &dofs = hm.dofs, &row_ptr = hm.row_ptr, &inc_ptr = hm.inc_ptr;
    const std::vector<uint8_t> &tags = hm.tags, &sbits = hm.sbits;
    const std::vector<uint32_t> &inc_elem = hm.inc_elem, &inc_pos = hm.inc_pos;
    const int64_t ndof = (int64_t)row_ptr.size() - 1, ne = (int64_t)tet.size();
    const int64_t ninc_total = (int64_t)inc_elem.size();
    const bool have_signs = !sbits.empty();
    if (ne <= 0 || ndof <= 0 || hm.nnz >= (int64_t(1) << 32)) return false;

    // an element with a repeated dof would update a diagonal slot or one slot twice
    for (int64_t e = 0; e < ne; e++)
        for (int a = 0; a < 6; a++)
            for (int b = a + 1; b < 6; b++)
                if (dofs[6 * e + a] >= 0 && dofs[6 * e + a] == dofs[6 * e + b]) return false;

    // ---- spatial layers and tiles ----
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (const double4 &p : xyz) {
        const double c[3] = {p.x, p.y, p.z};
        for (int a = 0; a < 3; a++) {
            lo[a] = std::min(lo[a], c[a]);
            hi[a] = std::max(hi[a], c[a]);
        }
    }
    double vol = 1.0, ext_max = 0.0;
    for (int a = 0; a < 3; a++) {
        vol *= hi[a] - lo[a];
        ext_max = std::max(ext_max, hi[a] - lo[a]);
    }
    const double nn = (double)xyz.size();
    double h = vol > 0.0 ? std::cbrt(vol / nn) : ext_max / std::max(1.0, std::cbrt(nn));
    if (!(h > 0.0)) h = 1.0;
    std::vector<int32_t> layer[3];
    for (int a = 0; a < 3; a++) axis_layers(xyz, a, h, layer[a]);
    constexpr int kTileLayers[3] = {4, 4, MAG_TILE_LAYERS_Z};
    int32_t ntile[3] = {1, 1, 1};
    for (int a = 0; a < 3; a++) {
        int32_t m = 0;
        for (int32_t v : layer[a]) m = std::max(m, v);
        ntile[a] = m / kTileLayers[a] + 1;
    }
    const int64_t tiles = (int64_t)ntile[0] * ntile[1] * ntile[2];
    if (tiles >= (int64_t(1) << 31)) return false;
    // tile of every row: that of its edge's lower node; a row without incidences
    // (an unused dof) joins the tile of the row before it
    std::vector<int32_t> row_tile((size_t)ndof, 0);
    {
        int32_t prev = 0;
        for (int64_t r = 0; r < ndof; r++) {
            if (inc_ptr[r + 1] > inc_ptr[r]) {
                const uint32_t ew = inc_elem[inc_ptr[r]];
                const int64_t e = ew & 0x1FFFFFFFu;
                const int l = (int)(ew >> 29);
                const int *t = &tet[e].x;
                const int32_t na = t[edge_a(l)], nb = t[edge_b(l)];
                const int32_t node = na < nb ? na : nb;
                prev = (layer[0][node] / kTileLayers[0]) +
                       ntile[0] * ((layer[1][node] / kTileLayers[1]) + ntile[1] * (layer[2][node] / kTileLayers[2]));
            }
            row_tile[r] = prev;
        }
    }
    // rows grouped by tile (stable: ascending ids within a tile)
    std::vector<int64_t> tstart((size_t)tiles + 1, 0);
    for (int64_t r = 0; r < ndof; r++) tstart[row_tile[r] + 1]++;
    for (int64_t t = 0; t < tiles; t++) tstart[t + 1] += tstart[t];
    std::vector<int32_t> order((size_t)ndof);
    {
        std::vector<int64_t> fill(tstart.begin(), tstart.end() - 1);
        for (int64_t r = 0; r < ndof; r++) order[fill[row_tile[r]]++] = (int32_t)r;
    }
    // blocks: each tile's rows, cut where a block would exceed its capacity
    std::vector<int64_t> bstart;  // index into order
    for (int64_t t = 0; t < tiles; t++) {
        int64_t k = tstart[t];
        const int64_t k1 = tstart[t + 1];
        while (k < k1) {
            bstart.push_back(k);
            int64_t bn = 0, bi = 0;
            while (k < k1) {
                const int32_t r = order[k];
                const int64_t rn = row_ptr[r + 1] - row_ptr[r], ri = inc_ptr[r + 1] - inc_ptr[r];
                if (rn > kCompactMaxRow || ri > kCompactMaxRow) return false;
                if (bn + rn > kTileMaxNnz || bi + ri > kTileMaxInc) break;
                bn += rn;
                bi += ri;
                k++;
            }
        }
    }
    bstart.push_back(ndof);
    const int64_t nb = (int64_t)bstart.size() - 1;
    if (nb >= (int64_t(1) << 31)) return false;

    std::vector<TileBlock> blocks((size_t)nb);
    std::vector<uint2> rows((size_t)ndof);
    std::vector<std::vector<HostRec>> brec((size_t)nb);
    std::vector<std::vector<uint2>> bchunk((size_t)nb);
    std::atomic<int> fail{0};

#pragma omp parallel
    {
        struct Inc {
            int64_t e;
            int l;
            int lr;     // block-local row
            int32_t k;  // incidence index
        };
        std::vector<Inc> incs;
        std::vector<int32_t> own_a, own_b, color, adj_ptr, adj, queue;
        std::vector<uint8_t> cnt;
#pragma omp for schedule(dynamic, 16)
        for (int64_t b = 0; b < nb; b++) {
            if (fail) continue;
            const int64_t k0 = bstart[b], k1 = bstart[b + 1];
            TileBlock &B = blocks[b];
            std::memset(&B, 0, sizeof B);
            B.row0 = (int32_t)k0;
            B.nrows = (int32_t)(k1 - k0);
            // row table and incidences
            int32_t bn = 0, bi = 0;
            incs.clear();
            for (int64_t k = k0; k < k1; k++) {
                const int32_t r = order[k];
                const int32_t rn = row_ptr[r + 1] - row_ptr[r];
                const int32_t i0 = inc_ptr[r], i1 = inc_ptr[r + 1];
                uint32_t diag = 0;
                for (int32_t t = i0; t < i1; t++) {
                    const uint32_t ew = inc_elem[t];
                    const int l = (int)(ew >> 29);
                    if (t == i0) diag = (inc_pos[t] >> (5 * l)) & 31u;
                    incs.push_back(Inc{(int64_t)(ew & 0x1FFFFFFFu), l, (int)(k - k0), t});
                }
                rows[k] = make_uint2((uint32_t)r, (uint32_t)bn | ((uint32_t)bi << 13) | (diag << 25));
                bn += rn;
                bi += i1 - i0;
            }
            B.nnz = bn;
            B.ninc = bi;
            // store chunks: runs of consecutive rows, cut at kTileChunk nonzeros
            std::vector<uint2> &ch = bchunk[b];
            ch.clear();
            {
                int32_t off = 0;
                int64_t k = k0;
                while (k < k1) {
                    int64_t k2 = k + 1;
                    while (k2 < k1 && order[k2] == order[k2 - 1] + 1) k2++;
                    const int64_t g0 = row_ptr[order[k]], g1 = row_ptr[order[k2 - 1] + 1];
                    for (int64_t g = g0; g < g1; g += kTileChunk) {
                        const int32_t len = (int32_t)std::min<int64_t>(kTileChunk, g1 - g);
                        ch.push_back(make_uint2((uint32_t)(off + (g - g0)) | ((uint32_t)len << 16), (uint32_t)g));
                    }
                    off += (int32_t)(g1 - g0);
                    k = k2;
                }
            }
            B.nchunks = (int32_t)ch.size();
            // distinct elements (ascending) and their records
            std::sort(incs.begin(), incs.end(), [](const Inc &x, const Inc &y) {
                return x.e != y.e ? x.e < y.e : x.l < y.l;
            });
            std::vector<HostRec> &rec = brec[b];
            rec.clear();
            for (size_t q = 0; q < incs.size(); q++) {
                const Inc &c = incs[q];
                if (q == 0 || incs[q - 1].e != c.e) {
                    HostRec h;
                    const int64_t e = c.e;
                    const int4 tt = tet[e];
                    h.w[0] = (uint32_t)tt.x;
                    h.w[1] = (uint32_t)tt.y;
                    h.w[2] = (uint32_t)tt.z;
                    h.w[3] = (uint32_t)tt.w;
                    for (int j = 0; j < 4; j++) h.w[4 + j] = (uint32_t)dofs[6 * e + j];
                    h.w[8] = (uint32_t)dofs[6 * e + 4];
                    h.w[9] = (uint32_t)dofs[6 * e + 5];
                    h.w[10] = (uint32_t)e;
                    unsigned sb = 0;
                    if (have_signs) {
                        sb = sbits[e];
                    } else {
                        const int n4[4] = {tt.x, tt.y, tt.z, tt.w};
                        for (int j = 0; j < 6; j++) sb |= (n4[edge_a(j)] < n4[edge_b(j)] ? 0u : 1u) << j;
                    }
                    h.w[11] = (uint32_t)tags[e] | (sb << 8);
                    for (int j = 12; j < 18; j++) h.w[j] = 0;
                    for (int j = 18; j < 24; j++) h.w[j] = kTileAbsent;
                    rec.push_back(h);
                } else if (incs[q - 1].l == c.l) {
                    fail = 1;  // one element twice in a row's incidences at the same local row
                }
                HostRec &h = rec.back();
                const uint2 rw = rows[k0 + c.lr];
                const int32_t r = order[k0 + c.lr];
                const uint32_t nzb = rw.y & 0x1FFFu, incb = (rw.y >> 13) & 0xFFFu;
                h.w[12 + c.l] = inc_pos[c.k];
                h.w[18 + c.l] = nzb | ((incb + (uint32_t)(c.k - inc_ptr[r])) << 16);
            }
            const int32_t nr = (int32_t)rec.size();
            // colour classes: conflict = two elements updating the same off-diagonal slot
            own_a.assign((size_t)bn, -1);
            own_b.assign((size_t)bn, -1);
            cnt.assign((size_t)bn, 0);
            for (int32_t i = 0; i < nr && !fail; i++) {
                const HostRec &h = rec[i];
                for (int l = 0; l < 6; l++) {
                    if (h.w[18 + l] == kTileAbsent) continue;
                    const uint32_t nzb = h.w[18 + l] & 0xFFFFu;
                    for (int j = 0; j < 6; j++) {
                        if (j == l) continue;
                        const uint32_t p = (h.w[12 + l] >> (5 * j)) & 31u;
                        if (p == (uint32_t)kCompactMaxRow) continue;
                        const uint32_t sl = nzb + p;
                        if (sl >= (uint32_t)bn || cnt[sl] >= 2) {
                            fail = 1;
                            break;
                        }
                        if (cnt[sl] == 0) own_a[sl] = i;
                        else own_b[sl] = i;
                        cnt[sl]++;
                    }
                }
            }
            if (fail) continue;
            // An absent column (a dof of -1) of a row points at the row's own diagonal
            // nonzero: the kernels add its discarded value there without a test, and the row
            // phase overwrites that slot with the diagonal's element-ordered sum afterwards.
            for (int32_t i = 0; i < nr; i++) {
                HostRec &h = rec[i];
                for (int l = 0; l < 6; l++) {
                    if (h.w[18 + l] == kTileAbsent) continue;
                    const uint32_t diagp = (h.w[12 + l] >> (5 * l)) & 31u;
                    for (int j = 0; j < 6; j++)
                        if (((h.w[12 + l] >> (5 * j)) & 31u) == (uint32_t)kCompactMaxRow)
                            h.w[12 + l] = (h.w[12 + l] & ~(31u << (5 * j))) | (diagp << (5 * j));
                }
            }
            // adjacency (CSR over records)
            adj_ptr.assign((size_t)nr + 1, 0);
            for (int32_t sl = 0; sl < bn; sl++)
                if (cnt[sl] == 2) {
                    adj_ptr[own_a[sl] + 1]++;
                    adj_ptr[own_b[sl] + 1]++;
                }
            for (int32_t i = 0; i < nr; i++) adj_ptr[i + 1] += adj_ptr[i];
            adj.assign((size_t)adj_ptr[nr], 0);
            {
                std::vector<int32_t> f(adj_ptr.begin(), adj_ptr.end() - 1);
                for (int32_t sl = 0; sl < bn; sl++)
                    if (cnt[sl] == 2) {
                        adj[f[own_a[sl]]++] = own_b[sl];
                        adj[f[own_b[sl]]++] = own_a[sl];
                    }
            }
            // two colours by breadth-first search where the graph is bipartite (components
            // flipped to balance the classes), else greedy in element order
            color.assign((size_t)nr, -1);
            bool two = true;
            int64_t size0 = 0, size1 = 0;
            for (int32_t s0 = 0; s0 < nr && two; s0++) {
                if (color[s0] >= 0) continue;
                queue.clear();
                queue.push_back(s0);
                color[s0] = 0;
                int64_t c0 = 1, c1 = 0;
                for (size_t qh = 0; qh < queue.size() && two; qh++) {
                    const int32_t u = queue[qh];
                    for (int32_t t = adj_ptr[u]; t < adj_ptr[u + 1]; t++) {
                        const int32_t w = adj[t];
                        if (color[w] < 0) {
                            color[w] = 1 - color[u];
                            (color[w] ? c1 : c0)++;
                            queue.push_back(w);
                        } else if (color[w] == color[u]) {
                            two = false;
                            break;
                        }
                    }
                }
                if (two && std::llabs((size0 + c1) - (size1 + c0)) < std::llabs((size0 + c0) - (size1 + c1))) {
                    for (int32_t u : queue) color[u] = 1 - color[u];
                    std::swap(c0, c1);
                }
                size0 += c0;
                size1 += c1;
            }
            int ncol = 2;
            if (!two) {
                color.assign((size_t)nr, -1);
                ncol = 0;
                for (int32_t u = 0; u < nr; u++) {
                    unsigned used = 0;
                    for (int32_t t = adj_ptr[u]; t < adj_ptr[u + 1]; t++)
                        if (color[adj[t]] >= 0) used |= 1u << color[adj[t]];
                    int c = 0;
                    while (c < 32 && (used >> c) & 1u) c++;
                    color[u] = c;
                    ncol = std::max(ncol, c + 1);
                }
                if (ncol > kTileMaxColors) {
                    fail = 1;
                    continue;
                }
            }
            // records by colour; within a colour in ascending element order, or (build option)
            // by the set of the element's rows in the block, most rows first, so that the
            // threads of a warp run the same rows
            std::vector<int32_t> idx((size_t)nr);
            std::vector<uint32_t> rkey((size_t)nr, 0u);
            for (int32_t i = 0; i < nr; i++) {
                idx[i] = i;
                if (MAG_TILE_SORT_ROWS) {
                    uint32_t m = 0;
                    for (int l = 0; l < 6; l++) m |= (rec[i].w[18 + l] != kTileAbsent ? 1u : 0u) << l;
                    rkey[i] = ((6u - (uint32_t)__builtin_popcount(m)) << 6) | m;
                }
            }
            std::stable_sort(idx.begin(), idx.end(), [&](int32_t x, int32_t y) {
                return color[x] != color[y] ? color[x] < color[y] : rkey[x] < rkey[y];
            });
            std::vector<HostRec> sorted((size_t)nr);
            for (int32_t i = 0; i < nr; i++) sorted[i] = rec[idx[i]];
            rec.swap(sorted);
            B.nrec = nr;
            B.ncolors = ncol;
            for (int c = 0; c < kTileMaxColors; c++) B.col_end[c] = 0;
            for (int32_t i = 0; i < nr; i++) B.col_end[color[idx[i]]] = i + 1;
            for (int c = 1; c < ncol; c++) B.col_end[c] = std::max(B.col_end[c], B.col_end[c - 1]);
        }
    }
    if (fail) return false;

    // concatenate: record and chunk offsets, planes
    int64_t nrec = 0, nch = 0;
    int32_t max_nnz = 0, max_inc = 0, max_col = 0, max_rows = 0, max_ch = 0;
    for (int64_t b = 0; b < nb; b++) {
        blocks[b].rec0 = (int32_t)nrec;
        blocks[b].chunk0 = (int32_t)nch;
        nrec += blocks[b].nrec;
        nch += blocks[b].nchunks;
        max_nnz = std::max(max_nnz, blocks[b].nnz);
        max_inc = std::max(max_inc, blocks[b].ninc);
        max_col = std::max(max_col, blocks[b].ncolors);
        max_rows = std::max(max_rows, blocks[b].nrows);
        max_ch = std::max(max_ch, blocks[b].nchunks);
        if (nrec >= (int64_t(1) << 31) || nch >= (int64_t(1) << 31)) return false;
    }
    std::vector<uint4> planes((size_t)(6 * nrec));
    std::vector<uint2> chunks((size_t)nch);
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t b = 0; b < nb; b++) {
        const std::vector<HostRec> &rec = brec[b];
        const int64_t o = blocks[b].rec0;
        for (size_t i = 0; i < rec.size(); i++)
            for (int k = 0; k < 6; k++) {
                const uint32_t *w = rec[i].w + 4 * k;
                planes[(size_t)k * nrec + o + i] = make_uint4(w[0], w[1], w[2], w[3]);
            }
        std::copy(bchunk[b].begin(), bchunk[b].end(), chunks.begin() + blocks[b].chunk0);
    }
    // coverage check: every incidence is one record slot
    {
        int64_t present = 0;
        for (int64_t i = 0; i < nrec; i++) {
            const uint4 a = planes[4 * nrec + i], c = planes[5 * nrec + i];
            const uint32_t sl[6] = {a.z, a.w, c.x, c.y, c.z, c.w};
            for (int l = 0; l < 6; l++) present += sl[l] != kTileAbsent;
        }
        if (present != ninc_total) return false;
    }
    out->blocks.swap(blocks);
    out->rows.swap(rows);
    out->chunks.swap(chunks);
    out->planes.swap(planes);
    out->nrec = nrec;
    out->max_nnz = max_nnz;
    out->max_inc = max_inc;
    out->max_colors = max_col;
    out->max_rows = max_rows;
    out->max_chunks = max_ch;
    return true;
}

int build_tile_plan(const TilePlanInput &in, TilePlan *plan, cudaStream_t s) {
    *plan = TilePlan{};
    if (in.wide || in.ne <= 0 || in.ndof <= 0 || in.nnz >= (int64_t(1) << 32)) return MAG_OK;
    const auto t_start = std::chrono::steady_clock::now();
    TileHostMesh hm;
    MAG_TRY(download(hm.xyz, in.xyz, in.nn, s));
    MAG_TRY(download(hm.tet, in.tet, in.ne, s));
    MAG_TRY(download(hm.dofs, in.dofs, 6 * in.ne, s));
    MAG_TRY(download(hm.tags, in.tags, in.ne, s));
    if (in.signbits) MAG_TRY(download(hm.sbits, in.signbits, in.ne, s));
    MAG_TRY(download(hm.row_ptr, in.row_ptr, in.ndof + 1, s));
    MAG_TRY(download(hm.inc_ptr, in.inc_ptr, in.ndof + 1, s));
    MAG_TRY(download(hm.inc_elem, in.inc_elem, in.ninc, s));
    MAG_TRY(download(hm.inc_pos, in.inc_pos, in.ninc, s));
    MAG_CUDA_TRY(cudaStreamSynchronize(s));
    hm.nnz = in.nnz;
    TileHostPlan hp;
    if (!plan_tiles_host(hm, &hp)) return MAG_OK;
    TilePlan p;
    const int64_t nb = (int64_t)hp.blocks.size(), nch = (int64_t)hp.chunks.size(), nrec = hp.nrec;
    p.nblocks = (int32_t)nb;
    p.nrows = in.ndof;
    p.nchunks = nch;
    p.nrec = nrec;
    p.nnz = in.nnz;
    p.max_nnz = hp.max_nnz;
    p.max_inc = hp.max_inc;
    p.max_colors = hp.max_colors;
    p.max_rows = hp.max_rows;
    p.max_chunks = hp.max_chunks;
    p.evals_per_elem = (double)nrec / (double)in.ne;
    // rows and chunks padded by 16 bytes: the kernel's L2 prefetches round to 16 bytes
    const size_t b_blk = (size_t)nb * sizeof(TileBlock), b_rows = hp.rows.size() * sizeof(uint2) + 16,
                 b_ch = (size_t)std::max<int64_t>(nch, 1) * sizeof(uint2) + 16,
                 b_rec = (size_t)std::max<int64_t>(6 * nrec, 1) * sizeof(uint4);
    if (cudaMalloc(&p.blocks, b_blk) != cudaSuccess || cudaMalloc(&p.rows, b_rows) != cudaSuccess ||
        cudaMalloc(&p.chunks, b_ch) != cudaSuccess || cudaMalloc(&p.recs, b_rec) != cudaSuccess) {
        free_tile_plan(&p);
        cudaGetLastError();
        return MAG_OK;  // no room: the other schedules remain
    }
    MAG_CUDA_TRY(cudaMemcpyAsync(p.blocks, hp.blocks.data(), b_blk, cudaMemcpyHostToDevice, s));
    MAG_CUDA_TRY(cudaMemcpyAsync(p.rows, hp.rows.data(), hp.rows.size() * sizeof(uint2), cudaMemcpyHostToDevice, s));
    if (nch) MAG_CUDA_TRY(cudaMemcpyAsync(p.chunks, hp.chunks.data(), nch * sizeof(uint2), cudaMemcpyHostToDevice, s));
    if (nrec)
        MAG_CUDA_TRY(cudaMemcpyAsync(p.recs, hp.planes.data(), 6 * nrec * sizeof(uint4), cudaMemcpyHostToDevice, s));
    MAG_CUDA_TRY(cudaStreamSynchronize(s));
    p.bytes = (int64_t)(b_blk + b_rows + b_ch + b_rec);
    p.build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
    p.ok = 1;
    *plan = p;
    return MAG_OK;
}

namespace {

// Shared memory of one CTA: the block's values (an even count of doubles), the incidence
// slots (double2), then the block's row table and store chunks (uint2 each).
size_t tile_smem_bytes(const TilePlan &tp, TileArgs *a) {
    a->smem_nnz = ((tp.max_nnz + 1) & ~1) + kTileSlotPad;
    a->smem_inc = tp.max_inc;
    a->smem_rows = tp.max_rows;
    a->smem_chunks = tp.max_chunks;
    return (size_t)a->smem_nnz * sizeof(double) + (size_t)a->smem_inc * sizeof(double2) +
           (size_t)(a->smem_rows + a->smem_chunks) * sizeof(uint2);
}

template <bool CALCJ, bool Q4, int MODE, int BT = kTileBT, int MINB = kTileMinB>
int launch(const TileArgs &a, const TilePlan &tp, size_t smem, cudaStream_t s) {
    auto kern = k_tile<BT, MINB, CALCJ, Q4, MODE>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return MAG_E_CUDA;
    // CTAs resident at once: how far ahead a CTA prefetches
    int dev = 0, nsm = 0, per = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, BT, smem) != cudaSuccess || per < 1)
        return MAG_E_CUDA;
    // (ahead >= nblocks: no CTA prefetches)
    const int ahead = tp.prefetch_waves > 0 ? per * nsm * tp.prefetch_waves : tp.nblocks;
    kern<<<tp.nblocks, BT, smem, s>>>(a, tp.nblocks, ahead);
    return cudaPeekAtLastError() == cudaSuccess ? MAG_OK : MAG_E_CUDA;
}

TileArgs make_args(const TilePlan &tp, const ElemData &m, const QuadParams &qp, int *err) {
    TileArgs a{};
    a.blocks = tp.blocks;
    a.rows = tp.rows;
    a.chunks = tp.chunks;
    a.recs = tp.recs;
    a.nrec = tp.nrec;
    a.xyz = m.xyz;
    a.qp = qp;
    a.err = err;
    a.ndof = tp.nrows;
    return a;
}

}  // namespace

int launch_tile_jacobian(const TilePlan &tp, const ElemData &m, const double *sol, const QuadParams &qp,
                         const MaterialParams &mp, int calc_j, double *vals, double *res, int *err,
                         cudaStream_t s) {
    if (!tp.ok || !qp.standard_curl) return MAG_E_UNSUPPORTED;
    TileArgs a = make_args(tp, m, qp, err);
    a.sol = sol;
    a.mp = mp;
    a.vals = vals;
    a.res = res;
    a.nnz_total = tp.nnz;
    size_t smem = tile_smem_bytes(tp, &a);
    const bool q4 = qp.nq == 4 && qp.uniform_w;
    if (calc_j && q4) {  // the launch shape of the Newton Jacobian (threads per CTA x CTAs per SM)
        switch (tp.variant) {
            case 1: return launch<true, true, kJacobian, 288, 2>(a, tp, smem, s);
            case 2: return launch<true, true, kJacobian, 256, 2>(a, tp, smem, s);
            case 3: return launch<true, true, kJacobian, 512, 1>(a, tp, smem, s);
            default: return launch<true, true, kJacobian>(a, tp, smem, s);
        }
    }
    if (calc_j) return launch<true, false, kJacobian>(a, tp, smem, s);
    return q4 ? launch<false, true, kJacobian>(a, tp, smem, s) : launch<false, false, kJacobian>(a, tp, smem, s);
}

const char *tile_variant_name(int v) {
    static const char *names[kTileVariants] = {"320 threads x 2 CTAs/SM", "288 threads x 2 CTAs/SM",
                                               "256 threads x 2 CTAs/SM", "512 threads x 1 CTA/SM"};
    return v >= 0 && v < kTileVariants ? names[v] : "";
}

int launch_tile_stiffness(const TilePlan &tp, const ElemData &m, const double *nu, const QuadParams &qp,
                          double *vals, int *err, cudaStream_t s) {
    if (!tp.ok || !qp.standard_curl) return MAG_E_UNSUPPORTED;
    TileArgs a = make_args(tp, m, qp, err);
    a.nu_e = nu;
    a.vals = vals;
    a.nnz_total = tp.nnz;
    size_t smem = tile_smem_bytes(tp, &a);
    const bool q4 = qp.nq == 4 && qp.uniform_w;
    return q4 ? launch<true, true, kStiffness>(a, tp, smem, s) : launch<true, false, kStiffness>(a, tp, smem, s);
}

int launch_tile_seeded(const TilePlan &tp, const ElemData &m, const double *sol, const double *bscale,
                       const QuadParams &qp, const MaterialParams &mp, double *vals, double *res, int *err,
                       cudaStream_t s) {
    if (!tp.ok || !qp.standard_curl) return MAG_E_UNSUPPORTED;
    TileArgs a = make_args(tp, m, qp, err);
    a.sol = sol;
    a.bscale = bscale;
    a.mp = mp;
    a.vals = vals;
    a.res = res;
    a.nnz_total = tp.nnz;
    size_t smem = tile_smem_bytes(tp, &a);
    const bool q4 = qp.nq == 4 && qp.uniform_w;
    return q4 ? launch<true, true, kSeeded>(a, tp, smem, s) : launch<true, false, kSeeded>(a, tp, smem, s);
}

namespace {

using ComplexKernel = void (*)(const TileComplexInstance *, const int2 *, int, int, int, int, int, int);

ComplexKernel complex_kernel(int variant, bool q4) {
    if (q4) return variant == 1 ? k_tile_complex<288, 2, true> : k_tile_complex<320, 2, true>;
    return variant == 1 ? k_tile_complex<288, 2, false> : k_tile_complex<320, 2, false>;
}
constexpr int kComplexThreads[kTileComplexVariants] = {320, 288};

}  // namespace

int build_tile_complex(const std::vector<TileComplexInput> &in, TileComplexBatch *b, cudaStream_t s) {
    *b = TileComplexBatch{};
    if (in.empty()) return MAG_OK;
    std::vector<TileComplexInstance> hi(in.size());
    int q4 = 1;
    for (size_t i = 0; i < in.size(); i++) {
        const TilePlan &tp = *in[i].tp;
        if (!tp.ok || !in[i].qp.standard_curl || in[i].qp.nq > kMaxQuad) return MAG_OK;
        TileComplexInstance &t = hi[i];
        t = TileComplexInstance{};
        t.a = make_args(tp, in[i].m, in[i].qp, in[i].err);
        t.a.nu_e = in[i].nu;
        t.a.nnz_total = tp.nnz;
        t.sigma = in[i].sigma;
        t.val_ref = in[i].qp.val_ref;
        t.omega = in[i].omega;
        t.cvals = in[i].vals;
        b->smem_nnz = std::max(b->smem_nnz, ((tp.max_nnz + 1) & ~1) + kTileSlotPad);
        b->smem_inc = std::max(b->smem_inc, tp.max_inc);
        b->smem_rows = std::max(b->smem_rows, tp.max_rows);
        b->smem_chunks = std::max(b->smem_chunks, tp.max_chunks);
        q4 &= (in[i].qp.nq == 4 && in[i].qp.uniform_w) ? 1 : 0;
    }
    // items: larger meshes first (a short tail), each mesh's blocks in plan order
    std::vector<int> order(in.size());
    for (size_t i = 0; i < in.size(); i++) order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return in[x].tp->nrec > in[y].tp->nrec; });
    std::vector<int2> items;
    for (int i : order)
        for (int k = 0; k < in[i].tp->nblocks; k++) items.push_back(make_int2(i, k));
    if (items.empty() || items.size() >= (size_t)INT32_MAX) return MAG_OK;
    b->q4 = q4;
    b->smem = (size_t)b->smem_nnz * sizeof(double) + (size_t)b->smem_inc * sizeof(double2) +
              (size_t)(b->smem_rows + b->smem_chunks) * sizeof(uint2) + (size_t)18 * kMaxQuad * sizeof(double);
    int dev = 0, nsm = 0;
    MAG_CUDA_TRY(cudaGetDevice(&dev));
    MAG_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    for (int v = 0; v < kTileComplexVariants; v++) {
        const ComplexKernel kern = complex_kernel(v, q4 != 0);
        int per = 0;
        if (cudaFuncSetAttribute((const void *)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->smem) !=
                cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void *)kern, kComplexThreads[v], b->smem) !=
                cudaSuccess || per < 1) {
            cudaGetLastError();
            *b = TileComplexBatch{};
            return MAG_OK;  // the blocks do not fit: the other batch variants remain
        }
        b->ahead[v] = per * nsm;
    }
    if (cudaMalloc(&b->inst, hi.size() * sizeof(TileComplexInstance)) != cudaSuccess ||
        cudaMalloc(&b->items, items.size() * sizeof(int2)) != cudaSuccess) {
        cudaGetLastError();
        free_tile_complex(b);
        return MAG_OK;
    }
    MAG_CUDA_TRY(cudaMemcpyAsync(b->inst, hi.data(), hi.size() * sizeof(TileComplexInstance), cudaMemcpyHostToDevice, s));
    MAG_CUDA_TRY(cudaMemcpyAsync(b->items, items.data(), items.size() * sizeof(int2), cudaMemcpyHostToDevice, s));
    MAG_CUDA_TRY(cudaStreamSynchronize(s));
    b->nitems = (int)items.size();
    b->ok = 1;
    return MAG_OK;
}

int launch_tile_complex(const TileComplexBatch &b, int variant, cudaStream_t s) {
    if (!b.ok || variant < 0 || variant >= kTileComplexVariants) return MAG_E_UNSUPPORTED;
    const ComplexKernel kern = complex_kernel(variant, b.q4 != 0);
    kern<<<b.nitems, kComplexThreads[variant], b.smem, s>>>(static_cast<const TileComplexInstance *>(b.inst), b.items,
                                                           b.nitems, b.ahead[variant], b.smem_nnz, b.smem_inc,
                                                           b.smem_rows, b.smem_chunks);
    return cudaPeekAtLastError() == cudaSuccess ? MAG_OK : MAG_E_CUDA;
}

const char *tile_complex_variant_name(int v) {
    static const char *names[kTileComplexVariants] = {"tile blocks, 320 threads x 2 CTAs/SM",
                                                      "tile blocks, 288 threads x 2 CTAs/SM"};
    return v >= 0 && v < kTileComplexVariants ? names[v] : "";
}

void free_tile_complex(TileComplexBatch *b) {
    if (b->inst) cudaFree(b->inst);
    if (b->items) cudaFree(b->items);
    *b = TileComplexBatch{};
}

}  // namespace mag
