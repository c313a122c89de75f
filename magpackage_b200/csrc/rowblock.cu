// Row-block Newton-Jacobian assembly (FP64, sm_100a): one launch, no scratch,
// no inter-CTA synchronisation.
//
// The CSR rows are cut into blocks of whole rows holding at most kBlockInc
// (row, incident element) pairs. A CTA takes one block:
//   phase A -- one thread per incidence (row a, element e, local edge loc):
//              gathers e's vertices, edge values and material, computes the
//              element's geometry, curls, B and nu(|B|^2) (the reference's
//              arithmetic, bit for bit) and from them the row loc of the 6x6
//              tangent and the residual entry loc; the 7 values go to shared
//              memory. Each element is evaluated once per row it touches.
//   phase B -- one thread per row adds its incidences' values, in ascending
//              element order, into the row's slots of a shared-memory
//              accumulator (the in-row positions come from the plan) and sums
//              the residual; the block's contiguous slice of CSR values is then
//              stored coalesced.
// HBM traffic is the algorithmic I/O plus the incidence plan; the price is the
// repeated element-level arithmetic.
//
// Variants further down: k_rowblock_shared evaluates each distinct element of a block
// once into a shared-memory record; k_rowblock_nz (the default) in addition places
// every off-diagonal entry straight into its nonzero's slot (an off-diagonal entry has
// at most two contributions, whose sum does not depend on order) and keeps the per-row
// element-ordered sum for diagonals and residuals only.
#include <vector>

#include "common.cuh"
#include "element.cuh"
#include "rowblock.cuh"

namespace mag {

namespace {

using namespace elem;

// Sum over quadrature points of v * (qw_q * |det J|), in point order from zero.
// Q4 = the standard rule: 4 equal weights, so the 4 products are one value u
// and the sum is ((u + u) + u) + u.
template <bool Q4>
__device__ __forceinline__ double qsum_w(double v, const QuadParams &qp, double w0, double adet) {
    double u = v * w0;
    if (Q4) return ((u + u) + u) + u;
    double acc = u;
    if (qp.uniform_w) {
        for (int q = 1; q < qp.nq; q++) acc = acc + u;
    } else {
        for (int q = 1; q < qp.nq; q++) acc = acc + v * (qp.qw[q] * adet);
    }
    return acc;
}

__device__ __forceinline__ void pick(const double C[6][3], int k, double out[3]) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
        double v = C[0][c];
        v = k == 1 ? C[1][c] : v;
        v = k == 2 ? C[2][c] : v;
        v = k == 3 ? C[3][c] : v;
        v = k == 4 ? C[4][c] : v;
        v = k == 5 ? C[5][c] : v;
        out[c] = v;
    }
}

struct RBArgs {
    ElemData m;
    RowPlan rp;
    const double *sol;
    QuadParams qp;
    MaterialParams mp;
    const int32_t *block_row;  // [nblocks+1] first row of each block
    double *vals;
    double *res;
    const double *nu_e;        // [Ne] per-element reluctivity (stiffness mode of k_rowblock_nz)
};

constexpr int kSv = 9;  // shared-memory stride (doubles) of one incidence's values

// Row loc of element e's signed tangent (row[0..5]) and residual entry (row[6]).
template <bool CALCJ, bool STDCURL, bool Q4>
__device__ __forceinline__ void element_row(const RBArgs &A, int64_t e, int loc, double *out) {
    int4 tt = A.m.tet[e];
    int d[6];
    load_dofs(A.m.dofs, e, d);
    unsigned sb = A.m.signbits ? A.m.signbits[e] : derived_signs(tt);
    int tag = A.m.tags[e];
    Geo g;
    geometry(A.m.xyz, tt, g);
    double a[6];
#pragma unroll
    for (int i = 0; i < 6; i++) a[i] = d[i] >= 0 ? flip(__ldg(A.sol + d[i]), (sb >> i) & 1) : 0.0;
    unsigned si = (sb >> loc) & 1;
    const double w0 = A.qp.qw[0] * g.adet;
    if (STDCURL) {
        double C[6][3];
        curls_standard(g, C);
        double B[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            double s = a[0] * C[0][c];
#pragma unroll
            for (int i = 1; i < 6; i++) s = s + a[i] * C[i][c];
            B[c] = s;
        }
        double nu, dnu;
        material_eval(A.mp, tag, dot3(B, B), nu, dnu);
        double Cl[3];
        pick(C, loc, Cl);
        double bl = dot3(B, Cl);
        out[6] = flip(qsum_w<Q4>(nu * bl, A.qp, w0, g.adet), si);
        if (CALCJ) {
            if (dnu == 0.0) {
#pragma unroll
                for (int j = 0; j < 6; j++)
                    out[j] = flip(qsum_w<Q4>(nu * dot3(Cl, C[j]), A.qp, w0, g.adet), si ^ ((sb >> j) & 1));
            } else {
                double gl = (2.0 * dnu) * bl;
#pragma unroll
                for (int j = 0; j < 6; j++)
                    out[j] = flip(qsum_w<Q4>(nu * dot3(Cl, C[j]) + gl * dot3(B, C[j]), A.qp, w0, g.adet),
                                  si ^ ((sb >> j) & 1));
            }
        }
    } else {
        double res[6], K[6][6];
        jacobian_block<CALCJ, false>(g, a, tag, A.qp, A.mp, res, K);
        double r = res[0];
#pragma unroll
        for (int i = 1; i < 6; i++) r = loc == i ? res[i] : r;
        out[6] = flip(r, si);
        if (CALCJ) {
#pragma unroll
            for (int j = 0; j < 6; j++) {
                double v = K[0][j];
#pragma unroll
                for (int i = 1; i < 6; i++) v = loc == i ? K[i][j] : v;
                out[j] = flip(v, si ^ ((sb >> j) & 1));
            }
        }
    }
}

template <bool CALCJ, bool STDCURL, bool Q4, bool WIDE>
__global__ void __launch_bounds__(kBlockInc, 4) k_rowblock(RBArgs A) {
    __shared__ double sv[kBlockInc * kSv];
    __shared__ double sacc[kBlockInc * 6];  // a block's nonzeros <= 6 per incidence
    __shared__ int s_rp[kBlockInc + 1], s_ip[kBlockInc + 1];
    const int tid = threadIdx.x;
    const int a0 = A.block_row[blockIdx.x], a1 = A.block_row[blockIdx.x + 1];
    const int nrows = a1 - a0;
    for (int r = tid; r <= nrows; r += kBlockInc) {
        s_rp[r] = A.rp.row_ptr[a0 + r];
        s_ip[r] = A.rp.inc_ptr[a0 + r];
    }
    __syncthreads();
    const int k0 = s_ip[0], ninc = s_ip[nrows] - k0;
    const int base = s_rp[0], span = s_rp[nrows] - base;
    // phase A: one incidence per thread
    if (tid < ninc) {
        uint32_t ew = __ldg(A.rp.inc_elem + k0 + tid);
        element_row<CALCJ, STDCURL, Q4>(A, (int64_t)(ew & 0x1FFFFFFFu), (int)(ew >> 29), sv + tid * kSv);
    }
    if (CALCJ)
        for (int i = tid; i < span; i += kBlockInc) sacc[i] = 0.0;
    __syncthreads();
    // phase B: one thread per row adds its incidences in ascending element order
    for (int r = tid; r < nrows; r += kBlockInc) {
        const int off = s_rp[r] - base;
        double racc = 0.0;
        for (int k = s_ip[r]; k < s_ip[r + 1]; k++) {
            const double *v = sv + (k - k0) * kSv;
            if (CALCJ) {
                if (!WIDE) {
                    uint32_t pw = __ldg(A.rp.inc_pos + k);
#pragma unroll
                    for (int j = 0; j < 6; j++) {
                        uint32_t p = (pw >> (5 * j)) & 31u;
                        if (p != (uint32_t)kCompactMaxRow) sacc[off + p] = sacc[off + p] + v[j];
                    }
                } else {
                    uint32_t w0 = __ldg(A.rp.inc_pos + 2 * (int64_t)k), w1 = __ldg(A.rp.inc_pos + 2 * (int64_t)k + 1);
#pragma unroll
                    for (int j = 0; j < 6; j++) {
                        uint32_t p = (j < 4 ? (w0 >> (8 * j)) : (w1 >> (8 * (j - 4)))) & 255u;
                        if (p != (uint32_t)kWideMaxRow) sacc[off + p] = sacc[off + p] + v[j];
                    }
                }
            }
            racc = racc + v[6];
        }
        A.res[a0 + r] = racc;
    }
    if (CALCJ) {
        __syncthreads();
        for (int i = tid; i < span; i += kBlockInc) A.vals[base + i] = sacc[i];
    }
}

// ---- shared-element variant --------------------------------------------------------

// In-row positions of incidence k's six columns (kCompactMaxRow / kWideMaxRow = no dof).
template <bool WIDE>
__device__ __forceinline__ void inc_positions(const RowPlan &rp, int64_t k, unsigned p[6]) {
    if (!WIDE) {
        const uint32_t pw = rp.inc_pos[k];
#pragma unroll
        for (int j = 0; j < 6; j++) p[j] = (pw >> (5 * j)) & 31u;
    } else {
        const uint32_t w0 = rp.inc_pos[2 * k], w1 = rp.inc_pos[2 * k + 1];
#pragma unroll
        for (int j = 0; j < 6; j++) p[j] = (j < 4 ? (w0 >> (8 * j)) : (w1 >> (8 * (j - 4)))) & 255u;
    }
}

// Per incidence (row order) bit j: an earlier incidence of the same row (a lower
// element) also adds to column j's position, so this one is the second of that
// off-diagonal entry's contributions. Sets *bad when an off-diagonal position of a row
// has more than two contributions or a column other than the element's own edge lands
// on the diagonal (a repeated dof), which the nonzero-pass kernel cannot place.
template <bool WIDE>
__global__ void __launch_bounds__(256) k_second_masks(RowPlan rp, uint8_t *__restrict__ second, int *__restrict__ bad) {
    const int64_t a = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (a >= rp.ndof) return;
    const unsigned none = WIDE ? (unsigned)kWideMaxRow : (unsigned)kCompactMaxRow;
    const int k0 = rp.inc_ptr[a], k1 = rp.inc_ptr[a + 1];
    for (int k = k0; k < k1; k++) {
        unsigned p[6];
        inc_positions<WIDE>(rp, k, p);
        const unsigned loc = rp.inc_elem[k] >> 29;
        unsigned pd = p[0];
#pragma unroll
        for (int j = 1; j < 6; j++) pd = loc == (unsigned)j ? p[j] : pd;
        unsigned mask = 0;
        for (int j = 0; j < 6; j++) {
            if ((unsigned)j == loc || p[j] == none) continue;
            if (p[j] == pd) atomicExch(bad, 1);
            int before = 0;
            for (int q = k0; q < k; q++) {
                unsigned pq[6];
                inc_positions<WIDE>(rp, q, pq);
                const unsigned lq = rp.inc_elem[q] >> 29;
#pragma unroll
                for (int i = 0; i < 6; i++) before += ((unsigned)i != lq && pq[i] == p[j]) ? 1 : 0;
            }
            if (before == 1) mask |= 1u << j;
            if (before > 1) atomicExch(bad, 1);
        }
        second[k] = (uint8_t)mask;
    }
}


// Per block: sort its (element, incidence) pairs, number the distinct elements in
// ascending order, and record each incidence's slot. Counts above MAXE set *overflow.
template <int BI, int MAXE>
__global__ void __launch_bounds__(BI) k_block_elems(RowPlan rp, const int32_t *__restrict__ block_row,
                                                           int32_t *__restrict__ blk_nelem,
                                                           int32_t *__restrict__ blk_k0,
                                                           int32_t *__restrict__ blk_elem,
                                                           uint16_t *__restrict__ inc_slot,
                                                           uint32_t *__restrict__ inc_sorted,
                                                           const uint8_t *__restrict__ second, int *overflow) {
    __shared__ unsigned long long key[BI];
    __shared__ int scan[BI];
    const int t = threadIdx.x;
    const int a0 = block_row[blockIdx.x], a1 = block_row[blockIdx.x + 1];
    const int k0 = rp.inc_ptr[a0], ninc = rp.inc_ptr[a1] - k0;
    uint32_t ew = t < ninc ? rp.inc_elem[k0 + t] : 0xFFFFFFFFu;
    key[t] = t < ninc ? ((unsigned long long)(ew & 0x1FFFFFFFu) << 8) | (unsigned)t : ~0ull;
    __syncthreads();
    // bitonic sort of BI keys
    for (int k = 2; k <= BI; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            const int p = t ^ j;
            if (p > t) {
                unsigned long long x = key[t], y = key[p];
                const bool up = (t & k) == 0;
                if ((x > y) == up) {
                    key[t] = y;
                    key[p] = x;
                }
            }
            __syncthreads();
        }
    }
    const unsigned long long me = key[t];
    const bool valid = me != ~0ull;
    const bool first = valid && (t == 0 || (key[t - 1] >> 8) != (me >> 8));
    scan[t] = first ? 1 : 0;
    __syncthreads();
    for (int off = 1; off < BI; off <<= 1) {  // inclusive scan
        int v = t >= off ? scan[t - off] : 0;
        __syncthreads();
        scan[t] += v;
        __syncthreads();
    }
    const int slot = scan[t] - 1;
    if (valid) {
        const int orig = (int)(me & 0xFF);
        const uint32_t loc = rp.inc_elem[k0 + orig] >> 29;
        inc_slot[k0 + orig] = (uint16_t)(slot | (loc << 8));
        if (inc_sorted)
            inc_sorted[k0 + t] = (uint32_t)slot | loc << 8 | (uint32_t)orig << 16 |
                                 (second ? (uint32_t)second[k0 + orig] << 24 : 0u);
        if (first) blk_elem[k0 + slot] = (int32_t)(me >> 8);
    }
    if (t == 0) {
        blk_k0[blockIdx.x] = k0;
        if (blockIdx.x == gridDim.x - 1) blk_k0[gridDim.x] = k0 + ninc;
    }
    if (t == BI - 1) {
        blk_nelem[blockIdx.x] = scan[t];
        if (overflow && scan[t] > MAXE) atomicExch(overflow, 1);
    }
}

constexpr int kSv2 = 7;  // shared-memory stride (doubles) of one incidence's values

// One distinct element of a block, evaluated once: what every row of the element needs.
struct ElemRec {
    double J[9];   // Jacobian columns (the standard curls are recomputed from these)
    double r2;     // 2 / det
    double b[6];   // B . C_j (unsigned curls)
    double nu, g2; // nu(|B|^2), 2 d nu / d|B|^2
    double adet;
};

// Shared-memory carve-up of one block of BI incidences with at most MAXE distinct elements.
template <int BI, int MAXE>
struct SharedLayout {
    static constexpr int rec = (int)sizeof(ElemRec) * MAXE;  // phase B reuses it as the row accumulator
    static constexpr int sv = 8 * BI * kSv2;
    static constexpr int rsb = 4 * MAXE;
    static constexpr int pos = 8 * BI;  // in-row positions (2 words per incidence when wide)
    static constexpr int bytes = rec + sv + rsb + pos + 8 * (BI + 1);
    static_assert(rec >= 8 * (BI * 6 + BI * 6 / 16 + 1), "the skewed row accumulator reuses the records");
    static_assert(rec % 16 == 0 && sv % 16 == 0, "alignment of the shared-memory carve-up");
};

// Shared-element row blocks. Phase A1: one thread per distinct element of the block
// gathers and evaluates it once (geometry, curls, B, nu(|B|^2)) into a shared record;
// A2: one thread per incidence forms its element row from the record; B: one thread per
// CSR row adds its incidences in ascending element order, as k_rowblock does, so the
// bits are the same.
// Row-accumulator address of the block's i-th nonzero: one pad word per 16, so row
// threads (rows ~16 nonzeros apart) adding at the same in-row position hit different banks.
__device__ __forceinline__ int skew(int i) { return i + (i >> 4); }

template <int BI, int MAXE, int MINB, bool CALCJ, bool Q4, bool WIDE>
__global__ void __launch_bounds__(BI, MINB) k_rowblock_shared(RBArgs A, const int32_t *__restrict__ blk_nelem,
                                                              const int32_t *__restrict__ blk_k0,
                                                              const int32_t *__restrict__ blk_elem,
                                                              const uint32_t *__restrict__ inc_sorted) {
    using L = SharedLayout<BI, MAXE>;
    extern __shared__ __align__(16) unsigned char rs_smem[];
    ElemRec *rec = reinterpret_cast<ElemRec *>(rs_smem);
    double *sv = reinterpret_cast<double *>(rs_smem + L::rec);
    unsigned *rsb = reinterpret_cast<unsigned *>(rs_smem + L::rec + L::sv);
    uint32_t *spos = reinterpret_cast<uint32_t *>(rs_smem + L::rec + L::sv + L::rsb);
    int *s_rp = reinterpret_cast<int *>(rs_smem + L::rec + L::sv + L::rsb + L::pos);
    int *s_ip = s_rp + (BI + 1);
    double *sacc = reinterpret_cast<double *>(rec);
    const int tid = threadIdx.x;
    // every prologue load depends only on the block index, so they all issue together
    const int a0 = A.block_row[blockIdx.x], a1 = A.block_row[blockIdx.x + 1];
    const int k0 = blk_k0[blockIdx.x], ninc = blk_k0[blockIdx.x + 1] - k0;
    const int nel = blk_nelem[blockIdx.x];
    const int nrows = a1 - a0;
    // phase A2 walks the incidences in element order (consecutive threads read the same or
    // neighbouring records); each writes its values at its row-order position
    const unsigned my_inc = tid < ninc ? __ldg(inc_sorted + k0 + tid) : 0u;
    if (CALCJ && tid < ninc) {
        if (WIDE) {
            spos[2 * tid] = __ldg(A.rp.inc_pos + 2 * (int64_t)(k0 + tid));
            spos[2 * tid + 1] = __ldg(A.rp.inc_pos + 2 * (int64_t)(k0 + tid) + 1);
        } else {
            spos[tid] = __ldg(A.rp.inc_pos + k0 + tid);
        }
    }
    for (int r = tid; r <= nrows; r += BI) {
        s_rp[r] = A.rp.row_ptr[a0 + r];
        s_ip[r] = A.rp.inc_ptr[a0 + r];
    }
    // phase A1: one thread per distinct element (the plan keeps nel <= MAXE)
    if (tid < nel && tid < MAXE) {
        unsigned sb;
        int tag;
        Geo g;
        double a[6];
        {
            const int64_t e = blk_elem[k0 + tid];
            int4 tt = A.m.tet[e];
            int d[6];
            load_dofs(A.m.dofs, e, d);
            sb = A.m.signbits ? A.m.signbits[e] : derived_signs(tt);
            tag = A.m.tags[e];
            geometry(A.m.xyz, tt, g);
#pragma unroll
            for (int i = 0; i < 6; i++) a[i] = d[i] >= 0 ? flip(__ldg(A.sol + d[i]), (sb >> i) & 1) : 0.0;
        }
        double C[6][3];
        curls_standard(g, C);
        double B[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            double v = a[0] * C[0][c];
#pragma unroll
            for (int i = 1; i < 6; i++) v = v + a[i] * C[i][c];
            B[c] = v;
        }
        double nu, dnu;
        material_eval(A.mp, tag, dot3(B, B), nu, dnu);
        ElemRec &R = rec[tid];
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) R.J[3 * r + c] = g.J[r][c];
        R.r2 = 2.0 * g.rdet;
#pragma unroll
        for (int j = 0; j < 6; j++) R.b[j] = dot3(B, C[j]);
        R.nu = nu;
        R.g2 = 2.0 * dnu;
        R.adet = g.adet;
        rsb[tid] = sb;
    }
    __syncthreads();
    const int base = s_rp[0], span = s_rp[nrows] - base;
    // phase A2: one thread per incidence, the element's row from its record
    if (tid < ninc) {
        const ElemRec &R = rec[my_inc & 0xFF];
        const int loc = (int)((my_inc >> 8) & 0xFF);
        const unsigned sb = rsb[my_inc & 0xFF];
        Geo g;
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) g.J[r][c] = R.J[3 * r + c];
        g.rdet = 0.5 * R.r2;  // exact: curls_standard forms 2 * rdet again
        g.adet = R.adet;
        double C[6][3];
        curls_standard(g, C);
        const unsigned si = (sb >> loc) & 1;
        const double w0 = A.qp.qw[0] * R.adet, nu = R.nu;
        double Cl[3];
        pick(C, loc, Cl);
        double bl = R.b[0];
#pragma unroll
        for (int j = 1; j < 6; j++) bl = loc == j ? R.b[j] : bl;
        double *out = sv + ((my_inc >> 16) & 0xFF) * kSv2;
        out[6] = flip(qsum_w<Q4>(nu * bl, A.qp, w0, R.adet), si);
        if (CALCJ) {
            if (R.g2 == 0.0) {
#pragma unroll
                for (int j = 0; j < 6; j++)
                    out[j] = flip(qsum_w<Q4>(nu * dot3(Cl, C[j]), A.qp, w0, R.adet), si ^ ((sb >> j) & 1));
            } else {
                const double gl = R.g2 * bl;
#pragma unroll
                for (int j = 0; j < 6; j++)
                    out[j] = flip(qsum_w<Q4>(nu * dot3(Cl, C[j]) + gl * R.b[j], A.qp, w0, R.adet),
                                  si ^ ((sb >> j) & 1));
            }
        }
    }
    __syncthreads();  // the records are dead from here on; sacc reuses their memory
    if (CALCJ) {
        for (int i = tid; i < span; i += BI) sacc[skew(i)] = 0.0;
        __syncthreads();
    }
    // phase B: one thread per row adds its incidences in ascending element order
    for (int r = tid; r < nrows; r += BI) {
        const int off = s_rp[r] - base;
        double racc = 0.0;
        for (int k = s_ip[r]; k < s_ip[r + 1]; k++) {
            const double *v = sv + (k - k0) * kSv2;
            if (CALCJ) {
                if (!WIDE) {
                    uint32_t pw = spos[k - k0];
#pragma unroll
                    for (int j = 0; j < 6; j++) {
                        uint32_t p = (pw >> (5 * j)) & 31u;
                        if (p != (uint32_t)kCompactMaxRow) sacc[skew(off + p)] = sacc[skew(off + p)] + v[j];
                    }
                } else {
                    uint32_t w0 = spos[2 * (k - k0)], w1 = spos[2 * (k - k0) + 1];
#pragma unroll
                    for (int j = 0; j < 6; j++) {
                        uint32_t p = (j < 4 ? (w0 >> (8 * j)) : (w1 >> (8 * (j - 4)))) & 255u;
                        if (p != (uint32_t)kWideMaxRow) sacc[skew(off + p)] = sacc[skew(off + p)] + v[j];
                    }
                }
            }
            racc = racc + v[6];
        }
        A.res[a0 + r] = racc;
    }
    if (CALCJ) {
        __syncthreads();
        for (int i = tid; i < span; i += BI) A.vals[base + i] = sacc[skew(i)];
    }
}

// ---- nonzero-pass variant ----------------------------------------------------------

// Shared-memory carve-up of one block of the nonzero-pass kernel.
template <int BI, int MAXE>
struct NzLayout {
    static constexpr int rec = (int)sizeof(ElemRec) * MAXE;
    static constexpr int nzv = 16 * kNzMaxSpan;  // two slots per CSR nonzero of the block
    static constexpr int sv = 16 * BI;           // per incidence (row order): residual, diagonal entry
    static constexpr int rsb = 4 * MAXE;
    static constexpr int pos = 8 * BI;           // in-row positions (2 words per incidence when wide)
    static constexpr int roff = 2 * BI;          // per incidence: its row's first nonzero in the block
    static constexpr int loc = BI;               // per incidence: the local edge of its row
    static constexpr int bytes = rec + nzv + sv + rsb + pos + roff + loc + 8 * (BI + 1);
    static_assert(rec % 16 == 0 && nzv % 16 == 0 && sv % 16 == 0, "alignment of the shared-memory carve-up");
};

// Shared-element row blocks with a nonzero pass. A1 as k_rowblock_shared. A2: one thread
// per incidence forms its element row and writes each off-diagonal entry straight into
// its CSR nonzero's slot (0 for the lower element, 1 for the higher: an off-diagonal
// entry has at most two contributions, whose sum does not depend on their order), and
// its diagonal entry and residual into per-incidence slots. B1: one thread per row sums
// the diagonal and the residual over its incidences in ascending element order. B2: one
// thread per nonzero stores (0 + slot 0) + slot 1, coalesced. Same bits as k_rowblock.
//
// STIFF: the curl-curl matrix K(nu) with the per-element reluctivity A.nu_e instead
// (assemble_curl_curl_kernel_mex.cpp:94-101: (C_i . C_j) nu w summed over the points, the
// Jacobian's entry with d nu = 0, same operation order); no solution, no residual.
template <int BI, int MAXE, int MINB, bool CALCJ, bool Q4, bool WIDE, bool STIFF = false>
__global__ void __launch_bounds__(BI, MINB) k_rowblock_nz(RBArgs A, const int32_t *__restrict__ blk_nelem,
                                                          const int32_t *__restrict__ blk_k0,
                                                          const int32_t *__restrict__ blk_elem,
                                                          const uint32_t *__restrict__ inc_sorted) {
    using L = NzLayout<BI, MAXE>;
    extern __shared__ __align__(16) unsigned char nz_smem[];
    ElemRec *rec = reinterpret_cast<ElemRec *>(nz_smem);
    double2 *nzv = reinterpret_cast<double2 *>(nz_smem + L::rec);
    double2 *sv = reinterpret_cast<double2 *>(nz_smem + L::rec + L::nzv);
    unsigned *rsb = reinterpret_cast<unsigned *>(nz_smem + L::rec + L::nzv + L::sv);
    uint32_t *spos = reinterpret_cast<uint32_t *>(nz_smem + L::rec + L::nzv + L::sv + L::rsb);
    uint16_t *sroff = reinterpret_cast<uint16_t *>(nz_smem + L::rec + L::nzv + L::sv + L::rsb + L::pos);
    uint8_t *sloc = nz_smem + L::rec + L::nzv + L::sv + L::rsb + L::pos + L::roff;
    int *s_ip = reinterpret_cast<int *>(nz_smem + L::rec + L::nzv + L::sv + L::rsb + L::pos + L::roff + L::loc);
    int *s_off = s_ip + (BI + 1);
    constexpr unsigned kNone = WIDE ? (unsigned)kWideMaxRow : (unsigned)kCompactMaxRow;
    const int tid = threadIdx.x;
    const int a0 = A.block_row[blockIdx.x], a1 = A.block_row[blockIdx.x + 1];
    const int k0 = blk_k0[blockIdx.x], ninc = blk_k0[blockIdx.x + 1] - k0;
    const int nel = blk_nelem[blockIdx.x];
    const int nrows = a1 - a0;
    const int base = A.rp.row_ptr[a0], span = A.rp.row_ptr[a1] - base;
    const unsigned my_inc = tid < ninc ? __ldg(inc_sorted + k0 + tid) : 0u;
    if (CALCJ && tid < ninc) {
        if (WIDE) {
            spos[2 * tid] = __ldg(A.rp.inc_pos + 2 * (int64_t)(k0 + tid));
            spos[2 * tid + 1] = __ldg(A.rp.inc_pos + 2 * (int64_t)(k0 + tid) + 1);
        } else {
            spos[tid] = __ldg(A.rp.inc_pos + k0 + tid);
        }
    }
    // per row: first incidence and first nonzero (block-relative); per incidence: its row's
    // first nonzero
    for (int r = tid; r <= nrows; r += BI) {
        const int ip = A.rp.inc_ptr[a0 + r] - k0, off = A.rp.row_ptr[a0 + r] - base;
        s_ip[r] = ip;
        s_off[r] = off;
        if (CALCJ && r < nrows) {
            const int ipn = A.rp.inc_ptr[a0 + r + 1] - k0;
            for (int k = ip; k < ipn; k++) sroff[k] = (uint16_t)off;
        }
    }
    if (CALCJ)
        for (int i = tid; i < span; i += BI) nzv[i] = make_double2(0.0, 0.0);
    // phase A1: one thread per distinct element (the plan keeps nel <= MAXE)
    if (tid < nel && tid < MAXE) {
        if (STIFF) {
            const int64_t e = blk_elem[k0 + tid];
            const int4 tt = A.m.tet[e];
            const unsigned sb = A.m.signbits ? A.m.signbits[e] : derived_signs(tt);
            Geo g;
            geometry(A.m.xyz, tt, g);
            ElemRec &R = rec[tid];
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
                for (int c = 0; c < 3; c++) R.J[3 * r + c] = g.J[r][c];
            R.r2 = 2.0 * g.rdet;
#pragma unroll
            for (int j = 0; j < 6; j++) R.b[j] = 0.0;
            R.nu = __ldg(A.nu_e + e);
            R.g2 = 0.0;
            R.adet = g.adet;
            rsb[tid] = sb;
        } else {
            const int64_t e = blk_elem[k0 + tid];
            const int4 tt = A.m.tet[e];
            int d[6];
            load_dofs(A.m.dofs, e, d);
            const unsigned sb = A.m.signbits ? A.m.signbits[e] : derived_signs(tt);
            const int tag = A.m.tags[e];
            Geo g;
            geometry(A.m.xyz, tt, g);
            double a[6];
#pragma unroll
            for (int i = 0; i < 6; i++) a[i] = d[i] >= 0 ? flip(__ldg(A.sol + d[i]), (sb >> i) & 1) : 0.0;
            double C[6][3];
            curls_standard(g, C);
            double B[3];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                double v = a[0] * C[0][c];
#pragma unroll
                for (int i = 1; i < 6; i++) v = v + a[i] * C[i][c];
                B[c] = v;
            }
            double nu, dnu;
            material_eval(A.mp, tag, dot3(B, B), nu, dnu);
            ElemRec &R = rec[tid];
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
                for (int c = 0; c < 3; c++) R.J[3 * r + c] = g.J[r][c];
            R.r2 = 2.0 * g.rdet;
#pragma unroll
            for (int j = 0; j < 6; j++) R.b[j] = dot3(B, C[j]);
            R.nu = nu;
            R.g2 = 2.0 * dnu;
            R.adet = g.adet;
            rsb[tid] = sb;
        }
    }
    __syncthreads();
    // phase A2: one thread per incidence, walking them in element order
    if (tid < ninc) {
        const ElemRec &R = rec[my_inc & 0xFF];
        const int loc = (int)((my_inc >> 8) & 0xFF);
        const int k = (int)((my_inc >> 16) & 0xFF);
        const unsigned second = my_inc >> 24;
        const unsigned sb = rsb[my_inc & 0xFF];
        Geo g;
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) g.J[r][c] = R.J[3 * r + c];
        g.rdet = 0.5 * R.r2;  // exact: curls_standard forms 2 * rdet again
        g.adet = R.adet;
        double C[6][3];
        curls_standard(g, C);
        const unsigned si = (sb >> loc) & 1;
        const double w0 = A.qp.qw[0] * R.adet, nu = R.nu;
        // the incidence's own curl read from the record by index, in curls_standard's
        // operation order: (J_p - J_m) r2 for edges 0-2, J_x r2 (negated for edge 4) for 3-5
        // (J_x - 0 is J_x exactly)
        const int cp = (0x102 >> (4 * (loc % 3))) & 3, cm = (0x021 >> (4 * (loc % 3))) & 3;
        const double r2 = R.r2;
        double Cl[3];
#pragma unroll
        for (int r = 0; r < 3; r++) {
            const double jm = loc < 3 ? R.J[3 * r + cm] : 0.0;
            const double v = (R.J[3 * r + (loc < 3 ? cp : 5 - loc)] - jm) * r2;
            Cl[r] = loc == 4 ? -v : v;
        }
        const double bl = R.b[loc];
        const double rv = flip(qsum_w<Q4>(nu * bl, A.qp, w0, R.adet), si);
        double dv = 0.0;
        if (CALCJ) {
            double v[6];
            if (R.g2 == 0.0) {
#pragma unroll
                for (int j = 0; j < 6; j++)
                    v[j] = flip(qsum_w<Q4>(nu * dot3(Cl, C[j]), A.qp, w0, R.adet), si ^ ((sb >> j) & 1));
            } else {
                const double gl = R.g2 * bl;
#pragma unroll
                for (int j = 0; j < 6; j++)
                    v[j] = flip(qsum_w<Q4>(nu * dot3(Cl, C[j]) + gl * R.b[j], A.qp, w0, R.adet), si ^ ((sb >> j) & 1));
            }
            unsigned p[6];
            if (!WIDE) {
                const uint32_t pw = spos[k];
#pragma unroll
                for (int j = 0; j < 6; j++) p[j] = (pw >> (5 * j)) & 31u;
            } else {
                const uint32_t w0p = spos[2 * k], w1p = spos[2 * k + 1];
#pragma unroll
                for (int j = 0; j < 6; j++) p[j] = (j < 4 ? (w0p >> (8 * j)) : (w1p >> (8 * (j - 4)))) & 255u;
            }
            double *slots = reinterpret_cast<double *>(nzv) + 2 * (int)sroff[k];
#pragma unroll
            for (int j = 0; j < 6; j++) {
                if (j == loc) dv = v[j];
                else if (p[j] != kNone) slots[2 * p[j] + ((second >> j) & 1)] = v[j];
            }
            sloc[k] = (uint8_t)loc;
        }
        sv[k] = make_double2(rv, dv);
    }
    __syncthreads();
    // phase B1: one thread per row, the diagonal and the residual in ascending element order
    for (int r = tid; r < nrows; r += BI) {
        const int i0 = s_ip[r], i1 = s_ip[r + 1];
        double racc = 0.0, dacc = 0.0;
        for (int k = i0; k < i1; k++) {
            const double2 v = sv[k];
            racc = racc + v.x;
            if (CALCJ) dacc = dacc + v.y;
        }
        if (!STIFF) A.res[a0 + r] = racc;
        if (CALCJ && i1 > i0) {
            const int l = sloc[i0];
            unsigned pd;
            if (!WIDE) {
                pd = (spos[i0] >> (5 * l)) & 31u;
            } else {
                pd = (l < 4 ? (spos[2 * i0] >> (8 * l)) : (spos[2 * i0 + 1] >> (8 * (l - 4)))) & 255u;
            }
            reinterpret_cast<double *>(nzv)[2 * (s_off[r] + (int)pd)] = dacc;
        }
    }
    if (CALCJ) {
        __syncthreads();
        // phase B2: one thread per nonzero
        for (int i = tid; i < span; i += BI) {
            const double2 v = nzv[i];
            A.vals[base + i] = (0.0 + v.x) + v.y;
        }
    }
}

}  // namespace

int build_second_masks(const RowPlan &rp, int64_t ninc, uint8_t **out, cudaStream_t s) {
    *out = nullptr;
    uint8_t *second = nullptr;
    int *d_bad = nullptr;
    int bad = 1;
    if (cudaMalloc(&second, (size_t)(ninc > 0 ? ninc : 1)) == cudaSuccess && cudaMalloc(&d_bad, 4) == cudaSuccess &&
        cudaMemsetAsync(d_bad, 0, 4, s) == cudaSuccess) {
        const unsigned g = (unsigned)((rp.ndof + 255) / 256);
        if (rp.wide) k_second_masks<true><<<g, 256, 0, s>>>(rp, second, d_bad);
        else k_second_masks<false><<<g, 256, 0, s>>>(rp, second, d_bad);
        if (cudaMemcpyAsync(&bad, d_bad, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            bad = 1;
    }
    if (d_bad) cudaFree(d_bad);
    cudaGetLastError();
    if (bad) {
        if (second) cudaFree(second);
        return MAG_OK;  // no masks: the nonzero-pass kernels are not available for this mesh
    }
    *out = second;
    return MAG_OK;
}

int build_rowblock_plan(const RowPlan &rp, RowBlockPlan *out, cudaStream_t s, int block_inc, bool with_shared,
                        const uint8_t *second) {
    *out = RowBlockPlan{};
    std::vector<int32_t> ip((size_t)rp.ndof + 1), rpp((size_t)rp.ndof + 1);
    MAG_CUDA_TRY(cudaMemcpyAsync(ip.data(), rp.inc_ptr, ip.size() * 4, cudaMemcpyDeviceToHost, s));
    MAG_CUDA_TRY(cudaMemcpyAsync(rpp.data(), rp.row_ptr, rpp.size() * 4, cudaMemcpyDeviceToHost, s));
    MAG_CUDA_TRY(cudaStreamSynchronize(s));
    std::vector<int32_t> starts;
    starts.reserve((size_t)(rp.ndof / 32) + 2);
    int64_t a = 0;
    while (a < rp.ndof) {
        starts.push_back((int32_t)a);
        int64_t b = a + 1;
        if (ip[b] - ip[a] > block_inc) {
            set_error("row-block plan: row %lld has %d incidences (at most %d)", (long long)a,
                      ip[b] - ip[a], block_inc);
            return MAG_E_UNSUPPORTED;
        }
        while (b < rp.ndof && ip[b + 1] - ip[a] <= block_inc && b - a < block_inc) b++;
        a = b;
    }
    starts.push_back((int32_t)rp.ndof);
    out->block_inc = block_inc;
    const int64_t ninc = ip[rp.ndof];
    const int max_elems = block_inc == kSharedBlockInc ? kSharedMaxElems : kMaxBlockElems;
    with_shared = with_shared && (block_inc == kSharedBlockInc || block_inc == kBlockInc);
    if (with_shared) {
        if (cudaMalloc(&out->blk_elem, (size_t)(ninc > 0 ? ninc : 1) * 4) != cudaSuccess ||
            cudaMalloc(&out->inc_slot, (size_t)(ninc > 0 ? ninc : 1) * 2) != cudaSuccess ||
            cudaMalloc(&out->inc_sorted, (size_t)(ninc > 0 ? ninc : 1) * 4) != cudaSuccess)
            with_shared = false;
    }
    // second-contributor bits (mesh-owned, built by build_second_masks) enable the nonzero-pass kernel
    bool nz = with_shared && second != nullptr;
    // Upload the blocks; for the shared-element lists, split any block whose distinct
    // elements exceed the kernel's capacity and rebuild (a few passes at most).
    for (int pass = 0;; pass++) {
        out->nblocks = (int32_t)starts.size() - 1;
        if (out->block_row) cudaFree(out->block_row);
        if (out->blk_nelem) cudaFree(out->blk_nelem);
        if (out->blk_k0) cudaFree(out->blk_k0);
        out->block_row = nullptr;
        out->blk_nelem = nullptr;
        out->blk_k0 = nullptr;
        MAG_CUDA_TRY(cudaMalloc(&out->block_row, starts.size() * 4));
        MAG_CUDA_TRY(cudaMemcpyAsync(out->block_row, starts.data(), starts.size() * 4, cudaMemcpyHostToDevice, s));
        if (!with_shared) break;
        if (cudaMalloc(&out->blk_nelem, (size_t)out->nblocks * 4) != cudaSuccess ||
            cudaMalloc(&out->blk_k0, (size_t)(out->nblocks + 1) * 4) != cudaSuccess) {
            with_shared = false;
            break;
        }
        if (block_inc == kSharedBlockInc)
            k_block_elems<kSharedBlockInc, kSharedMaxElems><<<out->nblocks, kSharedBlockInc, 0, s>>>(
                rp, out->block_row, out->blk_nelem, out->blk_k0, out->blk_elem, out->inc_slot, out->inc_sorted,
                second, nullptr);
        else
            k_block_elems<kBlockInc, kMaxBlockElems><<<out->nblocks, kBlockInc, 0, s>>>(
                rp, out->block_row, out->blk_nelem, out->blk_k0, out->blk_elem, out->inc_slot, out->inc_sorted,
                second, nullptr);
        std::vector<int32_t> nel((size_t)out->nblocks);
        if (cudaMemcpyAsync(nel.data(), out->blk_nelem, nel.size() * 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            with_shared = false;
            break;
        }
        std::vector<int32_t> next;
        next.reserve(starts.size() + 16);
        bool split = false;
        for (int32_t b = 0; b < out->nblocks; b++) {
            next.push_back(starts[b]);
            const bool over = nel[b] > max_elems || (nz && rpp[starts[b + 1]] - rpp[starts[b]] > kNzMaxSpan);
            if (over && starts[b + 1] - starts[b] > 1) {
                next.push_back(starts[b] + (starts[b + 1] - starts[b]) / 2);
                split = true;
            } else if (nel[b] > max_elems) {
                with_shared = false;  // one row alone exceeds the capacity
            } else if (nz && rpp[starts[b + 1]] - rpp[starts[b]] > kNzMaxSpan) {
                nz = false;  // one row alone exceeds the nonzero-pass capacity
            }
        }
        next.push_back(starts.back());
        if (!with_shared) break;
        if (!split) {
            out->shared_ok = 1;
            out->nz_ok = nz ? 1 : 0;
            break;
        }
        if (pass >= 4) {
            with_shared = false;
            break;
        }
        starts.swap(next);
    }
    MAG_CUDA_TRY(cudaStreamSynchronize(s));
    out->ok = 1;
    out->bytes = (int64_t)starts.size() * 4;
    if (out->shared_ok) {
        out->bytes += (int64_t)out->nblocks * 8 + ninc * 10;
    } else {
        cudaGetLastError();
        if (out->blk_nelem) cudaFree(out->blk_nelem);
        if (out->blk_k0) cudaFree(out->blk_k0);
        if (out->blk_elem) cudaFree(out->blk_elem);
        if (out->inc_slot) cudaFree(out->inc_slot);
        if (out->inc_sorted) cudaFree(out->inc_sorted);
        out->inc_sorted = nullptr;
        out->blk_nelem = nullptr;
        out->blk_k0 = nullptr;
        out->blk_elem = nullptr;
        out->inc_slot = nullptr;
    }
    return MAG_OK;
}

void free_rowblock_plan(RowBlockPlan *p) {
    if (p->block_row) cudaFree(p->block_row);
    if (p->blk_nelem) cudaFree(p->blk_nelem);
    if (p->blk_k0) cudaFree(p->blk_k0);
    if (p->blk_elem) cudaFree(p->blk_elem);
    if (p->inc_slot) cudaFree(p->inc_slot);
    if (p->inc_sorted) cudaFree(p->inc_sorted);
    *p = RowBlockPlan{};
}

int launch_rowblock_jacobian(const RowBlockPlan &bp, const ElemData &m, const RowPlan &rp, const double *sol,
                             const QuadParams &qp, const MaterialParams &mp, int calcj, double *vals,
                             double *res, cudaStream_t s) {
    if (!bp.ok) return MAG_E_UNSUPPORTED;
    RBArgs A{m, rp, sol, qp, mp, bp.block_row, vals, res};
    dim3 g(bp.nblocks), b(kBlockInc);
    const bool std_c = qp.standard_curl != 0, wide = rp.wide != 0;
    const bool q4 = qp.nq == 4 && qp.uniform_w;
#define MAG_RB(CJ, SC, Q, W) k_rowblock<CJ, SC, Q, W><<<g, b, 0, s>>>(A)
    if (calcj) {
        if (std_c && q4) {
            if (wide) MAG_RB(true, true, true, true); else MAG_RB(true, true, true, false);
        } else if (std_c) {
            if (wide) MAG_RB(true, true, false, true); else MAG_RB(true, true, false, false);
        } else {
            if (wide) MAG_RB(true, false, false, true); else MAG_RB(true, false, false, false);
        }
    } else {
        if (std_c && q4) MAG_RB(false, true, true, false);
        else if (std_c) MAG_RB(false, true, false, false);
        else MAG_RB(false, false, false, false);
    }
#undef MAG_RB
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) {
        set_error("row-block launch: %s", cudaGetErrorString(e));
        return MAG_E_CUDA;
    }
    return MAG_OK;
}

}  // namespace mag

namespace mag {

int launch_rowblock_shared_jacobian(const RowBlockPlan &bp, const ElemData &m, const RowPlan &rp,
                                    const double *sol, const QuadParams &qp, const MaterialParams &mp, int calcj,
                                    double *vals, double *res, cudaStream_t s) {
    if (!bp.ok || !bp.shared_ok || !qp.standard_curl) return MAG_E_UNSUPPORTED;
    RBArgs A{m, rp, sol, qp, mp, bp.block_row, vals, res};
    const bool wide = rp.wide != 0, q4 = qp.nq == 4 && qp.uniform_w;
#define MAG_RS(BI_, ME_, MB_, CJ, Q, W)                                                                   \
    do {                                                                                                 \
        auto kern = k_rowblock_shared<BI_, ME_, MB_, CJ, Q, W>;                                          \
        const int sm = SharedLayout<BI_, ME_>::bytes;                                                    \
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);                     \
        kern<<<bp.nblocks, BI_, sm, s>>>(A, bp.blk_nelem, bp.blk_k0, bp.blk_elem, bp.inc_sorted);        \
    } while (0)
#define MAG_RS_ALL(BI_, ME_, MB_)                                                                         \
    do {                                                                                                 \
        if (calcj) {                                                                                     \
            if (q4) {                                                                                    \
                if (wide) MAG_RS(BI_, ME_, MB_, true, true, true); else MAG_RS(BI_, ME_, MB_, true, true, false); \
            } else {                                                                                     \
                if (wide) MAG_RS(BI_, ME_, MB_, true, false, true); else MAG_RS(BI_, ME_, MB_, true, false, false); \
            }                                                                                            \
        } else {                                                                                         \
            if (q4) MAG_RS(BI_, ME_, MB_, false, true, false); else MAG_RS(BI_, ME_, MB_, false, false, false); \
        }                                                                                                \
    } while (0)
    static_assert(kSharedBlockInc == kBlockInc, "one block size for the shared-element kernels");
    MAG_RS_ALL(kSharedBlockInc, kSharedMaxElems, 4);
#undef MAG_RS_ALL
#undef MAG_RS
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) {
        set_error("shared row-block launch: %s", cudaGetErrorString(e));
        return MAG_E_CUDA;
    }
    return MAG_OK;
}

}  // namespace mag

namespace mag {

int launch_rowblock_nz_jacobian(const RowBlockPlan &bp, const ElemData &m, const RowPlan &rp, const double *sol,
                                const QuadParams &qp, const MaterialParams &mp, int calcj, double *vals,
                                double *res, cudaStream_t s) {
    if (!bp.ok || !bp.shared_ok || !bp.nz_ok || !qp.standard_curl) return MAG_E_UNSUPPORTED;
    RBArgs A{m, rp, sol, qp, mp, bp.block_row, vals, res};
    const bool wide = rp.wide != 0, q4 = qp.nq == 4 && qp.uniform_w;
    constexpr int BI = kSharedBlockInc, ME = kSharedMaxElems;
    constexpr int sm = NzLayout<BI, ME>::bytes;
#define MAG_NZ(CJ, Q, W)                                                                                 \
    do {                                                                                                 \
        auto kern = k_rowblock_nz<BI, ME, 4, CJ, Q, W>;                                                  \
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);                     \
        kern<<<bp.nblocks, BI, sm, s>>>(A, bp.blk_nelem, bp.blk_k0, bp.blk_elem, bp.inc_sorted);         \
    } while (0)
    if (calcj) {
        if (q4) {
            if (wide) MAG_NZ(true, true, true); else MAG_NZ(true, true, false);
        } else {
            if (wide) MAG_NZ(true, false, true); else MAG_NZ(true, false, false);
        }
    } else {
        if (q4) MAG_NZ(false, true, false); else MAG_NZ(false, false, false);
    }
#undef MAG_NZ
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) {
        set_error("nonzero-pass row-block launch: %s", cudaGetErrorString(e));
        return MAG_E_CUDA;
    }
    return MAG_OK;
}

}  // namespace mag

namespace mag {

int launch_rowblock_nz_stiffness(const RowBlockPlan &bp, const ElemData &m, const RowPlan &rp, const double *nu,
                                 const QuadParams &qp, double *vals, cudaStream_t s) {
    if (!bp.ok || !bp.shared_ok || !bp.nz_ok || !qp.standard_curl || !nu || !vals) return MAG_E_UNSUPPORTED;
    RBArgs A{m, rp, nullptr, qp, MaterialParams{}, bp.block_row, vals, nullptr, nu};
    const bool wide = rp.wide != 0, q4 = qp.nq == 4 && qp.uniform_w;
    constexpr int BI = kSharedBlockInc, ME = kSharedMaxElems;
    constexpr int sm = NzLayout<BI, ME>::bytes;
#define MAG_NZK(Q, W)                                                                                    \
    do {                                                                                                 \
        auto kern = k_rowblock_nz<BI, ME, 4, true, Q, W, true>;                                          \
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);                     \
        kern<<<bp.nblocks, BI, sm, s>>>(A, bp.blk_nelem, bp.blk_k0, bp.blk_elem, bp.inc_sorted);         \
    } while (0)
    if (q4) {
        if (wide) MAG_NZK(true, true); else MAG_NZK(true, false);
    } else {
        if (wide) MAG_NZK(false, true); else MAG_NZK(false, false);
    }
#undef MAG_NZK
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) {
        set_error("nonzero-pass stiffness launch: %s", cudaGetErrorString(e));
        return MAG_E_CUDA;
    }
    return MAG_OK;
}

}  // namespace mag
