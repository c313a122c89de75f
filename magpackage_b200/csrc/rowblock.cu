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
// repeated element-level arithmetic, so the kernel is FP64-bound.
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

}  // namespace

int build_rowblock_plan(const RowPlan &rp, RowBlockPlan *out, cudaStream_t s, int block_inc) {
    *out = RowBlockPlan{};
    std::vector<int32_t> ip((size_t)rp.ndof + 1);
    MAG_CUDA_TRY(cudaMemcpyAsync(ip.data(), rp.inc_ptr, ip.size() * 4, cudaMemcpyDeviceToHost, s));
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
    out->nblocks = (int32_t)starts.size() - 1;
    MAG_CUDA_TRY(cudaMalloc(&out->block_row, starts.size() * 4));
    MAG_CUDA_TRY(cudaMemcpyAsync(out->block_row, starts.data(), starts.size() * 4, cudaMemcpyHostToDevice, s));
    MAG_CUDA_TRY(cudaStreamSynchronize(s));
    out->bytes = (int64_t)starts.size() * 4;
    out->ok = 1;
    return MAG_OK;
}

void free_rowblock_plan(RowBlockPlan *p) {
    if (p->block_row) cudaFree(p->block_row);
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
