// Harmonic-balance (HBFEM) assembly, FP64 (sm_100a).
//
// Element phase (one thread per element) restates assemble_hbfem_kernel_mex.cpp:108-226
// operation for operation: the signed harmonic edge values, per quadrature point the
// physical curls, per time sample t the edge values A(t) = sum_h (Re A_h Re D(t,h) -
// Im A_h Im D(t,h)), B(t), nu(|B(t)|^2) from the B-H table (with the coefficient offsets
// the reference gateway forgets to set), H = nu B, and the harmonic residual
// R_h += w (C_i . H) P(h,t); the Jacobian block is w nu_dc C_r . C_c with nu_dc the
// time average of nu. Per (element, local row) it writes the signed block row into
// the common element scratch (reduced by k_rows_reduce) and its 2K residual entries
// into a second scratch that k_rows_reduce_harm sums per CSR row, in ascending element
// order, as MATLAB's sparse() does with the gateway's triplets.
#include "assemble.cuh"
#include "common.cuh"
#include "element.cuh"
#include "hbfem.cuh"

#include <type_traits>

namespace mag {

namespace {

using namespace elem;

struct HbArgs {
    ElemData m;
    const double *sr, *si;  // [K][ndof] harmonic solution (si may be NULL)
    const double *dr, *di;  // [K][N]: D(t, h) at h * N + t (di may be NULL)
    const double *pr, *pi;  // [N][K]: P(h, t) at t * K + h (pi may be NULL)
    int K, N;
    int64_t ndof;
    QuadParams qp;
    MaterialParams mp;
    double *scratch;  // [Ne][6][kScratchStride] block rows (NULL: residual only)
    double *rscr;     // [Ne][6][2K] residual entries (re | im)
};

// Index of (r, c), r <= c, in the upper triangle of a 6 x 6 block stored row by row.
__host__ __device__ constexpr int kb_at(int r, int c) { return r * 6 - r * (r - 1) / 2 + (c - r); }

// L lanes per element (L a power of two >= K): lane h of an element's group owns
// harmonic h. It keeps that harmonic's six signed edge values and residual accumulators in
// registers; the time-domain edge values A_k(t) = sum_h (Re A_kh Re D(t,h) - Im A_kh Im D(t,h))
// are summed from the lanes' terms, gathered by shuffles, in ascending h: the reference's
// order. B(t), nu, H and the DC block are the same on every lane of the group (same inputs,
// same operations); lane 0 keeps the DC block. No array lives in local memory.
#ifndef MAG_HBFEM_MINB
#define MAG_HBFEM_MINB 3  // resident CTAs per SM the element kernel is compiled for
#endif

template <bool CALCJ, int L>
__global__ void __launch_bounds__(128, MAG_HBFEM_MINB) k_hbfem_elems(HbArgs A) {
    const int lane = threadIdx.x & 31;
    const int sub = lane & (L - 1);
    const int base = lane & ~(L - 1);
    const int64_t e = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / L;
    // every lane stays to the end (the shuffles need the whole warp); an element past the
    // end is computed on element 0's data and not stored
    const bool valid = e < A.m.ne;
    const int64_t ee = valid ? e : 0;
    const int K = A.K, N = A.N;
    const bool own = sub < K;
    const int4 tt = A.m.tet[ee];
    int d[6];
    load_dofs(A.m.dofs, ee, d);
    const unsigned sb = A.m.signbits ? A.m.signbits[ee] : derived_signs(tt);
    const int tag = A.m.tags[ee];
    Geo g;
    geometry(A.m.xyz, tt, g);
    double arh[6], aih[6], rrh[6], rih[6];
#pragma unroll
    for (int k = 0; k < 6; k++) {
        const bool has = own && d[k] >= 0;
        const double xr = has ? __ldg(A.sr + sub * A.ndof + d[k]) : 0.0;
        const double xi = has && A.si ? __ldg(A.si + sub * A.ndof + d[k]) : 0.0;
        arh[k] = flip(xr, (sb >> k) & 1);
        aih[k] = flip(xi, (sb >> k) & 1);
        rrh[k] = 0.0;
        rih[k] = 0.0;
    }
    // The DC block is symmetric bit for bit (C_r . C_c and C_c . C_r are the same products
    // summed in the same order), so only its upper triangle is accumulated: kb[r][c], r <= c,
    // at kb_at(r, c), in shared memory (lane 0 of the group owns its element's 21 entries).
    __shared__ double kbs[128 / L][21];
    double *kb = kbs[threadIdx.x / L];
    if (CALCJ && sub == 0)
        for (int i = 0; i < 21; i++) kb[i] = 0.0;
    const bool imag_a = A.si && A.di;
    for (int q = 0; q < A.qp.nq; q++) {
        const double w = A.qp.qw[q] * g.adet;
        double C[6][3];
        curls_generic(g, A.qp.curl_ref, q, C);
        double sum_nu = 0.0;
        for (int t = 0; t < N; t++) {
            const double drh = own ? __ldg(A.dr + sub * N + t) : 0.0;
            const double dih = own && imag_a ? __ldg(A.di + sub * N + t) : 0.0;
            double at[6];
#pragma unroll
            for (int k = 0; k < 6; k++) {
                double term = arh[k] * drh;
                if (imag_a) term = term - aih[k] * dih;
                double acc = 0.0;
                for (int h = 0; h < K; h++) acc = acc + __shfl_sync(0xFFFFFFFFu, term, base + h);
                at[k] = acc;
            }
            double B[3] = {0.0, 0.0, 0.0};
#pragma unroll
            for (int i = 0; i < 6; i++)
#pragma unroll
                for (int c = 0; c < 3; c++) B[c] = B[c] + C[i][c] * at[i];
            const double bsq = B[0] * B[0] + B[1] * B[1] + B[2] * B[2];
            double nu, dnu;
            material_eval(A.mp, tag, bsq, nu, dnu);
            sum_nu = sum_nu + nu;
            const double H[3] = {nu * B[0], nu * B[1], nu * B[2]};
            if (own) {
                const double p_r = __ldg(A.pr + t * K + sub);
                const double p_i = A.pi ? __ldg(A.pi + t * K + sub) : 0.0;
#pragma unroll
                for (int i = 0; i < 6; i++) {
                    const double dot = C[i][0] * H[0] + C[i][1] * H[1] + C[i][2] * H[2];
                    rrh[i] = rrh[i] + w * dot * p_r;
                    if (A.pi) rih[i] = rih[i] + w * dot * p_i;
                }
            }
        }
        if (CALCJ && sub == 0) {
            const double nu_dc = sum_nu / (double)N;
#pragma unroll 1
            for (int c = 0; c < 6; c++)
#pragma unroll
                for (int r = 0; r <= c; r++) {
                    const double dot = C[r][0] * C[c][0] + C[r][1] * C[c][1] + C[r][2] * C[c][2];
                    kb[kb_at(r, c)] = kb[kb_at(r, c)] + w * nu_dc * dot;
                }
        }
    }
    if (!valid) return;
    double *rdst = A.rscr + e * 6 * 2 * K;
#pragma unroll
    for (int i = 0; i < 6; i++) {
        const unsigned si = (sb >> i) & 1;
        if (own) {
            rdst[i * 2 * K + sub] = flip(rrh[i], si);
            rdst[i * 2 * K + K + sub] = flip(rih[i], si);
        }
        if (CALCJ && sub == 0) {
            double row[6];
#pragma unroll
            for (int j = 0; j < 6; j++) row[j] = flip(kb[i <= j ? kb_at(i, j) : kb_at(j, i)], si ^ ((sb >> j) & 1));
            store_row(A.scratch + e * kScratchPerElem + i * kScratchStride, row, 0.0);
        }
    }
}

// out_re[h][row], out_im[h][row]: per CSR row and residual component, the incidences'
// entries summed from zero in ascending element order.
__global__ void __launch_bounds__(128) k_rows_reduce_harm(RowPlan rp, const double *__restrict__ rscr, int K,
                                                          double *__restrict__ out_re, double *__restrict__ out_im) {
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int W = 2 * K;
    if (idx >= rp.ndof * W) return;
    const int64_t a = idx / W;
    const int c = (int)(idx % W);
    double r = 0.0;
    for (int32_t t = rp.inc_ptr[a]; t < rp.inc_ptr[a + 1]; t++) {
        const uint32_t ew = rp.inc_elem[t];
        r = r + __ldg(rscr + ((int64_t)(ew & 0x1FFFFFFFu) * 6 + (ew >> 29)) * W + c);
    }
    if (c < K) out_re[(int64_t)c * rp.ndof + a] = r;
    else out_im[(int64_t)(c - K) * rp.ndof + a] = r;
}

}  // namespace

int launch_hbfem(const ElemData &m, const RowPlan &rp, int max_row, const double *sr, const double *si, int K,
                 const double *dr, const double *di, const double *pr, const double *pi, int N,
                 const QuadParams &qp, const MaterialParams &mp, double *scratch, double *rscr, double *vals,
                 double *out_re, double *out_im, cudaStream_t s) {
    if (K < 1 || K > kMaxHarm) return MAG_E_ARG;
    HbArgs A{m, sr, si, dr, di, pr, pi, K, N, rp.ndof, qp, mp, vals ? scratch : nullptr, rscr};
    const int L = K == 1 ? 1 : K == 2 ? 2 : K <= 4 ? 4 : K <= 8 ? 8 : 16;  // lanes per element
    const unsigned g = (unsigned)((m.ne * L + 127) / 128);
    auto go = [&](auto calcj, auto lanes) { k_hbfem_elems<decltype(calcj)::value, decltype(lanes)::value><<<g, 128, 0, s>>>(A); };
    using T = std::true_type;
    using F = std::false_type;
    switch (L) {
        case 1: vals ? go(T{}, std::integral_constant<int, 1>{}) : go(F{}, std::integral_constant<int, 1>{}); break;
        case 2: vals ? go(T{}, std::integral_constant<int, 2>{}) : go(F{}, std::integral_constant<int, 2>{}); break;
        case 4: vals ? go(T{}, std::integral_constant<int, 4>{}) : go(F{}, std::integral_constant<int, 4>{}); break;
        case 8: vals ? go(T{}, std::integral_constant<int, 8>{}) : go(F{}, std::integral_constant<int, 8>{}); break;
        default: vals ? go(T{}, std::integral_constant<int, 16>{}) : go(F{}, std::integral_constant<int, 16>{}); break;
    }
    if (cudaPeekAtLastError() != cudaSuccess) return MAG_E_CUDA;
    const int64_t nt = rp.ndof * 2 * K;
    k_rows_reduce_harm<<<(unsigned)((nt + 127) / 128), 128, 0, s>>>(rp, rscr, K, out_re, out_im);
    if (cudaPeekAtLastError() != cudaSuccess) return MAG_E_CUDA;
    if (vals) return launch_rows_reduce(rp, max_row, scratch, vals, nullptr, s);
    return MAG_OK;
}

}  // namespace mag
