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

// Resident CTAs per SM the element kernel is compiled for (registers <= 65536 / (128 x this)):
// with the harmonic count a compile-time constant (MAG_HBFEM_MINB) and at run time
// (MAG_HBFEM_MINB_RT). Measured at 40^3, K = 3, N = 32: run-time count 3.26 ms (3 CTAs/SM);
// constant count 2.24 ms (3 CTAs/SM, 168 registers) and 1.66 ms (2 CTAs/SM, 255 registers).
#ifndef MAG_HBFEM_MINB
#define MAG_HBFEM_MINB 2
#endif
#ifndef MAG_HBFEM_MINB_RT
#define MAG_HBFEM_MINB_RT 3
#endif

// KC: the harmonic count as a compile-time constant (0: A.K at run time, arrays sized for
// kMaxHarm); with a constant count the harmonic loops unroll and the arrays are indexed
// statically.
template <bool CALCJ, int KC>
__global__ void __launch_bounds__(128, KC > 0 ? MAG_HBFEM_MINB : MAG_HBFEM_MINB_RT) k_hbfem_elems(HbArgs A) {
    constexpr int KA = KC > 0 ? KC : kMaxHarm;
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= A.m.ne) return;
    const int K = KC > 0 ? KC : A.K, N = A.N;
    const int4 tt = A.m.tet[e];
    int d[6];
    load_dofs(A.m.dofs, e, d);
    const unsigned sb = A.m.signbits ? A.m.signbits[e] : derived_signs(tt);
    const int tag = A.m.tags[e];
    Geo g;
    geometry(A.m.xyz, tt, g);
    double ar[6][KA], ai[6][KA];
    for (int k = 0; k < 6; k++)
        for (int h = 0; h < K; h++) {
            const bool has = d[k] >= 0;
            const double xr = has ? __ldg(A.sr + h * A.ndof + d[k]) : 0.0;
            const double xi = has && A.si ? __ldg(A.si + h * A.ndof + d[k]) : 0.0;
            ar[k][h] = flip(xr, (sb >> k) & 1);
            ai[k][h] = flip(xi, (sb >> k) & 1);
        }
    double rr[6][KA], ri[6][KA];
    for (int k = 0; k < 6; k++)
        for (int h = 0; h < K; h++) {
            rr[k][h] = 0.0;
            ri[k][h] = 0.0;
        }
    // The DC block is symmetric bit for bit (C_r . C_c and C_c . C_r are the same products
    // summed in the same order), so only its upper triangle is accumulated: kb[r][c], r <= c,
    // at kb_at(r, c).
    double kb[21];
#pragma unroll
    for (int i = 0; i < 21; i++) kb[i] = 0.0;
    const bool imag_a = A.si && A.di;
    for (int q = 0; q < A.qp.nq; q++) {
        const double w = A.qp.qw[q] * g.adet;
        double C[6][3];
        curls_generic(g, A.qp.curl_ref, q, C);
        double sum_nu = 0.0;
        for (int t = 0; t < N; t++) {
            double at[6];
            for (int k = 0; k < 6; k++) {
                double acc = 0.0;
                for (int h = 0; h < K; h++) {
                    double term = ar[k][h] * __ldg(A.dr + h * N + t);
                    if (imag_a) term = term - ai[k][h] * __ldg(A.di + h * N + t);
                    acc = acc + term;
                }
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
            for (int h = 0; h < K; h++) {
                const double p_r = __ldg(A.pr + t * K + h);
                const double p_i = A.pi ? __ldg(A.pi + t * K + h) : 0.0;
#pragma unroll
                for (int i = 0; i < 6; i++) {
                    const double dot = C[i][0] * H[0] + C[i][1] * H[1] + C[i][2] * H[2];
                    rr[i][h] = rr[i][h] + w * dot * p_r;
                    if (A.pi) ri[i][h] = ri[i][h] + w * dot * p_i;
                }
            }
        }
        if (CALCJ) {
            const double nu_dc = sum_nu / (double)N;
#pragma unroll
            for (int c = 0; c < 6; c++)
#pragma unroll
                for (int r = 0; r <= c; r++) {
                    const double dot = C[r][0] * C[c][0] + C[r][1] * C[c][1] + C[r][2] * C[c][2];
                    kb[kb_at(r, c)] = kb[kb_at(r, c)] + w * nu_dc * dot;
                }
        }
    }
    double *rdst = A.rscr + (int64_t)e * 6 * 2 * K;
#pragma unroll
    for (int i = 0; i < 6; i++) {
        const unsigned si = (sb >> i) & 1;
        for (int h = 0; h < K; h++) {
            rdst[i * 2 * K + h] = flip(rr[i][h], si);
            rdst[i * 2 * K + K + h] = flip(ri[i][h], si);
        }
        if (CALCJ) {
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
    HbArgs A{m, sr, si, dr, di, pr, pi, K, N, rp.ndof, qp, mp, vals ? scratch : nullptr, rscr};
    const unsigned g = (unsigned)((m.ne + 127) / 128);
    switch (K) {
        case 1: vals ? k_hbfem_elems<true, 1><<<g, 128, 0, s>>>(A) : k_hbfem_elems<false, 1><<<g, 128, 0, s>>>(A); break;
        case 2: vals ? k_hbfem_elems<true, 2><<<g, 128, 0, s>>>(A) : k_hbfem_elems<false, 2><<<g, 128, 0, s>>>(A); break;
        case 3: vals ? k_hbfem_elems<true, 3><<<g, 128, 0, s>>>(A) : k_hbfem_elems<false, 3><<<g, 128, 0, s>>>(A); break;
        case 4: vals ? k_hbfem_elems<true, 4><<<g, 128, 0, s>>>(A) : k_hbfem_elems<false, 4><<<g, 128, 0, s>>>(A); break;
        default: vals ? k_hbfem_elems<true, 0><<<g, 128, 0, s>>>(A) : k_hbfem_elems<false, 0><<<g, 128, 0, s>>>(A);
    }
    if (cudaPeekAtLastError() != cudaSuccess) return MAG_E_CUDA;
    const int64_t nt = rp.ndof * 2 * K;
    k_rows_reduce_harm<<<(unsigned)((nt + 127) / 128), 128, 0, s>>>(rp, rscr, K, out_re, out_im);
    if (cudaPeekAtLastError() != cudaSuccess) return MAG_E_CUDA;
    if (vals) return launch_rows_reduce(rp, max_row, scratch, vals, nullptr, s);
    return MAG_OK;
}

}  // namespace mag
