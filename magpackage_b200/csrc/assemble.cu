// Element assembly kernels (FP64, sm_100a).
//
// Two phases per assembly:
//   phase 1 (element-parallel): each element's 6x6 block (with edge signs
//     applied) and its 6 residual/RHS entries go to a scratch slab laid out
//     [element][local row][8] = {row values 0..5, vector entry, pad}: one
//     64-byte aligned chunk per (element, local row).
//   phase 2 (row-parallel): every CSR row walks its incidence list, which the
//     pattern builder sorted by ascending element, and adds each incident
//     element's chunk into the row's slots. Every nonzero is therefore summed
//     in one fixed order (element order, the order of appearance that MATLAB's
//     sparse() sees in the MEX triplets), with no floating-point atomics.
//
// Bit-exactness. This translation unit is compiled with -fmad=false and the
// element arithmetic follows the reference's evaluation order
// (src/mex/assemble_jacobian_kernel_mex.cpp:61-152, MexElemUtils.hpp:35-66,
// MexMaterialUtils.hpp:24-87, assemble_curl_curl_kernel_mex.cpp:44-121,
// assemble_mass_kernel_mex.cpp:167-248, assemble_source_kernel_mex.cpp:46-114),
// so each element block equals the reference MEX output bit for bit. Where the
// reference repeats identical work per quadrature point (the Nedelec curl is
// constant), the value is computed once and the per-point products are
// accumulated in the reference's order, which yields the same bits.
#include "assemble.cuh"
#include "common.cuh"
#include "element.cuh"

namespace mag {

namespace {

using namespace elem;

// ---- phase 1: Jacobian + residual -------------------------------------------

template <bool CALCJ, bool STDCURL>
__global__ void __launch_bounds__(128) k_jacobian_elems(ElemData m, const double *__restrict__ sol,
                                                        QuadParams qp, MaterialParams mp,
                                                        double *__restrict__ scratch) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= m.ne) return;
    int4 t = m.tet[e];
    int d[6];
    load_dofs(m.dofs, e, d);
    unsigned sb = m.signbits ? m.signbits[e] : derived_signs(t);
    int tag = m.tags[e];
    Geo g;
    geometry(m.xyz, t, g);
    double a[6];
#pragma unroll
    for (int i = 0; i < 6; i++) a[i] = d[i] >= 0 ? flip(__ldg(sol + d[i]), (sb >> i) & 1) : 0.0;
    double res[6], K[6][6];
    jacobian_block<CALCJ, STDCURL>(g, a, tag, qp, mp, res, K);
    double *dst = scratch + e * kScratchPerElem;
#pragma unroll
    for (int i = 0; i < 6; i++) {
        double row[6];
#pragma unroll
        for (int j = 0; j < 6; j++) row[j] = CALCJ ? flip(K[i][j], ((sb >> i) ^ (sb >> j)) & 1) : 0.0;
        store_row(dst + i * kScratchStride, row, flip(res[i], (sb >> i) & 1));
    }
}

// ---- phase 1: Newton block with a seeded tangent ---------------------------
// Residual at the element's state B (as k_jacobian_elems); tangent evaluated at the
// seeded state beta_e * B: nu(|beta B|^2) Ci.Cj + 2 nu'(|beta B|^2) (beta B.Ci)(beta B.Cj).
// Standard curl table only (constant curls, so one evaluation per element).
__global__ void __launch_bounds__(128) k_jacobian_seeded_elems(ElemData m, const double *__restrict__ sol,
                                                               const double *__restrict__ bscale, QuadParams qp,
                                                               MaterialParams mp, double *__restrict__ scratch) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= m.ne) return;
    int4 t = m.tet[e];
    int d[6];
    load_dofs(m.dofs, e, d);
    unsigned sb = m.signbits ? m.signbits[e] : derived_signs(t);
    int tag = m.tags[e];
    Geo g;
    geometry(m.xyz, t, g);
    double a[6];
#pragma unroll
    for (int i = 0; i < 6; i++) a[i] = d[i] >= 0 ? flip(__ldg(sol + d[i]), (sb >> i) & 1) : 0.0;
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
    double w[kMaxQuad];
    for (int q = 0; q < qp.nq; q++) w[q] = qp.qw[q] * g.adet;
    double nu, dnu, num, dnum;
    material_eval(mp, tag, dot3(B, B), nu, dnu);
    const double be = bscale[e];
    material_eval(mp, tag, (be * be) * dot3(B, B), num, dnum);
    double b[6];
#pragma unroll
    for (int i = 0; i < 6; i++) b[i] = dot3(B, C[i]);
    double *dst = scratch + e * kScratchPerElem;
#pragma unroll
    for (int i = 0; i < 6; i++) {
        double row[6];
        const double gi = 2.0 * dnum * (be * b[i]);
#pragma unroll
        for (int j = 0; j < 6; j++)
            row[j] = flip(qsum(num * dot3(C[i], C[j]) + gi * (be * b[j]), w, qp.nq, qp.uniform_w),
                          ((sb >> i) ^ (sb >> j)) & 1);
        store_row(dst + i * kScratchStride, row, flip(qsum(nu * b[i], w, qp.nq, qp.uniform_w), (sb >> i) & 1));
    }
}

// Midpoint seed of the tangent: beta_e = (|B_e| + |B_hat_e|) / (2 |B_e|), |B_hat_e|^2 the
// point where the element's nonlinear nu(|B|^2) equals the predicted nu_hat_e (bisection;
// nu is nondecreasing in |B|^2 for the B-H tables used). beta = 1 for linear materials,
// nu_hat <= 0, or B = 0.
__global__ void __launch_bounds__(128) k_seed_midpoint(ElemData m, const double *__restrict__ sol,
                                                       const double *__restrict__ nu_hat, MaterialParams mp,
                                                       double max_scale, double *__restrict__ bscale) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= m.ne) return;
    const int tag = m.tags[e];
    const double target = nu_hat[e];
    double beta = 1.0;
    if (target > 0.0 && __ldg(mp.is_non + tag - 1) != 0.0) {
        int4 t = m.tet[e];
        int d[6];
        load_dofs(m.dofs, e, d);
        unsigned sb = m.signbits ? m.signbits[e] : derived_signs(t);
        Geo g;
        geometry(m.xyz, t, g);
        double C[6][3];
        curls_standard(g, C);
        double a[6];
#pragma unroll
        for (int i = 0; i < 6; i++) a[i] = d[i] >= 0 ? flip(__ldg(sol + d[i]), (sb >> i) & 1) : 0.0;
        double B[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            double v = a[0] * C[0][c];
#pragma unroll
            for (int i = 1; i < 6; i++) v = v + a[i] * C[i][c];
            B[c] = v;
        }
        const double bp = sqrt(dot3(B, B));
        if (bp > 0.0) {
            double lo = 0.0, hi = 4.0 * __ldg(mp.max_bsq + tag - 1), nu, dnu;
            material_eval(mp, tag, hi, nu, dnu);
            double s_hat = hi;
            if (target < nu) {
                material_eval(mp, tag, 0.0, nu, dnu);
                if (target <= nu) {
                    s_hat = 0.0;
                } else {
                    for (int it = 0; it < 64; it++) {
                        double mid = 0.5 * (lo + hi);
                        material_eval(mp, tag, mid, nu, dnu);
                        if (nu < target) lo = mid;
                        else hi = mid;
                    }
                    s_hat = 0.5 * (lo + hi);
                }
            }
            beta = 0.5 * (bp + sqrt(s_hat)) / bp;
            beta = fmin(fmax(beta, 1.0 / max_scale), max_scale);  // trust region of the seed
        }
    }
    bscale[e] = beta;
}

// ---- phase 1: curl-curl K(nu) ----------------------------------------------

template <bool STDCURL>
__global__ void __launch_bounds__(128) k_stiffness_elems(ElemData m, const double *__restrict__ nu_e,
                                                         QuadParams qp, double *__restrict__ scratch) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= m.ne) return;
    int4 t = m.tet[e];
    unsigned sb = m.signbits ? m.signbits[e] : derived_signs(t);
    Geo g;
    geometry(m.xyz, t, g);
    double nu = nu_e[e];
    double w[kMaxQuad];
    for (int q = 0; q < qp.nq; q++) w[q] = qp.qw[q] * g.adet;
    double K[6][6];
    if (STDCURL) {
        double C[6][3];
        curls_standard(g, C);
#pragma unroll
        for (int i = 0; i < 6; i++)
#pragma unroll
            for (int j = i; j < 6; j++) {
                double v = qsum(dot3(C[i], C[j]) * nu, w, qp.nq, qp.uniform_w);
                K[i][j] = v;
                K[j][i] = v;
            }
    } else {
#pragma unroll
        for (int i = 0; i < 6; i++)
#pragma unroll
            for (int j = 0; j < 6; j++) K[i][j] = 0.0;
        for (int q = 0; q < qp.nq; q++) {
            double C[6][3];
            curls_generic(g, qp.curl_ref, q, C);
#pragma unroll
            for (int i = 0; i < 6; i++)
#pragma unroll
                for (int j = 0; j < 6; j++) K[i][j] = K[i][j] + dot3(C[i], C[j]) * nu * w[q];
        }
    }
    double *dst = scratch + e * kScratchPerElem;
#pragma unroll
    for (int i = 0; i < 6; i++) {
        double row[6];
#pragma unroll
        for (int j = 0; j < 6; j++) row[j] = flip(K[i][j], ((sb >> i) ^ (sb >> j)) & 1);
        store_row(dst + i * kScratchStride, row, 0.0);
    }
}

// ---- phase 1: sigma-mass M(sigma) and source F ---------------------------------

__global__ void __launch_bounds__(128) k_mass_elems(ElemData m, const double *__restrict__ sigma_e,
                                                    QuadParams qp, double *__restrict__ scratch) {
    __shared__ double sref[18 * kMaxQuad];
    for (int i = threadIdx.x; i < 18 * qp.nq; i += blockDim.x) sref[i] = qp.val_ref[i];
    __syncthreads();
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= m.ne) return;
    int4 t = m.tet[e];
    unsigned sb = m.signbits ? m.signbits[e] : derived_signs(t);
    Geo g;
    geometry(m.xyz, t, g);
    double iv[3][3];
    inverse3(g, iv);
    double sigma = sigma_e ? sigma_e[e] : 1.0;
    double M[6][6];
#pragma unroll
    for (int i = 0; i < 6; i++)
#pragma unroll
        for (int j = 0; j < 6; j++) M[i][j] = 0.0;
    if (fabs(sigma) > 1e-12) {  // zero-sigma elements contribute explicit zeros
        for (int q = 0; q < qp.nq; q++) {
            double w = qp.qw[q] * g.adet;
            double N[6][3];
#pragma unroll
            for (int i = 0; i < 6; i++) {
                double r0 = sref[i + 18 * q], r1 = sref[i + 6 + 18 * q], r2 = sref[i + 12 + 18 * q];
#pragma unroll
                for (int c = 0; c < 3; c++) N[i][c] = iv[0][c] * r0 + iv[1][c] * r1 + iv[2][c] * r2;
            }
#pragma unroll
            for (int i = 0; i < 6; i++)
#pragma unroll
                for (int j = i; j < 6; j++) {
                    double v = M[i][j] + dot3(N[i], N[j]) * sigma * w;
                    M[i][j] = v;
                    M[j][i] = v;
                }
        }
    }
    double *dst = scratch + e * kScratchPerElem;
#pragma unroll
    for (int i = 0; i < 6; i++) {
        double row[6];
#pragma unroll
        for (int j = 0; j < 6; j++) row[j] = flip(M[i][j], ((sb >> i) ^ (sb >> j)) & 1);
        store_row(dst + i * kScratchStride, row, 0.0);
    }
}

__global__ void __launch_bounds__(128) k_source_elems(ElemData m, const double *__restrict__ js,
                                                      QuadParams qp, double *__restrict__ scratch) {
    __shared__ double sref[18 * kMaxQuad];
    for (int i = threadIdx.x; i < 18 * qp.nq; i += blockDim.x) sref[i] = qp.val_ref[i];
    __syncthreads();
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= m.ne) return;
    int4 t = m.tet[e];
    unsigned sb = m.signbits ? m.signbits[e] : derived_signs(t);
    Geo g;
    geometry(m.xyz, t, g);
    double iv[3][3];
    inverse3(g, iv);
    double jp[3] = {js[3 * e], js[3 * e + 1], js[3 * e + 2]};
    double jr[3];
#pragma unroll
    for (int r = 0; r < 3; r++) jr[r] = iv[r][0] * jp[0] + iv[r][1] * jp[1] + iv[r][2] * jp[2];
    double f[6] = {0, 0, 0, 0, 0, 0};
    if (fabs(jp[0]) > 1e-12 || fabs(jp[1]) > 1e-12 || fabs(jp[2]) > 1e-12) {
        for (int q = 0; q < qp.nq; q++) {
            double w = qp.qw[q] * g.adet;
#pragma unroll
            for (int i = 0; i < 6; i++) {
                double r[3] = {sref[i + 18 * q], sref[i + 6 + 18 * q], sref[i + 12 + 18 * q]};
                f[i] = f[i] + dot3(jr, r) * w;
            }
        }
    }
    double *dst = scratch + e * kScratchPerElem;
#pragma unroll
    for (int i = 0; i < 6; i++) dst[i * kScratchStride + 6] = flip(f[i], (sb >> i) & 1);
}

// ---- winding (coil current) vector ---------------------------------------------
// assemble_winding_kernel_mex.cpp:13-127 per element: zero outside the coil region
// (:54-61), else the direction (per-element field or uniform, :78-87) times the scale
// (:90-92), mapped by J^{-1} (:96) and integrated against the reference basis with
// no cut-off (:99-114), signed (:124). Writes the residual slot of the element scratch
// and/or the reference's (I, V) pairs (I = 0 outside the coil).
struct WindingArgs {
    int coil;
    const double *field;  // [Ne][3] or NULL
    double dir[3];
    double scale;
};

__global__ void __launch_bounds__(128) k_winding_elems(ElemData m, WindingArgs wa, QuadParams qp,
                                                       double *__restrict__ scratch, double *__restrict__ I,
                                                       double *__restrict__ V) {
    __shared__ double sref[18 * kMaxQuad];
    for (int i = threadIdx.x; i < 18 * qp.nq; i += blockDim.x) sref[i] = qp.val_ref[i];
    __syncthreads();
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= m.ne) return;
    double f[6] = {0, 0, 0, 0, 0, 0};
    const bool in_coil = (int)m.tags[e] == wa.coil;
    unsigned sb = 0;
    if (in_coil) {
        const int4 t = m.tet[e];
        sb = m.signbits ? m.signbits[e] : derived_signs(t);
        Geo g;
        geometry(m.xyz, t, g);
        double iv[3][3];
        inverse3(g, iv);
        const double *d = wa.field ? wa.field + 3 * e : wa.dir;
        const double jp[3] = {d[0] * wa.scale, d[1] * wa.scale, d[2] * wa.scale};
        double jr[3];
#pragma unroll
        for (int r = 0; r < 3; r++) jr[r] = iv[r][0] * jp[0] + iv[r][1] * jp[1] + iv[r][2] * jp[2];
        for (int q = 0; q < qp.nq; q++) {
            const double w = qp.qw[q] * g.adet;
#pragma unroll
            for (int i = 0; i < 6; i++) {
                const double r[3] = {sref[i + 18 * q], sref[i + 6 + 18 * q], sref[i + 12 + 18 * q]};
                f[i] = f[i] + dot3(jr, r) * w;
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 6; i++) {
        const double v = in_coil ? flip(f[i], (sb >> i) & 1) : 0.0;
        if (scratch) scratch[e * kScratchPerElem + i * kScratchStride + 6] = v;
        if (I) {
            I[6 * e + i] = in_coil ? (double)(m.dofs[6 * e + i] + 1) : 0.0;
            V[6 * e + i] = v;
        }
    }
}

// ---- element B (post-processing / predictor features) -------------------------

__global__ void __launch_bounds__(128) k_element_b(ElemData m, const double *__restrict__ sol,
                                                   double *__restrict__ bout, double *__restrict__ bsq,
                                                   MaterialParams mp, double *__restrict__ nu_out,
                                                   double *__restrict__ dnu_out) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= m.ne) return;
    int4 t = m.tet[e];
    int d[6];
    load_dofs(m.dofs, e, d);
    unsigned sb = m.signbits ? m.signbits[e] : derived_signs(t);
    Geo g;
    geometry(m.xyz, t, g);
    double C[6][3];
    curls_standard(g, C);
    double a[6];
#pragma unroll
    for (int i = 0; i < 6; i++) a[i] = d[i] >= 0 ? flip(__ldg(sol + d[i]), (sb >> i) & 1) : 0.0;
    double B[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        double s = a[0] * C[0][c];
#pragma unroll
        for (int i = 1; i < 6; i++) s = s + a[i] * C[i][c];
        B[c] = s;
    }
    if (bout) {
        bout[3 * e] = B[0];
        bout[3 * e + 1] = B[1];
        bout[3 * e + 2] = B[2];
    }
    if (bsq) bsq[e] = dot3(B, B);
    if (nu_out || dnu_out) {  // the reluctivity the Jacobian kernel evaluates for this element
        double nu, dnu;
        material_eval(mp, m.tags[e], dot3(B, B), nu, dnu);
        if (nu_out) nu_out[e] = nu;
        if (dnu_out) dnu_out[e] = dnu;
    }
}

// ---- phase 2: fixed-order row reduction --------------------------------------

template <bool MAT, bool VEC, bool WIDE>
__global__ void __launch_bounds__(128) k_rows_reduce(RowPlan rp, const double *__restrict__ scratch,
                                                     double *__restrict__ vals, double *__restrict__ vec) {
    extern __shared__ double sacc[];
    int64_t a0 = (int64_t)blockIdx.x * blockDim.x;
    int64_t a = a0 + threadIdx.x;
    int64_t a_end = a0 + blockDim.x < rp.ndof ? a0 + blockDim.x : rp.ndof;
    int32_t base = rp.row_ptr[a0];
    int32_t span = rp.row_ptr[a_end] - base;
    if (MAT) {
        for (int32_t i = threadIdx.x; i < span; i += blockDim.x) sacc[i] = 0.0;
        __syncthreads();
    }
    if (a < rp.ndof) {
        int32_t off = MAT ? rp.row_ptr[a] - base : 0;
        double r = 0.0;
        int32_t t1 = rp.inc_ptr[a + 1];
        for (int32_t t = rp.inc_ptr[a]; t < t1; t++) {
            uint32_t ew = rp.inc_elem[t];
            const double *src = scratch + (int64_t)(ew & 0x1FFFFFFFu) * kScratchPerElem +
                                (ew >> 29) * kScratchStride;
            if (MAT) {
                const double2 *p2 = reinterpret_cast<const double2 *>(src);
                double2 v01 = __ldg(p2), v23 = __ldg(p2 + 1), v45 = __ldg(p2 + 2);
                double v[6] = {v01.x, v01.y, v23.x, v23.y, v45.x, v45.y};
                if (!WIDE) {
                    uint32_t pw = rp.inc_pos[t];
#pragma unroll
                    for (int j = 0; j < 6; j++) {
                        uint32_t p = (pw >> (5 * j)) & 31u;
                        if (p != (uint32_t)kCompactMaxRow) sacc[off + p] = sacc[off + p] + v[j];
                    }
                } else {
                    uint32_t w0 = rp.inc_pos[2 * (int64_t)t], w1 = rp.inc_pos[2 * (int64_t)t + 1];
#pragma unroll
                    for (int j = 0; j < 6; j++) {
                        uint32_t p = (j < 4 ? (w0 >> (8 * j)) : (w1 >> (8 * (j - 4)))) & 255u;
                        if (p != (uint32_t)kWideMaxRow) sacc[off + p] = sacc[off + p] + v[j];
                    }
                }
            }
            if (VEC) r = r + __ldg(src + 6);
        }
        if (VEC) vec[a] = r;
    }
    if (MAT) {
        __syncthreads();
        for (int32_t i = threadIdx.x; i < span; i += blockDim.x) vals[base + i] = sacc[i];
    }
}

// ---- MEX layout -------------------------------------------------------------

// Scratch -> reference triplets: entry (i, j) of element e at 36e + 6j + i.
__global__ void k_to_triplets(const double *__restrict__ scratch, const int32_t *__restrict__ dofs,
                              int64_t ne, int calcj, double *__restrict__ I, double *__restrict__ J,
                              double *__restrict__ V, double *__restrict__ Ridx,
                              double *__restrict__ Rval) {
    int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= 36 * ne) return;
    int64_t e = s / 36;
    int r = (int)(s - 36 * e);
    int j = r / 6, i = r - 6 * j;
    const double *src = scratch + e * kScratchPerElem;
    if (calcj) {
        I[s] = (double)(dofs[6 * e + i] + 1);
        J[s] = (double)(dofs[6 * e + j] + 1);
        V[s] = src[i * kScratchStride + j];
    }
    if (Ridx && r < 6) {
        Ridx[6 * e + r] = (double)(dofs[6 * e + r] + 1);
        Rval[6 * e + r] = src[r * kScratchStride + 6];
    }
}

inline unsigned blocks(int64_t n, int b) { return (unsigned)((n + b - 1) / b); }

}  // namespace

// ---- launchers -----------------------------------------------------------------

int launch_jacobian_elems(const ElemData &m, const double *sol, const QuadParams &qp,
                          const MaterialParams &mp, int calcj, double *scratch, cudaStream_t s) {
    unsigned g = blocks(m.ne, 128);
    if (qp.standard_curl) {
        if (calcj) k_jacobian_elems<true, true><<<g, 128, 0, s>>>(m, sol, qp, mp, scratch);
        else k_jacobian_elems<false, true><<<g, 128, 0, s>>>(m, sol, qp, mp, scratch);
    } else {
        if (calcj) k_jacobian_elems<true, false><<<g, 128, 0, s>>>(m, sol, qp, mp, scratch);
        else k_jacobian_elems<false, false><<<g, 128, 0, s>>>(m, sol, qp, mp, scratch);
    }
    return cudaPeekAtLastError() == cudaSuccess ? MAG_OK : MAG_E_CUDA;
}

int launch_jacobian_seeded_elems(const ElemData &m, const double *sol, const double *bscale, const QuadParams &qp,
                                 const MaterialParams &mp, double *scratch, cudaStream_t s) {
    k_jacobian_seeded_elems<<<blocks(m.ne, 128), 128, 0, s>>>(m, sol, bscale, qp, mp, scratch);
    return cudaPeekAtLastError() == cudaSuccess ? MAG_OK : MAG_E_CUDA;
}

int launch_seed_midpoint(const ElemData &m, const double *sol, const double *nu_hat, const MaterialParams &mp,
                         double max_scale, double *bscale, cudaStream_t s) {
    k_seed_midpoint<<<blocks(m.ne, 128), 128, 0, s>>>(m, sol, nu_hat, mp, max_scale, bscale);
    return cudaPeekAtLastError() == cudaSuccess ? MAG_OK : MAG_E_CUDA;
}

int launch_stiffness_elems(const ElemData &m, const double *nu, const QuadParams &qp,
                           double *scratch, cudaStream_t s) {
    unsigned g = blocks(m.ne, 128);
    if (qp.standard_curl) k_stiffness_elems<true><<<g, 128, 0, s>>>(m, nu, qp, scratch);
    else k_stiffness_elems<false><<<g, 128, 0, s>>>(m, nu, qp, scratch);
    return cudaPeekAtLastError() == cudaSuccess ? MAG_OK : MAG_E_CUDA;
}

int launch_mass_elems(const ElemData &m, const double *sigma, const QuadParams &qp, double *scratch,
                      cudaStream_t s) {
    k_mass_elems<<<blocks(m.ne, 128), 128, 0, s>>>(m, sigma, qp, scratch);
    return cudaPeekAtLastError() == cudaSuccess ? MAG_OK : MAG_E_CUDA;
}

int launch_source_elems(const ElemData &m, const double *js, const QuadParams &qp, double *scratch,
                        cudaStream_t s) {
    k_source_elems<<<blocks(m.ne, 128), 128, 0, s>>>(m, js, qp, scratch);
    return cudaPeekAtLastError() == cudaSuccess ? MAG_OK : MAG_E_CUDA;
}

int launch_winding_elems(const ElemData &m, int coil, const double *field, const double dir[3], double scale,
                         const QuadParams &qp, double *scratch, double *I, double *V, cudaStream_t s) {
    WindingArgs wa{coil, field, {dir[0], dir[1], dir[2]}, scale};
    k_winding_elems<<<blocks(m.ne, 128), 128, 0, s>>>(m, wa, qp, scratch, I, V);
    return cudaPeekAtLastError() == cudaSuccess ? MAG_OK : MAG_E_CUDA;
}

int launch_element_b(const ElemData &m, const double *sol, double *b, double *bsq, cudaStream_t s,
                     const MaterialParams *mp, double *nu, double *dnu) {
    MaterialParams none{};
    k_element_b<<<blocks(m.ne, 128), 128, 0, s>>>(m, sol, b, bsq, mp ? *mp : none, mp ? nu : nullptr,
                                                  mp ? dnu : nullptr);
    return cudaPeekAtLastError() == cudaSuccess ? MAG_OK : MAG_E_CUDA;
}

int launch_rows_reduce(const RowPlan &rp, int max_row, const double *scratch, double *vals,
                       double *vec, cudaStream_t s) {
    const int b = 128;
    unsigned g = blocks(rp.ndof, b);
    size_t smem = vals ? (size_t)b * max_row * sizeof(double) : 0;
    if (smem > 200 * 1024) return MAG_E_UNSUPPORTED;
    bool mat = vals != nullptr, v = vec != nullptr;
#define MAG_P2(M, V, W)                                                                          \
    do {                                                                                         \
        auto kern = k_rows_reduce<M, V, W>;                                                      \
        if (smem > 48 * 1024)                                                                    \
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);  \
        kern<<<g, b, smem, s>>>(rp, scratch, vals, vec);                                         \
    } while (0)
    if (rp.wide) {
        if (mat && v) MAG_P2(true, true, true);
        else if (mat) MAG_P2(true, false, true);
        else if (v) MAG_P2(false, true, true);
    } else {
        if (mat && v) MAG_P2(true, true, false);
        else if (mat) MAG_P2(true, false, false);
        else if (v) MAG_P2(false, true, false);
    }
#undef MAG_P2
    return cudaPeekAtLastError() == cudaSuccess ? MAG_OK : MAG_E_CUDA;
}

int launch_to_triplets(const double *scratch, const int32_t *dofs, int64_t ne, int calcj, double *I,
                       double *J, double *V, double *Ridx, double *Rval, cudaStream_t s) {
    k_to_triplets<<<blocks(36 * ne, 256), 256, 0, s>>>(scratch, dofs, ne, calcj, I, J, V, Ridx, Rval);
    return cudaPeekAtLastError() == cudaSuccess ? MAG_OK : MAG_E_CUDA;
}

}  // namespace mag
