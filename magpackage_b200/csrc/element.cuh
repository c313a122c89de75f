// Per-element device math shared by the assembly kernels (FP64).
//
// Evaluation order follows the reference MEX sources operation for operation
// (src/mex/MexElemUtils.hpp:35-66, src/mex/MexMaterialUtils.hpp:24-87,
// src/mex/assemble_jacobian_kernel_mex.cpp:61-152), so translation units that
// include this header must be compiled with -fmad=false.
#pragma once

#include "common.cuh"

namespace mag {
namespace elem {

__device__ __forceinline__ unsigned derived_signs(int4 t) {
    // bit k set <=> local edge k runs from the larger to the smaller node id
    int n[4] = {t.x, t.y, t.z, t.w};
    unsigned b = 0;
#pragma unroll
    for (int k = 0; k < 6; k++) b |= (n[edge_a(k)] < n[edge_b(k)] ? 0u : 1u) << k;
    return b;
}

// -v when neg is set: negation is a flip of the sign bit, done here as one integer XOR of
// the high word instead of a select between v and -v.
__device__ __forceinline__ double flip(double v, unsigned neg) {
    return __longlong_as_double(__double_as_longlong(v) ^ ((long long)(neg & 1u) << 63));
}

struct Geo {
    double J[3][3];
    double det, rdet, adet;
};

__device__ __forceinline__ void geometry_v(double4 v0, double4 v1, double4 v2, double4 v3, Geo &g) {
    g.J[0][0] = v1.x - v0.x; g.J[1][0] = v1.y - v0.y; g.J[2][0] = v1.z - v0.z;
    g.J[0][1] = v2.x - v0.x; g.J[1][1] = v2.y - v0.y; g.J[2][1] = v2.z - v0.z;
    g.J[0][2] = v3.x - v0.x; g.J[1][2] = v3.y - v0.y; g.J[2][2] = v3.z - v0.z;
    const double(*J)[3] = g.J;
    double m0 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
    double m1 = J[1][0] * J[2][2] - J[1][2] * J[2][0];
    double m2 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
    g.det = J[0][0] * m0 - J[0][1] * m1 + J[0][2] * m2;
    g.rdet = 1.0 / g.det;
    g.adet = fabs(g.det);
}

__device__ __forceinline__ void geometry(const double4 *__restrict__ xyz, int4 t, Geo &g) {
    geometry_v(xyz[t.x], xyz[t.y], xyz[t.z], xyz[t.w], g);
}

// Physical curls of the six Whitney functions, C_i = J c_i / det, for the
// standard reference curls c = 2 grad(L_a) x grad(L_b):
//   (0,-2,2) (2,0,-2) (-2,2,0) (0,0,2) (0,-2,0) (2,0,0).
// The reference forms J c with three products and two additions; with these
// c entries that sum is exactly 2(J_b - J_a) (scaling by 2 and adding signed
// zeros are exact), and 2 d / det rounds like d * (2/det).
__device__ __forceinline__ void curls_standard(const Geo &g, double C[6][3]) {
    double r2 = 2.0 * g.rdet;
#pragma unroll
    for (int r = 0; r < 3; r++) {
        C[0][r] = (g.J[r][2] - g.J[r][1]) * r2;
        C[1][r] = (g.J[r][0] - g.J[r][2]) * r2;
        C[2][r] = (g.J[r][1] - g.J[r][0]) * r2;
        C[3][r] = g.J[r][2] * r2;
        C[4][r] = -(g.J[r][1] * r2);
        C[5][r] = g.J[r][0] * r2;
    }
}

// Any reference curl table (entry (i,c) of point q at i + 6c + 18q).
__device__ __forceinline__ void curls_generic(const Geo &g, const double *__restrict__ ref, int q,
                                              double C[6][3]) {
#pragma unroll
    for (int i = 0; i < 6; i++) {
        double c0 = ref[i + 18 * q], c1 = ref[i + 6 + 18 * q], c2 = ref[i + 12 + 18 * q];
#pragma unroll
        for (int r = 0; r < 3; r++) C[i][r] = (g.J[r][0] * c0 + g.J[r][1] * c1 + g.J[r][2] * c2) * g.rdet;
    }
}

__device__ __forceinline__ double dot3(const double *a, const double *b) {
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

// nu(s) and d nu/ds, s = |B|^2, per MexMaterialUtils.hpp:24-87.
__device__ __forceinline__ void material_eval(const MaterialParams &mp, int tag, double s,
                                              double &nu, double &dnu) {
    int m = tag - 1;
    if (__ldg(mp.is_non + m) == 0.0) {
        nu = __ldg(mp.lin + m);
        dnu = 0.0;
        return;
    }
    double smax = __ldg(mp.max_bsq + m);
    bool beyond = s > smax;
    double x = beyond ? smax : s;
    const double *b = mp.breaks + __ldg(mp.start + m);
    int pieces = __ldg(mp.count + m);
    int k = 0, lo = 0, hi = pieces - 1;
    // The last break <= x (0 if none), as the reference's binary search over the whole table
    // finds it (MexMaterialUtils.hpp:47-59). With buckets, the search runs inside the window
    // of x's uniform-in-s bucket i: the host stored the answers at the edges e(i-1) and e(i+2),
    // one bucket wider on each side than the bucket, so the answer for x lies in [lo, hi]
    // whichever neighbouring bucket the rounding of (x - origin) * scale picks, and the binary
    // search inside the window returns the same index (NaN or x below the first break: 0).
    const double scale = mp.bucket ? __ldg(mp.bucket_geom + 2 * m + 1) : 0.0;
    if (scale > 0.0) {
        const double f = (x - __ldg(mp.bucket_geom + 2 * m)) * scale;
        const int i = !(f >= 0.0) ? 0 : (f >= (double)(kMatBuckets - 1) ? kMatBuckets - 1 : (int)f);
        const int *w = mp.bucket + 2 * kMatBuckets * m + i;
        lo = __ldg(w);
        hi = __ldg(w + kMatBuckets);
        k = lo;
    }
    while (lo <= hi) {
        int mid = lo + (hi - lo) / 2;
        if (x >= __ldg(b + mid)) {
            k = mid;
            lo = mid + 1;
        } else {
            hi = mid - 1;
        }
    }
    if (k >= pieces) k = pieces - 1;
    if (k < 0) k = 0;
    const double *c = mp.coefs + __ldg(mp.coef_start + m) + 4 * k;
    double c0 = __ldg(c), c1 = __ldg(c + 1), c2 = __ldg(c + 2), c3 = __ldg(c + 3);
    double t = x - __ldg(b + k);
    double v = ((c0 * t + c1) * t + c2) * t + c3;
    double dv = (3.0 * c0 * t + 2.0 * c1) * t + c2;
    if (beyond) v = v + dv * (s - smax);
    double nu0 = __ldg(mp.lin + m);
    if (v > nu0 || v < 1e-7) {
        v = nu0;
        dv = 0.0;
    }
    nu = v;
    dnu = dv;
}

__device__ __forceinline__ void load_dofs(const int32_t *__restrict__ dofs, int64_t e, int d[6]) {
    const int2 *p = reinterpret_cast<const int2 *>(dofs + 6 * e);
    int2 a = p[0], b = p[1], c = p[2];
    d[0] = a.x; d[1] = a.y; d[2] = b.x; d[3] = b.y; d[4] = c.x; d[5] = c.y;
}

// Sum over quadrature points of v * w_q, accumulated in point order from zero.
__device__ __forceinline__ double qsum(double v, const double *w, int nq, int uniform) {
    double u = v * w[0];
    double acc = u;
    if (uniform) {
        for (int q = 1; q < nq; q++) acc = acc + u;
    } else {
        for (int q = 1; q < nq; q++) acc = acc + v * w[q];
    }
    return acc;
}

__device__ __forceinline__ void store_row(double *__restrict__ dst, const double k[6], double r) {
    double2 *p = reinterpret_cast<double2 *>(dst);
    p[0] = make_double2(k[0], k[1]);
    p[1] = make_double2(k[2], k[3]);
    p[2] = make_double2(k[4], k[5]);
    p[3] = make_double2(r, 0.0);
}

__device__ __forceinline__ void inverse3(const Geo &g, double iv[3][3]) {
    const double(*J)[3] = g.J;
    double s = 1.0 / g.det;
    iv[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) * s;
    iv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * s;
    iv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * s;
    iv[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) * s;
    iv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * s;
    iv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * s;
    iv[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) * s;
    iv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * s;
    iv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * s;
}


// Element Newton block: residual res[i] and tangent K[i][j] (signs not yet
// applied) from the element geometry g and the signed edge values a[6],
// evaluated as assemble_jacobian_kernel_mex.cpp:92-131 does.
template <bool CALCJ, bool STDCURL>
__device__ __forceinline__ void jacobian_block(const Geo &g, const double a[6], int tag,
                                               const QuadParams &qp, const MaterialParams &mp,
                                               double res[6], double K[6][6]) {
    double w[kMaxQuad];
    for (int q = 0; q < qp.nq; q++) w[q] = qp.qw[q] * g.adet;

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
        material_eval(mp, tag, dot3(B, B), nu, dnu);
        double b[6];
#pragma unroll
        for (int i = 0; i < 6; i++) {
            b[i] = dot3(B, C[i]);
            res[i] = qsum(nu * b[i], w, qp.nq, qp.uniform_w);
        }
        if (CALCJ) {
            if (dnu == 0.0) {
                // linear response: nu*Ci.Cj + (+-0) is symmetric bit for bit
#pragma unroll
                for (int i = 0; i < 6; i++)
#pragma unroll
                    for (int j = i; j < 6; j++) {
                        double v = qsum(nu * dot3(C[i], C[j]), w, qp.nq, qp.uniform_w);
                        K[i][j] = v;
                        K[j][i] = v;
                    }
            } else {
                double g2 = 2.0 * dnu;
#pragma unroll
                for (int i = 0; i < 6; i++) {
                    double gi = g2 * b[i];
#pragma unroll
                    for (int j = 0; j < 6; j++)
                        K[i][j] = qsum(nu * dot3(C[i], C[j]) + gi * b[j], w, qp.nq, qp.uniform_w);
                }
            }
        }
    } else {
#pragma unroll
        for (int i = 0; i < 6; i++) {
            res[i] = 0.0;
#pragma unroll
            for (int j = 0; j < 6; j++) K[i][j] = 0.0;
        }
        for (int q = 0; q < qp.nq; q++) {
            double C[6][3];
            curls_generic(g, qp.curl_ref, q, C);
            double B[3] = {0.0, 0.0, 0.0};
#pragma unroll
            for (int i = 0; i < 6; i++)
#pragma unroll
                for (int c = 0; c < 3; c++) B[c] = B[c] + a[i] * C[i][c];
            double nu, dnu;
            material_eval(mp, tag, dot3(B, B), nu, dnu);
#pragma unroll
            for (int i = 0; i < 6; i++) {
                double bi = dot3(B, C[i]);
                res[i] = res[i] + nu * bi * w[q];
                if (CALCJ) {
#pragma unroll
                    for (int j = 0; j < 6; j++)
                        K[i][j] = K[i][j] + (nu * dot3(C[i], C[j]) + 2.0 * dnu * bi * dot3(B, C[j])) * w[q];
                }
            }
        }
    }
}

}  // namespace elem
}  // namespace mag
