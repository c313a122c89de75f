/*
 * CPU restatement of the reference's four Nedelec element kernels.
 * TEST INFRASTRUCTURE ONLY (results to compare the GPU with; see oracle.h).
 *
 * The floating-point operations are evaluated in the same order as the
 * reference MEX sources so that this restatement is bit-identical to them
 * (compiled without FMA contraction, see oracle/Makefile). Sources followed:
 *   geometry       src/mex/MexElemUtils.hpp:35-66 (J columns = x_{k+1}-x_1,
 *                  det by first-row cofactors, inverse = adjugate * (1/det))
 *   material       src/mex/MexMaterialUtils.hpp:24-87
 *   Jacobian       src/mex/assemble_jacobian_kernel_mex.cpp:61-152
 *   curl-curl      src/mex/assemble_curl_curl_kernel_mex.cpp:44-121
 *   mass           src/mex/assemble_mass_kernel_mex.cpp:167-248
 *   source         src/mex/assemble_source_kernel_mex.cpp:46-114
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>

typedef struct {
    double g[3][3]; /* g[r][c]: row r (x,y,z), column c (edge vector c) */
} mat3;

/* Gather the 4 vertices of element e (1-based node ids stored as doubles). */
static void gather_vertices(const double *P, const double *T, int64_t e, double v[4][3]) {
    for (int a = 0; a < 4; a++) {
        int64_t node = (int64_t)T[4 * e + a] - 1;
        for (int c = 0; c < 3; c++) v[a][c] = P[3 * node + c];
    }
}

/* MexElemUtils.hpp:35-49: columns are the edge vectors from vertex 1; the
 * determinant is expanded along the first row. */
static double edge_matrix(const double v[4][3], mat3 *m) {
    for (int c = 0; c < 3; c++)
        for (int r = 0; r < 3; r++) m->g[r][c] = v[c + 1][r] - v[0][r];
    const double(*g)[3] = m->g;
    double m0 = g[1][1] * g[2][2] - g[1][2] * g[2][1];
    double m1 = g[1][0] * g[2][2] - g[1][2] * g[2][0];
    double m2 = g[1][0] * g[2][1] - g[1][1] * g[2][0];
    return g[0][0] * m0 - g[0][1] * m1 + g[0][2] * m2;
}

/* MexElemUtils.hpp:52-66: adjugate entries scaled by 1/det. */
static void inverse3(const mat3 *m, double det, mat3 *inv) {
    const double(*g)[3] = m->g;
    double s = 1.0 / det;
    inv->g[0][0] = (g[1][1] * g[2][2] - g[1][2] * g[2][1]) * s;
    inv->g[0][1] = (g[0][2] * g[2][1] - g[0][1] * g[2][2]) * s;
    inv->g[0][2] = (g[0][1] * g[1][2] - g[0][2] * g[1][1]) * s;
    inv->g[1][0] = (g[1][2] * g[2][0] - g[1][0] * g[2][2]) * s;
    inv->g[1][1] = (g[0][0] * g[2][2] - g[0][2] * g[2][0]) * s;
    inv->g[1][2] = (g[0][2] * g[1][0] - g[0][0] * g[1][2]) * s;
    inv->g[2][0] = (g[1][0] * g[2][1] - g[1][1] * g[2][0]) * s;
    inv->g[2][1] = (g[0][1] * g[2][0] - g[0][0] * g[2][1]) * s;
    inv->g[2][2] = (g[0][0] * g[1][1] - g[0][1] * g[1][0]) * s;
}

/* y = M x and y = M^T x, each component summed left to right. */
static void apply(const mat3 *m, const double x[3], double y[3]) {
    for (int r = 0; r < 3; r++) y[r] = m->g[r][0] * x[0] + m->g[r][1] * x[1] + m->g[r][2] * x[2];
}
static void apply_t(const mat3 *m, const double x[3], double y[3]) {
    for (int c = 0; c < 3; c++) y[c] = m->g[0][c] * x[0] + m->g[1][c] * x[1] + m->g[2][c] * x[2];
}

static double dot3(const double a[3], const double b[3]) {
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

/* Reference basis data is [6 x 3 x nq] column-major: entry (i, comp, q). */
static void ref_vec(const double *R, int i, int q, double out[3]) {
    for (int c = 0; c < 3; c++) out[c] = R[i + 6 * c + 18 * q];
}

/* MexMaterialUtils.hpp:24-87: reluctivity and d(nu)/d(|B|^2) at s = |B|^2.
 * Tags are 1-based; the material tables are indexed by tag-1. */
static void material_eval(double s, int tag, const double *lin, const double *isNon,
                          const double *maxB, const double *brk, const double *coe,
                          const double *start, const double *cnt, const double *coeStart,
                          double *nu_out, double *dnu_out) {
    int m = tag - 1;
    if (isNon[m] == 0.0) {
        *nu_out = lin[m];
        *dnu_out = 0.0;
        return;
    }
    double smax = maxB[m];
    int beyond = s > smax;
    double x = beyond ? smax : s;
    const double *b = brk + (int)start[m];
    int pieces = (int)cnt[m];
    /* largest k in [0, pieces-1] with x >= b[k]; k = 0 if none */
    int k = 0, lo = 0, hi = pieces - 1;
    while (lo <= hi) {
        int mid = lo + (hi - lo) / 2;
        if (x >= b[mid]) {
            k = mid;
            lo = mid + 1;
        } else {
            hi = mid - 1;
        }
    }
    if (k >= pieces) k = pieces - 1;
    if (k < 0) k = 0;
    const double *c = coe + (int)coeStart[m] + 4 * k;
    double t = x - b[k];
    double nu = ((c[0] * t + c[1]) * t + c[2]) * t + c[3];
    double dnu = (3.0 * c[0] * t + 2.0 * c[1]) * t + c[2];
    if (beyond) nu = nu + dnu * (s - smax);
    double nu0 = lin[m];
    if (nu > nu0 || nu < 1e-7) {
        nu = nu0;
        dnu = 0.0;
    }
    *nu_out = nu;
    *dnu_out = dnu;
}

void oracle_material_eval(const double *s, const double *Tags, int64_t n, const double *lin,
                          const double *isNon, const double *maxB, const double *brk,
                          const double *coe, const double *start, const double *cnt,
                          const double *coeStart, double *nu, double *dnu) {
    for (int64_t i = 0; i < n; i++)
        material_eval(s[i], (int)Tags[i], lin, isNon, maxB, brk, coe, start, cnt, coeStart, nu + i,
                      dnu + i);
}

void oracle_jacobian(const double *P, const double *T, int64_t Ne, const double *Dofs,
                     const double *Signs, const double *Tags, const double *SolA, const double *Qw,
                     int nq, const double *CurlRef, const double *lin, const double *isNon,
                     const double *maxB, const double *brk, const double *coe, const double *start,
                     const double *cnt, const double *coeStart, int calcJ, double *I, double *J,
                     double *V, double *Ridx, double *Rval) {
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < Ne; e++) {
        double v[4][3];
        mat3 m;
        gather_vertices(P, T, e, v);
        double det = edge_matrix(v, &m);
        double adet = fabs(det);
        double rdet = 1.0 / det;

        int dof[6];
        double sg[6], a[6];
        for (int i = 0; i < 6; i++) {
            dof[i] = (int)Dofs[6 * e + i];
            sg[i] = Signs[6 * e + i];
            a[i] = dof[i] - 1 >= 0 ? SolA[dof[i] - 1] * sg[i] : 0.0;
        }
        int tag = (int)Tags[e];
        double res[6] = {0, 0, 0, 0, 0, 0};
        double k[6][6] = {{0}};
        for (int q = 0; q < nq; q++) {
            double w = Qw[q] * adet;
            double cu[6][3];
            for (int i = 0; i < 6; i++) {
                double r[3], p[3];
                ref_vec(CurlRef, i, q, r);
                apply(&m, r, p); /* covariant Piola for curls: J c / det */
                for (int c = 0; c < 3; c++) cu[i][c] = p[c] * rdet;
            }
            double B[3] = {0, 0, 0};
            for (int i = 0; i < 6; i++)
                for (int c = 0; c < 3; c++) B[c] += a[i] * cu[i][c];
            double nu, dnu;
            material_eval(dot3(B, B), tag, lin, isNon, maxB, brk, coe, start, cnt, coeStart, &nu,
                          &dnu);
            for (int i = 0; i < 6; i++) {
                double bi = dot3(B, cu[i]);
                res[i] += nu * bi * w;
                if (!calcJ) continue;
                for (int j = 0; j < 6; j++) {
                    double cc = dot3(cu[i], cu[j]);
                    double bj = dot3(B, cu[j]);
                    k[i][j] += (nu * cc + 2.0 * dnu * bi * bj) * w;
                }
            }
        }
        for (int i = 0; i < 6; i++) {
            Ridx[6 * e + i] = (double)dof[i];
            Rval[6 * e + i] = res[i] * sg[i];
        }
        if (!calcJ) continue;
        /* column-major local order: column j outer, row i inner (:141-152) */
        for (int j = 0; j < 6; j++)
            for (int i = 0; i < 6; i++) {
                int64_t o = 36 * e + 6 * j + i;
                I[o] = (double)dof[i];
                J[o] = (double)dof[j];
                V[o] = k[i][j] * sg[i] * sg[j];
            }
    }
}

void oracle_curl_curl(const double *P, const double *T, int64_t Ne, const double *Dofs,
                      const double *Signs, const double *Nu, const double *Qw, int nq,
                      const double *CurlRef, double *I, double *J, double *V) {
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < Ne; e++) {
        double v[4][3];
        mat3 m;
        gather_vertices(P, T, e, v);
        double det = edge_matrix(v, &m);
        double adet = fabs(det);
        double rdet = 1.0 / det;
        double nu = Nu[e];
        double k[6][6] = {{0}};
        for (int q = 0; q < nq; q++) {
            double w = Qw[q] * adet;
            double cu[6][3];
            for (int i = 0; i < 6; i++) {
                double r[3], p[3];
                ref_vec(CurlRef, i, q, r);
                apply(&m, r, p);
                for (int c = 0; c < 3; c++) cu[i][c] = p[c] * rdet;
            }
            for (int i = 0; i < 6; i++)
                for (int j = 0; j < 6; j++) k[i][j] += dot3(cu[i], cu[j]) * nu * w;
        }
        for (int j = 0; j < 6; j++)
            for (int i = 0; i < 6; i++) {
                int64_t o = 36 * e + 6 * j + i;
                I[o] = (double)(int64_t)Dofs[6 * e + i];
                J[o] = (double)(int64_t)Dofs[6 * e + j];
                V[o] = k[i][j] * Signs[6 * e + i] * Signs[6 * e + j];
            }
    }
}

void oracle_mass(const double *P, const double *T, int64_t Ne, const double *Dofs,
                 const double *Signs, const double *Coeffs, int64_t ncoeff, const double *Qw, int nq,
                 const double *ValRef, double *I, double *J, double *V) {
    int per_element = Coeffs != 0 && ncoeff == Ne;
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < Ne; e++) {
        double v[4][3];
        mat3 m, inv;
        gather_vertices(P, T, e, v);
        double det = edge_matrix(v, &m);
        double adet = fabs(det);
        inverse3(&m, det, &inv);
        double sigma = per_element ? Coeffs[e] : 1.0;
        double k[6][6] = {{0}};
        if (fabs(sigma) > 1e-12) { /* zero-sigma elements still emit zeros (:69) */
            for (int q = 0; q < nq; q++) {
                double w = Qw[q] * adet;
                double nv[6][3];
                for (int i = 0; i < 6; i++) {
                    double r[3];
                    ref_vec(ValRef, i, q, r);
                    apply_t(&inv, r, nv[i]); /* N = J^{-T} N_ref */
                }
                for (int i = 0; i < 6; i++)
                    for (int j = 0; j < 6; j++) k[i][j] += dot3(nv[i], nv[j]) * sigma * w;
            }
        }
        for (int j = 0; j < 6; j++)
            for (int i = 0; i < 6; i++) {
                int64_t o = 36 * e + 6 * j + i;
                I[o] = (double)(int64_t)Dofs[6 * e + i];
                J[o] = (double)(int64_t)Dofs[6 * e + j];
                V[o] = k[i][j] * Signs[6 * e + i] * Signs[6 * e + j];
            }
    }
}

void oracle_source(const double *P, const double *T, int64_t Ne, const double *Dofs,
                   const double *Signs, const double *Js, const double *Qw, int nq,
                   const double *ValRef, double *I, double *V) {
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < Ne; e++) {
        double v[4][3];
        mat3 m, inv;
        gather_vertices(P, T, e, v);
        double det = edge_matrix(v, &m);
        double adet = fabs(det);
        inverse3(&m, det, &inv);
        double jp[3] = {Js[3 * e], Js[3 * e + 1], Js[3 * e + 2]};
        double jr[3];
        apply(&inv, jp, jr); /* (J^{-T})^T j = J^{-1} j, :69-76 */
        double f[6] = {0, 0, 0, 0, 0, 0};
        if (fabs(jp[0]) > 1e-12 || fabs(jp[1]) > 1e-12 || fabs(jp[2]) > 1e-12) {
            for (int q = 0; q < nq; q++) {
                double w = Qw[q] * adet;
                for (int i = 0; i < 6; i++) {
                    double r[3];
                    ref_vec(ValRef, i, q, r);
                    f[i] += dot3(jr, r) * w;
                }
            }
        }
        for (int i = 0; i < 6; i++) {
            I[6 * e + i] = (double)(int64_t)Dofs[6 * e + i];
            V[6 * e + i] = f[i] * Signs[6 * e + i];
        }
    }
}

/* Winding (coil current) vector element kernel, src/mex/assemble_winding_kernel_mex.cpp:13-127.
 * Elements whose tag is not the coil's give I = V = 0 (:54-61); the others use the
 * per-element direction DirField[3e..3e+2] or, when DirField is NULL, UniDir (:78-87),
 * scaled by Scale (:90-92), mapped by J^{-1} (:96) and integrated against the reference
 * basis without the source kernel's 1e-12 cut-off (:99-114). */
void oracle_winding(const double *P, const double *T, int64_t Ne, const double *Dofs,
                    const double *Signs, const double *Tags, double CoilID, const double *DirField,
                    const double *UniDir, double Scale, const double *Qw, int nq, const double *ValRef,
                    double *I, double *V) {
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < Ne; e++) {
        if ((int)Tags[e] != (int)CoilID) {
            for (int i = 0; i < 6; i++) I[6 * e + i] = V[6 * e + i] = 0.0;
            continue;
        }
        double v[4][3];
        mat3 m, inv;
        gather_vertices(P, T, e, v);
        double det = edge_matrix(v, &m);
        double adet = fabs(det);
        inverse3(&m, det, &inv);
        const double *d = DirField ? DirField + 3 * e : UniDir;
        double jp[3] = {d[0] * Scale, d[1] * Scale, d[2] * Scale};
        double jr[3];
        apply(&inv, jp, jr);
        double f[6] = {0, 0, 0, 0, 0, 0};
        for (int q = 0; q < nq; q++) {
            double w = Qw[q] * adet;
            for (int i = 0; i < 6; i++) {
                double r[3];
                ref_vec(ValRef, i, q, r);
                f[i] += dot3(jr, r) * w;
            }
        }
        for (int i = 0; i < 6; i++) {
            I[6 * e + i] = (double)(int64_t)Dofs[6 * e + i];
            V[6 * e + i] = f[i] * Signs[6 * e + i];
        }
    }
}

/* Harmonic-balance element kernel, restating src/mex/assemble_hbfem_kernel_mex.cpp:26-258
 * with the coefficient offsets passed (the gateway leaves them unset). For each element:
 * the signed harmonic edge values A_h (re, im), the time samples
 * A(t) = sum_h (Re A_h Re D(t,h) - Im A_h Im D(t,h)), per quadrature point the curls,
 * per time sample B(t), nu(|B(t)|^2), H = nu B, and the harmonic residual
 * R_h += w (C_i . H) P(h,t) (re, im); the Jacobian block is w nu_dc C_r . C_c with nu_dc
 * the time average of nu, repeated per harmonic and scaled by Scalings[h]. */
void oracle_hbfem(const double *P, const double *T, int64_t Ne, const double *Dofs,
                  const double *Signs, const double *Tags, const double *SolR, const double *SolI,
                  int64_t Ndof, int K, const double *DR, const double *DI, const double *PR,
                  const double *PI, int N, const double *Qw, int nq, const double *CurlRef,
                  const double *lin, const double *isNon, const double *maxB, const double *brk,
                  const double *coe, const double *start, const double *cnt, const double *coeStart,
                  int calcJ, const double *Scalings, double *I, double *J, double *V, double *Rrows,
                  double *Rcols, double *Rre, double *Rim) {
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < Ne; e++) {
        double *ar = malloc(sizeof(double) * 6 * K), *ai = malloc(sizeof(double) * 6 * K);
        double *at = malloc(sizeof(double) * 6 * N);
        double *rr = calloc((size_t)6 * K, sizeof(double)), *ri = calloc((size_t)6 * K, sizeof(double));
        double kb[36] = {0};
        double d[6], s[6];
        for (int k = 0; k < 6; k++) {
            d[k] = Dofs[6 * e + k];
            s[k] = Signs[6 * e + k];
            int64_t g = (int64_t)d[k] - 1;
            for (int h = 0; h < K; h++) {
                ar[k + 6 * h] = SolR[g + h * Ndof] * s[k];
                ai[k + 6 * h] = SolI ? SolI[g + h * Ndof] * s[k] : 0.0;
            }
        }
        for (int t = 0; t < N; t++)
            for (int k = 0; k < 6; k++) {
                double acc = 0.0;
                for (int h = 0; h < K; h++) {
                    double term = ar[k + 6 * h] * DR[t + h * N];
                    if (SolI && DI) term -= ai[k + 6 * h] * DI[t + h * N];
                    acc += term;
                }
                at[k + 6 * t] = acc;
            }
        double v[4][3];
        gather_vertices(P, T, e, v);
        mat3 Jm;
        double det = edge_matrix(v, &Jm);
        double rdet = 1.0 / det, adet = fabs(det);
        int tag = (int)Tags[e];
        for (int q = 0; q < nq; q++) {
            double w = Qw[q] * adet;
            double C[6][3];
            for (int i = 0; i < 6; i++) {
                double c[3];
                ref_vec(CurlRef, i, q, c);
                double y[3];
                apply(&Jm, c, y);
                for (int r = 0; r < 3; r++) C[i][r] = y[r] * rdet;
            }
            double sum_nu = 0.0;
            for (int t = 0; t < N; t++) {
                double B[3] = {0.0, 0.0, 0.0};
                for (int i = 0; i < 6; i++)
                    for (int r = 0; r < 3; r++) B[r] += C[i][r] * at[i + 6 * t];
                double bsq = B[0] * B[0] + B[1] * B[1] + B[2] * B[2];
                double nu, dnu;
                material_eval(bsq, tag, lin, isNon, maxB, brk, coe, start, cnt, coeStart, &nu, &dnu);
                sum_nu += nu;
                double H[3] = {nu * B[0], nu * B[1], nu * B[2]};
                for (int h = 0; h < K; h++) {
                    double pr = PR[h + t * K];
                    for (int i = 0; i < 6; i++) {
                        double dot = C[i][0] * H[0] + C[i][1] * H[1] + C[i][2] * H[2];
                        rr[i + 6 * h] += w * dot * pr;
                        if (PI) ri[i + 6 * h] += w * dot * PI[h + t * K];
                    }
                }
            }
            if (calcJ) {
                double nu_dc = sum_nu / N;
                for (int c = 0; c < 6; c++)
                    for (int r = 0; r < 6; r++) {
                        double dot = C[r][0] * C[c][0] + C[r][1] * C[c][1] + C[r][2] * C[c][2];
                        kb[r + 6 * c] += w * nu_dc * dot;
                    }
            }
        }
        int64_t oR = e * 6 * K;
        for (int h = 0, n = 0; h < K; h++)
            for (int k = 0; k < 6; k++, n++) {
                Rrows[oR + n] = d[k];
                Rcols[oR + n] = (double)(h + 1);
                Rre[oR + n] = rr[k + 6 * h] * s[k];
                Rim[oR + n] = ri[k + 6 * h] * s[k];
            }
        if (calcJ) {
            int64_t oK = e * 36 * K;
            for (int h = 0, n = 0; h < K; h++)
                for (int c = 0; c < 6; c++)
                    for (int r = 0; r < 6; r++, n++) {
                        I[oK + n] = d[r] + (double)h * (double)Ndof;
                        J[oK + n] = d[c] + (double)h * (double)Ndof;
                        V[oK + n] = kb[r + 6 * c] * Scalings[h] * s[r] * s[c];
                    }
        }
        free(ar);
        free(ai);
        free(at);
        free(rr);
        free(ri);
    }
}
