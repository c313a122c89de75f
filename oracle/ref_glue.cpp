/*
 * Oracle glue around the reference's own MEX element kernels (test infrastructure).
 *
 * oracle/Makefile compiles these reference sources UNCHANGED, each with its
 * mexFunction renamed by a -D flag so that several can live in one library:
 *   src/mex/assemble_jacobian_kernel_mex.cpp   -> ref_jacobian_mexFunction
 *   src/mex/assemble_curl_curl_kernel_mex.cpp  -> ref_curl_curl_mexFunction
 *   src/mex/assemble_mass_kernel_mex.cpp       -> ref_mass_mexFunction
 *   src/mex/assemble_source_kernel_mex.cpp     -> ref_source_mexFunction
 *   src/mex/assemble_hbfem_kernel_mex.cpp      -> ref_hbfem_mexFunction
 *   src/mex/assemble_winding_kernel_mex.cpp    -> ref_winding_mexFunction
 * This file implements the mex.h stand-in (oracle/mex_shim/mex.h) and exposes
 * plain C entry points that build the mxArray argument lists exactly as
 * Assembler.m does (Assembler.m:33,48,67,87,157-160,199-202) and hand the MEX outputs
 * back in caller-owned buffers. Nothing here is shipped or measured as product.
 */
#include "mex.h"

#include <csetjmp>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>

extern "C" {

/* ---- mex.h stand-in ---------------------------------------------------- */

static double *g_targets[8];
static size_t g_target_n[8];
static int g_ntargets = 0;
static int g_next = 0;
static jmp_buf g_err_jmp;
static char g_err_msg[512];

double *mxGetPr(const mxArray *a) { return a ? a->pr : nullptr; }
size_t mxGetM(const mxArray *a) { return a ? a->m : 0; }
size_t mxGetN(const mxArray *a) { return a ? a->n : 0; }
size_t mxGetNumberOfElements(const mxArray *a) { return a ? a->m * a->n : 0; }
double mxGetScalar(const mxArray *a) { return (a && a->pr && a->m * a->n) ? a->pr[0] : 0.0; }
int mxIsEmpty(const mxArray *a) { return !a || a->m * a->n == 0; }

mxArray *mxCreateDoubleMatrix(size_t m, size_t n, mxComplexity) {
    mxArray *a = (mxArray *)std::calloc(1, sizeof(mxArray));
    a->m = m;
    a->n = n;
    size_t cnt = m * n;
    if (g_next < g_ntargets && g_target_n[g_next] == cnt) {
        /* Hand out the caller's buffer; zero it like MATLAB's allocator does. */
        a->pr = g_targets[g_next];
        if (cnt) std::memset(a->pr, 0, cnt * sizeof(double));
        a->owns = 0;
    } else {
        a->pr = cnt ? (double *)std::calloc(cnt, sizeof(double)) : nullptr;
        a->owns = 1;
    }
    g_next++;
    return a;
}

void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...) {
    char body[400];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(body, sizeof body, fmt, ap);
    va_end(ap);
    std::snprintf(g_err_msg, sizeof g_err_msg, "%s: %s", id, body);
    std::longjmp(g_err_jmp, 1);
}

/* ---- renamed reference gateways --------------------------------------- */

void ref_jacobian_mexFunction(int, mxArray *[], int, const mxArray *[]);
void ref_curl_curl_mexFunction(int, mxArray *[], int, const mxArray *[]);
void ref_mass_mexFunction(int, mxArray *[], int, const mxArray *[]);
void ref_source_mexFunction(int, mxArray *[], int, const mxArray *[]);
void ref_hbfem_mexFunction(int, mxArray *[], int, const mxArray *[]);
void ref_winding_mexFunction(int, mxArray *[], int, const mxArray *[]);

const char *ref_last_error(void) { return g_err_msg; }

static mxArray wrap(const double *p, size_t m, size_t n) {
    mxArray a;
    a.pr = const_cast<double *>(p);
    a.m = m;
    a.n = n;
    a.owns = 0;
    return a;
}

static double now_s() {
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

typedef void (*mexfn)(int, mxArray *[], int, const mxArray *[]);

/* Calls one gateway; outputs land in `outs` (sizes `outn`), the call's wall
 * time (allocation + element loop, the cost MATLAB pays) in *seconds. */
static int run(mexfn fn, int nlhs, int nrhs, const mxArray *prhs, double **outs,
               const size_t *outn, double *seconds) {
    const mxArray *argp[32];
    mxArray *plhs[8] = {nullptr};
    for (int i = 0; i < nrhs; i++) argp[i] = &prhs[i];
    for (int i = 0; i < nlhs; i++) {
        g_targets[i] = outs[i];
        g_target_n[i] = outn[i];
    }
    g_ntargets = nlhs;
    g_next = 0;
    g_err_msg[0] = 0;
    int rc = 0;
    double t0 = now_s();
    if (setjmp(g_err_jmp) == 0) {
        fn(nlhs, plhs, nrhs, argp);
    } else {
        rc = -1;
    }
    double t1 = now_s();
    if (seconds) *seconds = t1 - t0;
    for (int i = 0; i < nlhs; i++) {
        if (!plhs[i]) continue;
        if (rc == 0 && plhs[i]->owns && outs[i] && plhs[i]->pr)
            std::memcpy(outs[i], plhs[i]->pr, outn[i] * sizeof(double));
        if (plhs[i]->owns) std::free(plhs[i]->pr);
        std::free(plhs[i]);
    }
    g_ntargets = 0;
    return rc;
}

/* [I,J,V,R_idx,R_val] = assemble_jacobian_kernel_mex(17 args), Assembler.m:199-202. */
int ref_jacobian(const double *P, size_t Nn, const double *T, size_t Ne, const double *Dofs,
                 const double *Signs, const double *Tags, const double *SolA, size_t Ndof,
                 const double *Qw, size_t nq, const double *CurlRef, const double *lin,
                 const double *isNon, const double *maxB, size_t nmat, const double *brk,
                 size_t nbrk, const double *coe, size_t ncoe, const double *start,
                 const double *cnt, const double *coeStart, int calcJ, double *I, double *J,
                 double *V, double *Ridx, double *Rval, double *seconds) {
    double cj = calcJ ? 1.0 : 0.0;
    mxArray in[17] = {
        wrap(P, 3, Nn),        wrap(T, 4, Ne),     wrap(Dofs, 6, Ne),  wrap(Signs, 6, Ne),
        wrap(Tags, 1, Ne),     wrap(SolA, Ndof, 1), wrap(Qw, 1, nq),    wrap(CurlRef, 18, nq),
        wrap(lin, nmat, 1),    wrap(isNon, nmat, 1), wrap(maxB, nmat, 1), wrap(brk, nbrk, 1),
        wrap(coe, ncoe, 1),    wrap(start, nmat, 1), wrap(cnt, nmat, 1), wrap(coeStart, nmat, 1),
        wrap(&cj, 1, 1)};
    size_t nK = calcJ ? Ne * 36 : 0;
    double *outs[5] = {I, J, V, Ridx, Rval};
    size_t outn[5] = {nK, nK, nK, Ne * 6, Ne * 6};
    return run(ref_jacobian_mexFunction, 5, 17, in, outs, outn, seconds);
}

/* [I,J,V] = assemble_curl_curl_kernel_mex(P,T,Dofs,Signs,Nu,Qw,CurlRef), Assembler.m:33. */
int ref_curl_curl(const double *P, size_t Nn, const double *T, size_t Ne, const double *Dofs,
                  const double *Signs, const double *Nu, const double *Qw, size_t nq,
                  const double *CurlRef, double *I, double *J, double *V, double *seconds) {
    mxArray in[7] = {wrap(P, 3, Nn),    wrap(T, 4, Ne), wrap(Dofs, 6, Ne),     wrap(Signs, 6, Ne),
                     wrap(Nu, Ne, 1),   wrap(Qw, 1, nq), wrap(CurlRef, 18, nq)};
    double *outs[3] = {I, J, V};
    size_t outn[3] = {Ne * 36, Ne * 36, Ne * 36};
    return run(ref_curl_curl_mexFunction, 3, 7, in, outs, outn, seconds);
}

/* [I,J,V] = assemble_mass_kernel_mex(P,T,Dofs,Signs,Coeffs,Qw,ValRef), Assembler.m:48,67.
 * ncoeff == 0 passes an empty Coeffs (sigma = 1 everywhere, mass_kernel_mex.cpp:155,187). */
int ref_mass(const double *P, size_t Nn, const double *T, size_t Ne, const double *Dofs,
             const double *Signs, const double *Coeffs, size_t ncoeff, const double *Qw, size_t nq,
             const double *ValRef, double *I, double *J, double *V, double *seconds) {
    mxArray in[7] = {wrap(P, 3, Nn),          wrap(T, 4, Ne),  wrap(Dofs, 6, Ne),   wrap(Signs, 6, Ne),
                     wrap(Coeffs, ncoeff, ncoeff ? 1 : 0), wrap(Qw, 1, nq), wrap(ValRef, 18, nq)};
    double *outs[3] = {I, J, V};
    size_t outn[3] = {Ne * 36, Ne * 36, Ne * 36};
    return run(ref_mass_mexFunction, 3, 7, in, outs, outn, seconds);
}

/* [I,V] = assemble_source_kernel_mex(P,T,Dofs,Signs,Js,Qw,ValRef), Assembler.m:87. */
int ref_source(const double *P, size_t Nn, const double *T, size_t Ne, const double *Dofs,
               const double *Signs, const double *Js, const double *Qw, size_t nq,
               const double *ValRef, double *I, double *V, double *seconds) {
    mxArray in[7] = {wrap(P, 3, Nn), wrap(T, 4, Ne), wrap(Dofs, 6, Ne), wrap(Signs, 6, Ne),
                     wrap(Js, 3, Ne), wrap(Qw, 1, nq), wrap(ValRef, 18, nq)};
    double *outs[2] = {I, V};
    size_t outn[2] = {Ne * 6, Ne * 6};
    return run(ref_source_mexFunction, 2, 7, in, outs, outn, seconds);
}

/* [I,V] = assemble_winding_kernel_mex(P,T,Dofs,Signs,Tags,CoilID,DirField,UniDir,Scale,Qw,ValRef),
 * Assembler.m:157-166. DirField NULL is passed as the empty []. */
int ref_winding(const double *P, size_t Nn, const double *T, size_t Ne, const double *Dofs,
                const double *Signs, const double *Tags, double CoilID, const double *DirField,
                const double *UniDir, double Scale, const double *Qw, size_t nq, const double *ValRef,
                double *I, double *V, double *seconds) {
    mxArray in[11] = {wrap(P, 3, Nn),       wrap(T, 4, Ne),          wrap(Dofs, 6, Ne),
                      wrap(Signs, 6, Ne),   wrap(Tags, 1, Ne),       wrap(&CoilID, 1, 1),
                      DirField ? wrap(DirField, 3, Ne) : wrap(nullptr, 0, 0),
                      wrap(UniDir, 3, 1),   wrap(&Scale, 1, 1),      wrap(Qw, 1, nq),
                      wrap(ValRef, 18, nq)};
    double *outs[2] = {I, V};
    size_t outn[2] = {Ne * 6, Ne * 6};
    return run(ref_winding_mexFunction, 2, 11, in, outs, outn, seconds);
}

/* [I,J,V,R_rows,R_cols,R_re,R_im] = assemble_hbfem_kernel_mex(22 args)
 * (assemble_hbfem_kernel_mex.cpp:26-57). SolR/SolI [Ndof x K], DR/DI [N x K],
 * PR/PI [K x N] column-major; a NULL imaginary part is passed as an empty array.
 * The gateway reads seven material arrays and leaves the coefficient offsets
 * unset, so only linear materials give defined results. */
int ref_hbfem(const double *P, size_t Nn, const double *T, size_t Ne, const double *Dofs,
              const double *Signs, const double *Tags, const double *SolR, const double *SolI, size_t Ndof,
              size_t K, const double *DR, const double *DI, const double *PR, const double *PI, size_t N,
              const double *Qw, size_t nq, const double *CurlRef, const double *lin, const double *isNon,
              const double *maxB, size_t nmat, const double *brk, size_t nbrk, const double *coe, size_t ncoe,
              const double *start, const double *cnt, int calcJ, const double *Scalings, double *I, double *J,
              double *V, double *Rrows, double *Rcols, double *Rre, double *Rim, double *seconds) {
    double cj = calcJ ? 1.0 : 0.0;
    mxArray in[22] = {
        wrap(P, 3, Nn),          wrap(T, 4, Ne),          wrap(Dofs, 6, Ne),      wrap(Signs, 6, Ne),
        wrap(Tags, 1, Ne),       wrap(SolR, Ndof, K),     wrap(SolI, SolI ? Ndof : 0, SolI ? K : 0),
        wrap(DR, N, K),          wrap(DI, DI ? N : 0, DI ? K : 0),
        wrap(PR, K, N),          wrap(PI, PI ? K : 0, PI ? N : 0),
        wrap(Qw, 1, nq),         wrap(CurlRef, 18, nq),
        wrap(lin, nmat, 1),      wrap(isNon, nmat, 1),    wrap(maxB, nmat, 1),    wrap(brk, nbrk, 1),
        wrap(coe, ncoe, 1),      wrap(start, nmat, 1),    wrap(cnt, nmat, 1),     wrap(&cj, 1, 1),
        wrap(Scalings, K, 1)};
    size_t nK = calcJ ? Ne * 36 * K : 0, nR = Ne * 6 * K;
    double *outs[7] = {I, J, V, Rrows, Rcols, Rre, Rim};
    size_t outn[7] = {nK, nK, nK, nR, nR, nR, nR};
    return run(ref_hbfem_mexFunction, 7, 22, in, outs, outn, seconds);
}

}  // extern "C"
