/*
 * A minimal MATLAB stand-in that runs one MEX gateway (linked into the same
 * shared object) from Python: dense and sparse double arrays with MATLAB's
 * storage (column-major; sparse as jc/ir/pr compressed columns), mxMalloc
 * memory released when the gateway raises, and mexErrMsgIdAndTxt returning to
 * the caller through longjmp like MATLAB's non-local exit. Test infrastructure.
 */
#include <csetjmp>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <set>

#include "mex.h"

struct mxArray_tag {
    double *pr = nullptr;
    mwIndex *jc = nullptr;
    mwIndex *ir = nullptr;
    size_t m = 0, n = 0, nzmax = 0;
    int sparse = 0;
    int owns = 0;
};

namespace {
std::jmp_buf g_jmp;
char g_msg[512];
std::set<void *> g_allocs;
}  // namespace

extern "C" {

double *mxGetPr(const mxArray *a) { return a ? a->pr : nullptr; }
size_t mxGetM(const mxArray *a) { return a ? a->m : 0; }
size_t mxGetN(const mxArray *a) { return a ? a->n : 0; }
size_t mxGetNumberOfElements(const mxArray *a) { return a ? a->m * a->n : 0; }
double mxGetScalar(const mxArray *a) {
    if (!a || !a->pr) return 0.0;
    if (a->sparse) return a->jc[1] > 0 && a->ir[0] == 0 ? a->pr[0] : 0.0;
    return a->m * a->n != 0 ? a->pr[0] : 0.0;
}
int mxIsEmpty(const mxArray *a) { return !a || a->m * a->n == 0; }
int mxIsSparse(const mxArray *a) { return a && a->sparse; }
mwIndex *mxGetJc(const mxArray *a) { return a ? a->jc : nullptr; }
mwIndex *mxGetIr(const mxArray *a) { return a ? a->ir : nullptr; }

mxArray *mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity) {
    mxArray *a = new mxArray_tag();
    a->m = m;
    a->n = n;
    a->pr = m * n != 0 ? (double *)std::calloc(m * n, sizeof(double)) : nullptr;
    a->owns = 1;
    return a;
}

mxArray *mxCreateSparse(mwSize m, mwSize n, mwSize nzmax, mxComplexity) {
    mxArray *a = new mxArray_tag();
    a->m = m;
    a->n = n;
    a->nzmax = nzmax ? nzmax : 1;  // MATLAB raises 0 to 1
    a->sparse = 1;
    a->jc = (mwIndex *)std::calloc(n + 1, sizeof(mwIndex));
    a->ir = (mwIndex *)std::calloc(a->nzmax, sizeof(mwIndex));
    a->pr = (double *)std::calloc(a->nzmax, sizeof(double));
    a->owns = 1;
    return a;
}

void mxDestroyArray(mxArray *a) {
    if (!a) return;
    if (a->owns) {
        std::free(a->pr);
        std::free(a->jc);
        std::free(a->ir);
    }
    delete a;
}

void *mxMalloc(size_t n) {
    void *p = std::malloc(n ? n : 1);
    g_allocs.insert(p);
    return p;
}

void mxFree(void *p) {
    g_allocs.erase(p);
    std::free(p);
}

void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...) {
    char body[400];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(body, sizeof body, fmt, ap);
    va_end(ap);
    std::snprintf(g_msg, sizeof g_msg, "%s: %s", id, body);
    std::longjmp(g_jmp, 1);
}

/* ---- driver entry points (ctypes) ------------------------------------------ */

/* A dense m x n argument over caller-owned column-major data. */
mxArray *rt_wrap(double *data, size_t m, size_t n) {
    mxArray *a = new mxArray_tag();
    a->pr = data;
    a->m = m;
    a->n = n;
    return a;
}

/* Call the gateway; 0 on return, 1 if it raised (message in msg). */
int rt_call(int nlhs, mxArray **plhs, int nrhs, mxArray **prhs, char *msg, int msg_len) {
    g_allocs.clear();
    g_msg[0] = 0;
    if (setjmp(g_jmp)) {
        for (void *p : g_allocs) std::free(p);
        g_allocs.clear();
        if (msg && msg_len > 0) std::snprintf(msg, (size_t)msg_len, "%s", g_msg);
        return 1;
    }
    mexFunction(nlhs, plhs, nrhs, (const mxArray **)prhs);
    return 0;
}

/* m, n, sparse flag and stored entries (nnz for sparse, m*n for dense). */
void rt_info(const mxArray *a, size_t *out) {
    out[0] = a->m;
    out[1] = a->n;
    out[2] = (size_t)a->sparse;
    out[3] = a->sparse ? a->jc[a->n] : a->m * a->n;
}

}  // extern "C"
