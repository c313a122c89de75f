// Sparse linear algebra around the assembled CSR: y = A x, the reference's
// Dirichlet elimination, and a preconditioned conjugate-gradient solve that
// stands in for the reference's MUMPS call (LinearSolver.m:22-46) in the
// transient Newton driver.
//
// Every reduction runs over a fixed grid in a fixed order, so a solve is
// bitwise reproducible. The CG iterations run as a captured CUDA graph of
// kPcgChunk iterations; each kernel returns at once when the device-side state
// says the solve has finished, and the host reads that state once per chunk.
#include <cstdint>
#include <cstring>
#include <new>

#include "common.cuh"
#include "sparse.cuh"

namespace mag {

namespace {

constexpr int kThreads = 256;
constexpr int kLanes = 8;  // lanes per CSR row in y = A x
constexpr int kPcgChunk = 32;

struct Csr {
    const int64_t *rp;
    const int32_t *ci;
    const double *v;
    int64_t n;
};

// Row i of A x with kLanes lanes; the value is valid in the group's lane 0.
__device__ __forceinline__ double row_dot(const Csr &A, int64_t i, int lane, const double *__restrict__ x) {
    double s = 0.0;
    if (i < A.n) {
        const int64_t a = A.rp[i], b = A.rp[i + 1];
        for (int64_t k = a + lane; k < b; k += kLanes) s = s + A.v[k] * __ldg(x + A.ci[k]);
    }
#pragma unroll
    for (int o = kLanes / 2; o > 0; o >>= 1) s = s + __shfl_down_sync(0xffffffffu, s, o, kLanes);
    return s;
}

// Fixed-order block sum of one value per thread; result valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double *sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = v + __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) t = t + sh[i];
    return t;
}

// Row loops over groups of kLanes threads run a block-uniform number of passes,
// so every lane reaches the shuffles in row_dot.
#define MAG_ROW_LOOP(n)                                                                                      \
    for (int64_t i = blockIdx.x * (int64_t)(kThreads / kLanes) + threadIdx.x / kLanes;                       \
         i - (threadIdx.x / kLanes) < (n); i += (int64_t)gridDim.x * (kThreads / kLanes))

__global__ void __launch_bounds__(kThreads) k_spmv(Csr A, const double *__restrict__ x, double *__restrict__ y) {
    const int lane = threadIdx.x % kLanes;
    MAG_ROW_LOOP(A.n) {
        double s = row_dot(A, i, lane, x);
        if (lane == 0 && i < A.n) y[i] = s;
    }
}

// M_free A M_free + M_fixed in place (BoundaryCondition.m:81-112), rhs[fixed] = 0.
__global__ void k_dirichlet(int64_t n, const int64_t *__restrict__ rp, const int32_t *__restrict__ ci,
                            double *__restrict__ v, const uint8_t *__restrict__ fixed, double *__restrict__ rhs) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool fi = fixed[i] != 0;
    for (int64_t k = rp[i]; k < rp[i + 1]; k++) {
        const int64_t j = ci[k];
        if (fi) v[k] = j == i ? 1.0 : 0.0;
        else if (fixed[j]) v[k] = 0.0;
    }
    if (rhs && fi) rhs[i] = 0.0;
}

// ---- preconditioned CG --------------------------------------------------------------

struct PcgState {
    double rz, alpha, beta, rr, bb, tol2;
    int done;  // 0 running, 1 converged, 2 iteration limit, 3 breakdown (p.Ap <= 0 or not finite)
    int iters, max_iter;
};

struct PcgBufs {
    double *x, *r, *p, *q, *z, *dinv, *part;
    PcgState *st;
    int nb;
};

// Auxiliary gradient space of the preconditioner: z = D^-1 r + G (D_N^-1 (G^T r)),
// G the (free edge x interior node) incidence of the discrete gradient and D_N the
// diagonal of G^T A G. The curl-curl part of A vanishes on gradients, so without this
// term the gradient modes are held only by the small regularisation and Jacobi-CG
// needs tens of thousands of iterations (a Hiptmair-type additive correction).
struct Aux {
    int64_t ni;
    const int64_t *g_rp;   // G   [n x ni]
    const int32_t *g_ci;
    const double *g_v;
    const int64_t *gt_rp;  // G^T [ni x n]
    const int32_t *gt_ci;
    const double *gt_v;
    const double *dn_inv;  // [ni]
    double *w;             // [ni] scratch
};

__global__ void __launch_bounds__(kThreads) k_aux_gt(Aux a, const double *__restrict__ r, const PcgState *st) {
    if (st && st->done) return;
    for (int64_t j = blockIdx.x * (int64_t)kThreads + threadIdx.x; j < a.ni; j += (int64_t)gridDim.x * kThreads) {
        double s = 0.0;
        for (int64_t k = a.gt_rp[j]; k < a.gt_rp[j + 1]; k++) s = s + a.gt_v[k] * r[a.gt_ci[k]];
        a.w[j] = a.dn_inv[j] * s;
    }
}

// z = D^-1 r (+ G w with the auxiliary space). First call (init): p = z and partials
// (r.z, r.r, b.b) with stride 3; later calls: (r.z, r.r) with stride 2.
template <bool AUX>
__global__ void __launch_bounds__(kThreads) k_pcg_precond(int64_t n, PcgBufs B, Aux a, const double *__restrict__ b,
                                                          int init) {
    if (!init && B.st->done) return;
    __shared__ double sh[kThreads / 32];
    double rz = 0.0, rr = 0.0, bb = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads) {
        double r = B.r[i];
        double z = B.dinv[i] * r;
        if (AUX)
            for (int64_t k = a.g_rp[i]; k < a.g_rp[i + 1]; k++) z = z + a.g_v[k] * a.w[a.g_ci[k]];
        B.z[i] = z;
        if (init) {
            B.p[i] = z;
            bb = bb + b[i] * b[i];
        }
        rz = rz + r * z;
        rr = rr + r * r;
    }
    double t0 = block_sum(rz, sh), t1 = block_sum(rr, sh), t2 = block_sum(bb, sh);
    if (threadIdx.x == 0) {
        const int st = init ? 3 : 2;
        B.part[st * blockIdx.x] = t0;
        B.part[st * blockIdx.x + 1] = t1;
        if (init) B.part[st * blockIdx.x + 2] = t2;
    }
}

// x = x0, r = b - A x0, dinv = 1/diag(A) (1 where the diagonal is missing or not positive)
__global__ void __launch_bounds__(kThreads) k_pcg_setup(Csr A, const double *__restrict__ b,
                                                        const double *__restrict__ x0, PcgBufs B) {
    const int lane = threadIdx.x % kLanes;
    MAG_ROW_LOOP(A.n) {
        double s = row_dot(A, i, lane, x0);
        if (lane == 0 && i < A.n) {
            double d = 0.0;
            for (int64_t k = A.rp[i]; k < A.rp[i + 1]; k++)
                if (A.ci[k] == i) d = A.v[k];
            B.dinv[i] = d > 0.0 ? 1.0 / d : 1.0;
            B.r[i] = b[i] - s;
            B.x[i] = x0[i];
        }
    }
}

__global__ void __launch_bounds__(kThreads) k_pcg_init_reduce(PcgBufs B, double rtol, int max_iter) {
    __shared__ double sh[kThreads / 32];
    double a = 0.0, c = 0.0, d = 0.0;
    for (int i = threadIdx.x; i < B.nb; i += kThreads) {
        a = a + B.part[3 * i];
        c = c + B.part[3 * i + 1];
        d = d + B.part[3 * i + 2];
    }
    double rz = block_sum(a, sh), rr = block_sum(c, sh), bb = block_sum(d, sh);
    if (threadIdx.x == 0) {
        PcgState s{};
        s.rz = rz;
        s.rr = rr;
        s.bb = bb;
        s.tol2 = rtol * rtol * bb;
        s.max_iter = max_iter;
        s.iters = 0;
        s.done = rr <= s.tol2 ? 1 : 0;
        *B.st = s;
    }
}

// q = A p and the partials of p.q
__global__ void __launch_bounds__(kThreads) k_pcg_spmv_dot(Csr A, PcgBufs B) {
    if (B.st->done) return;
    __shared__ double sh[kThreads / 32];
    const int lane = threadIdx.x % kLanes;
    double acc = 0.0;
    MAG_ROW_LOOP(A.n) {
        double s = row_dot(A, i, lane, B.p);
        if (lane == 0 && i < A.n) {
            B.q[i] = s;
            acc = acc + B.p[i] * s;
        }
    }
    double t = block_sum(acc, sh);
    if (threadIdx.x == 0) B.part[blockIdx.x] = t;
}

__global__ void __launch_bounds__(kThreads) k_pcg_alpha(PcgBufs B) {
    if (B.st->done) return;
    __shared__ double sh[kThreads / 32];
    double a = 0.0;
    for (int i = threadIdx.x; i < B.nb; i += kThreads) a = a + B.part[i];
    double pq = block_sum(a, sh);
    if (threadIdx.x == 0) {
        PcgState &s = *B.st;
        if (!(pq > 0.0) || !isfinite(pq)) s.done = 3;
        else s.alpha = s.rz / pq;
    }
}

// x += alpha p, r -= alpha q
__global__ void __launch_bounds__(kThreads) k_pcg_xr(int64_t n, PcgBufs B) {
    if (B.st->done) return;
    const double al = B.st->alpha;
    for (int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads) {
        B.x[i] = B.x[i] + al * B.p[i];
        B.r[i] = B.r[i] - al * B.q[i];
    }
}

__global__ void __launch_bounds__(kThreads) k_pcg_beta(PcgBufs B) {
    if (B.st->done) return;
    __shared__ double sh[kThreads / 32];
    double a = 0.0, c = 0.0;
    for (int i = threadIdx.x; i < B.nb; i += kThreads) {
        a = a + B.part[2 * i];
        c = c + B.part[2 * i + 1];
    }
    double rz = block_sum(a, sh), rr = block_sum(c, sh);
    if (threadIdx.x == 0) {
        PcgState &s = *B.st;
        s.iters++;
        s.rr = rr;
        s.beta = rz / s.rz;
        s.rz = rz;
        if (rr <= s.tol2) s.done = 1;
        else if (!isfinite(rr)) s.done = 3;
        else if (s.iters >= s.max_iter) s.done = 2;
    }
}

__global__ void __launch_bounds__(kThreads) k_pcg_dir(int64_t n, PcgBufs B) {
    if (B.st->done) return;
    const double be = B.st->beta;
    for (int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads)
        B.p[i] = B.z[i] + be * B.p[i];
}

int grid_for(int64_t threads) {
    static int nsm = 0;
    if (!nsm) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        if (nsm <= 0) nsm = 1;
    }
    int64_t want = (threads + kThreads - 1) / kThreads;
    int64_t cap = 4LL * nsm;
    return (int)(want < 1 ? 1 : (want < cap ? want : cap));
}

}  // namespace

struct PcgSolver {
    int64_t n = 0;
    PcgBufs B{};
    Aux aux{};
    double *w = nullptr;
    int64_t w_cap = 0;
    cudaStream_t s = nullptr;
    cudaGraphExec_t exec = nullptr;
    Csr key{};
    PcgState *h_st = nullptr;  // pinned
};

int csr_spmv(int64_t n, const int64_t *rp, const int32_t *ci, const double *v, const double *x, double *y,
             cudaStream_t s) {
    Csr A{rp, ci, v, n};
    k_spmv<<<grid_for(n * kLanes), kThreads, 0, s>>>(A, x, y);
    return cudaPeekAtLastError() == cudaSuccess ? MAG_OK : MAG_E_CUDA;
}

int csr_dirichlet(int64_t n, const int64_t *rp, const int32_t *ci, double *v, const uint8_t *fixed, double *rhs,
                  cudaStream_t s) {
    k_dirichlet<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, rp, ci, v, fixed, rhs);
    return cudaPeekAtLastError() == cudaSuccess ? MAG_OK : MAG_E_CUDA;
}

int pcg_create(int64_t n, PcgSolver **out) {
    *out = nullptr;
    PcgSolver *P = new (std::nothrow) PcgSolver();
    if (!P) return MAG_E_NOMEM;
    P->n = n;
    const int gs = grid_for(n * kLanes), gv = grid_for(n);
    P->B.nb = gs > gv ? gs : gv;
    size_t vb = (size_t)n * sizeof(double);
    double **bufs[] = {&P->B.x, &P->B.r, &P->B.p, &P->B.q, &P->B.z, &P->B.dinv};
    bool ok = true;
    for (double **b : bufs) ok = ok && cudaMalloc(b, vb) == cudaSuccess;
    ok = ok && cudaMalloc(&P->B.part, (size_t)3 * P->B.nb * sizeof(double)) == cudaSuccess;
    ok = ok && cudaMalloc(&P->B.st, sizeof(PcgState)) == cudaSuccess;
    ok = ok && cudaMallocHost(&P->h_st, sizeof(PcgState)) == cudaSuccess;
    ok = ok && cudaStreamCreateWithFlags(&P->s, cudaStreamNonBlocking) == cudaSuccess;
    if (!ok) {
        pcg_destroy(P);
        return MAG_E_NOMEM;
    }
    *out = P;
    return MAG_OK;
}

void pcg_destroy(PcgSolver *P) {
    if (!P) return;
    if (P->s) cudaStreamSynchronize(P->s);
    if (P->exec) cudaGraphExecDestroy(P->exec);
    double *bufs[] = {P->B.x, P->B.r, P->B.p, P->B.q, P->B.z, P->B.dinv, P->B.part, P->w};
    for (double *b : bufs)
        if (b) cudaFree(b);
    if (P->B.st) cudaFree(P->B.st);
    if (P->h_st) cudaFreeHost(P->h_st);
    if (P->s) cudaStreamDestroy(P->s);
    delete P;
}

int pcg_set_aux(PcgSolver *P, int64_t ni, const int64_t *g_rp, const int32_t *g_ci, const double *g_v,
                const int64_t *gt_rp, const int32_t *gt_ci, const double *gt_v, const double *dn_inv) {
    if (P->exec) {  // the captured iterations change shape
        cudaGraphExecDestroy(P->exec);
        P->exec = nullptr;
    }
    if (ni <= 0) {
        P->aux = Aux{};
        return MAG_OK;
    }
    if (ni > P->w_cap) {
        if (P->w) cudaFree(P->w);
        P->w = nullptr;
        P->w_cap = 0;
        if (cudaMalloc(&P->w, (size_t)ni * sizeof(double)) != cudaSuccess) {
            P->aux = Aux{};
            return MAG_E_NOMEM;
        }
        P->w_cap = ni;
    }
    P->aux = Aux{ni, g_rp, g_ci, g_v, gt_rp, gt_ci, gt_v, dn_inv, P->w};
    return MAG_OK;
}

namespace {

PcgBufs bufs_with(const PcgSolver *P, int nb) {
    PcgBufs b = P->B;
    b.nb = nb;
    return b;
}

void enqueue_iterations(PcgSolver *P, const Csr &A, cudaStream_t s) {
    const int gs = grid_for(P->n * kLanes), gv = grid_for(P->n);
    const PcgBufs Bs = bufs_with(P, gs), Bv = bufs_with(P, gv);
    for (int it = 0; it < kPcgChunk; it++) {
        k_pcg_spmv_dot<<<gs, kThreads, 0, s>>>(A, Bs);
        k_pcg_alpha<<<1, kThreads, 0, s>>>(Bs);
        k_pcg_xr<<<gv, kThreads, 0, s>>>(P->n, Bv);
        if (P->aux.ni > 0) {
            k_aux_gt<<<grid_for(P->aux.ni), kThreads, 0, s>>>(P->aux, P->B.r, P->B.st);
            k_pcg_precond<true><<<gv, kThreads, 0, s>>>(P->n, Bv, P->aux, nullptr, 0);
        } else {
            k_pcg_precond<false><<<gv, kThreads, 0, s>>>(P->n, Bv, P->aux, nullptr, 0);
        }
        k_pcg_beta<<<1, kThreads, 0, s>>>(Bv);
        k_pcg_dir<<<gv, kThreads, 0, s>>>(P->n, Bv);
    }
}

}  // namespace

int pcg_solve(PcgSolver *P, const int64_t *rp, const int32_t *ci, const double *v, const double *b, double *x,
              double rtol, int max_iter, int *iters, double *relres, int *status, cudaStream_t caller) {
    Csr A{rp, ci, v, P->n};
    cudaStream_t s = P->s;
    cudaEvent_t ev;
    MAG_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    cudaEventRecord(ev, caller);
    cudaStreamWaitEvent(s, ev, 0);
    const int gs = grid_for(P->n * kLanes), gv = grid_for(P->n);
    const PcgBufs Bv = bufs_with(P, gv);
    k_pcg_setup<<<gs, kThreads, 0, s>>>(A, b, x, P->B);
    if (P->aux.ni > 0) {
        k_aux_gt<<<grid_for(P->aux.ni), kThreads, 0, s>>>(P->aux, P->B.r, nullptr);
        k_pcg_precond<true><<<gv, kThreads, 0, s>>>(P->n, Bv, P->aux, b, 1);
    } else {
        k_pcg_precond<false><<<gv, kThreads, 0, s>>>(P->n, Bv, P->aux, b, 1);
    }
    k_pcg_init_reduce<<<1, kThreads, 0, s>>>(Bv, rtol, max_iter);
    cudaError_t le = cudaPeekAtLastError();
    if (le != cudaSuccess) {
        cudaEventDestroy(ev);
        set_error("pcg setup launch: %s", cudaGetErrorString(le));
        return MAG_E_CUDA;
    }
    if (!P->exec || memcmp(&P->key, &A, sizeof(Csr)) != 0) {
        if (P->exec) {
            cudaGraphExecDestroy(P->exec);
            P->exec = nullptr;
        }
        cudaGraph_t g;
        MAG_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        enqueue_iterations(P, A, s);
        MAG_CUDA_TRY(cudaStreamEndCapture(s, &g));
        cudaError_t e = cudaGraphInstantiate(&P->exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            cudaEventDestroy(ev);
            set_error("pcg graph: %s", cudaGetErrorString(e));
            return MAG_E_CUDA;
        }
        P->key = A;
    }
    for (;;) {
        MAG_CUDA_TRY(cudaMemcpyAsync(P->h_st, P->B.st, sizeof(PcgState), cudaMemcpyDeviceToHost, s));
        MAG_CUDA_TRY(cudaStreamSynchronize(s));
        if (P->h_st->done) break;
        MAG_CUDA_TRY(cudaGraphLaunch(P->exec, s));
    }
    MAG_CUDA_TRY(cudaMemcpyAsync(x, P->B.x, (size_t)P->n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    cudaEventRecord(ev, s);
    cudaStreamWaitEvent(caller, ev, 0);
    cudaEventDestroy(ev);
    const PcgState &h = *P->h_st;
    if (iters) *iters = h.iters;
    if (relres) *relres = h.bb > 0 ? sqrt(h.rr / h.bb) : sqrt(h.rr);
    if (status) *status = h.done;
    if (h.done == 3) {
        set_error("pcg breakdown after %d iterations (matrix not positive definite on the Krylov space)", h.iters);
        return MAG_E_GEOMETRY;
    }
    return MAG_OK;
}

}  // namespace mag
