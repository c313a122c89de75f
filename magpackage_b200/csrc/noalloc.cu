// mag_mex_jacobian_noalloc: the Jacobian/residual element assembly of
// mag_mex_jacobian for callers that must not allocate device memory.
//
// Who needs it: a MEX function handed mxGPUArray buffers, whose device memory
// belongs to MATLAB's allocator; hosts that run inside another runtime's
// memory pool or under a fixed memory budget; code on a path where a
// cudaMalloc would synchronise the device or is not allowed at all. Such a
// caller owns every input and output buffer and wants the library to touch
// nothing else.
//
// The element blocks that mag_mex_jacobian keeps in a cudaMalloc'd slab live
// here in one file-scope device array, g_noalloc_scratch, sized for
// kNoAllocMaxElements elements (12 MiB of blocks plus small tables; every GPU
// that loads this library holds the array until the process exits). Larger
// inputs are rejected with MAG_E_UNSUPPORTED. The array is shared by all
// calls and keeps the last call's contents; each call clears the words that
// must start at zero. Two calls whose kernels overlap on the GPU (different
// streams, or different host threads) race on the array: serialise them.
//
// The first call on each device looks up the array's device address with
// cudaGetSymbolAddress (with that device current) and caches it; make that first
// call before any stream capture begins. Each call copies the host tables from
// pageable memory and synchronises the stream. With CUDA's lazy module loading
// (the default) the array is committed on a device at that first call, not when
// the library is loaded, so a first call made under a tight memory budget can
// fail for lack of device memory (MAG_E_CUDA); make it early. Nothing here calls
// cudaMalloc, cudaFree or any allocating library routine.
// An element that fails the input checks makes the call return MAG_E_RANGE and
// leaves NaN in its triplet values and residual entries.
#include <mutex>

#include "common.cuh"
#include "element.cuh"

namespace mag {

namespace {

constexpr int64_t kNoAllocMaxElements = 32768;
constexpr int kNaMaxMat = 64;
constexpr int kNaMaxBreaks = 4096;
constexpr int kNaMaxCoefs = 16384;
constexpr int kNaMaxDevices = 64;

// Layout of g_noalloc_scratch, in doubles.
constexpr size_t kOffBlocks = 0;
constexpr size_t kOffLin = kOffBlocks + (size_t)kNoAllocMaxElements * kScratchPerElem;
constexpr size_t kOffIsNon = kOffLin + kNaMaxMat;
constexpr size_t kOffMaxB = kOffIsNon + kNaMaxMat;
constexpr size_t kOffBreaks = kOffMaxB + kNaMaxMat;
constexpr size_t kOffCoefs = kOffBreaks + kNaMaxBreaks;
constexpr size_t kOffInts = kOffCoefs + kNaMaxCoefs;       // 3 * kNaMaxMat int32
constexpr size_t kOffCurl = kOffInts + (3 * kNaMaxMat) / 2; // 18 * kMaxQuad doubles
constexpr size_t kOffErr = kOffCurl + 18 * kMaxQuad;        // one int32 error word
constexpr size_t kNoAllocDoubles = kOffErr + 32;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

std::mutex g_mu;
double *g_addr[kNaMaxDevices] = {nullptr};

int scratch_address(double **out) {
    int dev = 0;
    MAG_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNaMaxDevices) {
        set_error("mag_mex_jacobian_noalloc: device ordinal %d out of range", dev);
        return MAG_E_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            set_error("mag_mex_jacobian_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
            return MAG_E_CUDA;
        }
        g_addr[dev] = static_cast<double *>(p);
    }
    *out = g_addr[dev];
    return MAG_OK;
}

struct NaArgs {
    const double *P, *T, *Dofs, *Signs, *Tags, *Sol;
    int64_t nn, ne, ndof;
    int nmat;
};

// Reads the reference's MEX layout directly (1-based ids stored as doubles),
// checks every index before use, and writes the element's block.
template <bool CALCJ, bool STDCURL>
__global__ void __launch_bounds__(128) k_na_elems(NaArgs a, QuadParams qp, MaterialParams mp,
                                                  double *__restrict__ blocks, int *__restrict__ err) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= a.ne) return;
    double *dst = blocks + e * kScratchPerElem;
    // an element that fails a check flags the call and leaves NaN in its block, so the
    // triplets copied from it are visibly invalid rather than the previous call's values
    auto reject = [&]() {
        atomicOr(err, 1);
        const double nan = __longlong_as_double(0x7FF8000000000000LL);
        const double row[6] = {nan, nan, nan, nan, nan, nan};
        for (int i = 0; i < 6; i++) elem::store_row(dst + i * kScratchStride, row, nan);
    };
    int node[4];
    for (int k = 0; k < 4; k++) {
        double v = a.T[4 * e + k];
        if (!(v >= 1.0 && v < (double)a.nn + 1.0)) {
            reject();
            return;
        }
        node[k] = (int)v - 1;
    }
    int d[6];
    unsigned sb = 0;
    for (int k = 0; k < 6; k++) {
        double v = a.Dofs[6 * e + k], s = a.Signs[6 * e + k];
        if (!(v > -1.0 && v < (double)a.ndof + 1.0) || (s != 1.0 && s != -1.0)) {
            reject();
            return;
        }
        d[k] = (int)v - 1;
        sb |= (s < 0 ? 1u : 0u) << k;
    }
    double tv = a.Tags[e];
    if (!(tv >= 1.0 && tv < (double)a.nmat + 1.0)) {
        reject();
        return;
    }
    int tag = (int)tv;
    double4 v[4];
    for (int k = 0; k < 4; k++) {
        const int64_t p = 3 * (int64_t)node[k];
        v[k] = make_double4(a.P[p], a.P[p + 1], a.P[p + 2], 0.0);
        if (!isfinite(v[k].x) || !isfinite(v[k].y) || !isfinite(v[k].z)) {
            reject();
            return;
        }
    }
    elem::Geo g;
    // same arithmetic as elem::geometry, reading the [3 x Nn] layout
    g.J[0][0] = v[1].x - v[0].x; g.J[1][0] = v[1].y - v[0].y; g.J[2][0] = v[1].z - v[0].z;
    g.J[0][1] = v[2].x - v[0].x; g.J[1][1] = v[2].y - v[0].y; g.J[2][1] = v[2].z - v[0].z;
    g.J[0][2] = v[3].x - v[0].x; g.J[1][2] = v[3].y - v[0].y; g.J[2][2] = v[3].z - v[0].z;
    double m0 = g.J[1][1] * g.J[2][2] - g.J[1][2] * g.J[2][1];
    double m1 = g.J[1][0] * g.J[2][2] - g.J[1][2] * g.J[2][0];
    double m2 = g.J[1][0] * g.J[2][1] - g.J[1][1] * g.J[2][0];
    g.det = g.J[0][0] * m0 - g.J[0][1] * m1 + g.J[0][2] * m2;
    g.rdet = 1.0 / g.det;
    g.adet = fabs(g.det);
    double av[6];
    for (int i = 0; i < 6; i++) av[i] = d[i] >= 0 ? elem::flip(a.Sol[d[i]], (sb >> i) & 1) : 0.0;
    double res[6], K[6][6];
    elem::jacobian_block<CALCJ, STDCURL>(g, av, tag, qp, mp, res, K);
    for (int i = 0; i < 6; i++) {
        double row[6];
        for (int j = 0; j < 6; j++) row[j] = CALCJ ? elem::flip(K[i][j], ((sb >> i) ^ (sb >> j)) & 1) : 0.0;
        elem::store_row(dst + i * kScratchStride, row, elem::flip(res[i], (sb >> i) & 1));
    }
}

// Blocks -> the reference's triplet order (36e + 6j + i) and residual pairs.
__global__ void k_na_triplets(const double *__restrict__ blocks, const double *__restrict__ Dofs,
                              int64_t ne, int calcj, double *__restrict__ I, double *__restrict__ J,
                              double *__restrict__ V, double *__restrict__ Ridx, double *__restrict__ Rval) {
    int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= 36 * ne) return;
    int64_t e = s / 36;
    int r = (int)(s - 36 * e);
    int j = r / 6, i = r - 6 * j;
    const double *src = blocks + e * kScratchPerElem;
    if (calcj) {
        I[s] = (double)(int)Dofs[6 * e + i];
        J[s] = (double)(int)Dofs[6 * e + j];
        V[s] = src[i * kScratchStride + j];
    }
    if (r < 6) {
        Ridx[6 * e + r] = (double)(int)Dofs[6 * e + r];
        Rval[6 * e + r] = src[r * kScratchStride + 6];
    }
}

bool standard_curl(const double *curl, int nq) {
    static const double c[6][3] = {{0, -2, 2}, {2, 0, -2}, {-2, 2, 0}, {0, 0, 2}, {0, -2, 0}, {2, 0, 0}};
    for (int q = 0; q < nq; q++)
        for (int i = 0; i < 6; i++)
            for (int k = 0; k < 3; k++)
                if (curl[i + 6 * k + 18 * q] != c[i][k]) return false;
    return true;
}

}  // namespace
}  // namespace mag

using namespace mag;

extern "C" int mag_mex_jacobian_noalloc(
    const double *d_P, int64_t Nn, const double *d_T, int64_t Ne, const double *d_Dofs,
    const double *d_Signs, const double *d_Tags, const double *d_SolA, int64_t Ndof, const double *Qw,
    int nq, const double *CurlRef, const double *lin, const double *isNon, const double *maxB, int nmat,
    const double *brk, int nbrk, const double *coe, int ncoe, const double *start, const double *cnt,
    const double *coeStart, int calc_j, double *d_I, double *d_J, double *d_V, double *d_Ridx,
    double *d_Rval, void *stream) {
    if (!d_P || !d_T || !d_Dofs || !d_Signs || !d_Tags || !d_SolA || !Qw || !CurlRef || !lin || !isNon ||
        !maxB || !start || !cnt || !coeStart || !d_Ridx || !d_Rval || (calc_j && (!d_I || !d_J || !d_V)) ||
        Nn <= 0 || Ne <= 0 || Ndof <= 0 || nbrk < 0 || ncoe < 0 || (nbrk && !brk) || (ncoe && !coe)) {
        set_error("mag_mex_jacobian_noalloc: bad arguments");
        return MAG_E_ARG;
    }
    if (Ne > kNoAllocMaxElements || nmat < 1 || nmat > kNaMaxMat || nbrk > kNaMaxBreaks ||
        ncoe > kNaMaxCoefs || nq < 1 || nq > kMaxQuad || Nn >= (int64_t(1) << 31) ||
        Ndof >= (int64_t(1) << 31)) {
        set_error("mag_mex_jacobian_noalloc: size beyond its static scratch (at most %lld elements, "
                  "%d materials, %d breaks, %d coefficients, %d quadrature points); got Ne=%lld, "
                  "nmat=%d, nbrk=%d, ncoe=%d, nq=%d",
                  (long long)kNoAllocMaxElements, kNaMaxMat, kNaMaxBreaks, kNaMaxCoefs, kMaxQuad,
                  (long long)Ne, nmat, nbrk, ncoe, nq);
        return MAG_E_UNSUPPORTED;
    }
    int ints[3 * kNaMaxMat];
    for (int m = 0; m < nmat; m++) {
        int st = (int)start[m], c = (int)cnt[m], cs = (int)coeStart[m];
        if (isNon[m] != 0.0 && (c < 1 || st < 0 || st + c > nbrk || cs < 0 || cs + 4 * c > ncoe)) {
            set_error("mag_mex_jacobian_noalloc: spline table of tag %d out of range", m + 1);
            return MAG_E_RANGE;
        }
        ints[m] = st;
        ints[kNaMaxMat + m] = c;
        ints[2 * kNaMaxMat + m] = cs;
    }
    double *base = nullptr;
    MAG_TRY(scratch_address(&base));
    cudaStream_t s = (cudaStream_t)stream;
    int *d_err = reinterpret_cast<int *>(base + kOffErr);
    int *d_ints = reinterpret_cast<int *>(base + kOffInts);
    MAG_CUDA_TRY(cudaMemsetAsync(d_err, 0, sizeof(int), s));
    MAG_CUDA_TRY(cudaMemcpyAsync(base + kOffLin, lin, nmat * 8, cudaMemcpyHostToDevice, s));
    MAG_CUDA_TRY(cudaMemcpyAsync(base + kOffIsNon, isNon, nmat * 8, cudaMemcpyHostToDevice, s));
    MAG_CUDA_TRY(cudaMemcpyAsync(base + kOffMaxB, maxB, nmat * 8, cudaMemcpyHostToDevice, s));
    if (nbrk) MAG_CUDA_TRY(cudaMemcpyAsync(base + kOffBreaks, brk, nbrk * 8, cudaMemcpyHostToDevice, s));
    if (ncoe) MAG_CUDA_TRY(cudaMemcpyAsync(base + kOffCoefs, coe, ncoe * 8, cudaMemcpyHostToDevice, s));
    MAG_CUDA_TRY(cudaMemcpyAsync(d_ints, ints, sizeof ints, cudaMemcpyHostToDevice, s));
    MAG_CUDA_TRY(cudaMemcpyAsync(base + kOffCurl, CurlRef, 18 * nq * 8, cudaMemcpyHostToDevice, s));

    QuadParams qp{};
    qp.nq = nq;
    qp.uniform_w = 1;
    for (int q = 0; q < nq; q++) {
        qp.qw[q] = Qw[q];
        if (Qw[q] != Qw[0]) qp.uniform_w = 0;
    }
    qp.standard_curl = standard_curl(CurlRef, nq) ? 1 : 0;
    qp.curl_ref = base + kOffCurl;
    qp.val_ref = base + kOffCurl;
    MaterialParams mp{nmat, nbrk, ncoe, base + kOffLin, base + kOffIsNon, base + kOffMaxB,
                      base + kOffBreaks, base + kOffCoefs, d_ints, d_ints + kNaMaxMat,
                      d_ints + 2 * kNaMaxMat};
    NaArgs a{d_P, d_T, d_Dofs, d_Signs, d_Tags, d_SolA, Nn, Ne, Ndof, nmat};
    double *blocks = base + kOffBlocks;
    unsigned g = (unsigned)((Ne + 127) / 128);
    if (qp.standard_curl) {
        if (calc_j) k_na_elems<true, true><<<g, 128, 0, s>>>(a, qp, mp, blocks, d_err);
        else k_na_elems<false, true><<<g, 128, 0, s>>>(a, qp, mp, blocks, d_err);
    } else {
        if (calc_j) k_na_elems<true, false><<<g, 128, 0, s>>>(a, qp, mp, blocks, d_err);
        else k_na_elems<false, false><<<g, 128, 0, s>>>(a, qp, mp, blocks, d_err);
    }
    MAG_CUDA_TRY(cudaPeekAtLastError());
    k_na_triplets<<<(unsigned)((36 * Ne + 255) / 256), 256, 0, s>>>(blocks, d_Dofs, Ne, calc_j, d_I, d_J,
                                                                    d_V, d_Ridx, d_Rval);
    MAG_CUDA_TRY(cudaPeekAtLastError());
    int herr = 0;
    MAG_CUDA_TRY(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    MAG_CUDA_TRY(cudaStreamSynchronize(s));
    if (herr) {
        set_error("mag_mex_jacobian_noalloc: index, sign, tag or coordinate out of range (nodes 1..Nn, "
                  "dofs 0..numel(SolA), signs +-1, tags 1..nmat, finite P); outputs are incomplete");
        return MAG_E_RANGE;
    }
    return MAG_OK;
}
