// C ABI (include/magasm.h): the mesh handle, validation, and the
// MEX-compatible entry points.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <vector>

#include "assemble.cuh"
#include "batch.cuh"
#include "common.cuh"
#include "tile.cuh"
#include "rowblock.cuh"
#include "internal.h"
#include "mlp.cuh"
#include "sparse.cuh"
#include "hbfem.cuh"

namespace mag {

namespace {
thread_local char g_err[768] = "";
}

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

namespace {

constexpr int kB = 256;
inline unsigned grid(int64_t n) { return (unsigned)((n + kB - 1) / kB); }

// ---- input conversion / validation kernels ---------------------------------

__global__ void k_pack_xyz(const double *__restrict__ P, int64_t nn, double4 *__restrict__ xyz,
                           int *__restrict__ err) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= nn) return;
    double x = P[3 * i], y = P[3 * i + 1], z = P[3 * i + 2];
    if (!isfinite(x) || !isfinite(y) || !isfinite(z)) atomicExch(err, 1);
    xyz[i] = make_double4(x, y, z, 0.0);
}

// 1-based node ids stored as doubles (MEX layout) -> 0-based int32.
__global__ void k_index_from_double(const double *__restrict__ src, int64_t n, int32_t *__restrict__ dst,
                                    int64_t limit, int allow_zero, int *__restrict__ err,
                                    int *__restrict__ maxval = nullptr) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v = src[i];
    // the reference truncates with (int) before use
    int64_t k = (v > -2.0 && v < 4294967296.0) ? (int64_t)v : -2;
    if (k < (allow_zero ? 0 : 1) || k > limit) {
        atomicExch(err, 1);
        k = allow_zero ? 0 : 1;
    }
    dst[i] = (int32_t)(k - 1);
    if (maxval) atomicMax(maxval, (int)k);
}

__global__ void k_check_nodes(const int4 *__restrict__ tet, int64_t ne, int64_t nn, int *__restrict__ err) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= ne) return;
    int4 t = tet[e];
    if (t.x < 0 || t.y < 0 || t.z < 0 || t.w < 0 || t.x >= nn || t.y >= nn || t.z >= nn || t.w >= nn)
        atomicExch(err, 1);
}

__global__ void k_pack_tags_i32(const int32_t *__restrict__ src, int64_t ne, uint8_t *__restrict__ dst,
                                int *__restrict__ maxtag, int *__restrict__ err) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= ne) return;
    int32_t t = src[e];
    if (t < 1 || t > kMaxMaterials) {
        atomicExch(err, 1);
        t = 1;
    }
    dst[e] = (uint8_t)t;
    atomicMax(maxtag, t);
}

__global__ void k_pack_tags_f64(const double *__restrict__ src, int64_t ne, uint8_t *__restrict__ dst,
                                int *__restrict__ maxtag, int *__restrict__ err) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= ne) return;
    double v = src[e];
    int t = (v >= 1.0 && v < 256.0) ? (int)v : 0;
    if (t < 1 || t > kMaxMaterials) {
        atomicExch(err, 1);
        t = 1;
    }
    dst[e] = (uint8_t)t;
    atomicMax(maxtag, t);
}

// Signs: bit k of signbits[e] set <=> sign -1. Counts disagreements with the
// Mesh.m:134-135 rule so that matching signs need not be stored.
__global__ void k_pack_signs_i8(const int8_t *__restrict__ s, const int4 *__restrict__ tet, int64_t ne,
                                uint8_t *__restrict__ bits, int *__restrict__ mismatch,
                                int *__restrict__ err) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= ne) return;
    int4 t = tet[e];
    int n[4] = {t.x, t.y, t.z, t.w};
    unsigned b = 0, d = 0;
    for (int k = 0; k < 6; k++) {
        int8_t v = s[6 * e + k];
        if (v != 1 && v != -1) atomicExch(err, 1);
        b |= (v < 0 ? 1u : 0u) << k;
        d |= (n[edge_a(k)] < n[edge_b(k)] ? 0u : 1u) << k;
    }
    bits[e] = (uint8_t)b;
    if (b != d) atomicAdd(mismatch, 1);
}

__global__ void k_pack_signs_f64(const double *__restrict__ s, int64_t ne, uint8_t *__restrict__ bits,
                                 int *__restrict__ err) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= ne) return;
    unsigned b = 0;
    for (int k = 0; k < 6; k++) {
        double v = s[6 * e + k];
        if (v != 1.0 && v != -1.0) atomicExch(err, 1);
        b |= (v < 0 ? 1u : 0u) << k;
    }
    bits[e] = (uint8_t)b;
}

__global__ void k_check_geometry(const double4 *__restrict__ xyz, const int4 *__restrict__ tet,
                                 int64_t ne, int *__restrict__ err) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= ne) return;
    int4 t = tet[e];
    double4 a = xyz[t.x], b = xyz[t.y], c = xyz[t.z], d = xyz[t.w];
    double u0 = b.x - a.x, u1 = b.y - a.y, u2 = b.z - a.z;
    double v0 = c.x - a.x, v1 = c.y - a.y, v2 = c.z - a.z;
    double w0 = d.x - a.x, w1 = d.y - a.y, w2 = d.z - a.z;
    double det = u0 * (v1 * w2 - w1 * v2) - v0 * (u1 * w2 - w1 * u2) + w0 * (u1 * v2 - v1 * u2);
    if (!(det != 0.0) || !isfinite(det)) atomicExch(err, 1);
}

__global__ void k_i32_to_i64(const int32_t *__restrict__ a, int64_t n, int64_t *__restrict__ b) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) b[i] = a[i];
}

struct Dev {
    void *p = nullptr;
    cudaStream_t s = nullptr;
    explicit Dev(cudaStream_t st) : s(st) {}
    ~Dev() {
        if (p) cudaFreeAsync(p, s);
    }
    cudaError_t alloc(size_t bytes) { return cudaMallocAsync(&p, bytes ? bytes : 16, s); }
    template <class T> T *as() const { return static_cast<T *>(p); }
};

int sync_flag(const int *d, cudaStream_t s, int *h) {
    MAG_CUDA_TRY(cudaMemcpyAsync(h, d, sizeof(int), cudaMemcpyDeviceToHost, s));
    MAG_CUDA_TRY(cudaStreamSynchronize(s));
    return MAG_OK;
}

// Order-2 Nedelec reference data of get_quadrature_data.m:18-28 and
// nedelec_tet_p1.m:28-51, evaluated as those scripts do.
void default_reference_data(double qw[4], double curl[72], double val[72]) {
    const double a = 0.58541020, b = 0.13819660;
    const double xi[4] = {a, b, b, b}, eta[4] = {b, a, b, b}, zeta[4] = {b, b, a, b};
    const double G[4][3] = {{-1, -1, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int q = 0; q < 4; q++) {
        qw[q] = 1.0 / 24.0;
        double L[4] = {((1.0 - xi[q]) - eta[q]) - zeta[q], xi[q], eta[q], zeta[q]};
        for (int e = 0; e < 6; e++) {
            int i = edge_a(e), j = edge_b(e);
            double cr[3] = {G[i][1] * G[j][2] - G[i][2] * G[j][1], G[i][2] * G[j][0] - G[i][0] * G[j][2],
                            G[i][0] * G[j][1] - G[i][1] * G[j][0]};
            for (int c = 0; c < 3; c++) {
                val[e + 6 * c + 18 * q] = G[j][c] * L[i] - G[i][c] * L[j];
                curl[e + 6 * c + 18 * q] = 2.0 * cr[c];
            }
        }
    }
}

bool is_standard_curl(const double *curl, int nq) {
    static const double std_c[6][3] = {{0, -2, 2}, {2, 0, -2}, {-2, 2, 0}, {0, 0, 2}, {0, -2, 0}, {2, 0, 0}};
    for (int q = 0; q < nq; q++)
        for (int i = 0; i < 6; i++)
            for (int c = 0; c < 3; c++)
                if (curl[i + 6 * c + 18 * q] != std_c[i][c]) return false;
    return true;
}

}  // namespace

// Material tables on the device.
struct MaterialStore {
    void *mem = nullptr;
    MaterialParams mp{};
};

int upload_materials(const double *lin, const double *isnon, const double *maxb, int nmat,
                     const double *brk, int nbrk, const double *coe, int ncoe, const double *start,
                     const double *cnt, const double *coestart, MaterialStore *out, cudaStream_t s) {
    if (nmat <= 0 || !lin || !isnon || !maxb || !start || !cnt || !coestart || nbrk < 0 || ncoe < 0) {
        set_error("materials: bad arguments");
        return MAG_E_ARG;
    }
    // validate the spline windows on the host
    for (int m = 0; m < nmat; m++) {
        if (isnon[m] == 0.0) continue;
        int st = (int)start[m], c = (int)cnt[m], cs = (int)coestart[m];
        if (c < 1 || st < 0 || st + c > nbrk || cs < 0 || cs + 4 * c > ncoe) {
            set_error("materials: spline table of tag %d out of range", m + 1);
            return MAG_E_RANGE;
        }
    }
    // doubles: lin | isnon | maxb | breaks | coefs | bucket geometry (2 per material);
    // ints: start | count | coef_start | bucket windows (2 kMatBuckets per material)
    size_t nd = (size_t)5 * nmat + nbrk + ncoe, ni = (size_t)3 * nmat + (size_t)2 * kMatBuckets * nmat;
    size_t bytes = nd * 8 + ni * 4 + 64;
    char *host = new (std::nothrow) char[bytes];
    if (!host) return MAG_E_NOMEM;
    std::memset(host, 0, bytes);
    double *hd = reinterpret_cast<double *>(host);
    std::memcpy(hd, lin, nmat * 8);
    std::memcpy(hd + nmat, isnon, nmat * 8);
    std::memcpy(hd + 2 * nmat, maxb, nmat * 8);
    if (nbrk) std::memcpy(hd + 3 * nmat, brk, nbrk * 8);
    if (ncoe) std::memcpy(hd + 3 * nmat + nbrk, coe, ncoe * 8);
    double *geom = hd + 3 * nmat + nbrk + ncoe;
    int *hi = reinterpret_cast<int *>(hd + nd);
    for (int m = 0; m < nmat; m++) {
        hi[m] = (int)start[m];
        hi[nmat + m] = (int)cnt[m];
        hi[2 * nmat + m] = (int)coestart[m];
    }
    // Search windows of the spline lookup (see material_eval): for a table of strictly
    // increasing finite breaks below a finite MaxBSq, kMatBuckets buckets uniform in s from
    // the first break to MaxBSq; bucket i's window is [K(e(i-1)), K(e(i+2))] with K(y) the
    // last break <= y (0 if none) and e(j) = origin + j / scale. Other tables keep scale 0.
    int *win = hi + 3 * nmat;
    for (int m = 0; m < nmat; m++) {
        if (isnon[m] == 0.0) continue;
        const int st = (int)start[m], c = (int)cnt[m];
        const double *b = brk + st, smax = maxb[m];
        bool ok = std::isfinite(smax) && std::isfinite(b[0]) && smax > b[0];
        for (int j = 1; j < c && ok; j++) ok = std::isfinite(b[j]) && b[j] > b[j - 1];
        const double scale = ok ? (double)kMatBuckets / (smax - b[0]) : 0.0;
        if (!(scale > 0.0) || !std::isfinite(scale)) continue;
        auto K = [&](double y) {
            const int j = (int)(std::upper_bound(b, b + c, y) - b) - 1;
            return j < 0 ? 0 : j;
        };
        int *lo = win + 2 * kMatBuckets * m, *up = lo + kMatBuckets;
        for (int i = 0; i < kMatBuckets; i++) {
            lo[i] = K(b[0] + (double)(i - 1) / scale);
            up[i] = K(b[0] + (double)(i + 2) / scale);
        }
        geom[2 * m] = b[0];
        geom[2 * m + 1] = scale;
    }
    void *dmem = nullptr;
    cudaError_t ce = cudaMalloc(&dmem, bytes);
    if (ce != cudaSuccess) {
        delete[] host;
        set_error("materials: %s", cudaGetErrorString(ce));
        return MAG_E_NOMEM;
    }
    ce = cudaMemcpyAsync(dmem, host, bytes, cudaMemcpyHostToDevice, s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    delete[] host;
    if (ce != cudaSuccess) {
        cudaFree(dmem);
        set_error("materials: %s", cudaGetErrorString(ce));
        return MAG_E_CUDA;
    }
    if (out->mem) cudaFree(out->mem);
    out->mem = dmem;
    double *dd = static_cast<double *>(dmem);
    int *di = reinterpret_cast<int *>(dd + nd);
    out->mp = MaterialParams{nmat, nbrk, ncoe, dd, dd + nmat, dd + 2 * nmat, dd + 3 * nmat,
                             dd + 3 * nmat + nbrk, di, di + nmat, di + 2 * nmat, di + 3 * nmat,
                             dd + 3 * nmat + nbrk + ncoe};
    return MAG_OK;
}

int make_quad(const double *qw, int nq, const double *curl, const double *val, QuadParams *qp,
              double **d_ref, cudaStream_t s) {
    if (nq < 1 || nq > kMaxQuad || !qw || !curl || !val) {
        set_error("quadrature: need 1..%d points and both basis tables", kMaxQuad);
        return MAG_E_ARG;
    }
    QuadParams q{};
    q.nq = nq;
    q.uniform_w = 1;
    for (int i = 0; i < nq; i++) {
        q.qw[i] = qw[i];
        if (qw[i] != qw[0]) q.uniform_w = 0;
    }
    q.standard_curl = is_standard_curl(curl, nq) ? 1 : 0;
    double *d = nullptr;
    MAG_CUDA_TRY(cudaMalloc(&d, 2 * 18 * nq * sizeof(double)));
    cudaError_t ce = cudaMemcpyAsync(d, curl, 18 * nq * 8, cudaMemcpyHostToDevice, s);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(d + 18 * nq, val, 18 * nq * 8, cudaMemcpyHostToDevice, s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess) {
        cudaFree(d);
        set_error("quadrature: %s", cudaGetErrorString(ce));
        return MAG_E_CUDA;
    }
    q.curl_ref = d;
    q.val_ref = d + 18 * nq;
    if (*d_ref) cudaFree(*d_ref);
    *d_ref = d;
    *qp = q;
    return MAG_OK;
}

}  // namespace mag

using namespace mag;

struct mag_mesh {
    int64_t nn = 0, ne = 0, ndof = 0;
    double4 *xyz = nullptr;
    int4 *tet = nullptr;
    int32_t *dofs = nullptr;
    uint8_t *tags = nullptr;
    uint8_t *signbits = nullptr;
    int max_tag = 0;
    PatternBuffers pat;
    double *scratch = nullptr;
    QuadParams qp{};
    double *d_ref = nullptr;
    MaterialStore mat;
    int has_mat = 0;
    RowBlockPlan rowblock;
    RowBlockPlan rowshared;  // 256-incidence blocks with per-block distinct-element lists
    uint8_t *second = nullptr;  // per incidence: second-contributor bits (NULL: some row has > 2)
    TilePlan tile;              // spatial-tile blocks (default schedule)
    int *status = nullptr;      // device word: a tile kernel skipped an out-of-range plan index
    int schedule = MAG_SCHEDULE_ROW_BLOCKS;
    int64_t bytes = 0;

    ElemData elems() const { return ElemData{xyz, tet, dofs, tags, signbits, ne}; }
    RowPlan rows() const {
        return RowPlan{pat.row_ptr, pat.inc_ptr, pat.inc_elem, pat.inc_pos, ndof, pat.wide};
    }
};

namespace {

void destroy_mesh(mag_mesh *m) {
    if (!m) return;
    void *ptrs[] = {m->xyz, m->tet, m->dofs, m->tags, m->signbits, m->scratch, m->d_ref, m->mat.mem, m->second,
                    m->status};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    free_pattern(&m->pat, nullptr);
    free_tile_plan(&m->tile);
    free_rowblock_plan(&m->rowblock);
    free_rowblock_plan(&m->rowshared);
    cudaDeviceSynchronize();
    delete m;
}

int require_ready(const mag_mesh *m, bool need_mat) {
    if (!m) {
        set_error("null mesh handle");
        return MAG_E_ARG;
    }
    if (need_mat && !m->has_mat) {
        set_error("materials not set (mag_mesh_set_materials)");
        return MAG_E_ARG;
    }
    if (need_mat && m->mat.mp.nmat < m->max_tag) {
        set_error("material table has %d entries but the mesh uses tag %d", m->mat.mp.nmat, m->max_tag);
        return MAG_E_RANGE;
    }
    return MAG_OK;
}

int finish(cudaStream_t s) {
    (void)s;
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) {
        set_error("kernel launch failed: %s", cudaGetErrorString(e));
        return MAG_E_CUDA;
    }
    return MAG_OK;
}

}  // namespace

extern "C" {

int mag_version(void) { return 1; }
const char *mag_last_error(void) { return g_err; }

int mag_sync(void *stream) {
    const cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) {
        set_error("mag_sync: %s", cudaGetErrorString(e));
        return MAG_E_CUDA;
    }
    return MAG_OK;
}

int mag_generate_edges(const int32_t *d_T, int64_t Ne, int64_t Nn, int32_t *d_edges, int32_t *d_t2e,
                       int8_t *d_sign, int64_t *E_out, void *stream) {
    return generate_edges(d_T, Ne, Nn, d_edges, d_t2e, d_sign, E_out, (cudaStream_t)stream);
}

int mag_mesh_create(const double *d_P, int64_t Nn, const int32_t *d_T, int64_t Ne,
                    const int32_t *d_dofs, const int8_t *d_signs, const int32_t *d_tags,
                    int64_t num_dofs, mag_mesh **out, void *stream) {
    if (!out || !d_P || !d_T || !d_dofs || !d_tags || Nn <= 0 || Ne <= 0 || num_dofs <= 0) {
        set_error("mag_mesh_create: bad arguments");
        return MAG_E_ARG;
    }
    *out = nullptr;
    cudaStream_t s = (cudaStream_t)stream;
    mag_mesh *m = new (std::nothrow) mag_mesh();
    if (!m) return MAG_E_NOMEM;
    m->nn = Nn;
    m->ne = Ne;
    m->ndof = num_dofs;
    auto fail = [&](int code) {
        destroy_mesh(m);
        return code;
    };
    Dev err(s), mx(s), mism(s);
    if (err.alloc(4) != cudaSuccess || mx.alloc(4) != cudaSuccess || mism.alloc(4) != cudaSuccess) {
        set_error("mag_mesh_create: out of device memory");
        return fail(MAG_E_NOMEM);
    }
    cudaMemsetAsync(err.p, 0, 4, s);
    cudaMemsetAsync(mx.p, 0, 4, s);
    cudaMemsetAsync(mism.p, 0, 4, s);
    size_t b_xyz = Nn * sizeof(double4), b_tet = Ne * sizeof(int4), b_dofs = Ne * 6 * 4, b_tags = Ne;
    if (cudaMalloc(&m->xyz, b_xyz) != cudaSuccess || cudaMalloc(&m->tet, b_tet) != cudaSuccess ||
        cudaMalloc(&m->dofs, b_dofs) != cudaSuccess || cudaMalloc(&m->tags, b_tags) != cudaSuccess) {
        set_error("mag_mesh_create: out of device memory");
        return fail(MAG_E_NOMEM);
    }
    m->bytes = b_xyz + b_tet + b_dofs + b_tags;
    k_pack_xyz<<<grid(Nn), kB, 0, s>>>(d_P, Nn, m->xyz, err.as<int>());
    cudaMemcpyAsync(m->tet, d_T, b_tet, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(m->dofs, d_dofs, b_dofs, cudaMemcpyDeviceToDevice, s);
    k_check_nodes<<<grid(Ne), kB, 0, s>>>(m->tet, Ne, Nn, err.as<int>());
    int h = 0;
    if (sync_flag(err.as<int>(), s, &h) != MAG_OK) return fail(MAG_E_CUDA);
    if (h) {
        set_error("mag_mesh_create: node id out of range or non-finite coordinate");
        return fail(MAG_E_RANGE);
    }
    k_check_geometry<<<grid(Ne), kB, 0, s>>>(m->xyz, m->tet, Ne, err.as<int>());
    if (sync_flag(err.as<int>(), s, &h) != MAG_OK) return fail(MAG_E_CUDA);
    if (h) {
        set_error("mag_mesh_create: degenerate element (zero or non-finite det J)");
        return fail(MAG_E_GEOMETRY);
    }
    k_pack_tags_i32<<<grid(Ne), kB, 0, s>>>(d_tags, Ne, m->tags, mx.as<int>(), err.as<int>());
    if (sync_flag(err.as<int>(), s, &h) != MAG_OK) return fail(MAG_E_CUDA);
    if (h) {
        set_error("mag_mesh_create: region tag outside 1..%d", kMaxMaterials);
        return fail(MAG_E_RANGE);
    }
    if (sync_flag(mx.as<int>(), s, &m->max_tag) != MAG_OK) return fail(MAG_E_CUDA);
    if (d_signs) {
        if (cudaMalloc(&m->signbits, Ne) != cudaSuccess) return fail(MAG_E_NOMEM);
        k_pack_signs_i8<<<grid(Ne), kB, 0, s>>>(d_signs, m->tet, Ne, m->signbits, mism.as<int>(),
                                                err.as<int>());
        int mm = 0;
        if (sync_flag(err.as<int>(), s, &h) != MAG_OK || sync_flag(mism.as<int>(), s, &mm) != MAG_OK)
            return fail(MAG_E_CUDA);
        if (h) {
            set_error("mag_mesh_create: signs must be +1 or -1");
            return fail(MAG_E_ARG);
        }
        if (mm == 0) {  // identical to the derived rule: do not store them
            cudaFree(m->signbits);
            m->signbits = nullptr;
        } else {
            m->bytes += Ne;
        }
    }
    int rc = build_pattern(m->dofs, Ne, num_dofs, &m->pat, s);
    if (rc != MAG_OK) return fail(rc);
    m->bytes += (int64_t)(num_dofs + 1) * 8 + m->pat.nnz * 4 + m->pat.ninc * 4 * (m->pat.wide ? 3 : 2);
    if (cudaMalloc(&m->scratch, (size_t)Ne * kScratchPerElem * sizeof(double)) != cudaSuccess) {
        set_error("mag_mesh_create: out of device memory for the element scratch");
        return fail(MAG_E_NOMEM);
    }
    m->bytes += (int64_t)Ne * kScratchPerElem * 8;
    // optional schedules; the two-pass kernels always work
    if (build_rowblock_plan(m->rows(), &m->rowblock, s) == MAG_OK) {
        m->bytes += m->rowblock.bytes;
    } else {
        free_rowblock_plan(&m->rowblock);
        cudaGetLastError();
    }
    if (build_second_masks(m->rows(), m->pat.ninc, &m->second, s) == MAG_OK && m->second) m->bytes += m->pat.ninc;
    if (build_rowblock_plan(m->rows(), &m->rowshared, s, kSharedBlockInc, true, m->second) == MAG_OK &&
        m->rowshared.shared_ok) {
        m->bytes += m->rowshared.bytes;
    } else {
        free_rowblock_plan(&m->rowshared);
        cudaGetLastError();
    }
    if (cudaMalloc(&m->status, sizeof(int)) != cudaSuccess) return fail(MAG_E_NOMEM);
    cudaMemsetAsync(m->status, 0, sizeof(int), s);
    {
        const TilePlanInput ti{m->xyz, m->tet, m->dofs, m->tags, m->signbits, m->pat.row_ptr, m->pat.inc_ptr,
                               m->pat.inc_elem, m->pat.inc_pos, Nn, Ne, num_dofs, m->pat.nnz, m->pat.ninc,
                               m->pat.wide};
        rc = build_tile_plan(ti, &m->tile, s);
        if (rc != MAG_OK) return fail(rc);
        if (m->tile.ok) m->bytes += m->tile.bytes;
    }
    m->schedule = m->tile.ok               ? MAG_SCHEDULE_TILE_BLOCKS
                  : m->rowshared.nz_ok     ? MAG_SCHEDULE_NZ_ROW_BLOCKS
                  : m->rowshared.shared_ok ? MAG_SCHEDULE_SHARED_ROW_BLOCKS
                  : m->rowblock.ok         ? MAG_SCHEDULE_ROW_BLOCKS
                                           : MAG_SCHEDULE_TWO_PASS;
    double qw[4], curl[72], val[72];
    default_reference_data(qw, curl, val);
    rc = make_quad(qw, 4, curl, val, &m->qp, &m->d_ref, s);
    if (rc != MAG_OK) return fail(rc);
    *out = m;
    return MAG_OK;
}

int mag_mesh_destroy(mag_mesh *mesh) {
    destroy_mesh(mesh);
    return MAG_OK;
}

int mag_mesh_get_info(const mag_mesh *m, mag_mesh_info *info) {
    if (!m || !info) {
        set_error("mag_mesh_get_info: bad arguments");
        return MAG_E_ARG;
    }
    std::memset(info, 0, sizeof *info);
    info->num_nodes = m->nn;
    info->num_elements = m->ne;
    info->num_dofs = m->ndof;
    info->nnz = m->pat.nnz;
    info->num_incidences = m->pat.ninc;
    info->max_row_nnz = m->pat.max_row;
    info->wide_positions = m->pat.wide;
    info->signs_derived = m->signbits ? 0 : 1;
    info->schedule = m->schedule;
    info->tile_blocks = m->tile.ok ? m->tile.nblocks : 0;
    info->tile_colors = m->tile.ok ? m->tile.max_colors : 0;
    info->tile_evals_per_elem = m->tile.ok ? m->tile.evals_per_elem : 0.0;
    info->tile_plan_ms = m->tile.build_ms;
    info->device_bytes = m->bytes;
    info->shared_blocks = m->rowshared.shared_ok ? m->rowshared.nblocks : 0;
    info->reserved0 = 0;
    info->nz_pass = m->rowshared.nz_ok;
    return MAG_OK;
}

int mag_mesh_pattern(const mag_mesh *m, int64_t *d_row_ptr, int32_t *d_col_idx, void *stream) {
    if (!m || !d_row_ptr || !d_col_idx) {
        set_error("mag_mesh_pattern: bad arguments");
        return MAG_E_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    k_i32_to_i64<<<grid(m->ndof + 1), kB, 0, s>>>(m->pat.row_ptr, m->ndof + 1, d_row_ptr);
    MAG_CUDA_TRY(cudaMemcpyAsync(d_col_idx, m->pat.col_idx, m->pat.nnz * 4, cudaMemcpyDeviceToDevice, s));
    return finish(s);
}

int mag_mesh_set_quadrature(mag_mesh *m, const double *qw, int nq, const double *curl_ref,
                            const double *val_ref) {
    if (!m) {
        set_error("null mesh handle");
        return MAG_E_ARG;
    }
    return make_quad(qw, nq, curl_ref, val_ref, &m->qp, &m->d_ref, nullptr);
}

int mag_mesh_set_materials(mag_mesh *m, const double *lin_nu, const double *is_nonlinear,
                           const double *max_bsq, int nmat, const double *breaks, int nbreaks,
                           const double *coefs, int ncoefs, const double *spline_start,
                           const double *spline_count, const double *coef_start) {
    if (!m) {
        set_error("null mesh handle");
        return MAG_E_ARG;
    }
    int rc = upload_materials(lin_nu, is_nonlinear, max_bsq, nmat, breaks, nbreaks, coefs, ncoefs,
                              spline_start, spline_count, coef_start, &m->mat, nullptr);
    if (rc == MAG_OK) m->has_mat = 1;
    return rc;
}

int mag_assemble_jacobian(mag_mesh *m, const double *d_sol, double *d_vals, double *d_res, int calc_j,
                          void *stream) {
    MAG_TRY(require_ready(m, true));
    if (!d_sol || !d_res || (calc_j && !d_vals)) {
        set_error("mag_assemble_jacobian: bad arguments");
        return MAG_E_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    if (m->schedule == MAG_SCHEDULE_TILE_BLOCKS && m->tile.ok && m->qp.standard_curl) {
        MAG_TRY(launch_tile_jacobian(m->tile, m->elems(), d_sol, m->qp, m->mat.mp, calc_j, calc_j ? d_vals : nullptr,
                                     d_res, m->status, s));
        return finish(s);
    }
    if ((m->schedule == MAG_SCHEDULE_NZ_ROW_BLOCKS || m->schedule == MAG_SCHEDULE_TILE_BLOCKS) &&
        m->rowshared.nz_ok && m->qp.standard_curl) {
        MAG_TRY(launch_rowblock_nz_jacobian(m->rowshared, m->elems(), m->rows(), d_sol, m->qp, m->mat.mp, calc_j,
                                            calc_j ? d_vals : nullptr, d_res, s));
        return finish(s);
    }
    const bool rowsched = m->schedule == MAG_SCHEDULE_NZ_ROW_BLOCKS || m->schedule == MAG_SCHEDULE_TILE_BLOCKS;
    if ((m->schedule == MAG_SCHEDULE_SHARED_ROW_BLOCKS || rowsched) && m->rowshared.shared_ok &&
        m->qp.standard_curl) {
        MAG_TRY(launch_rowblock_shared_jacobian(m->rowshared, m->elems(), m->rows(), d_sol, m->qp, m->mat.mp,
                                                calc_j, calc_j ? d_vals : nullptr, d_res, s));
        return finish(s);
    }
    if (m->schedule == MAG_SCHEDULE_ROW_BLOCKS || m->schedule == MAG_SCHEDULE_SHARED_ROW_BLOCKS || rowsched) {
        MAG_TRY(launch_rowblock_jacobian(m->rowblock, m->elems(), m->rows(), d_sol, m->qp, m->mat.mp, calc_j,
                                         calc_j ? d_vals : nullptr, d_res, s));
        return finish(s);
    }
    MAG_TRY(launch_jacobian_elems(m->elems(), d_sol, m->qp, m->mat.mp, calc_j, m->scratch, s));
    MAG_TRY(launch_rows_reduce(m->rows(), m->pat.max_row, m->scratch, calc_j ? d_vals : nullptr, d_res, s));
    return finish(s);
}

int mag_assemble_stiffness(mag_mesh *m, const double *d_nu, double *d_vals, void *stream) {
    MAG_TRY(require_ready(m, false));
    if (!d_nu || !d_vals) {
        set_error("mag_assemble_stiffness: bad arguments");
        return MAG_E_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    if (m->schedule == MAG_SCHEDULE_TILE_BLOCKS && m->tile.ok && m->qp.standard_curl) {
        MAG_TRY(launch_tile_stiffness(m->tile, m->elems(), d_nu, m->qp, d_vals, m->status, s));
        return finish(s);
    }
    if ((m->schedule == MAG_SCHEDULE_NZ_ROW_BLOCKS || m->schedule == MAG_SCHEDULE_TILE_BLOCKS) &&
        m->rowshared.nz_ok && m->qp.standard_curl) {
        MAG_TRY(launch_rowblock_nz_stiffness(m->rowshared, m->elems(), m->rows(), d_nu, m->qp, d_vals, s));
        return finish(s);
    }
    MAG_TRY(launch_stiffness_elems(m->elems(), d_nu, m->qp, m->scratch, s));
    MAG_TRY(launch_rows_reduce(m->rows(), m->pat.max_row, m->scratch, d_vals, nullptr, s));
    return finish(s);
}

int mag_assemble_jacobian_seeded(mag_mesh *m, const double *d_sol, const double *d_bscale, double *d_vals,
                                 double *d_res, void *stream) {
    MAG_TRY(require_ready(m, true));
    if (!d_sol || !d_bscale || !d_vals || !d_res) {
        set_error("mag_assemble_jacobian_seeded: bad arguments");
        return MAG_E_ARG;
    }
    if (!m->qp.standard_curl) {
        set_error("mag_assemble_jacobian_seeded: needs the standard Nedelec curl table");
        return MAG_E_UNSUPPORTED;
    }
    cudaStream_t s = (cudaStream_t)stream;
    if (m->schedule == MAG_SCHEDULE_TILE_BLOCKS && m->tile.ok) {
        MAG_TRY(launch_tile_seeded(m->tile, m->elems(), d_sol, d_bscale, m->qp, m->mat.mp, d_vals, d_res, m->status,
                                   s));
        return finish(s);
    }
    MAG_TRY(launch_jacobian_seeded_elems(m->elems(), d_sol, d_bscale, m->qp, m->mat.mp, m->scratch, s));
    MAG_TRY(launch_rows_reduce(m->rows(), m->pat.max_row, m->scratch, d_vals, d_res, s));
    return finish(s);
}

int mag_assemble_hbfem(mag_mesh *m, const double *d_sol_re, const double *d_sol_im, int K, const double *d_d_re,
                       const double *d_d_im, const double *d_p_re, const double *d_p_im, int N, double *d_vals,
                       double *d_res_re, double *d_res_im, void *stream) {
    MAG_TRY(require_ready(m, true));
    if (!d_sol_re || !d_d_re || !d_p_re || !d_res_re || !d_res_im || K < 1 || N < 1) {
        set_error("mag_assemble_hbfem: bad arguments");
        return MAG_E_ARG;
    }
    if (K > kMaxHarm) {
        set_error("mag_assemble_hbfem: %d harmonics (at most %d per call)", K, kMaxHarm);
        return MAG_E_UNSUPPORTED;
    }
    cudaStream_t s = (cudaStream_t)stream;
    double *rscr = nullptr;
    MAG_CUDA_TRY(cudaMallocAsync((void **)&rscr, (size_t)m->ne * 6 * 2 * K * sizeof(double), s));
    int rc = launch_hbfem(m->elems(), m->rows(), m->pat.max_row, d_sol_re, d_sol_im, K, d_d_re, d_d_im, d_p_re,
                          d_p_im, N, m->qp, m->mat.mp, m->scratch, rscr, d_vals, d_res_re, d_res_im, s);
    cudaFreeAsync(rscr, s);
    if (rc != MAG_OK) {
        set_error("mag_assemble_hbfem: launch failed (%s)", cudaGetErrorString(cudaGetLastError()));
        return rc;
    }
    return finish(s);
}

int mag_seed_midpoint(mag_mesh *m, const double *d_sol, const double *d_nu_hat, double max_scale, double *d_bscale,
                      void *stream) {
    MAG_TRY(require_ready(m, true));
    if (!d_sol || !d_nu_hat || !d_bscale || !(max_scale >= 1.0)) {
        set_error("mag_seed_midpoint: bad arguments");
        return MAG_E_ARG;
    }
    if (!m->qp.standard_curl) {
        set_error("mag_seed_midpoint: needs the standard Nedelec curl table");
        return MAG_E_UNSUPPORTED;
    }
    cudaStream_t s = (cudaStream_t)stream;
    MAG_TRY(launch_seed_midpoint(m->elems(), d_sol, d_nu_hat, m->mat.mp, max_scale, d_bscale, s));
    return finish(s);
}

int mag_assemble_mass(mag_mesh *m, const double *d_sigma, double *d_vals, void *stream) {
    MAG_TRY(require_ready(m, false));
    if (!d_vals) {
        set_error("mag_assemble_mass: bad arguments");
        return MAG_E_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    MAG_TRY(launch_mass_elems(m->elems(), d_sigma, m->qp, m->scratch, s));
    MAG_TRY(launch_rows_reduce(m->rows(), m->pat.max_row, m->scratch, d_vals, nullptr, s));
    return finish(s);
}

int mag_assemble_source(mag_mesh *m, const double *d_js, double *d_out, void *stream) {
    MAG_TRY(require_ready(m, false));
    if (!d_js || !d_out) {
        set_error("mag_assemble_source: bad arguments");
        return MAG_E_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    MAG_TRY(launch_source_elems(m->elems(), d_js, m->qp, m->scratch, s));
    MAG_TRY(launch_rows_reduce(m->rows(), m->pat.max_row, m->scratch, nullptr, d_out, s));
    return finish(s);
}

int mag_assemble_winding(mag_mesh *m, int coil_id, const double *d_dir_field, const double *dir, double scale,
                         double *d_out, void *stream) {
    MAG_TRY(require_ready(m, false));
    if (!d_out || (!d_dir_field && !dir)) {
        set_error("mag_assemble_winding: bad arguments");
        return MAG_E_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const double zero[3] = {0.0, 0.0, 0.0};
    MAG_TRY(launch_winding_elems(m->elems(), coil_id, d_dir_field, dir ? dir : zero, scale, m->qp, m->scratch,
                                 nullptr, nullptr, s));
    MAG_TRY(launch_rows_reduce(m->rows(), m->pat.max_row, m->scratch, nullptr, d_out, s));
    return finish(s);
}

int mag_element_b(mag_mesh *m, const double *d_sol, double *d_b, double *d_bsq, void *stream) {
    MAG_TRY(require_ready(m, false));
    if (!d_sol || (!d_b && !d_bsq)) {
        set_error("mag_element_b: bad arguments");
        return MAG_E_ARG;
    }
    if (!m->qp.standard_curl) {
        set_error("mag_element_b: needs the standard Nedelec curl table");
        return MAG_E_UNSUPPORTED;
    }
    cudaStream_t s = (cudaStream_t)stream;
    MAG_TRY(launch_element_b(m->elems(), d_sol, d_b, d_bsq, s));
    return finish(s);
}

int mag_element_nu(mag_mesh *m, const double *d_sol, double *d_nu, double *d_dnu, void *stream) {
    MAG_TRY(require_ready(m, true));
    if (!d_sol || (!d_nu && !d_dnu)) {
        set_error("mag_element_nu: bad arguments");
        return MAG_E_ARG;
    }
    if (!m->qp.standard_curl) {
        set_error("mag_element_nu: needs the standard Nedelec curl table");
        return MAG_E_UNSUPPORTED;
    }
    cudaStream_t s = (cudaStream_t)stream;
    MAG_TRY(launch_element_b(m->elems(), d_sol, nullptr, nullptr, s, &m->mat.mp, d_nu, d_dnu));
    return finish(s);
}

int mag_mesh_set_option(mag_mesh *m, int option, int64_t value) {
    if (!m) {
        set_error("null mesh handle");
        return MAG_E_ARG;
    }
    if (option == MAG_OPTION_SCHEDULE) {
        if (value == MAG_SCHEDULE_RETIRED_1 || value == MAG_SCHEDULE_RETIRED_4 ||
            (value == MAG_SCHEDULE_ROW_BLOCKS && !m->rowblock.ok) ||
            (value == MAG_SCHEDULE_SHARED_ROW_BLOCKS && !m->rowshared.shared_ok) ||
            (value == MAG_SCHEDULE_NZ_ROW_BLOCKS && !m->rowshared.nz_ok) ||
            (value == MAG_SCHEDULE_TILE_BLOCKS && !m->tile.ok) || value < 0 || value > 6) {
            set_error("assembly schedule %lld is not available for this mesh", (long long)value);
            return MAG_E_UNSUPPORTED;
        }
        m->schedule = (int)value;
        return MAG_OK;
    }
    if (option == MAG_OPTION_TILE_VARIANT) {
        if (value < 0 || value >= kTileVariants) {
            set_error("tile variant %lld out of range (0..%d)", (long long)value, kTileVariants - 1);
            return MAG_E_ARG;
        }
        m->tile.variant = (int)value;
        return MAG_OK;
    }
    if (option == MAG_OPTION_TILE_PREFETCH) {
        if (value < 0 || value >= kTileDepths) {
            set_error("tile prefetch depth %lld out of range (0..%d)", (long long)value, kTileDepths - 1);
            return MAG_E_ARG;
        }
        m->tile.prefetch_waves = (int)value;
        return MAG_OK;
    }
    set_error("unknown option %d", option);
    return MAG_E_ARG;
}

int mag_mesh_tune(mag_mesh *m, const double *d_sol, double *d_vals, double *d_res, int reps, double *times_ms,
                  int *variant, int *depth, void *stream) {
    if (!m || !d_sol || !d_vals || !d_res || reps < 1) {
        set_error("mag_mesh_tune: bad arguments");
        return MAG_E_ARG;
    }
    if (m->schedule != MAG_SCHEDULE_TILE_BLOCKS || !m->tile.ok) {
        set_error("mag_mesh_tune: the mesh does not run the tile schedule");
        return MAG_E_UNSUPPORTED;
    }
    cudaStream_t s = (cudaStream_t)stream;
    cudaEvent_t e0, e1;
    MAG_CUDA_TRY(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return MAG_E_CUDA;
    }
    const int v0 = m->tile.variant, w0 = m->tile.prefetch_waves;
    int best_v = v0, best_w = w0, rc = MAG_OK;
    double best = 1e300;
    for (int v = 0; v < kTileVariants && rc == MAG_OK; v++)
        for (int w = 0; w < kTileDepths && rc == MAG_OK; w++) {
            m->tile.variant = v;
            m->tile.prefetch_waves = w;
            rc = mag_assemble_jacobian(m, d_sol, d_vals, d_res, 1, stream);  // warm-up
            if (rc != MAG_OK) break;
            cudaEventRecord(e0, s);
            for (int r = 0; r < reps && rc == MAG_OK; r++) rc = mag_assemble_jacobian(m, d_sol, d_vals, d_res, 1, stream);
            cudaEventRecord(e1, s);
            if (cudaEventSynchronize(e1) != cudaSuccess) rc = MAG_E_CUDA;
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            const double t = (double)ms / reps;
            if (times_ms) times_ms[v * kTileDepths + w] = t;
            if (rc == MAG_OK && t < best) {
                best = t;
                best_v = v;
                best_w = w;
            }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    m->tile.variant = rc == MAG_OK ? best_v : v0;
    m->tile.prefetch_waves = rc == MAG_OK ? best_w : w0;
    if (rc != MAG_OK) return rc;
    // the kept pair's outputs (every candidate gives the same bits)
    MAG_TRY(mag_assemble_jacobian(m, d_sol, d_vals, d_res, 1, stream));
    if (variant) *variant = best_v;
    if (depth) *depth = best_w;
    return MAG_OK;
}

int mag_mesh_check(mag_mesh *m, void *stream) {
    if (!m) {
        set_error("null mesh handle");
        return MAG_E_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    int h = 0;
    MAG_CUDA_TRY(cudaMemcpyAsync(&h, m->status, sizeof(int), cudaMemcpyDeviceToHost, s));
    MAG_CUDA_TRY(cudaStreamSynchronize(s));
    MAG_CUDA_TRY(cudaGetLastError());
    if (h) {
        MAG_CUDA_TRY(cudaMemsetAsync(m->status, 0, sizeof(int), s));
        MAG_CUDA_TRY(cudaStreamSynchronize(s));
        set_error("tile schedule: a plan index was out of range and was skipped (internal error); the last "
                  "assemblies are incomplete");
        return MAG_E_RANGE;
    }
    return MAG_OK;
}

int mag_csr_drop_zeros(const int64_t *d_row_ptr, const int32_t *d_col_idx, const double *d_vals,
                       int64_t nrows, int64_t *d_row_ptr_out, int32_t *d_col_out, double *d_vals_out,
                       int64_t *nnz_out, void *stream) {
    return csr_drop_zeros(d_row_ptr, d_col_idx, d_vals, nrows, d_row_ptr_out, d_col_out, d_vals_out,
                          nnz_out, (cudaStream_t)stream);
}

// ---- batched complex assembly -----------------------------------------------------

}  // extern "C"

struct mag_batch {
    BatchState st;
    int chosen = 0;
    double times[8] = {0};
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace {
void destroy_batch(mag_batch *b) {
    if (!b) return;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    batch_free_variants(&b->st);
    for (int32_t *p : b->st.owned)
        if (p) cudaFree(p);
    delete b;
}
}  // namespace

extern "C" {

int mag_batch_variants(void) { return batch_num_variants(); }

}  // extern "C"

namespace {
// Capture the chosen variant's launch in a CUDA graph (replacing any earlier one); capture
// needs a stream other than the legacy default.
int capture_batch(mag_batch *b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    cudaStream_t cs;
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) return MAG_E_CUDA;
    cudaError_t ce = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (ce == cudaSuccess) {
        batch_launch(b->st, b->chosen, cs);
        ce = cudaStreamEndCapture(cs, &b->graph);
    }
    if (ce == cudaSuccess) ce = cudaGraphInstantiate(&b->exec, b->graph, 0);
    cudaStreamDestroy(cs);
    if (ce != cudaSuccess) {
        set_error("batch graph capture failed: %s", cudaGetErrorString(ce));
        return MAG_E_CUDA;
    }
    return MAG_OK;
}
}  // namespace

extern "C" {

int mag_batch_create(mag_mesh *const *meshes, int n, const double *const *d_nu, const double *const *d_sigma,
                     const double *omega, double *const *d_vals, mag_batch **out, void *stream) {
    if (!meshes || n < 1 || !d_nu || !omega || !d_vals || !out) {
        set_error("mag_batch_create: bad arguments");
        return MAG_E_ARG;
    }
    *out = nullptr;
    cudaStream_t s = (cudaStream_t)stream;
    mag_batch *b = new (std::nothrow) mag_batch();
    if (!b) return MAG_E_NOMEM;
    auto fail = [&](int rc) {
        destroy_batch(b);
        return rc;
    };
    for (int i = 0; i < n; i++) {
        mag_mesh *m = meshes[i];
        if (!m || !d_nu[i] || !d_vals[i] || !m->rowblock.ok || !m->qp.standard_curl) {
            set_error("mag_batch_create: mesh %d is missing, has no row-block plan, or uses a "
                      "non-standard curl table", i);
            return fail(MAG_E_ARG);
        }
        BatchInstance bi{};
        bi.m = m->elems();
        bi.rp = m->rows();
        bi.nu = d_nu[i];
        bi.sigma = d_sigma ? d_sigma[i] : nullptr;
        bi.val_ref = m->qp.val_ref;
        bi.second = m->second;
        bi.nq = m->qp.nq;
        for (int q = 0; q < m->qp.nq; q++) bi.qw[q] = m->qp.qw[q];
        bi.nq4 = (m->qp.nq == 4 && m->qp.uniform_w) ? 1 : 0;
        bi.omega = omega[i];
        bi.vals = d_vals[i];
        b->st.inst_host.push_back(bi);
        b->st.tile_in.push_back(TileComplexInput{&m->tile, m->elems(), m->qp, d_nu[i], bi.sigma, omega[i],
                                                 d_vals[i], m->status});
        b->st.inst_ne.push_back(m->ne);
        b->st.block_row256.push_back(m->rowblock.block_row);
        b->st.nblocks256.push_back(m->rowblock.nblocks);
        RowBlockPlan p128;
        int rc = build_rowblock_plan(m->rows(), &p128, s, 128);
        if (rc != MAG_OK) return fail(rc);
        b->st.owned.push_back(p128.block_row);
        b->st.block_row128.push_back(p128.block_row);
        b->st.nblocks128.push_back(p128.nblocks);
    }
    int rc = batch_build(&b->st, s);
    if (rc != MAG_OK) return fail(rc);
    // autotune: time every variant on these inputs, keep the fastest
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return fail(MAG_E_CUDA);
    double best = 1e300;
    for (int v = 0; v < batch_num_variants(); v++) {
        b->times[v] = -1.0;  // not available for these meshes
        if (!batch_variant_available(b->st, v)) continue;
        rc = batch_launch(b->st, v, s);  // warm-up
        if (rc != MAG_OK) break;
        cudaEventRecord(e0, s);
        for (int r = 0; r < 3; r++) batch_launch(b->st, v, s);
        cudaEventRecord(e1, s);
        if (cudaEventSynchronize(e1) != cudaSuccess) {
            rc = MAG_E_CUDA;
            break;
        }
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        b->times[v] = ms / 3.0;
        if (b->times[v] < best) {
            best = b->times[v];
            b->chosen = v;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != MAG_OK) return fail(rc);
    rc = capture_batch(b);
    if (rc != MAG_OK) return fail(rc);
    *out = b;
    return MAG_OK;
}

int mag_batch_select(mag_batch *b, int variant) {
    if (!b || variant < 0 || variant >= batch_num_variants()) {
        set_error("mag_batch_select: bad arguments");
        return MAG_E_ARG;
    }
    if (!batch_variant_available(b->st, variant)) {
        set_error("mag_batch_select: variant %d is not available for these meshes", variant);
        return MAG_E_UNSUPPORTED;
    }
    b->chosen = variant;
    return capture_batch(b);
}

int mag_batch_assemble(mag_batch *b, void *stream) {
    if (!b || !b->exec) {
        set_error("mag_batch_assemble: bad handle");
        return MAG_E_ARG;
    }
    MAG_CUDA_TRY(cudaGraphLaunch(b->exec, (cudaStream_t)stream));
    return MAG_OK;
}

int mag_batch_tuning(const mag_batch *b, int *chosen, double *times_ms, char *name, int name_len) {
    if (!b) {
        set_error("mag_batch_tuning: bad handle");
        return MAG_E_ARG;
    }
    if (chosen) *chosen = b->chosen;
    if (times_ms)
        for (int v = 0; v < batch_num_variants(); v++) times_ms[v] = b->times[v];
    if (name && name_len > 0) {
        std::strncpy(name, batch_variant_name(b->chosen), name_len - 1);
        name[name_len - 1] = 0;
    }
    return MAG_OK;
}

int mag_batch_destroy(mag_batch *b) {
    destroy_batch(b);
    return MAG_OK;
}

// ---- reluctivity predictor MLP --------------------------------------------------------

}  // extern "C"

struct mag_mlp {
    float *params = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr, *partial = nullptr;
    __nv_bfloat16 *ops = nullptr;
    int *err = nullptr;
    int grid = 0, step = 0;
    long long spin_limit = 0;
};

namespace {
void destroy_mlp(mag_mlp *n) {
    if (!n) return;
    void *p[] = {n->params, n->grad, n->m, n->v, n->partial, n->ops, n->err};
    for (void *q : p)
        if (q) cudaFree(q);
    delete n;
}
int mlp_grid(int64_t n, int cap) {
    int64_t tiles = (n + 127) / 128;
    return (int)(tiles < cap ? (tiles < 1 ? 1 : tiles) : cap);
}
}  // namespace

extern "C" {

int mag_mlp_num_params(void) { return kMlpParams; }

int mag_mlp_create(const float *init_params, mag_mlp **out) {
    if (!init_params || !out) {
        set_error("mag_mlp_create: bad arguments");
        return MAG_E_ARG;
    }
    *out = nullptr;
    mag_mlp *n = new (std::nothrow) mag_mlp();
    if (!n) return MAG_E_NOMEM;
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    n->grid = 2 * (nsm > 0 ? nsm : 1);
    size_t pb = (size_t)kMlpParams * sizeof(float);
    if (cudaMalloc(&n->params, pb) != cudaSuccess || cudaMalloc(&n->grad, pb) != cudaSuccess ||
        cudaMalloc(&n->m, pb) != cudaSuccess || cudaMalloc(&n->v, pb) != cudaSuccess ||
        cudaMalloc(&n->partial, pb * n->grid) != cudaSuccess ||
        cudaMalloc(&n->ops, (size_t)kMlpOperandElems * sizeof(__nv_bfloat16)) != cudaSuccess ||
        cudaMalloc(&n->err, sizeof(int)) != cudaSuccess) {
        destroy_mlp(n);
        set_error("mag_mlp_create: out of device memory");
        return MAG_E_NOMEM;
    }
    cudaMemcpy(n->params, init_params, pb, cudaMemcpyHostToDevice);
    cudaMemset(n->m, 0, pb);
    cudaMemset(n->v, 0, pb);
    cudaMemset(n->err, 0, sizeof(int));
    if (mlp_pack(n->params, n->ops, nullptr) != MAG_OK || cudaDeviceSynchronize() != cudaSuccess) {
        destroy_mlp(n);
        set_error("mag_mlp_create: CUDA error");
        return MAG_E_CUDA;
    }
    *out = n;
    return MAG_OK;
}

int mag_mlp_destroy(mag_mlp *n) {
    destroy_mlp(n);
    return MAG_OK;
}

int mag_mlp_get_params(const mag_mlp *n, float *host) {
    if (!n || !host) return MAG_E_ARG;
    MAG_CUDA_TRY(cudaMemcpy(host, n->params, (size_t)kMlpParams * sizeof(float), cudaMemcpyDeviceToHost));
    return MAG_OK;
}

int mag_mlp_set_params(mag_mlp *n, const float *host) {
    if (!n || !host) return MAG_E_ARG;
    MAG_CUDA_TRY(cudaMemcpy(n->params, host, (size_t)kMlpParams * sizeof(float), cudaMemcpyHostToDevice));
    MAG_TRY(mlp_pack(n->params, n->ops, nullptr));
    MAG_CUDA_TRY(cudaDeviceSynchronize());
    return MAG_OK;
}

int mag_mlp_forward(mag_mlp *n, const float *d_feats, int64_t rows, float *d_y, float *d_z, void *stream) {
    if (!n || !d_feats || rows <= 0 || !d_y || ((uintptr_t)d_feats & 15)) {
        set_error("mag_mlp_forward: bad arguments");
        return MAG_E_ARG;
    }
    MlpForwardArgs a{d_feats, rows, n->params, n->ops, d_y, d_z, nullptr, nullptr, 0, 0, 0, 0, n->err,
                     n->spin_limit};
    return mlp_forward(a, mlp_grid(rows, 1 << 30), (cudaStream_t)stream);
}

int mag_mlp_predict_nu(mag_mlp *n, const float *d_feats, int64_t rows, const int32_t *d_rows, double y_scale,
                       double y_shift, double nu_min, double nu_max, double *d_nu, void *stream) {
    if (!n || !d_feats || rows <= 0 || !d_nu || !(nu_min > 0) || !(nu_max >= nu_min) || ((uintptr_t)d_feats & 15)) {
        set_error("mag_mlp_predict_nu: bad arguments");
        return MAG_E_ARG;
    }
    MlpForwardArgs a{d_feats, rows, n->params, n->ops, nullptr, nullptr, d_nu, d_rows, y_scale, y_shift,
                     nu_min, nu_max, n->err, n->spin_limit};
    return mlp_forward(a, mlp_grid(rows, 1 << 30), (cudaStream_t)stream);
}

int mag_mlp_gradient(mag_mlp *n, const float *d_feats, const float *d_target, int64_t rows, float loss_scale,
                     float *d_y, float *d_z, float *d_grad, void *stream) {
    if (!n || !d_feats || !d_target || rows <= 0 || !d_y || !d_z || ((uintptr_t)d_feats & 15)) {
        set_error("mag_mlp_gradient: bad arguments");
        return MAG_E_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    MlpForwardArgs fa{d_feats, rows, n->params, n->ops, d_y, d_z, nullptr, nullptr, 0, 0, 0, 0, n->err,
                      n->spin_limit};
    MAG_TRY(mlp_forward(fa, mlp_grid(rows, 1 << 30), s));
    MlpBackwardArgs ba{d_feats, d_z, d_y, d_target, rows, loss_scale, n->params, n->ops, n->partial,
                       d_grad ? d_grad : n->grad, n->err, n->spin_limit};
    return mlp_backward(ba, mlp_grid(rows, n->grid), s);
}

int mag_mlp_train_step(mag_mlp *n, const float *d_feats, const float *d_target, int64_t rows, float lr,
                       float *d_y, float *d_z, void *stream) {
    MAG_TRY(mag_mlp_gradient(n, d_feats, d_target, rows, 2.0f / (float)rows, d_y, d_z, nullptr, stream));
    cudaStream_t s = (cudaStream_t)stream;
    n->step++;
    MAG_TRY(mlp_adam(n->params, n->grad, n->m, n->v, lr, 0.9f, 0.999f, 1e-8f, n->step, s));
    return mlp_pack(n->params, n->ops, s);
}

int mag_mlp_train_epoch(mag_mlp *n, const float *d_feats, const float *d_target, int64_t rows,
                        const int64_t *d_perm, int64_t batch, float lr, float *d_xb, float *d_tb, float *d_y,
                        float *d_z, float *d_loss, void *stream) {
    if (!n || !d_feats || !d_target || !d_perm || rows <= 0 || batch <= 0 || !d_xb || !d_tb || !d_y || !d_z ||
        ((uintptr_t)d_feats & 15) || ((uintptr_t)d_xb & 15)) {
        set_error("mag_mlp_train_epoch: bad arguments");
        return MAG_E_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    for (int64_t off = 0; off + batch <= rows; off += batch) {
        MAG_TRY(mlp_gather(d_feats, d_target, d_perm, off, batch, d_xb, d_tb, s));
        MAG_TRY(mag_mlp_train_step(n, d_xb, d_tb, batch, lr, d_y, d_z, stream));
        if (d_loss) MAG_TRY(mlp_sqerr(d_y, d_tb, batch, d_loss, s));
    }
    return MAG_OK;
}

int mag_mlp_check(mag_mlp *n, void *stream) {
    if (!n) return MAG_E_ARG;
    int h = 0;
    cudaStream_t s = (cudaStream_t)stream;
    MAG_CUDA_TRY(cudaMemcpyAsync(&h, n->err, sizeof(int), cudaMemcpyDeviceToHost, s));
    MAG_CUDA_TRY(cudaStreamSynchronize(s));
    if (h) {
        // reported once: the word is cleared so that later calls start clean
        MAG_CUDA_TRY(cudaMemsetAsync(n->err, 0, sizeof(int), s));
        MAG_CUDA_TRY(cudaStreamSynchronize(s));
        set_error("an MLP kernel's bounded wait on its tensor-core completion gave up");
        return MAG_E_TIMEOUT;
    }
    return MAG_OK;
}

int mag_mlp_set_spin_limit(mag_mlp *n, int64_t polls) {
    if (!n || polls < 0) {
        set_error("mag_mlp_set_spin_limit: bad arguments");
        return MAG_E_ARG;
    }
    n->spin_limit = (long long)polls;
    return MAG_OK;
}

// ---- sparse algebra ---------------------------------------------------------------

int mag_csr_spmv(int64_t n, const int64_t *rp, const int32_t *ci, const double *v, const double *x, double *y,
                 void *stream) {
    if (n <= 0 || !rp || !ci || !v || !x || !y) {
        set_error("mag_csr_spmv: bad arguments");
        return MAG_E_ARG;
    }
    MAG_TRY(csr_spmv(n, rp, ci, v, x, y, (cudaStream_t)stream));
    return MAG_OK;
}

int mag_csr_apply_dirichlet(int64_t n, const int64_t *rp, const int32_t *ci, double *v, const uint8_t *fixed,
                            double *rhs, void *stream) {
    if (n <= 0 || !rp || !ci || !v || !fixed) {
        set_error("mag_csr_apply_dirichlet: bad arguments");
        return MAG_E_ARG;
    }
    MAG_TRY(csr_dirichlet(n, rp, ci, v, fixed, rhs, (cudaStream_t)stream));
    return MAG_OK;
}

}  // extern "C"

struct mag_pcg {
    PcgSolver *s = nullptr;
};

extern "C" {

int mag_pcg_create(int64_t n, mag_pcg **out) {
    if (n <= 0 || !out) {
        set_error("mag_pcg_create: bad arguments");
        return MAG_E_ARG;
    }
    *out = nullptr;
    mag_pcg *p = new (std::nothrow) mag_pcg();
    if (!p) return MAG_E_NOMEM;
    if (pcg_create(n, &p->s) != MAG_OK) {
        delete p;
        set_error("mag_pcg_create: out of device memory");
        return MAG_E_NOMEM;
    }
    *out = p;
    return MAG_OK;
}

int mag_pcg_destroy(mag_pcg *p) {
    if (p) {
        pcg_destroy(p->s);
        delete p;
    }
    return MAG_OK;
}

int mag_pcg_set_aux(mag_pcg *p, int64_t ni, const int64_t *g_rp, const int32_t *g_ci, const double *g_v,
                    const int64_t *gt_rp, const int32_t *gt_ci, const double *gt_v, const double *dn_inv) {
    if (!p || ni < 0 || (ni > 0 && (!g_rp || !g_ci || !g_v || !gt_rp || !gt_ci || !gt_v || !dn_inv))) {
        set_error("mag_pcg_set_aux: bad arguments");
        return MAG_E_ARG;
    }
    int rc = pcg_set_aux(p->s, ni, g_rp, g_ci, g_v, gt_rp, gt_ci, gt_v, dn_inv);
    if (rc != MAG_OK) set_error("mag_pcg_set_aux: out of device memory");
    return rc;
}

int mag_pcg_solve(mag_pcg *p, const int64_t *rp, const int32_t *ci, const double *v, const double *b, double *x,
                  double rtol, int max_iter, int *iters, double *relres, int *status, void *stream) {
    if (!p || !rp || !ci || !v || !b || !x || !(rtol >= 0) || max_iter <= 0) {
        set_error("mag_pcg_solve: bad arguments");
        return MAG_E_ARG;
    }
    return pcg_solve(p->s, rp, ci, v, b, x, rtol, max_iter, iters, relres, status, (cudaStream_t)stream);
}

// ---- MEX-compatible entry points ------------------------------------------------

namespace {

// ---- host <-> device copies of the MEX entry points ---------------------------------
// The MEX arrays are pageable host memory. cudaMemcpy to or from pageable memory passes
// through a small driver buffer; a large copy goes faster through two pinned chunks: the
// DMA of one chunk overlaps the host threads' copy of the other to or from the caller's
// array (which also touches its pages in parallel).
constexpr size_t kStageChunk = size_t(32) << 20;
constexpr size_t kStageMin = size_t(4) << 20;  // smaller copies go direct

struct PinnedStage {
    void *buf[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    bool tried = false;
};
PinnedStage g_stage;  // used under g_mex_mu

bool stage_ready() {
    if (!g_stage.tried) {
        g_stage.tried = true;
        for (int i = 0; i < 2; i++)
            if (cudaHostAlloc(&g_stage.buf[i], kStageChunk, cudaHostAllocDefault) != cudaSuccess ||
                cudaEventCreateWithFlags(&g_stage.ev[i], cudaEventDisableTiming) != cudaSuccess) {
                cudaGetLastError();
                for (int k = 0; k < 2; k++) {
                    if (g_stage.buf[k]) cudaFreeHost(g_stage.buf[k]);
                    if (g_stage.ev[k]) cudaEventDestroy(g_stage.ev[k]);
                    g_stage.buf[k] = nullptr;
                    g_stage.ev[k] = nullptr;
                }
                return false;
            }
    }
    return g_stage.buf[0] != nullptr;
}

void host_copy(void *dst, const void *src, size_t bytes) {
    constexpr size_t kPiece = size_t(1) << 20;
    const int64_t n = (int64_t)((bytes + kPiece - 1) / kPiece);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; k++) {
        const size_t o = (size_t)k * kPiece, len = bytes - o < kPiece ? bytes - o : kPiece;
        std::memcpy(static_cast<char *>(dst) + o, static_cast<const char *>(src) + o, len);
    }
}

// Device -> pageable host, synchronous on return.
int copy_to_host(void *dst, const void *src, size_t bytes, cudaStream_t s) {
    if (bytes < kStageMin || !stage_ready()) {
        MAG_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
        MAG_CUDA_TRY(cudaStreamSynchronize(s));
        return MAG_OK;
    }
    const size_t n = (bytes + kStageChunk - 1) / kStageChunk;
    for (size_t i = 0; i <= n; i++) {
        if (i < n) {
            const size_t o = i * kStageChunk, len = bytes - o < kStageChunk ? bytes - o : kStageChunk;
            MAG_CUDA_TRY(cudaMemcpyAsync(g_stage.buf[i % 2], static_cast<const char *>(src) + o, len,
                                         cudaMemcpyDeviceToHost, s));
            MAG_CUDA_TRY(cudaEventRecord(g_stage.ev[i % 2], s));
        }
        if (i > 0) {
            const size_t j = i - 1, o = j * kStageChunk, len = bytes - o < kStageChunk ? bytes - o : kStageChunk;
            MAG_CUDA_TRY(cudaEventSynchronize(g_stage.ev[j % 2]));
            host_copy(static_cast<char *>(dst) + o, g_stage.buf[j % 2], len);
        }
    }
    return MAG_OK;
}

// Pageable host -> device; the source may be reused when this returns.
int copy_to_device(void *dst, const void *src, size_t bytes, cudaStream_t s) {
    if (bytes < kStageMin || !stage_ready()) {
        MAG_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
        return MAG_OK;
    }
    const size_t n = (bytes + kStageChunk - 1) / kStageChunk;
    for (size_t i = 0; i < n; i++) {
        const size_t o = i * kStageChunk, len = bytes - o < kStageChunk ? bytes - o : kStageChunk;
        if (i >= 2) MAG_CUDA_TRY(cudaEventSynchronize(g_stage.ev[i % 2]));  // chunk i-2 has left the buffer
        host_copy(g_stage.buf[i % 2], static_cast<const char *>(src) + o, len);
        MAG_CUDA_TRY(cudaMemcpyAsync(static_cast<char *>(dst) + o, g_stage.buf[i % 2], len,
                                     cudaMemcpyHostToDevice, s));
        MAG_CUDA_TRY(cudaEventRecord(g_stage.ev[i % 2], s));
    }
    for (int k = 0; k < 2; k++) MAG_CUDA_TRY(cudaEventSynchronize(g_stage.ev[k]));
    return MAG_OK;
}

// A mesh given in the reference's MEX layout, converted to the device layout. The MEX
// entry points keep the last kMexCacheEntries of them (per device), keyed by the sizes
// and a content hash of P, T, Dofs and Signs, so that the Newton loop's calls with the
// same mesh (Assembler.m:199-202 every iteration and line-search step) neither upload
// nor convert nor plan it again; an array changed in place, or a new array at a reused
// address, hashes differently and is converted afresh. Tags are hashed separately and
// reconverted when they change.
struct MexMesh {
    Dev xyz, tet, dofs, tags, signs, scratch;
    ElemData ed{};
    int dev = -1;
    int64_t Nn = 0, Ne = 0;
    uint64_t h0 = 0, h1 = 0;       // content hash of P, T, Dofs, Signs
    int has_tags = 0;
    uint64_t t0 = 0, t1 = 0;       // content hash of Tags
    int max_tag = 0;
    int max_dof = 0;               // largest 1-based dof (0 = missing) the element arrays use
    PatternBuffers pat;            // CSR pattern of the sparse-returning entry points
    int64_t pat_ndof = -1;
    uint64_t stamp = 0;
    explicit MexMesh(cudaStream_t s) : xyz(s), tet(s), dofs(s), tags(s), signs(s), scratch(s) {}
    ~MexMesh() { free_pattern(&pat, nullptr); }
};

constexpr size_t kMexCacheEntries = 2;
std::mutex g_mex_mu;  // held for the whole of every MEX entry point (the cached scratch is shared)
std::vector<std::unique_ptr<MexMesh>> g_mex_cache;
uint64_t g_mex_clock = 0;

inline uint64_t mix64(uint64_t x) {
    x ^= x >> 33;
    x *= 0xFF51AFD7ED558CCDull;
    x ^= x >> 33;
    x *= 0xC4CEB9FE1A85EC53ull;
    x ^= x >> 33;
    return x;
}

// Two-lane 64-bit content hash of a host array, folded into (h0, h1); 1 MiB chunks
// are hashed on the host threads and combined in order.
void hash_host(const void *data, size_t bytes, uint64_t &h0, uint64_t &h1) {
    constexpr size_t C = size_t(1) << 20;
    const size_t n = (bytes + C - 1) / C;
    std::vector<uint64_t> a(n), b(n);
    const unsigned char *c = static_cast<const unsigned char *>(data);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < (int64_t)n; k++) {
        const size_t o = (size_t)k * C, len = bytes - o < C ? bytes - o : C;
        uint64_t x = 0x243F6A8885A308D3ull + (uint64_t)k, y = 0x13198A2E03707344ull ^ (uint64_t)k;
        size_t i = 0;
        for (; i + 8 <= len; i += 8) {
            uint64_t v;
            std::memcpy(&v, c + o + i, 8);
            x = (x ^ v) * 0x9E3779B97F4A7C15ull;
            x ^= x >> 29;
            y = (y + v) * 0xC2B2AE3D27D4EB4Full;
            y ^= y >> 31;
        }
        for (; i < len; i++) {
            x = (x ^ c[o + i]) * 0x9E3779B97F4A7C15ull;
            y = (y + c[o + i]) * 0xC2B2AE3D27D4EB4Full;
        }
        a[k] = mix64(x);
        b[k] = mix64(y ^ len);
    }
    for (size_t k = 0; k < n; k++) {
        h0 = mix64(h0 ^ a[k]) + k;
        h1 = mix64(h1 + b[k]) ^ k;
    }
    h0 = mix64(h0 ^ bytes);
    h1 = mix64(h1 + bytes);
}

// Upload the reference's double arrays (P, T, Dofs, Signs) and convert them.
int mex_convert(const double *P, int64_t Nn, const double *T, int64_t Ne, const double *Dofs,
                const double *Signs, MexMesh &mm, cudaStream_t s) {
    Dev err(s), mxd(s), Pd(s), Td(s), Dd(s), Sd(s);
    MAG_CUDA_TRY(err.alloc(4));
    MAG_CUDA_TRY(mxd.alloc(4));
    MAG_CUDA_TRY(cudaMemsetAsync(err.p, 0, 4, s));
    MAG_CUDA_TRY(cudaMemsetAsync(mxd.p, 0, 4, s));
    MAG_CUDA_TRY(Pd.alloc(Nn * 24));
    MAG_CUDA_TRY(Td.alloc(Ne * 32));
    MAG_CUDA_TRY(Dd.alloc(Ne * 48));
    MAG_CUDA_TRY(Sd.alloc(Ne * 48));
    MAG_CUDA_TRY(mm.xyz.alloc(Nn * sizeof(double4)));
    MAG_CUDA_TRY(mm.tet.alloc(Ne * 16));
    MAG_CUDA_TRY(mm.dofs.alloc(Ne * 24));
    MAG_CUDA_TRY(mm.tags.alloc(Ne));
    MAG_CUDA_TRY(mm.signs.alloc(Ne));
    MAG_TRY(copy_to_device(Pd.p, P, Nn * 24, s));
    MAG_TRY(copy_to_device(Td.p, T, Ne * 32, s));
    MAG_TRY(copy_to_device(Dd.p, Dofs, Ne * 48, s));
    MAG_TRY(copy_to_device(Sd.p, Signs, Ne * 48, s));
    k_pack_xyz<<<grid(Nn), kB, 0, s>>>(Pd.as<double>(), Nn, mm.xyz.as<double4>(), err.as<int>());
    k_index_from_double<<<grid(4 * Ne), kB, 0, s>>>(Td.as<double>(), 4 * Ne, mm.tet.as<int32_t>(), Nn, 0,
                                                    err.as<int>());
    k_index_from_double<<<grid(6 * Ne), kB, 0, s>>>(Dd.as<double>(), 6 * Ne, mm.dofs.as<int32_t>(),
                                                    (int64_t)INT32_MAX, 1, err.as<int>(), mxd.as<int>());
    k_pack_signs_f64<<<grid(Ne), kB, 0, s>>>(Sd.as<double>(), Ne, mm.signs.as<uint8_t>(), err.as<int>());
    MAG_CUDA_TRY(cudaMemsetAsync(mm.tags.p, 1, Ne, s));
    int h = 0;
    MAG_TRY(sync_flag(err.as<int>(), s, &h));
    if (h) {
        set_error("mex: index or sign out of range (nodes 1..Nn, dofs 0..numel(SolA), signs +-1)");
        return MAG_E_RANGE;
    }
    MAG_TRY(sync_flag(mxd.as<int>(), s, &mm.max_dof));
    mm.ed = ElemData{mm.xyz.as<double4>(), mm.tet.as<int4>(), mm.dofs.as<int32_t>(),
                     mm.tags.as<uint8_t>(), mm.signs.as<uint8_t>(), Ne};
    MAG_CUDA_TRY(mm.scratch.alloc((size_t)Ne * kScratchPerElem * 8));
    return MAG_OK;
}

int mex_set_tags(MexMesh &mm, const double *Tags, cudaStream_t s) {
    Dev err(s), mx(s), Gd(s);
    MAG_CUDA_TRY(err.alloc(4));
    MAG_CUDA_TRY(mx.alloc(4));
    MAG_CUDA_TRY(Gd.alloc(mm.Ne * 8));
    MAG_CUDA_TRY(cudaMemsetAsync(err.p, 0, 4, s));
    MAG_CUDA_TRY(cudaMemsetAsync(mx.p, 0, 4, s));
    MAG_TRY(copy_to_device(Gd.p, Tags, mm.Ne * 8, s));
    k_pack_tags_f64<<<grid(mm.Ne), kB, 0, s>>>(Gd.as<double>(), mm.Ne, mm.tags.as<uint8_t>(), mx.as<int>(),
                                               err.as<int>());
    int h = 0;
    MAG_TRY(sync_flag(err.as<int>(), s, &h));
    mm.has_tags = 0;
    if (h) {
        set_error("mex: tag out of range (tags 1..255)");
        return MAG_E_RANGE;
    }
    MAG_TRY(sync_flag(mx.as<int>(), s, &mm.max_tag));
    mm.has_tags = 1;
    return MAG_OK;
}

// The device mesh for these MEX arrays: from the cache, or converted and cached.
// dof_limit: every dof must be <= it (numel(SolA) for the Jacobian); Tags may be NULL.
// The caller holds g_mex_mu.
int mex_mesh(const double *P, int64_t Nn, const double *T, int64_t Ne, const double *Dofs,
             const double *Signs, const double *Tags, int64_t dof_limit, MexMesh **out, int *max_tag,
             cudaStream_t s) {
    *out = nullptr;
    if (!P || !T || !Dofs || !Signs || Nn <= 0 || Ne <= 0) {
        set_error("mex: bad arguments");
        return MAG_E_ARG;
    }
    int dev = 0;
    MAG_CUDA_TRY(cudaGetDevice(&dev));
    uint64_t h0 = 0x6A09E667F3BCC908ull, h1 = 0xBB67AE8584CAA73Bull;
    hash_host(P, (size_t)Nn * 24, h0, h1);
    hash_host(T, (size_t)Ne * 32, h0, h1);
    hash_host(Dofs, (size_t)Ne * 48, h0, h1);
    hash_host(Signs, (size_t)Ne * 48, h0, h1);
    MexMesh *mm = nullptr;
    for (auto &e : g_mex_cache)
        if (e->dev == dev && e->Nn == Nn && e->Ne == Ne && e->h0 == h0 && e->h1 == h1) mm = e.get();
    if (!mm) {
        std::unique_ptr<MexMesh> fresh(new (std::nothrow) MexMesh(s));
        if (!fresh) return MAG_E_NOMEM;
        if (g_mex_cache.size() >= kMexCacheEntries) {  // evict the least recently used
            size_t lru = 0;
            for (size_t i = 1; i < g_mex_cache.size(); i++)
                if (g_mex_cache[i]->stamp < g_mex_cache[lru]->stamp) lru = i;
            g_mex_cache.erase(g_mex_cache.begin() + (long)lru);
        }
        MAG_TRY(mex_convert(P, Nn, T, Ne, Dofs, Signs, *fresh, s));
        fresh->dev = dev;
        fresh->Nn = Nn;
        fresh->Ne = Ne;
        fresh->h0 = h0;
        fresh->h1 = h1;
        mm = fresh.get();
        g_mex_cache.push_back(std::move(fresh));
    }
    mm->stamp = ++g_mex_clock;
    if (Tags) {
        uint64_t t0 = 0x3C6EF372FE94F82Bull, t1 = 0xA54FF53A5F1D36F1ull;
        hash_host(Tags, (size_t)Ne * 8, t0, t1);
        if (!mm->has_tags || mm->t0 != t0 || mm->t1 != t1) {
            MAG_TRY(mex_set_tags(*mm, Tags, s));
            mm->t0 = t0;
            mm->t1 = t1;
        }
    }
    if (mm->max_dof > dof_limit) {
        set_error("mex: dof %d out of range (dofs 0..%lld)", mm->max_dof, (long long)dof_limit);
        return MAG_E_RANGE;
    }
    *max_tag = Tags ? mm->max_tag : 0;
    *out = mm;
    return MAG_OK;
}

// The CSR pattern of a cached MEX mesh with ndof rows (built on first use).
int mex_pattern(MexMesh &mm, int64_t ndof, cudaStream_t s) {
    if (mm.pat_ndof == ndof) return MAG_OK;
    free_pattern(&mm.pat, s);
    mm.pat = PatternBuffers{};
    mm.pat_ndof = -1;
    MAG_TRY(build_pattern(mm.dofs.as<int32_t>(), mm.Ne, ndof, &mm.pat, s));
    mm.pat_ndof = ndof;
    return MAG_OK;
}

int mex_download(MexMesh &mm, int64_t Ne, int calcj, double *I, double *J, double *V, double *Ridx,
                 double *Rval, cudaStream_t s) {
    Dev out(s);
    int64_t nk = calcj ? 36 * Ne : 0, nr = Ridx ? 6 * Ne : 0;
    MAG_CUDA_TRY(out.alloc((3 * nk + 2 * nr) * 8));
    double *dI = out.as<double>(), *dJ = dI + nk, *dV = dJ + nk, *dRi = dV + nk, *dRv = dRi + nr;
    MAG_TRY(launch_to_triplets(mm.scratch.as<double>(), mm.dofs.as<int32_t>(), Ne, calcj, dI, dJ, dV,
                               Ridx ? dRi : nullptr, Ridx ? dRv : nullptr, s));
    if (nk) {
        MAG_TRY(copy_to_host(I, dI, nk * 8, s));
        MAG_TRY(copy_to_host(J, dJ, nk * 8, s));
        MAG_TRY(copy_to_host(V, dV, nk * 8, s));
    }
    if (nr) {
        MAG_TRY(copy_to_host(Ridx, dRi, nr * 8, s));
        MAG_TRY(copy_to_host(Rval, dRv, nr * 8, s));
    }
    MAG_CUDA_TRY(cudaStreamSynchronize(s));
    return MAG_OK;
}

// The Jacobian element phase of the MEX entry points: upload, materials, quadrature,
// element blocks and residual entries into mm.scratch.
struct MexJacobian {
    MexMesh *mm = nullptr;
    MaterialStore ms{};
    double *q = nullptr;
    Dev sol;
    explicit MexJacobian(cudaStream_t s) : sol(s) {}
    ~MexJacobian() {
        if (ms.mem) cudaFree(ms.mem);
        if (q) cudaFree(q);
    }
    int run(const double *P, int64_t Nn, const double *T, int64_t Ne, const double *Dofs, const double *Signs,
            const double *Tags, const double *SolA, int64_t Ndof, const double *Qw, int nq,
            const double *CurlRef, const double *lin, const double *isNon, const double *maxB, int nmat,
            const double *brk, int nbrk, const double *coe, int ncoe, const double *start, const double *cnt,
            const double *coeStart, int calc_j, cudaStream_t s) {
        int max_tag = 0;
        MAG_TRY(mex_mesh(P, Nn, T, Ne, Dofs, Signs, Tags, Ndof, &mm, &max_tag, s));
        MAG_TRY(upload_materials(lin, isNon, maxB, nmat, brk, nbrk, coe, ncoe, start, cnt, coeStart, &ms, s));
        if (nmat < max_tag) {
            set_error("mag_mex_jacobian: tag %d has no material entry", max_tag);
            return MAG_E_RANGE;
        }
        QuadParams qp{};
        // the Jacobian kernel takes no basis values; reuse the curl table for the slot
        MAG_TRY(make_quad(Qw, nq, CurlRef, CurlRef, &qp, &q, s));
        // dofs must index SolA
        MAG_CUDA_TRY(sol.alloc(Ndof * 8));
        MAG_TRY(copy_to_device(sol.p, SolA, Ndof * 8, s));
        return launch_jacobian_elems(mm->ed, sol.as<double>(), qp, ms.mp, calc_j, mm->scratch.as<double>(), s);
    }
};

}  // namespace

int mag_mex_cache_clear(void) {
    std::lock_guard<std::mutex> lk(g_mex_mu);
    g_mex_cache.clear();
    MAG_CUDA_TRY(cudaDeviceSynchronize());
    return MAG_OK;
}

int mag_mex_jacobian(const double *P, int64_t Nn, const double *T, int64_t Ne, const double *Dofs,
                     const double *Signs, const double *Tags, const double *SolA, int64_t Ndof,
                     const double *Qw, int nq, const double *CurlRef, const double *lin,
                     const double *isNon, const double *maxB, int nmat, const double *brk, int nbrk,
                     const double *coe, int ncoe, const double *start, const double *cnt,
                     const double *coeStart, int calc_j, double *I, double *J, double *V,
                     double *R_idx, double *R_val) {
    cudaStream_t s = nullptr;
    if (Ne == 0) return MAG_OK;  // the gateway returns empty triplets for an empty mesh
    if (!Tags || !SolA || Ndof <= 0 || !R_idx || !R_val || (calc_j && (!I || !J || !V))) {
        set_error("mag_mex_jacobian: bad arguments");
        return MAG_E_ARG;
    }
    std::lock_guard<std::mutex> lk(g_mex_mu);
    MexJacobian mj(s);
    MAG_TRY(mj.run(P, Nn, T, Ne, Dofs, Signs, Tags, SolA, Ndof, Qw, nq, CurlRef, lin, isNon, maxB, nmat, brk,
                   nbrk, coe, ncoe, start, cnt, coeStart, calc_j, s));
    return mex_download(*mj.mm, Ne, calc_j, I, J, V, R_idx, R_val, s);
}

int mag_mex_curl_curl(const double *P, int64_t Nn, const double *T, int64_t Ne, const double *Dofs,
                      const double *Signs, const double *Nu, const double *Qw, int nq,
                      const double *CurlRef, double *I, double *J, double *V) {
    cudaStream_t s = nullptr;
    if (Ne == 0) return MAG_OK;  // the gateway returns empty triplets for an empty mesh
    if (!Nu || !I || !J || !V) {
        set_error("mag_mex_curl_curl: bad arguments");
        return MAG_E_ARG;
    }
    std::lock_guard<std::mutex> lk(g_mex_mu);
    MexMesh *mmp = nullptr;
    int max_tag = 0;
    MAG_TRY(mex_mesh(P, Nn, T, Ne, Dofs, Signs, nullptr, (int64_t)1 << 31, &mmp, &max_tag, s));
    MexMesh &mm = *mmp;
    QuadParams qp{};
    double *dq = nullptr;
    MAG_TRY(make_quad(Qw, nq, CurlRef, CurlRef, &qp, &dq, s));
    Dev nu(s);
    MAG_CUDA_TRY(nu.alloc(Ne * 8));
    MAG_CUDA_TRY(cudaMemcpyAsync(nu.p, Nu, Ne * 8, cudaMemcpyHostToDevice, s));
    int rc = launch_stiffness_elems(mm.ed, nu.as<double>(), qp, mm.scratch.as<double>(), s);
    if (rc == MAG_OK) rc = mex_download(mm, Ne, 1, I, J, V, nullptr, nullptr, s);
    cudaFree(dq);
    return rc;
}

int mag_mex_mass(const double *P, int64_t Nn, const double *T, int64_t Ne, const double *Dofs,
                 const double *Signs, const double *Coeffs, int64_t ncoeffs, const double *Qw, int nq,
                 const double *ValRef, double *I, double *J, double *V) {
    cudaStream_t s = nullptr;
    if (Ne == 0) return MAG_OK;  // the gateway returns empty triplets for an empty mesh
    if (!I || !J || !V) {
        set_error("mag_mex_mass: bad arguments");
        return MAG_E_ARG;
    }
    std::lock_guard<std::mutex> lk(g_mex_mu);
    MexMesh *mmp = nullptr;
    int max_tag = 0;
    MAG_TRY(mex_mesh(P, Nn, T, Ne, Dofs, Signs, nullptr, (int64_t)1 << 31, &mmp, &max_tag, s));
    MexMesh &mm = *mmp;
    QuadParams qp{};
    double *dq = nullptr;
    MAG_TRY(make_quad(Qw, nq, ValRef, ValRef, &qp, &dq, s));
    Dev sg(s);
    const double *dsig = nullptr;
    if (Coeffs && ncoeffs == Ne) {  // otherwise sigma = 1 (assemble_mass_kernel_mex.cpp:155)
        MAG_CUDA_TRY(sg.alloc(Ne * 8));
        MAG_CUDA_TRY(cudaMemcpyAsync(sg.p, Coeffs, Ne * 8, cudaMemcpyHostToDevice, s));
        dsig = sg.as<double>();
    }
    int rc = launch_mass_elems(mm.ed, dsig, qp, mm.scratch.as<double>(), s);
    if (rc == MAG_OK) rc = mex_download(mm, Ne, 1, I, J, V, nullptr, nullptr, s);
    cudaFree(dq);
    return rc;
}

}  // extern "C"

extern "C" {

int mag_mex_source(const double *P, int64_t Nn, const double *T, int64_t Ne, const double *Dofs,
                   const double *Signs, const double *Js, const double *Qw, int nq, const double *ValRef,
                   double *I, double *V) {
    cudaStream_t s = nullptr;
    if (Ne == 0) return MAG_OK;
    if (!Js || !I || !V) {
        set_error("mag_mex_source: bad arguments");
        return MAG_E_ARG;
    }
    std::lock_guard<std::mutex> lk(g_mex_mu);
    MexMesh *mmp = nullptr;
    int max_tag = 0;
    MAG_TRY(mex_mesh(P, Nn, T, Ne, Dofs, Signs, nullptr, (int64_t)1 << 31, &mmp, &max_tag, s));
    MexMesh &mm = *mmp;
    QuadParams qp{};
    double *dq = nullptr;
    MAG_TRY(make_quad(Qw, nq, ValRef, ValRef, &qp, &dq, s));
    Dev js(s), out(s);
    int rc = js.alloc(Ne * 24) == cudaSuccess && out.alloc(Ne * 96) == cudaSuccess ? MAG_OK : MAG_E_NOMEM;
    if (rc == MAG_OK && cudaMemcpyAsync(js.p, Js, Ne * 24, cudaMemcpyHostToDevice, s) != cudaSuccess) rc = MAG_E_CUDA;
    if (rc == MAG_OK) rc = launch_source_elems(mm.ed, js.as<double>(), qp, mm.scratch.as<double>(), s);
    double *dI = out.as<double>(), *dV = dI + 6 * Ne;
    if (rc == MAG_OK)
        rc = launch_to_triplets(mm.scratch.as<double>(), mm.dofs.as<int32_t>(), Ne, 0, nullptr, nullptr, nullptr,
                                dI, dV, s);
    if (rc == MAG_OK && (cudaMemcpyAsync(I, dI, Ne * 48, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                         cudaMemcpyAsync(V, dV, Ne * 48, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                         cudaStreamSynchronize(s) != cudaSuccess))
        rc = MAG_E_CUDA;
    cudaFree(dq);
    return rc;
}

int mag_mex_winding(const double *P, int64_t Nn, const double *T, int64_t Ne, const double *Dofs,
                    const double *Signs, const double *Tags, double CoilID, const double *DirField,
                    const double *UniDir, double Scale, const double *Qw, int nq, const double *ValRef, double *I,
                    double *V) {
    cudaStream_t s = nullptr;
    if (Ne == 0) return MAG_OK;
    if (!Tags || (!DirField && !UniDir) || !I || !V) {
        set_error("mag_mex_winding: bad arguments");
        return MAG_E_ARG;
    }
    std::lock_guard<std::mutex> lk(g_mex_mu);
    MexMesh *mmp = nullptr;
    int max_tag = 0;
    MAG_TRY(mex_mesh(P, Nn, T, Ne, Dofs, Signs, Tags, (int64_t)1 << 31, &mmp, &max_tag, s));
    MexMesh &mm = *mmp;
    QuadParams qp{};
    double *dq = nullptr;
    MAG_TRY(make_quad(Qw, nq, ValRef, ValRef, &qp, &dq, s));
    Dev field(s), out(s);
    int rc = out.alloc(Ne * 96) == cudaSuccess ? MAG_OK : MAG_E_NOMEM;
    if (rc == MAG_OK && DirField) {
        rc = field.alloc(Ne * 24) == cudaSuccess ? MAG_OK : MAG_E_NOMEM;
        if (rc == MAG_OK && cudaMemcpyAsync(field.p, DirField, Ne * 24, cudaMemcpyHostToDevice, s) != cudaSuccess)
            rc = MAG_E_CUDA;
    }
    const double zero[3] = {0.0, 0.0, 0.0};
    // (int)CoilID as the reference compares it; no tag of the mesh lies outside 1..255
    const int coil = (CoilID > -2147483648.0 && CoilID < 2147483648.0) ? (int)CoilID : -1;
    double *dI = out.as<double>(), *dV = dI + 6 * Ne;
    if (rc == MAG_OK)
        rc = launch_winding_elems(mm.ed, coil, DirField ? field.as<double>() : nullptr, UniDir ? UniDir : zero,
                                  Scale, qp, nullptr, dI, dV, s);
    if (rc == MAG_OK && (cudaMemcpyAsync(I, dI, Ne * 48, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                         cudaMemcpyAsync(V, dV, Ne * 48, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                         cudaStreamSynchronize(s) != cudaSuccess))
        rc = MAG_E_CUDA;
    cudaFree(dq);
    return rc;
}

}  // extern "C"

// ---- MATLAB sparse results of the MEX-compatible assemblies -----------------------

struct mag_sparse {
    int64_t n = 0, nnz = 0;
    int64_t *rp = nullptr;  // [n+1] column pointers
    int32_t *ci = nullptr;  // [nnz] row indices, ascending per column
    double *v = nullptr;    // [nnz]
};

namespace mag {
namespace {

// Transpose each element's 6x6 block in place (the residual slot stays). Summed by the
// row reduction, the transposed blocks give the CSR of V^T, which is the
// compressed-column storage of sparse(I, J, V): bit-exact also where the nonlinear
// term 2 dnu (B.C_i)(B.C_j), evaluated left to right, differs from its transpose in
// the last bit.
__global__ void k_transpose_blocks(double *__restrict__ scratch, int64_t ne) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= ne) return;
    double *b = scratch + e * kScratchPerElem;
#pragma unroll
    for (int i = 0; i < 6; i++)
#pragma unroll
        for (int j = i + 1; j < 6; j++) {
            const double t = b[i * kScratchStride + j];
            b[i * kScratchStride + j] = b[j * kScratchStride + i];
            b[j * kScratchStride + i] = t;
        }
}

__global__ void k_i32_to_u64(const int32_t *__restrict__ a, int64_t n, uint64_t *__restrict__ b) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) b[i] = (uint64_t)(uint32_t)a[i];
}

}  // namespace
}  // namespace mag

namespace {

void destroy_sparse(mag_sparse *sp) {
    if (!sp) return;
    if (sp->rp) cudaFree(sp->rp);
    if (sp->ci) cudaFree(sp->ci);
    if (sp->v) cudaFree(sp->v);
    delete sp;
}

int empty_sparse(int64_t ndof, mag_sparse **out) {
    mag_sparse *sp = new (std::nothrow) mag_sparse();
    if (!sp) return MAG_E_NOMEM;
    sp->n = ndof;
    if (cudaMalloc(&sp->rp, (ndof + 1) * 8) != cudaSuccess || cudaMemset(sp->rp, 0, (ndof + 1) * 8) != cudaSuccess) {
        destroy_sparse(sp);
        set_error("mex sparse: out of device memory");
        return MAG_E_NOMEM;
    }
    *out = sp;
    return MAG_OK;
}

// sparse(I, J, V, ndof, ndof) (and, when h_res is given, full(sparse(R_idx, 1, R_val, ndof, 1))
// into h_res) from the element blocks in mm.scratch: the mesh's CSR pattern, the
// fixed-order row reduction over transposed blocks, then MATLAB's storage rule
// (no explicit zeros). Missing dofs (0 in Dofs) contribute nothing, as the
// (I > 0) & (J > 0) filter of Assembler.m:37,52,71,205 drops them.
int mex_to_sparse(MexMesh &mm, int64_t Ne, int64_t ndof, bool with_matrix, double *h_res, mag_sparse **out,
                  cudaStream_t s) {
    MAG_TRY(mex_pattern(mm, ndof, s));
    const PatternBuffers &pat = mm.pat;
    const RowPlan rows{pat.row_ptr, pat.inc_ptr, pat.inc_elem, pat.inc_pos, ndof, pat.wide};
    Dev vals(s), rp64(s), res(s);
    if (with_matrix) {
        k_transpose_blocks<<<grid(Ne), kB, 0, s>>>(mm.scratch.as<double>(), Ne);
        MAG_CUDA_TRY(vals.alloc(pat.nnz * 8));
        MAG_CUDA_TRY(rp64.alloc((ndof + 1) * 8));
    }
    if (h_res) MAG_CUDA_TRY(res.alloc(ndof * 8));
    MAG_TRY(launch_rows_reduce(rows, pat.max_row, mm.scratch.as<double>(), with_matrix ? vals.as<double>() : nullptr,
                               h_res ? res.as<double>() : nullptr, s));
    if (h_res) {
        MAG_TRY(copy_to_host(h_res, res.p, ndof * 8, s));
        MAG_CUDA_TRY(cudaStreamSynchronize(s));
    }
    if (!with_matrix) return MAG_OK;
    k_i32_to_i64<<<grid(ndof + 1), kB, 0, s>>>(pat.row_ptr, ndof + 1, rp64.as<int64_t>());
    mag_sparse *sp = new (std::nothrow) mag_sparse();
    if (!sp) return MAG_E_NOMEM;
    sp->n = ndof;
    const size_t nz = pat.nnz > 0 ? (size_t)pat.nnz : 1;
    if (cudaMalloc(&sp->rp, (ndof + 1) * 8) != cudaSuccess || cudaMalloc(&sp->ci, nz * 4) != cudaSuccess ||
        cudaMalloc(&sp->v, nz * 8) != cudaSuccess) {
        destroy_sparse(sp);
        set_error("mex sparse: out of device memory");
        return MAG_E_NOMEM;
    }
    int rc = csr_drop_zeros(rp64.as<int64_t>(), pat.col_idx, vals.as<double>(), ndof, sp->rp, sp->ci, sp->v,
                            &sp->nnz, s);
    if (rc != MAG_OK) {
        destroy_sparse(sp);
        return rc;
    }
    *out = sp;
    return MAG_OK;
}

}  // namespace

extern "C" {

int mag_mex_jacobian_sparse(const double *P, int64_t Nn, const double *T, int64_t Ne, const double *Dofs,
                            const double *Signs, const double *Tags, const double *SolA, int64_t Ndof,
                            const double *Qw, int nq, const double *CurlRef, const double *lin,
                            const double *isNon, const double *maxB, int nmat, const double *brk, int nbrk,
                            const double *coe, int ncoe, const double *start, const double *cnt,
                            const double *coeStart, int calc_j, mag_sparse **J_out, double *R) {
    cudaStream_t s = nullptr;
    if (J_out) *J_out = nullptr;
    if (!SolA || Ndof <= 0 || !R || (calc_j && !J_out)) {
        set_error("mag_mex_jacobian_sparse: bad arguments");
        return MAG_E_ARG;
    }
    if (Ne == 0) {
        std::memset(R, 0, Ndof * 8);
        return calc_j ? empty_sparse(Ndof, J_out) : MAG_OK;
    }
    if (!Tags) {
        set_error("mag_mex_jacobian_sparse: bad arguments");
        return MAG_E_ARG;
    }
    std::lock_guard<std::mutex> lk(g_mex_mu);
    MexJacobian mj(s);
    MAG_TRY(mj.run(P, Nn, T, Ne, Dofs, Signs, Tags, SolA, Ndof, Qw, nq, CurlRef, lin, isNon, maxB, nmat, brk,
                   nbrk, coe, ncoe, start, cnt, coeStart, calc_j, s));
    return mex_to_sparse(*mj.mm, Ne, Ndof, calc_j != 0, R, J_out, s);
}

int mag_mex_curl_curl_sparse(const double *P, int64_t Nn, const double *T, int64_t Ne, const double *Dofs,
                             const double *Signs, const double *Nu, const double *Qw, int nq,
                             const double *CurlRef, int64_t Ndof, mag_sparse **out) {
    cudaStream_t s = nullptr;
    if (out) *out = nullptr;
    if (!out || Ndof <= 0 || (Ne > 0 && !Nu)) {
        set_error("mag_mex_curl_curl_sparse: bad arguments");
        return MAG_E_ARG;
    }
    if (Ne == 0) return empty_sparse(Ndof, out);
    std::lock_guard<std::mutex> lk(g_mex_mu);
    MexMesh *mmp = nullptr;
    int max_tag = 0;
    MAG_TRY(mex_mesh(P, Nn, T, Ne, Dofs, Signs, nullptr, Ndof, &mmp, &max_tag, s));
    MexMesh &mm = *mmp;
    QuadParams qp{};
    double *dq = nullptr;
    MAG_TRY(make_quad(Qw, nq, CurlRef, CurlRef, &qp, &dq, s));
    Dev nu(s);
    int rc = nu.alloc(Ne * 8) == cudaSuccess ? MAG_OK : MAG_E_NOMEM;
    if (rc == MAG_OK && cudaMemcpyAsync(nu.p, Nu, Ne * 8, cudaMemcpyHostToDevice, s) != cudaSuccess) rc = MAG_E_CUDA;
    if (rc == MAG_OK) rc = launch_stiffness_elems(mm.ed, nu.as<double>(), qp, mm.scratch.as<double>(), s);
    if (rc == MAG_OK) rc = mex_to_sparse(mm, Ne, Ndof, true, nullptr, out, s);
    cudaFree(dq);
    return rc;
}

int mag_mex_mass_sparse(const double *P, int64_t Nn, const double *T, int64_t Ne, const double *Dofs,
                        const double *Signs, const double *Coeffs, int64_t ncoeffs, const double *Qw, int nq,
                        const double *ValRef, int64_t Ndof, mag_sparse **out) {
    cudaStream_t s = nullptr;
    if (out) *out = nullptr;
    if (!out || Ndof <= 0) {
        set_error("mag_mex_mass_sparse: bad arguments");
        return MAG_E_ARG;
    }
    if (Ne == 0) return empty_sparse(Ndof, out);
    std::lock_guard<std::mutex> lk(g_mex_mu);
    MexMesh *mmp = nullptr;
    int max_tag = 0;
    MAG_TRY(mex_mesh(P, Nn, T, Ne, Dofs, Signs, nullptr, Ndof, &mmp, &max_tag, s));
    MexMesh &mm = *mmp;
    QuadParams qp{};
    double *dq = nullptr;
    MAG_TRY(make_quad(Qw, nq, ValRef, ValRef, &qp, &dq, s));
    Dev sg(s);
    const double *dsig = nullptr;
    int rc = MAG_OK;
    if (Coeffs && ncoeffs == Ne) {  // otherwise sigma = 1 (assemble_mass_kernel_mex.cpp:155)
        rc = sg.alloc(Ne * 8) == cudaSuccess ? MAG_OK : MAG_E_NOMEM;
        if (rc == MAG_OK && cudaMemcpyAsync(sg.p, Coeffs, Ne * 8, cudaMemcpyHostToDevice, s) != cudaSuccess)
            rc = MAG_E_CUDA;
        dsig = sg.as<double>();
    }
    if (rc == MAG_OK) rc = launch_mass_elems(mm.ed, dsig, qp, mm.scratch.as<double>(), s);
    if (rc == MAG_OK) rc = mex_to_sparse(mm, Ne, Ndof, true, nullptr, out, s);
    cudaFree(dq);
    return rc;
}

int mag_sparse_info(const mag_sparse *sp, int64_t *n, int64_t *nnz) {
    if (!sp) {
        set_error("mag_sparse_info: null handle");
        return MAG_E_ARG;
    }
    if (n) *n = sp->n;
    if (nnz) *nnz = sp->nnz;
    return MAG_OK;
}

int mag_sparse_copy(const mag_sparse *sp, uint64_t *jc, uint64_t *ir, double *pr) {
    if (!sp || !jc || (sp->nnz > 0 && (!ir || !pr))) {
        set_error("mag_sparse_copy: bad arguments");
        return MAG_E_ARG;
    }
    cudaStream_t s = nullptr;
    // column pointers are non-negative: the int64 bits are the mwIndex bits
    std::lock_guard<std::mutex> lk(g_mex_mu);  // the pinned staging buffers
    MAG_TRY(copy_to_host(jc, sp->rp, (sp->n + 1) * 8, s));
    if (sp->nnz > 0) {
        Dev wide(s);
        MAG_CUDA_TRY(wide.alloc(sp->nnz * 8));
        k_i32_to_u64<<<grid(sp->nnz), kB, 0, s>>>(sp->ci, sp->nnz, wide.as<uint64_t>());
        MAG_TRY(copy_to_host(ir, wide.p, sp->nnz * 8, s));
        MAG_TRY(copy_to_host(pr, sp->v, sp->nnz * 8, s));
    }
    MAG_CUDA_TRY(cudaStreamSynchronize(s));
    return MAG_OK;
}

int mag_sparse_destroy(mag_sparse *sp) {
    destroy_sparse(sp);
    return MAG_OK;
}

}  // extern "C"
