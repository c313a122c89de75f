// One-time integer work on the GPU: edge numbering (Mesh.generateEdges), the CSR
// pattern of the dof coupling, the per-row incidence plan used by the
// fixed-order value reduction, and MATLAB-style zero dropping.
//
// Sorting uses CUB's stable radix sort (header library shipped with the CUDA
// toolkit). Stability is what makes every row's incidence list come out in
// ascending element order, which fixes the summation order of the assembly.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_reduce.cuh>
#include <cub/device/device_scan.cuh>

#include "common.cuh"
#include "internal.h"

namespace mag {

namespace {

int bits_for(uint64_t n) {
    int b = 1;
    while (b < 64 && (uint64_t(1) << b) <= n) b++;
    return b;
}

constexpr int kBlock = 256;
inline unsigned grid_for(int64_t n, int block = kBlock) {
    return (unsigned)((n + block - 1) / block);
}

// ---- edges --------------------------------------------------------------

__global__ void k_edge_keys(const int32_t *__restrict__ T, int64_t ne, int64_t nn, int nb,
                            uint64_t *__restrict__ keys, uint32_t *__restrict__ slots,
                            int8_t *__restrict__ sign, int *__restrict__ err) {
    int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= 6 * ne) return;
    int64_t e = s / 6;
    int k = (int)(s - 6 * e);
    int32_t a = T[4 * e + edge_a(k)], b = T[4 * e + edge_b(k)];
    if (a < 0 || b < 0 || a >= nn || b >= nn || a == b) {
        atomicExch(err, 1);
        a = b = 0;
    }
    uint64_t lo = (uint64_t)(a < b ? a : b), hi = (uint64_t)(a < b ? b : a);
    keys[s] = (lo << nb) | hi;
    slots[s] = (uint32_t)s;
    // +1 iff the local start node carries the smaller global id (Mesh.m:134-135)
    sign[s] = (int8_t)(a < b ? 1 : -1);
}

__global__ void k_head_flags(const uint64_t *__restrict__ keys, int64_t n, int32_t *__restrict__ f) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    f[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}

__global__ void k_edge_scatter(const uint64_t *__restrict__ keys, const uint32_t *__restrict__ slots,
                               const int32_t *__restrict__ flags, const int32_t *__restrict__ ids,
                               int64_t n, int nb, int32_t *__restrict__ edges,
                               int32_t *__restrict__ t2e) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int32_t id = ids[i] - 1;
    t2e[slots[i]] = id;
    if (flags[i]) {
        uint64_t k = keys[i];
        edges[2 * (int64_t)id] = (int32_t)(k >> nb);
        edges[2 * (int64_t)id + 1] = (int32_t)(k & ((uint64_t(1) << nb) - 1));
    }
}

// ---- pattern ------------------------------------------------------------

__global__ void k_inc_keys(const int32_t *__restrict__ dofs, int64_t ne, int64_t ndof,
                           uint32_t *__restrict__ keys, uint32_t *__restrict__ vals,
                           int32_t *__restrict__ cnt, int *__restrict__ err) {
    int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= 6 * ne) return;
    int64_t e = s / 6;
    int k = (int)(s - 6 * e);
    int32_t d = dofs[s];
    if (d >= ndof || d < -1) {
        atomicExch(err, 1);
        d = -1;
    }
    keys[s] = d < 0 ? (uint32_t)ndof : (uint32_t)d;  // dof-less slots sort to the end
    vals[s] = (uint32_t)e | ((uint32_t)k << 29);
    if (d >= 0) atomicAdd(&cnt[d], 1);
}

// Sorted unique insert into a small per-thread list; returns false on overflow.
__device__ inline bool insert_sorted(int32_t *list, int &n, int cap, int32_t v) {
    int lo = 0, hi = n;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (list[mid] < v) lo = mid + 1; else hi = mid;
    }
    if (lo < n && list[lo] == v) return true;
    if (n >= cap) return false;
    for (int t = n; t > lo; t--) list[t] = list[t - 1];
    list[lo] = v;
    n++;
    return true;
}

__device__ inline int find_sorted(const int32_t *list, int n, int32_t v) {
    int lo = 0, hi = n;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (list[mid] < v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

constexpr int kRowCap = 256;

// Pass 1 (fill == false): count each row's distinct columns.
// Pass 2 (fill == true): write col_idx and every incidence's six in-row positions.
template <bool FILL>
__global__ void k_rows(const int32_t *__restrict__ dofs, const int32_t *__restrict__ inc_ptr,
                       const uint32_t *__restrict__ inc_elem, int64_t ndof,
                       int32_t *__restrict__ row_nnz, const int32_t *__restrict__ row_ptr,
                       int32_t *__restrict__ col_idx, uint32_t *__restrict__ inc_pos, int wide,
                       int *__restrict__ err) {
    int64_t a = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (a >= ndof) return;
    int32_t list[kRowCap];
    int n = 0;
    int32_t t0 = inc_ptr[a], t1 = inc_ptr[a + 1];
    for (int32_t t = t0; t < t1; t++) {
        uint32_t e = inc_elem[t] & 0x1FFFFFFFu;
        for (int j = 0; j < 6; j++) {
            int32_t d = dofs[6 * (int64_t)e + j];
            if (d < 0) continue;
            if (!insert_sorted(list, n, kRowCap, d)) {
                atomicExch(err, 2);
                return;
            }
        }
    }
    if (!FILL) {
        row_nnz[a] = n;
        return;
    }
    int32_t base = row_ptr[a];
    for (int i = 0; i < n; i++) col_idx[base + i] = list[i];
    for (int32_t t = t0; t < t1; t++) {
        uint32_t e = inc_elem[t] & 0x1FFFFFFFu;
        if (!wide) {
            uint32_t w = 0;
            for (int j = 0; j < 6; j++) {
                int32_t d = dofs[6 * (int64_t)e + j];
                uint32_t p = d < 0 ? (uint32_t)kCompactMaxRow : (uint32_t)find_sorted(list, n, d);
                w |= p << (5 * j);
            }
            inc_pos[t] = w;
        } else {
            uint32_t w0 = 0, w1 = 0;
            for (int j = 0; j < 6; j++) {
                int32_t d = dofs[6 * (int64_t)e + j];
                uint32_t p = d < 0 ? (uint32_t)kWideMaxRow : (uint32_t)find_sorted(list, n, d);
                if (j < 4) w0 |= p << (8 * j); else w1 |= p << (8 * (j - 4));
            }
            inc_pos[2 * (int64_t)t] = w0;
            inc_pos[2 * (int64_t)t + 1] = w1;
        }
    }
}

// ---- zero dropping --------------------------------------------------------

__global__ void k_count_nonzero(const int64_t *__restrict__ rp, const double *__restrict__ v,
                                int64_t nrows, int64_t *__restrict__ cnt) {
    int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= nrows) return;
    int64_t c = 0;
    for (int64_t t = rp[r]; t < rp[r + 1]; t++) c += (v[t] != 0.0);
    cnt[r] = c;
}

__global__ void k_compact(const int64_t *__restrict__ rp, const int32_t *__restrict__ ci,
                          const double *__restrict__ v, int64_t nrows,
                          const int64_t *__restrict__ rp_out, int32_t *__restrict__ ci_out,
                          double *__restrict__ v_out) {
    int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= nrows) return;
    int64_t o = rp_out[r];
    for (int64_t t = rp[r]; t < rp[r + 1]; t++) {
        double x = v[t];
        if (x != 0.0) {
            ci_out[o] = ci[t];
            v_out[o] = x;
            o++;
        }
    }
}

// Device scratch that frees itself on every return path.
struct DevBuf {
    void *p = nullptr;
    cudaStream_t s = nullptr;
    explicit DevBuf(cudaStream_t st) : s(st) {}
    ~DevBuf() {
        if (p) cudaFreeAsync(p, s);
    }
    cudaError_t alloc(size_t bytes) { return cudaMallocAsync(&p, bytes ? bytes : 16, s); }
    template <class T> T *as() const { return static_cast<T *>(p); }
};

int read_flag(const int *d_err, cudaStream_t s, int *out) {
    MAG_CUDA_TRY(cudaMemcpyAsync(out, d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    MAG_CUDA_TRY(cudaStreamSynchronize(s));
    return MAG_OK;
}

}  // namespace

int generate_edges(const int32_t *d_T, int64_t ne, int64_t nn, int32_t *d_edges, int32_t *d_t2e,
                   int8_t *d_sign, int64_t *E_out, cudaStream_t s) {
    if (ne <= 0 || nn <= 0 || !d_T || !d_edges || !d_t2e || !d_sign || !E_out) {
        set_error("generate_edges: bad arguments");
        return MAG_E_ARG;
    }
    if (6 * ne >= (int64_t(1) << 32) || nn >= (int64_t(1) << 31)) {
        set_error("generate_edges: mesh too large");
        return MAG_E_UNSUPPORTED;
    }
    int64_t n = 6 * ne;
    int nb = bits_for((uint64_t)nn);
    DevBuf keys(s), keys2(s), slots(s), slots2(s), flags(s), ids(s), err(s), tmp(s);
    MAG_CUDA_TRY(keys.alloc(n * 8));
    MAG_CUDA_TRY(keys2.alloc(n * 8));
    MAG_CUDA_TRY(slots.alloc(n * 4));
    MAG_CUDA_TRY(slots2.alloc(n * 4));
    MAG_CUDA_TRY(flags.alloc(n * 4));
    MAG_CUDA_TRY(ids.alloc(n * 4));
    MAG_CUDA_TRY(err.alloc(4));
    MAG_CUDA_TRY(cudaMemsetAsync(err.p, 0, 4, s));
    k_edge_keys<<<grid_for(n), kBlock, 0, s>>>(d_T, ne, nn, nb, keys.as<uint64_t>(),
                                               slots.as<uint32_t>(), d_sign, err.as<int>());
    size_t tb = 0, tb2 = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, keys.as<uint64_t>(), keys2.as<uint64_t>(),
                                    slots.as<uint32_t>(), slots2.as<uint32_t>(), (int64_t)n, 0,
                                    2 * nb, s);
    cub::DeviceScan::InclusiveSum(nullptr, tb2, flags.as<int32_t>(), ids.as<int32_t>(), (int64_t)n, s);
    MAG_CUDA_TRY(tmp.alloc(tb > tb2 ? tb : tb2));
    MAG_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp.p, tb, keys.as<uint64_t>(), keys2.as<uint64_t>(),
                                                 slots.as<uint32_t>(), slots2.as<uint32_t>(),
                                                 (int64_t)n, 0, 2 * nb, s));
    k_head_flags<<<grid_for(n), kBlock, 0, s>>>(keys2.as<uint64_t>(), n, flags.as<int32_t>());
    tb2 = tb > tb2 ? tb : tb2;
    MAG_CUDA_TRY(cub::DeviceScan::InclusiveSum(tmp.p, tb2, flags.as<int32_t>(), ids.as<int32_t>(),
                                               (int64_t)n, s));
    k_edge_scatter<<<grid_for(n), kBlock, 0, s>>>(keys2.as<uint64_t>(), slots2.as<uint32_t>(),
                                                  flags.as<int32_t>(), ids.as<int32_t>(), n, nb,
                                                  d_edges, d_t2e);
    MAG_CUDA_TRY(cudaGetLastError());
    int32_t last = 0;
    MAG_CUDA_TRY(cudaMemcpyAsync(&last, ids.as<int32_t>() + (n - 1), 4, cudaMemcpyDeviceToHost, s));
    int eflag = 0;
    MAG_TRY(read_flag(err.as<int>(), s, &eflag));
    if (eflag) {
        set_error("generate_edges: node id out of range or repeated node in an element");
        return MAG_E_RANGE;
    }
    *E_out = last;
    return MAG_OK;
}

int build_pattern(const int32_t *d_dofs, int64_t ne, int64_t ndof, PatternBuffers *out,
                  cudaStream_t s) {
    *out = PatternBuffers{};
    if (ne <= 0 || ndof <= 0 || !d_dofs) {
        set_error("build_pattern: bad arguments");
        return MAG_E_ARG;
    }
    if (ne >= (int64_t(1) << 29) || ndof >= (int64_t(1) << 31) - 2) {
        set_error("build_pattern: mesh too large (elements < 2^29, dofs < 2^31 supported)");
        return MAG_E_UNSUPPORTED;
    }
    int64_t n = 6 * ne;
    int nb = bits_for((uint64_t)ndof + 1);
    DevBuf keys(s), keys2(s), vals2(s), cnt(s), err(s), tmp(s), rownnz(s), maxrow(s);
    MAG_CUDA_TRY(keys.alloc(n * 4));
    MAG_CUDA_TRY(keys2.alloc(n * 4));
    MAG_CUDA_TRY(vals2.alloc(n * 4));
    MAG_CUDA_TRY(cnt.alloc((ndof + 1) * 4));
    MAG_CUDA_TRY(err.alloc(4));
    MAG_CUDA_TRY(rownnz.alloc((ndof + 1) * 4));
    MAG_CUDA_TRY(maxrow.alloc(4));
    MAG_CUDA_TRY(cudaMemsetAsync(err.p, 0, 4, s));
    MAG_CUDA_TRY(cudaMemsetAsync(cnt.p, 0, (ndof + 1) * 4, s));
    MAG_CUDA_TRY(cudaMemsetAsync(rownnz.p, 0, (ndof + 1) * 4, s));

    MAG_CUDA_TRY(cudaMallocAsync((void **)&out->inc_ptr, (ndof + 1) * 4, s));
    MAG_CUDA_TRY(cudaMallocAsync((void **)&out->row_ptr, (ndof + 1) * 4, s));
    MAG_CUDA_TRY(cudaMallocAsync((void **)&out->inc_elem, n * 4, s));

    k_inc_keys<<<grid_for(n), kBlock, 0, s>>>(d_dofs, ne, ndof, keys.as<uint32_t>(),
                                              out->inc_elem, cnt.as<int32_t>(), err.as<int>());
    // Stable sort by dof: each row's incidences stay in ascending element order.
    size_t tb = 0, tb2 = 0, tb3 = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, keys.as<uint32_t>(), keys2.as<uint32_t>(),
                                    out->inc_elem, vals2.as<uint32_t>(), (int64_t)n, 0, nb, s);
    cub::DeviceScan::ExclusiveSum(nullptr, tb2, cnt.as<int32_t>(), out->inc_ptr, (int64_t)ndof + 1, s);
    cub::DeviceReduce::Max(nullptr, tb3, rownnz.as<int32_t>(), maxrow.as<int32_t>(), (int64_t)ndof, s);
    size_t tbm = tb > tb2 ? tb : tb2;
    tbm = tbm > tb3 ? tbm : tb3;
    MAG_CUDA_TRY(tmp.alloc(tbm));
    MAG_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp.p, tb, keys.as<uint32_t>(), keys2.as<uint32_t>(),
                                                 out->inc_elem, vals2.as<uint32_t>(), (int64_t)n, 0,
                                                 nb, s));
    MAG_CUDA_TRY(cudaMemcpyAsync(out->inc_elem, vals2.p, n * 4, cudaMemcpyDeviceToDevice, s));
    tb2 = tbm;
    MAG_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp.p, tb2, cnt.as<int32_t>(), out->inc_ptr,
                                               (int64_t)ndof + 1, s));
    int32_t ninc = 0;
    MAG_CUDA_TRY(cudaMemcpyAsync(&ninc, out->inc_ptr + ndof, 4, cudaMemcpyDeviceToHost, s));
    int eflag = 0;
    MAG_TRY(read_flag(err.as<int>(), s, &eflag));
    if (eflag) {
        set_error("build_pattern: dof index out of range");
        return MAG_E_RANGE;
    }
    out->ninc = ninc;

    k_rows<false><<<grid_for(ndof, 128), 128, 0, s>>>(d_dofs, out->inc_ptr, out->inc_elem, ndof,
                                                       rownnz.as<int32_t>(), nullptr, nullptr,
                                                       nullptr, 0, err.as<int>());
    tb3 = tbm;
    MAG_CUDA_TRY(cub::DeviceReduce::Max(tmp.p, tb3, rownnz.as<int32_t>(), maxrow.as<int32_t>(),
                                        (int64_t)ndof, s));
    // row_nnz has a zero at index ndof, so the exclusive scan ends with nnz.
    tb2 = tbm;
    MAG_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp.p, tb2, rownnz.as<int32_t>(),
                                               out->row_ptr, (int64_t)ndof + 1, s));
    int32_t nnz = 0, mx = 0;
    MAG_CUDA_TRY(cudaMemcpyAsync(&nnz, out->row_ptr + ndof, 4, cudaMemcpyDeviceToHost, s));
    MAG_CUDA_TRY(cudaMemcpyAsync(&mx, maxrow.p, 4, cudaMemcpyDeviceToHost, s));
    MAG_TRY(read_flag(err.as<int>(), s, &eflag));
    if (eflag) {
        set_error("build_pattern: a row couples more than %d dofs", kRowCap);
        return MAG_E_UNSUPPORTED;
    }
    if (mx > kWideMaxRow) {
        set_error("build_pattern: a row has %d entries (at most %d supported)", mx, kWideMaxRow);
        return MAG_E_UNSUPPORTED;
    }
    out->nnz = nnz;
    out->max_row = mx;
    out->wide = mx > kCompactMaxRow ? 1 : 0;
    MAG_CUDA_TRY(cudaMallocAsync((void **)&out->col_idx, (size_t)nnz * 4 + 16, s));
    MAG_CUDA_TRY(cudaMallocAsync((void **)&out->inc_pos, (size_t)ninc * 4 * (out->wide ? 2 : 1) + 16, s));
    k_rows<true><<<grid_for(ndof, 128), 128, 0, s>>>(d_dofs, out->inc_ptr, out->inc_elem, ndof,
                                                      nullptr, out->row_ptr, out->col_idx,
                                                      out->inc_pos, out->wide, err.as<int>());
    MAG_CUDA_TRY(cudaGetLastError());
    MAG_CUDA_TRY(cudaStreamSynchronize(s));
    return MAG_OK;
}

void free_pattern(PatternBuffers *p, cudaStream_t s) {
    void *ptrs[] = {p->row_ptr, p->col_idx, p->inc_ptr, p->inc_elem, p->inc_pos};
    for (void *q : ptrs)
        if (q) cudaFreeAsync(q, s);
    *p = PatternBuffers{};
}

int csr_drop_zeros(const int64_t *rp, const int32_t *ci, const double *v, int64_t nrows,
                   int64_t *rp_out, int32_t *ci_out, double *v_out, int64_t *nnz_out,
                   cudaStream_t s) {
    if (nrows <= 0 || !rp || !ci || !v || !rp_out || !ci_out || !v_out || !nnz_out) {
        set_error("csr_drop_zeros: bad arguments");
        return MAG_E_ARG;
    }
    DevBuf cnt(s), tmp(s);
    MAG_CUDA_TRY(cnt.alloc((nrows + 1) * 8));
    MAG_CUDA_TRY(cudaMemsetAsync(cnt.p, 0, (nrows + 1) * 8, s));
    k_count_nonzero<<<grid_for(nrows), kBlock, 0, s>>>(rp, v, nrows, cnt.as<int64_t>());
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt.as<int64_t>(), rp_out, (int64_t)nrows + 1, s);
    MAG_CUDA_TRY(tmp.alloc(tb));
    MAG_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp.p, tb, cnt.as<int64_t>(), rp_out,
                                               (int64_t)nrows + 1, s));
    k_compact<<<grid_for(nrows), kBlock, 0, s>>>(rp, ci, v, nrows, rp_out, ci_out, v_out);
    MAG_CUDA_TRY(cudaGetLastError());
    MAG_CUDA_TRY(cudaMemcpyAsync(nnz_out, rp_out + nrows, 8, cudaMemcpyDeviceToHost, s));
    MAG_CUDA_TRY(cudaStreamSynchronize(s));
    return MAG_OK;
}

}  // namespace mag
