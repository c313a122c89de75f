// Batched complex frequency-domain assembly: A_i = K_i(nu) + j*omega_i*M_i(sigma)
// for many independent meshes in one persistent launch (FP64 -> complex128).
//
// Each instance is a mag_mesh with its own CSR pattern and row-block plan. The
// work queue is the list of (instance, row block) items of all instances;
// persistent CTAs take items b, b+G, b+2G, ... (items are independent, so no
// waits). An item is a row block (see rowblock.cu):
//   phase A -- one thread per incidence computes the element's row loc of the
//              curl-curl matrix (assemble_curl_curl_kernel_mex.cpp:64-101) and of
//              the sigma-mass matrix (assemble_mass_kernel_mex.cpp:186-230,
//              four distinct quadrature points), signed, into shared memory;
//   phase B -- when the mesh has second-contributor bits, phase A already placed
//              every off-diagonal entry of K and M into one of its nonzero's two
//              slots (at most two contributions, summed (0 + a) + b, which does not
//              depend on their order); one thread per row sums the diagonals in
//              ascending element order and one pass stores the pairs. Otherwise one
//              thread per row sums all entries in ascending element order. Either
//              way the pair is (K_ab, omega * M_ab): exactly what MATLAB forms for
//              K + 1j*omega*M from the two assembled matrices
//              (FrequencySolver.m:131), where 0*M adds nothing to the real part.
// Variants 4 and 5 run the same assembly on the meshes' tile blocks instead
// (k_tile_complex in tile.cu: one evaluation of each element per block it touches, K
// pass then M pass). The launch is captured once in a CUDA graph and replayed. The
// variant (schedule, block size, CTA residency) is chosen per batch by timing every
// available one (mag_batch_create).
#include <algorithm>
#include <vector>

#include "batch.cuh"
#include "common.cuh"
#include "element.cuh"

namespace mag {

namespace {

using namespace elem;

struct BatchItem {
    int32_t inst;
    int32_t block;
};

// Nonzeros of a block the slot path holds: four slot arrays (K and M, two slots per
// nonzero) plus per-incidence diagonals and row offsets fit in the 24 * BI doubles of the
// row-phase buffers. A block's span is at most 6 * BI; larger spans take the row phase.
template <int BI>
constexpr int kSlotSpan = 5 * BI;

template <int BI>
__device__ void complex_block(const BatchInstance &I, int blk, double *sk, double *sm, double *acc_k,
                              double *acc_m, int *s_rp, int *s_ip, const double *sval) {
    const int tid = threadIdx.x;
    const int a0 = I.block_row[blk], a1 = I.block_row[blk + 1];
    const int nrows = a1 - a0;
    for (int r = tid; r <= nrows; r += BI) {
        s_rp[r] = I.rp.row_ptr[a0 + r];
        s_ip[r] = I.rp.inc_ptr[a0 + r];
    }
    __syncthreads();
    const int k0 = s_ip[0], ninc = s_ip[nrows] - k0;
    const int base = s_rp[0], span = s_rp[nrows] - base;
    // slot path: each off-diagonal entry of K and M has at most two contributions (the
    // tetrahedra sharing a face) and (0 + a) + b does not depend on their order, so the
    // incidences place them directly; only the diagonals are summed per row
    const bool slots = I.second != nullptr && span <= kSlotSpan<BI>;
    double *slot_k = sk, *slot_m = sk + 2 * kSlotSpan<BI>;  // [span][2] each
    double *sdiag = sk + 4 * kSlotSpan<BI>;                   // [ninc][2]: K, M diagonal entries
    uint16_t *sroff = reinterpret_cast<uint16_t *>(sdiag + 2 * BI);  // [ninc]: row's first nonzero
    static_assert(4 * kSlotSpan<BI> + 2 * BI + BI / 4 <= 24 * BI, "slot path fits the row-phase buffers");
    if (slots) {
        for (int r = tid; r < nrows; r += BI)
            for (int k = s_ip[r]; k < s_ip[r + 1]; k++) sroff[k - k0] = (uint16_t)(s_rp[r] - base);
        for (int i = tid; i < 4 * span; i += BI) (i < 2 * span ? slot_k[i] : slot_m[i - 2 * span]) = 0.0;
        __syncthreads();
    }
    if (tid < ninc) {
        uint32_t ew = __ldg(I.rp.inc_elem + k0 + tid);
        const int64_t e = ew & 0x1FFFFFFFu;
        const int loc = (int)(ew >> 29);
        int4 tt = I.m.tet[e];
        unsigned sb = I.m.signbits ? I.m.signbits[e] : derived_signs(tt);
        unsigned si = (sb >> loc) & 1;
        Geo g;
        geometry(I.m.xyz, tt, g);
        // curl-curl row: sum_q (C_loc . C_j * nu) * w_q
        double C[6][3];
        curls_standard(g, C);
        double Cl[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            double v = C[0][c];
#pragma unroll
            for (int i = 1; i < 6; i++) v = loc == i ? C[i][c] : v;
            Cl[c] = v;
        }
        const double nu = I.nu[e];
        const double w0 = I.qw[0] * g.adet;
        double krow[6];
#pragma unroll
        for (int j = 0; j < 6; j++) {
            double u = (dot3(Cl, C[j]) * nu) * w0;
            double kv = I.nq4 ? ((u + u) + u) + u : u;
            if (!I.nq4)
                for (int q = 1; q < I.nq; q++) kv = kv + (dot3(Cl, C[j]) * nu) * (I.qw[q] * g.adet);
            krow[j] = flip(kv, si ^ ((sb >> j) & 1));
        }
        // sigma-mass row: sum_q (N_loc . N_j * sigma) * w_q, N = J^{-T} N_ref
        const double sigma = I.sigma ? I.sigma[e] : 1.0;
        double mrow[6] = {0, 0, 0, 0, 0, 0};
        if (fabs(sigma) > 1e-12) {
            double iv[3][3];
            inverse3(g, iv);
            for (int q = 0; q < I.nq; q++) {
                const double w = I.qw[q] * g.adet;
                double N[6][3];
#pragma unroll
                for (int i = 0; i < 6; i++) {
                    const double r0 = sval[i + 18 * q], r1 = sval[i + 6 + 18 * q], r2 = sval[i + 12 + 18 * q];
#pragma unroll
                    for (int c = 0; c < 3; c++) N[i][c] = iv[0][c] * r0 + iv[1][c] * r1 + iv[2][c] * r2;
                }
                double Nl[3];
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    double v = N[0][c];
#pragma unroll
                    for (int i = 1; i < 6; i++) v = loc == i ? N[i][c] : v;
                    Nl[c] = v;
                }
#pragma unroll
                for (int j = 0; j < 6; j++) mrow[j] = mrow[j] + dot3(Nl, N[j]) * sigma * w;
            }
        }
#pragma unroll
        for (int j = 0; j < 6; j++) mrow[j] = flip(mrow[j], si ^ ((sb >> j) & 1));
        if (slots) {
            unsigned p[6];
            if (!I.rp.wide) {
                const uint32_t pw = __ldg(I.rp.inc_pos + k0 + tid);
#pragma unroll
                for (int j = 0; j < 6; j++) p[j] = (pw >> (5 * j)) & 31u;
            } else {
                const uint32_t w0p = __ldg(I.rp.inc_pos + 2 * (int64_t)(k0 + tid));
                const uint32_t w1p = __ldg(I.rp.inc_pos + 2 * (int64_t)(k0 + tid) + 1);
#pragma unroll
                for (int j = 0; j < 6; j++) p[j] = (j < 4 ? (w0p >> (8 * j)) : (w1p >> (8 * (j - 4)))) & 255u;
            }
            const unsigned none = I.rp.wide ? (unsigned)kWideMaxRow : (unsigned)kCompactMaxRow;
            const unsigned second = __ldg(I.second + k0 + tid);
            const int off = sroff[tid];
#pragma unroll
            for (int j = 0; j < 6; j++) {
                if (j == loc) {
                    sdiag[2 * tid] = krow[j];
                    sdiag[2 * tid + 1] = mrow[j];
                } else if (p[j] != none) {
                    const int at = 2 * (off + (int)p[j]) + (int)((second >> j) & 1);
                    slot_k[at] = krow[j];
                    slot_m[at] = mrow[j];
                }
            }
        } else {
#pragma unroll
            for (int j = 0; j < 6; j++) {
                sk[tid * 6 + j] = krow[j];
                sm[tid * 6 + j] = mrow[j];
            }
        }
    }
    double2 *out = reinterpret_cast<double2 *>(I.vals);
    if (slots) {
        __syncthreads();
        // diagonals: one thread per row, its incidences in ascending element order
        for (int r = tid; r < nrows; r += BI) {
            const int i0 = s_ip[r] - k0, i1 = s_ip[r + 1] - k0;
            if (i1 <= i0) continue;
            double dk = 0.0, dm = 0.0;
            for (int k = i0; k < i1; k++) {
                dk = dk + sdiag[2 * k];
                dm = dm + sdiag[2 * k + 1];
            }
            const int kf = k0 + i0;
            const int l = (int)(__ldg(I.rp.inc_elem + kf) >> 29);
            unsigned pd;
            if (!I.rp.wide) {
                pd = (__ldg(I.rp.inc_pos + kf) >> (5 * l)) & 31u;
            } else {
                pd = (l < 4 ? (__ldg(I.rp.inc_pos + 2 * (int64_t)kf) >> (8 * l))
                            : (__ldg(I.rp.inc_pos + 2 * (int64_t)kf + 1) >> (8 * (l - 4)))) & 255u;
            }
            const int at = 2 * (s_rp[r] - base + (int)pd);
            slot_k[at] = dk;
            slot_m[at] = dm;
        }
        __syncthreads();
        for (int i = tid; i < span; i += BI)
            out[base + i] = make_double2((0.0 + slot_k[2 * i]) + slot_k[2 * i + 1],
                                         I.omega * ((0.0 + slot_m[2 * i]) + slot_m[2 * i + 1]));
        __syncthreads();
        return;
    }
    for (int i = tid; i < span; i += BI) {
        acc_k[i] = 0.0;
        acc_m[i] = 0.0;
    }
    __syncthreads();
    for (int r = tid; r < nrows; r += BI) {
        const int off = s_rp[r] - base;
        for (int k = s_ip[r]; k < s_ip[r + 1]; k++) {
            const double *vk = sk + (k - k0) * 6, *vm = sm + (k - k0) * 6;
            if (!I.rp.wide) {
                uint32_t pw = __ldg(I.rp.inc_pos + k);
#pragma unroll
                for (int j = 0; j < 6; j++) {
                    uint32_t p = (pw >> (5 * j)) & 31u;
                    if (p != (uint32_t)kCompactMaxRow) {
                        acc_k[off + p] = acc_k[off + p] + vk[j];
                        acc_m[off + p] = acc_m[off + p] + vm[j];
                    }
                }
            } else {
                uint32_t w0 = __ldg(I.rp.inc_pos + 2 * (int64_t)k), w1 = __ldg(I.rp.inc_pos + 2 * (int64_t)k + 1);
#pragma unroll
                for (int j = 0; j < 6; j++) {
                    uint32_t p = (j < 4 ? (w0 >> (8 * j)) : (w1 >> (8 * (j - 4)))) & 255u;
                    if (p != (uint32_t)kWideMaxRow) {
                        acc_k[off + p] = acc_k[off + p] + vk[j];
                        acc_m[off + p] = acc_m[off + p] + vm[j];
                    }
                }
            }
        }
    }
    __syncthreads();
    for (int i = tid; i < span; i += BI) out[base + i] = make_double2(acc_k[i], I.omega * acc_m[i]);
    __syncthreads();
}

template <int BI>
constexpr size_t batch_smem_bytes() {
    return (size_t)(4 * BI * 6 + 18 * kMaxQuad) * sizeof(double) + 2 * (BI + 1) * sizeof(int);
}

template <int BI, int MINB>
__global__ void __launch_bounds__(BI, MINB) k_batch_complex(const BatchInstance *__restrict__ inst,
                                                             const BatchItem *__restrict__ items, int nitems) {
    extern __shared__ double dyn[];
    double *sk = dyn, *sm = sk + BI * 6, *acc_k = sm + BI * 6, *acc_m = acc_k + BI * 6;
    double *sval = acc_m + BI * 6;
    int *s_rp = reinterpret_cast<int *>(sval + 18 * kMaxQuad), *s_ip = s_rp + BI + 1;
    int cur = -1;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const BatchItem w = items[it];
        const BatchInstance &I = inst[w.inst];
        if (w.inst != cur) {  // reference basis values of this instance
            __syncthreads();
            for (int i = threadIdx.x; i < 18 * I.nq; i += BI) sval[i] = I.val_ref[i];
            __syncthreads();
            cur = w.inst;
        }
        complex_block<BI>(I, w.block, sk, sm, acc_k, acc_m, s_rp, s_ip, sval);
    }
}

using KernelFn = void (*)(const BatchInstance *, const BatchItem *, int);

struct Variant {
    KernelFn fn;
    int threads;
    size_t smem;
    const char *name;
};

const Variant kVariants[] = {
    {k_batch_complex<256, 2>, 256, batch_smem_bytes<256>(), "256 incidences/CTA, 2 CTAs/SM"},
    {k_batch_complex<256, 3>, 256, batch_smem_bytes<256>(), "256 incidences/CTA, 3 CTAs/SM"},
    {k_batch_complex<128, 4>, 128, batch_smem_bytes<128>(), "128 incidences/CTA, 4 CTAs/SM"},
    {k_batch_complex<128, 6>, 128, batch_smem_bytes<128>(), "128 incidences/CTA, 6 CTAs/SM"},
};
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);

}  // namespace

int batch_build(BatchState *b, cudaStream_t s) {
    // items per variant (block size differs between variants)
    for (int v = 0; v < kNumVariants; v++) {
        const int bi = kVariants[v].threads;
        std::vector<BatchItem> items;
        std::vector<BatchInstance> insts = b->inst_host;
        for (int i = 0; i < (int)insts.size(); i++) {
            const int32_t *br = bi == 256 ? b->block_row256[i] : b->block_row128[i];
            insts[i].block_row = br;
            int nb = bi == 256 ? b->nblocks256[i] : b->nblocks128[i];
            for (int k = 0; k < nb; k++) items.push_back(BatchItem{i, k});
        }
        // big instances first within the queue keeps the tail short
        std::stable_sort(items.begin(), items.end(), [&](const BatchItem &x, const BatchItem &y) {
            return b->inst_ne[x.inst] > b->inst_ne[y.inst];
        });
        BatchVariantData &d = b->var[v];
        d.nitems = (int)items.size();
        MAG_CUDA_TRY(cudaMalloc(&d.items, items.size() * sizeof(BatchItem) + 16));
        MAG_CUDA_TRY(cudaMalloc(&d.inst, insts.size() * sizeof(BatchInstance)));
        MAG_CUDA_TRY(cudaMemcpyAsync(d.items, items.data(), items.size() * sizeof(BatchItem),
                                     cudaMemcpyHostToDevice, s));
        MAG_CUDA_TRY(cudaMemcpyAsync(d.inst, insts.data(), insts.size() * sizeof(BatchInstance),
                                     cudaMemcpyHostToDevice, s));
        int dev = 0, nsm = 0, per = 0;
        MAG_CUDA_TRY(cudaGetDevice(&dev));
        MAG_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        MAG_CUDA_TRY(cudaFuncSetAttribute((const void *)kVariants[v].fn,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)kVariants[v].smem));
        MAG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void *)kVariants[v].fn,
                                                                   kVariants[v].threads, kVariants[v].smem));
        d.grid = std::max(1, std::min(d.nitems, nsm * std::max(per, 1)));
    }
    MAG_CUDA_TRY(cudaStreamSynchronize(s));
    // the tile-block variants, when every mesh has a tile plan
    return build_tile_complex(b->tile_in, &b->tile, s);
}

int batch_launch(const BatchState &b, int variant, cudaStream_t s) {
    if (variant >= kNumVariants) {
        if (launch_tile_complex(b.tile, variant - kNumVariants, s) != MAG_OK) {
            set_error("batch launch (tile blocks): %s", cudaGetErrorString(cudaGetLastError()));
            return MAG_E_CUDA;
        }
        return MAG_OK;
    }
    const BatchVariantData &d = b.var[variant];
    const Variant &v = kVariants[variant];
    v.fn<<<d.grid, v.threads, v.smem, s>>>(static_cast<const BatchInstance *>(d.inst),
                                      static_cast<const BatchItem *>(d.items), d.nitems);
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) {
        set_error("batch launch: %s", cudaGetErrorString(e));
        return MAG_E_CUDA;
    }
    return MAG_OK;
}

int batch_num_variants() { return kNumVariants + kTileComplexVariants; }
bool batch_variant_available(const BatchState &b, int v) {
    if (v >= kNumVariants) return v < kNumVariants + kTileComplexVariants && b.tile.ok;
    return v >= 0 && b.var[v].nitems > 0;
}
const char *batch_variant_name(int v) {
    if (v >= kNumVariants) return tile_complex_variant_name(v - kNumVariants);
    return v >= 0 ? kVariants[v].name : "";
}

void batch_free_variants(BatchState *b) {
    free_tile_complex(&b->tile);
    for (auto &d : b->var) {
        if (d.items) cudaFree(d.items);
        if (d.inst) cudaFree(d.inst);
        d = BatchVariantData{};
    }
}

}  // namespace mag
