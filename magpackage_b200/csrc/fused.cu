// Fused single-launch Newton-Jacobian assembly (FP64, sm_100a).
//
// One cooperative launch of persistent CTAs walks a static schedule that
// interleaves two kinds of items:
//   element tile t  -- 256 elements: geometry, curls, B, nu(|B|^2), the 6x6
//                      tangent and the residual row, staged row by row
//                      through shared memory and stored as full 64-byte
//                      chunks into ring slot t mod R;
//   row chunk c     -- 32 CSR rows: one thread per nonzero walks its row's
//                      incidence list (ascending element order) and adds the
//                      matching value of each incident element's chunk; the
//                      diagonal thread also sums the residual.
// A chunk starts once every tile it reads is done; a tile reuses a ring slot
// once every chunk that read the slot's previous tile is done. The host turns
// both rules into one number per item: the schedule position before which
// every item must be complete. CTA b takes positions b, b+G, b+2G, ... in
// order and publishes how many it has finished, so "every item before p is
// done" is min over CTAs of (finished_b * G + b) >= p. Every requirement names
// earlier positions only and all CTAs are co-resident, so the earliest
// unfinished item can always proceed. The completed-prefix bound is loaded at
// the start of each item and reduced at its end, so an item whose requirement
// is already met starts without a round trip. The ring covers the mesh's reuse
// window (about one plane of hexahedra for these meshes), which keeps the
// element scratch in L2 instead of writing it to HBM and reading it back.
//
// Waits are bounded: after kSpinLimit polls a CTA records MAG_E_TIMEOUT in the
// error word, skips the item, still counts it as finished and moves on, so the
// launch always ends. Element arithmetic is bit-identical to the reference (see
// element.cuh; this file is compiled with -fmad=false) and each nonzero is
// summed in ascending element order, exactly like the two-pass kernels.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "element.cuh"
#include "fused.cuh"

namespace mag {

namespace {

using namespace elem;

__device__ __forceinline__ int ld_relaxed(const int *p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(int *p, int v) {
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ int warp_min(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ int match5(uint32_t w, uint32_t p) {
    const uint32_t L = 0x02108421u, H = 0x21084210u;  // low / high bit of each 5-bit field
    uint32_t x = w ^ (p * L);
    uint32_t z = (x - L) & ~x & H;
    return z ? ((__ffs(z) - 1) - 4) / 5 : -1;
}

__device__ __forceinline__ int match8(uint32_t w0, uint32_t w1, uint32_t p) {
    uint32_t x0 = w0 ^ (p * 0x01010101u);
    uint32_t z0 = (x0 - 0x01010101u) & ~x0 & 0x80808080u;
    if (z0) return ((__ffs(z0) - 1) - 7) / 8;
    uint32_t x1 = (w1 ^ (p * 0x0101u)) & 0xFFFFu;
    uint32_t z1 = (x1 - 0x0101u) & ~x1 & 0x8080u;
    return z1 ? 4 + ((__ffs(z1) - 1) - 7) / 8 : -1;
}

__device__ __forceinline__ double qsum_w(double v, const QuadParams &qp, double adet) {
    double u = v * (qp.qw[0] * adet);
    double acc = u;
    if (qp.uniform_w) {
        for (int q = 1; q < qp.nq; q++) acc = acc + u;
    } else {
        for (int q = 1; q < qp.nq; q++) acc = acc + v * (qp.qw[q] * adet);
    }
    return acc;
}

struct FusedArgs {
    ElemData m;
    RowPlan rp;
    const double *sol;
    QuadParams qp;
    MaterialParams mp;
    double *vals;
    double *res;
    const int32_t *sched;
    const int32_t *need;
    int *ctrl;
    double *ring;
    int nitems, ntiles, nchunks, ring_tiles;
};

// ---- element tile -------------------------------------------------------------

template <bool CALCJ, bool STDCURL>
__device__ void run_tile(const FusedArgs &A, int t, double *sbuf) {
    const int tid = threadIdx.x;
    const int64_t e = (int64_t)t * kTileElems + tid;
    const bool valid = e < A.m.ne;
    double C[6][3], b[6], nu = 0, dnu = 0, adet = 0;
    unsigned sb = 0;
    double Kg[6][6], rg[6];  // general path only
    if (valid) {
        int4 tt = A.m.tet[e];
        int d[6];
        load_dofs(A.m.dofs, e, d);
        sb = A.m.signbits ? A.m.signbits[e] : derived_signs(tt);
        int tag = A.m.tags[e];
        Geo g;
        geometry(A.m.xyz, tt, g);
        adet = g.adet;
        double a[6];
#pragma unroll
        for (int i = 0; i < 6; i++) a[i] = d[i] >= 0 ? flip(__ldg(A.sol + d[i]), (sb >> i) & 1) : 0.0;
        if (STDCURL) {
            curls_standard(g, C);
            double B[3];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                double s = a[0] * C[0][c];
#pragma unroll
                for (int i = 1; i < 6; i++) s = s + a[i] * C[i][c];
                B[c] = s;
            }
            material_eval(A.mp, tag, dot3(B, B), nu, dnu);
#pragma unroll
            for (int i = 0; i < 6; i++) b[i] = dot3(B, C[i]);
        } else {
            jacobian_block<CALCJ, false>(g, a, tag, A.qp, A.mp, rg, Kg);
        }
    }
    double *slot = A.ring + (size_t)(t % A.ring_tiles) * kTileElems * kScratchPerElem;
    const int64_t n_here = A.m.ne - (int64_t)t * kTileElems;
    const int nvalid = n_here < kTileElems ? (int)n_here : kTileElems;
#pragma unroll 1
    for (int i = 0; i < 6; i++) {
        if (valid) {
            double row[6], r;
            if (STDCURL) {
                r = qsum_w(nu * b[i], A.qp, adet);
                if (CALCJ) {
                    if (dnu == 0.0) {
#pragma unroll
                        for (int j = 0; j < 6; j++) row[j] = qsum_w(nu * dot3(C[i], C[j]), A.qp, adet);
                    } else {
                        double gi = (2.0 * dnu) * b[i];
#pragma unroll
                        for (int j = 0; j < 6; j++)
                            row[j] = qsum_w(nu * dot3(C[i], C[j]) + gi * b[j], A.qp, adet);
                    }
                }
            } else {
                r = rg[i];
#pragma unroll
                for (int j = 0; j < 6; j++) row[j] = Kg[i][j];
            }
            double *o = sbuf + tid * 9;
#pragma unroll
            for (int j = 0; j < 6; j++) o[j] = CALCJ ? flip(row[j], ((sb >> i) ^ (sb >> j)) & 1) : 0.0;
            o[6] = flip(r, (sb >> i) & 1);
            o[7] = 0.0;
        }
        __syncthreads();
        // kTileElems chunks x 64 bytes, in 16-byte pieces; a warp stores 8 whole chunks
#pragma unroll
        for (int q = 0; q < 4; q++) {
            int piece = tid + q * kTileElems;
            int c = piece >> 2, h = piece & 3;
            if (c < nvalid) {
                double2 v = make_double2(sbuf[c * 9 + 2 * h], sbuf[c * 9 + 2 * h + 1]);
                *reinterpret_cast<double2 *>(slot + (size_t)c * kScratchPerElem + i * kScratchStride + 2 * h) = v;
            }
        }
        __syncthreads();
    }
}

// ---- row chunk ----------------------------------------------------------------

template <bool CALCJ, bool WIDE>
__device__ void run_chunk(const FusedArgs &A, int c, int *srow) {
    const int tid = threadIdx.x;
    const int64_t a0 = (int64_t)c * kChunkRows;
    const int nrows = (int)((A.rp.ndof - a0) < kChunkRows ? (A.rp.ndof - a0) : kChunkRows);
    int *s_rp = srow, *s_ip = srow + kChunkRows + 1;
    if (tid <= nrows) {
        s_rp[tid] = A.rp.row_ptr[a0 + tid];
        s_ip[tid] = A.rp.inc_ptr[a0 + tid];
    }
    __syncthreads();
    const int base = s_rp[0];
    const size_t tile_doubles = (size_t)kTileElems * kScratchPerElem;
    if (CALCJ) {
        const int span = s_rp[nrows] - base;
        for (int s = tid; s < span; s += kTileElems) {
            int r = 0;
            while (r + 1 < nrows && s_rp[r + 1] - base <= s) r++;
            const uint32_t p = (uint32_t)(s - (s_rp[r] - base));
            double acc = 0.0, racc = 0.0;
            bool diag = false;
            for (int k = s_ip[r]; k < s_ip[r + 1]; k++) {
                int j;
                if (!WIDE) j = match5(__ldg(A.rp.inc_pos + k), p);
                else j = match8(__ldg(A.rp.inc_pos + 2 * (int64_t)k), __ldg(A.rp.inc_pos + 2 * (int64_t)k + 1), p);
                if (j < 0) continue;
                uint32_t ew = __ldg(A.rp.inc_elem + k);
                uint32_t e = ew & 0x1FFFFFFFu, loc = ew >> 29;
                const double *ch = A.ring + (size_t)((e / kTileElems) % (uint32_t)A.ring_tiles) * tile_doubles +
                                   (size_t)(e % kTileElems) * kScratchPerElem + loc * kScratchStride;
                acc = acc + __ldcg(ch + j);
                if (j == (int)loc) {
                    diag = true;
                    racc = racc + __ldcg(ch + 6);
                }
            }
            A.vals[base + s] = acc;
            if (diag) A.res[a0 + r] = racc;
        }
    } else {
        if (tid < nrows) {
            double racc = 0.0;
            for (int k = s_ip[tid]; k < s_ip[tid + 1]; k++) {
                uint32_t ew = __ldg(A.rp.inc_elem + k);
                uint32_t e = ew & 0x1FFFFFFFu, loc = ew >> 29;
                const double *ch = A.ring + (size_t)((e / kTileElems) % (uint32_t)A.ring_tiles) * tile_doubles +
                                   (size_t)(e % kTileElems) * kScratchPerElem + loc * kScratchStride;
                racc = racc + __ldcg(ch + 6);
            }
            A.res[a0 + tid] = racc;
        }
    }
}

template <bool CALCJ, bool STDCURL, bool WIDE>
__global__ void __launch_bounds__(kTileElems, 2) k_fused(FusedArgs A) {
    __shared__ double sbuf[kTileElems * 9];
    __shared__ int srow[2 * (kChunkRows + 1)];
    __shared__ int s_red[kTileElems / 32];
    __shared__ int s_done, s_skip;
    const int G = gridDim.x, b = blockIdx.x, tid = threadIdx.x;
    int *err = A.ctrl;
    int *progress = A.ctrl + kCtrlHeader;
    if (tid == 0) {
        s_done = 0;
        s_skip = 0;
    }
    __syncthreads();
    int finished = 0;
    for (int it = b; it < A.nitems; it += G, finished++) {
        const int code = __ldg(A.sched + it);
        const int np = __ldg(A.need + it);
        if (np > s_done) {  // block-uniform: wait until every item before np is finished
            long long spins = 0;
            for (;;) {
                int lo = 0x7FFFFFFF;
                for (int j = tid; j < G; j += kTileElems) {
                    int pos = j == b ? it : ld_relaxed(progress + j) * G + j;
                    lo = min(lo, pos);
                }
                lo = warp_min(lo);
                if ((tid & 31) == 0) s_red[tid >> 5] = lo;
                __syncthreads();
                if (tid == 0) {
                    int m = s_red[0];
                    for (int w = 1; w < kTileElems / 32; w++) m = min(m, s_red[w]);
                    s_done = max(s_done, m);
                    if (s_done < np && ++spins > kSpinLimit) {
                        atomicExch(err, MAG_E_TIMEOUT);
                        s_skip = 1;
                    }
                }
                __syncthreads();
                if (s_done >= np || s_skip) break;
                __nanosleep(128);
            }
            __threadfence();  // acquire: the progress loads above saw released counters
        }
        // start loading the completed-prefix bound for the next item
        int pre0 = 0x7FFFFFFF, pre1 = 0x7FFFFFFF;
        if (tid < G) pre0 = tid == b ? -1 : ld_relaxed(progress + tid);
        if (tid + kTileElems < G) pre1 = tid + kTileElems == b ? -1 : ld_relaxed(progress + tid + kTileElems);
        if (!s_skip) {
            if (code >= 0) run_tile<CALCJ, STDCURL>(A, code, sbuf);
            else run_chunk<CALCJ, WIDE>(A, -1 - code, srow);
        }
        __threadfence();  // release this item's writes; acquire for the loads just issued
        int lo = 0x7FFFFFFF;
        if (tid < G) lo = pre0 < 0 ? it + G : pre0 * G + tid;
        if (tid + kTileElems < G) lo = min(lo, pre1 < 0 ? it + G : pre1 * G + tid + kTileElems);
        lo = warp_min(lo);
        if ((tid & 31) == 0) s_red[tid >> 5] = lo;
        __syncthreads();
        if (tid == 0) {
            st_release(progress + b, finished + 1);
            int m = s_red[0];
            for (int w = 1; w < kTileElems / 32; w++) m = min(m, s_red[w]);
            s_done = max(s_done, m);
        }
        __syncthreads();
    }
}

// Per chunk, the last tile any of its rows reads (and the first, for planning).
__global__ void k_chunk_span(RowPlan rp, int nchunks, int32_t *lo, int32_t *hi) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nchunks) return;
    int64_t a0 = (int64_t)c * kChunkRows, a1 = a0 + kChunkRows < rp.ndof ? a0 + kChunkRows : rp.ndof;
    int mn = 0x7FFFFFFF, mx = -1;
    for (int k = rp.inc_ptr[a0]; k < rp.inc_ptr[a1]; k++) {
        int t = (int)((rp.inc_elem[k] & 0x1FFFFFFFu) / kTileElems);
        mn = t < mn ? t : mn;
        mx = t > mx ? t : mx;
    }
    lo[c] = mx < 0 ? -1 : mn;
    hi[c] = mx;
}

template <bool CALCJ, bool STDCURL, bool WIDE>
cudaError_t launch(FusedArgs &A, int grid, cudaStream_t s) {
    void *args[] = {&A};
    return cudaLaunchCooperativeKernel((const void *)k_fused<CALCJ, STDCURL, WIDE>, dim3(grid),
                                       dim3(kTileElems), args, 0, s);
}

}  // namespace

int build_fused_plan(const ElemData &m, const RowPlan &rp, int max_row, FusedPlan *fp, cudaStream_t s) {
    *fp = FusedPlan{};
    (void)max_row;
    const int ntiles = (int)((m.ne + kTileElems - 1) / kTileElems);
    const int nchunks = (int)((rp.ndof + kChunkRows - 1) / kChunkRows);
    // grid: every CTA resident at once (cooperative launch)
    int dev = 0, nsm = 0, per_sm = 0;
    MAG_CUDA_TRY(cudaGetDevice(&dev));
    MAG_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const void *variants[] = {
        (const void *)k_fused<true, true, false>,  (const void *)k_fused<true, true, true>,
        (const void *)k_fused<true, false, false>, (const void *)k_fused<true, false, true>,
        (const void *)k_fused<false, true, false>, (const void *)k_fused<false, true, true>,
        (const void *)k_fused<false, false, false>, (const void *)k_fused<false, false, true>};
    per_sm = 1 << 20;
    for (const void *f : variants) {
        int n = 0;
        MAG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f, kTileElems, 0));
        per_sm = std::min(per_sm, n);
    }
    if (per_sm < 1) {
        set_error("fused plan: kernel does not fit on an SM");
        return MAG_E_UNSUPPORTED;
    }
    const int grid = nsm * per_sm;

    int32_t *d_lo = nullptr, *d_hi = nullptr;
    MAG_CUDA_TRY(cudaMallocAsync((void **)&d_lo, (size_t)nchunks * 4 + 4, s));
    MAG_CUDA_TRY(cudaMallocAsync((void **)&d_hi, (size_t)nchunks * 4 + 4, s));
    k_chunk_span<<<(nchunks + 255) / 256, 256, 0, s>>>(rp, nchunks, d_lo, d_hi);
    std::vector<int32_t> lo(nchunks), hi(nchunks);
    MAG_CUDA_TRY(cudaMemcpyAsync(lo.data(), d_lo, (size_t)nchunks * 4, cudaMemcpyDeviceToHost, s));
    MAG_CUDA_TRY(cudaMemcpyAsync(hi.data(), d_hi, (size_t)nchunks * 4, cudaMemcpyDeviceToHost, s));
    MAG_CUDA_TRY(cudaStreamSynchronize(s));
    cudaFreeAsync(d_lo, s);
    cudaFreeAsync(d_hi, s);

    int span = 0;
    for (int c = 0; c < nchunks; c++)
        if (hi[c] >= 0) span = std::max(span, hi[c] - lo[c]);
    // Dependencies must point several "waves" (G consecutive items, one per CTA)
    // back, or the schedule degenerates into a grid-wide barrier per wave: a
    // chunk runs lag tiles after the last tile it reads, and a tile reuses a
    // slot lag tiles after the last chunk that read it, so ring >= span + 2 lag.
    const double chunks_per_tile = (double)nchunks / std::max(ntiles, 1);
    const int lag = std::max(2, (int)(kLagWaves * (double)grid / (1.0 + chunks_per_tile)) + 1);
    // chunk order: by the tile after which it may run (hi + lag), then index
    std::vector<int32_t> order(nchunks);
    for (int c = 0; c < nchunks; c++) order[c] = c;
    std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) { return hi[x] < hi[y]; });
    std::vector<int32_t> sched;
    sched.reserve((size_t)ntiles + nchunks);
    std::vector<int64_t> pos_tile(ntiles), pos_chunk(nchunks);
    size_t k = 0;
    while (k < order.size() && hi[order[k]] < 0) {  // rows touching no element
        pos_chunk[order[k]] = (int64_t)sched.size();
        sched.push_back(-1 - order[k]);
        k++;
    }
    for (int t = 0; t < ntiles; t++) {
        pos_tile[t] = (int64_t)sched.size();
        sched.push_back(t);
        while (k < order.size() && (hi[order[k]] + lag <= t || t == ntiles - 1)) {
            pos_chunk[order[k]] = (int64_t)sched.size();
            sched.push_back(-1 - order[k]);
            k++;
        }
    }
    // latest-reading chunk of every tile (reverse sweep, next-unassigned jumps)
    std::vector<int32_t> maxreader(ntiles, -1), nxt(ntiles + 1);
    for (int t = 0; t <= ntiles; t++) nxt[t] = t;
    auto find = [&](int t) {
        while (nxt[t] != t) {
            nxt[t] = nxt[nxt[t]];
            t = nxt[t];
        }
        return t;
    };
    for (int c = nchunks - 1; c >= 0; c--) {
        if (hi[c] < 0) continue;
        for (int t = find(lo[c]); t <= hi[c]; t = find(t)) {
            maxreader[t] = c;
            nxt[t] = t + 1;
        }
    }
    std::vector<int64_t> pmax(nchunks);
    int64_t run = -1;
    for (int c = 0; c < nchunks; c++) {
        run = std::max(run, pos_chunk[c]);
        pmax[c] = run;
    }
    // smallest ring for which every slot-reuse wait names earlier items only
    int ring = std::min(ntiles, span + 2 * lag + 8);
    std::vector<int32_t> need(sched.size(), 0);
    for (;;) {
        bool okr = true;
        for (int t = ring; t < ntiles; t++) {
            int r = maxreader[t - ring];
            if (r >= 0 && pmax[r] >= pos_tile[t]) {
                okr = false;
                break;
            }
        }
        if (okr) break;
        if (ring >= ntiles) {  // unreachable: with ring == ntiles no slot is reused
            set_error("fused plan: no valid schedule");
            return MAG_E_UNSUPPORTED;
        }
        ring = std::min(ntiles, ring + ring / 2 + 1);
    }
    for (int t = 0; t < ntiles; t++) {
        int32_t np = 0;
        if (t >= ring) {
            int r = maxreader[t - ring];
            if (r >= 0) np = (int32_t)(pmax[r] + 1);
        }
        need[pos_tile[t]] = np;
    }
    for (int c = 0; c < nchunks; c++) need[pos_chunk[c]] = hi[c] >= 0 ? (int32_t)(pos_tile[hi[c]] + 1) : 0;
    // the no-deadlock invariant: an item only ever waits on earlier positions
    for (size_t i = 0; i < need.size(); i++) {
        if (need[i] < 0 || (size_t)need[i] > i) {
            set_error("fused plan: item %zu would wait on a later item", i);
            return MAG_E_UNSUPPORTED;
        }
    }

    fp->ntiles = ntiles;
    fp->nchunks = nchunks;
    fp->nitems = (int32_t)sched.size();
    fp->ring_tiles = ring;
    fp->grid = std::min(grid, fp->nitems);
    fp->ctrl_bytes = (size_t)(kCtrlHeader + fp->grid) * 4;
    size_t ring_bytes = (size_t)ring * kTileElems * kScratchPerElem * 8;
    MAG_CUDA_TRY(cudaMalloc(&fp->sched, sched.size() * 4));
    MAG_CUDA_TRY(cudaMalloc(&fp->need, need.size() * 4));
    MAG_CUDA_TRY(cudaMalloc(&fp->ctrl, fp->ctrl_bytes));
    // the status word is read by mag_mesh_check whichever schedule ran: start it clear
    MAG_CUDA_TRY(cudaMemsetAsync(fp->ctrl, 0, fp->ctrl_bytes, s));
    MAG_CUDA_TRY(cudaMalloc(&fp->ring, ring_bytes));
    MAG_CUDA_TRY(cudaMemcpyAsync(fp->sched, sched.data(), sched.size() * 4, cudaMemcpyHostToDevice, s));
    MAG_CUDA_TRY(cudaMemcpyAsync(fp->need, need.data(), need.size() * 4, cudaMemcpyHostToDevice, s));
    MAG_CUDA_TRY(cudaStreamSynchronize(s));
    fp->bytes = (int64_t)(sched.size() * 8 + fp->ctrl_bytes + ring_bytes);
    fp->ok = 1;
    return MAG_OK;
}

void free_fused_plan(FusedPlan *fp) {
    void *ptrs[] = {fp->sched, fp->need, fp->ctrl, fp->ring};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    *fp = FusedPlan{};
}

int launch_fused_jacobian(const FusedPlan &fp, const ElemData &m, const RowPlan &rp, const double *sol,
                          const QuadParams &qp, const MaterialParams &mp, int calcj, double *vals,
                          double *res, cudaStream_t s) {
    if (!fp.ok) return MAG_E_UNSUPPORTED;
    MAG_CUDA_TRY(cudaMemsetAsync(fp.ctrl, 0, fp.ctrl_bytes, s));
    FusedArgs A{m, rp, sol, qp, mp, vals, res, fp.sched, fp.need, fp.ctrl, fp.ring,
                fp.nitems, fp.ntiles, fp.nchunks, fp.ring_tiles};
    cudaError_t e;
    const bool std_c = qp.standard_curl != 0, wide = rp.wide != 0;
    if (calcj) {
        if (std_c) e = wide ? launch<true, true, true>(A, fp.grid, s) : launch<true, true, false>(A, fp.grid, s);
        else e = wide ? launch<true, false, true>(A, fp.grid, s) : launch<true, false, false>(A, fp.grid, s);
    } else {
        if (std_c) e = wide ? launch<false, true, true>(A, fp.grid, s) : launch<false, true, false>(A, fp.grid, s);
        else e = wide ? launch<false, false, true>(A, fp.grid, s) : launch<false, false, false>(A, fp.grid, s);
    }
    if (e != cudaSuccess) {
        set_error("fused launch: %s", cudaGetErrorString(e));
        return MAG_E_CUDA;
    }
    return MAG_OK;
}

int fused_status(const FusedPlan &fp, cudaStream_t s) {
    if (!fp.ok) return MAG_OK;
    int h = 0;
    MAG_CUDA_TRY(cudaMemcpyAsync(&h, fp.ctrl, 4, cudaMemcpyDeviceToHost, s));
    MAG_CUDA_TRY(cudaStreamSynchronize(s));
    if (h) {
        set_error("a bounded device-side wait gave up; the last assembly's output is incomplete");
        return MAG_E_TIMEOUT;
    }
    return MAG_OK;
}

}  // namespace mag
