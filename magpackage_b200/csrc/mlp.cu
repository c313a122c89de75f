// Per-element reluctivity predictor: a 4 -> 64 -> 64 -> 64 -> 1 MLP with SiLU
// activations, BF16 tensor-core GEMMs (tcgen05, FP32 accumulators in TMEM) and
// FP32 master weights. Forward (inference and training) and backward kernels.
//
// Tile = 128 rows (elements) per CTA, 128 threads; thread t owns row t, and warp
// w reads TMEM lanes 32w..32w+31 (accumulator row m lives in lane m for M=128).
// Operands live in shared memory in the no-swizzle K-major "core matrix"
// layout: 8 rows x 16 bytes per core matrix, K-adjacent core matrices 128 B
// apart (leading byte offset), 8-row groups K*16 B apart (stride byte offset).
// One elected thread issues the MMAs (M=128, N=64, K=16 each) and commits them
// to an mbarrier; all threads wait with a bounded spin and read the
// accumulators with tcgen05.ld.
//
// Rounding points (mirrored by oracle/mlp_ref.py): layer inputs are rounded to
// BF16 before each MMA; accumulation, biases, activations, the last (64 -> 1)
// layer and all gradients are FP32. Inference halves W1..W3 and b1..b3 (exact),
// so that its accumulators hold z/2 and SiLU takes one FMA after the tanh.
#include <cuda_bf16.h>

#include <cstdint>

#include "mlp.cuh"

namespace mag {

namespace {

constexpr int kRows = 128;
constexpr int kH = 64;
constexpr long long kMbarSpin = 1LL << 24;

// ---- parameter layout (floats) -------------------------------------------------
// W1[64][4] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] w4[64] b4
constexpr int oW1 = 0, ob1 = oW1 + kH * 4, oW2 = ob1 + kH, ob2 = oW2 + kH * kH, oW3 = ob2 + kH,
              ob3 = oW3 + kH * kH, ow4 = ob3 + kH, ob4 = ow4 + kH;
static_assert(ob4 + 1 == kMlpParams, "parameter layout");

// ---- bf16 operand images (core-matrix K-major), element offsets -----------------
// W1p[64 out][16 in], W2[64][64], W3[64][64], W2T[64 in][64 out], W3T[64][64]
constexpr int kW1pElems = kH * 16, kWElems = kH * kH;
constexpr int bW1p = 0, bW2 = bW1p + kW1pElems, bW3 = bW2 + kWElems, bW2T = bW3 + kWElems,
              bW3T = bW2T + kWElems;
static_assert(bW3T + kWElems == kMlpOperandElems, "operand layout");

__host__ __device__ constexpr int core_off(int r, int k, int K) {
    // element offset of (row r, column k) in a K-major core-matrix image of width K
    return (r >> 3) * (K * 8) + (k >> 3) * 64 + (r & 7) * 8 + (k & 7);
}

// sigmoid(z) = (1 + tanh(z/2)) / 2 with the hardware tanh approximation (one MUFU
// operation; relative error about 2^-11, below the BF16 rounding every layer input gets).
__device__ __forceinline__ float sigmoid_fast(float z) {
    float t;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(0.5f * z));
    return 0.5f + 0.5f * t;
}
__device__ __forceinline__ float silu(float z) { return z * sigmoid_fast(z); }
__device__ __forceinline__ float dsilu(float z) {
    float s = sigmoid_fast(z);
    return s * (1.0f + z * (1.0f - s));
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint64_t smem_desc(const void *p, uint32_t lbo, uint32_t sbo) {
    uint64_t a = smem_u32(p);
    return ((a >> 4) & 0x3FFFull) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);  // version 1, no swizzle
}

// kind::f16 instruction descriptor: F32 accumulate, BF16 A and B, both K-major.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kH >> 3) << 17) |
                            ((uint32_t)(kRows >> 4) << 24);

__device__ __forceinline__ void mbar_init(uint64_t *bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait on phase `parity`; returns false if it gave up. limit = 0: kMbarSpin
// polls of the potentially blocking try_wait; limit > 0: that many polls of the
// non-blocking test_wait (a caller-set limit, small in tests, that really runs out).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, long long limit = 0) {
    uint32_t done = 0;
    if (limit > 0) {
        for (long long i = 0; i < limit; i++) {
            asm volatile(
                "{\n\t.reg .pred P1;\n\t"
                "mbarrier.test_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                "selp.b32 %0, 1, 0, P1;\n\t}"
                : "=r"(done)
                : "r"(smem_u32(bar)), "r"(parity)
                : "memory");
            if (done) return true;
        }
        return false;
    }
    for (long long i = 0; i < kMbarSpin; i++) {
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// D[128 x 64] (TMEM) = A[128 x K] * B[64 x K]^T, issued by one thread, completion on bar.
__device__ __forceinline__ void mma_issue(uint32_t tmem, const __nv_bfloat16 *A, const __nv_bfloat16 *B, int K,
                                          uint64_t *bar) {
    const uint32_t sbo = (uint32_t)K * 16;
    for (int kk = 0; kk < K / 16; kk++) {
        uint64_t ad = smem_desc(A + kk * 128, 128, sbo);  // 2 core matrices (256 B) per K=16 step
        uint64_t bd = smem_desc(B + kk * 128, 128, sbo);
        uint32_t acc = kk > 0 ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
            ::"r"(tmem), "l"(ad), "l"(bd), "r"(kIdesc), "r"(acc));
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// This thread's accumulator row (64 FP32 columns) from TMEM: four 16-column loads
// in flight, one wait.
__device__ __forceinline__ void tmem_row(uint32_t tmem, float out[kH]) {
    const uint32_t lane_base = (uint32_t)((threadIdx.x >> 5) * 32) << 16;
    uint32_t r[kH];
#pragma unroll
    for (int c = 0; c < kH; c += 16) {
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(r[c + 0]), "=r"(r[c + 1]), "=r"(r[c + 2]), "=r"(r[c + 3]), "=r"(r[c + 4]), "=r"(r[c + 5]),
              "=r"(r[c + 6]), "=r"(r[c + 7]), "=r"(r[c + 8]), "=r"(r[c + 9]), "=r"(r[c + 10]), "=r"(r[c + 11]),
              "=r"(r[c + 12]), "=r"(r[c + 13]), "=r"(r[c + 14]), "=r"(r[c + 15])
            : "r"(tmem + lane_base + (uint32_t)c));
    }
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < kH; i++) out[i] = __uint_as_float(r[i]);
}

// Columns c..c+15 of this thread's accumulator row from TMEM.
__device__ __forceinline__ void tmem_cols16(uint32_t tmem, int c, float out[16]) {
    const uint32_t lane_base = (uint32_t)((threadIdx.x >> 5) * 32) << 16;
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(tmem + lane_base + (uint32_t)c));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) out[i] = __uint_as_float(r[i]);
}

// A hidden layer's epilogue, 16 columns at a time (few live registers): z = acc + b,
// h = SiLU(z) as BF16 into the next layer's input image; z kept for training.
__device__ __forceinline__ void hidden_epilogue(uint32_t tmem, const float *bias, __nv_bfloat16 *img, int row_t,
                                                float *z_row) {
#pragma unroll
    for (int c = 0; c < kH; c += 16) {
        float z[16];
        tmem_cols16(tmem, c, z);
        __align__(16) __nv_bfloat162 hp[8];
#pragma unroll
        for (int i = 0; i < 16; i++) z[i] += bias[c + i];
#pragma unroll
        for (int i = 0; i < 8; i++) hp[i] = __floats2bfloat162_rn(silu(z[2 * i]), silu(z[2 * i + 1]));
        *reinterpret_cast<uint4 *>(img + core_off(row_t, c, kH)) = *reinterpret_cast<uint4 *>(hp);
        *reinterpret_cast<uint4 *>(img + core_off(row_t, c + 8, kH)) = *reinterpret_cast<uint4 *>(hp + 4);
        if (z_row)
#pragma unroll
            for (int i = 0; i < 16; i++) z_row[c + i] = z[i];
    }
}

// ---- inference epilogue: packed FP32 pairs (f32x2) ---------------------------------

__device__ __forceinline__ uint64_t pk2(float a, float b) {
    uint64_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void upk2(uint64_t v, float &a, float &b) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ uint64_t add2(uint64_t a, uint64_t b) {
    uint64_t r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ uint64_t fma2(uint64_t a, uint64_t b, uint64_t c) {
    uint64_t r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}

// SiLU of a hidden pair from its halved pre-activations h = z/2, packed as BF16 (z0's
// value in the low half). The inference kernel halves W1..W3 and b1..b3 (exact: a power of
// two), so the accumulators hold h, and z sigmoid(z) = h (1 + tanh h) = h + h tanh h: one
// single-precision tanh.approx per value and one packed FMA per pair.
// (A half-precision tanh of the pair, one MUFU operation for two values, was measured: 4 %
// faster at 8M rows, but its forward error, 6.7e-3 of max|y|, is above the 5.6e-3 bound.)
__device__ __forceinline__ uint32_t silu2h_bf16(uint64_t h) {
    float h0, h1, t0, t1;
    upk2(h, h0, h1);
    asm("tanh.approx.f32 %0, %1;" : "=f"(t0) : "f"(h0));
    asm("tanh.approx.f32 %0, %1;" : "=f"(t1) : "f"(h1));
    float p0, p1;
    upk2(fma2(h, pk2(t0, t1), h), p0, p1);
    uint32_t out;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(out) : "f"(p1), "f"(p0));
    return out;
}

// Inference form of hidden_epilogue: the same image, packed arithmetic on the halved
// accumulators and biases (h = z/2).
__device__ __forceinline__ void hidden_epilogue_infer(uint32_t tmem, const float *bias, __nv_bfloat16 *img,
                                                      int row_t) {
#pragma unroll
    for (int c = 0; c < kH; c += 16) {
        float z[16];
        tmem_cols16(tmem, c, z);
        __align__(16) uint32_t hp[8];
#pragma unroll
        for (int i = 0; i < 8; i += 2) {  // one 16-byte shared load of biases per two pairs
            const float4 b = *reinterpret_cast<const float4 *>(bias + c + 2 * i);
            hp[i] = silu2h_bf16(add2(pk2(z[2 * i], z[2 * i + 1]), pk2(b.x, b.y)));
            hp[i + 1] = silu2h_bf16(add2(pk2(z[2 * i + 2], z[2 * i + 3]), pk2(b.z, b.w)));
        }
        *reinterpret_cast<uint4 *>(img + core_off(row_t, c, kH)) = *reinterpret_cast<uint4 *>(hp);
        *reinterpret_cast<uint4 *>(img + core_off(row_t, c + 8, kH)) = *reinterpret_cast<uint4 *>(hp + 4);
    }
}

// Write this thread's row of 64 values as BF16 into a K=64 core-matrix image.
__device__ __forceinline__ void put_row64(__nv_bfloat16 *img, int row, const float v[kH]) {
#pragma unroll
    for (int kb = 0; kb < 8; kb++) {
        __align__(16) __nv_bfloat162 t[4];
#pragma unroll
        for (int i = 0; i < 4; i++) t[i] = __floats2bfloat162_rn(v[kb * 8 + 2 * i], v[kb * 8 + 2 * i + 1]);
        *reinterpret_cast<uint4 *>(img + core_off(row, kb * 8, kH)) = *reinterpret_cast<uint4 *>(t);
    }
}

struct Smem {
    __nv_bfloat16 act[kRows * kH];      // layer input image (K=64) or the K=16 input image
    __nv_bfloat16 w[2 * kWElems + kW1pElems];
    float vec[4 * kH + 1];              // b1 | b2 | b3 | w4 | b4 (forward kernel)
    uint64_t bar;
    uint32_t tmem;
    int fail;
};

__device__ __forceinline__ void load_ops(Smem &S, const __nv_bfloat16 *ops, int first, int count) {
    const uint4 *src = reinterpret_cast<const uint4 *>(ops + first);
    uint4 *dst = reinterpret_cast<uint4 *>(S.w);
    for (int i = threadIdx.x; i < count / 8; i += blockDim.x) dst[i] = src[i];
}

// load_ops with every weight halved (a power-of-two scale: exact for every weight above
// 2^-125 in magnitude, where BF16 values are normal).
__device__ __forceinline__ void load_ops_halved(Smem &S, const __nv_bfloat16 *ops, int first, int count) {
    const uint4 *src = reinterpret_cast<const uint4 *>(ops + first);
    uint4 *dst = reinterpret_cast<uint4 *>(S.w);
    const __nv_bfloat162 half2 = __floats2bfloat162_rn(0.5f, 0.5f);
    for (int i = threadIdx.x; i < count / 8; i += blockDim.x) {
        uint4 v = src[i];
        __nv_bfloat162 *p = reinterpret_cast<__nv_bfloat162 *>(&v);
#pragma unroll
        for (int j = 0; j < 4; j++) p[j] = __hmul2(p[j], half2);
        dst[i] = v;
    }
}

__device__ __forceinline__ void tmem_alloc(Smem &S) {
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem)),
                     "r"(kH));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
        tc_fence_before();  // the allocated address is read by every thread after the next barrier
    }
}

__device__ __forceinline__ void tmem_free(Smem &S) {
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x < 32) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(S.tmem), "r"(kH));
    }
}

// One layer: D = act * W^T; waits for completion; returns false on timeout. A wait
// that gives up first drains: the issued MMAs still read shared memory and write TMEM,
// so the kernel waits for their commit (default bound) before it leaves the tile loop
// and frees TMEM.
__device__ __forceinline__ bool run_layer(Smem &S, const __nv_bfloat16 *W, int K, uint32_t &phase,
                                          long long limit) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // smem writes -> tensor core
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x == 0) {
        tc_fence_after();
        mma_issue(S.tmem, S.act, W, K, &S.bar);
    }
    bool ok = mbar_wait(&S.bar, phase, limit);
    if (!ok) mbar_wait(&S.bar, phase);
    phase ^= 1u;
    tc_fence_after();
    // block-uniform outcome, so every thread leaves the tile loop together
    const bool any_fail = __syncthreads_or(ok ? 0 : 1) != 0;
    if (any_fail && threadIdx.x == 0) S.fail = 1;
    return !any_fail;
}

// The forward kernel's layer: one block-wide barrier per layer. The barrier before the
// MMA issue also settles whether any thread's previous wait gave up (`ok` is this
// thread's outcome of its last wait): then every thread leaves the tile loop together.
// A wait that gives up drains as in run_layer.
__device__ __forceinline__ bool run_layer_fwd(Smem &S, const __nv_bfloat16 *W, int K, uint32_t &phase,
                                              long long limit, bool &ok) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // smem writes -> tensor core
    tc_fence_before();
    if (__syncthreads_or(ok ? 0 : 1) != 0) {
        if (threadIdx.x == 0) S.fail = 1;
        return false;
    }
    if (threadIdx.x == 0) {
        tc_fence_after();
        mma_issue(S.tmem, S.act, W, K, &S.bar);
    }
    ok = mbar_wait(&S.bar, phase, limit);
    if (!ok) mbar_wait(&S.bar, phase);
    phase ^= 1u;
    tc_fence_after();
    return true;
}

// ---- forward ---------------------------------------------------------------------

// INFER: no pre-activations kept (prediction); the epilogues use the packed forms above.
template <bool INFER>
__global__ void __launch_bounds__(kRows, 6) k_mlp_forward(MlpForwardArgs a) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    Smem &S = *reinterpret_cast<Smem *>(smem_raw);
    const int t = threadIdx.x;
    if (t == 0) {
        mbar_init(&S.bar);
        S.fail = 0;
    }
    // all weight images: W1p | W2 | W3 (contiguous in the operand buffer). Inference halves
    // W1..W3 and b1..b3 (exact), so that the accumulators hold z/2 (silu2h_bf16).
    const float hs = INFER ? 0.5f : 1.0f;
    if (INFER) load_ops_halved(S, a.ops, bW1p, kW1pElems + 2 * kWElems);
    else load_ops(S, a.ops, bW1p, kW1pElems + 2 * kWElems);
    for (int i = t; i < kH; i += kRows) {
        S.vec[i] = hs * a.params[ob1 + i];
        S.vec[kH + i] = hs * a.params[ob2 + i];
        S.vec[2 * kH + i] = hs * a.params[ob3 + i];
        S.vec[3 * kH + i] = a.params[ow4 + i];
    }
    if (t == 0) S.vec[4 * kH] = a.params[ob4];
    tmem_alloc(S);
    __syncthreads();
    tc_fence_after();
    const __nv_bfloat16 *W1 = S.w, *W2 = S.w + kW1pElems, *W3 = S.w + kW1pElems + kWElems;
    const float *sb1 = S.vec, *sb2 = S.vec + kH, *sb3 = S.vec + 2 * kH, *sw4 = S.vec + 3 * kH;
    uint32_t phase = 0;
    bool ok = true;  // this thread's last tensor-core wait completed
    // The next tile's feature row (one 16-byte load: feature rows are 16 bytes, the buffer
    // 16-byte aligned) and output index are loaded one tile ahead, so their DRAM latency
    // overlaps the current tile's layers.
    const float4 *feats4 = reinterpret_cast<const float4 *>(a.feats);
    float4 f_next = make_float4(0.f, 0.f, 0.f, 0.f);
    int64_t dst_next = 0;
    {
        const int64_t r0 = (int64_t)blockIdx.x * kRows + t;
        if (r0 < a.n) {
            f_next = __ldg(feats4 + r0);
            dst_next = a.rows ? (int64_t)__ldg(a.rows + r0) : r0;
        }
    }
    for (int tile = blockIdx.x; tile * kRows < a.n; tile += gridDim.x) {
        const int64_t row = (int64_t)tile * kRows + t;
        const bool valid = row < a.n;
        const float4 f = f_next;
        const int64_t dst = dst_next;
        {
            const int64_t rn = row + (int64_t)gridDim.x * kRows;
            if (rn < a.n) {
                f_next = __ldg(feats4 + rn);
                dst_next = a.rows ? (int64_t)__ldg(a.rows + rn) : rn;
            }
        }
        float x[4] = {0, 0, 0, 0};
        if (valid) {
            x[0] = f.x;
            x[1] = f.y;
            x[2] = f.z;
            x[3] = f.w;
        }
        {  // input image, K = 16 (features 4..15 are zero)
            __align__(16) __nv_bfloat16 v[16];
            for (int i = 0; i < 16; i++) v[i] = __float2bfloat16_rn(i < 4 ? x[i] : 0.0f);
            *reinterpret_cast<uint4 *>(S.act + core_off(t, 0, 16)) = *reinterpret_cast<uint4 *>(v);
            *reinterpret_cast<uint4 *>(S.act + core_off(t, 8, 16)) = *reinterpret_cast<uint4 *>(v + 8);
        }
        float *zr = (a.z_out && valid) ? a.z_out + row * 3 * kH : nullptr;
        // layer 1
        // (a completed MMA has read its input image; the next layer's issue barrier orders
        // every thread's TMEM reads and image writes before the next MMA, also across tiles:
        // the next tile's first MMA is issued after its own barrier)
        if (!run_layer_fwd(S, W1, 16, phase, a.spin_limit, ok)) break;
        if (INFER) hidden_epilogue_infer(S.tmem, sb1, S.act, t);
        else hidden_epilogue(S.tmem, sb1, S.act, t, zr);
        // layer 2
        if (!run_layer_fwd(S, W2, kH, phase, a.spin_limit, ok)) break;
        if (INFER) hidden_epilogue_infer(S.tmem, sb2, S.act, t);
        else hidden_epilogue(S.tmem, sb2, S.act, t, zr ? zr + kH : nullptr);
        // layer 3 and the 64 -> 1 output, 16 columns at a time
        if (!run_layer_fwd(S, W3, kH, phase, a.spin_limit, ok)) break;
        float y = 0.0f;
        if (INFER) {  // pairs of halved pre-activations: single-precision tanh (the output is not rounded to BF16)
            uint64_t yacc = pk2(0.0f, 0.0f);
#pragma unroll
            for (int c = 0; c < kH; c += 16) {
                float z[16];
                tmem_cols16(S.tmem, c, z);
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    // biases and output weights by 16-byte shared loads, two pairs each
                    float4 b4, w4;
                    if ((i & 1) == 0) {
                        b4 = *reinterpret_cast<const float4 *>(sb3 + c + 2 * i);
                        w4 = *reinterpret_cast<const float4 *>(sw4 + c + 2 * i);
                    }
                    const float2 b = (i & 1) ? make_float2(b4.z, b4.w) : make_float2(b4.x, b4.y);
                    const float2 w = (i & 1) ? make_float2(w4.z, w4.w) : make_float2(w4.x, w4.y);
                    const uint64_t hh = add2(pk2(z[2 * i], z[2 * i + 1]), pk2(b.x, b.y));  // z/2
                    float h0, h1, t0, t1;
                    upk2(hh, h0, h1);
                    asm("tanh.approx.f32 %0, %1;" : "=f"(t0) : "f"(h0));
                    asm("tanh.approx.f32 %0, %1;" : "=f"(t1) : "f"(h1));
                    yacc = fma2(pk2(w.x, w.y), fma2(hh, pk2(t0, t1), hh), yacc);  // w4 silu(z)
                }
            }
            float y0, y1;
            upk2(yacc, y0, y1);
            y = y0 + y1;
        } else {
#pragma unroll
            for (int c = 0; c < kH; c += 16) {
                float z[16];
                tmem_cols16(S.tmem, c, z);
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    z[i] += sb3[c + i];
                    y += sw4[c + i] * silu(z[i]);
                }
                if (zr)
#pragma unroll
                    for (int i = 0; i < 16; i++) zr[2 * kH + c + i] = z[i];
            }
        }
        y += S.vec[4 * kH];
        if (valid && ok) {  // (after a wait that gave up, the kernel reports a timeout instead)
            if (a.y_out) a.y_out[row] = y;
            if (a.nu_out) {  // nu = exp(y * scale + shift), clamped to [nu_min, nu_max]
                double v = exp((double)y * a.y_scale + a.y_shift);
                v = v < a.nu_min ? a.nu_min : (v > a.nu_max ? a.nu_max : v);
                a.nu_out[dst] = v;
            }
        }
    }
    if (!ok) S.fail = 1;  // a wait of the last layer gave up
    tmem_free(S);         // (its barrier makes S.fail visible to thread 0)
    if (t == 0 && S.fail && a.err) atomicExch(a.err, 1);
}

// ---- backward --------------------------------------------------------------------

struct BwdSmem {
    Smem s;
    float dz[kRows * kH];   // current layer's dZ (FP32)
    float hin[kRows * kH];  // current layer's input (BF16-rounded, held as FP32)
};

// dW[o][i] += sum_r dz[r][o] * hin[r][i] (i < nin), db[o] += sum_r dz[r][o]; FP32, fixed row order.
__device__ __forceinline__ void weight_grads(const BwdSmem &S, int nin, float *gW, float *gb) {
    const int t = threadIdx.x;
    const int o = t >> 1, i0 = (t & 1) * 32;
    if (i0 < nin) {
        float acc[32];
        for (int i = 0; i < 32; i++) acc[i] = 0.0f;
        for (int r = 0; r < kRows; r++) {
            float d = S.dz[r * kH + o];
            for (int i = 0; i < 32 && i0 + i < nin; i++) acc[i] += d * S.hin[r * kH + i0 + i];
        }
        for (int i = 0; i < 32 && i0 + i < nin; i++) gW[o * nin + i0 + i] += acc[i];
    }
    if ((t & 1) == 0) {
        float b = 0.0f;
        for (int r = 0; r < kRows; r++) b += S.dz[r * kH + o];
        gb[o] += b;
    }
}

__global__ void __launch_bounds__(kRows, 1) k_mlp_backward(MlpBackwardArgs a) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    BwdSmem &B = *reinterpret_cast<BwdSmem *>(smem_raw);
    Smem &S = B.s;
    const int t = threadIdx.x;
    if (t == 0) {
        mbar_init(&S.bar);
        S.fail = 0;
    }
    load_ops(S, a.ops, bW2T, 2 * kWElems);  // W2T | W3T
    tmem_alloc(S);
    __syncthreads();
    tc_fence_after();
    const __nv_bfloat16 *W2T = S.w, *W3T = S.w + kWElems;
    const float *P = a.params;
    float *G = a.grad_partial + (size_t)blockIdx.x * kMlpParams;  // this CTA's partial gradient
    for (int i = t; i < kMlpParams; i += kRows) G[i] = 0.0f;
    __syncthreads();
    uint32_t phase = 0;
    for (int tile = blockIdx.x; tile * kRows < a.n; tile += gridDim.x) {
        const int64_t row = (int64_t)tile * kRows + t;
        const bool valid = row < a.n;
        float z3[kH], z2[kH], z1[kH], dz[kH], dh[kH];
        for (int o = 0; o < kH; o++) {
            z1[o] = valid ? a.z[(row * 3 + 0) * kH + o] : 0.0f;
            z2[o] = valid ? a.z[(row * 3 + 1) * kH + o] : 0.0f;
            z3[o] = valid ? a.z[(row * 3 + 2) * kH + o] : 0.0f;
        }
        const float dy = valid ? (a.y[row] - a.target[row]) * a.loss_scale : 0.0f;
        // last layer: dw4, db4, dz3
        for (int o = 0; o < kH; o++) dz[o] = dy * P[ow4 + o] * dsilu(z3[o]);
        {
            float h3[kH];
            for (int o = 0; o < kH; o++) h3[o] = silu(z3[o]);
            // dw4 / db4 reduced over rows through shared memory (fixed order)
            for (int o = 0; o < kH; o++) B.dz[t * kH + o] = dy * h3[o];
            __syncthreads();
            if (t < kH) {
                float s = 0.0f;
                for (int r = 0; r < kRows; r++) s += B.dz[r * kH + t];
                G[ow4 + t] += s;
            }
            if (t == kH) {
                float s = 0.0f;
                for (int r = 0; r < kRows; r++) {
                    int64_t rr = (int64_t)tile * kRows + r;
                    s += rr < a.n ? (a.y[rr] - a.target[rr]) * a.loss_scale : 0.0f;
                }
                G[ob4] += s;
            }
            __syncthreads();
        }
        // layer 3: dW3 += dz3^T h2, dh2 = dz3 W3
        for (int o = 0; o < kH; o++) {
            B.dz[t * kH + o] = dz[o];
            B.hin[t * kH + o] = __bfloat162float(__float2bfloat16_rn(silu(z2[o])));
        }
        __syncthreads();
        weight_grads(B, kH, G + oW3, G + ob3);
        put_row64(S.act, t, dz);
        if (!run_layer(S, W3T, kH, phase, a.spin_limit)) break;
        tmem_row(S.tmem, dh);
        tc_fence_before();
        __syncthreads();
        for (int o = 0; o < kH; o++) dz[o] = dh[o] * dsilu(z2[o]);
        // layer 2: dW2 += dz2^T h1, dh1 = dz2 W2
        for (int o = 0; o < kH; o++) {
            B.dz[t * kH + o] = dz[o];
            B.hin[t * kH + o] = __bfloat162float(__float2bfloat16_rn(silu(z1[o])));
        }
        __syncthreads();
        weight_grads(B, kH, G + oW2, G + ob2);
        put_row64(S.act, t, dz);
        if (!run_layer(S, W2T, kH, phase, a.spin_limit)) break;
        tmem_row(S.tmem, dh);
        tc_fence_before();
        __syncthreads();
        for (int o = 0; o < kH; o++) dz[o] = dh[o] * dsilu(z1[o]);
        // layer 1: dW1 += dz1^T x
        for (int o = 0; o < kH; o++) {
            B.dz[t * kH + o] = dz[o];
            B.hin[t * kH + o] = (o < 4 && valid) ? __bfloat162float(__float2bfloat16_rn(a.feats[row * 4 + o])) : 0.0f;
        }
        __syncthreads();
        weight_grads(B, 4, G + oW1, G + ob1);
        __syncthreads();
    }
    if (t == 0 && S.fail && a.err) atomicExch(a.err, 1);
    tmem_free(S);
}

// grad[p] = sum over CTAs (fixed order) of the partials.
__global__ void k_mlp_reduce(const float *__restrict__ partial, int nparts, float *__restrict__ grad) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kMlpParams) return;
    float s = 0.0f;
    for (int c = 0; c < nparts; c++) s += partial[(size_t)c * kMlpParams + p];
    grad[p] = s;
}

// Adam step on the FP32 master weights.
__global__ void k_mlp_adam(float *__restrict__ params, const float *__restrict__ grad, float *__restrict__ m,
                           float *__restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kMlpParams) return;
    float g = grad[p];
    float mm = b1 * m[p] + (1.0f - b1) * g;
    float vv = b2 * v[p] + (1.0f - b2) * g * g;
    m[p] = mm;
    v[p] = vv;
    params[p] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
}

// BF16 operand images from the FP32 master weights.
__global__ void k_mlp_pack(const float *__restrict__ P, __nv_bfloat16 *__restrict__ ops) {
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < kH * 16) {  // W1p [64 out][16 in], inputs 4..15 zero
        int o = idx / 16, i = idx % 16;
        ops[bW1p + core_off(o, i, 16)] = __float2bfloat16_rn(i < 4 ? P[oW1 + o * 4 + i] : 0.0f);
    }
    if (idx < kH * kH) {
        int o = idx / kH, i = idx % kH;
        ops[bW2 + core_off(o, i, kH)] = __float2bfloat16_rn(P[oW2 + o * kH + i]);
        ops[bW3 + core_off(o, i, kH)] = __float2bfloat16_rn(P[oW3 + o * kH + i]);
        // transposed images: row = input feature i, column = output feature o
        ops[bW2T + core_off(i, o, kH)] = __float2bfloat16_rn(P[oW2 + o * kH + i]);
        ops[bW3T + core_off(i, o, kH)] = __float2bfloat16_rn(P[oW3 + o * kH + i]);
    }
}

__global__ void k_mlp_gather(const float4 *__restrict__ feats, const float *__restrict__ target,
                             const int64_t *__restrict__ perm, int64_t off, int64_t b, float4 *__restrict__ xb,
                             float *__restrict__ tb) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= b) return;
    const int64_t r = perm[off + i];
    xb[i] = feats[r];
    tb[i] = target[r];
}

// One CTA of 1024 threads: strided partial sums, then a fixed tree over the shared array.
__global__ void __launch_bounds__(1024) k_mlp_sqerr(const float *__restrict__ y, const float *__restrict__ t,
                                                    int64_t b, float *__restrict__ acc) {
    __shared__ float part[1024];
    float v = 0.0f;
    for (int64_t i = threadIdx.x; i < b; i += 1024) {
        const float d = y[i] - t[i];
        v += d * d;
    }
    part[threadIdx.x] = v;
    __syncthreads();
    for (int w = 512; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *acc += part[0];
}

}  // namespace

int mlp_gather(const float *feats, const float *target, const int64_t *perm, int64_t off, int64_t b, float *xb,
               float *tb, cudaStream_t s) {
    k_mlp_gather<<<(unsigned)((b + 255) / 256), 256, 0, s>>>(reinterpret_cast<const float4 *>(feats), target, perm,
                                                            off, b, reinterpret_cast<float4 *>(xb), tb);
    return cudaPeekAtLastError() == cudaSuccess ? MAG_OK : MAG_E_CUDA;
}

int mlp_sqerr(const float *y, const float *t, int64_t b, float *acc, cudaStream_t s) {
    k_mlp_sqerr<<<1, 1024, 0, s>>>(y, t, b, acc);
    return cudaPeekAtLastError() == cudaSuccess ? MAG_OK : MAG_E_CUDA;
}

size_t mlp_forward_smem() { return sizeof(Smem) + 1024; }
size_t mlp_backward_smem() { return sizeof(BwdSmem) + 1024; }

int mlp_pack(const float *params, __nv_bfloat16 *ops, cudaStream_t s) {
    k_mlp_pack<<<(kH * kH + 255) / 256, 256, 0, s>>>(params, ops);
    return cudaPeekAtLastError() == cudaSuccess ? MAG_OK : MAG_E_CUDA;
}

int mlp_forward(const MlpForwardArgs &a, int grid, cudaStream_t s) {
    size_t sm = sizeof(Smem);
    auto kern = a.z_out ? k_mlp_forward<false> : k_mlp_forward<true>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    // The CTAs loop over tiles; launching several waves of them (48 per SM, about 9 tiles
    // each at 8M rows) lets SMs that finish early take more CTAs, which evens out the tail
    // (measured at 7.99M rows: 8 per SM 0.514 ms, 24 0.474, 48 0.467, 96 0.470, one tile per
    // CTA 0.654: the per-CTA weight load and TMEM allocation then dominate). A build option.
#ifndef MAG_MLP_CTAS_PER_SM
#define MAG_MLP_CTAS_PER_SM 48
#endif
    int dev = 0, nsm = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
        nsm > 0 && grid > MAG_MLP_CTAS_PER_SM * nsm)
        grid = MAG_MLP_CTAS_PER_SM * nsm;
    kern<<<grid, kRows, sm, s>>>(a);
    return cudaPeekAtLastError() == cudaSuccess ? MAG_OK : MAG_E_CUDA;
}

int mlp_backward(const MlpBackwardArgs &a, int grid, cudaStream_t s) {
    size_t sm = sizeof(BwdSmem);
    cudaFuncSetAttribute(k_mlp_backward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_mlp_backward<<<grid, kRows, sm, s>>>(a);
    if (cudaPeekAtLastError() != cudaSuccess) return MAG_E_CUDA;
    k_mlp_reduce<<<(kMlpParams + 255) / 256, 256, 0, s>>>(a.grad_partial, grid, a.grad);
    return cudaPeekAtLastError() == cudaSuccess ? MAG_OK : MAG_E_CUDA;
}

int mlp_adam(float *params, const float *grad, float *m, float *v, float lr, float b1, float b2, float eps,
             int step, cudaStream_t s) {
    float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    k_mlp_adam<<<(kMlpParams + 255) / 256, 256, 0, s>>>(params, grad, m, v, lr, b1, b2, eps, c1, c2);
    return cudaPeekAtLastError() == cudaSuccess ? MAG_OK : MAG_E_CUDA;
}

}  // namespace mag
