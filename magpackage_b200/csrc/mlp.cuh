// Reluctivity predictor MLP: launch interface (mlp.cu).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "common.cuh"

namespace mag {

constexpr int kMlpParams = 64 * 4 + 64 + 64 * 64 + 64 + 64 * 64 + 64 + 64 + 1;  // 8705
constexpr int kMlpOperandElems = 64 * 16 + 4 * 64 * 64;                       // BF16 images

struct MlpForwardArgs {
    const float *feats;     // [n][4]
    int64_t n;
    const float *params;    // FP32 master weights
    const __nv_bfloat16 *ops;
    float *y_out;           // [n] or NULL
    float *z_out;           // [n][3][64] pre-activations (training) or NULL
    double *nu_out;         // nu scattered to rows[i] (or i) or NULL
    const int32_t *rows;
    double y_scale, y_shift, nu_min, nu_max;
    int *err;
    long long spin_limit;   // polls before a tensor-core wait gives up; 0 = the default bound
};

struct MlpBackwardArgs {
    const float *feats, *z, *y, *target;
    int64_t n;
    float loss_scale;       // dL/dy = (y - target) * loss_scale
    const float *params;
    const __nv_bfloat16 *ops;
    float *grad_partial;    // [grid][kMlpParams]
    float *grad;            // [kMlpParams]
    int *err;
    long long spin_limit;
};

size_t mlp_forward_smem();
size_t mlp_backward_smem();
int mlp_pack(const float *params, __nv_bfloat16 *ops, cudaStream_t s);
int mlp_forward(const MlpForwardArgs &a, int grid, cudaStream_t s);
int mlp_backward(const MlpBackwardArgs &a, int grid, cudaStream_t s);
int mlp_adam(float *params, const float *grad, float *m, float *v, float lr, float b1, float b2, float eps,
             int step, cudaStream_t s);
// xb[i] = feats[perm[off + i]] (16-byte rows), tb[i] = target[perm[off + i]], i < b.
int mlp_gather(const float *feats, const float *target, const int64_t *perm, int64_t off, int64_t b, float *xb,
               float *tb, cudaStream_t s);
// *acc += sum_i (y_i - t_i)^2 over i < b, in a fixed order (one CTA).
int mlp_sqerr(const float *y, const float *t, int64_t b, float *acc, cudaStream_t s);

}  // namespace mag
