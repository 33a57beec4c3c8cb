// The learned edge proposal's network: a 10 -> 64 -> 64 -> 64 -> 32 MLP with
// ReLU hidden layers and a softmax output, run and trained on the tensor
// cores (dr_mlp.cu).  Parameters are one flat f32 array (PyTorch's
// nn.Linear convention, weight[out][in] row-major, then bias):
//   W1 [64][16] (inputs 10..15 are zero padding), b1 [64],
//   W2 [64][64], b2 [64], W3 [64][64], b3 [64], W4 [32][64], b4 [32].
// The kernels read a bf16 copy of the weights packed in the tensor cores'
// shared-memory layout (dr_mlp_pack).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#define DR_MLP_IN 16
#define DR_MLP_FEATURES 10
#define DR_MLP_HIDDEN 64
#define DR_MLP_OUT 32

enum : int {
    kMlpW1 = 0,
    kMlpB1 = kMlpW1 + 64 * 16,
    kMlpW2 = kMlpB1 + 64,
    kMlpB2 = kMlpW2 + 64 * 64,
    kMlpW3 = kMlpB2 + 64,
    kMlpB3 = kMlpW3 + 64 * 64,
    kMlpW4 = kMlpB3 + 64,
    kMlpB4 = kMlpW4 + 32 * 64,
    kMlpParams = kMlpB4 + 32
};
// packed bf16 weight images (bytes)
enum : int {
    kImgW1 = 0,
    kImgW2 = kImgW1 + 64 * 16 * 2,
    kImgW3 = kImgW2 + 64 * 64 * 2,
    kImgW4 = kImgW3 + 64 * 64 * 2,
    kImgBytes = kImgW4 + 32 * 64 * 2
};

// Status bit set when a tensor-core wait timed out.
#define DR_MLP_STATUS_TIMEOUT 16

cudaError_t dr_mlp_pack(const float *params, uint8_t *wimg, cudaStream_t st);
// Rows x[n][16] (bf16) -> logits[n][32] (f32, may be null) and softmax
// probabilities probs[n][32] (bf16, may be null).
cudaError_t dr_mlp_infer(const uint8_t *wimg, const float *params, const __nv_bfloat16 *x, long long n, float *logits,
                         __nv_bfloat16 *probs, int *status, int num_sms, cudaStream_t st);
// Gradient of the loss  sum_r sum_s -t[r][s] log q[r][s] / total  (q the
// softmax output, total = *target_total, the sum of all targets) w.r.t. the
// parameters, added to grads[kMlpParams]; the loss is added to *loss.
cudaError_t dr_mlp_grad(const uint8_t *wimg, const float *params, const __nv_bfloat16 *x, const float *targets,
                        long long n, const float *target_total, float *grads, float *loss, int *status, int num_sms,
                        cudaStream_t st);
cudaError_t dr_mlp_to_bf16(const float *x, __nv_bfloat16 *y, long long n, cudaStream_t st);
// *out = sum of x[0..n) (out is zeroed first)
cudaError_t dr_mlp_sum(const float *x, long long n, float *out, cudaStream_t st);
// One Adam step on params with grads (moments m, v); step counts from 1.
cudaError_t dr_mlp_adam(float *params, const float *grads, float *m, float *v, int step, float lr, cudaStream_t st);
