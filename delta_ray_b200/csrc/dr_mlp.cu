// Tensor-core kernels of the learned edge proposal's MLP (sm_100a).
//
// One CTA of 128 threads handles tiles of 128 rows: thread t owns row t.  The
// weights are staged once per CTA in shared memory (bf16, interleaved
// layout, dr_tcgen05.cuh); each layer is tcgen05.mma (M = 128 rows, K = 16 per
// instruction) from shared memory into a TMEM accumulator, issued by one
// thread and committed to an mbarrier; every thread then loads its row from
// TMEM (tcgen05.ld), adds the bias, applies ReLU and writes the bf16
// activation back to shared memory as the next layer's A operand.
//
// The gradient kernel keeps the three hidden activations and runs the
// backward pass on the tensor cores as well: dH = dZ * W reads the weight
// image as an MN-major B operand, and dW = dZ^T * H (M = 64 output features,
// K = the tile's 128 rows) reads dZ and H as MN-major operands; its TMEM
// accumulator uses the M = 64 layout (rows 16w..16w+15 in lanes 32w..32w+15).
// Each tile's weight gradient is added to the global f32 gradient with
// atomics.  All waits are bounded: on a timeout the kernel sets
// DR_MLP_STATUS_TIMEOUT in *status, waits once more, frees its TMEM and returns.
#include "dr_mlp.h"
#include "dr_tcgen05.cuh"

#include <atomic>

namespace {

constexpr int kTile = 128;
constexpr long long kWaitNs = 2000000000ll;  // 2 s per wait

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait on the mbarrier phase, made uniform across the CTA.
__device__ bool wait_mma(uint32_t mbar, uint32_t &phase) {
    bool ok = false;
    unsigned long long t0 = global_ns();
    while (true) {
        if (tc::mbar_wait(mbar, phase, 64)) {
            ok = true;
            break;
        }
        if (global_ns() - t0 > (unsigned long long)kWaitNs) break;
    }
    ok = __syncthreads_and(ok);
    if (ok) phase ^= 1u;
    tc::fence_after_sync();
    return ok;
}

// Generic shared-memory writes -> visible to the tensor cores; TMEM reads of
// every thread finished before the next MMA is issued.
__device__ __forceinline__ void sync_for_mma() {
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
}

__device__ __forceinline__ uint32_t lane_base(uint32_t tmem) { return tmem + ((threadIdx.x & ~31u) << 16); }

// D[tmem] = A (128 x K, K-major) * W^T (W: N x K image), K in steps of 16.
__device__ __forceinline__ void issue_forward(uint32_t tmem, uint32_t a, int K, uint32_t w, int N) {
    const uint32_t id = tc::idesc_bf16(128, N, 0, 0);
    for (int j = 0; j < K / 16; j++)
        tc::mma_bf16(tmem, tc::sdesc_k(a + j * 256, K), tc::sdesc_k(w + j * 256, K), id, j > 0);
}

// 64 f32 columns of this thread's row.
__device__ __forceinline__ void ld_row64(uint32_t tmem, float *v) {
    uint32_t ta = lane_base(tmem);
    tc::tmem_ld32(ta, v);
    tc::tmem_ld32(ta + 32, v + 32);
}

// bias + ReLU, bf16 row into H (128 x 64)
__device__ __forceinline__ void epilogue_relu(uint32_t tmem, const float *bias, uint8_t *H) {
    float v[64];
    ld_row64(tmem, v);
#pragma unroll
    for (int c = 0; c < 64; c++) v[c] = fmaxf(v[c] + bias[c], 0.f);
#pragma unroll
    for (int c = 0; c < 64; c += 8) tc::st_row8(H, threadIdx.x, c, 64, v + c);
}

__device__ __forceinline__ void load_weights(const uint8_t *wimg, const float *params, uint8_t *sW, float *sB) {
    for (int i = threadIdx.x; i < kImgBytes / 16; i += blockDim.x)
        reinterpret_cast<uint4 *>(sW)[i] = reinterpret_cast<const uint4 *>(wimg)[i];
    for (int i = threadIdx.x; i < 224; i += blockDim.x) {
        int src = i < 64 ? kMlpB1 + i : i < 128 ? kMlpB2 + i - 64 : i < 192 ? kMlpB3 + i - 128 : kMlpB4 + i - 192;
        sB[i] = params[src];
    }
}

__device__ __forceinline__ void load_features(const __nv_bfloat16 *x, long long row, long long n, uint8_t *sX) {
    uint4 lo = make_uint4(0, 0, 0, 0), hi = lo;
    if (row < n) {
        const uint4 *src = reinterpret_cast<const uint4 *>(x + row * DR_MLP_IN);
        lo = src[0];
        hi = src[1];
    }
    *reinterpret_cast<uint4 *>(sX + tc::imat_offset(threadIdx.x, 0, 16)) = lo;
    *reinterpret_cast<uint4 *>(sX + tc::imat_offset(threadIdx.x, 8, 16)) = hi;
}

// Forward through the three hidden layers of one tile (features already in
// sX); the last hidden activation ends in H3.  Returns false on a timeout.
__device__ bool hidden_layers(uint32_t tmem, uint32_t mbar, uint32_t &phase, const uint8_t *sW, const float *sB,
                              uint8_t *sX, uint8_t *H1, uint8_t *H2, uint8_t *H3) {
    const uint32_t aW = tc::smem_addr(sW);
    sync_for_mma();
    if (threadIdx.x == 0) {
        issue_forward(tmem, tc::smem_addr(sX), 16, aW + kImgW1, 64);
        tc::commit(mbar);
    }
    if (!wait_mma(mbar, phase)) return false;
    epilogue_relu(tmem, sB, H1);
    sync_for_mma();
    if (threadIdx.x == 0) {
        issue_forward(tmem, tc::smem_addr(H1), 64, aW + kImgW2, 64);
        tc::commit(mbar);
    }
    if (!wait_mma(mbar, phase)) return false;
    epilogue_relu(tmem, sB + 64, H2);
    sync_for_mma();
    if (threadIdx.x == 0) {
        issue_forward(tmem, tc::smem_addr(H2), 64, aW + kImgW3, 64);
        tc::commit(mbar);
    }
    if (!wait_mma(mbar, phase)) return false;
    epilogue_relu(tmem, sB + 128, H3);
    sync_for_mma();
    if (threadIdx.x == 0) {
        issue_forward(tmem, tc::smem_addr(H3), 64, aW + kImgW4, 32);
        tc::commit(mbar);
    }
    return wait_mma(mbar, phase);
}

__device__ void softmax32(const float *z, float *q) {
    float m = z[0];
#pragma unroll
    for (int s = 1; s < 32; s++) m = fmaxf(m, z[s]);
    float sum = 0.f;
#pragma unroll
    for (int s = 0; s < 32; s++) {
        q[s] = __expf(z[s] - m);
        sum += q[s];
    }
    float inv = 1.f / sum;
#pragma unroll
    for (int s = 0; s < 32; s++) q[s] *= inv;
}

// On a timeout: record it, give the outstanding commit one more bounded wait.
__device__ void on_timeout(uint32_t mbar, uint32_t phase, int *status) {
    if (threadIdx.x == 0 && status) atomicOr(status, DR_MLP_STATUS_TIMEOUT);
    unsigned long long t0 = global_ns();
    while (!tc::mbar_wait(mbar, phase, 64) && global_ns() - t0 < (unsigned long long)kWaitNs) {
    }
}

constexpr int kInferSmem = kImgBytes + 1024 + 4096 + 3 * 16384 + 64;

__global__ void __launch_bounds__(128) k_mlp_infer(const uint8_t *wimg, const float *params, const __nv_bfloat16 *x,
                                                   long long n, float *logits, __nv_bfloat16 *probs, int *status) {
    extern __shared__ __align__(1024) uint8_t sm[];
    uint8_t *sW = sm;
    float *sB = reinterpret_cast<float *>(sm + kImgBytes);
    uint8_t *sX = sm + kImgBytes + 1024;
    uint8_t *H1 = sX + 4096, *H2 = H1 + 16384, *H3 = H2 + 16384;
    uint64_t *bar = reinterpret_cast<uint64_t *>(H3 + 16384);
    uint32_t *slot = reinterpret_cast<uint32_t *>(bar + 1);
    const uint32_t mbar = tc::smem_addr(bar);
    if (threadIdx.x < 32) tc::tmem_alloc(tc::smem_addr(slot), 64);
    if (threadIdx.x == 0) tc::mbar_init(mbar, 1);
    load_weights(wimg, params, sW, sB);
    sync_for_mma();
    const uint32_t tmem = *slot;
    uint32_t phase = 0;
    bool ok = true;
    for (long long t0 = (long long)blockIdx.x * kTile; t0 < n; t0 += (long long)gridDim.x * kTile) {
        long long row = t0 + threadIdx.x;
        load_features(x, row, n, sX);
        if (!hidden_layers(tmem, mbar, phase, sW, sB, sX, H1, H2, H3)) {
            ok = false;
            break;
        }
        float z[32], q[32];
        tc::tmem_ld32(lane_base(tmem), z);
#pragma unroll
        for (int s = 0; s < 32; s++) z[s] += sB[192 + s];
        if (row < n) {
            if (logits) {
#pragma unroll
                for (int s = 0; s < 32; s += 4)
                    *reinterpret_cast<float4 *>(logits + row * 32 + s) = make_float4(z[s], z[s + 1], z[s + 2], z[s + 3]);
            }
            if (probs) {
                softmax32(z, q);
                __nv_bfloat162 h[16];
#pragma unroll
                for (int s = 0; s < 16; s++) h[s] = __floats2bfloat162_rn(q[2 * s], q[2 * s + 1]);
                uint4 *dst = reinterpret_cast<uint4 *>(probs + row * 32);
#pragma unroll
                for (int s = 0; s < 4; s++) dst[s] = reinterpret_cast<uint4 *>(h)[s];
            }
        }
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
    }
    if (!ok) on_timeout(mbar, phase, status);
    tc::fence_before_sync();
    __syncthreads();
    if (threadIdx.x < 32) tc::tmem_free(tmem, 64);
}

constexpr int kGradSmem = kImgBytes + 1024 + 1024 + 4096 + 4 * 16384 + 64;

__global__ void __launch_bounds__(128) k_mlp_grad(const uint8_t *wimg, const float *params, const __nv_bfloat16 *x,
                                                  const float *targets, long long n, const float *target_total,
                                                  float *grads, float *loss, int *status) {
    extern __shared__ __align__(1024) uint8_t sm[];
    uint8_t *sW = sm;
    float *sB = reinterpret_cast<float *>(sm + kImgBytes);
    float *sDB = reinterpret_cast<float *>(sm + kImgBytes + 1024);
    uint8_t *sX = sm + kImgBytes + 2048;
    uint8_t *H1 = sX + 4096, *H2 = H1 + 16384, *H3 = H2 + 16384, *sD = H3 + 16384;
    uint64_t *bar = reinterpret_cast<uint64_t *>(sD + 16384);
    uint32_t *slot = reinterpret_cast<uint32_t *>(bar + 1);
    const uint32_t mbar = tc::smem_addr(bar);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid < 32) tc::tmem_alloc(tc::smem_addr(slot), 128);
    if (tid == 0) tc::mbar_init(mbar, 1);
    load_weights(wimg, params, sW, sB);
    for (int i = tid; i < 224; i += blockDim.x) sDB[i] = 0.f;
    sync_for_mma();
    const uint32_t tmem = *slot, tmem_w = tmem + 64;  // [0, 64): forward / dH; [64, 128): dW (M = 64 layout)
    const uint32_t aW = tc::smem_addr(sW), aX = tc::smem_addr(sX), aD = tc::smem_addr(sD);
    const uint32_t aH[3] = {tc::smem_addr(H1), tc::smem_addr(H2), tc::smem_addr(H3)};
    uint8_t *Hs[3] = {H1, H2, H3};
    const float total = *target_total;
    const float inv_total = total > 0.f ? 1.f / total : 0.f;
    float loss_acc = 0.f;
    uint32_t phase = 0;
    bool ok = true;
    for (long long t0 = (long long)blockIdx.x * kTile; t0 < n && ok; t0 += (long long)gridDim.x * kTile) {
        long long row = t0 + tid;
        load_features(x, row, n, sX);
        if (!hidden_layers(tmem, mbar, phase, sW, sB, sX, H1, H2, H3)) {
            ok = false;
            break;
        }
        // softmax cross-entropy against the row's targets
        float z[32], q[32], t[32];
        tc::tmem_ld32(lane_base(tmem), z);
#pragma unroll
        for (int s = 0; s < 32; s++) z[s] += sB[192 + s];
        softmax32(z, q);
        float T = 0.f;
#pragma unroll
        for (int s = 0; s < 32; s++) {
            t[s] = row < n ? targets[row * 32 + s] : 0.f;
            T += t[s];
        }
#pragma unroll
        for (int s = 0; s < 32; s++) {
            if (t[s] > 0.f) loss_acc -= t[s] * __logf(fmaxf(q[s], 1e-30f)) * inv_total;
            z[s] = (T * q[s] - t[s]) * inv_total;  // dZ4
            atomicAdd(&sDB[192 + s], z[s]);
        }
#pragma unroll
        for (int c = 0; c < 32; c += 8) tc::st_row8(sD, tid, c, 32, z + c);
        // layers 4..1 backwards: dW_l = dZ_l^T H_{l-1}, dH_{l-1} = dZ_l W_l
        for (int l = 3; l >= 0; l--) {
            const int out = l == 3 ? 32 : 64;
            const int in = l == 0 ? 16 : 64;
            const uint32_t aIn = l == 0 ? aX : aH[l - 1];
            const uint32_t aWl = aW + (l == 0 ? kImgW1 : l == 1 ? kImgW2 : l == 2 ? kImgW3 : kImgW4);
            sync_for_mma();
            if (tid == 0) {
                if (l == 3) {  // dW4^T (64 x 32) = H3^T dZ4
                    const uint32_t id = tc::idesc_bf16(64, 32, 1, 1);
                    for (int j = 0; j < 8; j++)
                        tc::mma_bf16(tmem_w, tc::sdesc_mn(aIn + j * 2 * 1024, 64), tc::sdesc_mn(aD + j * 2 * 512, 32),
                                     id, j > 0);
                } else {  // dW_l (64 x in) = dZ_l^T H_{l-1}
                    const uint32_t id = tc::idesc_bf16(64, in, 1, 1);
                    for (int j = 0; j < 8; j++)
                        tc::mma_bf16(tmem_w, tc::sdesc_mn(aD + j * 2 * 1024, 64),
                                     tc::sdesc_mn(aIn + j * 2 * (in / 8) * 128, in), id, j > 0);
                }
                if (l > 0) {  // dH_{l-1} (128 x 64) = dZ_l (128 x out) W_l (out x 64)
                    const uint32_t id = tc::idesc_bf16(128, 64, 0, 1);
                    for (int j = 0; j < out / 16; j++)
                        tc::mma_bf16(tmem, tc::sdesc_k(aD + j * 256, out), tc::sdesc_mn(aWl + j * 2 * 1024, 64), id,
                                     j > 0);
                }
                tc::commit(mbar);
            }
            if (!wait_mma(mbar, phase)) {
                ok = false;
                break;
            }
            // weight gradient: lanes 0..15 of warp w hold rows 16w..16w+15
            {
                float g[64];
                uint32_t ta = lane_base(tmem_w);
                tc::tmem_ld32(ta, g);
                if (l == 1 || l == 2) tc::tmem_ld32(ta + 32, g + 32);
                if (lane < 16) {
                    int r = 16 * warp + lane;
                    if (l == 3) {  // r = input feature, g[o] = dW4[o][r]
                        for (int o = 0; o < 32; o++) atomicAdd(grads + kMlpW4 + o * 64 + r, g[o]);
                    } else if (l == 0) {
                        for (int i = 0; i < 16; i++) atomicAdd(grads + kMlpW1 + r * 16 + i, g[i]);
                    } else {
                        float *dst = grads + (l == 1 ? kMlpW2 : kMlpW3) + r * 64;
                        for (int i = 0; i < 64; i++) atomicAdd(dst + i, g[i]);
                    }
                }
            }
            if (l == 0) break;
            // dZ_{l-1} = dH_{l-1} * relu'(Z_{l-1}), into sD (the MMAs that read sD are complete)
            {
                float v[64], h[8];
                ld_row64(tmem, v);
                for (int c = 0; c < 64; c += 8) {
                    tc::ld_row8(Hs[l - 1], tid, c, 64, h);
#pragma unroll
                    for (int k = 0; k < 8; k++) {
                        v[c + k] = h[k] > 0.f ? v[c + k] : 0.f;
                        atomicAdd(&sDB[64 * (l - 1) + c + k], v[c + k]);
                    }
                    tc::st_row8(sD, tid, c, 64, v + c);
                }
            }
        }
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
    }
    if (!ok) on_timeout(mbar, phase, status);
    tc::fence_before_sync();
    __syncthreads();
    for (int i = tid; i < 224; i += blockDim.x) {
        int dst = i < 64 ? kMlpB1 + i : i < 128 ? kMlpB2 + i - 64 : i < 192 ? kMlpB3 + i - 128 : kMlpB4 + i - 192;
        atomicAdd(grads + dst, sDB[i]);
    }
    for (int off = 16; off > 0; off >>= 1) loss_acc += __shfl_down_sync(0xffffffffu, loss_acc, off);
    if (lane == 0 && loss) atomicAdd(loss, loss_acc);
    if (tid < 32) tc::tmem_free(tmem, 128);
}

__global__ void k_mlp_pack(const float *params, uint8_t *wimg) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    // W1 64 x 16, W2 64 x 64, W3 64 x 64, W4 32 x 64
    int base, C, off;
    if (i < 1024) {
        base = kMlpW1, C = 16, off = kImgW1;
    } else if (i < 1024 + 4096) {
        i -= 1024;
        base = kMlpW2, C = 64, off = kImgW2;
    } else if (i < 1024 + 8192) {
        i -= 1024 + 4096;
        base = kMlpW3, C = 64, off = kImgW3;
    } else if (i < 1024 + 8192 + 2048) {
        i -= 1024 + 8192;
        base = kMlpW4, C = 64, off = kImgW4;
    } else {
        return;
    }
    int r = i / C, c = i % C;
    *reinterpret_cast<__nv_bfloat16 *>(wimg + off + tc::imat_offset(r, c, C)) = __float2bfloat16_rn(params[base + i]);
}

__global__ void k_mlp_adam(float *p, const float *g, float *m, float *v, int n, float lr, float bc1, float bc2) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    float gi = g[i];
    float mi = b1 * m[i] + (1.f - b1) * gi;
    float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
}

// Opts the kernel in to its dynamic shared memory, once per device.
cudaError_t smem_attribute(const void *fn, int bytes, int which) {
    static std::atomic<unsigned long long> done[2];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    unsigned long long bit = 1ull << (dev & 63);
    if (done[which].load() & bit) return cudaSuccess;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) done[which].fetch_or(bit);
    return e;
}

__global__ void k_to_bf16(const float *x, __nv_bfloat16 *y, long long n) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = __float2bfloat16_rn(x[i]);
}

__global__ void k_sum(const float *x, long long n, float *out) {
    float s = 0.f;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        s += x[i];
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

int grid_for(long long n, int num_sms, int per_sm) {
    long long tiles = (n + kTile - 1) / kTile;
    long long cap = (long long)num_sms * per_sm;
    return (int)(tiles < cap ? (tiles > 0 ? tiles : 1) : cap);
}

}  // namespace

cudaError_t dr_mlp_pack(const float *params, uint8_t *wimg, cudaStream_t st) {
    k_mlp_pack<<<(1024 + 8192 + 2048 + 255) / 256, 256, 0, st>>>(params, wimg);
    return cudaGetLastError();
}

cudaError_t dr_mlp_infer(const uint8_t *wimg, const float *params, const __nv_bfloat16 *x, long long n, float *logits,
                         __nv_bfloat16 *probs, int *status, int num_sms, cudaStream_t st) {
    cudaError_t e = smem_attribute((const void *)k_mlp_infer, kInferSmem, 0);
    if (e != cudaSuccess) return e;
    if (n <= 0) return cudaSuccess;
    k_mlp_infer<<<grid_for(n, num_sms, 2), kTile, kInferSmem, st>>>(wimg, params, x, n, logits, probs, status);
    return cudaGetLastError();
}

cudaError_t dr_mlp_grad(const uint8_t *wimg, const float *params, const __nv_bfloat16 *x, const float *targets,
                        long long n, const float *target_total, float *grads, float *loss, int *status, int num_sms,
                        cudaStream_t st) {
    cudaError_t e = smem_attribute((const void *)k_mlp_grad, kGradSmem, 1);
    if (e != cudaSuccess) return e;
    if (n <= 0) return cudaSuccess;
    k_mlp_grad<<<grid_for(n, num_sms, 2), kTile, kGradSmem, st>>>(wimg, params, x, targets, n, target_total, grads,
                                                                  loss, status);
    return cudaGetLastError();
}

cudaError_t dr_mlp_adam(float *params, const float *grads, float *m, float *v, int step, float lr, cudaStream_t st) {
    float bc1 = 1.f - powf(0.9f, (float)step), bc2 = 1.f - powf(0.999f, (float)step);
    k_mlp_adam<<<(kMlpParams + 255) / 256, 256, 0, st>>>(params, grads, m, v, kMlpParams, lr, bc1, bc2);
    return cudaGetLastError();
}

cudaError_t dr_mlp_to_bf16(const float *x, __nv_bfloat16 *y, long long n, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    k_to_bf16<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(x, y, n);
    return cudaGetLastError();
}

cudaError_t dr_mlp_sum(const float *x, long long n, float *out, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(float), st);
    if (e != cudaSuccess || n <= 0) return e;
    k_sum<<<296, 256, 0, st>>>(x, n, out);
    return cudaGetLastError();
}
