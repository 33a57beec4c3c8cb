// Backward pass kernels.  The work is split by what it depends on, each stage
// reading the previous one's compacted output from HBM:
//   k_backward_paths   one thread per (pixel, lane): path adjoint of the
//                      pixel's samples, image, and the shading-point records
//   k_edge_traverse    one thread per shading point: edge-tree traversal,
//                      appends (point, edge, weight) items
//   k_edge_eval        one thread per item: two straddling rays, shading of
//                      both sides, dv0/dv1 scatter and dp
//   k_dp_propagate     one thread per point: the point's dp through its
//                      triangle and the camera (reference "last edge" rule)
//   k_primary_edges    one thread per primary-edge sample
// Gradients of the small, shared parameters (camera, constant materials,
// light intensities) are reduced per block in shared memory and flushed with
// one atomic per nonzero entry; per-vertex gradients go straight to global
// atomics (or shared memory too when the whole gradient fits).
#include "../../include/delta_ray_b200.h"
#include "dr_backward.cuh"
#include "dr_kernels.h"

namespace {

struct BlockGrad {
    float *sm;
    float *g;
    int head, tail_begin, tail_len;
    __device__ __forceinline__ void add(int i, float v) {
        if (v == 0.f) return;
        if (i < head) {
            atomicAdd(sm + i, v);
        } else if ((unsigned)(i - tail_begin) < (unsigned)tail_len) {
            atomicAdd(sm + head + (i - tail_begin), v);
        } else {
            atomicAdd(g + i, v);
        }
    }
};

__device__ __forceinline__ BlockGrad block_grad_begin(float *sm, float *g, const GradCacheCfg &c) {
    BlockGrad b;
    b.sm = sm;
    b.g = g;
    b.head = c.head;
    b.tail_begin = c.tail_begin;
    b.tail_len = c.tail_len;
    for (int i = threadIdx.x; i < c.head + c.tail_len; i += blockDim.x) sm[i] = 0.f;
    __syncthreads();
    return b;
}

__device__ __forceinline__ void block_grad_flush(const BlockGrad &b) {
    __syncthreads();
    for (int i = threadIdx.x; i < b.head + b.tail_len; i += blockDim.x) {
        float v = b.sm[i];
        if (v != 0.f) atomicAdd(b.g + (i < b.head ? i : b.tail_begin + (i - b.head)), v);
    }
}

__device__ __forceinline__ void set_status(int *status, int bit) { atomicOr(status, bit); }

inline int blocks_for(long long n, int bs) { return (int)((n + bs - 1) / bs); }

}  // namespace

__global__ void __launch_bounds__(128) k_backward_paths(DevScene s, int W, int H, int spp, int B, uint64_t seed,
                                                        int lanes_log2, const float *d_image, float *grad, float *img,
                                                        BackwardWorkspace ws, GradCacheCfg cfg) {
    extern __shared__ float sm[];
    BlockGrad bg = block_grad_begin(sm, grad, cfg);
    long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int G = 1 << lanes_log2;
    long long pix = gid >> lanes_log2;
    int lane = (int)(gid & (G - 1));
    bool active = pix < (long long)W * H;
    float3 acc = f3(0.f);
    if (active) {
        int x = (int)(pix % W), y = (int)(pix / W);
        float3 dc = f3(d_image[3 * pix], d_image[3 * pix + 1], d_image[3 * pix + 2]);
        auto push = [&](const PointRecord &pr) {
            long long i = atomicAdd(ws.pt_count, 1);
            if (i < ws.cap_points) pr.store(ws.pt + (size_t)i * DR_PT_WORDS);
            else set_status(ws.status, DR_STATUS_POINT_OVERFLOW);
        };
        for (int si = lane; si < spp; si += G) acc += backward_pixel_sample(s, x, y, W, H, spp, si, B, seed, dc, bg, push);
    }
    for (int off = G >> 1; off >= 1; off >>= 1) {
        acc.x += __shfl_down_sync(0xffffffffu, acc.x, off);
        acc.y += __shfl_down_sync(0xffffffffu, acc.y, off);
        acc.z += __shfl_down_sync(0xffffffffu, acc.z, off);
    }
    if (img && active && lane == 0) {
        img[3 * pix] = acc.x;
        img[3 * pix + 1] = acc.y;
        img[3 * pix + 2] = acc.z;
    }
    block_grad_flush(bg);
}

__global__ void __launch_bounds__(128) k_edge_traverse(DevScene s, uint64_t seed, BackwardWorkspace ws) {
    long long n = min((long long)*ws.pt_count, ws.cap_points);
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        PointRecord pt;
        pt.load(ws.pt + (size_t)p * DR_PT_WORDS);
        auto emit = [&](int tree, int ei, int j, float w) {
            long long i = atomicAdd(ws.item_count, 1);
            if (i < ws.cap_items) {
                int4 it;
                it.x = (int)p;
                it.y = (tree << 30) | ei;
                it.z = j;
                it.w = 0;
                ws.items[i] = it;
                ws.item_w[i] = w;
            } else {
                set_status(ws.status, DR_STATUS_ITEM_OVERFLOW);
            }
        };
        if (!traverse_point(s, pt, seed, emit)) set_status(ws.status, DR_STATUS_STACK_OVERFLOW);
    }
}

__global__ void __launch_bounds__(128) k_edge_eval(DevScene s, int W, int H, int spp, int B, uint64_t seed, int dp_mode,
                                                   float *grad, BackwardWorkspace ws, GradCacheCfg cfg) {
    extern __shared__ float sm[];
    BlockGrad bg = block_grad_begin(sm, grad, cfg);
    long long n = min((long long)*ws.item_count, ws.cap_items);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        int4 it = ws.items[i];
        PointRecord pt;
        pt.load(ws.pt + (size_t)it.x * DR_PT_WORDS);
        int tree = it.y >> 30, ei = it.y & ((1 << 30) - 1);
        float3 dp = eval_item(s, pt, tree, ei, it.z, ws.item_w[i], spp, B, seed, bg);
        if (is_zero(dp)) continue;
        if (dp_mode == DR_DP_SUM) {
            propagate_dp(s, pt, W, H, spp, seed, dp, bg);
        } else {
            ws.item_dp[3 * i] = dp.x;
            ws.item_dp[3 * i + 1] = dp.y;
            ws.item_dp[3 * i + 2] = dp.z;
            unsigned long long key = ((unsigned long long)(it.z + 1) << 32) | (unsigned long long)i;
            atomicMax(ws.pt_last + it.x, key);
        }
    }
    block_grad_flush(bg);
}

__global__ void __launch_bounds__(128) k_dp_propagate(DevScene s, int W, int H, int spp, uint64_t seed, float *grad,
                                                      BackwardWorkspace ws, GradCacheCfg cfg) {
    extern __shared__ float sm[];
    BlockGrad bg = block_grad_begin(sm, grad, cfg);
    long long n = min((long long)*ws.pt_count, ws.cap_points);
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        unsigned long long key = ws.pt_last[p];
        if (key == 0) continue;
        long long i = (long long)(key & 0xffffffffull);
        float3 dp = f3(ws.item_dp[3 * i], ws.item_dp[3 * i + 1], ws.item_dp[3 * i + 2]);
        PointRecord pt;
        pt.load(ws.pt + (size_t)p * DR_PT_WORDS);
        propagate_dp(s, pt, W, H, spp, seed, dp, bg);
    }
    block_grad_flush(bg);
}

__global__ void __launch_bounds__(128) k_primary_edges(DevScene s, int W, int H, int spp, int B, uint64_t seed,
                                                       const float *d_image, long long n, float *grad,
                                                       GradCacheCfg cfg) {
    extern __shared__ float sm[];
    BlockGrad bg = block_grad_begin(sm, grad, cfg);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        primary_edge_item(s, i, W, H, spp, B, seed, d_image, bg);
    block_grad_flush(bg);
}

cudaError_t dr_launch_backward(const DevScene &s, int W, int H, int spp, int B, uint64_t seed, const float *d_image,
                               float *grad, float *img, long long primary_edge_samples, int dp_mode,
                               const BackwardWorkspace &ws, const GradCacheCfg &cfg, int num_sms, cudaStream_t st,
                               int *launches, StageTimer *timer) {
    const int bs = 128;
    size_t smem = sizeof(float) * (size_t)(cfg.head + cfg.tail_len);
    int lanes_log2 = 0;
    while ((1 << (lanes_log2 + 1)) <= spp && (1 << (lanes_log2 + 1)) <= 32 && spp % (1 << (lanes_log2 + 1)) == 0)
        lanes_log2++;
    long long threads = ((long long)W * H) << lanes_log2;
    // resident-grid size for the grid-stride stages: a few blocks per SM
    int grid_ws = num_sms * 12;
    timer->begin(st);
    if (dp_mode != DR_DP_SUM) {
        cudaError_t e = cudaMemsetAsync(ws.pt_last, 0, sizeof(unsigned long long) * (size_t)ws.cap_points, st);
        if (e != cudaSuccess) return e;
    }
    k_backward_paths<<<blocks_for(threads, bs), bs, smem, st>>>(s, W, H, spp, B, seed, lanes_log2, d_image, grad, img,
                                                               ws, cfg);
    timer->mark(st, "k_backward_paths");
    k_edge_traverse<<<grid_ws, bs, 0, st>>>(s, seed, ws);
    timer->mark(st, "k_edge_traverse");
    k_edge_eval<<<grid_ws, bs, smem, st>>>(s, W, H, spp, B, seed, dp_mode, grad, ws, cfg);
    timer->mark(st, "k_edge_eval");
    *launches += 3;
    if (dp_mode != DR_DP_SUM) {
        k_dp_propagate<<<grid_ws, bs, smem, st>>>(s, W, H, spp, seed, grad, ws, cfg);
        timer->mark(st, "k_dp_propagate");
        *launches += 1;
    }
    long long npe = primary_edge_samples > 0 ? primary_edge_samples : (long long)spp * W * H;
    if (s.num_prim_edges > 0 && npe > 0) {
        long long nb = std::min<long long>(blocks_for(npe, bs), (long long)grid_ws * 4);
        k_primary_edges<<<(int)nb, bs, smem, st>>>(s, W, H, spp, B, seed, d_image, npe, grad, cfg);
        timer->mark(st, "k_primary_edges");
        *launches += 1;
    }
    return cudaGetLastError();
}
