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

// Reserves `count` consecutive slots for each lane of the (fully converged)
// warp with one atomic: returns the lane's first slot.
__device__ __forceinline__ long long warp_reserve(int *counter, int count) {
    const unsigned full = 0xffffffffu;
    int lane = threadIdx.x & 31;
    int incl = count;
    for (int off = 1; off < 32; off <<= 1) {
        int v = __shfl_up_sync(full, incl, off);
        if (lane >= off) incl += v;
    }
    int total = __shfl_sync(full, incl, 31);
    long long base = 0;
    if (lane == 31 && total > 0) base = atomicAdd(counter, total);
    base = __shfl_sync(full, base, 31);
    return base + incl - count;
}

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
    int x = active ? (int)(pix % W) : 0, y = active ? (int)(pix / W) : 0;
    float3 dc = active ? f3(d_image[3 * pix], d_image[3 * pix + 1], d_image[3 * pix + 2]) : f3(0.f);
    // warp-uniform trip count so that the point push can be warp-aggregated
    int iters = (spp + G - 1) >> lanes_log2;
    for (int it = 0; it < iters; it++) {
        int si = lane + (it << lanes_log2);
        PointRecord pr;
        bool has = false;
        if (active && si < spp) {
            auto push = [&](const PointRecord &p) {
                pr = p;
                has = true;
            };
            acc += backward_pixel_sample(s, x, y, W, H, spp, si, B, seed, dc, bg, push);
        }
        __syncwarp();
        long long slot = warp_reserve(ws.pt_count, has ? 1 : 0);
        if (has) {
            if (slot < ws.cap_points) pr.store(ws.pt + (size_t)slot * DR_PT_WORDS);
            else set_status(ws.status, DR_STATUS_POINT_OVERFLOW);
        }
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

#define DR_ITEM_BUF 24
__global__ void __launch_bounds__(128) k_edge_traverse(DevScene s, uint64_t seed, BackwardWorkspace ws) {
    long long n = min((long long)*ws.pt_count, ws.cap_points);
    long long stride = (long long)gridDim.x * blockDim.x;
    // warp-uniform loop: every lane of a warp takes the same number of trips
    for (long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += stride) {
        long long p = base + (threadIdx.x & 31);
        bool active = p < n;
        int buf_e[DR_ITEM_BUF];
        float buf_w[DR_ITEM_BUF];
        int buf_j[DR_ITEM_BUF];
        int nb = 0;
        auto write_item = [&](long long i, int te, int j, float w) {
            if (i < ws.cap_items) {
                int4 it;
                it.x = (int)p;
                it.y = te;
                it.z = j;
                it.w = 0;
                ws.items[i] = it;
                ws.item_w[i] = w;
            } else {
                set_status(ws.status, DR_STATUS_ITEM_OVERFLOW);
            }
        };
        if (active) {
            PointRecord pt;
            pt.load(ws.pt + (size_t)p * DR_PT_WORDS);
            auto emit = [&](int tree, int ei, int j, float w) {
                if (nb < DR_ITEM_BUF) {
                    buf_e[nb] = (tree << 30) | ei;
                    buf_j[nb] = j;
                    buf_w[nb] = w;
                    nb++;
                } else {  // rare: more edges than the lane buffer holds
                    write_item(atomicAdd(ws.item_count, 1), (tree << 30) | ei, j, w);
                }
            };
            if (!traverse_point(s, pt, seed, emit)) set_status(ws.status, DR_STATUS_STACK_OVERFLOW);
        }
        __syncwarp();
        long long slot = warp_reserve(ws.item_count, nb);
        for (int k = 0; k < nb; k++) write_item(slot + k, buf_e[k], buf_j[k], buf_w[k]);
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

namespace {
int path_lanes_log2(int spp) {
    int l = 0;
    while ((1 << (l + 1)) <= spp && (1 << (l + 1)) <= 32 && spp % (1 << (l + 1)) == 0) l++;
    return l;
}
// resident-grid size for the grid-stride stages: a few blocks per SM
int stage_grid(int num_sms) { return num_sms * 12; }
}  // namespace

cudaError_t dr_launch_backward_front(const DevScene &s, int W, int H, int spp, int B, uint64_t seed,
                                     const float *d_image, float *grad, float *img, long long primary_edge_samples,
                                     int dp_mode, const BackwardWorkspace &ws, const GradCacheCfg &cfg, int num_sms,
                                     cudaStream_t st, int *launches, StageTimer *timer) {
    const int bs = 128;
    size_t smem = sizeof(float) * (size_t)(cfg.head + cfg.tail_len);
    int lanes_log2 = path_lanes_log2(spp);
    long long threads = ((long long)W * H) << lanes_log2;
    int grid_ws = stage_grid(num_sms);
    timer->begin(st);
    if (dp_mode != DR_DP_SUM) {
        cudaError_t e = cudaMemsetAsync(ws.pt_last, 0, sizeof(unsigned long long) * (size_t)ws.cap_points, st);
        if (e != cudaSuccess) return e;
    }
    k_backward_paths<<<blocks_for(threads, bs), bs, smem, st>>>(s, W, H, spp, B, seed, lanes_log2, d_image, grad, img,
                                                               ws, cfg);
    timer->mark(st, "k_backward_paths");
    *launches += 1;
    long long npe = primary_edge_samples > 0 ? primary_edge_samples : (long long)spp * W * H;
    if (s.num_prim_edges > 0 && npe > 0) {
        long long nb = std::min<long long>(blocks_for(npe, bs), (long long)grid_ws * 4);
        k_primary_edges<<<(int)nb, bs, smem, st>>>(s, W, H, spp, B, seed, d_image, npe, grad, cfg);
        timer->mark(st, "k_primary_edges");
        *launches += 1;
    }
    return dr_launch_edge_traverse(s, seed, ws, num_sms, st, launches, timer);
}

cudaError_t dr_launch_edge_traverse(const DevScene &s, uint64_t seed, const BackwardWorkspace &ws, int num_sms,
                                    cudaStream_t st, int *launches, StageTimer *timer) {
    k_edge_traverse<<<stage_grid(num_sms), 128, 0, st>>>(s, seed, ws);
    timer->mark(st, "k_edge_traverse");
    *launches += 1;
    return cudaGetLastError();
}

cudaError_t dr_launch_backward_back(const DevScene &s, int W, int H, int spp, int B, uint64_t seed, float *grad,
                                    int dp_mode, const BackwardWorkspace &ws, const GradCacheCfg &cfg, int num_sms,
                                    cudaStream_t st, int *launches, StageTimer *timer) {
    const int bs = 128;
    size_t smem = sizeof(float) * (size_t)(cfg.head + cfg.tail_len);
    int grid_ws = stage_grid(num_sms);
    k_edge_eval<<<grid_ws, bs, smem, st>>>(s, W, H, spp, B, seed, dp_mode, grad, ws, cfg);
    timer->mark(st, "k_edge_eval");
    *launches += 1;
    if (dp_mode != DR_DP_SUM) {
        k_dp_propagate<<<grid_ws, bs, smem, st>>>(s, W, H, spp, seed, grad, ws, cfg);
        timer->mark(st, "k_dp_propagate");
        *launches += 1;
    }
    return cudaGetLastError();
}
