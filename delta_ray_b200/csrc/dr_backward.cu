// Backward pass, path half.  The work is split by what it depends on, each
// stage reading the previous one's compacted output from HBM:
//   k_backward_paths   one thread per (pixel, lane): path adjoint of the
//                      pixel's samples, image, and the shading-point records
//   k_edge_traverse    one thread per shading point: edge-tree traversal,
//                      appends (point, edge, weight) items
//   k_edge_line        one thread per item: the line sample on the edge
//   k_edge_connect     surviving line samples fetched one per lane: the
//                      connectivity of the two straddling rays (the edge's
//                      faces, bounded occlusion walks)
//   k_edge_pairs       candidates fetched one per lane: the other side's
//                      closest hit and the tests on both hits
//   k_edge_shade       one thread per kept sample: shading of both sides,
//                      dv0/dv1 scatter and dp
//   k_dp_propagate     one thread per point: the point's dp through its
//                      triangle and the camera (reference "last edge" rule)
//   k_primary_shade    one thread per primary-edge sample: the two camera rays
//                      beside the sampled edge point and their shades
//   k_primary_grad     one thread per primary-edge sample: Jacobians, scatter
// This file holds the path kernels and the stage sequencing; it is compiled
// without FMA contraction, so that the first vertex of every path (which
// decides which edges a shading point sees) has the bits of the reference's
// CPU arithmetic.  The edge kernels (dr_edge_kernels.cu) start from the
// stored vertex and are compiled without contraction too.
// Gradients of the small, shared parameters (camera, constant materials,
// light intensities) are reduced per block in shared memory and flushed with
// one atomic per nonzero entry; per-vertex gradients go straight to global
// atomics (or shared memory too when the whole gradient fits).
#include "../../include/delta_ray_b200.h"
#include "dr_backward.cuh"
#include "dr_block_grad.cuh"

template <bool kChains, int BMAX>
__global__ void __launch_bounds__(128, 8) k_backward_paths(DevScene s, int W, int H, int spp, int B, uint64_t seed,
                                                        int lanes_log2, const float *d_image, float *grad, float *img,
                                                        BackwardWorkspace ws, GradCacheCfg cfg) {
    extern __shared__ float sm[];
    BlockGradWarp bg;
    static_cast<BlockGrad &>(bg) = block_grad_begin(sm, grad, cfg);
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
                if (p.bounce == 0) {  // the first vertex: pushed warp-aggregated below
                    pr = p;
                    has = true;
                    return;
                }
                // vertices after specular samples (rare): one atomic each
                unsigned long long slot = atomicAdd(&ws.counters->points, 1ull);
                if (slot < (unsigned long long)ws.cap_points) p.store(ws.pt + (size_t)slot * DR_PT_WORDS);
                else set_status(&ws.counters->status, DR_STATUS_POINT_OVERFLOW);
            };
            acc += backward_pixel_sample<kChains, BMAX>(s, x, y, W, H, spp, si, B, seed, dc, bg, push);
        }
        __syncwarp();
        unsigned long long slot = warp_reserve(&ws.counters->points, has ? 1 : 0);
        if (has) {
            if (slot < (unsigned long long)ws.cap_points) pr.store(ws.pt + (size_t)slot * DR_PT_WORDS);
            else set_status(&ws.counters->status, DR_STATUS_POINT_OVERFLOW);
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

// Position adjoints of the shading points pushed back along their paths.
// DR_DP_REFERENCE_LAST: each point's last edge with a nonzero dp (the largest
// key ((j + 1) << 32 | item) in pt_last).  DR_DP_SUM (scenes with specular
// chains only): the dp sums k_edge_shade accumulated for points after the first
// vertex, whose chains are traced again here, in this IEEE compile unit.
template <bool kChains>
__global__ void __launch_bounds__(128, 6) k_dp_propagate(DevScene s, int W, int H, int spp, uint64_t seed, int dp_mode,
                                                      float *grad, BackwardWorkspace ws, GradCacheCfg cfg) {
    extern __shared__ float sm[];
    BlockGradWarp bg;
    static_cast<BlockGrad &>(bg) = block_grad_begin(sm, grad, cfg);
    long long n = min(min((long long)ws.counters->points, ws.cap_points), ws.pt_end);
    for (long long p = ws.pt_begin + (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n;
         p += (long long)gridDim.x * blockDim.x) {
        float3 dp;
        if (dp_mode == DR_DP_SUM) {
            float4 a = reinterpret_cast<const float4 *>(ws.pt_last)[p];
            dp = f3(a.x, a.y, a.z);
            if (is_zero(dp)) continue;
        } else {
            unsigned long long key = ws.pt_last[p];
            if (key == 0) continue;
            long long i = (long long)(key & 0xffffffffull);
            dp = f3(ws.item_dp[3 * i], ws.item_dp[3 * i + 1], ws.item_dp[3 * i + 2]);
        }
        PointRecord pt;
        pt.load(ws.pt + (size_t)p * DR_PT_WORDS);
        const PointView v = point_view(ws, pt.view, W, H, spp, seed);
        propagate_dp<kChains>(s, pt, v.W, v.H, v.spp, v.seed, dp, bg, v.cam, v.cam_off);
    }
    block_grad_flush(bg);
}

namespace {
int path_lanes_log2(int spp) {
    int l = 0;
    while ((1 << (l + 1)) <= spp && (1 << (l + 1)) <= 32 && spp % (1 << (l + 1)) == 0) l++;
    return l;
}
}  // namespace

cudaError_t dr_launch_backward_front(const DevScene &s, int W, int H, int spp, int B, uint64_t seed,
                                     const float *d_image, float *grad, float *img, long long primary_edge_samples,
                                     int dp_mode, const BackwardWorkspace &ws, const GradCacheCfg &cfg, int num_sms,
                                     cudaStream_t st, int *launches, StageTimer *timer, bool traverse, bool first) {
    const int bs = 128;
    size_t smem = sizeof(float) * (size_t)(cfg.head + cfg.tail_len);
    int lanes_log2 = path_lanes_log2(spp);
    long long threads = ((long long)W * H) << lanes_log2;
    if (first) timer->begin(st);  // a later view's front stage of a batched call continues the timing
    if (dp_mode != DR_DP_SUM || s.specular_chains) {
        // LAST: one key per point; SUM with chains: a float4 dp sum per point
        size_t per = dp_mode == DR_DP_SUM ? DR_PT_LAST_BYTES : sizeof(unsigned long long);
        cudaError_t e = cudaMemsetAsync(ws.pt_last, 0, per * (size_t)ws.cap_points, st);
        if (e != cudaSuccess) return e;
    }
    // variants: specular chains or not, direct lighting (B = 1) or not
    // deeper than the records' 64 bounces: the checkpointed form, segments of
    // 16 bounces traced again for the suffix sweep and the replay
    auto kernel = s.specular_chains
                      ? (B == 1 ? k_backward_paths<true, 1>
                                : (B > DR_MAX_BOUNCES ? k_backward_paths<true, -16> : k_backward_paths<true, DR_MAX_BOUNCES>))
                      : (B == 1 ? k_backward_paths<false, 1>
                                : (B > DR_MAX_BOUNCES ? k_backward_paths<false, -16>
                                                      : k_backward_paths<false, DR_MAX_BOUNCES>));
    kernel<<<blocks_for(threads, bs), bs, smem, st>>>(s, W, H, spp, B, seed, lanes_log2, d_image, grad, img, ws, cfg);
    timer->mark(st, "k_backward_paths");
    *launches += 1;
    long long npe = primary_edge_samples > 0 ? primary_edge_samples : (long long)spp * W * H;
    if (s.num_prim_edges > 0 && npe > 0) {
        // the edge-item queue is free until the traversal: it carries the
        // primary samples' color differences (16 B each) between the two kernels
        cudaError_t e = dr_launch_primary_edges(s, W, H, spp, B, seed, d_image, npe, grad, cfg,
                                                reinterpret_cast<float4 *>(ws.items), ws.cap_items, num_sms, st,
                                                launches, timer);
        if (e != cudaSuccess) return e;
    }
    if (!traverse) return cudaGetLastError();
    return dr_launch_edge_traverse(s, seed, ws, num_sms, st, launches, timer);
}

cudaError_t dr_launch_backward_back(const DevScene &s, int W, int H, int spp, int B, uint64_t seed, float *grad,
                                    int dp_mode, const BackwardWorkspace &ws, const GradCacheCfg &cfg, int num_sms,
                                    cudaStream_t st, int *launches, StageTimer *timer) {
    const int bs = 128;
    size_t smem = sizeof(float) * (size_t)(cfg.head + cfg.tail_len);
    int grid_ws = stage_grid(num_sms);
    cudaError_t e = dr_launch_edge_eval(s, W, H, spp, B, seed, dp_mode, grad, ws, cfg, num_sms, st, launches, timer);
    if (e != cudaSuccess) return e;
    if (dp_mode != DR_DP_SUM || s.specular_chains) {
        if (s.specular_chains) k_dp_propagate<true><<<grid_ws, bs, smem, st>>>(s, W, H, spp, seed, dp_mode, grad, ws, cfg);
        else k_dp_propagate<false><<<grid_ws, bs, smem, st>>>(s, W, H, spp, seed, dp_mode, grad, ws, cfg);
        timer->mark(st, "k_dp_propagate");
        *launches += 1;
    }
    return cudaGetLastError();
}

// Loads every kernel a backward call can launch (see dr_preload_edge_kernels).
cudaError_t dr_preload_backward_kernels() {
    const void *k[] = {
        (const void *)k_backward_paths<true, 1>, (const void *)k_backward_paths<true, DR_MAX_BOUNCES>,
        (const void *)k_backward_paths<true, -16>, (const void *)k_backward_paths<false, 1>,
        (const void *)k_backward_paths<false, DR_MAX_BOUNCES>, (const void *)k_backward_paths<false, -16>,
        (const void *)k_dp_propagate<true>, (const void *)k_dp_propagate<false>,
    };
    for (const void *f : k) {
        cudaFuncAttributes a;
        const cudaError_t e = cudaFuncGetAttributes(&a, f);
        if (e != cudaSuccess) return e;
    }
    return dr_preload_edge_kernels();
}
