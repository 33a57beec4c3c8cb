// Per-block helpers shared by the backward kernels: a shared-memory cache of
// the small, shared gradient entries, device status bits and warp-aggregated
// queue slots.
#pragma once

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

// The same cache, for kernels whose warps mostly add to the same entries
// (path adjoints, primary edges, position adjoints in small scenes:
// neighbouring samples hit the same triangle and material): a full warp adding
// to one entry sums with shuffles and adds once.
struct BlockGradWarp : BlockGrad {
    __device__ __forceinline__ void add(int i, float v) {
        if (__activemask() == 0xffffffffu && __match_any_sync(0xffffffffu, i) == 0xffffffffu) {
            for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
            if ((threadIdx.x & 31) != 0) return;
        }
        BlockGrad::add(i, v);
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
__device__ __forceinline__ unsigned long long warp_reserve(unsigned long long *counter, int count) {
    const unsigned full = 0xffffffffu;
    int lane = threadIdx.x & 31;
    int incl = count;
    for (int off = 1; off < 32; off <<= 1) {
        int v = __shfl_up_sync(full, incl, off);
        if (lane >= off) incl += v;
    }
    int total = __shfl_sync(full, incl, 31);
    unsigned long long base = 0;
    if (lane == 31 && total > 0) base = atomicAdd(counter, (unsigned long long)total);
    base = __shfl_sync(full, base, 31);
    return base + (unsigned long long)(incl - count);
}

inline int blocks_for(long long n, int bs) { return (int)((n + bs - 1) / bs); }

// resident-grid size for the grid-stride stages: a few blocks per SM
inline int stage_grid(int num_sms) { return num_sms * 12; }

// A shading point's render settings: its view's in a batched multi-view call
// (ws.views), else the call's.  cam is null for the scene's own camera.
struct PointView {
    int W, H, spp;
    uint64_t seed;
    const DevCamera *cam;
    int cam_off;
};
__device__ __forceinline__ PointView point_view(const BackwardWorkspace &ws, int view, int W, int H, int spp,
                                                uint64_t seed) {
    PointView v;
    if (ws.views) {
        const ViewParams &p = ws.views[view];
        v.W = p.W;
        v.H = p.H;
        v.spp = p.spp;
        v.seed = p.seed;
        v.cam = &p.cam;
        v.cam_off = p.cam_off;
    } else {
        v.W = W;
        v.H = H;
        v.spp = spp;
        v.seed = seed;
        v.cam = nullptr;
        v.cam_off = 0;
    }
    return v;
}
__device__ __forceinline__ uint64_t point_seed(const BackwardWorkspace &ws, int view, uint64_t seed) {
    return ws.views ? ws.views[view].seed : seed;
}

}  // namespace
