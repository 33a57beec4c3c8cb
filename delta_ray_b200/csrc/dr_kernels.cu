// CUDA kernels of the renderer: LBVH build and the forward pixel-sample kernel.
// The per-sample logic lives in the dr_*.cuh headers; kernels here only map
// threads to work and reduce results.
#include "dr_bvh.cuh"
#include "dr_kernels.h"
#include "dr_shading.cuh"

#include <cub/cub.cuh>

// ---------------------------------------------------------------------------
// LBVH build
// ---------------------------------------------------------------------------
__global__ void k_bvh_morton(BvhBuildIn in, uint32_t *keys, int *vals) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= in.n) return;
    keys[i] = tri_morton(in, i);
    vals[i] = i;
}

__global__ void k_bvh_leaves(const int *sorted_ids, const float *vtx, const int4 *tri, int n, float4 *leaf_tris,
                             Box *leaf_boxes) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int t = sorted_ids[i];
    int4 id = tri[t];
    float4 a, b, c;
    a.x = vtx[3 * id.x]; a.y = vtx[3 * id.x + 1]; a.z = vtx[3 * id.x + 2]; a.w = dr_i2f(t);
    b.x = vtx[3 * id.y]; b.y = vtx[3 * id.y + 1]; b.z = vtx[3 * id.y + 2]; b.w = 0.f;
    c.x = vtx[3 * id.z]; c.y = vtx[3 * id.z + 1]; c.z = vtx[3 * id.z + 2]; c.w = 0.f;
    leaf_tris[3 * i] = a;
    leaf_tris[3 * i + 1] = b;
    leaf_tris[3 * i + 2] = c;
    leaf_boxes[i] = tri_box(a, b, c);
}

__global__ void k_bvh_internal(const uint32_t *keys, int n, int2 *children, int *parent_internal, int *parent_leaf) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    lbvh_internal(keys, n, i, children, parent_internal, parent_leaf);
}

__device__ __forceinline__ Box load_box_cg(const Box *b) {
    Box r;
    const float *f = (const float *)b;
    for (int k = 0; k < 3; k++) {
        r.lo[k] = __ldcg(f + k);
        r.hi[k] = __ldcg(f + 3 + k);
    }
    return r;
}

__global__ void k_bvh_refit(int n, const int *parent_leaf, const int *parent_internal, const int2 *children,
                            const Box *leaf_boxes, Box *node_boxes, int *flags, float4 *nodes) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int p = parent_leaf[i];
    // each internal node is finished by the second of its two children; the
    // walk is bounded by the tree height (< n)
    for (int guard = 0; guard < n; guard++) {
        __threadfence();
        if (atomicAdd(flags + p, 1) == 0) return;
        __threadfence();
        int2 c = children[p];
        Box b0 = c.x < 0 ? leaf_boxes[~c.x] : load_box_cg(node_boxes + c.x);
        Box b1 = c.y < 0 ? leaf_boxes[~c.y] : load_box_cg(node_boxes + c.y);
        Box u = box_union(b0, b1);
        float *dst = (float *)(node_boxes + p);
        for (int k = 0; k < 3; k++) {
            __stcg(dst + k, u.lo[k]);
            __stcg(dst + 3 + k, u.hi[k]);
        }
        write_node(nodes + 4 * p, b0, b1, c.x, c.y);
        if (p == 0) return;
        p = parent_internal[p];
    }
}

static inline int blocks_for(long long n, int bs) { return (int)((n + bs - 1) / bs); }

// The build's working arrays, laid out in the caller's scratch.  After a
// build they hold the tree's topology (sorted leaf order, parent and child
// links), which a refit reuses.
struct LbvhScratch {
    uint32_t *keys, *keys2;
    int *vals, *vals2;  // vals2: triangle id of each leaf (Morton order)
    Box *leaf_boxes, *node_boxes;
    int2 *children;
    int *parent_internal, *parent_leaf, *flags;
    void *sort_tmp;
    size_t sort_bytes, used;
};

static LbvhScratch lbvh_layout(void *scratch, int n) {
    LbvhScratch l;
    char *p = (char *)scratch;
    auto take = [&](size_t bytes) {
        char *r = p;
        p += (bytes + 255) & ~(size_t)255;
        return (void *)r;
    };
    l.keys = (uint32_t *)take(sizeof(uint32_t) * n);
    l.keys2 = (uint32_t *)take(sizeof(uint32_t) * n);
    l.vals = (int *)take(sizeof(int) * n);
    l.vals2 = (int *)take(sizeof(int) * n);
    l.leaf_boxes = (Box *)take(sizeof(Box) * n);
    l.node_boxes = (Box *)take(sizeof(Box) * n);
    l.children = (int2 *)take(sizeof(int2) * n);
    l.parent_internal = (int *)take(sizeof(int) * n);
    l.parent_leaf = (int *)take(sizeof(int) * n);
    l.flags = (int *)take(sizeof(int) * n);
    l.sort_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, l.sort_bytes, l.keys, l.keys2, l.vals, l.vals2, n, 0, 30);
    l.sort_tmp = take(l.sort_bytes);
    l.used = (size_t)(p - (char *)scratch);
    return l;
}

cudaError_t dr_build_lbvh(const float *vtx, const int4 *tri, int n, float3 lo, float3 hi, float4 *nodes,
                          float4 *leaf_tris, void *scratch, size_t scratch_bytes, cudaStream_t st, int *launches) {
    if (n <= 0) return cudaSuccess;
    BvhBuildIn in;
    in.vtx = vtx;
    in.tri = tri;
    in.n = n;
    in.lo = lo;
    float3 ext = hi - lo;
    in.inv_ext = f3(ext.x > 0.f ? 1.f / ext.x : 0.f, ext.y > 0.f ? 1.f / ext.y : 0.f, ext.z > 0.f ? 1.f / ext.z : 0.f);
    LbvhScratch l = lbvh_layout(scratch, n);
    if (l.used > scratch_bytes) return cudaErrorMemoryAllocation;
    const int bs = 256;
    k_bvh_morton<<<blocks_for(n, bs), bs, 0, st>>>(in, l.keys, l.vals);
    cub::DeviceRadixSort::SortPairs(l.sort_tmp, l.sort_bytes, l.keys, l.keys2, l.vals, l.vals2, n, 0, 30, st);
    k_bvh_leaves<<<blocks_for(n, bs), bs, 0, st>>>(l.vals2, vtx, tri, n, leaf_tris, l.leaf_boxes);
    *launches += 3;
    if (n > 1) {
        cudaMemsetAsync(l.flags, 0, sizeof(int) * n, st);
        k_bvh_internal<<<blocks_for(n - 1, bs), bs, 0, st>>>(l.keys2, n, l.children, l.parent_internal,
                                                               l.parent_leaf);
        k_bvh_refit<<<blocks_for(n, bs), bs, 0, st>>>(n, l.parent_leaf, l.parent_internal, l.children, l.leaf_boxes,
                                                       l.node_boxes, l.flags, nodes);
        *launches += 2;
    }
    return cudaGetLastError();
}

cudaError_t dr_refit_lbvh(const float *vtx, const int4 *tri, int n, float4 *nodes, float4 *leaf_tris, void *scratch,
                          size_t scratch_bytes, cudaStream_t st, int *launches) {
    if (n <= 0) return cudaSuccess;
    LbvhScratch l = lbvh_layout(scratch, n);
    if (l.used > scratch_bytes) return cudaErrorMemoryAllocation;
    const int bs = 256;
    k_bvh_leaves<<<blocks_for(n, bs), bs, 0, st>>>(l.vals2, vtx, tri, n, leaf_tris, l.leaf_boxes);
    *launches += 1;
    if (n > 1) {
        cudaMemsetAsync(l.flags, 0, sizeof(int) * n, st);
        k_bvh_refit<<<blocks_for(n, bs), bs, 0, st>>>(n, l.parent_leaf, l.parent_internal, l.children, l.leaf_boxes,
                                                       l.node_boxes, l.flags, nodes);
        *launches += 1;
    }
    return cudaGetLastError();
}

size_t dr_lbvh_scratch_bytes(int n) { return lbvh_layout(nullptr, n).used; }

// One 4-wide node per internal node (widen_node).
__global__ void k_bvh_widen(const float4 *nodes, int n_internal, float4 *wide) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n_internal) return;
    widen_node(nodes, p, wide + (size_t)DR_WIDE_F4 * p);
}

cudaError_t dr_widen_lbvh(const float4 *nodes, int n, float4 *wide, cudaStream_t st, int *launches) {
    if (n <= 1) return cudaSuccess;
    k_bvh_widen<<<blocks_for(n - 1, 256), 256, 0, st>>>(nodes, n - 1, wide);
    *launches += 1;
    return cudaGetLastError();
}

__global__ void k_trace_rays(DevScene s, const float *rays, long long n, int *tri, float *t) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *r = rays + 6 * i;
    Hit h = trace_closest(s, f3(r[0], r[1], r[2]), f3(r[3], r[4], r[5]), 1e-3f);
    tri[i] = h.tri;
    t[i] = h.t;
}

__global__ void k_eval_math(int fn, const float *x, const float *y, float *out, long long n) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = dr_math_eval(fn, x[i], y ? y[i] : 0.f);
}

cudaError_t dr_launch_eval_math(int fn, const float *x, const float *y, float *out, long long n, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    k_eval_math<<<blocks_for(n, 256), 256, 0, st>>>(fn, x, y, out, n);
    return cudaGetLastError();
}

cudaError_t dr_launch_trace(const DevScene &s, const float *rays, long long n, int *tri, float *t, cudaStream_t st,
                            int *launches) {
    if (n <= 0) return cudaSuccess;
    k_trace_rays<<<blocks_for(n, 256), 256, 0, st>>>(s, rays, n, tri, t);
    *launches += 1;
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Forward render: one pixel sample per (pixel, lane) and a segmented warp
// reduction over the 2^lanes_log2 lanes of a pixel.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256, 4) k_render_forward(DevScene s, int W, int H, int spp, int B, uint64_t seed,
                                                        int lanes_log2, float *img) {
    long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int G = 1 << lanes_log2;
    long long pix = gid >> lanes_log2;
    int lane = (int)(gid & (G - 1));
    float3 acc = f3(0.f);
    bool active = pix < (long long)W * H;
    if (active) {
        int x = (int)(pix % W), y = (int)(pix / W);
        for (int si = lane; si < spp; si += G) acc += pixel_sample(s, x, y, W, H, spp, si, B, seed);
    }
    for (int off = G >> 1; off >= 1; off >>= 1) {
        acc.x += __shfl_down_sync(0xffffffffu, acc.x, off);
        acc.y += __shfl_down_sync(0xffffffffu, acc.y, off);
        acc.z += __shfl_down_sync(0xffffffffu, acc.z, off);
    }
    if (active && lane == 0) {
        img[3 * pix] = acc.x;
        img[3 * pix + 1] = acc.y;
        img[3 * pix + 2] = acc.z;
    }
}

cudaError_t dr_launch_forward(const DevScene &s, int W, int H, int spp, int B, uint64_t seed, float *img,
                              cudaStream_t st, int *launches, StageTimer *timer) {
    int lanes_log2 = 0;
    while ((1 << (lanes_log2 + 1)) <= spp && (1 << (lanes_log2 + 1)) <= 32 && spp % (1 << (lanes_log2 + 1)) == 0)
        lanes_log2++;
    long long threads = ((long long)W * H) << lanes_log2;
    const int bs = 256;
    timer->begin(st);
    k_render_forward<<<blocks_for(threads, bs), bs, 0, st>>>(s, W, H, spp, B, seed, lanes_log2, img);
    timer->mark(st, "k_render_forward");
    *launches += 1;
    return cudaGetLastError();
}

__global__ void k_accumulate(float *dst, const float *src, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] += src[i];
}

cudaError_t dr_launch_accumulate(float *dst, const float *src, long long n, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    long long blocks = (n + 255) / 256;
    k_accumulate<<<(int)(blocks < 4096 ? blocks : 4096), 256, 0, st>>>(dst, src, n);
    return cudaGetLastError();
}
