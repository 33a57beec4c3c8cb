// Host-callable launchers of the renderer's kernels (defined in the .cu files).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "dr_scene.cuh"

// LBVH over n triangles (dr_kernels.cu); `nodes` holds 4 float4 per internal
// node, `leaf_tris` 3 float4 per triangle; scratch >= dr_lbvh_scratch_bytes(n).
cudaError_t dr_build_lbvh(const float *vtx, const int4 *tri, int n, float3 lo, float3 hi, float4 *nodes,
                          float4 *leaf_tris, void *scratch, size_t scratch_bytes, cudaStream_t st, int *launches);
size_t dr_lbvh_scratch_bytes(int n);

cudaError_t dr_launch_trace(const DevScene &s, const float *rays, long long n, int *tri, float *t, cudaStream_t st,
                            int *launches);

cudaError_t dr_launch_forward(const DevScene &s, int W, int H, int spp, int B, uint64_t seed, float *img,
                              cudaStream_t st, int *launches);

// Backward pass (dr_backward.cu).  `ws` is the workspace described by
// BackwardWorkspace; status receives device error bits.
struct BackwardWorkspace {
    // secondary shading points (one slot per pixel sample at most)
    float *pt;         // [cap_points][PT_FLOATS] packed point records
    int *pt_count;     // [1]
    long long cap_points;
    // edge items produced by the edge-tree traversal
    int4 *items;       // (point id, edge list, edge index, edge ordinal j)
    float *item_w;     // edge weight
    int *item_count;   // [1]
    long long cap_items;
    float *item_dp;    // [cap_items][3] dp of each item (0 when it had none)
    int *pt_last;      // [cap_points] index of the last item with nonzero dp
    int *status;       // [1] error bits
};

cudaError_t dr_launch_backward(const DevScene &s, int W, int H, int spp, int B, uint64_t seed, const float *d_image,
                               float *grad, float *img, long long primary_edge_samples, int dp_mode,
                               const BackwardWorkspace &ws, cudaStream_t st, int *launches);

// Words of one packed secondary-point record in BackwardWorkspace::pt.
#define DR_PT_FLOATS 24

// Device status bits.
#define DR_STATUS_POINT_OVERFLOW 1
#define DR_STATUS_ITEM_OVERFLOW 2
#define DR_STATUS_STACK_OVERFLOW 4
