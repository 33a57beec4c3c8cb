// Rules of the edge trees' median-split build that make its result
// independent of the order in which values are combined, so that the GPU
// build (dr_scene_build.cu), the host build (dr_host_scene.h) and the oracle
// produce the same trees bit for bit:
//  - edge_ord_key: a float's position in the total order -NaN < -inf < ... <
//    -0 < +0 < ... < +inf < NaN, as an unsigned key.  Splits sort by it
//    (stably), boxes take minima and maxima in it.
//  - edge_fixed / edge_unfixed: the normal-cone axis sums unit normals
//    exactly, in 2^-38 fixed point (int64; |sum| < 2^62 for up to 2^23
//    edges per node), and converts the sum to float once.
//  - edge_split_dim: the split dimension of a node (edge_tree.cpp:116-153):
//    the largest extent of the centroid box (0-2), or for the directional
//    tree also of the scaled normal box (3-5), first one on ties; -1 when
//    that extent is zero (a leaf of several edges).
#pragma once

#include <stdint.h>

// Edge trees of at most this many edges follow the reference's split rule
// exactly (std::nth_element, built on the host in microseconds); larger
// trees follow the rule above and are built on the GPU.  The two rules give
// the same trees except where edges share a median coordinate; both are
// unbiased, but the reference's "last sampled edge wins" gradient depends on
// the order of the edges in the trees, so small scenes keep the reference's.
#define DR_TREE_EXACT_MAX_EDGES 16384

#include "dr_math.h"

DRM_FN uint32_t edge_ord_key(float x) {
    uint32_t b;
#ifdef __CUDA_ARCH__
    b = __float_as_uint(x);
#else
    std::memcpy(&b, &x, 4);
#endif
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
DRM_FN float edge_from_ord_key(uint32_t k) {
    uint32_t b = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
#ifdef __CUDA_ARCH__
    return __uint_as_float(b);
#else
    float x;
    std::memcpy(&x, &b, 4);
    return x;
#endif
}

constexpr double kEdgeFixedScale = 274877906944.0;          // 2^38
constexpr double kEdgeFixedInv = 3.637978807091713e-12;      // 2^-38
DRM_FN long long edge_fixed(float x) {
    double v = drm::mul((double)x, kEdgeFixedScale);
    if (v != v) return 0;
    if (v > 1125899906842624.0) v = 1125899906842624.0;  // 2^50
    if (v < -1125899906842624.0) v = -1125899906842624.0;
    return (long long)drm::round_int(v);
}
DRM_FN float edge_unfixed(long long s) {
#ifdef __CUDA_ARCH__
    double d = __ll2double_rn(s);
#else
    double d = (double)s;
#endif
    return (float)drm::mul(d, kEdgeFixedInv);
}

DRM_FN int edge_split_dim(float slx, float sly, float slz, float shx, float shy, float shz, bool dir, float dlx,
                          float dly, float dlz, float dhx, float dhy, float dhz) {
    float lo[6] = {slx, sly, slz, dlx, dly, dlz}, hi[6] = {shx, shy, shz, dhx, dhy, dhz};
    int dim = -1;
    float maxe = -__builtin_huge_valf();
    for (int a = 0; a < (dir ? 6 : 3); a++) {
        float e = hi[a] - lo[a];
        if (e > maxe) {
            dim = a;
            maxe = e;
        }
    }
    if (dim < 0 || hi[dim] == lo[dim]) return -1;
    return dim;
}
