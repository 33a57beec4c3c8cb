// LBVH construction (Karras 2012, "Maximizing parallelism in the construction
// of BVHs, octrees and k-d trees"): 30-bit Morton codes of triangle centroids,
// a stable radix sort, one thread per internal node to find its key range and
// split, then a bottom-up refit in which the second child to arrive at a node
// writes the node's two child boxes.
//
// Node layout (4 float4, 64 B): child 0 box (lo.xyz, hi.x), (hi.yz, child 1
// lo.xy), (child 1 lo.z, hi.xyz), (child ids as int bits).  A child id >= 0 is
// an internal node, < 0 is a leaf (~slot).  Leaves hold one triangle as 3
// float4 (v0, v1, v2; .w of v0 = global triangle id) in Morton order.
#pragma once

#include "dr_common.cuh"

HD uint32_t expand_bits10(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

HD uint32_t morton30(float x, float y, float z) {
    x = fminf(fmaxf(x * 1024.f, 0.f), 1023.f);
    y = fminf(fmaxf(y * 1024.f, 0.f), 1023.f);
    z = fminf(fmaxf(z * 1024.f, 0.f), 1023.f);
    return (expand_bits10((uint32_t)x) << 2) | (expand_bits10((uint32_t)y) << 1) | expand_bits10((uint32_t)z);
}

struct BvhBuildIn {
    const float *vtx;
    const int4 *tri;
    int n;
    float3 lo, inv_ext;
};

HD uint32_t tri_morton(const BvhBuildIn &in, int i) {
    int4 t = in.tri[i];
    float3 a = f3(in.vtx[3 * t.x], in.vtx[3 * t.x + 1], in.vtx[3 * t.x + 2]);
    float3 b = f3(in.vtx[3 * t.y], in.vtx[3 * t.y + 1], in.vtx[3 * t.y + 2]);
    float3 c = f3(in.vtx[3 * t.z], in.vtx[3 * t.z + 1], in.vtx[3 * t.z + 2]);
    float3 lo = f3(fminf(fminf(a.x, b.x), c.x), fminf(fminf(a.y, b.y), c.y), fminf(fminf(a.z, b.z), c.z));
    float3 hi = f3(fmaxf(fmaxf(a.x, b.x), c.x), fmaxf(fmaxf(a.y, b.y), c.y), fmaxf(fmaxf(a.z, b.z), c.z));
    float3 cen = (lo + hi) * 0.5f;
    return morton30((cen.x - in.lo.x) * in.inv_ext.x, (cen.y - in.lo.y) * in.inv_ext.y,
                    (cen.z - in.lo.z) * in.inv_ext.z);
}

HD int clz32(uint32_t x) {
#ifdef __CUDA_ARCH__
    return __clz((int)x);
#else
    return x == 0 ? 32 : __builtin_clz(x);
#endif
}

// common-prefix length of sorted keys i and j, ties broken by index
HD int lbvh_delta(const uint32_t *keys, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    uint32_t a = keys[i], b = keys[j];
    if (a == b) return 32 + clz32((uint32_t)(i ^ j));
    return clz32(a ^ b);
}

// Internal node i of n leaves: writes child ids and parent links.
HD void lbvh_internal(const uint32_t *keys, int n, int i, int2 *children, int *parent_internal, int *parent_leaf) {
    int dl = lbvh_delta(keys, n, i, i - 1), dr = lbvh_delta(keys, n, i, i + 1);
    int d = dr > dl ? 1 : -1;
    int dmin = d > 0 ? dl : dr;
    int lmax = 2;
    while (lbvh_delta(keys, n, i, i + lmax * d) > dmin) lmax *= 2;
    int l = 0;
    for (int t = lmax / 2; t >= 1; t /= 2)
        if (lbvh_delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
    int j = i + l * d;
    int dnode = lbvh_delta(keys, n, i, j);
    int s = 0;
    int step = l;
    do {
        step = (step + 1) >> 1;
        if (lbvh_delta(keys, n, i, i + (s + step) * d) > dnode) s += step;
    } while (step > 1);
    int gamma = i + s * d + (d < 0 ? -1 : 0);
    int lo = i < j ? i : j, hi = i < j ? j : i;
    int2 c;
    if (lo == gamma) {
        c.x = ~gamma;
        parent_leaf[gamma] = i;
    } else {
        c.x = gamma;
        parent_internal[gamma] = i;
    }
    if (hi == gamma + 1) {
        c.y = ~(gamma + 1);
        parent_leaf[gamma + 1] = i;
    } else {
        c.y = gamma + 1;
        parent_internal[gamma + 1] = i;
    }
    children[i] = c;
}

struct Box { float lo[3], hi[3]; };

HD Box tri_box(float4 a, float4 b, float4 c) {
    Box r;
    r.lo[0] = fminf(fminf(a.x, b.x), c.x);
    r.lo[1] = fminf(fminf(a.y, b.y), c.y);
    r.lo[2] = fminf(fminf(a.z, b.z), c.z);
    r.hi[0] = fmaxf(fmaxf(a.x, b.x), c.x);
    r.hi[1] = fmaxf(fmaxf(a.y, b.y), c.y);
    r.hi[2] = fmaxf(fmaxf(a.z, b.z), c.z);
    return r;
}

HD Box box_union(const Box &a, const Box &b) {
    Box r;
    for (int k = 0; k < 3; k++) {
        r.lo[k] = fminf(a.lo[k], b.lo[k]);
        r.hi[k] = fmaxf(a.hi[k], b.hi[k]);
    }
    return r;
}

HD void write_node(float4 *node, const Box &b0, const Box &b1, int c0, int c1) {
    float4 n0, n1, n2, n3;
    n0.x = b0.lo[0]; n0.y = b0.lo[1]; n0.z = b0.lo[2]; n0.w = b0.hi[0];
    n1.x = b0.hi[1]; n1.y = b0.hi[2]; n1.z = b1.lo[0]; n1.w = b1.lo[1];
    n2.x = b1.lo[2]; n2.y = b1.hi[0]; n2.z = b1.hi[1]; n2.w = b1.hi[2];
    n3.x = dr_i2f(c0); n3.y = dr_i2f(c1); n3.z = 0.f; n3.w = 0.f;
    node[0] = n0;
    node[1] = n1;
    node[2] = n2;
    node[3] = n3;
}
