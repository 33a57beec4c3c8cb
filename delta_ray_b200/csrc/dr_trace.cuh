// Ray casting on the LBVH and analytic re-intersection of the hit triangle.
//
// Hit rule (identical to the oracle's CPU BVH, so hit ids agree): a triangle is
// hit when Moller-Trumbore gives u >= 0, v >= 0, u + v <= 1 and
// tnear < t < tfar; the smallest t wins, equal t goes to the lower global
// triangle id.  The hit test is written with round-to-nearest intrinsics so
// that it evaluates exactly the same IEEE operations as the CPU oracle.
//
// Ray intervals follow scene.cpp of the reference: closest hit on
// (1e-3, inf) (scene.cpp:188-189), shadow rays on (1e-3 d, (1 - 1e-3) d)
// (scene.cpp:159-160).  The hit point itself is recomputed by intersect_tri
// exactly as intersect.h:100-148 does.
#pragma once

#include "dr_scene.cuh"

#ifdef DR_HOST_BUILD
HD float fmul_rn(float a, float b) { return a * b; }
HD float fadd_rn(float a, float b) { return a + b; }
HD float fsub_rn(float a, float b) { return a - b; }
HD float frcp_rn(float a) { return 1.f / a; }
#else
DEV float fmul_rn(float a, float b) { return __fmul_rn(a, b); }
DEV float fadd_rn(float a, float b) { return __fadd_rn(a, b); }
DEV float fsub_rn(float a, float b) { return __fsub_rn(a, b); }
DEV float frcp_rn(float a) { return __frcp_rn(a); }
#endif

#define DR_INF dr_i2f(0x7f800000)

// Node-visit counter, only in the CPU build of this code used by the tests.
#ifdef DR_HOST_BUILD
extern thread_local long long g_dr_visits;
#define DR_COUNT_VISIT() (g_dr_visits++)
#else
#define DR_COUNT_VISIT()
#endif
// Traversal stack depth.  The stack never overflows: along a root-to-leaf
// path of the Karras LBVH (dr_bvh.cuh) the nodes' common-prefix lengths
// (lbvh_delta) strictly increase.  Distinct 30-bit Morton keys give prefix
// lengths clz(a ^ b) in [2, 31], 30 values; equal keys give 32 + clz(i ^ j)
// with i, j < n < 2^31, at most 31 values.  So a path has at most 61 internal
// nodes, each pushes at most one entry, and 64 entries always suffice; the
// push guards below are never taken.
#define DR_STACK 64
static_assert(DR_STACK >= 30 + 31, "LBVH traversal stack shorter than the tree's depth bound");

// Moller-Trumbore with no contraction: the exact operation sequence of the
// oracle's hit test.  Returns false on a miss.
// The triangle's edge vectors e1 = b - a, e2 = c - a and the origin offset
// s = o - a, which rays from one origin share.
struct TriRay {
    float e1x, e1y, e1z, e2x, e2y, e2z, sx, sy, sz;
};
DEV TriRay tri_ray(float4 a, float4 b, float4 c, float3 o) {
    TriRay r;
    r.e1x = fsub_rn(b.x, a.x), r.e1y = fsub_rn(b.y, a.y), r.e1z = fsub_rn(b.z, a.z);
    r.e2x = fsub_rn(c.x, a.x), r.e2y = fsub_rn(c.y, a.y), r.e2z = fsub_rn(c.z, a.z);
    r.sx = fsub_rn(o.x, a.x), r.sy = fsub_rn(o.y, a.y), r.sz = fsub_rn(o.z, a.z);
    return r;
}
DEV bool hit_triangle(const TriRay &r, float3 d, float &t_out) {
    const float e1x = r.e1x, e1y = r.e1y, e1z = r.e1z, e2x = r.e2x, e2y = r.e2y, e2z = r.e2z;
    const float sx = r.sx, sy = r.sy, sz = r.sz;
    float px = fsub_rn(fmul_rn(d.y, e2z), fmul_rn(d.z, e2y));
    float py = fsub_rn(fmul_rn(d.z, e2x), fmul_rn(d.x, e2z));
    float pz = fsub_rn(fmul_rn(d.x, e2y), fmul_rn(d.y, e2x));
    float det = fadd_rn(fadd_rn(fmul_rn(e1x, px), fmul_rn(e1y, py)), fmul_rn(e1z, pz));
    if (det == 0.f) return false;
    float inv = frcp_rn(det);
    float u = fmul_rn(fadd_rn(fadd_rn(fmul_rn(sx, px), fmul_rn(sy, py)), fmul_rn(sz, pz)), inv);
    if (u < 0.f || u > 1.f) return false;
    float qx = fsub_rn(fmul_rn(sy, e1z), fmul_rn(sz, e1y));
    float qy = fsub_rn(fmul_rn(sz, e1x), fmul_rn(sx, e1z));
    float qz = fsub_rn(fmul_rn(sx, e1y), fmul_rn(sy, e1x));
    float v = fmul_rn(fadd_rn(fadd_rn(fmul_rn(d.x, qx), fmul_rn(d.y, qy)), fmul_rn(d.z, qz)), inv);
    if (v < 0.f || fadd_rn(u, v) > 1.f) return false;
    t_out = fmul_rn(fadd_rn(fadd_rn(fmul_rn(e2x, qx), fmul_rn(e2y, qy)), fmul_rn(e2z, qz)), inv);
    return true;
}
DEV bool hit_triangle(float4 a, float4 b, float4 c, float3 o, float3 d, float &t_out) {
    return hit_triangle(tri_ray(a, b, c, o), d, t_out);
}

HD float safe_inv(float x) {
    const float big = 1e30f;
    if (x == 0.f) return big;
    float r = 1.f / x;
    return r > big ? big : (r < -big ? -big : r);
}

// Slab test of one child box against [0, tmax]; returns the entry distance
// (>= 0) or -1 on a miss.  The far distance is widened by 2 gamma(3) (pbrt) so
// that a hit lying on a box face is never culled.
DEV float box_entry(float lx, float ly, float lz, float hx, float hy, float hz, float3 o, float3 inv, float tmax) {
    float t0x = (lx - o.x) * inv.x, t1x = (hx - o.x) * inv.x;
    float t0y = (ly - o.y) * inv.y, t1y = (hy - o.y) * inv.y;
    float t0z = (lz - o.z) * inv.z, t1z = (hz - o.z) * inv.z;
    float tn = fmaxf(fmaxf(fminf(t0x, t1x), fminf(t0y, t1y)), fmaxf(fminf(t0z, t1z), 0.f));
    float tf = fminf(fminf(fmaxf(t0x, t1x), fmaxf(t0y, t1y)), fminf(fmaxf(t0z, t1z), tmax * 1.0000004f));
    tf *= 1.0000004f;
    return tn <= tf ? tn : -1.f;
}

struct Hit {
    int tri;  // global triangle id, -1 for a miss
    float t;
};

// Closest hit on (tnear, inf) in the LBVH (nodes, tris) rooted at root.
DEV_NOINLINE Hit trace_closest_bvh(const float4 *DR_RESTRICT nodes, const float4 *DR_RESTRICT tris, int root, float3 o,
                                   float3 d, float tnear) {
    Hit h;
    h.tri = -1;
    h.t = DR_INF;
    float3 inv = f3(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z));
    int stack[DR_STACK];
    int sp = 0;
    int node = root;
    while (true) {
        DR_COUNT_VISIT();
        if (node < 0) {
            int leaf = ~node;
            float4 a = dr_ldg(tris + 3 * leaf), b = dr_ldg(tris + 3 * leaf + 1), c = dr_ldg(tris + 3 * leaf + 2);
            float t;
            if (hit_triangle(a, b, c, o, d, t) && t > tnear) {
                int id = dr_f2i(a.w);
                if (t < h.t || (t == h.t && id < h.tri)) {
                    h.t = t;
                    h.tri = id;
                }
            }
            if (sp == 0) break;
            node = stack[--sp];
            continue;
        }
        const float4 *n = nodes + 4 * node;
        float4 n0 = dr_ldg(n), n1 = dr_ldg(n + 1), n2 = dr_ldg(n + 2), n3 = dr_ldg(n + 3);
        float e0 = box_entry(n0.x, n0.y, n0.z, n0.w, n1.x, n1.y, o, inv, h.t);
        float e1 = box_entry(n1.z, n1.w, n2.x, n2.y, n2.z, n2.w, o, inv, h.t);
        int c0 = dr_f2i(n3.x), c1 = dr_f2i(n3.y);
        bool h0 = e0 >= 0.f, h1 = e1 >= 0.f;
        if (h0 && h1) {
            int nearc = e0 <= e1 ? c0 : c1, farc = e0 <= e1 ? c1 : c0;
            if (sp < DR_STACK) stack[sp++] = farc;
            node = nearc;
        } else if (h0) {
            node = c0;
        } else if (h1) {
            node = c1;
        } else {
            if (sp == 0) break;
            node = stack[--sp];
        }
    }
    return h;
}

// Scenes of at most DR_LINEAR_TRIS triangles are traced by testing every
// triangle: a loop that all lanes of a warp run in step, with no stack.  Both
// ways keep the smallest t, ties going to the smaller triangle id, so they
// agree unless the walk's widened box test (2 gamma(3)) rounds a hit lying
// within ~1e-6 of the closest one out of its box.

DEV_NOINLINE Hit trace_closest_linear(const float4 *DR_RESTRICT tris, int n, float3 o, float3 d, float tnear) {
    Hit h;
    h.tri = -1;
    h.t = DR_INF;
    for (int i = 0; i < n; i++) {
        float4 a = dr_ldg(tris + 3 * i), b = dr_ldg(tris + 3 * i + 1), c = dr_ldg(tris + 3 * i + 2);
        float t;
        if (hit_triangle(a, b, c, o, d, t) && t > tnear) {
            int id = dr_f2i(a.w);
            if (t < h.t || (t == h.t && id < h.tri)) {
                h.t = t;
                h.tri = id;
            }
        }
    }
    return h;
}

// Closest hits of two rays from one origin (the two sides of an edge sample)
// by testing every triangle; each triangle's tri_ray serves both rays.
DEV_NOINLINE void trace_closest_pair_linear(const float4 *DR_RESTRICT tris, int n, float3 o, float3 d0, float3 d1,
                                            float tnear, Hit &h0, Hit &h1) {
    h0.tri = h1.tri = -1;
    h0.t = h1.t = DR_INF;
    for (int i = 0; i < n; i++) {
        float4 a = dr_ldg(tris + 3 * i), b = dr_ldg(tris + 3 * i + 1), c = dr_ldg(tris + 3 * i + 2);
        TriRay r = tri_ray(a, b, c, o);
        int id = dr_f2i(a.w);
        float t;
        if (hit_triangle(r, d0, t) && t > tnear && (t < h0.t || (t == h0.t && id < h0.tri))) {
            h0.t = t;
            h0.tri = id;
        }
        if (hit_triangle(r, d1, t) && t > tnear && (t < h1.t || (t == h1.t && id < h1.tri))) {
            h1.t = t;
            h1.tri = id;
        }
    }
}

// Closest hits of two rays from one origin (the two sides of an edge sample,
// whose directions differ by a few 1e-3) in one walk of the LBVH: a node is
// entered when either ray enters one of its boxes before that ray's closest
// hit so far, nearer child first by the smaller of the two entries, and a
// leaf's triangle is tested against both rays with shared edge vectors.  Each
// ray gets the hit its own walk finds: a box the other ray's walk enters holds
// no closer hit for it (the test is conservative), and the rule (smallest t,
// ties to the smaller triangle id) does not depend on the order of the tests.
DEV_NOINLINE void trace_closest_pair_bvh(const float4 *DR_RESTRICT nodes, const float4 *DR_RESTRICT tris, int root,
                                         float3 o, float3 d0, float3 d1, float tnear, Hit &h0, Hit &h1) {
    h0.tri = h1.tri = -1;
    h0.t = h1.t = DR_INF;
    float3 i0 = f3(safe_inv(d0.x), safe_inv(d0.y), safe_inv(d0.z));
    float3 i1 = f3(safe_inv(d1.x), safe_inv(d1.y), safe_inv(d1.z));
    int stack[DR_STACK];
    int sp = 0;
    int node = root;
    while (true) {
        DR_COUNT_VISIT();
        if (node < 0) {
            int leaf = ~node;
            float4 a = dr_ldg(tris + 3 * leaf), b = dr_ldg(tris + 3 * leaf + 1), c = dr_ldg(tris + 3 * leaf + 2);
            TriRay r = tri_ray(a, b, c, o);
            int id = dr_f2i(a.w);
            float t;
            if (hit_triangle(r, d0, t) && t > tnear && (t < h0.t || (t == h0.t && id < h0.tri))) {
                h0.t = t;
                h0.tri = id;
            }
            if (hit_triangle(r, d1, t) && t > tnear && (t < h1.t || (t == h1.t && id < h1.tri))) {
                h1.t = t;
                h1.tri = id;
            }
            if (sp == 0) break;
            node = stack[--sp];
            continue;
        }
        const float4 *n = nodes + 4 * node;
        float4 n0 = dr_ldg(n), n1 = dr_ldg(n + 1), n2 = dr_ldg(n + 2), n3 = dr_ldg(n + 3);
        float a0 = box_entry(n0.x, n0.y, n0.z, n0.w, n1.x, n1.y, o, i0, h0.t);
        float b0 = box_entry(n0.x, n0.y, n0.z, n0.w, n1.x, n1.y, o, i1, h1.t);
        float a1 = box_entry(n1.z, n1.w, n2.x, n2.y, n2.z, n2.w, o, i0, h0.t);
        float b1 = box_entry(n1.z, n1.w, n2.x, n2.y, n2.z, n2.w, o, i1, h1.t);
        int c0 = dr_f2i(n3.x), c1 = dr_f2i(n3.y);
        bool x0 = a0 >= 0.f || b0 >= 0.f, x1 = a1 >= 0.f || b1 >= 0.f;
        if (x0 && x1) {
            float e0 = a0 >= 0.f ? (b0 >= 0.f ? fminf(a0, b0) : a0) : b0;
            float e1 = a1 >= 0.f ? (b1 >= 0.f ? fminf(a1, b1) : a1) : b1;
            int nearc = e0 <= e1 ? c0 : c1, farc = e0 <= e1 ? c1 : c0;
            if (sp < DR_STACK) stack[sp++] = farc;
            node = nearc;
        } else if (x0) {
            node = c0;
        } else if (x1) {
            node = c1;
        } else {
            if (sp == 0) break;
            node = stack[--sp];
        }
    }
}

DEV Hit trace_closest(const DevScene &s, float3 o, float3 d, float tnear) {
    if (s.num_tris == 0) {
        Hit h;
        h.tri = -1;
        h.t = DR_INF;
        return h;
    }
    if (s.num_tris <= DR_LINEAR_TRIS) return trace_closest_linear(s.bvh_tris, s.num_tris, o, d, tnear);
    // closest hits walk the binary nodes: a lane's own loop over them ran
    // faster than over the 4-wide nodes (the kernels that trace closest hits
    // measured 18-24 % slower with the 4-wide walk); the warp-stepped
    // occlusion walks of k_edge_connect take the 4-wide one (fewer steps)
    return trace_closest_bvh(s.bvh_nodes, s.bvh_tris, s.bvh_root, o, d, tnear);
}

// Any hit on (tnear, tfar).
DEV_NOINLINE bool trace_any_bvh(const float4 *DR_RESTRICT nodes, const float4 *DR_RESTRICT tris, int root, float3 o,
                                float3 d, float tnear, float tfar) {
    float3 inv = f3(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z));
    int stack[DR_STACK];
    int sp = 0;
    int node = root;
    while (true) {
        if (node < 0) {
            int leaf = ~node;
            float4 a = dr_ldg(tris + 3 * leaf), b = dr_ldg(tris + 3 * leaf + 1), c = dr_ldg(tris + 3 * leaf + 2);
            float t;
            if (hit_triangle(a, b, c, o, d, t) && t > tnear && t < tfar) return true;
            if (sp == 0) break;
            node = stack[--sp];
            continue;
        }
        const float4 *n = nodes + 4 * node;
        float4 n0 = dr_ldg(n), n1 = dr_ldg(n + 1), n2 = dr_ldg(n + 2), n3 = dr_ldg(n + 3);
        float e0 = box_entry(n0.x, n0.y, n0.z, n0.w, n1.x, n1.y, o, inv, tfar);
        float e1 = box_entry(n1.z, n1.w, n2.x, n2.y, n2.z, n2.w, o, inv, tfar);
        int c0 = dr_f2i(n3.x), c1 = dr_f2i(n3.y);
        bool h0 = e0 >= 0.f, h1 = e1 >= 0.f;
        if (h0 && h1) {
            if (sp < DR_STACK) stack[sp++] = c1;
            node = c0;
        } else if (h0) {
            node = c0;
        } else if (h1) {
            node = c1;
        } else {
            if (sp == 0) break;
            node = stack[--sp];
        }
    }
    return false;
}

// The 4-wide node of internal node p (DevScene::bvh_wide, DR_WIDE_F4 float4 at
// w): p's two children, each internal child replaced by its own two children
// with the boxes its node holds for them.  A walk from the root only reads
// the wide nodes of the root and of nodes two levels apart, so every binary
// node is tested in the same boxes as in the binary walk.
HD void widen_node(const float4 *nodes, int p, float4 *w) {
    float lo[3][4], hi[3][4];
    int ref[4];
    int k = 0;
    const float4 *np = nodes + 4 * p;
    const float4 a0 = np[0], a1 = np[1], a2 = np[2], a3 = np[3];
    const float pb[2][6] = {{a0.x, a0.y, a0.z, a0.w, a1.x, a1.y}, {a1.z, a1.w, a2.x, a2.y, a2.z, a2.w}};
    const int pc[2] = {dr_f2i(a3.x), dr_f2i(a3.y)};
    for (int j = 0; j < 2; j++) {
        if (pc[j] < 0) {  // a leaf child stands for itself
            for (int ax = 0; ax < 3; ax++) {
                lo[ax][k] = pb[j][ax];
                hi[ax][k] = pb[j][3 + ax];
            }
            ref[k++] = pc[j];
            continue;
        }
        const float4 *cp = nodes + 4 * pc[j];
        const float4 b0 = cp[0], b1 = cp[1], b2 = cp[2], b3 = cp[3];
        const float cb[2][6] = {{b0.x, b0.y, b0.z, b0.w, b1.x, b1.y}, {b1.z, b1.w, b2.x, b2.y, b2.z, b2.w}};
        const int cc[2] = {dr_f2i(b3.x), dr_f2i(b3.y)};
        for (int g = 0; g < 2; g++) {
            for (int ax = 0; ax < 3; ax++) {
                lo[ax][k] = cb[g][ax];
                hi[ax][k] = cb[g][3 + ax];
            }
            ref[k++] = cc[g];
        }
    }
    for (; k < 4; k++) {
        for (int ax = 0; ax < 3; ax++) {
            lo[ax][k] = 1.f;  // an empty box; the walks skip the slot by its id
            hi[ax][k] = 0.f;
        }
        ref[k] = DR_WIDE_EMPTY;
    }
    for (int ax = 0; ax < 3; ax++) {
        w[ax].x = lo[ax][0];
        w[ax].y = lo[ax][1];
        w[ax].z = lo[ax][2];
        w[ax].w = lo[ax][3];
        w[3 + ax].x = hi[ax][0];
        w[3 + ax].y = hi[ax][1];
        w[3 + ax].z = hi[ax][2];
        w[3 + ax].w = hi[ax][3];
    }
    w[6].x = dr_i2f(ref[0]);
    w[6].y = dr_i2f(ref[1]);
    w[6].z = dr_i2f(ref[2]);
    w[6].w = dr_i2f(ref[3]);
    w[7].x = w[7].y = w[7].z = w[7].w = 0.f;
}

// Steps of the walks over the LBVH's 4-wide form (see trace_before_wide);
// their stack holds up to three children per 4-wide level, and a path of at
// most 61 binary levels crosses at most 31 of those: 93 entries always
// suffice, so the push guards are never taken.
#define DR_WIDE_STACK 96
static_assert(DR_WIDE_STACK >= 3 * ((30 + 31 + 1) / 2), "4-wide traversal stack shorter than its depth bound");

// The children of wide node w whose boxes the ray enters before tmax, nearest
// first: n of them in c[0..n).
struct WideKids {
    int n;
    int c[4];
};
DEV void wide_swap(float &ka, int &ca, float &kb, int &cb) {
    if (kb < ka) {
        const float k = ka;
        ka = kb;
        kb = k;
        const int c = ca;
        ca = cb;
        cb = c;
    }
}
DEV WideKids wide_kids(const float4 *DR_RESTRICT w, float3 o, float3 inv, float tmax) {
    const float4 lx = dr_ldg(w), ly = dr_ldg(w + 1), lz = dr_ldg(w + 2);
    const float4 hx = dr_ldg(w + 3), hy = dr_ldg(w + 4), hz = dr_ldg(w + 5), rf = dr_ldg(w + 6);
    int c0 = dr_f2i(rf.x), c1 = dr_f2i(rf.y), c2 = dr_f2i(rf.z), c3 = dr_f2i(rf.w);
    float k0 = c0 != DR_WIDE_EMPTY ? box_entry(lx.x, ly.x, lz.x, hx.x, hy.x, hz.x, o, inv, tmax) : -1.f;
    float k1 = c1 != DR_WIDE_EMPTY ? box_entry(lx.y, ly.y, lz.y, hx.y, hy.y, hz.y, o, inv, tmax) : -1.f;
    float k2 = c2 != DR_WIDE_EMPTY ? box_entry(lx.z, ly.z, lz.z, hx.z, hy.z, hz.z, o, inv, tmax) : -1.f;
    float k3 = c3 != DR_WIDE_EMPTY ? box_entry(lx.w, ly.w, lz.w, hx.w, hy.w, hz.w, o, inv, tmax) : -1.f;
    WideKids r;
    r.n = (k0 >= 0.f) + (k1 >= 0.f) + (k2 >= 0.f) + (k3 >= 0.f);
    // misses sort last
    k0 = k0 >= 0.f ? k0 : DR_INF;
    k1 = k1 >= 0.f ? k1 : DR_INF;
    k2 = k2 >= 0.f ? k2 : DR_INF;
    k3 = k3 >= 0.f ? k3 : DR_INF;
    wide_swap(k0, c0, k1, c1);
    wide_swap(k2, c2, k3, c3);
    wide_swap(k0, c0, k2, c2);
    wide_swap(k1, c1, k3, c3);
    wide_swap(k1, c1, k2, c2);
    r.c[0] = c0;
    r.c[1] = c1;
    r.c[2] = c2;
    r.c[3] = c3;
    return r;
}
// The next node of a wide walk after wide node children k: the nearest, with
// the others stacked; false when the stack is empty too.
DEV bool wide_next(const WideKids &k, int *stack, int &sp, int &node) {
    if (k.n == 0) {
        if (sp == 0) return false;
        node = stack[--sp];
        return true;
    }
    if (k.n > 3 && sp < DR_WIDE_STACK) stack[sp++] = k.c[3];
    if (k.n > 2 && sp < DR_WIDE_STACK) stack[sp++] = k.c[2];
    if (k.n > 1 && sp < DR_WIDE_STACK) stack[sp++] = k.c[1];
    node = k.c[0];
    return true;
}

// The walk of trace_before_bvh as a resumable state: begin() sets it up,
// step() takes one node (a box pair or a leaf) and returns 0 while the walk
// goes on, 1 when a triangle hits ahead of (ta, ida), 2 when none does.
// Kernels that interleave many such walks step every walking lane together.
struct BeforeWalk {
    float3 o, d, inv;
    float tnear, ta;
    int ida, sp, node;
    int stack[DR_WIDE_STACK];
    DEV void begin(int root, float3 o_, float3 d_, float tnear_, float ta_, int ida_) {
        o = o_;
        d = d_;
        inv = f3(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z));
        tnear = tnear_;
        ta = ta_;
        ida = ida_;
        sp = 0;
        node = root;
    }
    // wide (may be null): the 4-wide form of the tree, walked in its place
    DEV int step(const float4 *DR_RESTRICT nodes, const float4 *DR_RESTRICT wide, const float4 *DR_RESTRICT tris) {
        if (node < 0) {
            const int leaf = ~node;
            float4 a = dr_ldg(tris + 3 * leaf), b = dr_ldg(tris + 3 * leaf + 1), c = dr_ldg(tris + 3 * leaf + 2);
            float t;
            if (hit_triangle(a, b, c, o, d, t) && t > tnear && (t < ta || (t == ta && dr_f2i(a.w) < ida))) return 1;
            if (sp == 0) return 2;
            node = stack[--sp];
            return 0;
        }
        if (wide) return wide_next(wide_kids(wide + (size_t)DR_WIDE_F4 * node, o, inv, ta), stack, sp, node) ? 0 : 2;
        const float4 *n = nodes + 4 * node;
        float4 n0 = dr_ldg(n), n1 = dr_ldg(n + 1), n2 = dr_ldg(n + 2), n3 = dr_ldg(n + 3);
        float e0 = box_entry(n0.x, n0.y, n0.z, n0.w, n1.x, n1.y, o, inv, ta);
        float e1 = box_entry(n1.z, n1.w, n2.x, n2.y, n2.z, n2.w, o, inv, ta);
        int c0 = dr_f2i(n3.x), c1 = dr_f2i(n3.y);
        bool h0 = e0 >= 0.f, h1 = e1 >= 0.f;
        if (h0 && h1) {
            int nearc = e0 <= e1 ? c0 : c1, farc = e0 <= e1 ? c1 : c0;
            if (sp < DR_STACK) stack[sp++] = farc;
            node = nearc;
        } else if (h0) {
            node = c0;
        } else if (h1) {
            node = c1;
        } else {
            if (sp == 0) return 2;
            node = stack[--sp];
        }
        return 0;
    }
};

// Whether a triangle hits ahead of (ta, ida) under the closest-hit rule: at t
// on (tnear, ta), or at ta with a smaller id.  Boxes are culled at ta (the
// widened test keeps every box holding such a hit), nearer child first.
DEV_NOINLINE bool trace_before_bvh(const float4 *DR_RESTRICT nodes, const float4 *DR_RESTRICT tris, int root,
                                   float3 o, float3 d, float tnear, float ta, int ida) {
    float3 inv = f3(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z));
    int stack[DR_STACK];
    int sp = 0;
    int node = root;
    while (true) {
        if (node < 0) {
            int leaf = ~node;
            float4 a = dr_ldg(tris + 3 * leaf), b = dr_ldg(tris + 3 * leaf + 1), c = dr_ldg(tris + 3 * leaf + 2);
            float t;
            if (hit_triangle(a, b, c, o, d, t) && t > tnear && (t < ta || (t == ta && dr_f2i(a.w) < ida)))
                return true;
            if (sp == 0) break;
            node = stack[--sp];
            continue;
        }
        const float4 *n = nodes + 4 * node;
        float4 n0 = dr_ldg(n), n1 = dr_ldg(n + 1), n2 = dr_ldg(n + 2), n3 = dr_ldg(n + 3);
        float e0 = box_entry(n0.x, n0.y, n0.z, n0.w, n1.x, n1.y, o, inv, ta);
        float e1 = box_entry(n1.z, n1.w, n2.x, n2.y, n2.z, n2.w, o, inv, ta);
        int c0 = dr_f2i(n3.x), c1 = dr_f2i(n3.y);
        bool h0 = e0 >= 0.f, h1 = e1 >= 0.f;
        if (h0 && h1) {
            int nearc = e0 <= e1 ? c0 : c1, farc = e0 <= e1 ? c1 : c0;
            if (sp < DR_STACK) stack[sp++] = farc;
            node = nearc;
        } else if (h0) {
            node = c0;
        } else if (h1) {
            node = c1;
        } else {
            if (sp == 0) break;
            node = stack[--sp];
        }
    }
    return false;
}

// ---------------------------------------------------------------------------
// Walks of the 4-wide form of the LBVH (DevScene::bvh_wide), taken by the
// warp-stepped occlusion walks (BeforeWalk) and by trace_before; closest and
// any hits walk the binary nodes (see trace_closest).  Each step tests
// a node's (up to) four children, the binary walk's two levels at once, in
// the same boxes, and goes on with the nearest child entered, the others
// stacked nearest on top.  The hits are those of the binary walks: a box is
// culled only beyond the best hit so far, and the closest-hit rule (smallest
// t, ties to the smaller triangle id) does not depend on the order.
DEV_NOINLINE bool trace_before_wide(const float4 *DR_RESTRICT wide, const float4 *DR_RESTRICT tris, int root,
                                    float3 o, float3 d, float tnear, float ta, int ida) {
    const float3 inv = f3(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z));
    int stack[DR_WIDE_STACK];
    int sp = 0;
    int node = root;
    while (true) {
        if (node < 0) {
            const int leaf = ~node;
            float4 a = dr_ldg(tris + 3 * leaf), b = dr_ldg(tris + 3 * leaf + 1), c = dr_ldg(tris + 3 * leaf + 2);
            float t;
            if (hit_triangle(a, b, c, o, d, t) && t > tnear && (t < ta || (t == ta && dr_f2i(a.w) < ida)))
                return true;
            if (sp == 0) break;
            node = stack[--sp];
            continue;
        }
        if (!wide_next(wide_kids(wide + (size_t)DR_WIDE_F4 * node, o, inv, ta), stack, sp, node)) break;
    }
    return false;
}

// trace_before_bvh on the scene's tree (the 4-wide form where there is one)
DEV bool trace_before(const DevScene &s, float3 o, float3 d, float tnear, float ta, int ida) {
    if (s.bvh_wide) return trace_before_wide(s.bvh_wide, s.bvh_tris, s.bvh_root, o, d, tnear, ta, ida);
    return trace_before_bvh(s.bvh_nodes, s.bvh_tris, s.bvh_root, o, d, tnear, ta, ida);
}

DEV_NOINLINE bool trace_any_linear(const float4 *DR_RESTRICT tris, int n, float3 o, float3 d, float tnear,
                                   float tfar) {
    for (int i = 0; i < n; i++) {
        float4 a = dr_ldg(tris + 3 * i), b = dr_ldg(tris + 3 * i + 1), c = dr_ldg(tris + 3 * i + 2);
        float t;
        if (hit_triangle(a, b, c, o, d, t) && t > tnear && t < tfar) return true;
    }
    return false;
}

DEV bool trace_any(const DevScene &s, float3 o, float3 d, float tnear, float tfar) {
    if (s.num_tris == 0) return false;
    if (s.num_tris <= DR_LINEAR_TRIS) return trace_any_linear(s.bvh_tris, s.num_tris, o, d, tnear, tfar);
    // binary, as closest hits (the 4-wide any-hit walk made the shading
    // kernels' shadow rays 8 % slower)
    return trace_any_bvh(s.bvh_nodes, s.bvh_tris, s.bvh_root, o, d, tnear, tfar);
}

// occluded(scene, ray, max_t) of the reference (scene.cpp:147-166)
DEV bool occluded(const DevScene &s, float3 o, float3 d, float max_t) {
    return trace_any(s, o, d, max_t * 1e-3f, max_t * (1.f - 1e-3f));
}

// ---------------------------------------------------------------------------
// Surface points and analytic re-intersection (intersect.h:100-148)
// ---------------------------------------------------------------------------
struct SurfacePoint {
    float3 p, ng;
    Frame f;
    float2 uv;
};

struct TriData {
    float3 v0, v1, v2;
    float3 n0, n1, n2;
    float2 t0, t1, t2;  // uvs (defaults (0,0),(1,0),(1,1): intersect.h:115-117)
    bool has_n;
    int shape;
};

DEV TriData load_tri(const DevScene &s, int tri) {
    TriData td;
    int4 id = tri_vids(s, tri);
    td.shape = id.w;
    td.v0 = vtx3(s.vtx, id.x);
    td.v1 = vtx3(s.vtx, id.y);
    td.v2 = vtx3(s.vtx, id.z);
    DevShape sh = s.shapes[id.w];
    td.has_n = sh.has_n != 0;
    if (td.has_n) {
        td.n0 = vtx3(s.nrm, id.x);
        td.n1 = vtx3(s.nrm, id.y);
        td.n2 = vtx3(s.nrm, id.z);
    } else {
        td.n0 = td.n1 = td.n2 = f3(0.f);
    }
    if (sh.has_uv) {
        td.t0.x = dr_ldg(s.uv + 2 * id.x); td.t0.y = dr_ldg(s.uv + 2 * id.x + 1);
        td.t1.x = dr_ldg(s.uv + 2 * id.y); td.t1.y = dr_ldg(s.uv + 2 * id.y + 1);
        td.t2.x = dr_ldg(s.uv + 2 * id.z); td.t2.y = dr_ldg(s.uv + 2 * id.z + 1);
    } else {
        td.t0.x = 0.f; td.t0.y = 0.f;
        td.t1.x = 1.f; td.t1.y = 0.f;
        td.t2.x = 1.f; td.t2.y = 1.f;
    }
    return td;
}

struct IsectFwd {  // forward intermediates of intersect_tri, kept for its adjoint
    float3 e1, e2, pvec, s, qvec, cg, ns;
    float div, ru, rv, rt, u, v, w, t;
    bool div_fixed, flip;
};

// `ad`: reciprocal-multiply divisions, as the reference's differentiated pass
// computes them (see sample_primary).
DEV SurfacePoint intersect_tri(const TriData &td, float3 o, float3 d, IsectFwd *fw = nullptr, bool ad = false) {
    IsectFwd f;
    f.e1 = td.v1 - td.v0;
    f.e2 = td.v2 - td.v0;
    f.pvec = cross(d, f.e2);
    f.div = dot(f.pvec, f.e1);
    f.div_fixed = f.div == 0.f;
    if (f.div_fixed) f.div = 1e-8f;  // intersect.h:80-83
    f.s = o - td.v0;
    f.ru = dot(f.s, f.pvec);
    f.qvec = cross(f.s, f.e1);
    f.rv = dot(d, f.qvec);
    f.rt = dot(f.e2, f.qvec);
    if (ad) {
        float inv = 1.f / f.div;
        f.u = f.ru * inv;
        f.v = f.rv * inv;
        f.t = f.rt * inv;
    } else {
        f.u = f.ru / f.div;
        f.v = f.rv / f.div;
        f.t = f.rt / f.div;
    }
    f.w = 1.f - (f.u + f.v);
    SurfacePoint sp;
    sp.uv.x = f.w * td.t0.x + f.u * td.t1.x + f.v * td.t2.x;
    sp.uv.y = f.w * td.t0.y + f.u * td.t1.y + f.v * td.t2.y;
    sp.p = o + d * f.t;
    f.cg = cross(td.v1 - td.v0, td.v2 - td.v0);
    float3 gn = normalize(f.cg);
    float3 sn = gn;
    f.flip = false;
    if (td.has_n) {
        f.ns = f.w * td.n0 + f.u * td.n1 + f.v * td.n2;
        sn = normalize(f.ns);
        if (dot(gn, sn) < 0.f) {
            gn = -gn;
            f.flip = true;
        }
    }
    sp.ng = gn;
    sp.f = make_frame(sn);
    if (fw) *fw = f;
    return sp;
}

struct TriGrad {
    float3 v0, v1, v2, n0, n1, n2;
};

// Adjoint of intersect_tri.  d_p, d_ng, d_frame, d_uv are output adjoints;
// accumulates vertex / normal adjoints into g and ray adjoints into d_o, d_d.
DEV void d_intersect_tri(const TriData &td, float3 o, float3 d, const IsectFwd &f, float3 d_p, float3 d_ng,
                         const Frame &d_frame, float2 d_uv, TriGrad &g, float3 &d_o, float3 &d_d) {
    float3 gn0 = normalize(f.cg);
    float3 sn = td.has_n ? normalize(f.ns) : gn0;
    float3 d_sn = d_make_frame(sn, d_frame);
    float d_u = 0.f, d_v = 0.f, d_w = 0.f;
    float3 d_gn;
    if (td.has_n) {
        float3 d_ns = d_normalize(f.ns, d_sn);
        d_w += dot(d_ns, td.n0);
        d_u += dot(d_ns, td.n1);
        d_v += dot(d_ns, td.n2);
        g.n0 += f.w * d_ns;
        g.n1 += f.u * d_ns;
        g.n2 += f.v * d_ns;
        d_gn = f.flip ? -d_ng : d_ng;
    } else {
        d_gn = d_ng + d_sn;
    }
    float3 d_cg = d_normalize(f.cg, d_gn);
    float3 d_e1 = f3(0.f), d_e2 = f3(0.f);
    d_cross(f.e1, f.e2, d_cg, d_e1, d_e2);
    // hit = o + d t
    d_o += d_p;
    d_d += d_p * f.t;
    float d_t = dot(d_p, d);
    // uv = w t0 + u t1 + v t2
    d_w += d_uv.x * td.t0.x + d_uv.y * td.t0.y;
    d_u += d_uv.x * td.t1.x + d_uv.y * td.t1.y;
    d_v += d_uv.x * td.t2.x + d_uv.y * td.t2.y;
    d_u -= d_w;
    d_v -= d_w;
    float inv = 1.f / f.div;
    float d_ru = d_u * inv, d_rv = d_v * inv, d_rt = d_t * inv;
    float d_div = -(d_u * f.ru + d_v * f.rv + d_t * f.rt) * inv * inv;
    if (f.div_fixed) d_div = 0.f;
    float3 d_s = d_ru * f.pvec;
    float3 d_pvec = d_ru * f.s;
    d_d += d_rv * f.qvec;
    float3 d_qvec = d_rv * d;
    d_e2 += d_rt * f.qvec;
    d_qvec += d_rt * f.e2;
    d_cross(f.s, f.e1, d_qvec, d_s, d_e1);
    d_o += d_s;
    g.v0 -= d_s;
    d_pvec += d_div * f.e1;
    d_e1 += d_div * f.pvec;
    d_cross(d, f.e2, d_pvec, d_d, d_e2);
    g.v1 += d_e1;
    g.v0 -= d_e1;
    g.v2 += d_e2;
    g.v0 -= d_e2;
}
