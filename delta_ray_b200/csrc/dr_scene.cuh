// Device-resident scene: flat, read-only arrays in HBM, one struct of raw
// pointers passed by value to every kernel.
//
// Geometry is global over all shapes: vertex i of shape s lives at
// shapes[s].vtx_off + i, triangle j at shapes[s].tri_off + j.  Global triangle
// ids therefore order (shape, triangle) exactly as the reference's Embree
// (geomID, primID) pairs (scene.cpp:100-135).
#pragma once

#include "../../include/delta_ray_b200.h"
#include "dr_common.cuh"

struct DevCamera {
    M4 c2w, w2c;
    float fov, aspect, clip_near;
    int fisheye;
};

struct DevMaterial {
    float kd[3], ks[3], rough;  // constant channels
    int tex_kd, tex_ks, tex_r;  // texel offsets in DevScene::texels, -1 for constants
    int kd_w, kd_h, ks_w, ks_h, r_w, r_h;
    float uv_kd[2], uv_ks[2], uv_r[2];
    int two_sided;
    int model;  // DR_MICROFACET_BLINN_PHONG or DR_MICROFACET_GGX
    int grad_kd, grad_ks, grad_r;  // offsets in the flat gradient
};

struct DevShape {
    int vtx_off, tri_off, nv, nt;
    int mat, light;  // light: index of the light using this shape, -1 if none
    int has_uv, has_n;
    int grad_v, grad_n;  // flat gradient offsets (grad_n = -1 without normals)
};

struct DevLight {
    int shape;
    float I[3];
    int cdf_off;  // offset of the triangle CDF (ntri + 1 floats) and func (ntri floats)
    int ntri;
    float area;   // total area (scene.cpp:40-47)
    float func_int;
    float bc[3], br;  // bounding sphere of the light's AABB (aabb.h:266-270)
    int grad;         // flat gradient offset of d_intensity
};

struct DevEdge { int shape, v0, v1, f0, f1; };  // local vertex / triangle ids

// What the silhouette test of a tree edge needs, computed once per scene
// build (dr_edges.cuh: edge_record): its end points v0, v1, the vertices a, b
// of its two faces opposite it and the faces' unit normals n0, n1;
// r[0] = (v0, n0.x), r[1] = (v1, n0.y), r[2] = (a, n0.z), r[3] = (b, n1.x),
// r[4] = (n1.y, n1.z, always, 0): always != 0 for edges that are silhouettes
// from everywhere (no shading normals, or one face).
struct EdgeRec { float4 r[5]; };

struct DevEdgeNode {
    float lo[3], hi[3];
    float axis[3], angle;
    int offset;  // leaf: first edge; interior: index of the second child
    int nprims;  // 0 for interior nodes
    float total_length;
    int pad;
};

// Paths keep at most DR_MAX_LINKS differentiable specular vertices: later
// ones are treated as constants and are no secondary-edge shading points, so
// a pixel sample hands at most DR_MAX_LINKS + 1 points to edge sampling.
#define DR_MAX_LINKS 8

// Scenes of at most DR_LINEAR_TRIS triangles are traced by testing every
// triangle (dr_trace.cuh); they need the LBVH's leaf array only, which the
// host fills in triangle order.
#define DR_LINEAR_TRIS 16

// A subtree of a point's edge-tree traversal, to be walked on its own (the
// node-keyed draws make its result independent of who walks it and when):
// the point, node | tree << 29 | mode << 30, the node's bound and the three
// path pmfs (cone, all, learned).
struct EdgeTask {
    int point, code;
    float bb, cpmf, apmf, lpmf;
};

// A 4-wide node of the LBVH (DevScene::bvh_wide): float4 0-5 the four child
// boxes by coordinate (lo.x of children 0-3, lo.y, lo.z, hi.x, hi.y, hi.z),
// float4 6 the children (internal node ids, ~leaf for leaves, DR_WIDE_EMPTY
// for an empty slot), float4 7 unused (a node fills one 128-byte line).
#define DR_WIDE_F4 8
#define DR_WIDE_EMPTY 0x7fffffff

struct DevScene {
    DevCamera cam;
    // flat-gradient offset of the camera's block (0; in a batched multi-view
    // call, the view's own block after the scene's gradient) and the view's
    // index, which its shading points carry
    int cam_off, view_id;
    // geometry
    const float *vtx;  // [V][3] global
    const float *nrm;  // [V][3] or null
    const float *uv;   // [V][2] or null
    const int4 *tri;   // global vertex ids (x, y, z) and shape id (w)
    const int *tri_local;
    int num_tris;
    // LBVH
    const float4 *bvh_nodes;  // 4 float4 per internal node (two child boxes + child ids)
    const float4 *bvh_tris;   // 3 float4 per leaf, leaf order (xyz, .w of the first = tri id)
    int bvh_root;             // >= 0 internal node, < 0 leaf (~leaf slot)
    // the same tree read four children at a time: for each internal node, its
    // children's children (a leaf child stands for itself) as one 4-wide node,
    // DR_WIDE_F4 float4 (null: the walks read the binary nodes)
    const float4 *bvh_wide;
    // shapes, materials, lights
    const DevShape *shapes;
    int num_shapes;
    const DevMaterial *mats;
    int num_mats;
    const float *texels;
    const DevLight *lights;
    int num_lights;
    const float *light_sel_cdf;  // [num_lights + 1]
    const float *light_sel_func; // [num_lights]
    float light_sel_func_int;
    float total_light_intensity;
    const float *light_tri_cdf;   // per light: ntri + 1 entries at cdf_off
    const float *light_tri_func;  // per light: ntri entries at cdf_off
    // edges
    const DevEdge *prim_edges;
    int num_prim_edges;
    const float *prim_cdf;  // [n + 1]
    const float *prim_func; // [n]
    float prim_func_int;
    const DevEdgeNode *sil_nodes;
    const DevEdge *sil_edges;
    int num_sil_nodes;
    const DevEdgeNode *nrm_nodes;
    const DevEdge *nrm_edges;
    int num_nrm_nodes;
    const EdgeRec *sil_rec, *nrm_rec;  // per tree edge, in the trees' edge order
    const float *ltc;      // 128*128 row-major 3x3, Blinn-Phong lobes
    const float *ltc_ggx;  // the same for GGX lobes
    int grad_total;
    // per render call: sub-pixel offsets over the whole pixel (u) instead of
    // the reference's [0, 1/spp) (u / spp)
    int full_pixel_jitter;
    // per render call: the backward pass holds the BSDF sampling pdf constant
    int detached_pdf;
    // per render call: a secondary-edge sample is divided by the two lobes'
    // mixture density instead of the picked lobe's pmf * line pdf
    int edge_lobe_mis;
    // per render call: specular samples can occur (a material with roughness
    // <= 0.01 and a specular lobe, and max_bounces >= 1), so the backward pass
    // differentiates through the vertices they reach
    int specular_chains;
    // the edge trees are large: traversals run in two stages (k_edge_expand,
    // then one thread per handed-on subtree)
    int split_traversal;
};

// --- accessors -------------------------------------------------------------
DEV float3 vtx3(const float *DR_RESTRICT a, int i) {
    return f3(dr_ldg(a + 3 * i), dr_ldg(a + 3 * i + 1), dr_ldg(a + 3 * i + 2));
}
DEV DevShape shape_of(const DevScene &s, int shape) { return s.shapes[shape]; }
DEV float3 shape_vertex(const DevScene &s, int shape, int local_v) {
    return vtx3(s.vtx, s.shapes[shape].vtx_off + local_v);
}
DEV int4 tri_vids(const DevScene &s, int tri) { return s.tri[tri]; }
DEV float3 face_normal(const DevScene &s, int shape, int local_tri) {
    int4 t = s.tri[s.shapes[shape].tri_off + local_tri];
    float3 a = vtx3(s.vtx, t.x), b = vtx3(s.vtx, t.y), c = vtx3(s.vtx, t.z);
    return normalize(cross(b - a, c - a));
}

// pbrt Distribution1D::sample_discrete (distribution.h:56-63) over a cdf of
// count + 1 entries: upper_bound, then clamp to [0, count - 1].
DEV int sample_discrete(const float *cdf, const float *func, float func_int, int count, float u, float *pmf) {
    int lo = 0, hi = count + 1;  // first index with cdf[i] > u
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (dr_ldg(cdf + mid) > u) hi = mid;
        else lo = mid + 1;
    }
    int off = lo - 1;
    off = off <= 0 ? 0 : (off >= count - 1 ? count - 1 : off);
    if (pmf) *pmf = dr_ldg(func + off) / (func_int * count);
    return off;
}
