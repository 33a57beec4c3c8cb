// Host-side scene preprocessing (plain C++): restates Scene::Scene
// (scene.cpp:19-136) and build_double_edge_tree (edge_tree.cpp:263-316):
// light samplers, the unique edge list in (shape, v0, v1) order, the
// primary-edge sampler over camera silhouettes clipped to the screen, and the
// two median-split edge trees.  Used by the library (dr_api.cu) and by the
// CPU build of the kernel logic in the tests.
#pragma once

#include <algorithm>
#include <atomic>
#include <cmath>
#include <thread>
#include <cstring>
#include <map>
#include <memory>
#include <tuple>
#include <vector>

#include <stdexcept>
#include <string>

#include "../../include/delta_ray_b200.h"
#include "dr_edge_rules.h"
#include "dr_scene.cuh"

namespace drhost {

// Invalid scene input; `code` is a dr_status value.
struct SceneError : std::runtime_error {
    int code;
    explicit SceneError(const std::string &m, int c = DR_ERR_INVALID_ARGUMENT) : std::runtime_error(m), code(c) {}
};

// ---- small host vector helpers (same float expressions as the device) ----
struct V3 { float x, y, z; };
inline V3 v3(float x, float y, float z) { return V3{x, y, z}; }
inline V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
inline V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
inline V3 operator*(float s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
inline V3 operator/(V3 a, float s) { float i = 1.f / s; return a * i; }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
inline float length(V3 a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
inline V3 normalize(V3 a) { return a / length(a); }
inline float get(V3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
inline void set(V3 &a, int i, float v) { if (i == 0) a.x = v; else if (i == 1) a.y = v; else a.z = v; }
inline float luminance(V3 a) { return 0.212671f * a.x + 0.715160f * a.y + 0.072169f * a.z; }

// Total order of floats (-0 before +0), the order of the GPU build's radix
// sort keys and atomic min / max: boxes and splits built with it do not
// depend on the order in which values are combined.
inline float tmin(float a, float b) { return edge_ord_key(b) < edge_ord_key(a) ? b : a; }
inline float tmax(float a, float b) { return edge_ord_key(b) > edge_ord_key(a) ? b : a; }

struct HAABB {
    V3 lo{INFINITY, INFINITY, INFINITY}, hi{-INFINITY, -INFINITY, -INFINITY};
    // std::min / std::max, as the reference
    void add(V3 p) {
        lo = v3(std::min(lo.x, p.x), std::min(lo.y, p.y), std::min(lo.z, p.z));
        hi = v3(std::max(hi.x, p.x), std::max(hi.y, p.y), std::max(hi.z, p.z));
    }
    void add(const HAABB &b) { add(b.lo); add(b.hi); }
    // in the total order (the product's split rule for large trees)
    void add_t(V3 p) {
        lo = v3(tmin(lo.x, p.x), tmin(lo.y, p.y), tmin(lo.z, p.z));
        hi = v3(tmax(hi.x, p.x), tmax(hi.y, p.y), tmax(hi.z, p.z));
    }
    void add_t(const HAABB &b) { add_t(b.lo); add_t(b.hi); }
};

struct HCam {
    float c2w[16], w2c[16];
    float fov, aspect, clip_near;
    bool fisheye;
};

V3 xfm_point(const float *M, V3 p) {
    float t0 = M[0] * p.x + M[1] * p.y + M[2] * p.z + M[3];
    float t1 = M[4] * p.x + M[5] * p.y + M[6] * p.z + M[7];
    float t2 = M[8] * p.x + M[9] * p.y + M[10] * p.z + M[11];
    float t3 = M[12] * p.x + M[13] * p.y + M[14] * p.z + M[15];
    float inv_w = 1.f / t3;
    return v3(t0, t1, t2) * inv_w;
}

struct V2 { float x, y; };

V2 project_local(const HCam &c, V3 l) {
    if (c.fisheye) {
        V3 d = normalize(l);
        float phi = dr_atan2f(d.y, d.x), theta = dr_acosf(d.z), r = theta * 2.f / DR_PI;
        return V2{0.5f * (-r * dr_cosf(phi) + 1.f), 0.5f * (-r * dr_sinf(phi) + 1.f)};
    }
    return V2{(-l.x / (l.z * c.fov) + 1.f) * 0.5f, (-l.y / (l.z * c.fov * c.aspect) + 1.f) * 0.5f};
}

// camera.h:216-242
bool project(const HCam &c, V3 p0, V3 p1, V2 *s0, V2 *s1) {
    V3 a = xfm_point(c.w2c, p0), b = xfm_point(c.w2c, p1);
    if (a.z < c.clip_near && b.z < c.clip_near) return false;
    if (a.z < c.clip_near) {
        V3 dir = a - b;
        float t = -(b.z - c.clip_near) / dir.z;
        a = b + t * dir;
    } else if (b.z < c.clip_near) {
        V3 dir = b - a;
        float t = -(a.z - c.clip_near) / dir.z;
        b = a + t * dir;
    }
    *s0 = project_local(c, a);
    *s1 = project_local(c, b);
    return true;
}

// Cohen-Sutherland clip to [0,1]^2 (line_clip.h:13-102)
bool clip_line(V2 a, V2 b, V2 *oa, V2 *ob) {
    auto code = [](V2 v) {
        int c = 0;
        if (v.x < 0.f) c |= 1; else if (v.x > 1.f) c |= 2;
        if (v.y < 0.f) c |= 4; else if (v.y > 1.f) c |= 8;
        return c;
    };
    int c0 = code(a), c1 = code(b);
    for (int guard = 0; guard < 64; guard++) {
        if (!(c0 | c1)) { *oa = a; *ob = b; return true; }
        if (c0 & c1) return false;
        int out = c0 ? c0 : c1;
        V2 v{0.f, 0.f};
        if (out & 8) { v.x = a.x + (b.x - a.x) * (1.f - a.y) / (b.y - a.y); v.y = 1.f; }
        else if (out & 4) { v.x = a.x + (b.x - a.x) * (0.f - a.y) / (b.y - a.y); v.y = 0.f; }
        else if (out & 2) { v.y = a.y + (b.y - a.y) * (1.f - a.x) / (b.x - a.x); v.x = 1.f; }
        else { v.y = a.y + (b.y - a.y) * (0.f - a.x) / (b.x - a.x); v.x = 0.f; }
        if (out == c0) { a = v; c0 = code(a); } else { b = v; c1 = code(b); }
    }
    return false;
}

struct HShape {
    std::vector<float> v, n, uv;
    std::vector<int> idx;
    int nv = 0, nt = 0, mat = 0, light = -1;
    V3 vtx(int i) const { return v3(v[3 * i], v[3 * i + 1], v[3 * i + 2]); }
    V3 nrm(int i) const { return v3(n[3 * i], n[3 * i + 1], n[3 * i + 2]); }
    V3 face_normal(int t) const {
        V3 a = vtx(idx[3 * t]), b = vtx(idx[3 * t + 1]), c = vtx(idx[3 * t + 2]);
        return normalize(cross(b - a, c - a));
    }
};

// pbrt Distribution1D (distribution.h:7-36)
struct HDist {
    std::vector<float> func, cdf;
    float func_int = 0.f;
    void build(const std::vector<float> &f) {
        int n = (int)f.size();
        func = f;
        cdf.assign(n + 1, 0.f);
        for (int i = 1; i <= n; i++) cdf[i] = cdf[i - 1] + func[i - 1] / n;
        func_int = cdf[n];
        for (int i = 1; i <= n; i++) cdf[i] = func_int == 0.f ? float(i) / float(n) : cdf[i] / func_int;
    }
};

struct PrimInfo {
    int prim;
    V3 n0, n1, sc, dc;
    HAABB sb, db;
};

struct BuildNode {
    HAABB sb;
    V3 axis;
    float angle;
    int first = 0, n = 0;
    std::unique_ptr<BuildNode> c[2];
};

struct HostScene;

// The edge trees' median split (edge_tree.cpp:49-173).  Trees of at most
// DR_TREE_EXACT_MAX_EDGES edges follow the reference exactly: std::nth_element
// with the same comparator (equal centroids resolve as in the reference),
// float normal sums in range order, std::min / std::max boxes.  Larger trees
// follow the product's rule (PRODUCT), which the GPU build (dr_scene_build.cu)
// reproduces bit for bit:
//  - a node's range is ordered by a stable sort on the split coordinate's
//    total-order key (edge_ord_key) and split at its middle (the same two
//    halves as nth_element except where edges share the median coordinate);
//  - the cone axis's normal sum is exact: fixed point (edge_fixed), converted
//    to float once;
//  - boxes take total-order minima and maxima (-0 below +0).
// A leaf covers pi[start, end): leaves in depth-first order cover pi in
// order, so the edges are laid out as pi once the tree is built.  The two
// halves of a large node are built on two threads (disjoint ranges of pi; the
// result is the serial one).
template <bool DIR, bool PRODUCT>
std::unique_ptr<BuildNode> build_node(std::vector<PrimInfo> &pi, int start, int end, std::atomic<int> *total,
                                      int depth) {
    auto node = std::make_unique<BuildNode>();
    total->fetch_add(1, std::memory_order_relaxed);
    HAABB sb;
    for (int i = start; i < end; i++) {
        if (PRODUCT) sb.add_t(pi[i].sb);
        else sb.add(pi[i].sb);
    }
    V3 nsum = v3(0.f, 0.f, 0.f);
    if (PRODUCT) {
        long long fs[3] = {0, 0, 0};
        for (int i = start; i < end; i++) {
            fs[0] += edge_fixed(pi[i].n0.x) + edge_fixed(pi[i].n1.x);
            fs[1] += edge_fixed(pi[i].n0.y) + edge_fixed(pi[i].n1.y);
            fs[2] += edge_fixed(pi[i].n0.z) + edge_fixed(pi[i].n1.z);
        }
        nsum = v3(edge_unfixed(fs[0]), edge_unfixed(fs[1]), edge_unfixed(fs[2]));
    } else {
        for (int i = start; i < end; i++) nsum = nsum + pi[i].n0 + pi[i].n1;
    }
    V3 axis = normalize(nsum);
    float cmin = 1.f;
    for (int i = start; i < end; i++) {
        cmin = std::min(cmin, dot(pi[i].n0, axis));
        cmin = std::min(cmin, dot(pi[i].n1, axis));
    }
    node->sb = sb;
    node->axis = axis;
    node->angle = dr_acosf(cmin);
    int n = end - start;
    auto leaf = [&]() {
        node->first = start;
        node->n = n;
    };
    if (n == 1) {
        leaf();
        return node;
    }
    HAABB scb, dcb;
    for (int i = start; i < end; i++) {
        if (PRODUCT) {
            scb.add_t(pi[i].sc);
            if (DIR) dcb.add_t(pi[i].dc);
        } else {
            scb.add(pi[i].sc);
            if (DIR) dcb.add(pi[i].dc);
        }
    }
    int dim = edge_split_dim(scb.lo.x, scb.lo.y, scb.lo.z, scb.hi.x, scb.hi.y, scb.hi.z, DIR, dcb.lo.x, dcb.lo.y,
                             dcb.lo.z, dcb.hi.x, dcb.hi.y, dcb.hi.z);
    if (dim < 0) {
        leaf();
        return node;
    }
    bool spatial = dim < 3;
    int d = spatial ? dim : dim - 3;
    int mid = (start + end) / 2;
    if (PRODUCT) {
        std::stable_sort(pi.begin() + start, pi.begin() + end, [d, spatial](const PrimInfo &a, const PrimInfo &b) {
            return spatial ? edge_ord_key(get(a.sc, d)) < edge_ord_key(get(b.sc, d))
                           : edge_ord_key(get(a.dc, d)) < edge_ord_key(get(b.dc, d));
        });
    } else {
        std::nth_element(&pi[start], &pi[mid], &pi[end - 1] + 1, [d, spatial](const PrimInfo &a, const PrimInfo &b) {
            return spatial ? get(a.sc, d) < get(b.sc, d) : get(a.dc, d) < get(b.dc, d);
        });
    }
    if (n >= 16384 && depth < 4) {
        std::thread left([&]() { node->c[0] = build_node<DIR, PRODUCT>(pi, start, mid, total, depth + 1); });
        node->c[1] = build_node<DIR, PRODUCT>(pi, mid, end, total, depth + 1);
        left.join();
    } else {
        node->c[0] = build_node<DIR, PRODUCT>(pi, start, mid, total, depth + 1);
        node->c[1] = build_node<DIR, PRODUCT>(pi, mid, end, total, depth + 1);
    }
    return node;
}

struct HostScene {
    HCam cam;
    std::vector<HShape> shapes;
    std::vector<DevMaterial> mats;
    // unique edges of the meshes before the degenerate/coplanar filter, in
    // (shape, v0, v1) order; valid while the triangle indices stay the same
    std::vector<DevEdge> topo_edges;
    bool topo_valid = false;
    // some material can take a "specular" BSDF sample (roughness <= 0.01 with a
    // nonzero specular lobe, material.h:410): the backward pass does not
    // differentiate through such bounces
    bool specular_bounces = false;
    std::vector<float> texels;
    std::vector<DevLight> lights;
    std::vector<float> light_tri_cdf, light_tri_func;
    HDist light_sel;
    float total_light_intensity = 0.f;
    std::vector<DevEdge> prim_edges;
    std::vector<DevEdge> kept_edges;  // edges after dropping degenerate and flat ones
    HDist prim_dist;
    std::vector<DevEdgeNode> sil_nodes, nrm_nodes;
    std::vector<DevEdge> sil_edges, nrm_edges;
    std::vector<float> ltc, ltc_ggx;
    size_t grad_total = 0;
    // flat gradient layout (include/delta_ray_b200.h)
    std::vector<size_t> layout_mat, layout_vtx, layout_nrm, layout_light;

    V3 ev0(const DevEdge &e) const { return shapes[e.shape].vtx(e.v0); }
    V3 ev1(const DevEdge &e) const { return shapes[e.shape].vtx(e.v1); }

    V3 non_shared(const DevEdge &e, int f) const {
        const HShape &s = shapes[e.shape];
        for (int i = 0; i < 3; i++) {
            int v = s.idx[3 * f + i];
            if (v != e.v0 && v != e.v1) return s.vtx(v);
        }
        return v3(0.f, 0.f, 0.f);
    }
    // edge.h:59-79
    bool is_silhouette(V3 p, const DevEdge &e) const {
        if (shapes[e.shape].n.empty()) return true;
        if (e.f0 == -1 || e.f1 == -1) return true;
        V3 v0 = ev0(e), v1 = ev1(e), a = non_shared(e, e.f0), b = non_shared(e, e.f1);
        V3 n0 = normalize(cross(v0 - a, v1 - a)), n1 = normalize(cross(v1 - b, v0 - b));
        bool f0 = dot(p - v0, n0) > 0.f && dot(p - v1, n0) > 0.f && dot(p - a, n0) > 0.f;
        bool f1 = dot(p - v0, n1) > 0.f && dot(p - v1, n1) > 0.f && dot(p - b, n1) > 0.f;
        return (f0 && !f1) || (!f0 && f1);
    }

    int flatten(std::vector<DevEdgeNode> &nodes, const std::vector<DevEdge> &ordered, const BuildNode *b, int *off) {
        int my = (*off)++;
        DevEdgeNode &ln = nodes[my];
        ln.lo[0] = b->sb.lo.x; ln.lo[1] = b->sb.lo.y; ln.lo[2] = b->sb.lo.z;
        ln.hi[0] = b->sb.hi.x; ln.hi[1] = b->sb.hi.y; ln.hi[2] = b->sb.hi.z;
        ln.axis[0] = b->axis.x; ln.axis[1] = b->axis.y; ln.axis[2] = b->axis.z;
        ln.angle = b->angle;
        ln.pad = 0;
        if (b->n > 0) {
            ln.offset = b->first;
            ln.nprims = b->n;
            float tl = 0.f;
            for (int i = 0; i < b->n; i++) {
                const DevEdge &e = ordered[b->first + i];
                tl += length(ev1(e) - ev0(e));
            }
            ln.total_length = tl;
        } else {
            nodes[my].nprims = 0;
            flatten(nodes, ordered, b->c[0].get(), off);
            int second = flatten(nodes, ordered, b->c[1].get(), off);
            nodes[my].offset = second;
            nodes[my].total_length = nodes[my + 1].total_length + nodes[second].total_length;
        }
        return my;
    }

    template <bool DIR> void build_tree(const std::vector<DevEdge> &edges, std::vector<DevEdgeNode> &nodes,
                                        std::vector<DevEdge> &ordered) {
        nodes.clear();
        ordered.clear();
        if (edges.empty()) return;
        const bool product = edges.size() > (size_t)DR_TREE_EXACT_MAX_EDGES;
        std::vector<PrimInfo> pi(edges.size());
        HAABB world;
        for (size_t i = 0; i < edges.size(); i++) {
            HAABB b;
            if (product) {
                b.add_t(ev0(edges[i]));
                b.add_t(ev1(edges[i]));
            } else {
                b.add(ev0(edges[i]));
                b.add(ev1(edges[i]));
            }
            pi[i].prim = (int)i;
            pi[i].sb = b;
            pi[i].sc = 0.5f * b.lo + 0.5f * b.hi;
            pi[i].n0 = pi[i].n1 = v3(0.f, 0.f, 0.f);
            if (product) world.add_t(b);
            else world.add(b);
        }
        if (DIR) {
            float factor = length(world.hi - world.lo) / 8.f;
            for (size_t i = 0; i < edges.size(); i++) {
                const DevEdge &e = edges[i];
                const HShape &sh = shapes[e.shape];
                V3 sn = normalize(sh.nrm(e.v0) + sh.nrm(e.v1));
                V3 n0 = sh.face_normal(e.f0), n1 = sh.face_normal(e.f1);
                if (dot(n0, sn) < 0.f) n0 = -n0;
                if (dot(n1, sn) < 0.f) n1 = -n1;
                pi[i].n0 = n0;
                pi[i].n1 = n1;
                HAABB d;
                if (product) {
                    d.add_t(n0 * factor);
                    d.add_t(n1 * factor);
                } else {
                    d.add(n0 * factor);
                    d.add(n1 * factor);
                }
                pi[i].db = d;
                pi[i].dc = 0.5f * (d.lo + d.hi);
            }
        }
        std::atomic<int> total(0);
        auto root = product ? build_node<DIR, true>(pi, 0, (int)edges.size(), &total, 0)
                            : build_node<DIR, false>(pi, 0, (int)edges.size(), &total, 0);
        ordered.resize(edges.size());
        for (size_t i = 0; i < edges.size(); i++) ordered[i] = edges[pi[i].prim];
        nodes.resize(total.load());
        int off = 0;
        flatten(nodes, ordered, root.get(), &off);
    }

    // The primary-edge sampler of camera c (edge_tree.cpp:263-294): the kept
    // edges that are silhouettes from the camera, by clipped screen length.
    void primary_for(const HCam &c, std::vector<DevEdge> &pe, HDist &pd) const {
        pe.clear();
        std::vector<float> lens;
        V3 org = xfm_point(c.c2w, v3(0.f, 0.f, 0.f));
        for (const DevEdge &e : kept_edges) {
            V2 a, b;
            float dist = 0.f;
            if (project(c, ev0(e), ev1(e), &a, &b)) {
                V2 ca, cb;
                if (clip_line(a, b, &ca, &cb))
                    dist = std::sqrt((cb.x - ca.x) * (cb.x - ca.x) + (cb.y - ca.y) * (cb.y - ca.y));
            }
            if (!is_silhouette(org, e)) dist = 0.f;
            if (dist > 0.f) {
                pe.push_back(e);
                lens.push_back(dist);
            }
        }
        pd = HDist();
        if (!lens.empty()) pd.build(lens);
    }

    // lights (light samplers) and, unless the GPU builds them, the edges
    void preprocess(bool edges = true) {
        preprocess_lights();
        if (edges) preprocess_edges();
    }

    void preprocess_lights() {
        // lights (scene.cpp:26-52)
        std::vector<float> imp;
        total_light_intensity = 0.f;
        light_tri_cdf.clear();
        light_tri_func.clear();
        for (size_t li = 0; li < lights.size(); li++) {
            DevLight &L = lights[li];
            float lum = luminance(v3(L.I[0], L.I[1], L.I[2]));
            imp.push_back(lum);
            total_light_intensity += lum;
            const HShape &sh = shapes[L.shape];
            std::vector<float> areas;
            HAABB b;
            float asum = 0.f;
            for (int t = 0; t < sh.nt; t++) {
                V3 a = sh.vtx(sh.idx[3 * t]), bb = sh.vtx(sh.idx[3 * t + 1]), cc = sh.vtx(sh.idx[3 * t + 2]);
                float ar = 0.5f * length(cross(bb - a, cc - a));
                asum += ar;
                areas.push_back(ar);
                b.add(a);
                b.add(bb);
                b.add(cc);
            }
            HDist d;
            d.build(areas);
            L.cdf_off = (int)light_tri_cdf.size();
            L.ntri = sh.nt;
            L.func_int = d.func_int;
            L.area = asum;
            V3 c = (b.lo + b.hi) / 2.f;
            L.bc[0] = c.x; L.bc[1] = c.y; L.bc[2] = c.z;
            V3 dd = b.hi - c;
            L.br = length(dd);
            light_tri_cdf.insert(light_tri_cdf.end(), d.cdf.begin(), d.cdf.end());
            light_tri_func.insert(light_tri_func.end(), d.func.begin(), d.func.end());
            light_tri_func.push_back(0.f);  // keep func and cdf offsets aligned (ntri + 1 slots)
        }
        if (!imp.empty()) light_sel.build(imp);
    }

    void preprocess_edges() {
        // unique edges in (shape, v0, v1) order (scene.cpp:54-97); they depend
        // on the triangle indices only, so an update with new positions reuses them
        if (!topo_valid) {
            std::map<std::tuple<int, int, int>, DevEdge> emap;
            for (int si = 0; si < (int)shapes.size(); si++) {
                const HShape &sh = shapes[si];
                for (int t = 0; t < sh.nt; t++) {
                    int ind[3] = {sh.idx[3 * t], sh.idx[3 * t + 1], sh.idx[3 * t + 2]};
                    for (int k = 0; k < 3; k++) {
                        int a = ind[k], b = ind[(k + 1) % 3];
                        if (a > b) std::swap(a, b);
                        auto key = std::make_tuple(si, a, b);
                        auto it = emap.find(key);
                        if (it == emap.end()) emap[key] = DevEdge{si, a, b, t, -1};
                        else it->second.f1 = t;
                    }
                }
            }
            topo_edges.clear();
            for (auto &kv : emap) topo_edges.push_back(kv.second);
            topo_valid = true;
        }
        std::vector<DevEdge> edges;
        for (const DevEdge &e : topo_edges) {
            V3 d = ev0(e) - ev1(e);
            if (std::fabs(d.x) + std::fabs(d.y) + std::fabs(d.z) < 1e-10f) continue;
            if (e.f1 != -1) {
                float ang = std::fabs(dot(shapes[e.shape].face_normal(e.f0), shapes[e.shape].face_normal(e.f1)));
                if (ang == 1.f || ang == -1.f) continue;
            }
            edges.push_back(e);
        }
        kept_edges = edges;
        primary_for(cam, prim_edges, prim_dist);
        std::vector<DevEdge> sil, nrm;
        for (const DevEdge &e : edges) {
            if (e.f0 == -1 || e.f1 == -1 || shapes[e.shape].n.empty()) sil.push_back(e);
            else nrm.push_back(e);
        }
        build_tree<false>(sil, sil_nodes, sil_edges);
        build_tree<true>(nrm, nrm_nodes, nrm_edges);
    }
};

// Blinn-Phong LTC table used when the caller supplies none: isotropic
// identity matrices, i.e. edges are importance-sampled by the cosine lobe.
std::vector<float> default_ltc() {
    std::vector<float> t(128 * 128 * 9, 0.f);
    for (int i = 0; i < 128 * 128; i++) t[9 * i] = t[9 * i + 4] = t[9 * i + 8] = 1.f;
    return t;
}

template <class Fetch> void load_desc(HostScene &h, const dr_scene_desc *d, Fetch fetch) {
    if (!d) throw SceneError("scene descriptor is NULL");
    if (d->num_shapes < 0 || d->num_materials < 0 || d->num_lights < 0)
        throw SceneError("negative count in scene descriptor");
    h = HostScene();
    auto m16 = [&](const float *p, float *dst, const char *what) {
        auto v = fetch(p, 16, what);
        std::memcpy(dst, v.data(), 64);
    };
    m16(d->camera.cam_to_world, h.cam.c2w, "cam_to_world");
    m16(d->camera.world_to_cam, h.cam.w2c, "world_to_cam");
    h.cam.fov = d->camera.fov_factor;
    h.cam.aspect = d->camera.aspect_ratio;
    h.cam.clip_near = d->camera.clip_near;
    h.cam.fisheye = d->camera.fisheye != 0;
    size_t g = 64;
    for (int i = 0; i < d->num_materials; i++) {
        const dr_material_desc &m = d->materials[i];
        DevMaterial dm;
        std::memset(&dm, 0, sizeof(dm));
        auto channel = [&](const float *p, int w, int hh, int ch, float *cval, int *tex, int *ow, int *oh,
                           int *grad, const char *what) {
            if (w < 0 || hh < 0 || (w == 0) != (hh == 0)) throw SceneError(what);
            *grad = (int)g;
            if (w == 0) {
                auto v = fetch(p, ch, what);
                for (int c = 0; c < ch; c++) cval[c] = v[c];
                *tex = -1;
                *ow = *oh = 0;
                g += ch;
            } else {
                auto v = fetch(p, (size_t)w * hh * ch, what);
                *tex = (int)h.texels.size();
                h.texels.insert(h.texels.end(), v.begin(), v.end());
                *ow = w;
                *oh = hh;
                g += (size_t)w * hh * ch;
            }
        };
        channel(m.diffuse, m.diffuse_w, m.diffuse_h, 3, dm.kd, &dm.tex_kd, &dm.kd_w, &dm.kd_h, &dm.grad_kd, "diffuse");
        channel(m.specular, m.specular_w, m.specular_h, 3, dm.ks, &dm.tex_ks, &dm.ks_w, &dm.ks_h, &dm.grad_ks,
                "specular");
        channel(m.roughness, m.roughness_w, m.roughness_h, 1, &dm.rough, &dm.tex_r, &dm.r_w, &dm.r_h, &dm.grad_r,
                "roughness");
        auto uvs = [&](const float *p, float *dst, const char *what) {
            auto v = fetch(p, 2, what);
            dst[0] = v[0];
            dst[1] = v[1];
        };
        uvs(m.diffuse_uv_scale, dm.uv_kd, "diffuse_uv_scale");
        uvs(m.specular_uv_scale, dm.uv_ks, "specular_uv_scale");
        uvs(m.roughness_uv_scale, dm.uv_r, "roughness_uv_scale");
        dm.two_sided = m.two_sided != 0;
        if (m.microfacet != DR_MICROFACET_BLINN_PHONG && m.microfacet != DR_MICROFACET_GGX)
            throw SceneError("unknown microfacet model");
        dm.model = m.microfacet;
        {
            // can this material's BSDF sample be "specular" (material.h:410)?
            auto range = [&](int tex, int w, int hh, int ch, const float *cval, float &lo, float &hi) {
                lo = 1e30f;
                hi = -1e30f;
                size_t n = tex < 0 ? (size_t)ch : (size_t)w * hh * ch;
                const float *v = tex < 0 ? cval : h.texels.data() + tex;
                for (size_t k = 0; k < n; k++) {
                    lo = std::min(lo, v[k]);
                    hi = std::max(hi, v[k]);
                }
            };
            float rlo, rhi, slo, shi;
            range(dm.tex_r, dm.r_w, dm.r_h, 1, &dm.rough, rlo, rhi);
            range(dm.tex_ks, dm.ks_w, dm.ks_h, 3, dm.ks, slo, shi);
            if (rlo <= 0.01f && (shi > 0.f || slo < 0.f)) h.specular_bounces = true;
        }
        h.mats.push_back(dm);
        h.layout_mat.push_back((size_t)dm.grad_kd);
        h.layout_mat.push_back((size_t)dm.grad_ks);
        h.layout_mat.push_back((size_t)dm.grad_r);
    }
    for (int i = 0; i < d->num_shapes; i++) {
        const dr_shape_desc &s = d->shapes[i];
        if (s.num_vertices < 0 || s.num_triangles < 0) throw SceneError("negative mesh size");
        if (s.material_id < 0 || s.material_id >= d->num_materials)
            throw SceneError("shape material_id out of range");
        HShape hs;
        hs.nv = s.num_vertices;
        hs.nt = s.num_triangles;
        hs.mat = s.material_id;
        hs.v = fetch(s.vertices, 3 * (size_t)hs.nv, "vertices");
        hs.idx = fetch(s.indices, 3 * (size_t)hs.nt, "indices");
        for (int v : hs.idx)
            if (v < 0 || v >= hs.nv) throw SceneError("triangle index out of range");
        if (s.uvs) hs.uv = fetch(s.uvs, 2 * (size_t)hs.nv, "uvs");
        if (s.normals) hs.n = fetch(s.normals, 3 * (size_t)hs.nv, "normals");
        h.layout_vtx.push_back(g);
        g += 3 * (size_t)hs.nv;
        if (s.normals) {
            h.layout_nrm.push_back(g);
            g += 3 * (size_t)hs.nv;
        } else {
            h.layout_nrm.push_back((size_t)-1);
        }
        h.shapes.push_back(std::move(hs));
    }
    for (int i = 0; i < d->num_lights; i++) {
        const dr_light_desc &l = d->lights[i];
        if (l.shape_id < 0 || l.shape_id >= d->num_shapes)
            throw SceneError("light shape_id out of range");
        DevLight L;
        std::memset(&L, 0, sizeof(L));
        L.shape = l.shape_id;
        auto I = fetch(l.intensity, 3, "intensity");
        L.I[0] = I[0]; L.I[1] = I[1]; L.I[2] = I[2];
        L.grad = (int)g;
        h.layout_light.push_back(g);
        g += 3;
        h.shapes[L.shape].light = i;
        h.lights.push_back(L);
    }
    h.grad_total = g;
    if (g > (size_t)0x7fffffff) throw SceneError("scene too large for 32-bit gradient offsets");
    h.ltc = d->ltc_table ? fetch(d->ltc_table, 128 * 128 * 9, "ltc_table") : default_ltc();
    h.ltc_ggx = d->ltc_table_ggx ? fetch(d->ltc_table_ggx, 128 * 128 * 9, "ltc_table_ggx") : default_ltc();
}


// Global (all-shape) geometry arrays in upload order.
struct FlatScene {
    std::vector<float> vtx, nrm, uv;
    std::vector<int4> tri;
    std::vector<int> tri_local;
    std::vector<DevShape> shapes;
    bool any_n = false, any_uv = false;
    float3 lo, hi;
};

inline void flatten(const HostScene &h, FlatScene &f) {
    f = FlatScene();
    for (auto &s : h.shapes) {
        f.any_n |= !s.n.empty();
        f.any_uv |= !s.uv.empty();
    }
    HAABB bounds;
    for (int si = 0; si < (int)h.shapes.size(); si++) {
        const HShape &s = h.shapes[si];
        DevShape ds;
        ds.vtx_off = (int)(f.vtx.size() / 3);
        ds.tri_off = (int)f.tri.size();
        ds.nv = s.nv;
        ds.nt = s.nt;
        ds.mat = s.mat;
        ds.light = s.light;
        ds.has_uv = !s.uv.empty();
        ds.has_n = !s.n.empty();
        ds.grad_v = (int)h.layout_vtx[si];
        ds.grad_n = h.layout_nrm[si] == (size_t)-1 ? -1 : (int)h.layout_nrm[si];
        f.vtx.insert(f.vtx.end(), s.v.begin(), s.v.end());
        if (f.any_n) {
            if (ds.has_n) f.nrm.insert(f.nrm.end(), s.n.begin(), s.n.end());
            else f.nrm.insert(f.nrm.end(), 3 * (size_t)s.nv, 0.f);
        }
        if (f.any_uv) {
            if (ds.has_uv) f.uv.insert(f.uv.end(), s.uv.begin(), s.uv.end());
            else f.uv.insert(f.uv.end(), 2 * (size_t)s.nv, 0.f);
        }
        for (int t = 0; t < s.nt; t++) {
            int4 q;
            q.x = ds.vtx_off + s.idx[3 * t];
            q.y = ds.vtx_off + s.idx[3 * t + 1];
            q.z = ds.vtx_off + s.idx[3 * t + 2];
            q.w = si;
            f.tri.push_back(q);
            f.tri_local.push_back(t);
        }
        for (int i = 0; i < s.nv; i++) bounds.add(s.vtx(i));
        f.shapes.push_back(ds);
    }
    f.lo.x = bounds.lo.x; f.lo.y = bounds.lo.y; f.lo.z = bounds.lo.z;
    f.hi.x = bounds.hi.x; f.hi.y = bounds.hi.y; f.hi.z = bounds.hi.z;
}

// Where each array of the scene lives (device or, in tests, host memory).
struct ScenePtrs {
    const float *vtx, *nrm, *uv;
    const int4 *tri;
    const int *tri_local;
    const float4 *bvh_nodes, *bvh_tris, *bvh_wide = nullptr;
    const DevShape *shapes;
    const DevMaterial *mats;
    const float *texels;
    const DevLight *lights;
    const float *light_sel_cdf, *light_sel_func, *light_tri_cdf, *light_tri_func;
    const DevEdge *prim_edges;
    const float *prim_cdf, *prim_func;
    const DevEdgeNode *sil_nodes;
    const DevEdge *sil_edges;
    const DevEdgeNode *nrm_nodes;
    const DevEdge *nrm_edges;
    const float *ltc, *ltc_ggx;
};

inline void fill_devscene(DevScene &ds, const HostScene &h, const FlatScene &f, const ScenePtrs &p) {
    std::memset(&ds, 0, sizeof(ds));
    std::memcpy(ds.cam.c2w.m, h.cam.c2w, 64);
    std::memcpy(ds.cam.w2c.m, h.cam.w2c, 64);
    ds.cam.fov = h.cam.fov;
    ds.cam.aspect = h.cam.aspect;
    ds.cam.clip_near = h.cam.clip_near;
    ds.cam.fisheye = h.cam.fisheye;
    int n = (int)f.tri.size();
    ds.vtx = p.vtx;
    ds.nrm = f.any_n ? p.nrm : nullptr;
    ds.uv = f.any_uv ? p.uv : nullptr;
    ds.tri = p.tri;
    ds.tri_local = p.tri_local;
    ds.num_tris = n;
    ds.bvh_nodes = p.bvh_nodes;
    ds.bvh_tris = p.bvh_tris;
    ds.bvh_wide = p.bvh_wide;
    ds.bvh_root = n > 1 ? 0 : ~0;
    ds.shapes = p.shapes;
    ds.num_shapes = (int)h.shapes.size();
    ds.mats = p.mats;
    ds.num_mats = (int)h.mats.size();
    ds.texels = p.texels;
    ds.lights = p.lights;
    ds.num_lights = (int)h.lights.size();
    ds.light_sel_cdf = p.light_sel_cdf;
    ds.light_sel_func = p.light_sel_func;
    ds.light_sel_func_int = h.light_sel.func_int;
    ds.total_light_intensity = h.total_light_intensity;
    ds.light_tri_cdf = p.light_tri_cdf;
    ds.light_tri_func = p.light_tri_func;
    ds.prim_edges = p.prim_edges;
    ds.num_prim_edges = (int)h.prim_edges.size();
    ds.prim_cdf = p.prim_cdf;
    ds.prim_func = p.prim_func;
    ds.prim_func_int = h.prim_dist.func_int;
    ds.sil_nodes = p.sil_nodes;
    ds.sil_edges = p.sil_edges;
    ds.num_sil_nodes = (int)h.sil_nodes.size();
    ds.nrm_nodes = p.nrm_nodes;
    ds.nrm_edges = p.nrm_edges;
    ds.num_nrm_nodes = (int)h.nrm_nodes.size();
    ds.ltc = p.ltc;
    ds.ltc_ggx = p.ltc_ggx;
    ds.full_pixel_jitter = 0;  // set per render call
    ds.detached_pdf = 0;
    ds.edge_lobe_mis = 0;
    ds.specular_chains = 0;
    ds.split_traversal = 0;
    ds.grad_total = (int)h.grad_total;
}

}  // namespace drhost
