// Test infrastructure: the renderer's per-sample kernel logic (the
// __host__ __device__ functions of delta_ray_b200/csrc) compiled for the CPU
// with DR_HOST_BUILD, driven sequentially.  Tests compare it with the oracle
// and use it to inspect the traversal.  Never part of the product: the product
// runs this code only on the GPU.
#include <algorithm>
#include <cstring>
#include <numeric>
#include <vector>

thread_local long long g_dr_visits = 0;

// Synthetic learned proposal for the harness (hh_set_proposal): per shading
// point, 32 skewed pseudo-random slot probabilities from a hash of the point's
// sample id and bounce.
static int g_prop_seed = 0;
static float g_prop_alpha = 0.f;
// hh_set_split(1): walk each point's trees to depth 4, hand the subtrees
// there on as tasks and walk those after all points (the GPU's two-stage
// traversal of large trees)
static int g_split = 0;
// hh_set_checkpoints(k): later hh_render calls trace paths in the checkpointed
// form, segments of k bounces (0: the per-bounce records)
static int g_ckpt = 0;

#include "../../delta_ray_b200/csrc/dr_backward.cuh"
#include "../../delta_ray_b200/csrc/dr_bvh.cuh"
#include "../../delta_ray_b200/csrc/dr_host_scene.h"

namespace {

// host replica of the device LBVH build (dr_kernels.cu: dr_build_lbvh)
void build_lbvh(const float *vtx, const int4 *tri, int n, float3 lo, float3 hi, std::vector<float4> &nodes,
                std::vector<float4> &leaves) {
    BvhBuildIn in;
    in.vtx = vtx;
    in.tri = tri;
    in.n = n;
    in.lo = lo;
    float3 ext = hi - lo;
    in.inv_ext = f3(ext.x > 0.f ? 1.f / ext.x : 0.f, ext.y > 0.f ? 1.f / ext.y : 0.f, ext.z > 0.f ? 1.f / ext.z : 0.f);
    std::vector<uint32_t> keys(n);
    std::vector<int> order(n);
    for (int i = 0; i < n; i++) keys[i] = tri_morton(in, i);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return keys[a] < keys[b]; });
    std::vector<uint32_t> skeys(n);
    for (int i = 0; i < n; i++) skeys[i] = keys[order[i]];
    leaves.assign(3 * std::max(1, n), float4{});
    std::vector<Box> leaf_boxes(std::max(1, n)), node_boxes(std::max(1, n));
    for (int i = 0; i < n; i++) {
        int t = order[i];
        const int *id = &tri[t].x;
        float4 v[3];
        for (int k = 0; k < 3; k++) {
            v[k].x = vtx[3 * id[k]];
            v[k].y = vtx[3 * id[k] + 1];
            v[k].z = vtx[3 * id[k] + 2];
            v[k].w = 0.f;
        }
        v[0].w = dr_i2f(t);
        for (int k = 0; k < 3; k++) leaves[3 * i + k] = v[k];
        leaf_boxes[i] = tri_box(v[0], v[1], v[2]);
    }
    nodes.assign(4 * std::max(1, n - 1), float4{});
    if (n < 2) return;
    std::vector<int2> children(n);
    std::vector<int> pint(n, -1), pleaf(n, -1), flags(n, 0);
    for (int i = 0; i < n - 1; i++) lbvh_internal(skeys.data(), n, i, children.data(), pint.data(), pleaf.data());
    for (int i = 0; i < n; i++) {
        int p = pleaf[i];
        while (true) {
            if (flags[p]++ == 0) break;
            int2 c = children[p];
            Box b0 = c.x < 0 ? leaf_boxes[~c.x] : node_boxes[c.x];
            Box b1 = c.y < 0 ? leaf_boxes[~c.y] : node_boxes[c.y];
            node_boxes[p] = box_union(b0, b1);
            write_node(&nodes[4 * p], b0, b1, c.x, c.y);
            if (p == 0) break;
            p = pint[p];
        }
    }
}

struct HostSceneBundle {
    drhost::HostScene h;
    drhost::FlatScene f;
    std::vector<float4> nodes, leaves;
    std::vector<EdgeRec> recs;
    DevScene ds;
};

struct HostSink {
    std::vector<double> *g;
    void add(int i, float v) { (*g)[i] += v; }
};

void make_scene(const dr_scene_desc *desc, HostSceneBundle &b) {
    drhost::load_desc(b.h, desc, [](auto p, size_t n, const char *) {
        using T = typename std::remove_const<typename std::remove_pointer<decltype(p)>::type>::type;
        return std::vector<T>(p, p + n);
    });
    b.h.preprocess();
    drhost::flatten(b.h, b.f);
    build_lbvh(b.f.vtx.data(), b.f.tri.data(), (int)b.f.tri.size(), b.f.lo, b.f.hi, b.nodes, b.leaves);
    drhost::ScenePtrs p;
    p.vtx = b.f.vtx.data();
    p.nrm = b.f.nrm.data();
    p.uv = b.f.uv.data();
    p.tri = b.f.tri.data();
    p.tri_local = b.f.tri_local.data();
    p.bvh_nodes = b.nodes.data();
    p.bvh_tris = b.leaves.data();
    p.shapes = b.f.shapes.data();
    p.mats = b.h.mats.data();
    p.texels = b.h.texels.data();
    p.lights = b.h.lights.data();
    p.light_sel_cdf = b.h.light_sel.cdf.data();
    p.light_sel_func = b.h.light_sel.func.data();
    p.light_tri_cdf = b.h.light_tri_cdf.data();
    p.light_tri_func = b.h.light_tri_func.data();
    p.prim_edges = b.h.prim_edges.data();
    p.prim_cdf = b.h.prim_dist.cdf.data();
    p.prim_func = b.h.prim_dist.func.data();
    p.sil_nodes = b.h.sil_nodes.data();
    p.sil_edges = b.h.sil_edges.data();
    p.nrm_nodes = b.h.nrm_nodes.data();
    p.nrm_edges = b.h.nrm_edges.data();
    p.ltc = b.h.ltc.data();
    p.ltc_ggx = b.h.ltc_ggx.data();
    drhost::fill_devscene(b.ds, b.h, b.f, p);
    const size_t ns = b.h.sil_edges.size(), nn = b.h.nrm_edges.size();
    b.recs.resize(std::max<size_t>(1, ns + nn));
    for (size_t i = 0; i < ns; i++) b.recs[i] = edge_record(b.ds, b.h.sil_edges[i]);
    for (size_t i = 0; i < nn; i++) b.recs[ns + i] = edge_record(b.ds, b.h.nrm_edges[i]);
    b.ds.sil_rec = b.recs.data();
    b.ds.nrm_rec = b.recs.data() + ns;
}

}  // namespace

extern "C" {

// Forward (d_image == NULL) or backward render with the kernel logic on the
// CPU.  `parts` selects the backward terms: 1 path adjoint, 2 secondary
// edges, 4 primary edges.  stats: [points, items].
int hh_render(const dr_scene_desc *desc, const dr_render_desc *rd, const float *d_image, float *image, float *grad,
              int parts, long long *stats) {
    HostSceneBundle b;
    make_scene(desc, b);
    b.ds.full_pixel_jitter = (rd->flags & DR_FLAG_FULL_PIXEL_JITTER) != 0;
    b.ds.detached_pdf = (rd->flags & DR_FLAG_DETACHED_PDF) != 0;
    b.ds.edge_lobe_mis = (rd->flags & DR_FLAG_EDGE_LOBE_MIS) != 0;
    b.ds.specular_chains = b.h.specular_bounces && rd->max_bounces >= 1;
    const DevScene &s = b.ds;
    int W = rd->width, H = rd->height, spp = rd->spp, B = rd->max_bounces;
    uint64_t seed = rd->seed;
    std::vector<double> g(b.h.grad_total, 0.0);
    HostSink sink{&g};
    std::vector<PointRecord> pts;
    auto push = [&](const PointRecord &pr) { pts.push_back(pr); };
    // the kernels' two instantiations, chosen as the launchers choose them
    auto sample = [&](int x, int y, int si, float3 dc, HostSink &gs) {
        if (g_ckpt == 4)
            return s.specular_chains ? backward_pixel_sample<true, -4>(s, x, y, W, H, spp, si, B, seed, dc, gs, push)
                                     : backward_pixel_sample<false, -4>(s, x, y, W, H, spp, si, B, seed, dc, gs, push);
        if (g_ckpt == 8)
            return s.specular_chains ? backward_pixel_sample<true, -8>(s, x, y, W, H, spp, si, B, seed, dc, gs, push)
                                     : backward_pixel_sample<false, -8>(s, x, y, W, H, spp, si, B, seed, dc, gs, push);
        if (g_ckpt == 16)
            return s.specular_chains ? backward_pixel_sample<true, -16>(s, x, y, W, H, spp, si, B, seed, dc, gs, push)
                                     : backward_pixel_sample<false, -16>(s, x, y, W, H, spp, si, B, seed, dc, gs, push);
        return s.specular_chains ? backward_pixel_sample<true>(s, x, y, W, H, spp, si, B, seed, dc, gs, push)
                                 : backward_pixel_sample<false>(s, x, y, W, H, spp, si, B, seed, dc, gs, push);
    };
    auto prop = [&](const PointRecord &pt, float3 dp) {
        if (s.specular_chains) propagate_dp<true>(s, pt, W, H, spp, seed, dp, sink);
        else propagate_dp<false>(s, pt, W, H, spp, seed, dp, sink);
    };
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            float3 acc = f3(0.f);
            float3 dc = d_image ? f3(d_image[3 * (y * W + x)], d_image[3 * (y * W + x) + 1], d_image[3 * (y * W + x) + 2])
                                : f3(0.f);
            for (int si = 0; si < spp; si++) {
                if (!d_image) acc += pixel_sample(s, x, y, W, H, spp, si, B, seed);
                else if (parts & 1) acc += sample(x, y, si, dc, sink);
                else {
                    std::vector<double> tmp(g.size(), 0.0);
                    HostSink ts{&tmp};
                    acc += sample(x, y, si, dc, ts);
                }
            }
            image[3 * (y * W + x)] = acc.x;
            image[3 * (y * W + x) + 1] = acc.y;
            image[3 * (y * W + x) + 2] = acc.z;
        }
    long long nitems = 0;
    if (d_image && (parts & 2)) {
        struct Item { int pt, tree, ei, j; float w; };
        std::vector<Item> items;
        std::vector<uint16_t> q(32);
        for (int p = 0; p < (int)pts.size(); p++) {
            auto emit = [&](int tree, int ei, int j, float w, int) { items.push_back(Item{p, tree, ei, j, w}); };
            EdgeProposal pr;
            pr.q = nullptr;
            pr.alpha = g_prop_alpha;
            pr.codes = false;
            if (g_prop_seed) {
                float v[32], sum = 0.f;
                for (int k = 0; k < 32; k++) {
                    uint64_t h = (pts[p].sid + 1) * 0x9E3779B97F4A7C15ull ^ ((uint64_t)pts[p].bounce << 40) ^
                                 ((uint64_t)k << 48) ^ (uint64_t)g_prop_seed * 0xD1B54A32D192ED03ull;
                    h ^= h >> 31;
                    h *= 0xBF58476D1CE4E5B9ull;
                    h ^= h >> 29;
                    float u = (float)((h >> 40) + 1) / (float)(1ull << 24);
                    v[k] = u * u * u * u;
                    sum += v[k];
                }
                for (int k = 0; k < 32; k++) {  // to bf16 bits, round to nearest even
                    float f = v[k] / sum;
                    uint32_t b;
                    memcpy(&b, &f, 4);
                    b += 0x7FFFu + ((b >> 16) & 1u);
                    q[k] = (uint16_t)(b >> 16);
                }
                pr.q = q.data();
            }
            if (g_split) {
                std::vector<EdgeTask> tasks;
                auto defer = [&](int code, float bb, float c, float a, float l) {
                    tasks.push_back(EdgeTask{p, code, bb, c, a, l});
                };
                if (pr.q) traverse_point<true, 4>(s, pts[p], seed, emit, pr, &defer);
                else traverse_point<false, 4>(s, pts[p], seed, emit, pr, &defer);
                for (const EdgeTask &t : tasks) {
                    if (pr.q) traverse_point_task<true>(s, pts[p], seed, t, emit, pr);
                    else traverse_point_task<false>(s, pts[p], seed, t, emit, pr);
                }
            } else if (pr.q) {
                traverse_point<true>(s, pts[p], seed, emit, pr);
            } else {
                traverse_point<false>(s, pts[p], seed, emit, pr);
            }
        }
        nitems = (long long)items.size();
        std::vector<int> last(pts.size(), -1);
        std::vector<float3> last_dp(pts.size(), f3(0.f));
        for (const Item &it : items) {
            float3 dp = eval_item(s, pts[it.pt], it.tree, it.ei, it.j, it.w, spp, B, seed, sink);
            if (is_zero(dp)) continue;
            if (rd->dp_mode == DR_DP_SUM) {
                prop(pts[it.pt], dp);
            } else if (it.j > last[it.pt]) {
                last[it.pt] = it.j;
                last_dp[it.pt] = dp;
            }
        }
        if (rd->dp_mode != DR_DP_SUM)
            for (size_t p = 0; p < pts.size(); p++)
                if (last[p] >= 0) prop(pts[p], last_dp[p]);
    }
    if (d_image && (parts & 4)) {
        long long npe = rd->primary_edge_samples > 0 ? rd->primary_edge_samples : (long long)spp * W * H;
        for (long long i = 0; i < npe; i++) primary_edge_item(s, i, W, H, spp, B, seed, d_image, sink);
    }
    if (grad)
        for (size_t i = 0; i < g.size(); i++) grad[i] = (float)g[i];
    if (stats) {
        stats[0] = (long long)pts.size();
        stats[1] = nitems;
    }
    return 0;
}

// The edge-tree traversal (no evaluation) of shading points [p0, p1) of a
// backward render: the path stage runs over the whole image, then only those
// points are walked, two-stage when `split` (subtrees at depth 8 handed on and
// walked after the point, as the GPU's k_edge_expand / k_edge_tasks do).
// Every `step`-th point of the range is walked.  Returns the number of
// sampled edges; *points receives the point count.
long long hh_traverse_range(const dr_scene_desc *desc, const dr_render_desc *rd, long long p0, long long p1, int split,
                            long long *points, long long step) {
    HostSceneBundle b;
    make_scene(desc, b);
    b.ds.specular_chains = b.h.specular_bounces && rd->max_bounces >= 1;
    const DevScene &s = b.ds;
    int W = rd->width, H = rd->height, spp = rd->spp, B = rd->max_bounces;
    std::vector<double> g(b.h.grad_total, 0.0);
    HostSink sink{&g};
    std::vector<PointRecord> pts;
    auto push = [&](const PointRecord &pr) { pts.push_back(pr); };
    const float3 one = f3(1.f, 1.f, 1.f);
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++)
            for (int si = 0; si < spp; si++) {
                if (s.specular_chains) backward_pixel_sample<true>(s, x, y, W, H, spp, si, B, rd->seed, one, sink, push);
                else backward_pixel_sample<false>(s, x, y, W, H, spp, si, B, rd->seed, one, sink, push);
            }
    *points = (long long)pts.size();
    long long n = 0;
    EdgeProposal pr;
    pr.q = nullptr;
    pr.alpha = 0.f;
    pr.codes = false;
    auto emit = [&](int, int, int, float, int) { n++; };
    if (step < 1) step = 1;
    for (long long p = std::max(0ll, p0); p < std::min((long long)pts.size(), p1); p += step) {
        if (split) {
            std::vector<EdgeTask> tasks;
            auto defer = [&](int code, float bb, float c, float a, float l) {
                tasks.push_back(EdgeTask{(int)p, code, bb, c, a, l});
            };
            traverse_point<false, 8>(s, pts[p], rd->seed, emit, pr, &defer);
            for (const EdgeTask &t : tasks) traverse_point_task<false>(s, pts[p], rd->seed, t, emit, pr);
        } else {
            traverse_point<false>(s, pts[p], rd->seed, emit, pr);
        }
    }
    return n;
}

void hh_set_split(int on) { g_split = on; }
void hh_set_checkpoints(int k) { g_ckpt = k; }

// The synthetic proposal of later hh_render calls (seed 0: none).
void hh_set_proposal(int seed, float alpha) {
    g_prop_seed = seed;
    g_prop_alpha = alpha;
}

// Builds the LBVH over the scene and traces rays [n][6]; returns node visits.
long long hh_trace(const dr_scene_desc *desc, const float *rays, int n, int *out_tri, float *out_t) {
    HostSceneBundle b;
    make_scene(desc, b);
    g_dr_visits = 0;
    for (int i = 0; i < n; i++) {
        const float *r = rays + 6 * i;
        Hit h = trace_closest(b.ds, f3(r[0], r[1], r[2]), f3(r[3], r[4], r[5]), 1e-3f);
        out_tri[i] = h.tri;
        out_t[i] = h.t;
    }
    return g_dr_visits;
}

// The scene's edge data as the host builds it (what: 0 silhouette-tree nodes,
// 1 silhouette-tree edges, 2 normal-tree nodes, 3 normal-tree edges,
// 4 primary edges, 5 primary cdf, 6 primary func, 7 primary func integral):
// the bytes are copied to out (up to capacity), the element count returned.
long long hh_scene_edges(const dr_scene_desc *desc, int what, void *out, long long capacity) {
    HostSceneBundle b;
    make_scene(desc, b);
    const void *src = nullptr;
    size_t elem = 0, count = 0;
    const auto &h = b.h;
    switch (what) {
    case 0: src = h.sil_nodes.data(); elem = sizeof(DevEdgeNode); count = h.sil_nodes.size(); break;
    case 1: src = h.sil_edges.data(); elem = sizeof(DevEdge); count = h.sil_edges.size(); break;
    case 2: src = h.nrm_nodes.data(); elem = sizeof(DevEdgeNode); count = h.nrm_nodes.size(); break;
    case 3: src = h.nrm_edges.data(); elem = sizeof(DevEdge); count = h.nrm_edges.size(); break;
    case 4: src = h.prim_edges.data(); elem = sizeof(DevEdge); count = h.prim_edges.size(); break;
    case 5: src = h.prim_dist.cdf.data(); elem = 4; count = h.prim_dist.cdf.size(); break;
    case 6: src = h.prim_dist.func.data(); elem = 4; count = h.prim_dist.func.size(); break;
    case 7: src = &h.prim_dist.func_int; elem = 4; count = 1; break;
    default: return -1;
    }
    size_t bytes = std::min((size_t)capacity, elem * count);
    if (out && bytes) std::memcpy(out, src, bytes);
    return (long long)count;
}

// Closest hits of n ray pairs [n][9] (origin, two directions) through the
// paired LBVH walk (trace_closest_pair_bvh) and through two single walks:
// out [n][4] = pair hit 0, pair hit 1, single hit 0, single hit 1.
void hh_trace_pairs(const dr_scene_desc *desc, const float *rays, int n, int *out) {
    HostSceneBundle b;
    make_scene(desc, b);
    for (int i = 0; i < n; i++) {
        const float *r = rays + 9 * i;
        float3 o = f3(r[0], r[1], r[2]), d0 = f3(r[3], r[4], r[5]), d1 = f3(r[6], r[7], r[8]);
        Hit h0, h1;
        trace_closest_pair_bvh(b.ds.bvh_nodes, b.ds.bvh_tris, b.ds.bvh_root, o, d0, d1, 1e-3f, h0, h1);
        out[4 * i] = h0.tri;
        out[4 * i + 1] = h1.tri;
        out[4 * i + 2] = trace_closest_bvh(b.ds.bvh_nodes, b.ds.bvh_tris, b.ds.bvh_root, o, d0, 1e-3f).tri;
        out[4 * i + 3] = trace_closest_bvh(b.ds.bvh_nodes, b.ds.bvh_tris, b.ds.bvh_root, o, d1, 1e-3f).tri;
    }
}

// The occlusion test of the ray stage (a triangle hitting ahead of (ta, ida))
// through the binary walk and through the 4-wide walk, for rays [n][6] with
// their ta[n], ida[n]: out [n][2].
void hh_trace_before(const dr_scene_desc *desc, const float *rays, const float *ta, const int *ida, int n, int *out) {
    HostSceneBundle b;
    make_scene(desc, b);
    const int ni = b.ds.num_tris - 1;
    std::vector<float4> wide((size_t)DR_WIDE_F4 * std::max(ni, 1));
    for (int p = 0; p < ni; p++) widen_node(b.ds.bvh_nodes, p, wide.data() + (size_t)DR_WIDE_F4 * p);
    for (int i = 0; i < n; i++) {
        const float *r = rays + 6 * i;
        const float3 o = f3(r[0], r[1], r[2]), d = f3(r[3], r[4], r[5]);
        out[2 * i] = trace_before_bvh(b.ds.bvh_nodes, b.ds.bvh_tris, b.ds.bvh_root, o, d, 1e-3f, ta[i], ida[i]);
        out[2 * i + 1] = trace_before_wide(wide.data(), b.ds.bvh_tris, b.ds.bvh_root, o, d, 1e-3f, ta[i], ida[i]);
    }
}

// The reproducible transcendental functions (dr_math.h) on n inputs.
// The silhouette test of edge-tree nodes, filtered and unfiltered, for n
// (node, point) pairs: node k from lo[3k..], hi[3k..], axis[3k..], angle[k];
// point p[3k..].  out[2k] filtered, out[2k + 1] float evaluation alone.
void hh_silhouette(const float *lo, const float *hi, const float *axis, const float *angle, const float *p,
                   long long n, int *out) {
    for (long long k = 0; k < n; k++) {
        DevEdgeNode nd{};
        for (int a = 0; a < 3; a++) {
            nd.lo[a] = lo[3 * k + a];
            nd.hi[a] = hi[3 * k + a];
            nd.axis[a] = axis[3 * k + a];
        }
        nd.angle = angle[k];
        float3 q = f3(p[3 * k], p[3 * k + 1], p[3 * k + 2]);
        out[2 * k] = contains_silhouette(nd, q);
        out[2 * k + 1] = contains_silhouette_exact(nd, q);
    }
}

void hh_math(int fn, const float *x, const float *y, float *out, long long n) {
    for (long long i = 0; i < n; i++) out[i] = dr_math_eval(fn, x[i], y ? y[i] : 0.f);
}

}  // extern "C"
