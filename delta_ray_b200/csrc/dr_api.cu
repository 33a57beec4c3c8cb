// Host side of the C ABI (include/delta_ray_b200.h): scene preprocessing,
// uploads, the device LBVH build and the render entry points.
//
// Scene preprocessing restates Scene::Scene (scene.cpp:19-136) and
// build_double_edge_tree (edge_tree.cpp:263-316): light samplers, the unique
// edge list in (shape, v0, v1) order, the primary-edge sampler over camera
// silhouettes clipped to the screen, and the two median-split edge trees.  It
// runs once per scene (the reference reruns it twice per optimisation step).
#include "../../include/delta_ray_b200.h"
#include "dr_host_scene.h"
#include "dr_kernels.h"
#include "dr_mlp.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <atomic>
#include <cstring>
#include <map>
#include <memory>
#include <chrono>
#include <mutex>
#include <random>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

namespace {

thread_local std::string g_last_error;

struct DrError : std::runtime_error {
    dr_status code;
    DrError(dr_status c, const std::string &m) : std::runtime_error(m), code(c) {}
};

void check_cuda(cudaError_t e, const char *what) {
    if (e != cudaSuccess) {
        dr_status c = e == cudaErrorMemoryAllocation ? DR_ERR_OUT_OF_MEMORY : DR_ERR_CUDA;
        throw DrError(c, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    DevBuf() {}
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    void reserve(size_t b) {
        if (b <= bytes && p) return;
        release();
        if (b == 0) b = 16;
        check_cuda(cudaMalloc(&p, b), "cudaMalloc");
        bytes = b;
    }
    template <typename T> void upload(const std::vector<T> &v) {
        reserve(sizeof(T) * v.size());
        if (!v.empty()) check_cuda(cudaMemcpy(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice), "upload");
    }
    template <typename T> T *as() const { return (T *)p; }
};

// Copies count elements from a host or device pointer (unified addressing).
template <typename T> std::vector<T> fetch(const T *src, size_t count, const char *what) {
    std::vector<T> v(count);
    if (count == 0) return v;
    if (!src) throw DrError(DR_ERR_INVALID_ARGUMENT, std::string(what) + " is NULL");
    check_cuda(cudaMemcpy(v.data(), src, sizeof(T) * count, cudaMemcpyDefault), what);
    return v;
}

// Backward work queues: shading points, sampled edges and their adjoints, tens
// of bytes per pixel sample and per edge sample.  A destroyed scene hands its
// queues to a one-slot cache per device and the next scene on that device
// takes them from there, so a loop that builds a new scene every step (as the
// reference's RenderFunction does) allocates them once.  Only idle queues are
// cached; `idle` orders their reuse after the last kernels that touched them.
// What a backward call leaves for the next one on the same queues about its
// edge stage: edges per shading point, and, when it streamed, the edges of
// each of kItemBuckets equal ranges of its points.
constexpr int kItemBuckets = 1024;
struct EdgeStats {
    double items_per_point = 0;  // 0: no call yet
    std::vector<unsigned long long> buckets;  // empty: the last call did not stream
    long long bucket_points = 0;              // the points the buckets cover
    DevBuf dev;                               // the reduction's output
};

struct BackwardQueues {
    DevBuf pt, items, item_w, item_dp, pt_last, pt_items, counts, survivors, hits, side_rad, tasks, tasks2;
    DevBuf walk_ctx, leafq;  // the level walk of the subtrees
    DevBuf line_ctx;         // the points' line-sample setups
    long long cap_items = 0;     // grown on overflow, kept with the buffers
    double points_per_sample = 1;  // shading points per pixel sample the last overflow asked for
    EdgeStats stats;
    cudaEvent_t idle = nullptr;
    ~BackwardQueues() {
        if (idle) cudaEventDestroy(idle);
    }
};

// The caches are never destroyed: freeing device memory during static
// destruction would race the CUDA runtime's own teardown.
std::mutex &cache_mutex() {
    static std::mutex *m = new std::mutex();
    return *m;
}
std::map<int, std::unique_ptr<BackwardQueues>> &queue_cache() {
    static auto *c = new std::map<int, std::unique_ptr<BackwardQueues>>();
    return *c;
}

std::unique_ptr<BackwardQueues> take_queues(int device, cudaStream_t st) {
    std::unique_ptr<BackwardQueues> q;
    {
        std::lock_guard<std::mutex> lk(cache_mutex());
        auto it = queue_cache().find(device);
        if (it != queue_cache().end()) q = std::move(it->second);
    }
    if (!q) return std::unique_ptr<BackwardQueues>(new BackwardQueues());
    if (q->idle) check_cuda(cudaStreamWaitEvent(st, q->idle, 0), "cudaStreamWaitEvent");
    return q;
}

void give_back_queues(int device, std::unique_ptr<BackwardQueues> q) {
    if (!q) return;
    std::lock_guard<std::mutex> lk(cache_mutex());
    auto &slot = queue_cache()[device];
    // keep the larger set; the other one is freed here
    if (!slot || slot->cap_items < q->cap_items) slot = std::move(q);
}

// Device copies of LTC tables, one per device and lobe (Blinn-Phong, GGX),
// shared by the scenes that use the same table.
struct LtcCache {
    std::vector<float> host;
    std::shared_ptr<DevBuf> dev;
};
std::map<std::pair<int, int>, LtcCache> &ltc_cache() {
    static auto *c = new std::map<std::pair<int, int>, LtcCache>();
    return *c;
}

// slot: 0 Blinn-Phong table, 1 GGX table
std::shared_ptr<DevBuf> device_ltc(int device, int slot, const std::vector<float> &table) {
    std::lock_guard<std::mutex> lk(cache_mutex());
    LtcCache &c = ltc_cache()[std::make_pair(device, slot)];
    if (c.dev && c.host == table) return c.dev;
    std::shared_ptr<DevBuf> d(new DevBuf());
    d->upload(table);
    c.host = table;
    c.dev = d;
    return d;
}

}  // namespace

using namespace drhost;

// The learned edge proposal of a scene: network parameters with their Adam
// moments, and the per-call buffers (features, slot probabilities, training
// rows and targets).
struct ProposalState {
    int train = 1;
    float alpha = 0.5f, lr = 1e-3f;
    long long train_points = 32768;
    long long steps = 0;
    float last_loss = 0.f;
    DevBuf params, m, v, grads, img, loss, total, status;
    DevBuf x, xt, q, targets;
};

struct dr_scene {
    int device = 0;
    HostScene h;
    // the scene's arrays (geometry, materials, lights, samplers, edge trees,
    // LBVH nodes) share one allocation; bvh_scratch keeps the LBVH topology
    // that an update refits
    DevBuf arena, bvh_scratch;
    std::shared_ptr<DevBuf> ltc, ltc_ggx;
    std::unique_ptr<BackwardQueues> queues;  // taken at the first backward call
    std::unique_ptr<ProposalState> proposal;  // set by dr_scene_set_proposal
    DevBuf view_grad, view_prim_edges, view_prim_cdf, view_prim_func;  // dr_render_backward_views
    std::vector<std::unique_ptr<DevBuf>> batch_prim;  // per view of a batched call: primary edges, cdf, func
    DevBuf view_table;                                 // its ViewParams
    float3 lo, hi;                            // scene bounds
    DevScene ds;
    StageTimer timer;
    bool timer_ready = false;
    std::vector<std::pair<std::string, float>> timings;
    long long last_points = 0, last_items = 0;
    // work counts of the last backward call: points, items, line samples kept
    // for rays, samples kept for shading, handed-on subtrees, items of the
    // first traversal stage, edge-tree nodes visited by the point walks and by
    // the subtree walks
    long long last_work[10] = {};
    int num_vertices = 0, num_tris = 0, num_sms = 148;
    int bvh_built_tris = 0;  // triangle count of the LBVH topology kept in bvh_scratch
    // scenes of more than kGpuEdgeTris triangles build their edges, edge trees
    // and primary-edge sampler on the GPU (dr_scene_build.cu): the unique
    // edges (kept while the triangle indices stay the same), the working
    // lists and scratch, and the arena of the results
    bool gpu_edges = false;
    DevBuf edge_topo, edge_lists, edge_scratch, edge_arena;
    DevBuf edge_recs;  // silhouette-test records of both trees' edges
    size_t num_sil_edges = 0, num_nrm_edges = 0;
    int topo_count = 0;
    bool topo_dev_valid = false;
    const DevEdge *kept_dev = nullptr;
    int num_kept = 0;
    float edge_build_ms = 0.f;  // host wall time of the last edge build (tooling)
    ~dr_scene() {
        if (timer_ready)
            for (int i = 0; i <= StageTimer::kMax; i++) cudaEventDestroy(timer.ev[i]);
        give_back_queues(device, std::move(queues));
    }
    int last_launches = 0;
    dr_tuning tune{64, 3, 0, 0, 0};  // dr_scene_set_tuning
};

namespace {

// Host-side layout of the scene arena: each array at a 256-byte aligned
// offset.  Arrays with a host source are packed into a pinned staging buffer
// and reach the device in one copy.
struct ArenaLayout {
    struct Part {
        const void *src;
        size_t bytes, off;
    };
    std::vector<Part> parts;
    size_t total = 0;
    template <typename T> size_t add(const std::vector<T> &v) { return space(sizeof(T) * v.size(), v.data()); }
    size_t space(size_t bytes, const void *src = nullptr) {
        size_t off = total;
        parts.push_back({src, bytes, off});
        total += (std::max<size_t>(bytes, 16) + 255) & ~size_t(255);
        return off;
    }
};

// Pinned staging buffer of the arena uploads, one per process, grown on demand.
struct Staging {
    std::mutex m;
    void *p = nullptr;
    size_t bytes = 0;
};
Staging &staging() {
    static Staging s;
    return s;
}

void upload_arena(DevBuf &arena, const ArenaLayout &lay, cudaStream_t st) {
    arena.reserve(lay.total);
    Staging &sg = staging();
    std::lock_guard<std::mutex> lk(sg.m);
    if (sg.bytes < lay.total) {
        if (sg.p) cudaFreeHost(sg.p);
        sg.p = nullptr;
        sg.bytes = 0;
        check_cuda(cudaMallocHost(&sg.p, lay.total), "cudaMallocHost");
        sg.bytes = lay.total;
    }
    size_t end = 0;  // bytes of the arena that carry host data
    for (const auto &pt : lay.parts)
        if (pt.src && pt.bytes) {
            memcpy((char *)sg.p + pt.off, pt.src, pt.bytes);
            end = std::max(end, pt.off + pt.bytes);
        }
    if (end) check_cuda(cudaMemcpyAsync(arena.p, sg.p, end, cudaMemcpyHostToDevice, st), "scene upload");
    // the staging buffer is reused by the next upload
    check_cuda(cudaStreamSynchronize(st), "scene upload");
}

void build_edges_gpu(dr_scene *sc, cudaStream_t st);
void build_edge_records(dr_scene *sc, cudaStream_t st);

void upload_scene(dr_scene *sc, cudaStream_t st, bool refit = false) {
    HostScene &h = sc->h;
    check_cuda(cudaSetDevice(sc->device), "cudaSetDevice");
    FlatScene f;
    flatten(h, f);
    sc->num_vertices = (int)(f.vtx.size() / 3);
    sc->lo = f.lo;
    sc->hi = f.hi;
    sc->num_tris = (int)f.tri.size();
    const int n = sc->num_tris;
    ArenaLayout lay;
    const size_t o_vtx = lay.add(f.vtx), o_nrm = lay.add(f.nrm), o_uv = lay.add(f.uv), o_tri = lay.add(f.tri),
                 o_tri_local = lay.add(f.tri_local), o_shapes = lay.add(f.shapes), o_mats = lay.add(h.mats),
                 o_texels = lay.add(h.texels), o_lights = lay.add(h.lights),
                 o_light_sel_cdf = lay.add(h.light_sel.cdf), o_light_sel_func = lay.add(h.light_sel.func),
                 o_light_tri_cdf = lay.add(h.light_tri_cdf), o_light_tri_func = lay.add(h.light_tri_func),
                 o_prim_edges = lay.add(h.prim_edges), o_prim_cdf = lay.add(h.prim_dist.cdf),
                 o_prim_func = lay.add(h.prim_dist.func), o_sil_nodes = lay.add(h.sil_nodes),
                 o_sil_edges = lay.add(h.sil_edges), o_nrm_nodes = lay.add(h.nrm_nodes),
                 o_nrm_edges = lay.add(h.nrm_edges);
    // LBVH nodes and leaves: written by the build / refit kernels, except for
    // scenes traced without the tree, whose leaves (triangle order) come from here
    std::vector<float4> leaves;
    const bool linear = n > 0 && n <= DR_LINEAR_TRIS;
    if (linear) {
        leaves.resize(3 * (size_t)n);
        for (int t = 0; t < n; t++) {
            const int4 id = f.tri[t];
            const int v[3] = {id.x, id.y, id.z};
            for (int k = 0; k < 3; k++) {
                float4 &q = leaves[3 * t + k];
                q.x = f.vtx[3 * v[k]];
                q.y = f.vtx[3 * v[k] + 1];
                q.z = f.vtx[3 * v[k] + 2];
                q.w = k == 0 ? dr_i2f(t) : 0.f;
            }
        }
    }
    const size_t o_bvh_nodes = lay.space(sizeof(float4) * 4 * (size_t)std::max(1, n - 1));
    const size_t o_bvh_tris = linear ? lay.add(leaves) : lay.space(sizeof(float4) * 3 * (size_t)std::max(1, n));
    const size_t o_bvh_wide = lay.space(sizeof(float4) * DR_WIDE_F4 * (size_t)(linear ? 1 : std::max(1, n - 1)));
    upload_arena(sc->arena, lay, st);
    char *base = (char *)sc->arena.p;
    sc->ltc = device_ltc(sc->device, 0, h.ltc);
    sc->ltc_ggx = device_ltc(sc->device, 1, h.ltc_ggx);
    float *vtx = (float *)(base + o_vtx);
    int4 *tri = (int4 *)(base + o_tri);
    float4 *bvh_nodes = (float4 *)(base + o_bvh_nodes), *bvh_tris = (float4 *)(base + o_bvh_tris);
    // device LBVH
    if (n > 0 && !linear) {
        // the build's working arrays stay with the scene: an update with new
        // vertex positions refits the same tree (closest hits do not depend on
        // the tree's shape, ties going to the lower triangle id)
        size_t sb = dr_lbvh_scratch_bytes(n);
        if (refit && sc->bvh_built_tris == n && sc->bvh_scratch.bytes >= sb) {
            check_cuda(dr_refit_lbvh(vtx, tri, n, bvh_nodes, bvh_tris, sc->bvh_scratch.p, sc->bvh_scratch.bytes, st,
                                     &sc->last_launches),
                       "LBVH refit");
        } else {
            sc->bvh_scratch.reserve(sb);
            check_cuda(dr_build_lbvh(vtx, tri, n, f.lo, f.hi, bvh_nodes, bvh_tris, sc->bvh_scratch.p,
                                     sc->bvh_scratch.bytes, st, &sc->last_launches),
                       "LBVH build");
            sc->bvh_built_tris = n;
        }
        check_cuda(dr_widen_lbvh(bvh_nodes, n, (float4 *)(base + o_bvh_wide), st, &sc->last_launches), "LBVH widen");
        check_cuda(cudaStreamSynchronize(st), "LBVH build");
    }
    ScenePtrs ptr;
    ptr.vtx = vtx;
    ptr.nrm = (float *)(base + o_nrm);
    ptr.uv = (float *)(base + o_uv);
    ptr.tri = tri;
    ptr.tri_local = (int *)(base + o_tri_local);
    ptr.bvh_nodes = bvh_nodes;
    ptr.bvh_tris = bvh_tris;
    ptr.bvh_wide = n > 1 && !linear ? (const float4 *)(base + o_bvh_wide) : nullptr;
    ptr.shapes = (DevShape *)(base + o_shapes);
    ptr.mats = (DevMaterial *)(base + o_mats);
    ptr.texels = (float *)(base + o_texels);
    ptr.lights = (DevLight *)(base + o_lights);
    ptr.light_sel_cdf = (float *)(base + o_light_sel_cdf);
    ptr.light_sel_func = (float *)(base + o_light_sel_func);
    ptr.light_tri_cdf = (float *)(base + o_light_tri_cdf);
    ptr.light_tri_func = (float *)(base + o_light_tri_func);
    ptr.prim_edges = (DevEdge *)(base + o_prim_edges);
    ptr.prim_cdf = (float *)(base + o_prim_cdf);
    ptr.prim_func = (float *)(base + o_prim_func);
    ptr.sil_nodes = (DevEdgeNode *)(base + o_sil_nodes);
    ptr.sil_edges = (DevEdge *)(base + o_sil_edges);
    ptr.nrm_nodes = (DevEdgeNode *)(base + o_nrm_nodes);
    ptr.nrm_edges = (DevEdge *)(base + o_nrm_edges);
    ptr.ltc = sc->ltc->as<float>();
    ptr.ltc_ggx = sc->ltc_ggx->as<float>();
    fill_devscene(sc->ds, h, f, ptr);
    sc->num_sil_edges = h.sil_edges.size();
    sc->num_nrm_edges = h.nrm_edges.size();
    if (sc->gpu_edges) build_edges_gpu(sc, st);
    build_edge_records(sc, st);
}

// The silhouette-test records of both trees' edges (after every build).
void build_edge_records(dr_scene *sc, cudaStream_t st) {
    const size_t ns = sc->num_sil_edges, nn = sc->num_nrm_edges;
    sc->edge_recs.reserve(sizeof(EdgeRec) * std::max<size_t>(1, ns + nn));
    EdgeRec *r = sc->edge_recs.as<EdgeRec>();
    check_cuda(dr_launch_edge_records(sc->ds, sc->ds.sil_edges, (int)ns, r, st), "edge records");
    check_cuda(dr_launch_edge_records(sc->ds, sc->ds.nrm_edges, (int)nn, r + ns, st), "edge records");
    check_cuda(cudaStreamSynchronize(st), "edge records");
    sc->last_launches += 2;
    sc->ds.sil_rec = r;
    sc->ds.nrm_rec = r + ns;
}

// Edges of a flattened tree: the last node in depth-first order is a leaf
// whose range ends at the edge count.
size_t edge_count_of(const dr_scene *scene, const DevEdgeNode *nodes, int num_nodes) {
    (void)scene;
    DevEdgeNode last;
    check_cuda(cudaMemcpy(&last, nodes + (num_nodes - 1), sizeof(last), cudaMemcpyDeviceToHost), "tree read");
    return (size_t)last.offset + (size_t)last.nprims;
}

// Scenes of more than this many triangles build their edge data on the GPU.
constexpr int kGpuEdgeTris = 8192;

// The edge data of a large scene on the GPU (dr_scene_build.cu): unique
// edges, the kept / silhouette / normal sets, both edge trees and the
// primary-edge sampler.  Trees of at most DR_TREE_EXACT_MAX_EDGES edges
// follow the reference's split rule and are built on the host from the
// GPU's edge lists (cheap at that size); larger ones on the GPU.
void build_edges_gpu(dr_scene *sc, cudaStream_t st) {
    auto t0 = std::chrono::steady_clock::now();
    HostScene &h = sc->h;
    DevScene &ds = sc->ds;
    const int T = sc->num_tris;
    sc->edge_scratch.reserve(dr_edges_scratch_bytes(T));
    if (!sc->topo_dev_valid) {
        sc->edge_topo.reserve(sizeof(DevEdge) * 3 * (size_t)std::max(1, T));
        check_cuda(dr_extract_edges(ds, sc->num_vertices, sc->edge_topo.as<DevEdge>(), &sc->topo_count,
                                    sc->edge_scratch.p, sc->edge_scratch.bytes, st, &sc->last_launches),
                   "edge extraction");
        sc->topo_dev_valid = true;
    }
    const int nt = sc->topo_count;
    sc->edge_lists.reserve(sizeof(DevEdge) * 3 * (size_t)std::max(1, nt));
    DevEdge *kept = sc->edge_lists.as<DevEdge>(), *sil = kept + nt, *nrm = sil + nt;
    int cnt[3];
    check_cuda(dr_split_edges(ds, sc->edge_topo.as<DevEdge>(), nt, kept, sil, nrm, cnt, sc->edge_scratch.p,
                              sc->edge_scratch.bytes, st, &sc->last_launches),
               "edge split");
    const int nk = cnt[0], ns = cnt[1], nn = cnt[2];
    const bool gs = ns > DR_TREE_EXACT_MAX_EDGES, gn = nn > DR_TREE_EXACT_MAX_EDGES;
    std::vector<DevEdgeNode> hs_nodes, hn_nodes;
    std::vector<DevEdge> hs_edges, hn_edges;
    auto host_tree = [&](const DevEdge *src, int n, bool dir, std::vector<DevEdgeNode> &nodes,
                         std::vector<DevEdge> &ordered) {
        std::vector<DevEdge> list(n);
        if (n)
            check_cuda(cudaMemcpy(list.data(), src, sizeof(DevEdge) * n, cudaMemcpyDeviceToHost), "edge download");
        if (dir) h.build_tree<true>(list, nodes, ordered);
        else h.build_tree<false>(list, nodes, ordered);
    };
    if (!gs) host_tree(sil, ns, false, hs_nodes, hs_edges);
    if (!gn) host_tree(nrm, nn, true, hn_nodes, hn_edges);
    // kept | silhouette edges | normal edges | silhouette nodes | normal nodes | primary edges | cdf | func
    ArenaLayout lay;
    const size_t o_kept = lay.space(sizeof(DevEdge) * (size_t)nk);
    const size_t o_se = gs ? lay.space(sizeof(DevEdge) * (size_t)ns) : lay.add(hs_edges);
    const size_t o_ne = gn ? lay.space(sizeof(DevEdge) * (size_t)nn) : lay.add(hn_edges);
    const size_t o_sn = gs ? lay.space(sizeof(DevEdgeNode) * 2 * (size_t)ns) : lay.add(hs_nodes);
    const size_t o_nn = gn ? lay.space(sizeof(DevEdgeNode) * 2 * (size_t)nn) : lay.add(hn_nodes);
    const size_t o_prim = lay.space(sizeof(DevEdge) * (size_t)nk), o_cdf = lay.space(sizeof(float) * (nk + 1)),
                 o_func = lay.space(sizeof(float) * (size_t)nk);
    upload_arena(sc->edge_arena, lay, st);
    char *b = (char *)sc->edge_arena.p;
    if (nk)
        check_cuda(cudaMemcpyAsync(b + o_kept, kept, sizeof(DevEdge) * nk, cudaMemcpyDeviceToDevice, st),
                   "kept edges");
    int n_sn = (int)hs_nodes.size(), n_nn = (int)hn_nodes.size();
    if (gs || gn) sc->edge_scratch.reserve(std::max(sc->edge_scratch.bytes, dr_tree_scratch_bytes(std::max(ns, nn))));
    if (gs)
        check_cuda(dr_build_edge_tree(ds, false, sil, ns, (DevEdgeNode *)(b + o_sn), (DevEdge *)(b + o_se), &n_sn,
                                      sc->edge_scratch.p, sc->edge_scratch.bytes, st, &sc->last_launches),
                   "silhouette edge tree");
    if (gn)
        check_cuda(dr_build_edge_tree(ds, true, nrm, nn, (DevEdgeNode *)(b + o_nn), (DevEdge *)(b + o_ne), &n_nn,
                                      sc->edge_scratch.p, sc->edge_scratch.bytes, st, &sc->last_launches),
                   "normal edge tree");
    int np = 0;
    float fi = 0.f;
    check_cuda(dr_build_primary(ds, ds.cam, (const DevEdge *)(b + o_kept), nk, (DevEdge *)(b + o_prim),
                                (float *)(b + o_cdf), (float *)(b + o_func), &np, &fi, sc->edge_scratch.p,
                                sc->edge_scratch.bytes, st, &sc->last_launches),
               "primary-edge sampler");
    sc->kept_dev = (const DevEdge *)(b + o_kept);
    sc->num_kept = nk;
    ds.prim_edges = (const DevEdge *)(b + o_prim);
    ds.num_prim_edges = np;
    ds.prim_cdf = (const float *)(b + o_cdf);
    ds.prim_func = (const float *)(b + o_func);
    ds.prim_func_int = fi;
    ds.sil_nodes = (const DevEdgeNode *)(b + o_sn);
    ds.sil_edges = (const DevEdge *)(b + o_se);
    ds.num_sil_nodes = ns ? n_sn : 0;
    ds.nrm_nodes = (const DevEdgeNode *)(b + o_nn);
    ds.nrm_edges = (const DevEdge *)(b + o_ne);
    ds.num_nrm_nodes = nn ? n_nn : 0;
    sc->num_sil_edges = (size_t)ns;
    sc->num_nrm_edges = (size_t)nn;
    sc->edge_build_ms =
        std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// Shared-memory gradient cache of the backward kernels: everything when the
// flat gradient is small, else the camera + material block and the lights.
GradCacheCfg grad_cache_cfg(const HostScene &h) {
    const int cap = 6144;  // floats (24 KB of shared memory per block)
    GradCacheCfg c;
    int total = (int)h.grad_total;
    if (total <= cap) {
        c.head = total;
        c.tail_begin = total;
        c.tail_len = 0;
        return c;
    }
    int first_vtx = h.layout_vtx.empty() ? total : (int)h.layout_vtx[0];
    c.head = std::min(first_vtx, cap / 2);
    int first_light = h.layout_light.empty() ? total : (int)h.layout_light[0];
    c.tail_begin = first_light;
    c.tail_len = std::min(total - first_light, cap / 2);
    return c;
}

void collect_timings(dr_scene *sc, cudaStream_t st) {
    sc->timings.clear();
    if (!sc->timer.on) return;
    check_cuda(cudaStreamSynchronize(st), "timing sync");
    for (int i = 0; i < sc->timer.n; i++) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, sc->timer.ev[i], sc->timer.ev[i + 1]);
        sc->timings.emplace_back(sc->timer.names[i], ms);
    }
}

// Edge trees above this many nodes are walked in two stages (k_edge_expand,
// k_edge_tasks): their points' walks are long and uneven.
constexpr int kSplitTraversalNodes = 4096;
// Queues of the two-stage walk (the first stage's subtrees, each level's nodes
// in two halves by class, the leaves): up to 128 entries per point, at most
// 4 GiB each; a node that finds no room is walked depth first by its lane.
constexpr long long kTasksPerPoint = 128, kMaxTasks = (4ll << 30) / sizeof(EdgeTask);

// The scene's device view with this call's per-render settings.
DevScene call_scene(const dr_scene *sc, const dr_render_desc *rd) {
    DevScene ds = sc->ds;
    ds.full_pixel_jitter = (rd->flags & DR_FLAG_FULL_PIXEL_JITTER) != 0;
    ds.detached_pdf = (rd->flags & DR_FLAG_DETACHED_PDF) != 0;
    ds.edge_lobe_mis = (rd->flags & DR_FLAG_EDGE_LOBE_MIS) != 0;
    ds.specular_chains = sc->h.specular_bounces && rd->max_bounces >= 1;
    ds.split_traversal = sc->ds.num_sil_nodes > kSplitTraversalNodes || sc->ds.num_nrm_nodes > kSplitTraversalNodes;
    return ds;
}

void check_render_desc(const dr_scene *sc, const dr_render_desc *rd) {
    if (!sc) throw DrError(DR_ERR_INVALID_ARGUMENT, "scene is NULL");
    if (!rd) throw DrError(DR_ERR_INVALID_ARGUMENT, "render descriptor is NULL");
    if (rd->width <= 0 || rd->height <= 0 || rd->spp <= 0 || rd->max_bounces < 0)
        throw DrError(DR_ERR_INVALID_ARGUMENT, "width, height and spp must be positive, max_bounces >= 0");
    if ((long long)rd->width * rd->height > (1ll << 28))
        throw DrError(DR_ERR_INVALID_ARGUMENT, "image too large");
    if ((long long)rd->width * rd->height * rd->spp >= (1ll << 31))
        throw DrError(DR_ERR_INVALID_ARGUMENT, "width * height * spp must be below 2^31 per call");
    for (int i = 0; i < 7; i++)
        if (rd->reserved[i] != 0) throw DrError(DR_ERR_INVALID_ARGUMENT, "reserved fields must be zero");
    if (rd->flags &
        ~(int)(DR_FLAG_FULL_PIXEL_JITTER | DR_FLAG_DETACHED_PDF | DR_FLAG_EDGE_LOBE_MIS | DR_FLAG_LEARNED_PROPOSAL))
        throw DrError(DR_ERR_INVALID_ARGUMENT, "unknown render flags");
    if (rd->max_bounces > 256) throw DrError(DR_ERR_NOT_SUPPORTED, "max_bounces above 256");
    if (sc->ds.num_lights == 0) throw DrError(DR_ERR_INVALID_ARGUMENT, "scene has no lights");
}

// Item queue limit of dr_render_backward: 8 GiB of edge items (64 bytes each:
// the item, its weight, its dp and its slot in the survivor queue of the
// evaluation wavefront).  Edge stages with more items stream.
constexpr long long kMaxQueueItems = (8ll << 30) / 64;
// the first call's probe of the edge counts (run_backward): every 32nd point,
// in calls of at least 2^20 pixel samples (about 30 probed points per bucket
// of the chunk plan at 640x480, 4 spp; the forecast's margin covers the rest)
constexpr long long kProbeStride = 32, kProbeMinSamples = 1ll << 20;
std::atomic<long long> g_item_queue_limit{0};  // dr_set_item_queue_limit (0: kMaxQueueItems)
long long max_queue_items() {
    long long l = g_item_queue_limit.load();
    return l > 0 ? l : kMaxQueueItems;
}
// the bound of one scene's calls: its tuned bound if it has one, and the
// process-wide bound, whichever is smaller
long long queue_limit(const dr_scene *scene) {
    const long long l = max_queue_items(), t = scene->tune.queue_items;
    return t > 0 && t < l ? t : l;
}

void check_backward_args(const dr_scene *scene, const dr_render_desc *rd, const float *d_image_dev,
                         const float *grad_dev) {
    check_render_desc(scene, rd);
    if (!d_image_dev || !grad_dev) throw DrError(DR_ERR_INVALID_ARGUMENT, "d_image and grad must be non-NULL");
    if (rd->dp_mode != DR_DP_REFERENCE_LAST && rd->dp_mode != DR_DP_SUM)
        throw DrError(DR_ERR_INVALID_ARGUMENT, "unknown dp_mode");
}

// Shading points a backward call starts with room for: one per pixel sample,
// twice that when specular samples can add vertices after the first.
long long initial_point_cap(const dr_scene *scene, const dr_render_desc *rd, double per_sample) {
    double samples = (double)rd->width * rd->height * rd->spp;
    double f = std::max(per_sample, (scene->h.specular_bounces && rd->max_bounces >= 2) ? 2.0 : 1.0);
    return std::max(1ll, (long long)std::ceil(samples * f));
}

// The backward pass on the queues bound in ws (counters zeroed here).
// Path adjoints and primary edges run first, with the edge traversal of all
// shading points behind them; if the sampled edges outgrow the item queue,
// `grow(n)` is asked for room for n items (it returns the capacity it bound),
// and the edge stage then streams: points in chunks whose items fit, each
// chunk traversed, evaluated and its position adjoints propagated before the
// next.  If the shading points (more than one per pixel sample after specular
// samples) outgrow their queue, `grow_points(n)` is asked for room for n and
// the front runs again (the same points: the streams are deterministic).
// Returns (shading points, edge items).
// One view's front stage in a batched multi-view backward call: its device
// view (camera, primary-edge sampler, camera-gradient offset, index), render
// settings, adjoint and image.
struct FrontCall {
    DevScene ds;
    dr_render_desc rd;
    const float *d_image;
    float *image;
};

// fronts (may be null): a batched multi-view call.  Each view's front stage
// runs in turn into the shared point queue, then one edge stage serves every
// view's points (ws.views gives each point its view's settings); the
// gradient has grad_len floats (the scene's, then one camera block per view).
template <class Grow, class GrowPoints>
std::pair<long long, long long> run_backward(dr_scene *scene, const dr_render_desc *rd, const float *d_image_dev,
                                             float *grad_dev, float *image_dev, BackwardWorkspace &ws,
                                             cudaStream_t st, StageTimer *timer, Grow grow, GrowPoints grow_points,
                                             ProposalState *prop = nullptr, const DevScene *view = nullptr,
                                             EdgeStats *stats = nullptr, const std::vector<FrontCall> *fronts = nullptr,
                                             long long grad_len = 0) {
    const DevScene ds = fronts ? (*fronts)[0].ds : view ? *view : call_scene(scene, rd);
    const GradCacheCfg cfg = grad_cache_cfg(scene->h);
    BackwardCounters c;
    auto read = [&]() {
        if (timer->failed)
            throw DrError(DR_ERR_CUDA, std::string("kernel ") + timer->failed + " failed: " +
                                           cudaGetErrorString(timer->failed_err));
        check_cuda(cudaMemcpyAsync(&c, ws.counters, sizeof(c), cudaMemcpyDeviceToHost, st), "status read");
        check_cuda(cudaStreamSynchronize(st), "backward");
        if (c.status & ~(DR_STATUS_ITEM_OVERFLOW | DR_STATUS_POINT_OVERFLOW))
            throw DrError(DR_ERR_DEVICE_STATUS, "device reported status " + std::to_string(c.status));
    };
    long long work[10] = {};
    // with the DR_DEBUG_SYNC diagnostic, a launch error names the kernel that failed
    auto check_launch = [&](cudaError_t e, const char *what) {
        if (e != cudaSuccess && timer->failed)
            throw DrError(DR_ERR_CUDA, std::string("kernel ") + timer->failed + " failed: " +
                                           cudaGetErrorString(timer->failed_err));
        check_cuda(e, what);
    };
    auto back = [&]() {
        check_launch(dr_launch_backward_back(ds, rd->width, rd->height, rd->spp, rd->max_bounces, rd->seed, grad_dev,
                                           rd->dp_mode, ws, cfg, scene->num_sms, st, &scene->last_launches, timer),
                   "backward launch");
        // the stage's work counts (the counters of the evaluation wavefront
        // and the task queue restart with every chunk)
        read();
        work[2] += (long long)c.survivors;
        work[3] += (long long)c.hits;
        work[4] += (long long)(c.tasks + c.handed_total);
        work[5] += (long long)(ds.split_traversal ? c.items_expand : c.items);
        work[8] += (long long)c.cands;
    };
    // edges per bucket of points [p0, p0 + np) from ws.pt_items
    auto read_buckets_at = [&](long long p0, long long np, std::vector<unsigned long long> &out) {
        stats->dev.reserve(sizeof(unsigned long long) * kItemBuckets);
        check_cuda(dr_launch_item_buckets(ws.pt_items + p0, np, kItemBuckets, stats->dev.as<unsigned long long>(),
                                          st),
                   "item buckets");
        scene->last_launches += 1;
        out.resize(kItemBuckets);
        check_cuda(cudaMemcpyAsync(out.data(), stats->dev.p, sizeof(unsigned long long) * kItemBuckets,
                                   cudaMemcpyDeviceToHost, st),
                   "bucket read");
        check_cuda(cudaStreamSynchronize(st), "item buckets");
    };
    auto read_buckets = [&](long long P, std::vector<unsigned long long> &out) { read_buckets_at(0, P, out); };
    // ends of chunks of points [p0, p0 + np) whose edges, by buckets `b` over
    // that range (scaled by `scale`), stay within `budget`; ascending, inside
    // (p0, p0 + np)
    auto plan_ends = [](const std::vector<unsigned long long> &b, long long p0, long long np, double budget,
                        double scale, std::vector<long long> &ends) {
        double acc = 0;
        long long last = p0;
        for (int i = 0; i < (int)b.size(); i++) {
            const long long at = p0 + (long long)i * np / (long long)b.size();
            if (acc > 0 && acc + (double)b[i] * scale > budget && at > last) {
                ends.push_back(at);
                last = at;
                acc = 0;
            }
            acc += (double)b[i] * scale;
        }
    };
    // when the last call's edges per point predict more items than the queue
    // can ever hold, the edge stage streams from the start instead of
    // traversing every point once only to find that out
    long long samples = (long long)rd->width * rd->height * rd->spp;
    if (fronts) {
        samples = 0;
        for (const FrontCall &f : *fronts) samples += (long long)f.rd.width * f.rd.height * f.rd.spp;
    }
    const bool stream_first = prop == nullptr && stats && stats->items_per_point > 0 &&
                              (double)samples * stats->items_per_point > (double)queue_limit(scene);
    // a scene's first call of many samples (no edge counts yet) first walks
    // every kProbeStride-th point only: their edge counts forecast the
    // others', and a call whose forecast overflows the queue streams from
    // that forecast instead of walking every point once to count its edges
    const bool probe = !stream_first && prop == nullptr && stats && stats->items_per_point <= 0 && ws.pt_items &&
                       samples >= kProbeMinSamples;
    for (int attempt = 0;; attempt++) {
        check_cuda(cudaMemsetAsync(ws.counters, 0, sizeof(BackwardCounters), st), "memset");
        check_cuda(cudaMemsetAsync(grad_dev, 0, sizeof(float) * (grad_len > 0 ? grad_len : scene->h.grad_total), st),
                   "memset");
        ws.pt_begin = 0;
        ws.pt_end = ws.cap_points;
        if (fronts) {
            for (size_t k = 0; k < fronts->size(); k++) {
                const FrontCall &f = (*fronts)[k];
                check_launch(dr_launch_backward_front(f.ds, f.rd.width, f.rd.height, f.rd.spp, f.rd.max_bounces,
                                                      f.rd.seed, f.d_image, grad_dev, f.image,
                                                      f.rd.primary_edge_samples, f.rd.dp_mode, ws, cfg,
                                                      scene->num_sms, st, &scene->last_launches, timer, false, k == 0),
                             "backward launch");
            }
        } else {
            check_launch(dr_launch_backward_front(ds, rd->width, rd->height, rd->spp, rd->max_bounces, rd->seed,
                                                  d_image_dev, grad_dev, image_dev, rd->primary_edge_samples,
                                                  rd->dp_mode, ws, cfg, scene->num_sms, st, &scene->last_launches,
                                                  timer, prop == nullptr && !stream_first && !probe),
                         "backward launch");
        }
        read();
        if (!(c.status & DR_STATUS_POINT_OVERFLOW)) break;
        const long long needed = (long long)c.points;
        if (attempt > 0 || grow_points(needed) < needed)
            throw DrError(DR_ERR_OUT_OF_MEMORY, std::to_string(needed) + " shading points exceed the point queue (" +
                                                    std::to_string(ws.cap_points) + ")");
    }
    const long long P = std::min((long long)c.points, ws.cap_points);
    bool probe_streams = false;
    long long probe_needed = 0;
    if (probe) {
        timer->mark(st, "host_point_count");
        check_cuda(cudaMemsetAsync(ws.pt_items, 0, sizeof(int) * (size_t)std::max(P, 1ll), st), "memset");
        ws.pt_stride = kProbeStride;
        check_launch(dr_launch_edge_traverse(ds, rd->seed, ws, scene->num_sms, st, &scene->last_launches, timer),
                     "edge traversal launch");
        read();
        ws.pt_stride = 1;
        // the items counter counts past the queue's end
        probe_needed = (long long)c.items * kProbeStride;
        probe_streams = (double)probe_needed > 0.8 * (double)queue_limit(scene);
        check_cuda(cudaMemsetAsync(&ws.counters->items, 0, 16, st), "memset");
        check_cuda(cudaMemsetAsync(&ws.counters->tasks, 0, sizeof(unsigned long long), st), "memset");
    }
    if ((fronts && !stream_first) || (probe && !probe_streams)) {
        // the views' points walked together (or every point after a probe
        // that forecast room for all of their edges)
        timer->mark(st, "host_point_count");
        check_launch(dr_launch_edge_traverse(ds, rd->seed, ws, scene->num_sms, st, &scene->last_launches, timer),
                     "edge traversal launch");
        read();
    }
    if (prop) {
        // the proposal: features and slot probabilities of every point, then
        // the traversal that draws edges with them
        ProposalState &pr = *prop;
        pr.x.reserve(sizeof(uint16_t) * 16 * (size_t)std::max(P, 1ll));
        pr.q.reserve(sizeof(uint16_t) * 32 * (size_t)std::max(P, 1ll));
        ws.proposal_q = pr.q.as<uint16_t>();
        ws.proposal_alpha = pr.alpha;
        ws.train_stride = 1;
        ws.train_n = 0;
        if (pr.train) {
            ws.train_stride = std::max(1ll, P / std::max(1ll, pr.train_points));
            ws.train_n = std::min(pr.train_points, (P + ws.train_stride - 1) / ws.train_stride);
            pr.xt.reserve(sizeof(uint16_t) * 16 * (size_t)std::max(ws.train_n, 1ll));
            pr.targets.reserve(sizeof(float) * 32 * (size_t)std::max(ws.train_n, 1ll));
            check_cuda(cudaMemsetAsync(pr.targets.p, 0, sizeof(float) * 32 * (size_t)ws.train_n, st), "memset");
            ws.train_targets = pr.targets.as<float>();
        }
        float3 ctr = (scene->lo + scene->hi) * 0.5f, ext = (scene->hi - scene->lo) * 0.5f;
        float3 ih = f3(ext.x > 0.f ? 1.f / ext.x : 0.f, ext.y > 0.f ? 1.f / ext.y : 0.f, ext.z > 0.f ? 1.f / ext.z : 0.f);
        check_cuda(cudaMemsetAsync(pr.status.p, 0, sizeof(int), st), "memset");
        timer->mark(st, "host_point_count");
        check_cuda(dr_launch_proposal_features(ds, ws, P, ctr, ih, pr.x.p, pr.train ? pr.xt.p : nullptr, st),
                   "proposal features");
        timer->mark(st, "k_proposal_features");
        check_cuda(dr_mlp_infer(pr.img.as<uint8_t>(), pr.params.as<float>(), pr.x.as<__nv_bfloat16>(), P, nullptr,
                                pr.q.as<__nv_bfloat16>(), pr.status.as<int>(), scene->num_sms, st),
                   "proposal inference");
        timer->mark(st, "k_mlp_infer");
        scene->last_launches += 2;
        check_cuda(dr_launch_edge_traverse(ds, rd->seed, ws, scene->num_sms, st, &scene->last_launches, timer),
                   "edge traversal launch");
        read();
        int mst = 0;
        check_cuda(cudaMemcpy(&mst, pr.status.p, sizeof(int), cudaMemcpyDeviceToHost), "status read");
        if (mst) throw DrError(DR_ERR_DEVICE_STATUS, "proposal network reported status " + std::to_string(mst));
    }
    long long items = 0;
    bool streamed = false;
    if (!stream_first && !probe_streams && !(c.status & DR_STATUS_ITEM_OVERFLOW)) {
        timer->mark(st, "host_queue_check");
        back();
        items = (long long)c.items;
    } else {
        // The chunks of points whose edges fit the queue.  After a full pass
        // every point's edges are counted and the streams repeat them exactly,
        // so the plan from them is exact; from the last call's buckets or its
        // edges per point it is a forecast, and a chunk that overflows is cut.
        streamed = true;
        std::vector<unsigned long long> b;
        double scale = 1, margin = 0.85;
        long long needed;
        if (probe_streams) {
            // the probe's counts, every kProbeStride-th point's
            read_buckets(P, b);
            scale = (double)kProbeStride;
            needed = probe_needed;
        } else if (!stream_first) {
            needed = (long long)c.items;
            if (ws.pt_items && stats) {
                read_buckets(P, b);
                margin = 0.97;
            }
        } else if (!stats->buckets.empty() && stats->bucket_points > 0) {
            b = stats->buckets;
            scale = (double)P / (double)stats->bucket_points;
            unsigned long long t = 0;
            for (unsigned long long x : b) t += x;
            needed = (long long)std::ceil((double)t * scale);
        } else {
            needed = (long long)std::ceil((double)P * stats->items_per_point);
        }
        long long cap = grow(needed + needed / 8 + 1);
        std::vector<long long> ends;  // chunk ends, ascending
        if (!b.empty()) {
            plan_ends(b, 0, P, margin * (double)cap, scale, ends);
        } else if (needed > cap) {
            const long long chunk = std::max(1ll, (long long)((double)P * cap / needed * 0.9));
            for (long long e = chunk; e < P; e += chunk) ends.push_back(e);
        }
        ends.push_back(P);
        size_t ci = 0;
        long long p0 = 0;
        while (p0 < P) {
            while (ends[ci] <= p0) ci++;
            const long long p1 = ends[ci];
            ws.pt_begin = p0;
            ws.pt_end = p1;
            // reset the item counter and the status word (items, status, pad)
            check_cuda(cudaMemsetAsync(&ws.counters->items, 0, 16, st), "memset");
            check_launch(dr_launch_edge_traverse(ds, rd->seed, ws, scene->num_sms, st, &scene->last_launches, timer),
                         "edge traversal launch");
            read();
            if (c.status & DR_STATUS_ITEM_OVERFLOW) {
                needed = (long long)c.items;
                cap = grow(needed + needed / 8 + 1);
                if (cap >= needed) continue;  // the same chunk again, with room for it
                if (p1 - p0 == 1)
                    throw DrError(DR_ERR_OUT_OF_MEMORY, "one shading point samples " + std::to_string(needed) +
                                                            " edges; the item queue holds " + std::to_string(cap));
                // the pass counted every point of the chunk: the chunk is cut
                // exactly from those counts, and its rest follows in pieces
                std::vector<long long> cuts;
                if (ws.pt_items && stats) {
                    std::vector<unsigned long long> cb;
                    read_buckets_at(p0, p1 - p0, cb);
                    plan_ends(cb, p0, p1 - p0, 0.97 * (double)cap, 1.0, cuts);
                }
                if (cuts.empty() || cuts.back() >= p1)
                    cuts.assign(1, p0 + std::max(1ll, (long long)((double)(p1 - p0) * cap / needed * 0.9)));
                ends.insert(ends.begin() + ci, cuts.begin(), cuts.end());
                continue;
            }
            back();
            items += (long long)c.items;
            p0 = p1;
        }
    }
    if (prop && prop->train && ws.train_n > 0) {
        // one training step on the contribution magnitudes the edges reported
        ProposalState &pr = *prop;
        timer->mark(st, "proposal_targets");
        check_cuda(dr_mlp_sum(pr.targets.as<float>(), ws.train_n * 32, pr.total.as<float>(), st), "target sum");
        check_cuda(cudaMemsetAsync(pr.grads.p, 0, sizeof(float) * kMlpParams, st), "memset");
        check_cuda(cudaMemsetAsync(pr.loss.p, 0, sizeof(float), st), "memset");
        check_cuda(dr_mlp_grad(pr.img.as<uint8_t>(), pr.params.as<float>(), pr.xt.as<__nv_bfloat16>(),
                               pr.targets.as<float>(), ws.train_n, pr.total.as<float>(), pr.grads.as<float>(),
                               pr.loss.as<float>(), pr.status.as<int>(), scene->num_sms, st),
                   "proposal gradient");
        timer->mark(st, "k_mlp_grad");
        check_cuda(dr_mlp_adam(pr.params.as<float>(), pr.grads.as<float>(), pr.m.as<float>(), pr.v.as<float>(),
                               (int)(pr.steps + 1), pr.lr, st),
                   "proposal update");
        check_cuda(dr_mlp_pack(pr.params.as<float>(), pr.img.as<uint8_t>(), st), "weight pack");
        scene->last_launches += 4;
        float loss = 0.f;
        int mst = 0;
        check_cuda(cudaMemcpyAsync(&loss, pr.loss.p, sizeof(float), cudaMemcpyDeviceToHost, st), "loss read");
        check_cuda(cudaMemcpyAsync(&mst, pr.status.p, sizeof(int), cudaMemcpyDeviceToHost, st), "status read");
        check_cuda(cudaStreamSynchronize(st), "proposal training");
        if (mst) throw DrError(DR_ERR_DEVICE_STATUS, "proposal network reported status " + std::to_string(mst));
        pr.last_loss = loss;
        pr.steps++;
    }
    check_cuda(cudaStreamSynchronize(st), "backward");
    if (stats && P > 0) {
        stats->items_per_point = (double)items / (double)P;
        // a streamed call leaves its buckets (every point's count is final now)
        if (streamed && ws.pt_items) read_buckets(P, stats->buckets);
        else stats->buckets.clear();
        stats->bucket_points = P;
    }
    work[0] = P;
    work[1] = items;
    work[6] = (long long)c.visits_walk;
    work[7] = (long long)c.visits_tasks;
    work[9] = (long long)c.spilled;
    std::memcpy(scene->last_work, work, sizeof(work));
    return {P, items};
}

template <typename F> dr_status guard(F f) {
    try {
        f();
        return DR_OK;
    } catch (const DrError &e) {
        g_last_error = e.what();
        return e.code;
    } catch (const SceneError &e) {
        g_last_error = e.what();
        return (dr_status)e.code;
    } catch (const std::exception &e) {
        g_last_error = e.what();
        return DR_ERR_INVALID_ARGUMENT;
    }
}

}  // namespace

namespace {
unsigned char *noalloc_scratch();
}  // namespace

extern "C" {

int dr_abi_version(void) { return DR_ABI_VERSION; }

dr_status dr_set_item_queue_limit(int64_t items) {
    return guard([&]() {
        if (items < 0) throw DrError(DR_ERR_INVALID_ARGUMENT, "negative item queue limit");
        g_item_queue_limit.store((long long)items);
    });
}

dr_status dr_scene_create(const dr_scene_desc *desc, int device, dr_scene **out) {
    return guard([&]() {
        if (!out) throw DrError(DR_ERR_INVALID_ARGUMENT, "out is NULL");
        *out = nullptr;
        int ndev = 0;
        check_cuda(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
        if (device < 0 || device >= ndev) throw DrError(DR_ERR_INVALID_ARGUMENT, "device index out of range");
        check_cuda(cudaSetDevice(device), "cudaSetDevice");
        std::unique_ptr<dr_scene> sc(new dr_scene());
        sc->device = device;
        sc->timer.sync = std::getenv("DR_DEBUG_SYNC") != nullptr;
        check_cuda(cudaDeviceGetAttribute(&sc->num_sms, cudaDevAttrMultiProcessorCount, device), "device query");
        load_desc(sc->h, desc, [](auto p, size_t n, const char *w) { return fetch(p, n, w); });
        long long ntri = 0;
        for (auto &sh : sc->h.shapes) ntri += sh.nt;
        sc->gpu_edges = ntri > kGpuEdgeTris;
        sc->h.preprocess(!sc->gpu_edges);
        sc->last_launches = 0;
        upload_scene(sc.get(), 0);
        // loads the module holding the no-alloc backward's scratch array and
        // the kernels a backward call launches now, so that a later no-alloc
        // call on this device takes no memory
        noalloc_scratch();
        check_cuda(dr_preload_backward_kernels(), "kernel preload");
        *out = sc.release();
    });
}

dr_status dr_scene_update(dr_scene *scene, const dr_scene_desc *desc) {
    return guard([&]() {
        if (!scene) throw DrError(DR_ERR_INVALID_ARGUMENT, "scene is NULL");
        std::vector<std::pair<int, int>> sizes;
        for (auto &s : scene->h.shapes) sizes.emplace_back(s.nv, s.nt);
        if (!desc || desc->num_shapes != (int)sizes.size())
            throw DrError(DR_ERR_INVALID_ARGUMENT, "update must describe the same shapes");
        for (int i = 0; i < desc->num_shapes; i++)
            if (desc->shapes[i].num_vertices != sizes[i].first || desc->shapes[i].num_triangles != sizes[i].second)
                throw DrError(DR_ERR_INVALID_ARGUMENT, "update must keep every mesh's topology");
        check_cuda(cudaSetDevice(scene->device), "cudaSetDevice");
        // the meshes keep their triangles: the edge topology and the LBVH's
        // topology carry over, everything that depends on positions is redone
        std::vector<DevEdge> topo = std::move(scene->h.topo_edges);
        bool topo_valid = scene->h.topo_valid;
        std::vector<std::vector<int>> old_idx;
        for (auto &sh : scene->h.shapes) old_idx.push_back(std::move(sh.idx));
        load_desc(scene->h, desc, [](auto p, size_t n, const char *w) { return fetch(p, n, w); });
        bool same_indices = true;
        for (int i = 0; i < desc->num_shapes && same_indices; i++) same_indices = scene->h.shapes[i].idx == old_idx[i];
        if (same_indices && topo_valid) {
            scene->h.topo_edges = std::move(topo);
            scene->h.topo_valid = true;
        }
        if (!same_indices) scene->topo_dev_valid = false;
        scene->h.preprocess(!scene->gpu_edges);
        scene->last_launches = 0;
        upload_scene(scene, 0, same_indices);
    });
}

dr_status dr_scene_destroy(dr_scene *scene) {
    return guard([&]() {
        if (!scene) return;
        cudaSetDevice(scene->device);
        delete scene;
    });
}

dr_status dr_scene_grad_layout(const dr_scene *scene, dr_grad_layout *layout) {
    return guard([&]() {
        if (!scene || !layout) throw DrError(DR_ERR_INVALID_ARGUMENT, "NULL argument");
        layout->total = scene->h.grad_total;
        layout->camera = 0;
        layout->material = scene->h.layout_mat.data();
        layout->shape_vertices = scene->h.layout_vtx.data();
        layout->shape_normals = scene->h.layout_nrm.data();
        layout->light = scene->h.layout_light.data();
    });
}

dr_status dr_render_forward(dr_scene *scene, const dr_render_desc *rd, float *image_dev, void *stream) {
    return guard([&]() {
        check_render_desc(scene, rd);
        if (!image_dev) throw DrError(DR_ERR_INVALID_ARGUMENT, "image is NULL");
        check_cuda(cudaSetDevice(scene->device), "cudaSetDevice");
        scene->last_launches = 0;
        check_cuda(dr_launch_forward(call_scene(scene, rd), rd->width, rd->height, rd->spp, rd->max_bounces, rd->seed, image_dev,
                                     (cudaStream_t)stream, &scene->last_launches, &scene->timer),
                   "forward launch");
        if (scene->timer.failed)
            throw DrError(DR_ERR_CUDA, std::string("kernel ") + scene->timer.failed + " failed: " +
                                           cudaGetErrorString(scene->timer.failed_err));
        collect_timings(scene, (cudaStream_t)stream);
    });
}

namespace {
// The backward pass of dr_render_backward on the library's cached queues;
// `view` (may be null) replaces the scene's device view (another camera).
void backward_on_queues(dr_scene *scene, const dr_render_desc *rd, const DevScene *view, const float *d_image_dev,
                        float *grad_dev, float *image_dev, cudaStream_t st,
                        const std::vector<FrontCall> *fronts = nullptr, long long grad_len = 0,
                        const ViewParams *views_dev = nullptr) {
    if (!scene->queues) {
        scene->queues = take_queues(scene->device, st);
        // another scene's edge statistics say nothing about this one
        EdgeStats &es = scene->queues->stats;
        es.items_per_point = 0;
        es.buckets.clear();
        es.bucket_points = 0;
    }
    BackwardQueues &q = *scene->queues;
    long long cap_points = initial_point_cap(scene, rd, q.points_per_sample);
    double samples_total = (double)rd->width * rd->height * rd->spp;
    if (fronts) {
        cap_points = 0;
        samples_total = 0;
        for (const FrontCall &f : *fronts) {
            cap_points += initial_point_cap(scene, &f.rd, q.points_per_sample);
            samples_total += (double)f.rd.width * f.rd.height * f.rd.spp;
        }
    }
    long long cap_items =
        std::min(queue_limit(scene), std::max(q.cap_items, std::max<long long>(cap_points * 4, 1 << 16)));
    q.counts.reserve(sizeof(BackwardCounters));
    if (!q.idle) check_cuda(cudaEventCreateWithFlags(&q.idle, cudaEventDisableTiming), "cudaEventCreate");
    // marks the queues busy up to here on every way out, errors included
    struct MarkIdle {
        cudaEvent_t e;
        cudaStream_t st;
        ~MarkIdle() { cudaEventRecord(e, st); }
    } mark_idle{q.idle, st};
    BackwardWorkspace ws{};
    ws.hand_steps = scene->tune.hand_steps;
    ws.task_rounds = scene->tune.task_rounds;
    ws.level_walk = scene->tune.depth_first ? 0 : 1;
    const bool split = view ? view->split_traversal : call_scene(scene, rd).split_traversal;
    const bool lbvh = (view ? view->num_tris : call_scene(scene, rd).num_tris) > DR_LINEAR_TRIS;
    auto bind_items = [&]() {
        q.items.reserve(sizeof(int4) * cap_items);
        q.item_w.reserve(sizeof(float) * cap_items);
        q.item_dp.reserve(sizeof(float) * 3 * cap_items);
        q.survivors.reserve(sizeof(float4) * 2 * cap_items);
        q.hits.reserve(sizeof(int4) * cap_items);
        q.side_rad.reserve(sizeof(float4) * 2 * cap_items);
        q.cap_items = cap_items;
        ws.items = q.items.as<int4>();
        ws.item_w = q.item_w.as<float>();
        ws.item_dp = q.item_dp.as<float>();
        ws.survivors = q.survivors.as<float4>();
        ws.hits = q.hits.as<int4>();
        ws.side_rad = q.side_rad.as<float4>();
        ws.cap_items = cap_items;
    };
    auto bind_points = [&]() {
        q.pt.reserve(sizeof(float) * DR_PT_FLOATS * cap_points);
        q.pt_last.reserve(DR_PT_LAST_BYTES * cap_points);
        ws.pt = q.pt.as<float>();
        ws.pt_last = q.pt_last.as<unsigned long long>();
        q.pt_items.reserve(sizeof(int) * cap_points);
        ws.pt_items = q.pt_items.as<int>();
        if (split && ws.level_walk) {
            q.walk_ctx.reserve(sizeof(float4) * DR_CTX_F4 * cap_points);
            ws.walk_ctx = q.walk_ctx.as<float4>();
        }
        if (lbvh) {
            q.line_ctx.reserve(sizeof(float4) * DR_LCTX_F4 * cap_points);
            ws.line_ctx = q.line_ctx.as<float4>();
        }
        ws.cap_points = cap_points;
    };
    bind_points();
    ws.counters = q.counts.as<BackwardCounters>();
    bind_items();
    if (split) {
        long long cap_tasks = std::min(kMaxTasks, std::max(1ll << 16, kTasksPerPoint * cap_points));
        q.tasks.reserve(sizeof(EdgeTask) * cap_tasks);
        q.tasks2.reserve(sizeof(EdgeTask) * cap_tasks);
        ws.tasks = q.tasks.as<EdgeTask>();
        ws.tasks2 = q.tasks2.as<EdgeTask>();
        ws.cap_tasks = cap_tasks;
        if (ws.level_walk) {
            q.leafq.reserve(sizeof(EdgeTask) * cap_tasks);
            ws.leafq = q.leafq.as<EdgeTask>();
            ws.cap_leaves = cap_tasks;
        }
    }
    // the item queue grows to what the traversal reported, up to its limit
    // (the grown queue is kept for later calls)
    auto grow = [&](long long want) {
        long long target = std::min(want, queue_limit(scene));
        if (target > cap_items) {
            cap_items = target;
            bind_items();
        }
        return cap_items;
    };
    // the point queue grows to what the path stage reported (the ratio is
    // kept for later calls)
    auto grow_points = [&](long long want) {
        cap_points = want + want / 16 + 1;
        q.points_per_sample = (double)cap_points / samples_total;
        bind_points();
        return cap_points;
    };
    ProposalState *prop = nullptr;
    if (rd->flags & DR_FLAG_LEARNED_PROPOSAL) {
        if (!scene->proposal)
            throw DrError(DR_ERR_INVALID_ARGUMENT, "DR_FLAG_LEARNED_PROPOSAL without dr_scene_set_proposal");
        prop = scene->proposal.get();
    }
    ws.views = views_dev;
    auto counts = run_backward(scene, rd, d_image_dev, grad_dev, image_dev, ws, st, &scene->timer, grow, grow_points,
                               prop, view, &q.stats, fronts, grad_len);
    scene->last_points = counts.first;
    scene->last_items = counts.second;
}
}  // namespace

dr_status dr_render_backward(dr_scene *scene, const dr_render_desc *rd, const float *d_image_dev, float *grad_dev,
                             float *image_dev, void *stream) {
    return guard([&]() {
        check_backward_args(scene, rd, d_image_dev, grad_dev);
        check_cuda(cudaSetDevice(scene->device), "cudaSetDevice");
        cudaStream_t st = (cudaStream_t)stream;
        scene->last_launches = 0;
        backward_on_queues(scene, rd, nullptr, d_image_dev, grad_dev, image_dev, st);
        collect_timings(scene, st);
    });
}

dr_status dr_scene_get_tuning(const dr_scene *scene, dr_tuning *out) {
    return guard([&]() {
        if (!scene || !out) throw DrError(DR_ERR_INVALID_ARGUMENT, "scene or out is NULL");
        *out = scene->tune;
    });
}

dr_status dr_scene_set_tuning(dr_scene *scene, const dr_tuning *tuning) {
    return guard([&]() {
        if (!scene || !tuning) throw DrError(DR_ERR_INVALID_ARGUMENT, "scene or tuning is NULL");
        if (tuning->hand_steps < 1 || tuning->hand_steps > 4096 || tuning->task_rounds < 1 ||
            tuning->task_rounds > 8 || tuning->queue_items < 0 || tuning->depth_first < 0 ||
            tuning->depth_first > 1 || tuning->reserved != 0)
            throw DrError(DR_ERR_INVALID_ARGUMENT, "tuning out of range (hand_steps 1..4096, task_rounds 1..8, "
                                                   "queue_items >= 0, depth_first 0 or 1, reserved 0)");
        scene->tune = *tuning;
    });
}

dr_status dr_scene_autotune(dr_scene *scene, const dr_render_desc *rd, const float *d_image_dev, float *grad_dev,
                            int max_trials, dr_tune_report *report, void *stream) {
    dr_tuning start{};
    bool started = false;
    dr_status status = guard([&]() {
        check_backward_args(scene, rd, d_image_dev, grad_dev);
        if (max_trials < 1) throw DrError(DR_ERR_INVALID_ARGUMENT, "max_trials must be positive");
        check_cuda(cudaSetDevice(scene->device), "cudaSetDevice");
        cudaStream_t st = (cudaStream_t)stream;
        start = scene->tune;
        started = true;
        // one backward call under the scene's current setting, host wall time
        // up to the end of its stream work (what a caller waits for)
        auto run = [&]() {
            check_cuda(cudaStreamSynchronize(st), "cudaStreamSynchronize");
            const auto t0 = std::chrono::steady_clock::now();
            scene->last_launches = 0;
            backward_on_queues(scene, rd, nullptr, d_image_dev, grad_dev, nullptr, st);
            check_cuda(cudaStreamSynchronize(st), "cudaStreamSynchronize");
            return std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
        };
        run();  // queues sized and edge counts kept for the chunk plans
        int trials = 0;
        auto time_of = [&](const dr_tuning &t) {
            scene->tune = t;
            trials++;
            return std::min(run(), run());
        };
        dr_tuning best = start;
        float best_ms = time_of(start);
        const float start_ms = best_ms;
        auto consider = [&](dr_tuning t) {
            if (trials >= max_trials) return;
            if (t.hand_steps == best.hand_steps && t.task_rounds == best.task_rounds &&
                t.queue_items == best.queue_items && t.depth_first == best.depth_first)
                return;
            const float ms = time_of(t);
            if (ms < best_ms) {
                best_ms = ms;
                best = t;
            }
        };
        // the subtree stage's walk, and for the depth-first one its rounds
        // and hand-on steps, matter only where points hand subtrees to it
        if (scene->last_work[4] > 0) {
            for (int d : {0, 1}) {
                dr_tuning t = best;
                t.depth_first = d;
                consider(t);
            }
            if (best.depth_first)
                for (int r : {1, 2, 3, 4}) {
                    dr_tuning t = best;
                    t.task_rounds = r;
                    consider(t);
                }
            if (best.depth_first && best.task_rounds > 1)
                for (int h : {16, 32, 64, 128, 256}) {
                    dr_tuning t = best;
                    t.hand_steps = h;
                    consider(t);
                }
        }
        // smaller item queues: more chunks, each one's queues nearer to L2
        const long long base = std::min(max_queue_items(), std::max<long long>(scene->last_items, 1 << 16));
        for (int d : {2, 4, 8}) {
            dr_tuning t = best;
            t.queue_items = std::max<long long>(base / d, 1 << 16);
            consider(t);
        }
        scene->tune = best;
        if (report) {
            report->best = best;
            report->best_ms = best_ms;
            report->start_ms = start_ms;
            report->trials = trials;
        }
    });
    if (status != DR_OK && started) scene->tune = start;  // a failed search leaves the setting as it was
    return status;
}

dr_status dr_render_backward_views(dr_scene *scene, int n_views, const dr_view_desc *views, float *grad_dev,
                                   float *camera_grads_dev, void *stream) {
    return guard([&]() {
        if (!scene || n_views < 0 || (n_views > 0 && !views) || !grad_dev)
            throw DrError(DR_ERR_INVALID_ARGUMENT, "invalid view batch");
        check_cuda(cudaSetDevice(scene->device), "cudaSetDevice");
        cudaStream_t st = (cudaStream_t)stream;
        scene->last_launches = 0;
        const long long total = scene->h.grad_total;
        check_cuda(cudaMemsetAsync(grad_dev, 0, sizeof(float) * total, st), "memset");
        // view v's device scene: its camera and a primary-edge sampler built
        // from it into the given buffers
        auto setup_view = [&](int v, DevBuf &pe_buf, DevBuf &pc_buf, DevBuf &pf_buf) {
            const dr_view_desc &vw = views[v];
            HCam hc;
            auto m16 = [&](const float *p, float *dst, const char *what) {
                std::vector<float> m = fetch(p, 16, what);
                std::memcpy(dst, m.data(), 64);
            };
            m16(vw.camera.cam_to_world, hc.c2w, "view cam_to_world");
            m16(vw.camera.world_to_cam, hc.w2c, "view world_to_cam");
            hc.fov = vw.camera.fov_factor;
            hc.aspect = vw.camera.aspect_ratio;
            hc.clip_near = vw.camera.clip_near;
            hc.fisheye = vw.camera.fisheye != 0;
            int n_prim = 0;
            float prim_func_int = 0.f;
            if (scene->gpu_edges) {
                DevCamera dc;
                std::memcpy(dc.c2w.m, hc.c2w, 64);
                std::memcpy(dc.w2c.m, hc.w2c, 64);
                dc.fov = hc.fov;
                dc.aspect = hc.aspect;
                dc.clip_near = hc.clip_near;
                dc.fisheye = hc.fisheye;
                const int nk = scene->num_kept;
                pe_buf.reserve(sizeof(DevEdge) * std::max(1, nk));
                pc_buf.reserve(sizeof(float) * (nk + 1));
                pf_buf.reserve(sizeof(float) * std::max(1, nk));
                check_cuda(dr_build_primary(scene->ds, dc, scene->kept_dev, nk, pe_buf.as<DevEdge>(),
                                            pc_buf.as<float>(), pf_buf.as<float>(), &n_prim, &prim_func_int,
                                            scene->edge_scratch.p, scene->edge_scratch.bytes, st,
                                            &scene->last_launches),
                           "view primary-edge sampler");
            } else {
                std::vector<DevEdge> pe;
                HDist pd;
                scene->h.primary_for(hc, pe, pd);
                pe_buf.upload(pe);
                pc_buf.upload(pd.cdf);
                pf_buf.upload(pd.func);
                n_prim = (int)pe.size();
                prim_func_int = pd.func_int;
            }
            DevScene ds = call_scene(scene, &vw.render);
            std::memcpy(ds.cam.c2w.m, hc.c2w, 64);
            std::memcpy(ds.cam.w2c.m, hc.w2c, 64);
            ds.cam.fov = hc.fov;
            ds.cam.aspect = hc.aspect;
            ds.cam.clip_near = hc.clip_near;
            ds.cam.fisheye = hc.fisheye;
            ds.prim_edges = pe_buf.as<DevEdge>();
            ds.num_prim_edges = n_prim;
            ds.prim_cdf = pc_buf.as<float>();
            ds.prim_func = pf_buf.as<float>();
            ds.prim_func_int = prim_func_int;
            return ds;
        };
        for (int v = 0; v < n_views; v++)
            check_backward_args(scene, &views[v].render, views[v].d_image, grad_dev);
        // One edge stage for every view when they differ only in camera,
        // size, samples, seed and adjoint (the kernels take those per point).
        bool batched = n_views > 1;
        for (int v = 1; v < n_views && batched; v++) {
            const dr_render_desc &a = views[0].render, &b = views[v].render;
            batched = a.max_bounces == b.max_bounces && a.flags == b.flags && a.dp_mode == b.dp_mode;
        }
        if (views && n_views > 0 && (views[0].render.flags & DR_FLAG_LEARNED_PROPOSAL)) batched = false;
        long long points = 0, items = 0;
        if (batched) {
            const long long glen = total + 64ll * n_views;
            scene->view_grad.reserve(sizeof(float) * glen);
            float *vg = scene->view_grad.as<float>();
            while ((int)scene->batch_prim.size() < 3 * n_views)
                scene->batch_prim.emplace_back(new DevBuf());
            std::vector<FrontCall> fronts(n_views);
            std::vector<ViewParams> table(n_views);
            for (int v = 0; v < n_views; v++) {
                FrontCall &f = fronts[v];
                f.ds = setup_view(v, *scene->batch_prim[3 * v], *scene->batch_prim[3 * v + 1],
                                  *scene->batch_prim[3 * v + 2]);
                f.ds.cam_off = (int)(total + 64ll * v);
                f.ds.view_id = v;
                f.rd = views[v].render;
                f.d_image = views[v].d_image;
                f.image = views[v].image;
                ViewParams &t = table[v];
                t.cam = f.ds.cam;
                t.W = f.rd.width;
                t.H = f.rd.height;
                t.spp = f.rd.spp;
                t.cam_off = f.ds.cam_off;
                t.seed = f.rd.seed;
            }
            scene->view_table.upload(table);
            backward_on_queues(scene, &fronts[0].rd, &fronts[0].ds, fronts[0].d_image, vg, nullptr, st, &fronts, glen,
                               scene->view_table.as<ViewParams>());
            points = scene->last_points;
            items = scene->last_items;
            // the views' summed gradient (camera block zero) and their camera blocks
            check_cuda(cudaMemcpyAsync(grad_dev + 64, vg + 64, sizeof(float) * (total - 64), cudaMemcpyDeviceToDevice,
                                       st),
                       "gradient copy");
            if (camera_grads_dev)
                check_cuda(cudaMemcpyAsync(camera_grads_dev, vg + total, sizeof(float) * 64 * (size_t)n_views,
                                           cudaMemcpyDeviceToDevice, st),
                           "camera gradients");
            check_cuda(cudaStreamSynchronize(st), "views");
        } else {
            scene->view_grad.reserve(sizeof(float) * total);
            float *vg = scene->view_grad.as<float>();
            for (int v = 0; v < n_views; v++) {
                const dr_view_desc &vw = views[v];
                // the view's sampler (the previous view's kernels have finished)
                DevScene ds = setup_view(v, scene->view_prim_edges, scene->view_prim_cdf, scene->view_prim_func);
                backward_on_queues(scene, &vw.render, &ds, vw.d_image, vg, vw.image, st);
                points += scene->last_points;
                items += scene->last_items;
                check_cuda(dr_launch_accumulate(grad_dev + 64, vg + 64, total - 64, st), "gradient sum");
                if (camera_grads_dev)
                    check_cuda(cudaMemcpyAsync(camera_grads_dev + 64 * (size_t)v, vg, 64 * sizeof(float),
                                               cudaMemcpyDeviceToDevice, st),
                               "camera gradient");
                check_cuda(cudaStreamSynchronize(st), "view");
            }
        }
        scene->last_points = points;
        scene->last_items = items;
        collect_timings(scene, st);
    });
}

int dr_mlp_param_count(void) { return kMlpParams; }

dr_status dr_scene_set_proposal(dr_scene *scene, const dr_proposal_desc *d) {
    return guard([&]() {
        if (!scene || !d) throw DrError(DR_ERR_INVALID_ARGUMENT, "scene and desc must be non-NULL");
        if (!(d->mix >= 0.f && d->mix <= 1.f)) throw DrError(DR_ERR_INVALID_ARGUMENT, "mix must lie in [0, 1]");
        if (!(d->learning_rate >= 0.f)) throw DrError(DR_ERR_INVALID_ARGUMENT, "learning_rate must be >= 0");
        check_cuda(cudaSetDevice(scene->device), "cudaSetDevice");
        bool fresh = !scene->proposal;
        if (fresh) {
            auto pr = std::make_unique<ProposalState>();
            for (DevBuf *b : {&pr->params, &pr->m, &pr->v, &pr->grads}) b->reserve(sizeof(float) * kMlpParams);
            pr->img.reserve(kImgBytes);
            pr->loss.reserve(sizeof(float));
            pr->total.reserve(sizeof(float));
            pr->status.reserve(sizeof(int));
            scene->proposal = std::move(pr);
        }
        ProposalState &pr = *scene->proposal;
        pr.train = d->train != 0;
        pr.alpha = d->mix;
        pr.lr = d->learning_rate;
        pr.train_points = d->train_points > 0 ? (long long)d->train_points : 32768;
        if (d->params || fresh) {
            std::vector<float> p(kMlpParams);
            if (d->params) {
                p = fetch(d->params, kMlpParams, "params");
            } else {  // nn.Linear's initialisation, W1 with the 10 real inputs as fan-in
                std::mt19937 gen(0);
                std::uniform_real_distribution<float> u(-1.f, 1.f);
                const int ends[8] = {kMlpB1, kMlpW2, kMlpB2, kMlpW3, kMlpB3, kMlpW4, kMlpB4, kMlpParams};
                for (int i = 0, blk = 0; i < kMlpParams; i++) {
                    while (i >= ends[blk]) blk++;
                    float fan = blk < 2 ? (float)DR_MLP_FEATURES : (float)DR_MLP_HIDDEN;
                    p[i] = u(gen) / std::sqrt(fan);
                }
            }
            pr.params.upload(p);
            check_cuda(cudaMemset(pr.m.p, 0, sizeof(float) * kMlpParams), "memset");
            check_cuda(cudaMemset(pr.v.p, 0, sizeof(float) * kMlpParams), "memset");
            pr.steps = 0;
            pr.last_loss = 0.f;
            check_cuda(dr_mlp_pack(pr.params.as<float>(), pr.img.as<uint8_t>(), 0), "weight pack");
            check_cuda(cudaDeviceSynchronize(), "weight pack");
        }
    });
}

dr_status dr_scene_proposal_state(const dr_scene *scene, float *params_out, float *last_loss, int64_t *steps) {
    return guard([&]() {
        if (!scene) throw DrError(DR_ERR_INVALID_ARGUMENT, "scene is NULL");
        if (!scene->proposal) throw DrError(DR_ERR_INVALID_ARGUMENT, "the scene has no proposal");
        check_cuda(cudaSetDevice(scene->device), "cudaSetDevice");
        const ProposalState &pr = *scene->proposal;
        if (params_out)
            check_cuda(cudaMemcpy(params_out, pr.params.p, sizeof(float) * kMlpParams, cudaMemcpyDefault),
                       "params read");
        if (last_loss) *last_loss = pr.last_loss;
        if (steps) *steps = pr.steps;
    });
}

namespace {
// Device buffers of one network call: bf16 rows, packed weights, status word.
struct MlpScratch {
    DevBuf x16, img, status, total;
    void bind(const float *x_dev, int64_t n, const float *params_dev, cudaStream_t st) {
        x16.reserve(sizeof(__nv_bfloat16) * DR_MLP_IN * (size_t)std::max<int64_t>(n, 1));
        img.reserve(kImgBytes);
        status.reserve(sizeof(int));
        total.reserve(sizeof(float));
        check_cuda(cudaMemsetAsync(status.p, 0, sizeof(int), st), "memset");
        check_cuda(dr_mlp_to_bf16(x_dev, x16.as<__nv_bfloat16>(), n * DR_MLP_IN, st), "bf16 rows");
        check_cuda(dr_mlp_pack(params_dev, img.as<uint8_t>(), st), "weight pack");
    }
    void check(cudaStream_t st) {
        int s = 0;
        check_cuda(cudaMemcpyAsync(&s, status.p, sizeof(int), cudaMemcpyDeviceToHost, st), "status read");
        check_cuda(cudaStreamSynchronize(st), "network");
        if (s) throw DrError(DR_ERR_DEVICE_STATUS, "network kernel reported status " + std::to_string(s));
    }
};
int current_sms() {
    int dev = 0, sms = 148;
    check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "device query");
    return sms;
}
}  // namespace

dr_status dr_mlp_forward(const float *params_dev, const float *x_dev, int64_t n, float *logits_dev, void *stream) {
    return guard([&]() {
        if (n < 0 || (n > 0 && (!params_dev || !x_dev || !logits_dev)))
            throw DrError(DR_ERR_INVALID_ARGUMENT, "invalid network buffers");
        cudaStream_t st = (cudaStream_t)stream;
        MlpScratch m;
        m.bind(x_dev, n, params_dev, st);
        check_cuda(dr_mlp_infer(m.img.as<uint8_t>(), params_dev, m.x16.as<__nv_bfloat16>(), n, logits_dev, nullptr,
                                m.status.as<int>(), current_sms(), st),
                   "network forward");
        m.check(st);
    });
}

dr_status dr_mlp_gradient(const float *params_dev, const float *x_dev, const float *targets_dev, int64_t n,
                          float *grads_dev, float *loss_dev, void *stream) {
    return guard([&]() {
        if (n < 0 || !params_dev || !grads_dev || !loss_dev || (n > 0 && (!x_dev || !targets_dev)))
            throw DrError(DR_ERR_INVALID_ARGUMENT, "invalid network buffers");
        cudaStream_t st = (cudaStream_t)stream;
        MlpScratch m;
        m.bind(x_dev, n, params_dev, st);
        check_cuda(cudaMemsetAsync(grads_dev, 0, sizeof(float) * kMlpParams, st), "memset");
        check_cuda(cudaMemsetAsync(loss_dev, 0, sizeof(float), st), "memset");
        check_cuda(dr_mlp_sum(targets_dev, n * DR_MLP_OUT, m.total.as<float>(), st), "target sum");
        check_cuda(dr_mlp_grad(m.img.as<uint8_t>(), params_dev, m.x16.as<__nv_bfloat16>(), targets_dev, n,
                               m.total.as<float>(), grads_dev, loss_dev, m.status.as<int>(), current_sms(), st),
                   "network gradient");
        m.check(st);
    });
}

dr_status dr_eval_math(int fn, const float *x_dev, const float *y_dev, float *out_dev, int64_t n, void *stream) {
    return guard([&]() {
        if (fn < 0 || fn > 7 || n < 0 || (n > 0 && (!x_dev || !out_dev)))
            throw DrError(DR_ERR_INVALID_ARGUMENT, "dr_eval_math: bad function number or NULL buffer");
        if ((fn == 3 || fn == 7) && n > 0 && !y_dev)
            throw DrError(DR_ERR_INVALID_ARGUMENT, "dr_eval_math: atan2 and pow need y");
        check_cuda(dr_launch_eval_math(fn, x_dev, y_dev, out_dev, n, (cudaStream_t)stream), "math kernel");
        check_cuda(cudaStreamSynchronize((cudaStream_t)stream), "math kernel");
    });
}

dr_status dr_trace_rays(dr_scene *scene, const float *rays_dev, int64_t n, int *tri_dev, float *t_dev, void *stream) {
    return guard([&]() {
        if (!scene) throw DrError(DR_ERR_INVALID_ARGUMENT, "scene is NULL");
        if (n < 0 || (n > 0 && (!rays_dev || !tri_dev || !t_dev)))
            throw DrError(DR_ERR_INVALID_ARGUMENT, "invalid ray buffers");
        check_cuda(cudaSetDevice(scene->device), "cudaSetDevice");
        scene->last_launches = 0;
        check_cuda(dr_launch_trace(scene->ds, rays_dev, n, tri_dev, t_dev, (cudaStream_t)stream,
                                   &scene->last_launches),
                   "trace launch");
    });
}

dr_status dr_scene_set_profiling(dr_scene *scene, int enable) {
    return guard([&]() {
        if (!scene) throw DrError(DR_ERR_INVALID_ARGUMENT, "scene is NULL");
        check_cuda(cudaSetDevice(scene->device), "cudaSetDevice");
        if (enable && !scene->timer_ready) {
            for (int i = 0; i <= StageTimer::kMax; i++)
                check_cuda(cudaEventCreate(&scene->timer.ev[i]), "cudaEventCreate");
            scene->timer_ready = true;
        }
        scene->timer.on = enable != 0;
    });
}

dr_status dr_scene_last_timings(const dr_scene *scene, int index, char *name, size_t name_len, float *ms) {
    return guard([&]() {
        if (!scene || !ms) throw DrError(DR_ERR_INVALID_ARGUMENT, "NULL argument");
        if (index < 0 || index >= (int)scene->timings.size()) throw DrError(DR_ERR_INVALID_ARGUMENT, "no such stage");
        const auto &t = scene->timings[index];
        if (name && name_len > 0) {
            size_t c = std::min(t.first.size(), name_len - 1);
            std::memcpy(name, t.first.data(), c);
            name[c] = 0;
        }
        *ms = t.second;
    });
}

dr_status dr_scene_last_counts(const dr_scene *scene, int64_t *points, int64_t *items) {
    return guard([&]() {
        if (!scene || !points || !items) throw DrError(DR_ERR_INVALID_ARGUMENT, "NULL argument");
        *points = scene->last_points;
        *items = scene->last_items;
    });
}

dr_status dr_scene_edge_data(const dr_scene *scene, int what, void *out_host, int64_t capacity_bytes,
                             int64_t *count, float *build_ms) {
    return guard([&]() {
        if (!scene || !count) throw DrError(DR_ERR_INVALID_ARGUMENT, "NULL argument");
        const DevScene &ds = scene->ds;
        const void *src = nullptr;
        size_t elem = 0, n = 0;
        switch (what) {
        case 0: src = ds.sil_nodes; elem = sizeof(DevEdgeNode); n = ds.num_sil_nodes; break;
        case 1:
            src = ds.sil_edges;
            elem = sizeof(DevEdge);
            n = ds.num_sil_nodes ? edge_count_of(scene, ds.sil_nodes, ds.num_sil_nodes) : 0;
            break;
        case 2: src = ds.nrm_nodes; elem = sizeof(DevEdgeNode); n = ds.num_nrm_nodes; break;
        case 3:
            src = ds.nrm_edges;
            elem = sizeof(DevEdge);
            n = ds.num_nrm_nodes ? edge_count_of(scene, ds.nrm_nodes, ds.num_nrm_nodes) : 0;
            break;
        case 4: src = ds.prim_edges; elem = sizeof(DevEdge); n = ds.num_prim_edges; break;
        case 5: src = ds.prim_cdf; elem = 4; n = ds.num_prim_edges ? ds.num_prim_edges + 1 : 0; break;
        case 6: src = ds.prim_func; elem = 4; n = ds.num_prim_edges; break;
        case 7: break;
        default: throw DrError(DR_ERR_INVALID_ARGUMENT, "no such edge array");
        }
        *count = what == 7 ? 1 : (int64_t)n;
        if (build_ms) *build_ms = scene->gpu_edges ? scene->edge_build_ms : 0.f;
        if (!out_host || capacity_bytes <= 0) return;
        check_cuda(cudaSetDevice(scene->device), "cudaSetDevice");
        if (what == 7) {
            if (capacity_bytes >= 4) std::memcpy(out_host, &ds.prim_func_int, 4);
            return;
        }
        size_t bytes = std::min((size_t)capacity_bytes, elem * n);
        if (bytes) check_cuda(cudaMemcpy(out_host, src, bytes, cudaMemcpyDeviceToHost), "edge data copy");
    });
}

dr_status dr_scene_last_work(const dr_scene *scene, int64_t *counts, int n) {
    return guard([&]() {
        if (!scene || !counts || n < 0) throw DrError(DR_ERR_INVALID_ARGUMENT, "NULL argument");
        for (int i = 0; i < n && i < 10; i++) counts[i] = scene->last_work[i];
    });
}

dr_status dr_scene_last_launch_count(const dr_scene *scene, int *count) {
    return guard([&]() {
        if (!scene || !count) throw DrError(DR_ERR_INVALID_ARGUMENT, "NULL argument");
        *count = scene->last_launches;
    });
}

size_t dr_last_error(char *buf, size_t len) {
    size_t n = g_last_error.size();
    if (buf && len > 0) {
        size_t c = std::min(n, len - 1);
        std::memcpy(buf, g_last_error.data(), c);
        buf[c] = 0;
    }
    return n;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// dr_render_backward_noalloc: the backward pass with its work queues in a
// fixed device array that is part of the library's module image, so that a
// call allocates no device memory.
// ---------------------------------------------------------------------------
namespace {
constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;  // per device
constexpr long long kNoAllocMaxSamples = 65536;            // width * height * spp
}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {
// Device address of the current device's copy of the array.  It is looked up
// on every call rather than cached, so that a context that was reset and made
// again (cudaDeviceReset) gets the address of its own copy.  The lookup loads
// the module that holds the array when CUDA loads modules lazily; scene
// creation makes the same lookup, so that the array's memory is taken there
// and a no-alloc call never loads a module itself.
unsigned char *noalloc_scratch() {
    void *p = nullptr;
    check_cuda(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress");
    if (!p) throw DrError(DR_ERR_CUDA, "cudaGetSymbolAddress returned NULL");
    return (unsigned char *)p;
}
}  // namespace

extern "C" {

dr_status dr_render_backward_noalloc(dr_scene *scene, const dr_render_desc *rd, const float *d_image_dev,
                                     float *grad_dev, float *image_dev, void *stream) {
    return guard([&]() {
        check_backward_args(scene, rd, d_image_dev, grad_dev);
        long long npix = (long long)rd->width * rd->height * rd->spp;
        if (rd->flags & DR_FLAG_LEARNED_PROPOSAL)
            throw DrError(DR_ERR_NOT_SUPPORTED, "the no-alloc backward does not run the learned proposal");
        if (npix > kNoAllocMaxSamples)
            throw DrError(DR_ERR_INVALID_ARGUMENT,
                          "width * height * spp = " + std::to_string(npix) + " exceeds the " +
                              std::to_string(kNoAllocMaxSamples) +
                              " pixel samples of the no-alloc backward's fixed scratch; use dr_render_backward");
        check_cuda(cudaSetDevice(scene->device), "cudaSetDevice");
        cudaStream_t st = (cudaStream_t)stream;
        scene->last_launches = 0;
        scene->timings.clear();  // this path records no stage timings
        unsigned char *base = noalloc_scratch();
        // layout: counters | point records | point keys | items | item weights | item dp | survivors | hits
        auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
        // scenes with specular chains: room for the points of every bounce,
        // up to half the scratch (the rest holds edge items)
        long long cap_points = npix;
        if (scene->h.specular_bounces && rd->max_bounces >= 1) {
            long long want = npix * std::min(rd->max_bounces + 1, DR_MAX_LINKS + 1);
            long long fit = (long long)(kNoAllocScratchBytes / 2 / (sizeof(float) * DR_PT_FLOATS + DR_PT_LAST_BYTES));
            cap_points = std::max(npix, std::min(want, fit));
        }
        size_t off = 256;
        BackwardWorkspace ws{};
        ws.counters = (BackwardCounters *)base;
        ws.pt = (float *)(base + off);
        off += up(sizeof(float) * DR_PT_FLOATS * (size_t)cap_points);
        ws.pt_last = (unsigned long long *)(base + off);
        off += up(DR_PT_LAST_BYTES * (size_t)cap_points);
        long long cap_items = (long long)((kNoAllocScratchBytes - off - 5 * 256) /
                                          (2 * sizeof(int4) + 4 * sizeof(float) + 2 * sizeof(float4)));
        ws.items = (int4 *)(base + off);
        off += up(sizeof(int4) * (size_t)cap_items);
        ws.item_w = (float *)(base + off);
        off += up(sizeof(float) * (size_t)cap_items);
        ws.item_dp = (float *)(base + off);
        off += up(sizeof(float) * 3 * (size_t)cap_items);
        ws.survivors = (float4 *)(base + off);
        off += up(sizeof(float4) * 2 * (size_t)cap_items);
        ws.hits = (int4 *)(base + off);
        off += up(sizeof(int4) * (size_t)cap_items);
        if (off > kNoAllocScratchBytes) throw DrError(DR_ERR_INVALID_ARGUMENT, "scratch layout does not fit");
        ws.cap_points = cap_points;
        ws.cap_items = cap_items;
        // what must start at zero, the queue counters and the gradient, is
        // cleared by run_backward (the point keys of the "last edge" rule by
        // the launcher); the queue cannot grow, so large edge stages stream
        StageTimer quiet;  // no profiling events on this path
        auto counts = run_backward(scene, rd, d_image_dev, grad_dev, image_dev, ws, st, &quiet,
                                   [&](long long) { return cap_items; }, [&](long long) { return cap_points; });
        scene->last_points = counts.first;
        scene->last_items = counts.second;
    });
}

}  // extern "C"
