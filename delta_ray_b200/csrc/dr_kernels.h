// Host-callable launchers of the renderer's kernels (defined in the .cu files).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "dr_scene.cuh"

// Optional per-stage timing: events recorded on the launch stream around each
// kernel when `on` is set (costs one event record per stage).
// With `sync` set (the DR_DEBUG_SYNC environment variable, a diagnostic), every
// mark synchronizes the stream and remembers the first kernel that failed.
struct StageTimer {
    // a streamed edge stage marks its kernels once per chunk of points, the
    // level walk's two once per level
    static const int kMax = 4096;
    bool on = false;
    bool sync = false;
    const char *failed = nullptr;
    cudaError_t failed_err = cudaSuccess;
    int n = 0;
    cudaEvent_t ev[kMax + 1];
    const char *names[kMax];
    void begin(cudaStream_t st) {
        n = 0;
        if (on) cudaEventRecord(ev[0], st);
    }
    void mark(cudaStream_t st, const char *name) {
        if (sync && !failed) {
            cudaError_t e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) {
                failed = name;
                failed_err = e;
            }
        }
        if (!on || n >= kMax) return;
        names[n++] = name;
        cudaEventRecord(ev[n], st);
    }
};

// LBVH over n triangles (dr_kernels.cu); `nodes` holds 4 float4 per internal
// node, `leaf_tris` 3 float4 per triangle; scratch >= dr_lbvh_scratch_bytes(n).
cudaError_t dr_build_lbvh(const float *vtx, const int4 *tri, int n, float3 lo, float3 hi, float4 *nodes,
                          float4 *leaf_tris, void *scratch, size_t scratch_bytes, cudaStream_t st, int *launches);
size_t dr_lbvh_scratch_bytes(int n);
// The 4-wide form of an LBVH over n triangles (DR_WIDE_F4 float4 per
// internal node, DevScene::bvh_wide), from its binary nodes; after every build
// and refit.
cudaError_t dr_widen_lbvh(const float4 *nodes, int n, float4 *wide, cudaStream_t st, int *launches);
// Recomputes the boxes of an LBVH built by dr_build_lbvh over the same
// triangles (same scratch, kept since the build) for new vertex positions.
cudaError_t dr_refit_lbvh(const float *vtx, const int4 *tri, int n, float4 *nodes, float4 *leaf_tris, void *scratch,
                          size_t scratch_bytes, cudaStream_t st, int *launches);

// GPU build of a scene's edge data (dr_scene_build.cu).  Each call finishes
// (synchronizes `st`) before it returns its counts.
// Unique edges (scene.cpp:54-97) into out (capacity 3 * s.num_tris).
size_t dr_edges_scratch_bytes(int ntri);
cudaError_t dr_extract_edges(const DevScene &s, int num_vertices, DevEdge *out, int *count_host, void *scratch,
                             size_t scratch_bytes, cudaStream_t st, int *launches);
// The kept edges and the silhouette and normal sets (capacity n each);
// counts_host: kept, silhouette, normal.  Scratch: dr_edges_scratch_bytes.
cudaError_t dr_split_edges(const DevScene &s, const DevEdge *topo, int n, DevEdge *kept, DevEdge *sil, DevEdge *nrm,
                           int counts_host[3], void *scratch, size_t scratch_bytes, cudaStream_t st, int *launches);
// The primary-edge sampler of camera cam over n kept edges: prim (capacity
// n), cdf (n + 1), func (n).  Scratch: dr_edges_scratch_bytes.
cudaError_t dr_build_primary(const DevScene &s, const DevCamera &cam, const DevEdge *kept, int n, DevEdge *prim,
                             float *cdf, float *func, int *count_host, float *func_int_host, void *scratch,
                             size_t scratch_bytes, cudaStream_t st, int *launches);
// A median-split edge tree of n edges (the product's rule, dr_edge_rules.h):
// nodes (capacity 2n - 1) in the flattened layout, the edges in leaf order.
size_t dr_tree_scratch_bytes(int n);
cudaError_t dr_build_edge_tree(const DevScene &s, bool dir, const DevEdge *edges, int n, DevEdgeNode *nodes,
                               DevEdge *ordered, int *num_nodes_host, void *scratch, size_t scratch_bytes,
                               cudaStream_t st, int *launches);

cudaError_t dr_launch_eval_math(int fn, const float *x, const float *y, float *out, long long n, cudaStream_t st);
cudaError_t dr_launch_trace(const DevScene &s, const float *rays, long long n, int *tri, float *t, cudaStream_t st,
                            int *launches);

cudaError_t dr_launch_forward(const DevScene &s, int W, int H, int spp, int B, uint64_t seed, float *img,
                              cudaStream_t st, int *launches, StageTimer *timer);

// Backward pass (dr_backward.cu).
// Queue counters on the device.  They are 64-bit and keep counting past a
// queue's capacity, so the host learns how many entries a launch needed.
struct BackwardCounters {
    unsigned long long points;  // shading points appended by k_backward_paths
    unsigned long long items;   // edge items appended by the last k_edge_traverse
    int status;                 // DR_STATUS_* bits
    int pad;
    unsigned long long survivors;  // line samples k_edge_line kept for the ray stage
    unsigned long long hits;       // samples the ray stage kept for k_edge_shade (follows survivors)
    unsigned long long tasks;      // subtrees k_edge_expand handed on to k_edge_tasks
    // work counts for the roofline's byte model: edge-tree nodes visited by
    // the point walks (k_edge_traverse / k_edge_expand) and by k_edge_tasks,
    // and the item count when k_edge_expand finished
    unsigned long long visits_walk, visits_tasks, items_expand;
    unsigned long long task_next;  // next task of k_edge_tasks (lanes fetch them one by one)
    // the ray stage: line samples fetched by k_edge_connect, its candidates
    // (records in `hits`, flagged by k_edge_pairs; `hits` counts the flagged
    // ones), candidates fetched by k_edge_pairs
    unsigned long long ray_next, cands, pair_next;
    // subtrees handed on between rounds of k_edge_tasks (two queues, used in
    // turn) and their total
    unsigned long long handed[2], handed_total;
    // leaves the level walk's launch queued for k_edge_leaves; the nodes it
    // queued for the next level, per class (front and back half of the
    // queue, two queues used in turn); subtrees a full queue left to a lane's
    // depth-first walk
    unsigned long long leaf_n, level_n[2][2], spilled;
};

// A view of a batched multi-view backward call: what the edge stage needs of
// the view its shading points came from.
struct ViewParams {
    DevCamera cam;
    int W, H, spp;
    int cam_off;  // the view's camera block in the flat gradient
    uint64_t seed;
};

struct BackwardWorkspace {
    float *pt;                   // [cap_points][DR_PT_FLOATS] shading-point records
    long long cap_points;
    int4 *items;                 // sampled edges: (point, tree << 30 | edge, ordinal j, 0)
    float *item_w;               // edge weight
    long long cap_items;
    float *item_dp;              // [cap_items][3] position adjoint of each item
    // [cap_points] x DR_PT_LAST_BYTES: DR_DP_REFERENCE_LAST keeps ((j + 1) << 32 | item)
    // of the point's last item with dp != 0 in the first 8 bytes; DR_DP_SUM on
    // scenes with specular chains sums the dp of points after the first vertex
    // as a float4
    unsigned long long *pt_last;
    BackwardCounters *counters;
    // points [pt_begin, min(pt_end, counters->points)) go through the edge
    // stage (traversal, edge evaluation, k_dp_propagate) of one launch
    long long pt_begin, pt_end;
    // the traversal kernels walk every pt_stride-th point of that range only
    // (the first call's forecast of the edge counts); 1 otherwise
    long long pt_stride = 1;
    // learned edge proposal (null: the reference's sampling): [cap_points][32]
    // bf16 slot probabilities, the mixture weight, and the training targets of
    // points p = k * train_stride, k < train_n ([train_n][32] f32 contribution
    // magnitudes per slot)
    // line samples that survived the first phase of edge evaluation:
    // [cap_items][2] float4 (item index bits, sample_p; d sample_p / d l, density)
    float4 *survivors;
    // [cap_items] per candidate of the ray stage (survivor index, closest-hit
    // triangle of the right and the left ray, kept ? 1 : 0)
    int4 *hits;
    // [cap_items][2] the two sides' radiance per candidate (k_edge_radiance;
    // null: k_edge_shade shades the sides itself)
    float4 *side_rad;
    // subtrees of large trees' traversals handed on to a second stage
    // (null: one thread walks each point whole)
    EdgeTask *tasks;
    long long cap_tasks;
    // [cap_tasks] the second queue of the rounds of k_edge_tasks (null: one
    // round, no subtree handed on)
    EdgeTask *tasks2;
    // the subtree walks of k_edge_tasks: steps a walk takes before it hands
    // its shallowest pending subtree on, and launches (rounds) per chunk of
    // points (the scene's tuning, dr_scene_set_tuning)
    int hand_steps = 64, task_rounds = 3;
    // the level-by-level walk of the subtrees (level_walk != 0; otherwise
    // k_edge_tasks walks each depth first): every point's walk context
    // ([cap_points][DR_CTX_F4] float4, k_walk_ctx) and the queue of the
    // leaves each level reached (cap_leaves entries); the levels' own queues
    // are `tasks` and `tasks2`, used in turn
    int level_walk = 1;
    float4 *walk_ctx;
    // [cap_points][DR_LCTX_F4] each point's line-sample setup (k_line_ctx;
    // null: k_edge_line sets it up per edge)
    float4 *line_ctx;
    EdgeTask *leafq;
    long long cap_leaves;
    // per view of a batched multi-view call (null: the call's own settings);
    // each point's settings are views[point.view]
    const ViewParams *views;
    // [cap_points] edges each point's traversal sampled, written by the point
    // walk and added to by its subtrees (null: not kept); the streamed edge
    // stage plans its chunks from them
    int *pt_items;
    const uint16_t *proposal_q;
    float proposal_alpha;
    float *train_targets;
    long long train_stride, train_n;
};

// Which part of the flat gradient a block caches in shared memory:
// [0, head) and [tail_begin, tail_begin + tail_len).
struct GradCacheCfg {
    int head, tail_begin, tail_len;
};

// The backward pass runs in two halves with a host check between them: the
// front half (path adjoints, primary edges, edge traversal) fills the point
// and item queues; when the item queue overflowed, the host grows it to the
// reported count and re-runs only the traversal; the back half evaluates the
// queued edge samples.
cudaError_t dr_launch_backward_front(const DevScene &s, int W, int H, int spp, int B, uint64_t seed,
                                     const float *d_image, float *grad, float *img, long long primary_edge_samples,
                                     int dp_mode, const BackwardWorkspace &ws, const GradCacheCfg &cfg, int num_sms,
                                     cudaStream_t st, int *launches, StageTimer *timer, bool traverse = true,
                                     bool first = true);
// Features of the learned edge proposal for points [0, n): x[n][16] bf16
// (position normalised by the scene centre c and inverse half extent ih,
// shading normal, roughness, incoming direction, zeros); points
// p = k * train_stride (k < train_n) are also written to xt[k].
cudaError_t dr_launch_proposal_features(const DevScene &s, const BackwardWorkspace &ws, long long n, float3 c,
                                        float3 ih, void *x, void *xt, cudaStream_t st);
// Load every kernel a backward call can launch (CUDA loads kernels lazily, at
// their first launch, taking device memory for their code).
cudaError_t dr_preload_backward_kernels();
cudaError_t dr_preload_edge_kernels();
cudaError_t dr_launch_edge_traverse(const DevScene &s, uint64_t seed, const BackwardWorkspace &ws, int num_sms,
                                    cudaStream_t st, int *launches, StageTimer *timer);
// The silhouette-test records of n tree edges (dr_edges.cuh: edge_record).
cudaError_t dr_launch_edge_records(const DevScene &s, const DevEdge *edges, int n, EdgeRec *out, cudaStream_t st);
// out[b] = edges sampled by points [b P / nb, (b + 1) P / nb) (ws.pt_items)
cudaError_t dr_launch_item_buckets(const int *pt_items, long long P, int nb, unsigned long long *out,
                                   cudaStream_t st);
// dst[0..n) += src[0..n)
cudaError_t dr_launch_accumulate(float *dst, const float *src, long long n, cudaStream_t st);
// Launchers of the edge half (dr_edge_kernels.cu).  Edge evaluation is a
// three-kernel wavefront: line samples, their rays, their shading.
cudaError_t dr_launch_edge_eval(const DevScene &s, int W, int H, int spp, int B, uint64_t seed, int dp_mode,
                                float *grad, const BackwardWorkspace &ws, const GradCacheCfg &cfg, int num_sms,
                                cudaStream_t st, int *launches, StageTimer *timer);
// Primary edges as two kernels (k_primary_shade, k_primary_grad) that pass
// each sample's color difference through `scratch` (cap samples at a time).
cudaError_t dr_launch_primary_edges(const DevScene &s, int W, int H, int spp, int B, uint64_t seed,
                                    const float *d_image, long long n, float *grad, const GradCacheCfg &cfg,
                                    float4 *scratch, long long cap, int num_sms, cudaStream_t st, int *launches,
                                    StageTimer *timer);
cudaError_t dr_launch_backward_back(const DevScene &s, int W, int H, int spp, int B, uint64_t seed, float *grad,
                                    int dp_mode, const BackwardWorkspace &ws, const GradCacheCfg &cfg, int num_sms,
                                    cudaStream_t st, int *launches, StageTimer *timer);

// float4 of one point's walk context in BackwardWorkspace::walk_ctx.
#define DR_CTX_F4 11
// float4 of one point's line-sample setup in BackwardWorkspace::line_ctx.
#define DR_LCTX_F4 6

// Words of one packed secondary-point record in BackwardWorkspace::pt.
#define DR_PT_FLOATS 24

// Device status bits.
#define DR_PT_LAST_BYTES 16
#define DR_STATUS_POINT_OVERFLOW 1
#define DR_STATUS_ITEM_OVERFLOW 2
#define DR_STATUS_STACK_OVERFLOW 4
