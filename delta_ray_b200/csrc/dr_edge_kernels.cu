// Backward pass, edge half: edge-tree traversal of the shading points, the
// secondary edge samples they drew, and the primary (screen-space) edges.
// Compiled without FMA contraction, like the path half: the edge-tree choices,
// line samples and ray tests must take the oracle's branches.
#include "../../include/delta_ray_b200.h"
#include "dr_backward.cuh"
#include "dr_block_grad.cuh"

#include <cooperative_groups.h>
#include <cuda_bf16.h>

namespace cg = cooperative_groups;

// Resident blocks per SM (of 128 threads) of the persistent walk kernels,
// settable at build time for tuning sweeps.
#ifndef DR_TASKS_BLOCKS
#define DR_TASKS_BLOCKS 6
#endif
#ifndef DR_CONNECT_BLOCKS
#define DR_CONNECT_BLOCKS 8
#endif
// and of the line and side-radiance kernels (a sweep at the 640x480
// heightfield: radiance 3 / 4 / 6 / 8 blocks 264 / 249 / 223 / 234 ms per
// step; line 4 and 6 the same; connect 6 / 8 / 10: 458 / 436 / 516; the
// level walk 6 and 8 the same)
#ifndef DR_LINE_BLOCKS
#define DR_LINE_BLOCKS 4
#endif
#ifndef DR_RADIANCE_BLOCKS
#define DR_RADIANCE_BLOCKS 6
#endif

#define DR_ITEM_BUF 24
// One thread per shading point in [pt_begin, pt_end).  A point's items collect
// in a lane buffer; a full buffer reserves DR_ITEM_BUF slots with one atomic
// (points of large glossy scenes sample thousands of edges), and the last
// partial buffers of a warp share one atomic.
// A lane's buffer of sampled edges: a full buffer reserves DR_ITEM_BUF slots
// of the item queue with one atomic; flush_warp() (all lanes of a converged
// warp) writes the rest with one atomic per warp.
struct ItemWriter {
    const BackwardWorkspace &ws;
    int buf_p[DR_ITEM_BUF], buf_e[DR_ITEM_BUF], buf_j[DR_ITEM_BUF];
    float buf_w[DR_ITEM_BUF];
    uint8_t buf_c[DR_ITEM_BUF];
    int nb = 0;
    __device__ explicit ItemWriter(const BackwardWorkspace &w) : ws(w) {}
    __device__ void write(unsigned long long first, int cnt) {
        unsigned long long cap = (unsigned long long)ws.cap_items;
        if (first + (unsigned long long)cnt > cap) set_status(&ws.counters->status, DR_STATUS_ITEM_OVERFLOW);
        for (int k = 0; k < cnt; k++) {
            unsigned long long i = first + (unsigned long long)k;
            if (i >= cap) break;
            int4 it;
            it.x = buf_p[k];
            it.y = buf_e[k];
            it.z = buf_j[k];
            it.w = buf_c[k];
            ws.items[i] = it;
            ws.item_w[i] = buf_w[k];
        }
    }
    __device__ void add(int p, int tree, int ei, int j, float w, int code) {
        if (nb == DR_ITEM_BUF) {
            write(atomicAdd(&ws.counters->items, (unsigned long long)DR_ITEM_BUF), DR_ITEM_BUF);
            nb = 0;
        }
        buf_p[nb] = p;
        buf_e[nb] = (tree << 30) | ei;
        buf_j[nb] = j;
        buf_w[nb] = w;
        buf_c[nb] = (uint8_t)code;
        nb++;
    }
    __device__ void flush_warp() {
        __syncwarp();
        write(warp_reserve(&ws.counters->items, nb), nb);
        nb = 0;
    }
};

__device__ __forceinline__ EdgeProposal point_proposal(const BackwardWorkspace &ws, long long p) {
    EdgeProposal pr;
    pr.q = ws.proposal_q ? ws.proposal_q + 32 * (size_t)p : nullptr;
    pr.alpha = ws.proposal_alpha;
    pr.codes = ws.train_targets != nullptr;
    return pr;
}

// The points a traversal launch walks: pt_begin, pt_begin + pt_stride, ...
// below min(pt_end, the points the path stage pushed); returns their number.
__device__ __forceinline__ long long strided_points(const BackwardWorkspace &ws) {
    const long long n = min(min((long long)ws.counters->points, ws.cap_points), ws.pt_end);
    return n > ws.pt_begin ? (n - ws.pt_begin + ws.pt_stride - 1) / ws.pt_stride : 0;
}

// One thread per shading point in [pt_begin, pt_end) walks the point's trees
// (small trees: every point's walk is short).
// Adds each warp's node-visit count to a counter (every lane calls it).
__device__ __forceinline__ void add_visits(unsigned long long *counter, int visits) {
    unsigned long long v = (unsigned long long)visits;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(counter, v);
}

template <bool PROP>
__global__ void __launch_bounds__(128, 6) k_edge_traverse(DevScene s, uint64_t seed, BackwardWorkspace ws) {
    const long long m = strided_points(ws);
    long long stride = (long long)gridDim.x * blockDim.x;
    ItemWriter out(ws);
    int visits = 0;
    // warp-uniform loop: every lane of a warp takes the same number of trips
    for (long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < m; base += stride) {
        const long long k = base + (threadIdx.x & 31);
        const long long p = ws.pt_begin + k * ws.pt_stride;
        if (k < m) {
            PointRecord pt;
            pt.load(ws.pt + (size_t)p * DR_PT_WORDS);
            int cnt = 0;
            auto emit = [&](int tree, int ei, int j, float w, int code) {
                out.add((int)p, tree, ei, j, w, code);
                cnt++;
            };
            if (!traverse_point<PROP>(s, pt, point_seed(ws, pt.view, seed), emit, point_proposal(ws, p),
                                      (NoDefer *)nullptr, &visits))
                set_status(&ws.counters->status, DR_STATUS_STACK_OVERFLOW);
            if (ws.pt_items) ws.pt_items[p] = cnt;
        }
        out.flush_warp();
    }
    add_visits(&ws.counters->visits_walk, visits);
}

// Large trees, first stage: each point's walk stops DR_TASK_CUT levels below
// the roots and hands the subtrees there on as tasks (a lane buffers 8 and
// reserves their slots with one atomic; if the task queue is full, the lane
// walks them itself).  The node-keyed draws make the sampled edges the same
// as those of the one-pass walk.
#define DR_TASK_CUT 8
#define DR_TASK_BUF 8
template <bool PROP>
__global__ void __launch_bounds__(128, 4) k_edge_expand(DevScene s, uint64_t seed, BackwardWorkspace ws) {
    const long long m = strided_points(ws);
    long long stride = (long long)gridDim.x * blockDim.x;
    ItemWriter out(ws);
    int visits = 0;
    for (long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < m; base += stride) {
        const long long k = base + (threadIdx.x & 31);
        const long long p = ws.pt_begin + k * ws.pt_stride;
        if (k < m) {
            PointRecord pt;
            pt.load(ws.pt + (size_t)p * DR_PT_WORDS);
            const EdgeProposal pr = point_proposal(ws, p);
            int cnt = 0;
            auto emit = [&](int tree, int ei, int j, float w, int code) {
                out.add((int)p, tree, ei, j, w, code);
                cnt++;
            };
            EdgeTask tb[DR_TASK_BUF];
            int nt = 0;
            bool ok = true;
            // every reserved slot below the queue's capacity is written (the
            // second stage reads all of them); subtrees beyond it are walked here
            auto flush = [&]() {
                unsigned long long first = atomicAdd(&ws.counters->tasks, (unsigned long long)nt);
                for (int k = 0; k < nt; k++) {
                    if (first + (unsigned long long)k < (unsigned long long)ws.cap_tasks)
                        ws.tasks[first + k] = tb[k];
                    else
                        ok &= traverse_point_task<PROP>(s, pt, point_seed(ws, pt.view, seed), tb[k], emit, pr, &visits);
                }
                nt = 0;
            };
            auto defer = [&](int code, float bb, float c, float a, float l) {
                if (nt == DR_TASK_BUF) flush();
                tb[nt++] = EdgeTask{(int)p, code, bb, c, a, l};
            };
            ok &= traverse_point<PROP, DR_TASK_CUT>(s, pt, point_seed(ws, pt.view, seed), emit, pr, &defer, &visits);
            if (nt > 0) flush();
            if (!ok) set_status(&ws.counters->status, DR_STATUS_STACK_OVERFLOW);
            if (ws.pt_items) ws.pt_items[p] = cnt;  // the subtrees add theirs
        }
        out.flush_warp();
    }
    add_visits(&ws.counters->visits_walk, visits);
}

// Large trees, second stage: the handed-on subtrees, fetched one per lane.
// Subtree sizes vary by orders of magnitude, so a lane that finishes its walk
// takes the next task (lanes that need one share an atomic) while the other
// lanes of its warp keep stepping theirs: every step of the loop walks one
// node per busy lane.  A full item buffer reserves its slots with one atomic
// of its own; the partial buffers go out together at the end.
__device__ __forceinline__ long long next_task(unsigned long long *counter) {
    cg::coalesced_group g = cg::coalesced_threads();
    unsigned long long first = 0;
    if (g.thread_rank() == 0) first = atomicAdd(counter, (unsigned long long)g.size());
    return (long long)(g.shfl(first, 0) + g.thread_rank());
}

// Rounds (ws.task_rounds launches per chunk): the subtrees come from `in`
// (*in_n of them); with HAND, a walk that has taken ws.hand_steps steps with
// two or more subtrees pending hands the shallowest one (the largest) to
// `hand_q` (*hand_n) for the next round, so that no lane walks a long subtree
// alone at the end of the launch.  The last round hands nothing on.
template <bool PROP, bool HAND>
__global__ void __launch_bounds__(128, DR_TASKS_BLOCKS) k_edge_tasks(DevScene s, uint64_t seed, BackwardWorkspace ws,
                                                                   const EdgeTask *in, const unsigned long long *in_n,
                                                                   EdgeTask *hand_q, unsigned long long *hand_n) {
    const long long n = (long long)min(*in_n, (unsigned long long)ws.cap_tasks);
    ItemWriter out(ws);
    int visits = 0, point = 0, cnt = 0;
    bool ok = true;
    EdgeWalk<PROP> w;
    auto emit = [&](int ei, int key, float wt, int code) {
        if (wt != 0.f) {
            out.add(point, w.tree, ei, key, wt, code);
            cnt++;
        }
    };
    NoDefer nd;
    int steps = 0;
    while (true) {
        if (!w.busy()) {
            if (cnt > 0 && ws.pt_items) atomicAdd(ws.pt_items + point, cnt);
            cnt = 0;
            const long long k = next_task(&ws.counters->task_next);
            if (k >= n) break;
            const EdgeTask t = in[k];
            PointRecord pt;
            pt.load(ws.pt + (size_t)t.point * DR_PT_WORDS);
            point = t.point;
            start_point_task<PROP>(w, s, pt, point_seed(ws, pt.view, seed), t, point_proposal(ws, t.point));
            steps = 0;
        }
        w.step(emit, nd, &visits);
        ok &= w.ok;
        if (HAND && ++steps >= ws.hand_steps && w.n >= 2) {
            steps = 0;
            const unsigned long long slot = atomicAdd(hand_n, 1ull);
            if (slot < (unsigned long long)ws.cap_tasks) hand_q[slot] = w.take_bottom(point);
        }
    }
    if (!ok) set_status(&ws.counters->status, DR_STATUS_STACK_OVERFLOW);
    out.flush_warp();
    add_visits(&ws.counters->visits_tasks, visits);
}

// ---------------------------------------------------------------------------
// The subtrees walked level by level.  Each launch of k_edge_level takes one
// level of nodes of every handed-on subtree (a queue of EdgeTask, one node of
// one point's walk each), decides their children exactly as the depth-first
// walk does (node_children) and queues the children it walks: interior ones
// for the next level, leaves for k_edge_leaves.  Every lane of a warp works on
// a node of the same kind at the same point of the code (the depth-first
// walk's lanes ran 8-10 of 32 on average: leaves, interior nodes, task fetches
// and hand-offs in one loop), and no walk stack is kept.  What a node's
// decision needs of its shading point comes from the point's walk context
// (k_walk_ctx, 176 B), read from L2.  The node draws are keyed by node, so
// the sampled edges are those of the depth-first walk.

// Walk context of one point, DR_CTX_F4 float4: 0-4 the bound context (p, n,
// the frame around wi, the normal in it), 5 roughness, exponent, model, the
// light cone's cosine, 6 the cone's axis and the learned-descent flag,
// 7 the node draws' key (sample id, bounce) and the view, 8-10 the shading
// frame (the proposal's direction bins).

// The point's two walks start at the root of the tree its draw picks
// (traverse_edges: edge_tree.cpp:685-725): the root tasks of the cone and the
// all walk, with the root's bound and the tree's pick probability, go to the
// first level's queue (`tasks`), and the point's edge count starts at 0.
template <bool PROP>
__global__ void __launch_bounds__(128, 8) k_walk_ctx(DevScene s, uint64_t seed, BackwardWorkspace ws) {
    const long long m = strided_points(ws);
    const long long stride = (long long)gridDim.x * blockDim.x;
    // warp-uniform loop: the root tasks' append is warp-aggregated
    for (long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < m; base += stride) {
        const long long k = base + (threadIdx.x & 31);
        EdgeTask root;
        int nroot = 0;
        if (k < m) {
            const long long p = ws.pt_begin + k * ws.pt_stride;
            PointRecord pt;
            pt.load(ws.pt + (size_t)p * DR_PT_WORDS);
            // as start_point_task / start_subtree
            const SurfacePoint sp = pt.surface();
            const DevMaterial &mt = s.mats[material_of_tri(s, pt.tri)];
            const float dl = luminance(get_kd(s, mt, sp.uv)), sl = luminance(get_ks(s, mt, sp.uv));
            const float rough = get_rough(s, mt, sp.uv);
            const BoundCtx bc = bound_ctx(pt.wi, sp, dl, sl, rough, mt.model);
            const uint64_t pseed = point_seed(ws, pt.view, seed);
            if (dot(pt.wi, sp.f.n) >= 0.f && (s.num_nrm_nodes > 0 || s.num_sil_nodes > 0)) {
                // the tree pick draws after the point's edge sample, as traverse_point
                Rng prng;
                prng.init(pseed, kStreamEdgePoint, pt.sid, (uint32_t)pt.bounce);
                draw_edge(prng);
                int tree;
                float pmf = 1.f;
                if (s.num_nrm_nodes == 0) {
                    tree = 0;
                } else if (s.num_sil_nodes == 0) {
                    tree = 1;
                } else {
                    float ni = s.nrm_nodes[0].total_length, si = s.sil_nodes[0].total_length;
                    float np = ni / (ni + si), spm = si / (ni + si);
                    float u = prng.next();
                    if (u < np) {
                        tree = 1;
                        pmf = np;
                    } else {
                        tree = 0;
                        pmf = spm;
                    }
                }
                root.point = (int)p;
                root.code = tree << 29;
                root.bb = bsdf_bound((tree ? s.nrm_nodes : s.sil_nodes)[0], bc);
                root.cpmf = root.apmf = root.lpmf = pmf;
                nroot = 2;
            }
            if (ws.pt_items) ws.pt_items[p] = 0;  // the leaves add the point's edges
            const ConeSpec cone = light_cone(s, pt.light, sp.p);
            float learned = 0.f;
            if constexpr (PROP) {
                NodeRng r;
                r.seed = point_seed(ws, pt.view, seed);
                r.sid = pt.sid;
                r.bounce = (uint32_t)pt.bounce;
                learned = r.draw(1, DR_NODE_MIX_DRAW) < ws.proposal_alpha ? 1.f : 0.f;
            }
            const bool lobe = sl > 0.f;  // the frame around wi is set only with a specular lobe
            const Frame hf = lobe ? bc.hf : Frame{f3(0.f), f3(0.f), f3(0.f)};
            const float3 ln = lobe ? bc.ln : f3(0.f);
            float4 *o = ws.walk_ctx + (size_t)p * DR_CTX_F4;
            o[0] = make_float4(bc.p.x, bc.p.y, bc.p.z, bc.n.x);
            o[1] = make_float4(bc.n.y, bc.n.z, bc.dl, bc.sl);
            o[2] = make_float4(hf.t.x, hf.t.y, hf.t.z, hf.b.x);
            o[3] = make_float4(hf.b.y, hf.b.z, hf.n.x, hf.n.y);
            o[4] = make_float4(hf.n.z, ln.x, ln.y, ln.z);
            o[5] = make_float4(bc.rough, bc.expo, __int_as_float(bc.model), cone.cos_angle);
            o[6] = make_float4(cone.d.x, cone.d.y, cone.d.z, learned);
            o[7] = make_float4(__uint_as_float((uint32_t)pt.sid), __uint_as_float((uint32_t)(pt.sid >> 32)),
                               __uint_as_float((uint32_t)pt.bounce), __int_as_float(pt.view));
            if constexpr (PROP) {
                o[8] = make_float4(sp.f.t.x, sp.f.t.y, sp.f.t.z, sp.f.b.x);
                o[9] = make_float4(sp.f.b.y, sp.f.b.z, sp.f.n.x, sp.f.n.y);
                o[10] = make_float4(sp.f.n.z, 0.f, 0.f, 0.f);
            }
        }
        __syncwarp();
        // the cone walk's root (mode 0), then the all walk's (mode 1)
        const unsigned long long slot = warp_reserve(&ws.counters->tasks, nroot);
        for (int j = 0; j < nroot; j++) {
            if (slot + j >= (unsigned long long)ws.cap_tasks) {  // room for two per point: never short
                set_status(&ws.counters->status, DR_STATUS_STACK_OVERFLOW);
                break;
            }
            EdgeTask t = root;
            t.code |= j << 30;
            ws.tasks[slot + j] = t;
        }
    }
}

// A point's walk context: what node_children needs (`f` only with PROP).
struct WalkPoint {
    BoundCtx bc;
    ConeSpec cone;
    NodeRng rng;
    Frame f;
    bool learned;
};
template <bool PROP>
__device__ __forceinline__ WalkPoint load_walk_point(const BackwardWorkspace &ws, int point, uint64_t seed) {
    const float4 *c = ws.walk_ctx + (size_t)point * DR_CTX_F4;
    const float4 a = c[0], b = c[1], d2 = c[2], d3 = c[3], d4 = c[4], d5 = c[5], d6 = c[6], d7 = c[7];
    WalkPoint w;
    w.bc.p = f3(a.x, a.y, a.z);
    w.bc.n = f3(a.w, b.x, b.y);
    w.bc.dl = b.z;
    w.bc.sl = b.w;
    w.bc.hf.t = f3(d2.x, d2.y, d2.z);
    w.bc.hf.b = f3(d2.w, d3.x, d3.y);
    w.bc.hf.n = f3(d3.z, d3.w, d4.x);
    w.bc.ln = f3(d4.y, d4.z, d4.w);
    w.bc.rough = d5.x;
    w.bc.expo = d5.y;
    w.bc.model = __float_as_int(d5.z);
    w.cone.o = w.bc.p;
    w.cone.d = f3(d6.x, d6.y, d6.z);
    w.cone.cos_angle = d5.w;
    w.learned = d6.w != 0.f;
    w.rng.sid = (uint64_t)__float_as_uint(d7.x) | ((uint64_t)__float_as_uint(d7.y) << 32);
    w.rng.bounce = __float_as_uint(d7.z);
    w.rng.seed = point_seed(ws, __float_as_int(d7.w), seed);
    if constexpr (PROP) {
        const float4 f8 = c[8], f9 = c[9], f10 = c[10];
        w.f.t = f3(f8.x, f8.y, f8.z);
        w.f.b = f3(f8.w, f9.x, f9.y);
        w.f.n = f3(f9.z, f9.w, f10.x);
    } else {
        w.f.t = w.f.b = w.f.n = f3(0.f);
    }
    return w;
}

template <bool PROP> __device__ __forceinline__ EdgeTask child_task(int point, int hi, const EdgeItem<PROP> &c) {
    EdgeTask t;
    t.point = point;
    t.code = c.node | hi;
    t.bb = c.bb;
    t.cpmf = c.cpmf;
    t.apmf = c.apmf;
    t.lpmf = 0.f;
    if constexpr (PROP) t.lpmf = c.lpmf;
    return t;
}

// A subtree that found no room in a level's queue: the lane walks it depth
// first (its items through `spill`).  Out of line: the rare path keeps its
// registers and stack to itself.
template <bool PROP>
__device__ __noinline__ void walk_here(const DevScene &s, uint64_t seed, const BackwardWorkspace &ws, const EdgeTask &t,
                          ItemWriter &spill, int *visits, bool &ok) {
    PointRecord pt;
    pt.load(ws.pt + (size_t)t.point * DR_PT_WORDS);
    int cnt = 0;
    auto emit = [&](int tree, int ei, int j, float w, int code) {
        spill.add(t.point, tree, ei, j, w, code);
        cnt++;
    };
    ok &= traverse_point_task<PROP>(s, pt, point_seed(ws, pt.view, seed), t, emit, point_proposal(ws, t.point),
                                    visits);
    if (cnt > 0 && ws.pt_items) atomicAdd(ws.pt_items + t.point, cnt);
    atomicAdd(&ws.counters->spilled, 1ull);
}

// The class of a node in the level queues: 0 for nodes whose decision takes
// the exact bounds and the cone tests (the cone walk's, and the all walk's on
// the cone walk's path), 1 for the all walk's others (no cone tests; filtered
// bounds where they split).  Each class fills its own half of a queue, so that
// a warp's lanes mostly run the same code.  (Splitting instead by whether the
// node's children take filtered bounds was slower: 490-520 -> 586 ms per step
// at the 640x480 heightfield.)
template <bool PROP> __device__ __forceinline__ int node_class(int mode, const EdgeItem<PROP> &c) {
    return (mode == 0 || c.cpmf != 0.f) ? 0 : 1;
}

#ifndef DR_LEVEL_BLOCKS
#define DR_LEVEL_BLOCKS 8
#endif
// `in` holds in_n[0] nodes of class 0 from its start and (in_n1 != null)
// in_n1[0] of class 1 from its middle; out_n[c] counts the class-c nodes
// queued in `out`'s half c.
template <bool PROP>
__global__ void __launch_bounds__(128, DR_LEVEL_BLOCKS) k_edge_level(DevScene s, uint64_t seed, BackwardWorkspace ws,
                                                                   const EdgeTask *in, const unsigned long long *in_n,
                                                                   const unsigned long long *in_n1, EdgeTask *out,
                                                                   unsigned long long *out_n) {
    const unsigned long long half = (unsigned long long)ws.cap_tasks / 2;
    const long long n0 = (long long)min(*in_n, in_n1 ? half : (unsigned long long)ws.cap_tasks);
    const long long n = n0 + (in_n1 ? (long long)min(*in_n1, half) : 0);
    const long long stride = (long long)gridDim.x * blockDim.x;
    ItemWriter spill(ws);
    int visits = 0;
    bool ok = true;
    // warp-uniform loop: the queue appends are warp-aggregated
    for (long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += stride) {
        const long long i = base + (threadIdx.x & 31);
        EdgeTask kid[2], lf[2];
        int nk = 0, nl = 0, kc[2] = {0, 0};
        if (i < n) {
            const EdgeTask t = in[i < n0 ? i : (long long)half + (i - n0)];
            const int tree = (t.code >> 29) & 1, mode = (t.code >> 30) & 1, nid = t.code & DR_NODE_MASK;
            const DevEdgeNode *nodes = tree ? s.nrm_nodes : s.sil_nodes;
            const DevEdgeNode &node = nodes[nid];
            if (!(t.bb <= 0.f)) {
                if (node.nprims > 0) {
                    lf[nl++] = t;  // a leaf handed on as it is
                } else {
                    ++visits;
                    const WalkPoint w = load_walk_point<PROP>(ws, t.point, seed);
                    const EdgeItem<PROP> it = edge_item<PROP>(nid, t.bb, t.cpmf, t.apmf, t.lpmf);
                    ChildPick<PROP> c;
                    const EdgeProposal pr = point_proposal(ws, t.point);
                    if (node_children<PROP>(nodes, w.bc, w.cone, w.rng, pr, w.f, mode == 0, tree == 1,
                                            PROP && mode == 1 && w.learned, it, node, nid, c)) {
                        const int hi = (tree << 29) | (mode << 30);
                        if (c.push_l) {
                            if (c.l_leaf) {
                                lf[nl++] = child_task<PROP>(t.point, hi, c.left);
                            } else {
                                kc[nk] = node_class<PROP>(mode, c.left);
                                kid[nk++] = child_task<PROP>(t.point, hi, c.left);
                            }
                        }
                        if (c.push_r) {
                            if (c.r_leaf) {
                                lf[nl++] = child_task<PROP>(t.point, hi, c.right);
                            } else {
                                kc[nk] = node_class<PROP>(mode, c.right);
                                kid[nk++] = child_task<PROP>(t.point, hi, c.right);
                            }
                        }
                    }
                }
            }
        }
        __syncwarp();
        const int n1 = (nk > 0 && kc[0]) + (nk > 1 && kc[1]);
        unsigned long long ko[2];
        ko[0] = warp_reserve(out_n, nk - n1);
        ko[1] = warp_reserve(out_n + 1, n1);
        const unsigned long long kl = warp_reserve(&ws.counters->leaf_n, nl);
        for (int j = 0; j < nk; j++) {
            const unsigned long long slot = ko[kc[j]]++;
            if (slot < half) out[kc[j] ? half + slot : slot] = kid[j];
            else walk_here<PROP>(s, seed, ws, kid[j], spill, &visits, ok);
        }
        for (int j = 0; j < nl; j++) {
            if (kl + j < (unsigned long long)ws.cap_leaves) ws.leafq[kl + j] = lf[j];
            else walk_here<PROP>(s, seed, ws, lf[j], spill, &visits, ok);
        }
        spill.flush_warp();
    }
    if (!ok) set_status(&ws.counters->status, DR_STATUS_STACK_OVERFLOW);
    add_visits(&ws.counters->visits_tasks, visits);
}

// The leaves a level reached: each leaf's silhouette edges (the edge records'
// test) as items, weighted as EdgeWalk::leaf weighs them; the warp appends
// them together, one edge of every lane's leaf at a time.
template <bool PROP>
__global__ void __launch_bounds__(128, 8) k_edge_leaves(DevScene s, BackwardWorkspace ws) {
    const long long n = (long long)min(ws.counters->leaf_n, (unsigned long long)ws.cap_leaves);
    const long long stride = (long long)gridDim.x * blockDim.x;
    const unsigned long long cap = (unsigned long long)ws.cap_items;
    int visits = 0;
    for (long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += stride) {
        const long long i = base + (threadIdx.x & 31);
        int point = -1, tree = 0, mode = 0, off = 0, np = 0;
        float w = 0.f;
        float3 p = f3(0.f);
        Frame f;
        bool codes = false;
        if (i < n) {
            const EdgeTask t = ws.leafq[i];
            tree = (t.code >> 29) & 1;
            mode = (t.code >> 30) & 1;
            const DevEdgeNode &node = (tree ? s.nrm_nodes : s.sil_nodes)[t.code & DR_NODE_MASK];
            point = t.point;
            off = node.offset;
            np = node.nprims;
            ++visits;
            const float4 c0 = ws.walk_ctx[(size_t)point * DR_CTX_F4];
            p = f3(c0.x, c0.y, c0.z);
            float apmf = t.apmf;
            if constexpr (PROP) apmf = ws.proposal_alpha * t.lpmf + (1.f - ws.proposal_alpha) * t.apmf;
            const float denom = t.cpmf * t.cpmf + apmf * apmf;
            w = mode == 0 ? t.cpmf / denom : apmf / denom;
            if constexpr (PROP) {
                codes = ws.train_targets != nullptr;
                if (codes) {
                    const float4 *c = ws.walk_ctx + (size_t)point * DR_CTX_F4;
                    const float4 f8 = c[8], f9 = c[9], f10 = c[10];
                    f.t = f3(f8.x, f8.y, f8.z);
                    f.b = f3(f8.w, f9.x, f9.y);
                    f.n = f3(f9.z, f9.w, f10.x);
                }
            }
            if (w == 0.f) np = 0;  // no item of weight 0 is kept
        }
        const EdgeRec *recs = tree ? s.nrm_rec : s.sil_rec;
        const DevEdge *edges = tree ? s.nrm_edges : s.sil_edges;
        int cnt = 0;
        const int most = __reduce_max_sync(0xffffffffu, (unsigned)np);
        for (int k = 0; k < most; k++) {
            const int ei = off + k;
            const bool e = k < np && is_silhouette_rec(recs + ei, p);
            int code = 0;
            if constexpr (PROP)
                if (e && codes) code = dir_bin(f, 0.5f * (edge_v0(s, edges[ei]) + edge_v1(s, edges[ei])) - p);
            const unsigned long long slot = warp_reserve(&ws.counters->items, e ? 1 : 0);
            if (e) {
                if (slot < cap) {
                    ws.items[slot] = make_int4(point, (tree << 30) | ei, (mode << 27) | ei, code);
                    ws.item_w[slot] = w;
                } else {
                    set_status(&ws.counters->status, DR_STATUS_ITEM_OVERFLOW);
                }
                cnt++;
            }
        }
        if (ws.pt_items) {  // lanes of the same point add their counts together
            const unsigned grp = __match_any_sync(0xffffffffu, point);
            const unsigned sum = __reduce_add_sync(grp, (unsigned)cnt);
            if ((int)(threadIdx.x & 31) == __ffs(grp) - 1 && point >= 0 && sum > 0)
                atomicAdd(ws.pt_items + point, (int)sum);
        }
    }
    add_visits(&ws.counters->visits_tasks, visits);
}

// What follows an item's evaluation: the proposal's training target and the
// position adjoint (pushed back now in DR_DP_SUM mode, else keyed for the
// reference's "last edge" rule).
template <bool EXT, class G>
__device__ __forceinline__ void finish_item(const DevScene &s, const BackwardWorkspace &ws, const int4 &it,
                                            long long i, const PointRecord &pt, float3 dp, float mag, int W, int H,
                                            int spp, uint64_t seed, int dp_mode, G &bg) {
    if (EXT && ws.train_targets && mag > 0.f && it.x % ws.train_stride == 0 && it.x / ws.train_stride < ws.train_n) {
        // the proposal's training target: contribution magnitude per direction bin
        atomicAdd(ws.train_targets + 32 * (size_t)(it.x / ws.train_stride) + (it.w & 31), mag);
    }
    if (is_zero(dp)) return;
    if (dp_mode == DR_DP_SUM) {
        if (pt.bounce == 0) {
            const PointView v = point_view(ws, pt.view, W, H, spp, seed);
            propagate_dp<false>(s, pt, v.W, v.H, v.spp, v.seed, dp, bg, v.cam, v.cam_off);
        } else {  // after specular samples: summed here, the chain is traced by k_dp_propagate
            float *a = reinterpret_cast<float *>(ws.pt_last) + 4 * (size_t)it.x;
            atomicAdd(a, dp.x);
            atomicAdd(a + 1, dp.y);
            atomicAdd(a + 2, dp.z);
        }
    } else {
        ws.item_dp[3 * i] = dp.x;
        ws.item_dp[3 * i + 1] = dp.y;
        ws.item_dp[3 * i + 2] = dp.z;
        unsigned long long key = ((unsigned long long)(it.z + 1) << 32) | (unsigned long long)i;
        atomicMax(ws.pt_last + it.x, key);
    }
}

// Edge evaluation as a wavefront, each stage compacting what it keeps so that
// the next runs with full warps.  k_edge_line: the line sample of every item
// (silhouette test, LTC lobe, point on the edge) and the hits of its two rays
// on the edge's own faces; often most items end here (edges in the point's
// own plane, below the lobe's horizon or outside the clipped segment, rays
// that miss both faces).  The ray stage (k_edge_connect, k_edge_pairs): the
// occlusion of each survivor's rays and the tests on their hits; with direct
// lighting only, a sample neither of whose rays hits an emitter ends here too.
// k_edge_shade: the shading and the Jacobians of the rest.
//
// EXT: DR_FLAG_EDGE_LOBE_MIS or proposal training in use; GI: max_bounces > 1
// (the shade calls of the two sides); the launcher picks the variant.
// Each point's line-sample setup (line_setup: the point's edge draw, lobe
// pick and LTC transforms), the same for all of its thousands of edges: the
// line kernel reads it instead of setting it up per edge.  Layout, float4:
// 0-2 minv and 3-5 m with the lobe's pick probability, the draw's u, ok and
// the point's position in the last words of the two matrices' rows.
__global__ void __launch_bounds__(128, 8) k_line_ctx(DevScene s, uint64_t seed, BackwardWorkspace ws) {
    const long long n = min(min((long long)ws.counters->points, ws.cap_points), ws.pt_end);
    for (long long p = ws.pt_begin + (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n;
         p += (long long)gridDim.x * blockDim.x) {
        PointRecord pt;
        pt.load(ws.pt + (size_t)p * DR_PT_WORDS);
        Rng prng;
        prng.init(point_seed(ws, pt.view, seed), kStreamEdgePoint, pt.sid, (uint32_t)pt.bounce);
        const EdgeSample es = draw_edge(prng);
        const LineSetup ls = line_setup(s, es, pt.wi, pt.tri, pt.surface());
        const float *a = ls.minv.m, *b = ls.m.m;
        float4 *o = ws.line_ctx + (size_t)p * DR_LCTX_F4;
        o[0] = make_float4(a[0], a[1], a[2], a[3]);
        o[1] = make_float4(a[4], a[5], a[6], a[7]);
        o[2] = make_float4(a[8], b[0], b[1], b[2]);
        o[3] = make_float4(b[3], b[4], b[5], b[6]);
        o[4] = make_float4(b[7], b[8], ls.mpmf, es.u);
        o[5] = make_float4(ls.ok ? 1.f : 0.f, pt.p.x, pt.p.y, pt.p.z);
    }
}

template <bool EXT>
__global__ void __launch_bounds__(128, DR_LINE_BLOCKS) k_edge_line(DevScene s, uint64_t seed, BackwardWorkspace ws) {
    long long n = (long long)min(ws.counters->items, (unsigned long long)ws.cap_items);
    long long stride = (long long)gridDim.x * blockDim.x;
    // warp-uniform loop: the survivor append is warp-aggregated
    for (long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += stride) {
        long long i = base + (threadIdx.x & 31);
        EdgeLine el;
        bool ok = false;
        if (i < n) {
            int4 it = ws.items[i];
            const int tree = it.y >> 30, ei = it.y & ((1 << 30) - 1);
            PointRecord pt;
            if (!EXT && ws.line_ctx) {
                const float4 *c = ws.line_ctx + (size_t)it.x * DR_LCTX_F4;
                const float4 c0 = c[0], c1 = c[1], c2 = c[2], c3 = c[3], c4 = c[4], c5 = c[5];
                LineSetup ls;
                const float ma[9] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w, c2.x};
                const float mb[9] = {c2.y, c2.z, c2.w, c3.x, c3.y, c3.z, c3.w, c4.x, c4.y};
                for (int k = 0; k < 9; k++) {
                    ls.minv.m[k] = ma[k];
                    ls.m.m[k] = mb[k];
                }
                ls.mpmf = c4.z;
                EdgeSample es;
                es.u = c4.w;
                es.bsdf_component = 0.f;  // the lobe pick is in the setup
                pt.p = f3(c5.y, c5.z, c5.w);
                const DevEdge &edge = tree ? s.nrm_edges[ei] : s.sil_edges[ei];
                SurfacePoint unused;
                ok = c5.x != 0.f && line_sample_from<false>(s, ls, es, edge, pt.p, unused, f3(0.f), el,
                                                             (tree ? s.nrm_rec : s.sil_rec) + ei);
            } else {
                pt.load(ws.pt + (size_t)it.x * DR_PT_WORDS);
                ok = item_line<EXT>(s, pt, tree, ei, point_seed(ws, pt.view, seed), el);
            }
            if (ok) {
                // the connectivity test's first part: a sample neither of whose
                // rays hits one of the edge's faces is connected on no side
                // (three in four samples of a large mesh end here)
                const DevEdge &edge = tree ? s.nrm_edges[ei] : s.sil_edges[ei];
                float3 sdir, rdir, ldir;
                edge_side_dirs(el, edge_v0(s, edge), edge_v1(s, edge), pt.p, sdir, rdir, ldir);
                Hit fr, fl;
                hit_faces_pair(s, edge, pt.p, rdir, ldir, 1e-3f, fr, fl);
                ok = fr.tri >= 0 || fl.tri >= 0;
            }
        }
        __syncwarp();
        unsigned long long slot = warp_reserve(&ws.counters->survivors, ok ? 1 : 0);
        if (ok) {
            ws.survivors[2 * slot] = make_float4(__int_as_float((int)i), el.sample_p.x, el.sample_p.y, el.sample_p.z);
            ws.survivors[2 * slot + 1] = make_float4(el.mwt.x, el.mwt.y, el.mwt.z, el.q);
        }
    }
}

// The ray stage of an LBVH scene in two kernels.  k_edge_connect decides
// each line sample's connectivity (the edge's faces and one or two bounded
// occlusion walks; most samples end here) and queues the few that go on;
// k_edge_pairs traces the other side's closest hit of those and runs the
// remaining tests.  Walk lengths vary widely, so both fetch their work one
// item per lane (a lane takes the next as soon as it is done) rather than a
// warp's worth at a time.
__global__ void __launch_bounds__(128, DR_CONNECT_BLOCKS) k_edge_connect(DevScene s, BackwardWorkspace ws) {
    const long long n = (long long)min(ws.counters->survivors, (unsigned long long)ws.cap_items);
    // A state machine per lane, stepped by the whole warp.  When at least
    // half the warp has no walk (or none has), those lanes take line samples
    // together (a sample's setup and face tests cost about ten walk steps)
    // until each has one that needs an occlusion walk; otherwise every
    // walking lane takes one node, at the same point of the code.  (Lanes
    // that ran their walks to the end before taking the next sample, and
    // lanes that took one as soon as they were idle, left the warp split
    // into groups issuing on their own: 5.1 and 3.8 of 32 lanes active.)
    long long k = 0;
    int phase = 0;  // 0 no walk, 1 walking the right ray, 2 walking the left ray
    bool more = true, cr = false;
    float3 p = f3(0.f), rdir = f3(0.f), ldir = f3(0.f);
    Hit fr, fl;
    fr.tri = fl.tri = -1;
    fr.t = fl.t = 0.f;
    BeforeWalk w;
    auto candidate = [&](int side, int face) {
        const long long j = next_task(&ws.counters->cands);
        ws.hits[j] = make_int4((int)k, face, side, 0);
    };
    while (true) {
        const unsigned walking = __ballot_sync(0xffffffffu, phase != 0);
        const unsigned idle = __ballot_sync(0xffffffffu, phase == 0 && more);
        if (walking == 0 && idle == 0) break;  // every lane's queue has ended
        const bool fetch = idle != 0 && (__popc(idle) >= 16 || walking == 0);
        while (fetch && phase == 0 && more) {
            k = next_task(&ws.counters->ray_next);
            if (k >= n) {
                more = false;
                break;
            }
            const float4 a = ws.survivors[2 * k];
            const int4 it = ws.items[__float_as_int(a.x)];
            const float *pw = ws.pt + (size_t)it.x * DR_PT_WORDS;  // the point's position: words 0-2
            const int tree = it.y >> 30, ei = it.y & ((1 << 30) - 1);
            const DevEdge &edge = tree ? s.nrm_edges[ei] : s.sil_edges[ei];
            p = f3(pw[0], pw[1], pw[2]);
            EdgeLine el;
            el.sample_p = f3(a.y, a.z, a.w);
            float3 sdir;
            edge_side_dirs(el, edge_v0(s, edge), edge_v1(s, edge), p, sdir, rdir, ldir);
            // the connectivity test of edge_connect_bvh, its walks stepped below
            hit_faces_pair(s, edge, p, rdir, ldir, 1e-3f, fr, fl);
            if (fr.tri >= 0) {
                w.begin(s.bvh_root, p, rdir, 1e-3f, fr.t, fr.tri);
                phase = 1;
            } else if (fl.tri >= 0) {
                cr = false;
                w.begin(s.bvh_root, p, ldir, 1e-3f, fl.t, fl.tri);
                phase = 2;
            }
        }
        if (fetch || phase == 0) continue;
        const int r = w.step(s.bvh_nodes, s.bvh_wide, s.bvh_tris);
        if (r == 0) continue;
        if (phase == 1) {
            cr = r == 2;  // no triangle ahead of the right face hit
            if (fl.tri >= 0) {  // the left side decides (both connected, or neither, ends the sample)
                w.begin(s.bvh_root, p, ldir, 1e-3f, fl.t, fl.tri);
                phase = 2;
            } else {
                if (cr) candidate(0, fr.tri);  // the left ray hits no face: not connected
                phase = 0;
            }
        } else {
            const bool cl = r == 2;
            if (cr != cl) candidate(cr ? 0 : 1, cr ? fr.tri : fl.tri);
            phase = 0;
        }
    }
}

template <bool DIRECT>
__global__ void __launch_bounds__(128, 4) k_edge_pairs(DevScene s, BackwardWorkspace ws) {
    const long long n = (long long)min(ws.counters->cands, (unsigned long long)ws.cap_items);
    while (true) {
        const long long j = next_task(&ws.counters->pair_next);
        if (j >= n) break;
        const int4 c = ws.hits[j];
        const float4 a = ws.survivors[2 * (long long)c.x];
        const int4 it = ws.items[__float_as_int(a.x)];
        // the point's position and triangle: words 0-2 and 17 of its record
        const float *w = ws.pt + (size_t)it.x * DR_PT_WORDS;
        const int tree = it.y >> 30, ei = it.y & ((1 << 30) - 1);
        const DevEdge &edge = tree ? s.nrm_edges[ei] : s.sil_edges[ei];
        const float3 p = f3(w[0], w[1], w[2]);
        EdgeLine el;
        el.sample_p = f3(a.y, a.z, a.w);
        float3 sdir, rdir, ldir;
        edge_side_dirs(el, edge_v0(s, edge), edge_v1(s, edge), p, sdir, rdir, ldir);
        EdgeHits eh;
        const bool ok = edge_rays_rest(s, dr_f2i(w[17]), p, rdir, ldir, c.z, c.y, DIRECT, eh);
        ws.hits[j] = make_int4(c.x, ok ? eh.r : -1, ok ? eh.l : -1, ok ? 1 : 0);
        if (ok) next_task(&ws.counters->hits);  // the count of kept samples
    }
}

// Scenes traced by testing every triangle (at most DR_LINEAR_TRIS): the rays
// are cheap, so the line sample and its rays run in one kernel without the
// survivor queue in between; a kept sample's survivor and hit records go to
// one slot (hits[slot].x = slot), which k_edge_shade reads as it does the
// records of the ray stage.
template <bool EXT, bool DIRECT>
__global__ void __launch_bounds__(128, 8) k_edge_line_rays(DevScene s, uint64_t seed, BackwardWorkspace ws) {
    long long n = (long long)min(ws.counters->items, (unsigned long long)ws.cap_items);
    long long stride = (long long)gridDim.x * blockDim.x;
    // warp-uniform loop: the append is warp-aggregated
    for (long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += stride) {
        long long i = base + (threadIdx.x & 31);
        EdgeLine el;
        EdgeHits eh;
        bool ok = false;
        if (i < n) {
            int4 it = ws.items[i];
            PointRecord pt;
            pt.load(ws.pt + (size_t)it.x * DR_PT_WORDS);
            int tree = it.y >> 30, ei = it.y & ((1 << 30) - 1);
            ok = item_line<EXT>(s, pt, tree, ei, point_seed(ws, pt.view, seed), el);
            if (ok) {
                const DevEdge &edge = tree ? s.nrm_edges[ei] : s.sil_edges[ei];
                ok = edge_rays(s, el, edge, pt.tri, pt.p, DIRECT, eh);
            }
        }
        __syncwarp();
        unsigned long long slot = warp_reserve(&ws.counters->cands, ok ? 1 : 0);
        if (ok) {
            ws.survivors[2 * slot] = make_float4(__int_as_float((int)i), el.sample_p.x, el.sample_p.y, el.sample_p.z);
            ws.survivors[2 * slot + 1] = make_float4(el.mwt.x, el.mwt.y, el.mwt.z, el.q);
            ws.hits[slot] = make_int4((int)slot, eh.r, eh.l, 1);
            next_task(&ws.counters->hits);  // the count of kept samples
        }
    }
}

// More than one bounce: the two sides' radiance of every kept sample (the
// multi-bounce shading) in a kernel of its own, [2 h] and [2 h + 1] of
// ws.side_rad; k_edge_shade then runs without the path-tracing code, whose
// size made the fused kernel wait on instruction fetches.
__global__ void __launch_bounds__(128, DR_RADIANCE_BLOCKS) k_edge_radiance(DevScene s, int B, uint64_t seed,
                                                                    BackwardWorkspace ws) {
    long long n = (long long)min(ws.counters->cands, (unsigned long long)ws.cap_items);
    for (long long h = (long long)blockIdx.x * blockDim.x + threadIdx.x; h < n; h += (long long)gridDim.x * blockDim.x) {
        int4 hr = ws.hits[h];
        if (hr.w == 0) continue;
        EdgeHits eh;
        eh.r = hr.y;
        eh.l = hr.z;
        float4 a = ws.survivors[2 * (long long)hr.x];
        long long i = __float_as_int(a.x);
        EdgeLine el;
        el.sample_p = f3(a.y, a.z, a.w);
        int4 it = ws.items[i];
        PointRecord pt;
        pt.load(ws.pt + (size_t)it.x * DR_PT_WORDS);
        float3 shr, shl;
        item_side_radiance(s, pt, it.y >> 30, it.y & ((1 << 30) - 1), it.z, B, point_seed(ws, pt.view, seed), el, eh,
                           shr, shl);
        ws.side_rad[2 * h] = make_float4(shr.x, shr.y, shr.z, shl.x);
        ws.side_rad[2 * h + 1] = make_float4(shl.y, shl.z, 0.f, 0.f);
    }
}

// PRE: the sides' radiance comes from k_edge_radiance.
template <bool EXT, bool GI, bool PRE>
__global__ void __launch_bounds__(128, 4) k_edge_shade(DevScene s, int W, int H, int spp, int B, uint64_t seed,
                                                    int dp_mode, float *grad, BackwardWorkspace ws, GradCacheCfg cfg) {
    extern __shared__ float sm[];
    BlockGrad bg = block_grad_begin(sm, grad, cfg);
    long long n = (long long)min(ws.counters->cands, (unsigned long long)ws.cap_items);
    for (long long h = (long long)blockIdx.x * blockDim.x + threadIdx.x; h < n; h += (long long)gridDim.x * blockDim.x) {
        int4 hr = ws.hits[h];
        if (hr.w == 0) continue;  // a candidate the ray stage dropped
        EdgeHits eh;
        eh.r = hr.y;
        eh.l = hr.z;
        long long k = hr.x;
        float4 a = ws.survivors[2 * k], b = ws.survivors[2 * k + 1];
        long long i = __float_as_int(a.x);
        EdgeLine el;
        el.sample_p = f3(a.y, a.z, a.w);
        el.mwt = f3(b.x, b.y, b.z);
        el.q = b.w;
        int4 it = ws.items[i];
        PointRecord pt;
        pt.load(ws.pt + (size_t)it.x * DR_PT_WORDS);
        int tree = it.y >> 30, ei = it.y & ((1 << 30) - 1);
        const PointView v = point_view(ws, pt.view, W, H, spp, seed);
        float mag = 0.f;
        float3 dp;
        if constexpr (PRE) {
            const float4 r0 = ws.side_rad[2 * h], r1 = ws.side_rad[2 * h + 1];
            const float3 rad[2] = {f3(r0.x, r0.y, r0.z), f3(r0.w, r1.x, r1.y)};
            dp = item_shade<EXT, GI, BlockGrad, true>(s, pt, tree, ei, it.z, ws.item_w[i], v.spp, B, v.seed, bg, &mag,
                                                     el, &eh, rad);
        } else {
            dp = item_shade<EXT, GI>(s, pt, tree, ei, it.z, ws.item_w[i], v.spp, B, v.seed, bg, &mag, el, &eh);
        }
        finish_item<EXT>(s, ws, it, i, pt, dp, mag, W, H, spp, seed, dp_mode, bg);
    }
    block_grad_flush(bg);
}

// Primary edges (delta_ray.cpp:1478-1522) in two kernels: k_primary_shade
// samples the edge point and shades the camera rays on its two sides (the
// code of a forward path), k_primary_grad redraws the sample and turns the
// color difference into the scene and camera gradients.
template <int BMAX>
__global__ void __launch_bounds__(128, 6) k_primary_shade(DevScene s, int B, uint64_t seed, long long i0, long long n,
                                                       float4 *out) {
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        out[k] = primary_shade_item<BMAX>(s, i0 + k, B, seed);
}

__global__ void __launch_bounds__(128, 8) k_primary_grad(DevScene s, int W, int H, int spp, uint64_t seed,
                                                      const float *d_image, long long i0, long long n,
                                                      const float4 *in, float *grad, GradCacheCfg cfg) {
    extern __shared__ float sm[];
    BlockGradWarp bg;
    static_cast<BlockGrad &>(bg) = block_grad_begin(sm, grad, cfg);
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        primary_grad_item(s, i0 + k, W, H, spp, seed, d_image, in[k], bg);
    block_grad_flush(bg);
}

__global__ void k_add_count(unsigned long long *dst, const unsigned long long *src, unsigned long long cap) {
    *dst += *src < cap ? *src : cap;
}

// *dst += min(*src, cap) on the device (the entries a queue received)
cudaError_t dr_launch_accumulate_count(unsigned long long *dst, const unsigned long long *src, long long cap,
                                       cudaStream_t st) {
    k_add_count<<<1, 1, 0, st>>>(dst, src, (unsigned long long)cap);
    return cudaGetLastError();
}

__global__ void k_edge_records(DevScene s, const DevEdge *edges, int n, EdgeRec *out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = edge_record(s, edges[i]);
}

cudaError_t dr_launch_edge_records(const DevScene &s, const DevEdge *edges, int n, EdgeRec *out, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    k_edge_records<<<(n + 255) / 256, 256, 0, st>>>(s, edges, n, out);
    return cudaGetLastError();
}

// Edges sampled per bucket of points: bucket b sums pt_items over points
// [b P / nb, (b + 1) P / nb).
__global__ void k_item_buckets(const int *pt_items, long long P, int nb, unsigned long long *out) {
    const int b = blockIdx.x;
    const long long p0 = (long long)b * P / nb, p1 = (long long)(b + 1) * P / nb;
    unsigned long long sum = 0;
    for (long long p = p0 + threadIdx.x; p < p1; p += blockDim.x) sum += (unsigned long long)(unsigned)pt_items[p];
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    __shared__ unsigned long long part[8];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) t += part[i];
        out[b] = t;
    }
}

cudaError_t dr_launch_item_buckets(const int *pt_items, long long P, int nb, unsigned long long *out,
                                   cudaStream_t st) {
    if (nb <= 0) return cudaSuccess;
    k_item_buckets<<<nb, 256, 0, st>>>(pt_items, P, nb, out);
    return cudaGetLastError();
}

cudaError_t dr_launch_edge_traverse(const DevScene &s, uint64_t seed, const BackwardWorkspace &ws, int num_sms,
                                    cudaStream_t st, int *launches, StageTimer *timer) {
    const bool prop = ws.proposal_q != nullptr;
    if (ws.tasks && s.split_traversal) {
        cudaError_t e = cudaMemsetAsync(&ws.counters->tasks, 0, sizeof(unsigned long long), st);
        if (e == cudaSuccess) e = cudaMemsetAsync(&ws.counters->handed_total, 0, sizeof(unsigned long long), st);
        if (e != cudaSuccess) return e;
        if (ws.level_walk && ws.walk_ctx && ws.leafq && ws.tasks2) {
            // the walks level by level from the roots: ping-pong between the
            // two queues, each level's leaves after it; the host looks every
            // 8 levels whether a level queued nothing (a walk ends within its
            // tree's depth, a few dozen levels)
            if (prop) k_walk_ctx<true><<<stage_grid(num_sms), 128, 0, st>>>(s, seed, ws);
            else k_walk_ctx<false><<<stage_grid(num_sms), 128, 0, st>>>(s, seed, ws);
            timer->mark(st, "k_walk_ctx");
            *launches += 1;
            // the roots fill `tasks` from its start; the levels fill their
            // queues by class
            const EdgeTask *in = ws.tasks;
            const unsigned long long *in_n = &ws.counters->tasks, *in_n1 = nullptr;
            for (int level = 0;; level++) {
                EdgeTask *out = (level & 1) ? ws.tasks : ws.tasks2;
                unsigned long long *out_n = ws.counters->level_n[level & 1];
                e = cudaMemsetAsync(out_n, 0, 2 * sizeof(unsigned long long), st);
                if (e == cudaSuccess) e = cudaMemsetAsync(&ws.counters->leaf_n, 0, sizeof(unsigned long long), st);
                if (e != cudaSuccess) return e;
                if (prop)
                    k_edge_level<true><<<num_sms * DR_LEVEL_BLOCKS, 128, 0, st>>>(s, seed, ws, in, in_n, in_n1, out, out_n);
                else
                    k_edge_level<false><<<num_sms * DR_LEVEL_BLOCKS, 128, 0, st>>>(s, seed, ws, in, in_n, in_n1, out, out_n);
                timer->mark(st, "k_edge_level");
                if (prop) k_edge_leaves<true><<<num_sms * 8, 128, 0, st>>>(s, ws);
                else k_edge_leaves<false><<<num_sms * 8, 128, 0, st>>>(s, ws);
                timer->mark(st, "k_edge_leaves");
                *launches += 2;
                in = out;
                in_n = out_n;
                in_n1 = out_n + 1;
                if ((level & 7) == 7) {
                    unsigned long long left[2] = {0, 0};
                    e = cudaMemcpyAsync(left, in_n, sizeof(left), cudaMemcpyDeviceToHost, st);
                    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
                    if (e != cudaSuccess) return e;
                    if (left[0] + left[1] == 0) break;
                    // node ids have 27 bits: no tree is deeper than that
                    if (level >= 4096) return cudaErrorInvalidValue;
                }
            }
            *launches += 1;
            return cudaGetLastError();
        }
        if (prop) k_edge_expand<true><<<stage_grid(num_sms), 128, 0, st>>>(s, seed, ws);
        else k_edge_expand<false><<<stage_grid(num_sms), 128, 0, st>>>(s, seed, ws);
        timer->mark(st, "k_edge_expand");
        // the item count of the first stage (the roofline's work counts)
        e = cudaMemcpyAsync(&ws.counters->items_expand, &ws.counters->items, sizeof(unsigned long long),
                            cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return e;
        // the subtrees in rounds: the first stage's, then those handed on
        // (ping-pong between the two queues); one round without a second queue
        const int rounds = ws.tasks2 ? ws.task_rounds : 1;
        const EdgeTask *in = ws.tasks;
        const unsigned long long *in_n = &ws.counters->tasks;
        for (int r = 0; r < rounds; r++) {
            EdgeTask *out = (r & 1) ? ws.tasks : ws.tasks2;
            unsigned long long *out_n = &ws.counters->handed[r & 1];
            e = cudaMemsetAsync(&ws.counters->task_next, 0, sizeof(unsigned long long), st);
            if (e == cudaSuccess) e = cudaMemsetAsync(out_n, 0, sizeof(unsigned long long), st);
            if (e != cudaSuccess) return e;
            const bool hand = r + 1 < rounds;
            auto k = prop ? (hand ? k_edge_tasks<true, true> : k_edge_tasks<true, false>)
                          : (hand ? k_edge_tasks<false, true> : k_edge_tasks<false, false>);
            k<<<stage_grid(num_sms), 128, 0, st>>>(s, seed, ws, in, in_n, out, out_n);
            timer->mark(st, "k_edge_tasks");
            *launches += 1;
            if (hand) {
                e = dr_launch_accumulate_count(&ws.counters->handed_total, out_n, ws.cap_tasks, st);
                if (e != cudaSuccess) return e;
                *launches += 1;
            }
            in = out;
            in_n = out_n;
        }
        *launches += 1;
        return cudaGetLastError();
    }
    if (prop) k_edge_traverse<true><<<stage_grid(num_sms), 128, 0, st>>>(s, seed, ws);
    else k_edge_traverse<false><<<stage_grid(num_sms), 128, 0, st>>>(s, seed, ws);
    timer->mark(st, "k_edge_traverse");
    *launches += 1;
    return cudaGetLastError();
}

cudaError_t dr_launch_edge_eval(const DevScene &s, int W, int H, int spp, int B, uint64_t seed, int dp_mode,
                                float *grad, const BackwardWorkspace &ws, const GradCacheCfg &cfg, int num_sms,
                                cudaStream_t st, int *launches, StageTimer *timer) {
    size_t smem = sizeof(float) * (size_t)(cfg.head + cfg.tail_len);
    const bool ext = s.edge_lobe_mis || ws.train_targets;
    const int grid = stage_grid(num_sms);
    // the survivor and hit counters (adjacent) and those of the ray stage
    cudaError_t e = cudaMemsetAsync(&ws.counters->survivors, 0, 2 * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(&ws.counters->ray_next, 0, 3 * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    if (s.num_tris <= DR_LINEAR_TRIS) {
        auto line_rays = ext ? (B > 1 ? k_edge_line_rays<true, false> : k_edge_line_rays<true, true>)
                             : (B > 1 ? k_edge_line_rays<false, false> : k_edge_line_rays<false, true>);
        line_rays<<<grid, 128, 0, st>>>(s, seed, ws);
        timer->mark(st, "k_edge_line_rays");
        *launches -= 1;
    } else {
        if (!ext && ws.line_ctx) {
            k_line_ctx<<<grid, 128, 0, st>>>(s, seed, ws);
            timer->mark(st, "k_line_ctx");
            *launches += 1;
        }
        if (ext) k_edge_line<true><<<grid, 128, 0, st>>>(s, seed, ws);
        else k_edge_line<false><<<grid, 128, 0, st>>>(s, seed, ws);
        timer->mark(st, "k_edge_line");
        k_edge_connect<<<grid, 128, 0, st>>>(s, ws);
        timer->mark(st, "k_edge_connect");
        if (B > 1) k_edge_pairs<false><<<grid, 128, 0, st>>>(s, ws);
        else k_edge_pairs<true><<<grid, 128, 0, st>>>(s, ws);
        timer->mark(st, "k_edge_pairs");
        *launches += 1;
    }
    const bool pre = B > 1 && ws.side_rad != nullptr;
    if (pre) {
        k_edge_radiance<<<grid, 128, 0, st>>>(s, B, seed, ws);
        timer->mark(st, "k_edge_radiance");
        *launches += 1;
    }
    auto shade = ext ? (B > 1 ? (pre ? k_edge_shade<true, true, true> : k_edge_shade<true, true, false>)
                              : k_edge_shade<true, false, false>)
                     : (B > 1 ? (pre ? k_edge_shade<false, true, true> : k_edge_shade<false, true, false>)
                              : k_edge_shade<false, false, false>);
    shade<<<grid, 128, smem, st>>>(s, W, H, spp, B, seed, dp_mode, grad, ws, cfg);
    timer->mark(st, "k_edge_shade");
    *launches += 3;
    return cudaGetLastError();
}

cudaError_t dr_launch_primary_edges(const DevScene &s, int W, int H, int spp, int B, uint64_t seed,
                                    const float *d_image, long long n, float *grad, const GradCacheCfg &cfg,
                                    float4 *scratch, long long cap, int num_sms, cudaStream_t st, int *launches,
                                    StageTimer *timer) {
    const int bs = 128;
    size_t smem = sizeof(float) * (size_t)(cfg.head + cfg.tail_len);
    auto shade = B == 1 ? k_primary_shade<1> : k_primary_shade<(1 << 30)>;
    for (long long i0 = 0; i0 < n; i0 += cap) {
        long long m = std::min(cap, n - i0);
        int nb = (int)std::min<long long>(blocks_for(m, bs), (long long)stage_grid(num_sms) * 4);
        shade<<<nb, bs, 0, st>>>(s, B, seed, i0, m, scratch);
        timer->mark(st, "k_primary_shade");
        k_primary_grad<<<nb, bs, smem, st>>>(s, W, H, spp, seed, d_image, i0, m, scratch, grad, cfg);
        timer->mark(st, "k_primary_grad");
        *launches += 2;
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// The learned proposal's inputs of each shading point: position normalised to
// the scene bounds, shading normal, roughness, incoming direction.
__global__ void k_proposal_features(DevScene s, BackwardWorkspace ws, long long n, float3 c, float3 ih,
                                    __nv_bfloat16 *x, __nv_bfloat16 *xt) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    PointRecord pt;
    pt.load(ws.pt + (size_t)p * DR_PT_WORDS);
    float rough = get_rough(s, s.mats[material_of_tri(s, pt.tri)], pt.uv);
    float f[16] = {(pt.p.x - c.x) * ih.x, (pt.p.y - c.y) * ih.y, (pt.p.z - c.z) * ih.z, pt.n.x, pt.n.y, pt.n.z,
                   rough, pt.wi.x, pt.wi.y, pt.wi.z, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    __nv_bfloat162 h[8];
    for (int k = 0; k < 8; k++) h[k] = __floats2bfloat162_rn(f[2 * k], f[2 * k + 1]);
    uint4 *dst = reinterpret_cast<uint4 *>(x + 16 * (size_t)p);
    dst[0] = reinterpret_cast<uint4 *>(h)[0];
    dst[1] = reinterpret_cast<uint4 *>(h)[1];
    if (xt && p % ws.train_stride == 0 && p / ws.train_stride < ws.train_n) {
        uint4 *dt = reinterpret_cast<uint4 *>(xt + 16 * (size_t)(p / ws.train_stride));
        dt[0] = reinterpret_cast<uint4 *>(h)[0];
        dt[1] = reinterpret_cast<uint4 *>(h)[1];
    }
}

cudaError_t dr_launch_proposal_features(const DevScene &s, const BackwardWorkspace &ws, long long n, float3 c,
                                        float3 ih, void *x, void *xt, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    k_proposal_features<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(s, ws, n, c, ih, (__nv_bfloat16 *)x,
                                                                      (__nv_bfloat16 *)xt);
    return cudaGetLastError();
}

// Loads every kernel of the edge half that a backward call can launch.  CUDA
// loads a kernel lazily, at its first launch, and the load takes device
// memory for its code; dr_scene_create calls this so that a later
// dr_render_backward_noalloc call finds its kernels loaded.
cudaError_t dr_preload_edge_kernels() {
    const void *k[] = {
        (const void *)k_edge_traverse<false>, (const void *)k_edge_traverse<true>,
        (const void *)k_edge_expand<false>, (const void *)k_edge_expand<true>,
        (const void *)k_edge_tasks<false, false>, (const void *)k_edge_tasks<false, true>,
        (const void *)k_edge_tasks<true, false>, (const void *)k_edge_tasks<true, true>,
        (const void *)k_walk_ctx<false>, (const void *)k_walk_ctx<true>,
        (const void *)k_edge_level<false>, (const void *)k_edge_level<true>,
        (const void *)k_edge_leaves<false>, (const void *)k_edge_leaves<true>,
        (const void *)k_edge_line_rays<false, false>, (const void *)k_edge_line_rays<false, true>,
        (const void *)k_edge_line_rays<true, false>, (const void *)k_edge_line_rays<true, true>,
        (const void *)k_edge_line<false>, (const void *)k_edge_line<true>, (const void *)k_line_ctx,
        (const void *)k_edge_connect, (const void *)k_edge_pairs<false>, (const void *)k_edge_pairs<true>,
        (const void *)k_edge_radiance,
        (const void *)k_edge_shade<false, false, false>, (const void *)k_edge_shade<false, true, false>,
        (const void *)k_edge_shade<false, true, true>, (const void *)k_edge_shade<true, false, false>,
        (const void *)k_edge_shade<true, true, false>, (const void *)k_edge_shade<true, true, true>,
        (const void *)k_primary_shade<1>, (const void *)k_primary_shade<(1 << 30)>,
        (const void *)k_primary_grad, (const void *)k_add_count, (const void *)k_item_buckets,
    };
    for (const void *f : k) {
        cudaFuncAttributes a;
        const cudaError_t e = cudaFuncGetAttributes(&a, f);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}
