// GPU build of a scene's edge data: the unique edges of the meshes
// (scene.cpp:54-97), their filter and split into the silhouette and normal
// sets (scene.cpp:76-97, edge_tree.cpp:263-316), the median-split edge trees
// (edge_tree.cpp:49-261) and the primary-edge sampler over camera silhouettes
// (edge_tree.cpp:263-328).  Large scenes build here; small ones on the host
// (dr_host_scene.h), with the same results.
//
// Edges.  Every triangle side becomes a 64-bit key (lower, higher global
// vertex id) with the triangle as value; a stable radix sort groups equal
// keys in (shape, triangle, side) order, as the reference's std::map visits
// them: a run's first triangle is f0, its last f1 (-1 for a run of one).
//
// Trees.  One level of the tree at a time: each node's range of positions in
// the permutation `perm` is reduced (boxes as total-order minima and maxima,
// the cone axis's normal sum in exact fixed point: dr_edge_rules.h), the
// split dimension chosen, and one stable radix sort over all positions,
// keyed by (node start, split coordinate), orders every splitting node's
// range; its two halves are the children.  Leaves keep their positions
// (key = position).  Subtree sizes and total lengths then go bottom up,
// depth-first indices top down, and the nodes are written in the reference's
// flattened layout (flatten_bvh, edge_tree.cpp:175-205).  The result equals
// the host build of the same rule.
#include <cub/cub.cuh>

#include <algorithm>
#include <utility>
#include <vector>

#include "dr_edge_rules.h"
#include "dr_edges.cuh"
#include "dr_kernels.h"

namespace {

constexpr int kBS = 256;
inline int nblocks(long long n, int bs = kBS) { return (int)std::max<long long>(1, (n + bs - 1) / bs); }
inline int bits_for(long long n) {
    int b = 1;
    while ((1ll << b) < n) b++;
    return b;
}

// ---------------------------------------------------------------- edges ---

__global__ void k_side_keys(const int4 *tri, int ntri, int vbits, unsigned long long *keys, int *vals) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntri) return;
    int4 tr = tri[t];
    int v[3] = {tr.x, tr.y, tr.z};
    for (int k = 0; k < 3; k++) {
        int a = v[k], b = v[(k + 1) % 3];
        if (a > b) {
            int c = a;
            a = b;
            b = c;
        }
        keys[3 * t + k] = ((unsigned long long)(unsigned)a << vbits) | (unsigned)b;
        vals[3 * t + k] = t;
    }
}

__global__ void k_run_heads(const unsigned long long *keys, int n, int *head) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    head[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}

__global__ void k_count_from_scan(const int *flag, const int *idx, int n, int *count) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *count = n > 0 ? idx[n - 1] + flag[n - 1] : 0;
}

__global__ void k_write_edges(const unsigned long long *keys, const int *vals, const int *head, const int *idx, int n,
                              int vbits, const int4 *tri, const int *tri_local, const DevShape *shapes, DevEdge *out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !head[i]) return;
    int j = i + 1;
    while (j < n && !head[j]) j++;
    int t0 = vals[i], t1 = j - i >= 2 ? vals[j - 1] : -1;
    unsigned long long k = keys[i];
    int a = (int)(k >> vbits), b = (int)(k & ((1ull << vbits) - 1));
    int s = tri[t0].w;
    int off = shapes[s].vtx_off;
    DevEdge e;
    e.shape = s;
    e.v0 = a - off;
    e.v1 = b - off;
    e.f0 = tri_local[t0];
    e.f1 = t1 >= 0 ? tri_local[t1] : -1;
    out[idx[i]] = e;
}

// The reference drops degenerate edges and edges between exactly coplanar
// faces (scene.cpp:76-90); the rest are silhouette-tree edges (boundary, or
// a mesh without shading normals) or normal-tree edges.
__global__ void k_classify_edges(DevScene s, const DevEdge *topo, int n, int *keep, int *sil, int *nrm) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    DevEdge e = topo[i];
    float3 d = edge_v0(s, e) - edge_v1(s, e);
    bool k = true;
    if (fabsf(d.x) + fabsf(d.y) + fabsf(d.z) < 1e-10f) {
        k = false;
    } else if (e.f1 != -1) {
        float ang = fabsf(dot(face_normal(s, e.shape, e.f0), face_normal(s, e.shape, e.f1)));
        if (ang == 1.f || ang == -1.f) k = false;
    }
    bool silhouette = e.f0 == -1 || e.f1 == -1 || !s.shapes[e.shape].has_n;
    keep[i] = k;
    sil[i] = k && silhouette;
    nrm[i] = k && !silhouette;
}

// ------------------------------------------------------ primary sampler ---

// Cohen-Sutherland clip to [0,1]^2 (line_clip.h:13-102), as the host build
__device__ bool clip_unit(float2 a, float2 b, float2 &oa, float2 &ob) {
    auto code = [](float2 v) {
        int c = 0;
        if (v.x < 0.f) c |= 1;
        else if (v.x > 1.f) c |= 2;
        if (v.y < 0.f) c |= 4;
        else if (v.y > 1.f) c |= 8;
        return c;
    };
    int c0 = code(a), c1 = code(b);
    for (int guard = 0; guard < 64; guard++) {
        if (!(c0 | c1)) {
            oa = a;
            ob = b;
            return true;
        }
        if (c0 & c1) return false;
        int out = c0 ? c0 : c1;
        float2 v = make_float2(0.f, 0.f);
        if (out & 8) {
            v.x = a.x + (b.x - a.x) * (1.f - a.y) / (b.y - a.y);
            v.y = 1.f;
        } else if (out & 4) {
            v.x = a.x + (b.x - a.x) * (0.f - a.y) / (b.y - a.y);
            v.y = 0.f;
        } else if (out & 2) {
            v.y = a.y + (b.y - a.y) * (1.f - a.x) / (b.x - a.x);
            v.x = 1.f;
        } else {
            v.y = a.y + (b.y - a.y) * (0.f - a.x) / (b.x - a.x);
            v.x = 0.f;
        }
        if (out == c0) {
            a = v;
            c0 = code(a);
        } else {
            b = v;
            c1 = code(b);
        }
    }
    return false;
}

// clipped screen length of a kept edge that is a silhouette from the camera
// (edge_tree.cpp:263-294), 0 otherwise
__global__ void k_primary_lengths(DevScene s, DevCamera cam, const DevEdge *kept, int n, float *len, int *flag) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    DevEdge e = kept[i];
    float3 org = xfm_point(cam.c2w, f3(0.f, 0.f, 0.f));
    float2 a, b;
    float dist = 0.f;
    if (project(cam, edge_v0(s, e), edge_v1(s, e), a, b)) {
        float2 ca, cb;
        if (clip_unit(a, b, ca, cb)) dist = sqrtf((cb.x - ca.x) * (cb.x - ca.x) + (cb.y - ca.y) * (cb.y - ca.y));
    }
    if (!is_silhouette(s, org, e)) dist = 0.f;
    len[i] = dist;
    flag[i] = dist > 0.f;
}

// pbrt's Distribution1D (distribution.h:7-36) over the selected lengths, in
// the reference's sequential float order (one thread)
__global__ void k_distribution(const float *func, const int *count, float *cdf, float *func_int) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    int n = *count;
    if (n <= 0) {
        *func_int = 0.f;
        return;
    }
    cdf[0] = 0.f;
    float c = 0.f;
    for (int i = 1; i <= n; i++) {
        c = c + func[i - 1] / n;
        cdf[i] = c;
    }
    float fi = c;
    for (int i = 1; i <= n; i++) cdf[i] = fi == 0.f ? float(i) / float(n) : cdf[i] / fi;
    *func_int = fi;
}

// ---------------------------------------------------------------- trees ---

// warp-aggregated atomics: lanes of a warp that all belong to one node
// combine first (most lanes do, in the upper levels)
__device__ unsigned warp_min(unsigned v) {
    for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ unsigned warp_max(unsigned v) {
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ unsigned long long warp_sum(unsigned long long v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

struct PrimRec {
    float sblo[3], sbhi[3], sc[3], dc[3], n0[3], n1[3];
};

// A node of the build, by level; boxes as total-order keys
struct BNode {
    int start, end, c0, c1;
    int leaf, dim, size, pre;
    unsigned sb_lo[3], sb_hi[3], sc_lo[3], sc_hi[3], dc_lo[3], dc_hi[3];
    unsigned long long fs[3];
    unsigned cmin;
    float axis[3];
    float tl;
    int pad;
};

__device__ float tmin_f(float a, float b) { return edge_ord_key(b) < edge_ord_key(a) ? b : a; }
__device__ float tmax_f(float a, float b) { return edge_ord_key(b) > edge_ord_key(a) ? b : a; }

// per-edge records: box of the two endpoints (total order), its centre
__global__ void k_prims(DevScene s, const DevEdge *edges, int n, PrimRec *prims, int *perm, unsigned *world) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned wk[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    if (i < n) {
        DevEdge e = edges[i];
        float3 v0 = edge_v0(s, e), v1 = edge_v1(s, e);
        PrimRec r;
        float p0[3] = {v0.x, v0.y, v0.z}, p1[3] = {v1.x, v1.y, v1.z};
        const float inf = __int_as_float(0x7f800000);
        for (int a = 0; a < 3; a++) {
            float lo = tmin_f(tmin_f(inf, p0[a]), p1[a]);
            float hi = tmax_f(tmax_f(-inf, p0[a]), p1[a]);
            r.sblo[a] = lo;
            r.sbhi[a] = hi;
            r.sc[a] = 0.5f * lo + 0.5f * hi;
            r.dc[a] = 0.f;
            r.n0[a] = r.n1[a] = 0.f;
            wk[a] = edge_ord_key(lo);
            wk[3 + a] = edge_ord_key(hi);
        }
        prims[i] = r;
        perm[i] = i;
    }
    // the world box: one atomic per warp and bound
    for (int a = 0; a < 3; a++) {
        unsigned lo = warp_min(wk[a]), hi = warp_max(wk[3 + a]);
        if ((threadIdx.x & 31) == 0) {
            atomicMin(world + a, lo);
            atomicMax(world + 3 + a, hi);
        }
    }
}

// normal-tree records: the two face normals oriented by the shading normals
// and their box scaled by the world diagonal / 8 (edge_tree.cpp:211-236)
__global__ void k_prims_dir(DevScene s, const DevEdge *edges, int n, PrimRec *prims, const unsigned *world) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float3 wl = f3(edge_from_ord_key(world[0]), edge_from_ord_key(world[1]), edge_from_ord_key(world[2]));
    float3 wh = f3(edge_from_ord_key(world[3]), edge_from_ord_key(world[4]), edge_from_ord_key(world[5]));
    float factor = length(wh - wl) / 8.f;
    DevEdge e = edges[i];
    const DevShape sh = s.shapes[e.shape];
    float3 sn = normalize(vtx3(s.nrm, sh.vtx_off + e.v0) + vtx3(s.nrm, sh.vtx_off + e.v1));
    float3 n0 = face_normal(s, e.shape, e.f0), n1 = face_normal(s, e.shape, e.f1);
    if (dot(n0, sn) < 0.f) n0 = -n0;
    if (dot(n1, sn) < 0.f) n1 = -n1;
    float3 a = n0 * factor, b = n1 * factor;
    float pa[3] = {a.x, a.y, a.z}, pb[3] = {b.x, b.y, b.z};
    float m0[3] = {n0.x, n0.y, n0.z}, m1[3] = {n1.x, n1.y, n1.z};
    const float inf = __int_as_float(0x7f800000);
    PrimRec &r = prims[i];
    for (int k = 0; k < 3; k++) {
        float lo = tmin_f(tmin_f(inf, pa[k]), pb[k]);
        float hi = tmax_f(tmax_f(-inf, pa[k]), pb[k]);
        r.dc[k] = 0.5f * (lo + hi);
        r.n0[k] = m0[k];
        r.n1[k] = m1[k];
    }
}

__global__ void k_nodes_reset(BNode *nodes, int first, int count) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    BNode &b = nodes[first + i];
    for (int a = 0; a < 3; a++) {
        b.sb_lo[a] = b.sc_lo[a] = b.dc_lo[a] = 0xffffffffu;
        b.sb_hi[a] = b.sc_hi[a] = b.dc_hi[a] = 0u;
        b.fs[a] = 0ull;
    }
    b.cmin = edge_ord_key(1.f);
    b.leaf = 0;
    b.c0 = b.c1 = -1;
}

template <bool DIR>
__global__ void k_level_reduce(const int *elem_node, const int *perm, const PrimRec *prims, int n, BNode *nodes) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int node = i < n ? elem_node[i] : -1;
    unsigned v[18];
    unsigned long long f[3] = {0ull, 0ull, 0ull};
    if (node >= 0) {
        const PrimRec &r = prims[perm[i]];
        for (int a = 0; a < 3; a++) {
            v[a] = edge_ord_key(r.sblo[a]);
            v[3 + a] = edge_ord_key(r.sbhi[a]);
            v[6 + a] = edge_ord_key(r.sc[a]);
            v[9 + a] = edge_ord_key(r.sc[a]);
            v[12 + a] = edge_ord_key(r.dc[a]);
            v[15 + a] = edge_ord_key(r.dc[a]);
            if (DIR) f[a] = (unsigned long long)(edge_fixed(r.n0[a]) + edge_fixed(r.n1[a]));
        }
    }
    int lead = __shfl_sync(0xffffffffu, node, 0);
    bool uniform = __all_sync(0xffffffffu, node == lead);
    if (uniform) {
        if (lead < 0) return;
        for (int a = 0; a < 3; a++) {
            v[a] = warp_min(v[a]);
            v[3 + a] = warp_max(v[3 + a]);
            v[6 + a] = warp_min(v[6 + a]);
            v[9 + a] = warp_max(v[9 + a]);
            if (DIR) {
                v[12 + a] = warp_min(v[12 + a]);
                v[15 + a] = warp_max(v[15 + a]);
                f[a] = warp_sum(f[a]);
            }
        }
        if ((threadIdx.x & 31) != 0) return;
    } else if (node < 0) {
        return;
    }
    BNode &b = nodes[node];
    for (int a = 0; a < 3; a++) {
        atomicMin(&b.sb_lo[a], v[a]);
        atomicMax(&b.sb_hi[a], v[3 + a]);
        atomicMin(&b.sc_lo[a], v[6 + a]);
        atomicMax(&b.sc_hi[a], v[9 + a]);
        if (DIR) {
            atomicMin(&b.dc_lo[a], v[12 + a]);
            atomicMax(&b.dc_hi[a], v[15 + a]);
            atomicAdd(&b.fs[a], f[a]);
        }
    }
}

template <bool DIR> __global__ void k_level_decide(BNode *nodes, int first, int count) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    BNode &b = nodes[first + i];
    float3 nsum = f3(edge_unfixed((long long)b.fs[0]), edge_unfixed((long long)b.fs[1]), edge_unfixed((long long)b.fs[2]));
    float3 axis = normalize(nsum);
    b.axis[0] = axis.x;
    b.axis[1] = axis.y;
    b.axis[2] = axis.z;
    int dim = -1;
    if (b.end - b.start > 1)
        dim = edge_split_dim(edge_from_ord_key(b.sc_lo[0]), edge_from_ord_key(b.sc_lo[1]),
                             edge_from_ord_key(b.sc_lo[2]), edge_from_ord_key(b.sc_hi[0]),
                             edge_from_ord_key(b.sc_hi[1]), edge_from_ord_key(b.sc_hi[2]), DIR,
                             edge_from_ord_key(b.dc_lo[0]), edge_from_ord_key(b.dc_lo[1]),
                             edge_from_ord_key(b.dc_lo[2]), edge_from_ord_key(b.dc_hi[0]),
                             edge_from_ord_key(b.dc_hi[1]), edge_from_ord_key(b.dc_hi[2]));
    b.dim = dim;
    b.leaf = dim < 0;
}

// the cone angle's minimum cosine (NaN products skipped, as std::min(cmin, x)
// keeps cmin for a NaN x)
__global__ void k_level_cone(const int *elem_node, const int *perm, const PrimRec *prims, int n, BNode *nodes) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int node = i < n ? elem_node[i] : -1;
    unsigned k = 0xffffffffu;
    if (node >= 0) {
        const PrimRec &r = prims[perm[i]];
        const BNode &b = nodes[node];
        float3 axis = f3(b.axis[0], b.axis[1], b.axis[2]);
        float d0 = dot(f3(r.n0[0], r.n0[1], r.n0[2]), axis), d1 = dot(f3(r.n1[0], r.n1[1], r.n1[2]), axis);
        if (d0 == d0) k = edge_ord_key(d0);
        if (d1 == d1) k = min(k, edge_ord_key(d1));
    }
    int lead = __shfl_sync(0xffffffffu, node, 0);
    if (__all_sync(0xffffffffu, node == lead)) {
        k = warp_min(k);
        if ((threadIdx.x & 31) != 0) return;
    }
    if (node >= 0 && k != 0xffffffffu) atomicMin(&nodes[node].cmin, k);
}

__global__ void k_level_keys(const int *elem_node, const int *perm, const PrimRec *prims, int n, const BNode *nodes,
                             unsigned long long *keys) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int node = elem_node[i];
    unsigned long long k = (unsigned long long)i << 32;  // finished positions stay where they are
    if (node >= 0 && !nodes[node].leaf) {
        const BNode &b = nodes[node];
        const PrimRec &r = prims[perm[i]];
        float c = b.dim < 3 ? r.sc[b.dim] : r.dc[b.dim - 3];
        k = ((unsigned long long)b.start << 32) | edge_ord_key(c);
    }
    keys[i] = k;
}

__global__ void k_level_children(BNode *nodes, int first, int count, int *next) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    BNode &b = nodes[first + i];
    if (b.leaf) return;
    int mid = (b.start + b.end) / 2;
    int c = atomicAdd(next, 2);
    b.c0 = c;
    b.c1 = c + 1;
    nodes[c].start = b.start;
    nodes[c].end = mid;
    nodes[c + 1].start = mid;
    nodes[c + 1].end = b.end;
}

__global__ void k_level_assign(int *elem_node, int n, const BNode *nodes) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int node = elem_node[i];
    if (node < 0) return;
    const BNode &b = nodes[node];
    elem_node[i] = b.leaf ? -1 : (i < (b.start + b.end) / 2 ? b.c0 : b.c1);
}

// bottom up: subtree sizes and total edge lengths (a leaf sums its edges'
// lengths in order, an interior node adds its children's)
__global__ void k_sizes(DevScene s, BNode *nodes, int first, int count, const int *perm, const DevEdge *edges) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    BNode &b = nodes[first + i];
    if (b.leaf) {
        float tl = 0.f;
        for (int j = b.start; j < b.end; j++) {
            DevEdge e = edges[perm[j]];
            tl += length(edge_v1(s, e) - edge_v0(s, e));
        }
        b.tl = tl;
        b.size = 1;
    } else {
        b.tl = nodes[b.c0].tl + nodes[b.c1].tl;
        b.size = 1 + nodes[b.c0].size + nodes[b.c1].size;
    }
}

// top down: depth-first indices (left child right after its parent)
__global__ void k_preorder(BNode *nodes, int first, int count) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    BNode &b = nodes[first + i];
    if (first + i == 0) b.pre = 0;
    if (b.leaf) return;
    nodes[b.c0].pre = b.pre + 1;
    nodes[b.c1].pre = b.pre + 1 + nodes[b.c0].size;
}

__global__ void k_write_nodes(const BNode *nodes, int count, DevEdgeNode *out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const BNode &b = nodes[i];
    DevEdgeNode o;
    for (int a = 0; a < 3; a++) {
        o.lo[a] = edge_from_ord_key(b.sb_lo[a]);
        o.hi[a] = edge_from_ord_key(b.sb_hi[a]);
        o.axis[a] = b.axis[a];
    }
    o.angle = dr_acosf(edge_from_ord_key(b.cmin));
    o.offset = b.leaf ? b.start : nodes[b.c1].pre;
    o.nprims = b.leaf ? b.end - b.start : 0;
    o.total_length = b.tl;
    o.pad = 0;
    out[b.pre] = o;
}

__global__ void k_gather_edges(const int *perm, int n, const DevEdge *edges, DevEdge *out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = edges[perm[i]];
}

// bump allocator over a caller's scratch buffer
struct Bump {
    char *p, *end;
    template <typename T> T *take(size_t count) {
        size_t bytes = (sizeof(T) * count + 255) & ~size_t(255);
        T *r = (T *)p;
        p += bytes;
        return r;
    }
};

}  // namespace

// ------------------------------------------------------------ entry points ---

namespace {
template <typename F> cudaError_t sync_read(cudaStream_t st, F f) {
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    f();
    return cudaSuccess;
}
size_t sort_tmp_bytes(int n) {
    size_t b = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, b, (unsigned long long *)nullptr, (unsigned long long *)nullptr,
                                    (int *)nullptr, (int *)nullptr, std::max(1, n));
    return b;
}
size_t select_tmp_bytes(int n) {
    size_t b = 0, c = 0;
    cub::DeviceSelect::Flagged(nullptr, b, (DevEdge *)nullptr, (int *)nullptr, (DevEdge *)nullptr, (int *)nullptr,
                               std::max(1, n));
    cub::DeviceSelect::Flagged(nullptr, c, (float *)nullptr, (int *)nullptr, (float *)nullptr, (int *)nullptr,
                               std::max(1, n));
    return std::max(b, c);
}
size_t scan_tmp_bytes(int n) {
    size_t b = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, b, (int *)nullptr, (int *)nullptr, std::max(1, n));
    return b;
}
}  // namespace

size_t dr_edges_scratch_bytes(int ntri) {
    int n3 = 3 * std::max(1, ntri);
    size_t phase1 = (size_t)n3 * (2 * 8 + 4 * 4) + std::max(sort_tmp_bytes(n3), scan_tmp_bytes(n3));
    size_t phase2 = (size_t)n3 * (3 * 4 + 3 * sizeof(DevEdge)) + select_tmp_bytes(n3) + 256;
    size_t prim = (size_t)n3 * (4 + 4 + sizeof(DevEdge)) + select_tmp_bytes(n3) + 256;
    return std::max(std::max(phase1, phase2), prim) + 16 * 256;
}

cudaError_t dr_extract_edges(const DevScene &s, int num_vertices, DevEdge *out, int *count_host, void *scratch,
                             size_t scratch_bytes, cudaStream_t st, int *launches) {
    const int ntri = s.num_tris;
    *count_host = 0;
    if (ntri <= 0) return cudaSuccess;
    const int n3 = 3 * ntri;
    const int vbits = bits_for(std::max(2, num_vertices));
    Bump bp{(char *)scratch, (char *)scratch + scratch_bytes};
    auto *keys = bp.take<unsigned long long>(n3), *keys2 = bp.take<unsigned long long>(n3);
    int *vals = bp.take<int>(n3), *vals2 = bp.take<int>(n3), *head = bp.take<int>(n3), *idx = bp.take<int>(n3);
    int *count = bp.take<int>(1);
    size_t tmp_bytes = std::max(sort_tmp_bytes(n3), scan_tmp_bytes(n3));
    void *tmp = bp.take<char>(tmp_bytes);
    if (bp.p > bp.end) return cudaErrorMemoryAllocation;
    k_side_keys<<<nblocks(ntri), kBS, 0, st>>>(s.tri, ntri, vbits, keys, vals);
    cudaError_t e = cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, keys, keys2, vals, vals2, n3, 0, 2 * vbits, st);
    if (e != cudaSuccess) return e;
    k_run_heads<<<nblocks(n3), kBS, 0, st>>>(keys2, n3, head);
    e = cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, head, idx, n3, st);
    if (e != cudaSuccess) return e;
    k_count_from_scan<<<1, 32, 0, st>>>(head, idx, n3, count);
    k_write_edges<<<nblocks(n3), kBS, 0, st>>>(keys2, vals2, head, idx, n3, vbits, s.tri, s.tri_local, s.shapes, out);
    if (launches) *launches += 6;
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(count_host, count, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(st);
}

cudaError_t dr_split_edges(const DevScene &s, const DevEdge *topo, int n, DevEdge *kept, DevEdge *sil, DevEdge *nrm,
                           int counts_host[3], void *scratch, size_t scratch_bytes, cudaStream_t st, int *launches) {
    counts_host[0] = counts_host[1] = counts_host[2] = 0;
    if (n <= 0) return cudaSuccess;
    Bump bp{(char *)scratch, (char *)scratch + scratch_bytes};
    int *fk = bp.take<int>(n), *fs = bp.take<int>(n), *fn = bp.take<int>(n), *cnt = bp.take<int>(3);
    size_t tmp_bytes = select_tmp_bytes(n);
    void *tmp = bp.take<char>(tmp_bytes);
    if (bp.p > bp.end) return cudaErrorMemoryAllocation;
    k_classify_edges<<<nblocks(n), kBS, 0, st>>>(s, topo, n, fk, fs, fn);
    cudaError_t e = cub::DeviceSelect::Flagged(tmp, tmp_bytes, topo, fk, kept, cnt, n, st);
    if (e == cudaSuccess) e = cub::DeviceSelect::Flagged(tmp, tmp_bytes, topo, fs, sil, cnt + 1, n, st);
    if (e == cudaSuccess) e = cub::DeviceSelect::Flagged(tmp, tmp_bytes, topo, fn, nrm, cnt + 2, n, st);
    if (e != cudaSuccess) return e;
    if (launches) *launches += 4;
    e = cudaMemcpyAsync(counts_host, cnt, 3 * sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(st);
}

cudaError_t dr_build_primary(const DevScene &s, const DevCamera &cam, const DevEdge *kept, int n, DevEdge *prim,
                             float *cdf, float *func, int *count_host, float *func_int_host, void *scratch,
                             size_t scratch_bytes, cudaStream_t st, int *launches) {
    *count_host = 0;
    *func_int_host = 0.f;
    if (n <= 0) return cudaSuccess;
    Bump bp{(char *)scratch, (char *)scratch + scratch_bytes};
    float *len = bp.take<float>(n);
    int *flag = bp.take<int>(n), *cnt = bp.take<int>(2);
    float *fi = bp.take<float>(1);
    size_t tmp_bytes = select_tmp_bytes(n);
    void *tmp = bp.take<char>(tmp_bytes);
    if (bp.p > bp.end) return cudaErrorMemoryAllocation;
    k_primary_lengths<<<nblocks(n), kBS, 0, st>>>(s, cam, kept, n, len, flag);
    cudaError_t e = cub::DeviceSelect::Flagged(tmp, tmp_bytes, kept, flag, prim, cnt, n, st);
    if (e == cudaSuccess) e = cub::DeviceSelect::Flagged(tmp, tmp_bytes, len, flag, func, cnt + 1, n, st);
    if (e != cudaSuccess) return e;
    k_distribution<<<1, 32, 0, st>>>(func, cnt, cdf, fi);
    if (launches) *launches += 4;
    e = cudaMemcpyAsync(count_host, cnt, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(func_int_host, fi, sizeof(float), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(st);
}

size_t dr_tree_scratch_bytes(int n) {
    n = std::max(1, n);
    return (size_t)n * (sizeof(PrimRec) + 4 * 4 + 2 * 8) + (size_t)2 * n * sizeof(BNode) + sort_tmp_bytes(n) +
           16 * 256;
}

cudaError_t dr_build_edge_tree(const DevScene &s, bool dir, const DevEdge *edges, int n, DevEdgeNode *out_nodes,
                               DevEdge *ordered, int *num_nodes_host, void *scratch, size_t scratch_bytes,
                               cudaStream_t st, int *launches) {
    *num_nodes_host = 0;
    if (n <= 0) return cudaSuccess;
    Bump bp{(char *)scratch, (char *)scratch + scratch_bytes};
    PrimRec *prims = bp.take<PrimRec>(n);
    int *perm = bp.take<int>(n), *perm2 = bp.take<int>(n), *elem_node = bp.take<int>(n);
    auto *keys = bp.take<unsigned long long>(n), *keys2 = bp.take<unsigned long long>(n);
    BNode *nodes = bp.take<BNode>(2 * (size_t)n);
    unsigned *world = bp.take<unsigned>(6);
    int *next = bp.take<int>(1);
    size_t tmp_bytes = sort_tmp_bytes(n);
    void *tmp = bp.take<char>(tmp_bytes);
    if (bp.p > bp.end) return cudaErrorMemoryAllocation;
    int nl = 0;
    auto L = [&](int k) { nl += k; };
    // per-edge records, the world box, the root
    const unsigned wl_init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    cudaError_t e = cudaMemcpyAsync(world, wl_init, sizeof(wl_init), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    k_prims<<<nblocks(n), kBS, 0, st>>>(s, edges, n, prims, perm, world);
    L(1);
    if (dir) {
        k_prims_dir<<<nblocks(n), kBS, 0, st>>>(s, edges, n, prims, world);
        L(1);
    }
    e = cudaMemsetAsync(elem_node, 0, sizeof(int) * n, st);
    const int root[2] = {0, n};
    if (e == cudaSuccess) e = cudaMemcpyAsync(nodes, root, sizeof(root), cudaMemcpyHostToDevice, st);
    const int one = 1;
    if (e == cudaSuccess) e = cudaMemcpyAsync(next, &one, sizeof(int), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    // level by level
    std::vector<std::pair<int, int>> levels;  // (first node, count)
    int first = 0, count = 1;
    const int kbits = 32 + bits_for(n + 1);
    while (count > 0) {
        // a median split halves every range: at most ceil(log2 n) + 1 levels
        if (levels.size() > 40 || first + count > 2 * n) return cudaErrorIllegalState;
        levels.emplace_back(first, count);
        k_nodes_reset<<<nblocks(count), kBS, 0, st>>>(nodes, first, count);
        if (dir) k_level_reduce<true><<<nblocks(n), kBS, 0, st>>>(elem_node, perm, prims, n, nodes);
        else k_level_reduce<false><<<nblocks(n), kBS, 0, st>>>(elem_node, perm, prims, n, nodes);
        if (dir) k_level_decide<true><<<nblocks(count), kBS, 0, st>>>(nodes, first, count);
        else k_level_decide<false><<<nblocks(count), kBS, 0, st>>>(nodes, first, count);
        L(3);
        // the silhouette tree has no normals: its cone axis is NaN and its
        // minimum cosine stays 1, as in the reference
        if (dir) {
            k_level_cone<<<nblocks(n), kBS, 0, st>>>(elem_node, perm, prims, n, nodes);
            L(1);
        }
        k_level_keys<<<nblocks(n), kBS, 0, st>>>(elem_node, perm, prims, n, nodes, keys);
        e = cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, keys, keys2, perm, perm2, n, 0, kbits, st);
        if (e != cudaSuccess) return e;
        std::swap(perm, perm2);
        k_level_children<<<nblocks(count), kBS, 0, st>>>(nodes, first, count, next);
        k_level_assign<<<nblocks(n), kBS, 0, st>>>(elem_node, n, nodes);
        L(4);
        int total = 0;
        e = cudaMemcpyAsync(&total, next, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return e;
        first += count;
        count = total - first;
    }
    const int num_nodes = first;
    for (int l = (int)levels.size() - 1; l >= 0; l--) {
        k_sizes<<<nblocks(levels[l].second), kBS, 0, st>>>(s, nodes, levels[l].first, levels[l].second, perm, edges);
        L(1);
    }
    for (auto &lv : levels) {
        k_preorder<<<nblocks(lv.second), kBS, 0, st>>>(nodes, lv.first, lv.second);
        L(1);
    }
    k_write_nodes<<<nblocks(num_nodes), kBS, 0, st>>>(nodes, num_nodes, out_nodes);
    k_gather_edges<<<nblocks(n), kBS, 0, st>>>(perm, n, edges, ordered);
    L(2);
    if (launches) *launches += nl;
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    *num_nodes_host = num_nodes;
    return cudaStreamSynchronize(st);
}
