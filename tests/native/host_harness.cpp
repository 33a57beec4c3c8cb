// Test infrastructure: the renderer's __host__ __device__ kernel logic compiled
// for the CPU (DR_HOST_BUILD), so that tests can inspect it without a GPU.
// Never part of the product: the product runs this code only on the GPU.
#include <algorithm>
#include <numeric>
#include <vector>

#include "../../delta_ray_b200/csrc/dr_bvh.cuh"
#include "../../delta_ray_b200/csrc/dr_trace.cuh"

thread_local long long g_dr_visits = 0;

namespace {

// host replica of the device LBVH build (dr_kernels.cu: dr_build_lbvh)
void build_lbvh(const float *vtx, const int4 *tri, int n, std::vector<float4> &nodes, std::vector<float4> &leaves) {
    float3 lo = f3(1e30f), hi = f3(-1e30f);
    for (int i = 0; i < n; i++) {
        const int *t = &tri[i].x;
        for (int k = 0; k < 3; k++) {
            const float *p = vtx + 3 * t[k];
            lo = f3(std::min(lo.x, p[0]), std::min(lo.y, p[1]), std::min(lo.z, p[2]));
            hi = f3(std::max(hi.x, p[0]), std::max(hi.y, p[1]), std::max(hi.z, p[2]));
        }
    }
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
    leaves.assign(3 * n, float4{});
    std::vector<Box> leaf_boxes(n), node_boxes(std::max(1, n));
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

}  // namespace

extern "C" {

// Builds the LBVH over (vtx, tri) and traces n rays [n][6]; writes the hit
// triangle, t, and returns the total number of BVH nodes visited.
long long hh_trace(const float *vtx, const int *tri4, int ntri, const float *rays, int n, int *out_tri, float *out_t) {
    std::vector<float4> nodes, leaves;
    build_lbvh(vtx, (const int4 *)tri4, ntri, nodes, leaves);
    DevScene s;
    std::memset(&s, 0, sizeof(s));
    s.num_tris = ntri;
    s.bvh_nodes = nodes.data();
    s.bvh_tris = leaves.data();
    s.bvh_root = ntri > 1 ? 0 : ~0;
    g_dr_visits = 0;
    for (int i = 0; i < n; i++) {
        const float *r = rays + 6 * i;
        Hit h = trace_closest(s, f3(r[0], r[1], r[2]), f3(r[3], r[4], r[5]), 1e-3f);
        out_tri[i] = h.tri;
        out_t[i] = h.t;
    }
    return g_dr_visits;
}

// LBVH statistics: depth histogram max and the sum of node box surface areas.
void hh_bvh_stats(const float *vtx, const int *tri4, int ntri, double *out) {
    std::vector<float4> nodes, leaves;
    build_lbvh(vtx, (const int4 *)tri4, ntri, nodes, leaves);
    int maxd = 0;
    double area = 0.0;
    std::vector<std::pair<int, int>> st;
    st.push_back({0, 0});
    while (!st.empty()) {
        auto [nd, d] = st.back();
        st.pop_back();
        maxd = std::max(maxd, d);
        if (nd < 0) continue;
        const float4 *q = &nodes[4 * nd];
        float b0[6] = {q[0].x, q[0].y, q[0].z, q[0].w, q[1].x, q[1].y};
        float b1[6] = {q[1].z, q[1].w, q[2].x, q[2].y, q[2].z, q[2].w};
        for (float *b : {b0, b1}) {
            float dx = b[3] - b[0], dy = b[4] - b[1], dz = b[5] - b[2];
            area += 2.0 * (dx * dy + dy * dz + dz * dx);
        }
        st.push_back({dr_f2i(q[3].x), d + 1});
        st.push_back({dr_f2i(q[3].y), d + 1});
    }
    out[0] = maxd;
    out[1] = area;
}

}  // extern "C"
