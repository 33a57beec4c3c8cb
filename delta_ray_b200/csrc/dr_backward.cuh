// Per-sample backward procedures, shared by the CUDA kernels (dr_backward.cu)
// and the CPU build used by the tests.  They restate render_sample
// (delta_ray.cpp:694-1005) and the primary-edge pass (delta_ray.cpp:1468-1550)
// with hand-written adjoints instead of the reference's tape:
//
//  1. backward_pixel_sample: traces the path once, storing per bounce the
//     next hit and the bounce's contribution X_k and throughput factor r_k;
//     the suffix radiance S_k = X_k + r_k S_{k+1} then gives every factor's
//     adjoint, and a replay of the stored bounces (no ray traversal) runs
//     the local adjoints.  Gradients through diffuse-sampled bounces are cut
//     as in pathtrace.h:149-159,245-247; only the first vertex's geometry is
//     differentiated.  The first vertex becomes a secondary-edge shading
//     point (pathtrace.h:218-227).
//  2. traverse_point: samples the shading point's edges from the edge tree.
//  3. eval_item: one sampled edge: dv0/dv1 and the point's position adjoint dp.
//  4. propagate_dp: dp pushed back through the first vertex to the triangle
//     and the camera (delta_ray.cpp:975-1002).
//  5. primary_edge_item: one primary-edge sample.
//
// Random numbers come from Philox streams: kStreamPixel (per pixel sample),
// kStreamEdgePoint (per shading point: edge sample and traversal draws),
// kStreamEdgeItem (per sampled edge: its light and secondary samples) and
// kStreamPrimaryEdge (per primary-edge sample).
#pragma once

#include "dr_adjoint.cuh"
#include "dr_edges.cuh"

#define DR_MAX_BOUNCES 64
#define DR_PT_WORDS 24

// Secondary shading point record (packed floats; ints stored as bits).
struct PointRecord {
    float3 p, n, ng;
    float2 uv;
    float3 wi, d_color;
    int tri;
    uint64_t sid;
    int light;
    int bounce;
    HD void store(float *w) const {
        w[0] = p.x; w[1] = p.y; w[2] = p.z;
        w[3] = n.x; w[4] = n.y; w[5] = n.z;
        w[6] = ng.x; w[7] = ng.y; w[8] = ng.z;
        w[9] = uv.x; w[10] = uv.y;
        w[11] = wi.x; w[12] = wi.y; w[13] = wi.z;
        w[14] = d_color.x; w[15] = d_color.y; w[16] = d_color.z;
        w[17] = dr_i2f(tri);
        w[18] = dr_i2f((int)(uint32_t)sid);
        w[19] = dr_i2f((int)(uint32_t)(sid >> 32));
        w[20] = dr_i2f(light);
        w[21] = dr_i2f(bounce);
        w[22] = 0.f;
        w[23] = 0.f;
    }
    HD void load(const float *w) {
        p = f3(w[0], w[1], w[2]);
        n = f3(w[3], w[4], w[5]);
        ng = f3(w[6], w[7], w[8]);
        uv.x = w[9];
        uv.y = w[10];
        wi = f3(w[11], w[12], w[13]);
        d_color = f3(w[14], w[15], w[16]);
        tri = dr_f2i(w[17]);
        sid = (uint64_t)(uint32_t)dr_f2i(w[18]) | ((uint64_t)(uint32_t)dr_f2i(w[19]) << 32);
        light = dr_f2i(w[20]);
        bounce = dr_f2i(w[21]);
    }
    HD SurfacePoint surface() const {
        SurfacePoint sp;
        sp.p = p;
        sp.ng = ng;
        sp.f = make_frame(n);
        sp.uv = uv;
        return sp;
    }
};

struct BounceRecord {
    int next_tri;  // hit of the BSDF-sampled ray, -1 when the path ended here
    float3 X;      // radiance added at this vertex (NEE + emitter hit), before T_k
    float3 r;      // throughput factor f / (pdf q)
    float q;       // Russian-roulette survival probability (1 before bounce 5)
};

// Direction sampled at a vertex, with the two-sided flip of pathtrace.h:116-133.
DEV float3 sampled_direction(const DevScene &s, const BSDFSample &bs, float3 wi, int tri, const SurfacePoint &sp,
                             bool &specular) {
    int mi = material_of_tri(s, tri);
    SurfacePoint use = sp;
    if (s.mats[mi].two_sided && dot(wi, sp.f.n) < 0.f) {
        use.f = frame_neg(sp.f);
        use.ng = -sp.ng;
    }
    return sample_bsdf_dir(s, mi, use, wi, bs, specular);
}

// The pixel sample's screen position (delta_ray.cpp:1236-1237,657-658).
DEV void pixel_sample_position(int x, int y, int W, int H, int spp, uint64_t sid, uint64_t seed, bool full_jitter,
                               float &sx, float &sy, Rng &r) {
    r.init(seed, kStreamPixel, sid, 0);
    float ux = r.next(), uy = r.next();
    float sub_x = full_jitter ? ux : ux / spp;
    float sub_y = full_jitter ? uy : uy / spp;
    sx = float((x + sub_x) / W);
    sy = float((y + sub_y) / H);
}

// Returns the sample's image contribution; accumulates its gradient into g
// and hands its first vertex to push_point(const PointRecord&).
template <class G, class Push>
DEV float3 backward_pixel_sample(const DevScene &s, int x, int y, int W, int H, int spp, int si, int B, uint64_t seed,
                                 float3 d_color, G &g, Push &push_point) {
    const float sw = 1.f / spp;
    uint64_t sid = ((uint64_t)y * W + x) * spp + si;
    Rng r;
    float sx, sy;
    pixel_sample_position(x, y, W, H, spp, sid, seed, s.full_pixel_jitter != 0, sx, sy, r);
    Ray ray = sample_primary(s.cam, sx, sy, true);
    if (abs_sum(ray.d) == 0.f) return f3(0.f);
    Hit h0 = trace_closest(s, ray.o, ray.d, 1e-3f);
    if (h0.tri < 0) return f3(0.f);
    TriData td0 = load_tri(s, h0.tri);
    IsectFwd fw0;
    SurfacePoint sp0 = intersect_tri(td0, ray.o, ray.d, &fw0, true);
    LightSample ls = draw_light(r);
    const Rng r_sec = r;  // stream position of the first secondary sample
    const float3 wi = -ray.d;
    // ---- pass 1: trace, keep the bounces ----
    BounceRecord rec[DR_MAX_BOUNCES];
    int nb = 0;
    float3 color = f3(0.f);
    int li0 = light_of_tri(s, h0.tri);
    bool prim_emit = li0 >= 0 && dot(sp0.f.n, wi) > 0.f;
    if (prim_emit) color += light_intensity(s, li0);
    float3 thr = f3(1.f), cwi = wi;
    int ctri = h0.tri;
    SurfacePoint csp = sp0;
    for (int b = 0; b < B; b++) {
        SecondarySample ss = draw_secondary(r);
        float3 N = nee(s, ls, wi, ctri, csp);
        color += thr * N;
        nb = b + 1;
        rec[b].next_tri = -1;
        rec[b].X = N;
        rec[b].r = f3(0.f);
        rec[b].q = 1.f;
        BounceHit bh = sample_bsdf_scene(s, ss.bsdf, cwi, ctri, csp);
        if (bh.tri < 0) break;
        float3 wo = normalize(bh.sp.p - csp.p);
        int mi = material_of_tri(s, ctri);
        float pdf = bsdf_pdf(s, mi, csp, cwi, wo);
        if (pdf <= 0.f) break;
        float3 f = bsdf(s, mi, csp, cwi, wo);
        if (sum(f) <= 0.f) break;
        rec[b].next_tri = bh.tri;
        int nli = light_of_tri(s, bh.tri);
        if (nli >= 0 && dot(bh.sp.f.n, -wo) > 0.f) {
            float lpdf = light_pdf(s, bh.tri) * length_sq(bh.sp.p - csp.p) / fabsf(dot(wo, bh.sp.ng));
            float mis = sq(pdf) / (sq(lpdf) + sq(pdf));
            float3 em = f * light_intensity(s, nli) * (mis / pdf);
            color += thr * em;
            rec[b].X += em;
        }
        float3 rb = f / pdf;
        thr = thr * rb;
        if (b >= 5) {
            float q = fminf(max3(thr), 0.95f);
            if (ss.rr >= q) break;
            thr = thr / q;
            rb = rb / q;
            rec[b].q = q;
        }
        rec[b].r = rb;
        cwi = -wo;
        ctri = bh.tri;
        csp = bh.sp;
    }
    color = color * sw;
    if (is_zero(d_color)) return color;  // render_sample_fast: no derivatives, no edges
    // ---- the first vertex is a secondary-edge shading point ----
    {
        PointRecord pr;
        pr.p = sp0.p;
        pr.n = sp0.f.n;
        pr.ng = sp0.ng;
        pr.uv = sp0.uv;
        pr.wi = wi;
        pr.d_color = d_color;
        pr.tri = h0.tri;
        pr.sid = sid;
        pr.light = sample_discrete(s.light_sel_cdf, s.light_sel_func, s.light_sel_func_int, s.num_lights, ls.sel,
                                   nullptr);
        pr.bounce = 0;
        if (B >= 1) push_point(pr);
    }
    // ---- suffix radiance S_{k+1}, stored in rec[k].X ----
    float3 S = f3(0.f);
    for (int k = nb - 1; k >= 0; k--) {
        float3 Sk = rec[k].X + rec[k].r * S;
        rec[k].X = S;  // now holds S_{k+1}
        S = Sk;
    }
    // ---- pass 2: replay with adjoints ----
    const float3 dC = d_color * sw;
    if (prim_emit) {
        const DevLight &L = s.lights[li0];
        g.add(L.grad + 0, dC.x);
        g.add(L.grad + 1, dC.y);
        g.add(L.grad + 2, dC.z);
    }
    SpGrad g0;  // adjoints of the first vertex (frame, uv) and of wi
    g0.zero();
    float3 d_p0 = f3(0.f);
    Rng rr = r_sec;
    thr = f3(1.f);
    cwi = wi;
    ctri = h0.tri;
    csp = sp0;
    for (int k = 0; k < nb; k++) {
        SecondarySample ss = draw_secondary(rr);
        const bool first = k == 0;
        float3 a = dC * thr;
        {
            SpGrad gn;
            gn.zero();
            float3 dp = f3(0.f);
            d_nee(s, ls, wi, ctri, csp, a, g, gn, dp);
            g0.dwi += gn.dwi;  // NEE always uses the primary wi (pathtrace.h:213-216)
            if (first) {
                frame_add(g0.df, gn.df);
                g0.duv.x += gn.duv.x;
                g0.duv.y += gn.duv.y;
                d_p0 += dp;
            }
        }
        int nt = rec[k].next_tri;
        if (nt < 0) break;
        bool spec;
        float3 dir = sampled_direction(s, ss.bsdf, cwi, ctri, csp, spec);
        SurfacePoint nsp = intersect_tri(load_tri(s, nt), csp.p, dir);
        float3 wo = normalize(nsp.p - csp.p);
        int mi = material_of_tri(s, ctri);
        float pdf = bsdf_pdf(s, mi, csp, cwi, wo);
        float3 f = bsdf(s, mi, csp, cwi, wo);
        float3 d_f = f3(0.f);
        float d_pdf = 0.f;
        int nli = light_of_tri(s, nt);
        if (nli >= 0 && dot(nsp.f.n, -wo) > 0.f) {
            float lpdf = light_pdf(s, nt) * length_sq(nsp.p - csp.p) / fabsf(dot(wo, nsp.ng));
            float mis = sq(pdf) / (sq(lpdf) + sq(pdf));
            float3 I = light_intensity(s, nli);
            float c = mis / pdf;
            d_f += a * I * c;
            const DevLight &L = s.lights[nli];
            g.add(L.grad + 0, a.x * f.x * c);
            g.add(L.grad + 1, a.y * f.y * c);
            g.add(L.grad + 2, a.z * f.z * c);
            d_pdf -= dot(a * f, I) * mis / (pdf * pdf);
        }
        // r_k = f / (pdf q): its adjoint is dC T_k S_{k+1}
        float3 dr = a * rec[k].X;
        float q = rec[k].q;
        if (!is_zero(dr)) {
            d_f += dr * (1.f / (pdf * q));
            d_pdf -= dot(dr, f) / (pdf * pdf * q);
        }
        SpGrad gb;
        gb.zero();
        d_bsdf(s, mi, csp, cwi, wo, d_f, g, gb);
        if (!s.detached_pdf) d_bsdf_pdf(s, mi, csp, cwi, wo, d_pdf, g, gb);
        if (first) {
            frame_add(g0.df, gb.df);
            g0.duv.x += gb.duv.x;
            g0.duv.y += gb.duv.y;
            g0.dwi += gb.dwi;
        }
        thr = thr * rec[k].r;
        cwi = -wo;
        ctri = nt;
        csp = nsp;
    }
    // ---- first vertex geometry -> triangle and camera ----
    TriGrad tg;
    tg.v0 = tg.v1 = tg.v2 = tg.n0 = tg.n1 = tg.n2 = f3(0.f);
    float3 d_o = f3(0.f), d_d = f3(0.f);
    d_intersect_tri(td0, ray.o, ray.d, fw0, d_p0, f3(0.f), g0.df, g0.duv, tg, d_o, d_d);
    d_d -= g0.dwi;
    scatter_tri_vertices(s, h0.tri, tg.v0, tg.v1, tg.v2, g);
    if (td0.has_n) {
        // the first vertex's normal adjoint goes to all three (delta_ray.cpp:1261-1269)
        int4 id = s.tri[h0.tri];
        const DevShape &sh = s.shapes[id.w];
        int b = sh.grad_n - 3 * sh.vtx_off;
        const int v[3] = {id.x, id.y, id.z};
        for (int k = 0; k < 3; k++) {
            g.add(b + 3 * v[k], tg.n0.x);
            g.add(b + 3 * v[k] + 1, tg.n0.y);
            g.add(b + 3 * v[k] + 2, tg.n0.z);
        }
    }
    d_sample_primary(s.cam, sx, sy, d_o, d_d, g, 0);
    return color;
}

// Cone towards the bounding sphere of the light picked by the primary light
// sample (delta_ray.cpp:878-890).
DEV ConeSpec light_cone(const DevScene &s, int li, float3 p) {
    const DevLight &L = s.lights[li];
    float3 bc = f3(L.bc[0], L.bc[1], L.bc[2]);
    float3 dl = bc - p;
    float tan_a = L.br / length(dl);
    ConeSpec c;
    c.o = p;
    c.d = normalize(dl);
    c.cos_angle = tan_a <= 1.f ? 1.f / sqrtf(tan_a * tan_a + 1.f) : 0.f;
    return c;
}

// Samples the point's edges; emit(tree, edge_index, j, weight) for every
// sampled edge of nonzero weight, j counting all sampled edges in order.
template <class Emit>
DEV bool traverse_point(const DevScene &s, const PointRecord &pt, uint64_t seed, Emit &emit) {
    Rng prng;
    prng.init(seed, kStreamEdgePoint, pt.sid, (uint32_t)pt.bounce);
    draw_edge(prng);  // the point's edge sample; eval_item redraws it
    SurfacePoint sp = pt.surface();
    ConeSpec cone = light_cone(s, pt.light, sp.p);
    int j = 0;
    auto em = [&](int tree, int ei, float w) {
        if (w != 0.f) emit(tree, ei, j, w);
        j++;
    };
    return traverse_edges(s, pt.wi, pt.tri, sp, cone, prng, em);
}

// One sampled edge (delta_ray.cpp:901-973); returns dp, scatters dv0 / dv1.
template <class G>
DEV float3 eval_item(const DevScene &s, const PointRecord &pt, int tree, int ei, int j, float w, int spp, int B,
                     uint64_t seed, G &g) {
    Rng prng;
    prng.init(seed, kStreamEdgePoint, pt.sid, (uint32_t)pt.bounce);
    EdgeSample es = draw_edge(prng);
    Rng irng;
    irng.init(seed, kStreamEdgeItem, pt.sid, ((uint32_t)pt.bounce << 16) | (uint32_t)j);
    LightSample els = draw_light(irng);
    const DevEdge &edge = tree ? s.nrm_edges[ei] : s.sil_edges[ei];
    float3 weight = f3(1.f) * ((1.f / spp) * w);
    EdgeResult er = shading_edge_sample(s, es, edge, els, irng, B - pt.bounce - 1, pt.wi, pt.tri, pt.surface(),
                                        weight, pt.d_color, B == 1);
    if (!is_zero(er.dv0) || !is_zero(er.dv1)) {
        const DevShape &sh = s.shapes[edge.shape];
        g.add(sh.grad_v + 3 * edge.v0 + 0, er.dv0.x);
        g.add(sh.grad_v + 3 * edge.v0 + 1, er.dv0.y);
        g.add(sh.grad_v + 3 * edge.v0 + 2, er.dv0.z);
        g.add(sh.grad_v + 3 * edge.v1 + 0, er.dv1.x);
        g.add(sh.grad_v + 3 * edge.v1 + 1, er.dv1.y);
        g.add(sh.grad_v + 3 * edge.v1 + 2, er.dv1.z);
    }
    return er.dp;
}

// dp of a first-vertex shading point pushed back to its triangle and the camera.
template <class G>
DEV void propagate_dp(const DevScene &s, const PointRecord &pt, int W, int H, int spp, uint64_t seed, float3 dp, G &g) {
    uint64_t pix = pt.sid / (uint64_t)spp;
    int x = (int)(pix % (uint64_t)W), y = (int)(pix / (uint64_t)W);
    Rng r;
    float sx, sy;
    pixel_sample_position(x, y, W, H, spp, pt.sid, seed, s.full_pixel_jitter != 0, sx, sy, r);
    Ray ray = sample_primary(s.cam, sx, sy, true);
    TriData td = load_tri(s, pt.tri);
    IsectFwd fw;
    intersect_tri(td, ray.o, ray.d, &fw, true);
    TriGrad tg;
    tg.v0 = tg.v1 = tg.v2 = tg.n0 = tg.n1 = tg.n2 = f3(0.f);
    float3 d_o = f3(0.f), d_d = f3(0.f);
    Frame zf = frame_zero();
    float2 zuv;
    zuv.x = zuv.y = 0.f;
    d_intersect_tri(td, ray.o, ray.d, fw, dp, f3(0.f), zf, zuv, tg, d_o, d_d);
    scatter_tri_vertices(s, pt.tri, tg.v0, tg.v1, tg.v2, g);
    d_sample_primary(s.cam, sx, sy, d_o, d_d, g, 0);
}

// Primary-edge sample i (delta_ray.cpp:1478-1522).
template <class G>
DEV void primary_edge_item(const DevScene &s, long long i, int W, int H, int spp, int B, uint64_t seed,
                           const float *d_image, G &g) {
    if (s.num_prim_edges == 0) return;
    Rng r;
    r.init(seed, kStreamPrimaryEdge, (uint64_t)i, 0);
    float pmf = 0.f;
    int id = sample_discrete(s.prim_cdf, s.prim_func, s.prim_func_int, s.num_prim_edges, r.next(), &pmf);
    float w = pmf > 0.f ? 1.f / pmf : 0.f;
    if (w <= 0.f) return;
    EdgeSample es = draw_edge(r);
    LightSample ls = draw_light(r);
    PrimaryEdgeResult pr;
    primary_edge_sample(s, es, s.prim_edges[id], ls, r, B, d_image, W, H, w / spp, pr);
    if (!pr.ok) return;
    const DevShape &sh = s.shapes[pr.edge.shape];
    g.add(sh.grad_v + 3 * pr.edge.v0 + 0, pr.dv0.x);
    g.add(sh.grad_v + 3 * pr.edge.v0 + 1, pr.dv0.y);
    g.add(sh.grad_v + 3 * pr.edge.v0 + 2, pr.dv0.z);
    g.add(sh.grad_v + 3 * pr.edge.v1 + 0, pr.dv1.x);
    g.add(sh.grad_v + 3 * pr.edge.v1 + 1, pr.dv1.y);
    g.add(sh.grad_v + 3 * pr.edge.v1 + 2, pr.dv1.z);
    for (int q = 0; q < 16; q++) g.add(16 + q, pr.dw2c[q]);
}
