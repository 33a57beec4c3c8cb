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
// the checkpointed form (BMAX < 0): up to DR_CKPT_SEGS segments of -BMAX bounces
#define DR_CKPT_SEGS 16
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
    int view = 0;  // the view of a batched multi-view call (0 otherwise)
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
        w[22] = dr_i2f(view);
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
        view = dr_f2i(w[22]);
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

// Adjoint of the specular lobe's sampled direction (sample_bsdf_dir with
// bs.w > dpmf): dir = 2 (wi.h) h - wi, h = to_world(f, (st cos phi, st sin phi,
// ct)), ct from the lobe's inverse cdf at bs.u0 (roughness-dependent).  f is
// the frame the sample used (flipped for two-sided back faces by the caller).
// Accumulates d_f, d_wi and returns d(roughness).
DEV float d_specular_direction(const DevScene &s, int mi, const Frame &f, float3 wi, float rough, const BSDFSample &bs,
                               float3 d_dir, Frame &d_f, float3 &d_wi) {
    const DevMaterial &m = s.mats[mi];
    float phi = 2.f * DR_PI * bs.u1;
    float sphi = dr_sinf(phi), cphi = dr_cosf(phi);
    float ct, dct_dr = 0.f;
    if (m.model == DR_MICROFACET_GGX) {
        float A = ggx_A(rough);
        float num = 1.f - bs.u0, den = 1.f + (A - 1.f) * bs.u0;
        ct = sqrtf(num / den);
        if (ct > 0.f) dct_dr = (-num * bs.u0 / (2.f * ct * den * den)) * ggx_dA_drough(rough);
    } else {
        float e = roughness_to_phong(rough);
        float ie = 1.f / (e + 2.0f);
        ct = dr_powf(bs.u0, ie);
        if (2.f / rough > 0.f && bs.u0 > 0.f) dct_dr = ct * dr_logf(bs.u0) * (-ie * ie) * (-2.f / (rough * rough));
    }
    float st = sqrtf(fmaxf(1.f - ct * ct, 0.f));
    float3 hl = f3(st * cphi, st * sphi, ct);
    float3 h = to_world(f, hl);
    float wh = dot(wi, h), hd = dot(h, d_dir);
    d_wi += 2.f * hd * h - d_dir;
    float3 d_h = 2.f * wh * d_dir + 2.f * hd * wi;
    d_f.t += hl.x * d_h;
    d_f.b += hl.y * d_h;
    d_f.n += hl.z * d_h;
    float3 d_hl = f3(dot(d_h, f.t), dot(d_h, f.b), dot(d_h, f.n));
    float d_ct = d_hl.z;
    if (st > 0.f) d_ct += (d_hl.x * cphi + d_hl.y * sphi) * (-ct / st);
    return d_ct * dct_dr;
}

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

// Geometry adjoints of one path vertex (position, shading frame, uv).
struct VertexGrad {
    float3 dp;
    Frame df;
    float2 duv;
    HD void zero() {
        dp = f3(0.f);
        df = frame_zero();
        duv.x = duv.y = 0.f;
    }
};

// A specular sample (pathtrace.h:141-159 keeps the vertex such a sample
// reaches differentiable): the link from vertex k to vertex k + 1, with what
// the reverse sweep needs of vertex k.
struct SpecLink {
    int tri;        // triangle of vertex k + 1
    int from;       // link that reached vertex k; -1: the first vertex; -2: vertex k is not differentiable
    int mi;         // material of vertex k
    bool flip;      // the sample used vertex k's frame flipped (two-sided back face)
    bool wo_live;   // wo_k = normalize(p_{k+1} - p_k) is differentiable: every sample so far was specular
    float3 o, dir;  // the sampled ray (origin p_k)
    Frame f;        // vertex k's frame as the sample used it
    float3 wi;      // vertex k's incoming direction
    float2 uv;      // vertex k's uv
    BSDFSample bs;  // the sample drawn at vertex k
    VertexGrad vg;  // adjoints of vertex k + 1
    float3 dwo;     // adjoint of wo_k
};

struct NoGrad {
    HD void add(int, float) {}
};

// Normal adjoint of a differentiated intersection: the reference adds the
// first vertex's normal adjoint to all three vertices (delta_ray.cpp:1261-1269).
template <class G> DEV void scatter_tri_normals(const DevScene &s, int tri, float3 dn0, G &g) {
    int4 id = s.tri[tri];
    const DevShape &sh = s.shapes[id.w];
    int b = sh.grad_n - 3 * sh.vtx_off;
    const int v[3] = {id.x, id.y, id.z};
    for (int k = 0; k < 3; k++) {
        g.add(b + 3 * v[k], dn0.x);
        g.add(b + 3 * v[k] + 1, dn0.y);
        g.add(b + 3 * v[k] + 2, dn0.z);
    }
}

// Reverse sweep over links[0..n), last first: vertex k + 1's adjoints go
// through its intersection (hit triangle positions; normals when `normals`)
// and the sampled direction (vertex k's position, frame, uv and incoming
// direction; the roughness texels when `materials`) to vertex k.  The first
// vertex's adjoints end in v0 and d_wi (the primary wi).
template <class G>
DEV void sweep_links(const DevScene &s, SpecLink *links, int n, VertexGrad &v0, float3 &d_wi, bool normals,
                     bool materials, G &g) {
    NoGrad ng;
    for (int l = n - 1; l >= 0; l--) {
        SpecLink &L = links[l];
        TriData td = load_tri(s, L.tri);
        IsectFwd fw;
        SurfacePoint nsp = intersect_tri(td, L.o, L.dir, &fw, true);
        VertexGrad *from = L.from == -1 ? &v0 : (L.from >= 0 ? &links[L.from].vg : nullptr);
        if (L.wo_live && !is_zero(L.dwo)) {
            float3 dv = d_normalize(nsp.p - L.o, L.dwo);
            L.vg.dp += dv;
            if (from) from->dp -= dv;
        }
        TriGrad tg;
        tg.v0 = tg.v1 = tg.v2 = tg.n0 = tg.n1 = tg.n2 = f3(0.f);
        float3 d_o = f3(0.f), d_dir = f3(0.f);
        d_intersect_tri(td, L.o, L.dir, fw, L.vg.dp, f3(0.f), L.vg.df, L.vg.duv, tg, d_o, d_dir);
        scatter_tri_vertices(s, L.tri, tg.v0, tg.v1, tg.v2, g);
        if (normals && td.has_n) scatter_tri_normals(s, L.tri, tg.n0, g);
        if (is_zero(d_dir) && (!from || is_zero(d_o))) continue;
        if (from) from->dp += d_o;
        const DevMaterial &m = s.mats[L.mi];
        Frame dfu = frame_zero();
        float3 dwi_k = f3(0.f);
        float dr = d_specular_direction(s, L.mi, L.f, L.wi, get_rough(s, m, L.uv), L.bs, d_dir, dfu, dwi_k);
        float2 duv;
        duv.x = duv.y = 0.f;
        if (dr != 0.f) {
            if (materials) d_rough(s, m, L.uv, dr, g, duv);
            else d_rough(s, m, L.uv, dr, ng, duv);
        }
        if (from) {
            if (L.flip) dfu = frame_neg(dfu);
            frame_add(from->df, dfu);
            from->duv.x += duv.x;
            from->duv.y += duv.y;
        }
        if (L.from == -1) d_wi += dwi_k;
        else if (L.from >= 0 && links[L.from].wo_live) links[L.from].dwo -= dwi_k;  // wi_k = -wo_{k-1}
    }
}

// Returns the sample's image contribution; accumulates its gradient into g
// and hands every secondary-edge shading point to push_point(const
// PointRecord&): the first vertex and the vertices after it that specular
// samples reached before the first non-specular one (pathtrace.h:218-227).
//
// The reference's AD (pathtrace.h:104-297) keeps the geometry of the first
// vertex and of every vertex reached by a specular sample differentiable; an
// outgoing direction wo_k stays differentiable while every sample so far was
// specular; NEE at every vertex uses the primary wi.  The replay accumulates
// each vertex's local adjoints, then a reverse sweep over the specular links
// pushes vertex k + 1's adjoints through its intersection and the sampled
// direction to vertex k, the roughness and the hit triangle.
// The trace's state before a bounce: where a trace resumes (a checkpoint).
struct PathState {
    Rng r;           // the pixel sample's stream at this bounce
    int ctri;        // the current vertex's triangle
    SurfacePoint csp;
    float3 cwi, thr;  // incoming direction; throughput so far (with roulette)
    bool all_spec;    // every sample so far was specular
};

// Bounce b of the trace (pass 1): the record (next hit, radiance X added at
// this vertex, throughput factor r, roulette probability q), the state moved
// on to the next vertex.  color (may be null) receives the bounce's radiance
// in the trace's own order of additions; push (may be null) the vertex
// reached when it is a secondary-edge shading point.  False when the path
// ends at this bounce (the record is then the last, possibly with a hit).
template <bool kChains, class Push>
DEV bool trace_bounce(const DevScene &s, const LightSample &ls, float3 wi, int b, int B, PathState &ps,
                      BounceRecord &rec, float3 *color, bool want_grad, float3 d_color, uint64_t sid, int light_pick,
                      Push *push) {
    SecondarySample ss = draw_secondary(ps.r);
    float3 N = nee(s, ls, wi, ps.ctri, ps.csp);
    if (color) *color += ps.thr * N;
    rec.next_tri = -1;
    rec.X = N;
    rec.r = f3(0.f);
    rec.q = 1.f;
    bool spec;
    float3 dir = sampled_direction(s, ss.bsdf, ps.cwi, ps.ctri, ps.csp, spec);
    if (abs_sum(dir) <= 0.f) return false;
    Hit bh = trace_closest(s, ps.csp.p, dir, 1e-3f);
    if (bh.tri < 0) return false;
    // a specular sample's hit keeps the reference's AD arithmetic (its
    // position decides which edges a later shading point sees)
    SurfacePoint nsp = intersect_tri(load_tri(s, bh.tri), ps.csp.p, dir, nullptr, spec);
    float3 wo = normalize(nsp.p - ps.csp.p);
    int mi = material_of_tri(s, ps.ctri);
    float pdf = bsdf_pdf(s, mi, ps.csp, ps.cwi, wo);
    if (pdf <= 0.f) return false;
    float3 f = bsdf(s, mi, ps.csp, ps.cwi, wo);
    if (sum(f) <= 0.f) return false;
    rec.next_tri = bh.tri;
    int nli = light_of_tri(s, bh.tri);
    if (nli >= 0 && dot(nsp.f.n, -wo) > 0.f) {
        float lpdf = light_pdf(s, bh.tri) * length_sq(nsp.p - ps.csp.p) / fabsf(dot(wo, nsp.ng));
        float mis = sq(pdf) / (sq(lpdf) + sq(pdf));
        float3 em = f * light_intensity(s, nli) * (mis / pdf);
        if (color) *color += ps.thr * em;
        rec.X += em;
    }
    float3 rb = f / pdf;
    ps.thr = ps.thr * rb;
    if (b >= 5) {
        float q = fminf(max3(ps.thr), 0.95f);
        if (ss.rr >= q) return false;
        ps.thr = ps.thr / q;
        rb = rb / q;
        rec.q = q;
    }
    rec.r = rb;
    ps.all_spec = ps.all_spec && spec;
    ps.cwi = -wo;
    ps.ctri = bh.tri;
    ps.csp = nsp;
    // vertex b + 1 is a secondary-edge shading point while every sample was specular
    if (kChains && push && want_grad && ps.all_spec && b + 1 < B && b + 1 <= DR_MAX_LINKS) {
        PointRecord pr;
        pr.p = nsp.p;
        pr.n = nsp.f.n;
        pr.ng = nsp.ng;
        pr.uv = nsp.uv;
        pr.wi = ps.cwi;
        pr.d_color = d_color * ps.thr;  // the edge weight carries the path throughput
        pr.tri = bh.tri;
        pr.sid = sid;
        pr.light = light_pick;
        pr.bounce = b + 1;
        pr.view = s.view_id;
        (*push)(pr);
    }
    return true;
}

// kChains = false compiles the variant for scenes without specular samples
// (no chain bookkeeping); both give the same result on such scenes.
// BMAX bounds max_bounces at compile time (1 for direct lighting, whose
// variant drops the bounce-record array and the loops' later trips).
template <bool kChains, int BMAX = DR_MAX_BOUNCES, class G, class Push>
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
    const int light_pick =
        sample_discrete(s.light_sel_cdf, s.light_sel_func, s.light_sel_func_int, s.num_lights, ls.sel, nullptr);
    // ---- pass 1: trace, keep the bounces (or checkpoints) ----
    constexpr int CK = BMAX < 0 ? -BMAX : 0;  // segment length of the checkpointed form
    constexpr int NREC = CK ? CK : BMAX;
    constexpr int NCK = CK ? DR_CKPT_SEGS : 1;
    if (B > (CK ? CK * NCK : BMAX)) B = CK ? CK * NCK : BMAX;
    BounceRecord rec[NREC];
    PathState ck[NCK];
    int nb = 0;
    float3 color = f3(0.f);
    int li0 = light_of_tri(s, h0.tri);
    bool prim_emit = li0 >= 0 && dot(sp0.f.n, wi) > 0.f;
    if (prim_emit) color += light_intensity(s, li0);
    bool want_grad = !is_zero(d_color);
    if (want_grad && B >= 1) {
        PointRecord pr;
        pr.p = sp0.p;
        pr.n = sp0.f.n;
        pr.ng = sp0.ng;
        pr.uv = sp0.uv;
        pr.wi = wi;
        pr.d_color = d_color;
        pr.tri = h0.tri;
        pr.sid = sid;
        pr.light = light_pick;
        pr.bounce = 0;
        pr.view = s.view_id;
        push_point(pr);
    }
    PathState ps;
    ps.r = r;
    ps.ctri = h0.tri;
    ps.csp = sp0;
    ps.cwi = wi;
    ps.thr = f3(1.f);
    ps.all_spec = true;
    for (int b = 0; b < B; b++) {
        if (CK && b % (CK ? CK : 1) == 0) ck[b / (CK ? CK : 1)] = ps;
        nb = b + 1;
        if (!trace_bounce<kChains>(s, ls, wi, b, B, ps, rec[CK ? b % (CK ? CK : 1) : b], &color, want_grad, d_color,
                                   sid, light_pick, &push_point))
            break;
    }
    color = color * sw;
    if (!want_grad) return color;  // render_sample_fast: no derivatives, no edges
    // ---- suffix radiance S_{k+1}, stored in rec[k].X ----
    // Checkpointed: a segment's records are traced again from its checkpoint
    // (the same streams, so the same bits); the sweep keeps only the suffix at
    // each segment's start, and pass 2 traces each segment once more.
    float3 sseg[NCK + 1];
    const int nseg = CK ? (nb + (CK ? CK : 1) - 1) / (CK ? CK : 1) : 0;
    auto retrace = [&](int j) {  // rec[0, len) of segment j
        PathState q = ck[j];
        const int b0 = j * (CK ? CK : 1), len = nb - b0 < (CK ? CK : 1) ? nb - b0 : (CK ? CK : 1);
        for (int i = 0; i < len; i++)
            trace_bounce<kChains, Push>(s, ls, wi, b0 + i, B, q, rec[i], nullptr, want_grad, d_color, sid, light_pick,
                                        nullptr);
        return len;
    };
    if (CK) {
        float3 S = f3(0.f);
        sseg[nseg] = S;
        for (int j = nseg - 1; j >= 0; j--) {
            const int len = retrace(j);
            for (int i = len - 1; i >= 0; i--) S = rec[i].X + rec[i].r * S;
            sseg[j] = S;
        }
    } else {
        float3 S = f3(0.f);
        for (int k = nb - 1; k >= 0; k--) {
            float3 Sk = rec[k].X + rec[k].r * S;
            rec[k].X = S;  // now holds S_{k+1}
            S = Sk;
        }
    }
    // ---- pass 2: replay with adjoints ----
    const float3 dC = d_color * sw;
    if (prim_emit) {
        const DevLight &L = s.lights[li0];
        g.add(L.grad + 0, dC.x);
        g.add(L.grad + 1, dC.y);
        g.add(L.grad + 2, dC.z);
    }
    VertexGrad v0g;  // adjoints of the first vertex
    v0g.zero();
    float3 d_wi = f3(0.f);  // adjoint of the primary wi
    SpecLink links[DR_MAX_LINKS];
    int nlinks = 0;
    int vlink = -1;            // link that reached the current vertex (-1: first vertex, or not differentiable)
    bool vlive = true;         // the current vertex's geometry is differentiable
    bool wi_live = true;       // the current vertex's incoming direction is differentiable
    Rng rr = r_sec;
    float3 thr = f3(1.f), cwi = wi;
    int ctri = h0.tri;
    SurfacePoint csp = sp0;
    for (int k = 0; k < nb; k++) {
        if (CK && k % (CK ? CK : 1) == 0) {  // the segment's records, each X turned into S_{k+1}
            const int j = k / (CK ? CK : 1), len = retrace(j);
            float3 S = sseg[j + 1];
            for (int i = len - 1; i >= 0; i--) {
                float3 Si = rec[i].X + rec[i].r * S;
                rec[i].X = S;
                S = Si;
            }
        }
        const BounceRecord &rk = rec[CK ? k % (CK ? CK : 1) : k];
        SecondarySample ss = draw_secondary(rr);
        float3 a = dC * thr;
        VertexGrad *vg = !vlive ? nullptr : (vlink < 0 ? &v0g : &links[vlink].vg);
        {
            SpGrad gn;
            gn.zero();
            float3 dp = f3(0.f);
            d_nee(s, ls, wi, ctri, csp, a, g, gn, dp);
            d_wi += gn.dwi;  // NEE always uses the primary wi (pathtrace.h:213-216)
            if (vg) {
                frame_add(vg->df, gn.df);
                vg->duv.x += gn.duv.x;
                vg->duv.y += gn.duv.y;
                vg->dp += dp;
            }
        }
        int nt = rk.next_tri;
        if (nt < 0) break;
        int mi = material_of_tri(s, ctri);
        SurfacePoint use = csp;
        bool flip = s.mats[mi].two_sided && dot(cwi, csp.f.n) < 0.f;
        if (flip) {
            use.f = frame_neg(csp.f);
            use.ng = -csp.ng;
        }
        bool spec;
        float3 dir = sample_bsdf_dir(s, mi, use, cwi, ss.bsdf, spec);
        SurfacePoint nsp = intersect_tri(load_tri(s, nt), csp.p, dir, nullptr, spec);
        float3 wo = normalize(nsp.p - csp.p);
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
        float3 dr = a * rk.X;
        float q = rk.q;
        if (!is_zero(dr)) {
            d_f += dr * (1.f / (pdf * q));
            d_pdf -= dot(dr, f) / (pdf * pdf * q);
        }
        SpGrad gb;
        gb.zero();
        d_bsdf(s, mi, csp, cwi, wo, d_f, g, gb);
        if (!s.detached_pdf) d_bsdf_pdf(s, mi, csp, cwi, wo, d_pdf, g, gb);
        if (vg) {
            frame_add(vg->df, gb.df);
            vg->duv.x += gb.duv.x;
            vg->duv.y += gb.duv.y;
        }
        // the incoming direction: the primary wi, or -wo_{k-1} while differentiable
        if (k == 0) d_wi += gb.dwi;
        else if (wi_live && vlink >= 0) links[vlink].dwo -= gb.dwi;
        // the vertex this sample reached is differentiable only for a specular sample
        int next_link = -1;
        if (kChains && spec && nlinks < DR_MAX_LINKS) {
            SpecLink &L = links[nlinks];
            L.tri = nt;
            L.from = vlive ? vlink : -2;
            L.mi = mi;
            L.flip = flip;
            L.wo_live = wi_live;
            L.o = csp.p;
            L.dir = dir;
            L.f = use.f;
            L.wi = cwi;
            L.uv = csp.uv;
            L.bs = ss.bsdf;
            L.vg.zero();
            L.dwo = L.wo_live ? gb.dwo : f3(0.f);
            next_link = nlinks++;
        }
        thr = thr * rk.r;
        wi_live = wi_live && spec;
        vlive = next_link >= 0;
        vlink = next_link;
        cwi = -wo;
        ctri = nt;
        csp = nsp;
    }
    if (kChains) sweep_links(s, links, nlinks, v0g, d_wi, true, true, g);
    // ---- first vertex geometry -> triangle and camera ----
    TriGrad tg;
    tg.v0 = tg.v1 = tg.v2 = tg.n0 = tg.n1 = tg.n2 = f3(0.f);
    float3 d_o = f3(0.f), d_d = f3(0.f);
    d_intersect_tri(td0, ray.o, ray.d, fw0, v0g.dp, f3(0.f), v0g.df, v0g.duv, tg, d_o, d_d);
    d_d -= d_wi;
    scatter_tri_vertices(s, h0.tri, tg.v0, tg.v1, tg.v2, g);
    if (td0.has_n) scatter_tri_normals(s, h0.tri, tg.n0, g);
    d_sample_primary(s.cam, sx, sy, d_o, d_d, g, s.cam_off);
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

// Samples the point's edges; emit(tree, edge_index, j, weight, slot_code) for
// every sampled edge of nonzero weight, j its key in the traversal order
// (mode << 27 | edge index: keys grow in the order the reference visits).
// CUT > 0: subtrees at depth CUT go to defer(code, bb, cpmf, apmf, lpmf)
// (EdgeTask fields) instead of being walked here.
template <bool PROP, int CUT = 0, class Emit, class Defer = NoDefer>
DEV bool traverse_point(const DevScene &s, const PointRecord &pt, uint64_t seed, Emit &emit, const EdgeProposal &pr,
                        Defer *defer = nullptr, int *visits = nullptr) {
    Rng prng;
    prng.init(seed, kStreamEdgePoint, pt.sid, (uint32_t)pt.bounce);
    draw_edge(prng);  // the point's edge sample; eval_item redraws it
    NodeRng nrng;
    nrng.seed = seed;
    nrng.sid = pt.sid;
    nrng.bounce = (uint32_t)pt.bounce;
    SurfacePoint sp = pt.surface();
    ConeSpec cone = light_cone(s, pt.light, sp.p);
    auto em = [&](int tree, int ei, int key, float w, int code) {
        if (w != 0.f) emit(tree, ei, key, w, code);
    };
    NoDefer nd;
    if constexpr (CUT > 0)
        return traverse_edges<PROP, CUT>(s, pt.wi, pt.tri, sp, cone, prng, nrng, em, pr, *defer, visits);
    return traverse_edges<PROP, 0>(s, pt.wi, pt.tri, sp, cone, prng, nrng, em, pr, nd, visits);
}

// Starts the walk of one handed-on subtree of the point (see traverse_point).
template <bool PROP>
DEV void start_point_task(EdgeWalk<PROP> &w, const DevScene &s, const PointRecord &pt, uint64_t seed,
                          const EdgeTask &task, const EdgeProposal &pr) {
    NodeRng nrng;
    nrng.seed = seed;
    nrng.sid = pt.sid;
    nrng.bounce = (uint32_t)pt.bounce;
    SurfacePoint sp = pt.surface();
    ConeSpec cone = light_cone(s, pt.light, sp.p);
    start_subtree<PROP>(w, s, pt.wi, pt.tri, sp, cone, nrng, task, pr);
}

// Walks one handed-on subtree of the point to the end.
template <bool PROP, class Emit>
DEV bool traverse_point_task(const DevScene &s, const PointRecord &pt, uint64_t seed, const EdgeTask &task,
                             Emit &emit, const EdgeProposal &pr, int *visits = nullptr) {
    EdgeWalk<PROP> w;
    start_point_task<PROP>(w, s, pt, seed, task, pr);
    auto em = [&](int ei, int key, float wt, int code) {
        if (wt != 0.f) emit(w.tree, ei, key, wt, code);
    };
    NoDefer nd;
    while (w.busy()) w.step(em, nd, visits);
    return w.ok;
}

// One sampled edge (delta_ray.cpp:901-973); returns dp, scatters dv0 / dv1;
// *mag (if given) receives the sample's contribution magnitude |dv0|_1 + |dv1|_1.
// EXT = false compiles the variant without DR_FLAG_EDGE_LOBE_MIS and without
// the magnitude (the kernels choose it when neither is in use).
// The item's line sample (first phase); false: the item contributes nothing.
template <bool EXT = true>
DEV bool item_line(const DevScene &s, const PointRecord &pt, int tree, int ei, uint64_t seed, EdgeLine &el) {
    Rng prng;
    prng.init(seed, kStreamEdgePoint, pt.sid, (uint32_t)pt.bounce);
    EdgeSample es = draw_edge(prng);
    const DevEdge &edge = tree ? s.nrm_edges[ei] : s.sil_edges[ei];
    return edge_line_sample<EXT>(s, es, edge, pt.wi, pt.tri, pt.surface(), el, (tree ? s.nrm_rec : s.sil_rec) + ei);
}

// The item's shading from its line sample; as eval_item.  `hits` (may be
// null): the closest hits of the sample's two rays, which edge_rays kept.
// The two sides' radiance of a kept edge sample (edge_side_radiance), with
// the item's own light sample and random stream as item_shade draws them.
DEV bool item_side_radiance(const DevScene &s, const PointRecord &pt, int tree, int ei, int j, int B,
                            uint64_t seed, const EdgeLine &el, const EdgeHits &hits, float3 &shr, float3 &shl) {
    Rng irng;
    irng.init(seed, kStreamEdgeItem, pt.sid, ((uint32_t)pt.bounce << 28) | (uint32_t)j);
    LightSample els = draw_light(irng);
    const DevEdge &edge = tree ? s.nrm_edges[ei] : s.sil_edges[ei];
    return edge_side_radiance(s, el, edge, els, irng, B - pt.bounce - 1, pt.wi, pt.tri, pt.surface(), hits, shr,
                              shl);
}

// PRE: the sides' radiance `rad` comes from item_side_radiance (see
// edge_shade_hits).
template <bool EXT = true, bool MAYBE_GI = true, class G, bool PRE = false>
DEV float3 item_shade(const DevScene &s, const PointRecord &pt, int tree, int ei, int j, float w, int spp, int B,
                      uint64_t seed, G &g, float *mag, const EdgeLine &el, const EdgeHits *hits = nullptr,
                      const float3 *rad = nullptr) {
    Rng irng;
    irng.init(seed, kStreamEdgeItem, pt.sid, ((uint32_t)pt.bounce << 28) | (uint32_t)j);
    LightSample els = draw_light(irng);
    const DevEdge &edge = tree ? s.nrm_edges[ei] : s.sil_edges[ei];
    float3 weight = f3(1.f) * ((1.f / spp) * w);
    EdgeResult er;
    if constexpr (PRE)
        er = edge_shade_hits<MAYBE_GI, true>(s, el, edge, els, irng, B - pt.bounce - 1, pt.wi, pt.tri, pt.surface(),
                                             weight, pt.d_color, B == 1, *hits, rad);
    else
        er = hits ? edge_shade_hits<MAYBE_GI>(s, el, edge, els, irng, B - pt.bounce - 1, pt.wi, pt.tri, pt.surface(),
                                              weight, pt.d_color, B == 1, *hits)
                  : edge_shade_sample<MAYBE_GI>(s, el, edge, els, irng, B - pt.bounce - 1, pt.wi, pt.tri,
                                                pt.surface(), weight, pt.d_color, B == 1);
    if (EXT && mag) *mag = abs_sum(er.dv0) + abs_sum(er.dv1);
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

template <bool EXT = true, bool MAYBE_GI = true, class G>
DEV float3 eval_item(const DevScene &s, const PointRecord &pt, int tree, int ei, int j, float w, int spp, int B,
                     uint64_t seed, G &g, float *mag = nullptr) {
    EdgeLine el;
    if (!item_line<EXT>(s, pt, tree, ei, seed, el)) {
        if (EXT && mag) *mag = 0.f;
        return f3(0.f);
    }
    return item_shade<EXT, MAYBE_GI>(s, pt, tree, ei, j, w, spp, B, seed, g, mag, el);
}

// dp of a shading point pushed back along its path to the camera and the
// triangles' positions (the second sweep of delta_ray.cpp:975-1002, which
// scatters neither normals nor material parameters).  A point after the first
// vertex was reached by specular samples only: its chain is traced again.
// cam (may be null): the point's camera and camera-gradient offset when it is
// not the scene's (a view of a batched multi-view call).
template <bool kChains, class G>
DEV void propagate_dp(const DevScene &s, const PointRecord &pt, int W, int H, int spp, uint64_t seed, float3 dp, G &g,
                      const DevCamera *cam = nullptr, int cam_off = 0) {
    const DevCamera &pc = cam ? *cam : s.cam;
    const int pco = cam ? cam_off : s.cam_off;
    uint64_t pix = pt.sid / (uint64_t)spp;
    int x = (int)(pix % (uint64_t)W), y = (int)(pix / (uint64_t)W);
    Rng r;
    float sx, sy;
    pixel_sample_position(x, y, W, H, spp, pt.sid, seed, s.full_pixel_jitter != 0, sx, sy, r);
    Ray ray = sample_primary(pc, sx, sy, true);
    VertexGrad v0;
    v0.zero();
    float3 d_wi = f3(0.f);
    int tri0 = pt.tri;
    if (!kChains || pt.bounce == 0) {
        v0.dp = dp;
    } else {
        SpecLink links[DR_MAX_LINKS];
        Hit h = trace_closest(s, ray.o, ray.d, 1e-3f);
        if (h.tri < 0) return;
        tri0 = h.tri;
        SurfacePoint csp = intersect_tri(load_tri(s, h.tri), ray.o, ray.d, nullptr, true);
        float3 cwi = -ray.d;
        int ctri = h.tri;
        draw_light(r);
        if (pt.bounce > DR_MAX_LINKS) return;
        const int n = pt.bounce;
        for (int k = 0; k < n; k++) {
            SecondarySample ss = draw_secondary(r);
            int mi = material_of_tri(s, ctri);
            SurfacePoint use = csp;
            bool flip = s.mats[mi].two_sided && dot(cwi, csp.f.n) < 0.f;
            if (flip) {
                use.f = frame_neg(csp.f);
                use.ng = -csp.ng;
            }
            bool spec;
            float3 dir = sample_bsdf_dir(s, mi, use, cwi, ss.bsdf, spec);
            Hit bh = trace_closest(s, csp.p, dir, 1e-3f);
            if (bh.tri < 0 || !spec) return;  // not the chain that reached the point
            SpecLink &L = links[k];
            L.tri = bh.tri;
            L.from = k - 1;
            L.mi = mi;
            L.flip = flip;
            L.wo_live = true;
            L.o = csp.p;
            L.dir = dir;
            L.f = use.f;
            L.wi = cwi;
            L.uv = csp.uv;
            L.bs = ss.bsdf;
            L.vg.zero();
            L.dwo = f3(0.f);
            SurfacePoint nsp = intersect_tri(load_tri(s, bh.tri), csp.p, dir, nullptr, true);
            cwi = -normalize(nsp.p - csp.p);
            ctri = bh.tri;
            csp = nsp;
        }
        links[n - 1].vg.dp = dp;
        sweep_links(s, links, n, v0, d_wi, false, false, g);
    }
    TriData td = load_tri(s, tri0);
    IsectFwd fw;
    intersect_tri(td, ray.o, ray.d, &fw, true);
    TriGrad tg;
    tg.v0 = tg.v1 = tg.v2 = tg.n0 = tg.n1 = tg.n2 = f3(0.f);
    float3 d_o = f3(0.f), d_d = f3(0.f);
    d_intersect_tri(td, ray.o, ray.d, fw, v0.dp, f3(0.f), v0.df, v0.duv, tg, d_o, d_d);
    d_d -= d_wi;
    scatter_tri_vertices(s, tri0, tg.v0, tg.v1, tg.v2, g);
    d_sample_primary(pc, sx, sy, d_o, d_d, g, pco);
}

// The gradients of one primary-edge sample.
template <class G> DEV void scatter_primary(const DevScene &s, const PrimaryEdgeResult &pr, G &g) {
    if (!pr.ok) return;
    const DevShape &sh = s.shapes[pr.edge.shape];
    g.add(sh.grad_v + 3 * pr.edge.v0 + 0, pr.dv0.x);
    g.add(sh.grad_v + 3 * pr.edge.v0 + 1, pr.dv0.y);
    g.add(sh.grad_v + 3 * pr.edge.v0 + 2, pr.dv0.z);
    g.add(sh.grad_v + 3 * pr.edge.v1 + 0, pr.dv1.x);
    g.add(sh.grad_v + 3 * pr.edge.v1 + 1, pr.dv1.y);
    g.add(sh.grad_v + 3 * pr.edge.v1 + 2, pr.dv1.z);
    for (int q = 0; q < 16; q++) g.add(s.cam_off + 16 + q, pr.dw2c[q]);
}

// Primary-edge sample i (delta_ray.cpp:1478-1522).
template <int BMAX = 1 << 30, class G>
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
    primary_edge_sample<BMAX>(s, es, s.prim_edges[id], ls, r, B, d_image, W, H, w / spp, pr);
    scatter_primary(s, pr, g);
}

// The primary-edge sample i in two halves (k_primary_shade, k_primary_grad),
// with the same draws and arithmetic as primary_edge_item.  The first returns
// (rcol - lcol, 1), or w = 0 when the sample ends before its gradient.
template <int BMAX>
DEV float4 primary_shade_item(const DevScene &s, long long i, int B, uint64_t seed) {
    float4 none;
    none.x = none.y = none.z = none.w = 0.f;
    if (s.num_prim_edges == 0) return none;
    Rng r;
    r.init(seed, kStreamPrimaryEdge, (uint64_t)i, 0);
    float pmf = 0.f;
    int id = sample_discrete(s.prim_cdf, s.prim_func, s.prim_func_int, s.num_prim_edges, r.next(), &pmf);
    float w = pmf > 0.f ? 1.f / pmf : 0.f;
    if (w <= 0.f) return none;
    EdgeSample es = draw_edge(r);
    LightSample ls = draw_light(r);
    PrimaryGeom pg;
    if (!primary_edge_geom(s.cam, s, es, s.prim_edges[id], pg)) return none;
    float3 diff;
    if (!primary_edge_colors<BMAX>(s, pg, s.prim_edges[id], ls, r, B, diff)) return none;
    float4 c;
    c.x = diff.x;
    c.y = diff.y;
    c.z = diff.z;
    c.w = 1.f;
    return c;
}

template <class G>
DEV void primary_grad_item(const DevScene &s, long long i, int W, int H, int spp, uint64_t seed, const float *d_image,
                           float4 c, G &g) {
    if (c.w == 0.f) return;
    Rng r;
    r.init(seed, kStreamPrimaryEdge, (uint64_t)i, 0);
    float pmf = 0.f;
    int id = sample_discrete(s.prim_cdf, s.prim_func, s.prim_func_int, s.num_prim_edges, r.next(), &pmf);
    float w = 1.f / pmf;
    EdgeSample es = draw_edge(r);
    PrimaryGeom pg;
    primary_edge_geom(s.cam, s, es, s.prim_edges[id], pg);
    PrimaryEdgeResult pr;
    primary_edge_grad(s, pg, s.prim_edges[id], f3(c.x, c.y, c.z), d_image, W, H, w / spp, pr);
    scatter_primary(s, pr, g);
}
