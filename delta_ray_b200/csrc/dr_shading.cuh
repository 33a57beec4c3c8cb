// Forward light transport: camera rays, materials, lights and the path tracer.
//
// Semantics (including the reference's quirks) follow, function by function:
//   sample_primary     camera.h:48-84
//   tex lookups        material.h:84-239 (bilinear, wrap-around, uv scaling)
//   bsdf               material.h:257-351 (Lambert + Blinn-Phong, rational
//                      Smith G1, Schlick Fresnel)
//   sample_bsdf_dir    material.h:353-412 (lobe chosen by luminance; "specular"
//                      only when roughness <= 0.01)
//   bsdf_pdf           material.h:414-462
//   sample_light/pdf   scene.h:49-108, sample.h:6-24
//   eval / nee         pathtrace.h:7-102 (MIS weights are constants)
//   shade              pathtrace.h:179-297 (NEE at every bounce uses the
//                      *primary* light sample and the *primary* wi; Russian
//                      roulette from bounce 5)
#pragma once

#include "dr_trace.cuh"

#ifdef DR_HOST_BUILD
#include <cmath>
HD bool dr_isfinite(float x) { return std::isfinite(x); }
#else
DEV bool dr_isfinite(float x) { return isfinite(x); }
#endif

DEV bool is_light_tri(const DevScene &s, int tri) { return s.shapes[s.tri[tri].w].light >= 0; }
DEV int light_of_tri(const DevScene &s, int tri) { return s.shapes[s.tri[tri].w].light; }
DEV int material_of_tri(const DevScene &s, int tri) { return s.shapes[s.tri[tri].w].mat; }

// ---------------------------------------------------------------------------
// Camera
// ---------------------------------------------------------------------------
struct Ray { float3 o, d; };

// `ad`: use the arithmetic of the reference's differentiated pass, where a
// division by a differentiable value is a multiply by its reciprocal
// (autodiff.h:161-186); the backward pass needs those exact bits for the
// shading point that edge sampling starts from.
// Fisheye branches of the camera routines are out of line: they are rarely
// taken and their trigonometry is large.  r.d = 0 outside the image circle.
DEV_NOINLINE float3 fisheye_dir(float sx, float sy) {
    float x = 2.f * (sx - 0.5f), y = 2.f * (sy - 0.5f);
    if (x * x + y * y > 1.f) return f3(0.f);
    float rr = sqrtf(x * x + y * y);
    float phi = dr_atan2f(y, x);
    float theta = rr * DR_PI / 2.f;
    float3 dir = f3(-dr_cosf(phi) * dr_sinf(theta), -dr_sinf(phi) * dr_sinf(theta), dr_cosf(theta));
    return normalize(dir);
}

DEV Ray sample_primary(const DevCamera &c, float sx, float sy, bool ad = false) {
    Ray r;
    r.o = xfm_point(c.c2w, f3(0.f));
    if (c.fisheye) {
        float3 d = fisheye_dir(sx, sy);
        r.d = is_zero(d) ? d : xfm_vector(c.c2w, d);
        return r;
    }
    float ndcx = (sx - 0.5f) * -2.f;
    float ndcy = ad ? ((sy - 0.5f) * -2.f) * (1.f / c.aspect) : (sy - 0.5f) * -2.f / c.aspect;
    float3 dir = f3(c.fov * ndcx, c.fov * ndcy, 1.f);
    r.d = xfm_vector(c.c2w, normalize(dir));
    return r;
}

// ---------------------------------------------------------------------------
// Materials
// ---------------------------------------------------------------------------
HD int modulo(int a, int b) {
    int r = a % b;
    return r < 0 ? r + b : r;
}

struct TexFoot {  // bilinear footprint of one lookup (for the adjoint)
    int xf, yf;   // wrapped floor texel
    int xc, yc;   // wrapped ceil texel
    float u, v;   // fractional position
};

DEV TexFoot tex_foot(int w, int h, float2 uv) {
    TexFoot t;
    int xf = (int)floorf(uv.x * w), yf = (int)floorf(uv.y * h);
    t.u = (uv.x * (float)w) - (float)xf;
    t.v = (uv.y * (float)h) - (float)yf;
    t.xf = modulo(xf, w);
    t.yf = modulo(yf, h);
    t.xc = modulo(xf + 1, w);
    t.yc = modulo(yf + 1, h);
    return t;
}

DEV float tex_fetch(const DevScene &s, int off, int w, int ch, int y, int x, int c) {
    return dr_ldg(s.texels + off + (y * w + x) * ch + c);
}

// Bilinear lookups out of line (called from many sites); constants inline.
DEV_NOINLINE float3 tex3_bilinear(const DevScene &s, int off, int w, int h, float2 uv) {
    TexFoot t = tex_foot(w, h, uv);
    float3 r;
    for (int c = 0; c < 3; c++) {
        float ff = tex_fetch(s, off, w, 3, t.yf, t.xf, c), fc = tex_fetch(s, off, w, 3, t.yc, t.xf, c);
        float cf = tex_fetch(s, off, w, 3, t.yf, t.xc, c), cc = tex_fetch(s, off, w, 3, t.yc, t.xc, c);
        comp_set(r, c, ff * (1.f - t.u) * (1.f - t.v) + fc * (1.f - t.u) * t.v + cf * t.u * (1.f - t.v) + cc * t.u * t.v);
    }
    return r;
}
DEV float3 tex3(const DevScene &s, int off, int w, int h, const float *cval, float2 uv) {
    if (off < 0) return f3(cval[0], cval[1], cval[2]);
    return tex3_bilinear(s, off, w, h, uv);
}

DEV_NOINLINE float tex1_bilinear(const DevScene &s, int off, int w, int h, float2 uv) {
    TexFoot t = tex_foot(w, h, uv);
    float ff = tex_fetch(s, off, w, 1, t.yf, t.xf, 0), fc = tex_fetch(s, off, w, 1, t.yc, t.xf, 0);
    float cf = tex_fetch(s, off, w, 1, t.yf, t.xc, 0), cc = tex_fetch(s, off, w, 1, t.yc, t.xc, 0);
    return ff * (1.f - t.u) * (1.f - t.v) + fc * (1.f - t.u) * t.v + cf * t.u * (1.f - t.v) + cc * t.u * t.v;
}
DEV float tex1(const DevScene &s, int off, int w, int h, float cval, float2 uv) {
    if (off < 0) return cval;
    return tex1_bilinear(s, off, w, h, uv);
}

DEV float2 scale_uv(float2 uv, const float *sc) {
    float2 r;
    r.x = uv.x * sc[0];
    r.y = uv.y * sc[1];
    return r;
}
DEV float3 get_kd(const DevScene &s, const DevMaterial &m, float2 uv) {
    return tex3(s, m.tex_kd, m.kd_w, m.kd_h, m.kd, scale_uv(uv, m.uv_kd));
}
DEV float3 get_ks(const DevScene &s, const DevMaterial &m, float2 uv) {
    return tex3(s, m.tex_ks, m.ks_w, m.ks_h, m.ks, scale_uv(uv, m.uv_ks));
}
DEV float get_rough(const DevScene &s, const DevMaterial &m, float2 uv) {
    return tex1(s, m.tex_r, m.r_w, m.r_h, m.rough, scale_uv(uv, m.uv_r));
}
DEV float roughness_to_phong(float r) { return fmaxf(2.f / r, 0.f); }

// rational approximation of the Smith G1 term with the "projected roughness"
// of material.h:305-335
DEV float smith_g1(const Frame &f, float3 n, float3 m, float3 v, float rough) {
    float c = dot(v, n);
    if (dot(v, m) * c <= 0.f) return 0.f;
    float tan_t = sqrtf(fmaxf(1.f / (c * c) - 1.f, 0.f));
    if (tan_t == 0.f) return 1.f;
    float3 vl = to_local(f, v);
    float s2 = 1.f - vl.z * vl.z;
    float alpha;
    if (s2 <= 0.f) {
        alpha = sqrtf(rough);
    } else {
        float inv = 1.f / s2;
        alpha = sqrtf(vl.x * vl.x * inv * rough + vl.y * vl.y * inv * rough);
    }
    float a = 1.f / (alpha * tan_t);
    if (a >= 1.6f) return 1.f;
    float a2 = a * a;
    return (3.535f * a + 2.181f * a2) / (1.0f + 2.276f * a + 2.577f * a2);
}

// GGX lobe (Walter et al. 2007, "Microfacet Models for Refraction through
// Rough Surfaces"; no counterpart in the reference): alpha = max(r^2, 1e-4),
// A = alpha^2, D(h) = A / (pi ((n.h)^2 (A - 1) + 1)^2), exact Smith G1.
DEV float ggx_A(float rough) {
    float a = fmaxf(rough * rough, 1e-4f);
    return a * a;
}
DEV float ggx_D(float z, float A) {
    float k = z * z * (A - 1.f) + 1.f;
    return A / (DR_PI * k * k);
}
DEV float ggx_g1(float3 n, float3 m, float3 v, float A) {
    float c = dot(v, n);
    if (dot(v, m) * c <= 0.f) return 0.f;
    float t2 = fmaxf(1.f / (c * c) - 1.f, 0.f);
    return 2.f / (1.f + sqrtf(1.f + A * t2));
}

DEV float3 bsdf(const DevScene &s, int mi, const SurfacePoint &sp, float3 wi, float3 wo) {
    const DevMaterial &m = s.mats[mi];
    float3 n = sp.f.n;
    if (m.two_sided && dot(wi, n) < 0.f) n = -n;
    float bcos = dot(n, wo);
    if (bcos <= 5e-3f) return f3(0.f);
    float3 kd = get_kd(s, m, sp.uv), ks = get_ks(s, m, sp.uv);
    float rough = get_rough(s, m, sp.uv);
    float3 res = kd * bcos / DR_PI;
    if (sum(ks) > 0.f && dot(wi, n) > 0.f) {
        float3 h = normalize(wi + wo);
        float3 hl = to_local(sp.f, h);
        if (hl.z > 0.f) {
            float D, G;
            if (m.model == DR_MICROFACET_GGX) {
                float A = ggx_A(rough);
                D = ggx_D(hl.z, A);
                G = ggx_g1(n, h, wi, A) * ggx_g1(n, h, wo, A);
            } else {
                float e = roughness_to_phong(rough);
                D = dr_powf(fmaxf(hl.z, 0.f), e) * (e + 2.f) / float(2 * 3.14159265358979323846);
                G = smith_g1(sp.f, n, h, wi, rough) * smith_g1(sp.f, n, h, wo, rough);
            }
            float cd = dot(h, wo);
            float fr = dr_powf(fmaxf(1.f - cd, 0.f), 5.f);
            float3 F = f3(ks.x + (1.f - ks.x) * fr, ks.y + (1.f - ks.y) * fr, ks.z + (1.f - ks.z) * fr);
            res += F * D * G / (4.f * dot(wi, n));
        }
    }
    return res;
}

DEV float bsdf_pdf(const DevScene &s, int mi, const SurfacePoint &sp, float3 wi, float3 wo) {
    const DevMaterial &m = s.mats[mi];
    float3 kd = get_kd(s, m, sp.uv), ks = get_ks(s, m, sp.uv);
    float dw = luminance(kd), sw = luminance(ks), ws = dw + sw;
    if (ws <= 0.f) return 0.f;
    float dpmf = dw / ws, spmf = sw / ws;
    float dpdf = 0.f;
    if (dpmf > 0.f) {
        float c = dot(sp.f.n, wo);
        c = m.two_sided ? fabsf(c) : fmaxf(c, 0.f);
        dpdf = dpmf * c / DR_PI;
    }
    float spdf = 0.f;
    if (spmf > 0.f) {
        float3 h = normalize(wi + wo);
        float3 hl = to_local(sp.f, h);
        if (hl.z > 0.f) {
            if (m.model == DR_MICROFACET_GGX) {
                // half vectors are drawn with density D(h) (n.h)
                float D = ggx_D(hl.z, ggx_A(get_rough(s, m, sp.uv)));
                spdf = spmf * D * hl.z / (4.f * fabsf(dot(wo, h)));
            } else {
                float e = roughness_to_phong(get_rough(s, m, sp.uv));
                float D = dr_powf(hl.z, e) * (e + 2.f) / float(2 * 3.14159265358979323846);
                spdf = spmf * D / (4.f * fabsf(dot(wo, h)));
            }
        }
    }
    return dpdf + spdf;
}

DEV float3 cos_hemisphere(float u0, float u1) {  // vector.h:533-538
    float phi = 2.f * DR_PI * u0;
    float tmp = sqrtf(1.f - u1);
    return f3(dr_cosf(phi) * tmp, dr_sinf(phi) * tmp, sqrtf(u1));
}

// Direction sampled at a surface point (material-level sample_bsdf).
DEV float3 sample_bsdf_dir(const DevScene &s, int mi, const SurfacePoint &sp, float3 wi, const BSDFSample &bs,
                           bool &specular) {
    const DevMaterial &m = s.mats[mi];
    specular = false;
    float3 kd = get_kd(s, m, sp.uv), ks = get_ks(s, m, sp.uv);
    float dw = luminance(kd), sw = luminance(ks), ws = dw + sw;
    if (ws <= 0.f) return f3(0.f);
    float dpmf = dw / ws;
    if (bs.w <= dpmf) {
        if (dpmf <= 0.f) return f3(0.f);
        return to_world(sp.f, cos_hemisphere(bs.u0, bs.u1));
    }
    if (sw <= 0.f) return f3(0.f);
    float rough = get_rough(s, m, sp.uv);
    float phi = 2.f * DR_PI * bs.u1;
    float sphi = dr_sinf(phi), cphi = dr_cosf(phi);
    float ct;
    if (m.model == DR_MICROFACET_GGX) {
        float A = ggx_A(rough);
        ct = sqrtf((1.f - bs.u0) / (1.f + (A - 1.f) * bs.u0));
    } else {
        ct = dr_powf(bs.u0, 1.0f / (roughness_to_phong(rough) + 2.0f));
    }
    float st = sqrtf(fmaxf(1.f - ct * ct, 0.f));
    float3 h = to_world(sp.f, f3(st * cphi, st * sphi, ct));
    specular = rough <= 0.01f;
    return 2.f * dot(wi, h) * h - wi;
}

// ---------------------------------------------------------------------------
// Lights
// ---------------------------------------------------------------------------
struct LightPoint {
    int tri;  // global triangle id
    int light;
    float b1, b2;  // barycentric weights of e1, e2
    SurfacePoint sp;
};

DEV LightPoint sample_light_point(const DevScene &s, const LightSample &ls) {
    LightPoint lp;
    lp.light = sample_discrete(s.light_sel_cdf, s.light_sel_func, s.light_sel_func_int, s.num_lights, ls.sel, nullptr);
    const DevLight &L = s.lights[lp.light];
    int ti = sample_discrete(s.light_tri_cdf + L.cdf_off, s.light_tri_func + L.cdf_off, L.func_int, L.ntri,
                             ls.tri_sel, nullptr);
    lp.tri = s.shapes[L.shape].tri_off + ti;
    int4 id = s.tri[lp.tri];
    float3 v0 = vtx3(s.vtx, id.x), v1 = vtx3(s.vtx, id.y), v2 = vtx3(s.vtx, id.z);
    float a = sqrtf(ls.u0);
    lp.b1 = 1.f - a;
    lp.b2 = a * ls.u1;
    float3 e1 = v1 - v0, e2 = v2 - v0;
    float3 nn = normalize(cross(e1, e2));
    lp.sp.p = v0 + e1 * lp.b1 + e2 * lp.b2;
    lp.sp.ng = nn;
    lp.sp.f = make_frame(nn);
    lp.sp.uv.x = ls.u0;
    lp.sp.uv.y = ls.u1;
    return lp;
}

DEV float light_pdf(const DevScene &s, int tri) {
    if (tri < 0) return 0.f;
    int li = light_of_tri(s, tri);
    if (li < 0) return 0.f;
    const DevLight &L = s.lights[li];
    float lpmf = luminance(f3(L.I[0], L.I[1], L.I[2])) / s.total_light_intensity;
    int4 id = s.tri[tri];
    float3 v0 = vtx3(s.vtx, id.x), v1 = vtx3(s.vtx, id.y), v2 = vtx3(s.vtx, id.z);
    float area = 0.5f * length(cross(v1 - v0, v2 - v0));
    float tri_pmf = area / L.area;
    return lpmf * tri_pmf / area;
}

DEV float3 light_intensity(const DevScene &s, int li) {
    const DevLight &L = s.lights[li];
    return f3(L.I[0], L.I[1], L.I[2]);
}

// contribution of a point on an emitter (pathtrace.h:7-57); shadow ray tested
DEV float3 eval_light(const DevScene &s, float3 wi, int stri, const SurfacePoint &sp, int ltri, const SurfacePoint &lp) {
    if (stri < 0 || ltri < 0) return f3(0.f);
    int li = light_of_tri(s, ltri);
    if (li < 0) return f3(0.f);
    float3 dv = lp.p - sp.p;
    float dist = length(dv);
    if (dist == 0.f) return f3(0.f);
    float3 nd = dv / dist;
    if (occluded(s, sp.p, nd, dist)) return f3(0.f);
    float3 b = bsdf(s, material_of_tri(s, stri), sp, wi, nd);
    float lcos = dot(lp.f.n, -nd);
    if (lcos <= 0.f) return f3(0.f);
    float d2 = sq(dist);
    float3 lc = light_intensity(s, li) * (lcos / d2);
    return b * lc;
}

// next_event_estimation (pathtrace.h:59-102)
DEV float3 nee(const DevScene &s, const LightSample &ls, float3 wi, int stri, const SurfacePoint &sp) {
    if (stri < 0) return f3(0.f);
    LightPoint lp = sample_light_point(s, ls);
    float3 ldir = normalize(lp.sp.p - sp.p);
    float lcos = fabsf(dot(ldir, lp.sp.ng));
    float lpdf = light_pdf(s, lp.tri);
    float bpdf = bsdf_pdf(s, material_of_tri(s, stri), sp, wi, ldir) * lcos / length_sq(lp.sp.p - sp.p);
    float mis = sq(lpdf) / (sq(bpdf) + sq(lpdf));
    return eval_light(s, wi, stri, sp, lp.tri, lp.sp) * (mis / lpdf);
}

// Scene-level BSDF sampling with the two-sided flip (pathtrace.h:104-162).
// Returns the hit (tri = -1 on a miss or a black BSDF) and the hit point.
struct BounceHit {
    int tri;
    bool specular;
    float3 dir;
    SurfacePoint sp;
};

DEV BounceHit sample_bsdf_scene(const DevScene &s, const BSDFSample &bs, float3 wi, int stri, const SurfacePoint &sp) {
    BounceHit bh;
    bh.tri = -1;
    bh.specular = false;
    if (stri < 0) return bh;
    int mi = material_of_tri(s, stri);
    SurfacePoint use = sp;
    if (s.mats[mi].two_sided && dot(wi, sp.f.n) < 0.f) {
        use.f = frame_neg(sp.f);
        use.ng = -sp.ng;
    }
    bool spec;
    float3 dir = sample_bsdf_dir(s, mi, use, wi, bs, spec);
    if (length(dir) <= 0.f) return bh;
    Hit h = trace_closest(s, use.p, dir, 1e-3f);
    if (h.tri < 0) return bh;
    bh.tri = h.tri;
    bh.specular = spec;
    bh.dir = dir;
    bh.sp = intersect_tri(load_tri(s, h.tri), use.p, dir);
    return bh;
}

// shade (pathtrace.h:179-297), forward only.  `rng` is positioned at the first
// secondary sample; it is taken by value so callers can replay the same draws.
// BMAX bounds max_bounces at compile time (1: the direct-lighting variant).
template <int BMAX = 1 << 30>
DEV float3 shade(const DevScene &s, float3 wi, int ptri, const SurfacePoint &psp, const LightSample &ls, Rng rng,
                 int max_bounces, bool include_primary_light) {
    if (max_bounces > BMAX) max_bounces = BMAX;
    float3 color = f3(0.f);
    if (ptri < 0) return color;
    if (include_primary_light) {
        int li = light_of_tri(s, ptri);
        if (li >= 0 && dot(psp.f.n, wi) > 0.f) color += light_intensity(s, li);
    }
    float3 thr = f3(1.f);
    float3 cwi = wi;
    int ctri = ptri;
    SurfacePoint csp = psp;
    for (int b = 0; b < max_bounces; b++) {
        SecondarySample ss = draw_secondary(rng);
        color += thr * nee(s, ls, wi, ctri, csp);
        BounceHit bh = sample_bsdf_scene(s, ss.bsdf, cwi, ctri, csp);
        if (bh.tri < 0) break;
        float3 wo = normalize(bh.sp.p - csp.p);
        int mi = material_of_tri(s, ctri);
        float pdf = bsdf_pdf(s, mi, csp, cwi, wo);
        if (pdf <= 0.f) break;
        float3 be = bsdf(s, mi, csp, cwi, wo);
        if (sum(be) <= 0.f) break;
        int nli = light_of_tri(s, bh.tri);
        if (nli >= 0 && dot(bh.sp.f.n, -wo) > 0.f) {
            float3 contrib = be * light_intensity(s, nli);
            float lpdf = light_pdf(s, bh.tri) * length_sq(bh.sp.p - csp.p) / fabsf(dot(wo, bh.sp.ng));
            float mis = sq(pdf) / (sq(lpdf) + sq(pdf));
            color += thr * contrib * (mis / pdf);
        }
        thr = thr * (be / pdf);
        if (b >= 5) {
            float q = fminf(max3(thr), 0.95f);
            if (ss.rr >= q) break;
            thr = thr / q;
        }
        cwi = -wo;
        ctri = bh.tri;
        csp = bh.sp;
    }
    return color;
}

// One pixel sample's radiance contribution (render_sample_fast,
// delta_ray.cpp:640-692; sub-pixel jitter in [0, 1/spp) as :1236-1237).
DEV float3 pixel_sample(const DevScene &s, int x, int y, int W, int H, int spp, int si, int B, uint64_t seed) {
    Rng r;
    r.init(seed, kStreamPixel, ((uint64_t)y * W + x) * spp + si, 0);
    float ux = r.next(), uy = r.next();
    float sub_x = s.full_pixel_jitter ? ux : ux / spp;
    float sub_y = s.full_pixel_jitter ? uy : uy / spp;
    Ray ray = sample_primary(s.cam, float((x + sub_x) / W), float((y + sub_y) / H));
    if (abs_sum(ray.d) == 0.f) return f3(0.f);
    Hit h = trace_closest(s, ray.o, ray.d, 1e-3f);
    if (h.tri < 0) return f3(0.f);
    SurfacePoint sp = intersect_tri(load_tri(s, h.tri), ray.o, ray.d);
    LightSample ls = draw_light(r);
    float3 c = shade(s, -ray.d, h.tri, sp, ls, r, B, true);
    return c * (1.f / spp);
}
