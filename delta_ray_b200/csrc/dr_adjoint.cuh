// Hand-written adjoints of the forward light-transport functions.
//
// The reference differentiates with a per-sample tape (autodiff.h); these
// functions compute the same partial derivatives directly: each d_* function
// recomputes the forward intermediates it needs and walks its statements in
// reverse, with the derivative rules of autodiff.h:84-324 (including its
// conventions at kinks: fabs, max and min pass the gradient to the selected
// operand, dr_powf(x, a) differentiates a through dr_logf(max(x, 1e-6))).
//
// Gradients are written through a sink `G` with add(flat_index, value); the
// flat layout is the C ABI's (camera at 0, then materials, shapes, lights).
#pragma once

#include "dr_shading.cuh"

#define DR_INV_2PI (1.f / float(2 * 3.14159265358979323846))

// Adjoints of a shading point's inputs collected by the material functions.
struct SpGrad {
    Frame df;     // shading frame
    float2 duv;   // uv (through textures)
    float3 dwi;   // incoming direction
    float3 dwo;   // outgoing direction
    HD void zero() {
        df = frame_zero();
        duv.x = duv.y = 0.f;
        dwi = f3(0.f);
        dwo = f3(0.f);
    }
};

// d/d(value) of one material channel (constant or bilinear texture): texel
// adjoints go to the flat gradient where delta_ray.cpp:1362-1441 puts them
// (the floor-floor texel's adjoint lands on the ceil-ceil texel and so on),
// the uv adjoint is returned through d_uv.  `finite_only` skips non-finite
// contributions as delta_ray.cpp:846-851 does for constant roughness.
// the texel part, out of line (many call sites)
template <class G>
DEV_NOINLINE void d_tex_texels(const DevScene &s, int off, int w, int h, int ch, int grad_base, const float *uv_scale,
                               float2 uv, const float *dval, G &g, float2 &d_uv) {
    float2 su = scale_uv(uv, uv_scale);
    TexFoot t = tex_foot(w, h, su);
    float du = 0.f, dv = 0.f;
    for (int c = 0; c < ch; c++) {
        float d = dval[c];
        if (d == 0.f) continue;
        float ff = tex_fetch(s, off, w, ch, t.yf, t.xf, c), fc = tex_fetch(s, off, w, ch, t.yc, t.xf, c);
        float cf = tex_fetch(s, off, w, ch, t.yf, t.xc, c), cc = tex_fetch(s, off, w, ch, t.yc, t.xc, c);
        g.add(grad_base + (t.yc * w + t.xc) * ch + c, d * (1.f - t.u) * (1.f - t.v));
        g.add(grad_base + (t.yc * w + t.xf) * ch + c, d * (1.f - t.u) * t.v);
        g.add(grad_base + (t.yf * w + t.xc) * ch + c, d * t.u * (1.f - t.v));
        g.add(grad_base + (t.yf * w + t.xf) * ch + c, d * t.u * t.v);
        du += d * (-ff * (1.f - t.v) - fc * t.v + cf * (1.f - t.v) + cc * t.v);
        dv += d * (-ff * (1.f - t.u) + fc * (1.f - t.u) - cf * t.u + cc * t.u);
    }
    d_uv.x += du * (float)w * uv_scale[0];
    d_uv.y += dv * (float)h * uv_scale[1];
}
template <class G>
DEV void d_tex_channel(const DevScene &s, int off, int w, int h, int ch, int grad_base, const float *uv_scale,
                       float2 uv, const float *dval, G &g, float2 &d_uv, bool finite_only) {
    if (off < 0) {
        for (int c = 0; c < ch; c++) {
            float v = dval[c];
            if (finite_only && !dr_isfinite(v)) continue;
            g.add(grad_base + c, v);
        }
        return;
    }
    d_tex_texels(s, off, w, h, ch, grad_base, uv_scale, uv, dval, g, d_uv);
}

template <class G> DEV void d_kd(const DevScene &s, const DevMaterial &m, float2 uv, float3 d, G &g, float2 &duv) {
    float v[3] = {d.x, d.y, d.z};
    d_tex_channel(s, m.tex_kd, m.kd_w, m.kd_h, 3, m.grad_kd, m.uv_kd, uv, v, g, duv, false);
}
template <class G> DEV void d_ks(const DevScene &s, const DevMaterial &m, float2 uv, float3 d, G &g, float2 &duv) {
    float v[3] = {d.x, d.y, d.z};
    d_tex_channel(s, m.tex_ks, m.ks_w, m.ks_h, 3, m.grad_ks, m.uv_ks, uv, v, g, duv, false);
}
template <class G> DEV void d_rough(const DevScene &s, const DevMaterial &m, float2 uv, float d, G &g, float2 &duv) {
    d_tex_channel(s, m.tex_r, m.r_w, m.r_h, 1, m.grad_r, m.uv_r, uv, &d, g, duv, true);
}

// adjoint of smith_g1(f, n, m, v, rough) (material.h:305-335)
DEV void d_smith_g1(const Frame &f, float3 n, float3 m, float3 v, float rough, float d_out, Frame &df, float3 &dn,
                    float3 &dm, float3 &dv, float &dr) {
    float c = dot(v, n);
    if (dot(v, m) * c <= 0.f) return;
    float tan_t = sqrtf(fmaxf(1.f / (c * c) - 1.f, 0.f));
    if (tan_t == 0.f) return;
    float3 vl = to_local(f, v);
    float s2 = 1.f - vl.z * vl.z;
    float alpha, inv = 0.f, cp2 = 0.f, sp2 = 0.f;
    if (s2 <= 0.f) {
        alpha = sqrtf(rough);
    } else {
        inv = 1.f / s2;
        cp2 = vl.x * vl.x * inv;
        sp2 = vl.y * vl.y * inv;
        alpha = sqrtf(cp2 * rough + sp2 * rough);
    }
    float q = alpha * tan_t;
    float a = 1.f / q;
    if (a >= 1.6f) return;
    float a2 = a * a;
    float num = 3.535f * a + 2.181f * a2, den = 1.0f + 2.276f * a + 2.577f * a2;
    float d_num = d_out / den, d_den = -d_out * num / (den * den);
    float d_a = 3.535f * d_num + 2.276f * d_den;
    float d_a2 = 2.181f * d_num + 2.577f * d_den;
    d_a += 2.f * a * d_a2;
    float d_q = -d_a / (q * q);
    float d_alpha = d_q * tan_t, d_tan = d_q * alpha;
    if (s2 <= 0.f) {
        dr += d_alpha * 0.5f / alpha;
    } else {
        float d_w2 = d_alpha * 0.5f / alpha;
        dr += d_w2 * (cp2 + sp2);
        float d_cp2 = d_w2 * rough, d_sp2 = d_w2 * rough;
        float3 dvl = f3(d_cp2 * inv * 2.f * vl.x, d_sp2 * inv * 2.f * vl.y, 0.f);
        float d_inv = d_cp2 * vl.x * vl.x + d_sp2 * vl.y * vl.y;
        float d_s2 = -d_inv * inv * inv;
        dvl.z += d_s2 * (-2.f * vl.z);
        d_to_local(f, v, dvl, df, dv);
    }
    float d_t2 = d_tan * 0.5f / tan_t;
    float cc = c * c;
    float d_cc = -d_t2 / (cc * cc);
    float d_c = d_cc * 2.f * c;
    dv += d_c * n;
    dn += d_c * v;
}

// adjoint of ggx_g1(n, m, v, A): G1 = 2 / (1 + S), S = sqrt(1 + A t2),
// t2 = 1 / c^2 - 1, c = v.n
DEV void d_ggx_g1(float3 n, float3 m, float3 v, float A, float d_out, float3 &dn, float3 &dv, float &dA) {
    float c = dot(v, n);
    if (dot(v, m) * c <= 0.f) return;
    float q = 1.f / (c * c) - 1.f;
    float t2 = fmaxf(q, 0.f);
    float S = sqrtf(1.f + A * t2);
    float dS = d_out * (-2.f / ((1.f + S) * (1.f + S)));
    float d_t2 = dS * A / (2.f * S);
    dA += dS * t2 / (2.f * S);
    if (q > 0.f) {
        float d_c = d_t2 * (-2.f / (c * c * c));
        dv += d_c * n;
        dn += d_c * v;
    }
}

// partial derivatives of ggx_D(z, A) = A / (pi k^2), k = z^2 (A - 1) + 1
DEV void ggx_D_partials(float z, float A, float &dDdz, float &dDdA) {
    float k = z * z * (A - 1.f) + 1.f;
    float ik3 = 1.f / (DR_PI * k * k * k);
    dDdz = -4.f * A * z * (A - 1.f) * ik3;
    dDdA = (k - 2.f * A * z * z) * ik3;
}

// d A / d roughness of ggx_A (A = r^4 above the clamp)
DEV float ggx_dA_drough(float rough) {
    float r2 = rough * rough;
    return r2 > 1e-4f ? 4.f * r2 * rough : 0.f;
}

// adjoint of bsdf (material.h:257-351); accumulates into sg and the material gradient
template <class G>
DEV void d_bsdf(const DevScene &s, int mi, const SurfacePoint &sp, float3 wi, float3 wo, float3 d_out, G &g,
                SpGrad &sg) {
    if (is_zero(d_out)) return;
    const DevMaterial &m = s.mats[mi];
    float sgn = (m.two_sided && dot(wi, sp.f.n) < 0.f) ? -1.f : 1.f;
    float3 n = sp.f.n * sgn;
    float bcos = dot(n, wo);
    if (bcos <= 5e-3f) return;
    float3 kd = get_kd(s, m, sp.uv), ks = get_ks(s, m, sp.uv);
    float rough = get_rough(s, m, sp.uv);
    float3 dkd = d_out * (bcos / DR_PI);
    float d_bcos = dot(d_out, kd) / DR_PI;
    float3 dn = f3(0.f);
    float3 dks = f3(0.f);
    float dr = 0.f;
    if (sum(ks) > 0.f && dot(wi, n) > 0.f) {
        float3 hr = wi + wo;
        float3 h = normalize(hr);
        float3 hl = to_local(sp.f, h);
        if (hl.z > 0.f) {
            const bool ggx = m.model == DR_MICROFACET_GGX;
            bool e_pos = false;
            float e = 0.f, pz = 0.f, P = 0.f, A = 0.f, D, G1i, G1o;
            if (ggx) {
                A = ggx_A(rough);
                D = ggx_D(hl.z, A);
                G1i = ggx_g1(n, h, wi, A);
                G1o = ggx_g1(n, h, wo, A);
            } else {
                e_pos = 2.f / rough > 0.f;
                e = roughness_to_phong(rough);
                pz = fmaxf(hl.z, 0.f);
                P = dr_powf(pz, e);
                D = P * (e + 2.f) * DR_INV_2PI;
                G1i = smith_g1(sp.f, n, h, wi, rough);
                G1o = smith_g1(sp.f, n, h, wo, rough);
            }
            float Gt = G1i * G1o;
            float cd = dot(h, wo);
            float om = 1.f - cd;
            float fr = dr_powf(fmaxf(om, 0.f), 5.f);
            float3 F = f3(ks.x + (1.f - ks.x) * fr, ks.y + (1.f - ks.y) * fr, ks.z + (1.f - ks.z) * fr);
            float denom = 4.f * dot(wi, n);
            float inv_den = 1.f / denom;
            float3 dF = d_out * (D * Gt * inv_den);
            float dFsum = dot(d_out, F);
            float d_D = dFsum * Gt * inv_den;
            float d_G = dFsum * D * inv_den;
            float d_denom = -dFsum * D * Gt * inv_den * inv_den;
            dks = dF * (1.f - fr);
            float d_fr = dF.x * (1.f - ks.x) + dF.y * (1.f - ks.y) + dF.z * (1.f - ks.z);
            float d_om = om >= 0.f ? d_fr * 5.f * dr_powf(om, 4.f) : 0.f;
            float d_cd = -d_om;
            float3 dh = d_cd * wo;
            sg.dwo += d_cd * h;
            float d_z;
            if (ggx) {
                float dA = 0.f, dDdz, dDdA;
                d_ggx_g1(n, h, wi, A, d_G * G1o, dn, sg.dwi, dA);
                d_ggx_g1(n, h, wo, A, d_G * G1i, dn, sg.dwo, dA);
                ggx_D_partials(hl.z, A, dDdz, dDdA);
                d_z = d_D * dDdz;
                dA += d_D * dDdA;
                dr += dA * ggx_dA_drough(rough);
            } else {
                d_smith_g1(sp.f, n, h, wi, rough, d_G * G1o, sg.df, dn, dh, sg.dwi, dr);
                d_smith_g1(sp.f, n, h, wo, rough, d_G * G1i, sg.df, dn, dh, sg.dwo, dr);
                float d_P = d_D * (e + 2.f) * DR_INV_2PI;
                float d_e = d_D * P * DR_INV_2PI;
                d_z = d_P * e * dr_powf(pz, e - 1.f);
                d_e += d_P * P * dr_logf(fmaxf(pz, 1e-6f));
                if (e_pos) dr += d_e * (-2.f / (rough * rough));
            }
            sg.dwi += (4.f * d_denom) * n;
            dn += (4.f * d_denom) * wi;
            d_to_local(sp.f, h, f3(0.f, 0.f, d_z), sg.df, dh);
            float3 dhr = d_normalize(hr, dh);
            sg.dwi += dhr;
            sg.dwo += dhr;
        }
    }
    dn += d_bcos * wo;
    sg.dwo += d_bcos * n;
    sg.df.n += sgn * dn;
    d_kd(s, m, sp.uv, dkd, g, sg.duv);
    if (!is_zero(dks)) d_ks(s, m, sp.uv, dks, g, sg.duv);
    if (dr != 0.f) d_rough(s, m, sp.uv, dr, g, sg.duv);
}

// adjoint of bsdf_pdf (material.h:414-462)
template <class G>
DEV void d_bsdf_pdf(const DevScene &s, int mi, const SurfacePoint &sp, float3 wi, float3 wo, float d_out, G &g,
                    SpGrad &sg) {
    if (d_out == 0.f) return;
    const DevMaterial &m = s.mats[mi];
    float3 kd = get_kd(s, m, sp.uv), ks = get_ks(s, m, sp.uv);
    float dw = luminance(kd), sw = luminance(ks), ws = dw + sw;
    if (ws <= 0.f) return;
    float dpmf = dw / ws, spmf = sw / ws;
    float d_dpmf = 0.f, d_spmf = 0.f, dr = 0.f;
    if (dpmf > 0.f) {
        float c = dot(sp.f.n, wo);
        float c2 = m.two_sided ? fabsf(c) : fmaxf(c, 0.f);
        d_dpmf += d_out * c2 / DR_PI;
        float d_c2 = d_out * dpmf / DR_PI;
        float d_c = m.two_sided ? (c >= 0.f ? d_c2 : -d_c2) : (c >= 0.f ? d_c2 : 0.f);
        sg.df.n += d_c * wo;
        sg.dwo += d_c * sp.f.n;
    }
    if (spmf > 0.f) {
        float3 hr = wi + wo;
        float3 h = normalize(hr);
        float3 hl = to_local(sp.f, h);
        if (hl.z > 0.f) {
            float rough = get_rough(s, m, sp.uv);
            float dwh = dot(wo, h);
            float Q = 4.f * fabsf(dwh);
            float d_hlz, d_Q;
            if (m.model == DR_MICROFACET_GGX) {
                // spdf = spmf D z / Q
                float A = ggx_A(rough);
                float D = ggx_D(hl.z, A);
                d_spmf += d_out * D * hl.z / Q;
                float d_D = d_out * spmf * hl.z / Q;
                d_Q = -d_out * spmf * D * hl.z / (Q * Q);
                float dDdz, dDdA;
                ggx_D_partials(hl.z, A, dDdz, dDdA);
                d_hlz = d_out * spmf * D / Q + d_D * dDdz;
                dr += d_D * dDdA * ggx_dA_drough(rough);
            } else {
                bool e_pos = 2.f / rough > 0.f;
                float e = roughness_to_phong(rough);
                float P = dr_powf(hl.z, e);
                float D = P * (e + 2.f) * DR_INV_2PI;
                d_spmf += d_out * D / Q;
                float d_D = d_out * spmf / Q;
                d_Q = -d_out * spmf * D / (Q * Q);
                float d_P = d_D * (e + 2.f) * DR_INV_2PI;
                float d_e = d_D * P * DR_INV_2PI;
                d_hlz = d_P * e * dr_powf(hl.z, e - 1.f);
                d_e += d_P * P * dr_logf(fmaxf(hl.z, 1e-6f));
                if (e_pos) dr += d_e * (-2.f / (rough * rough));
            }
            float d_dwh = 4.f * d_Q * (dwh >= 0.f ? 1.f : -1.f);
            sg.dwo += d_dwh * h;
            float3 dh = d_dwh * wo;
            d_to_local(sp.f, h, f3(0.f, 0.f, d_hlz), sg.df, dh);
            float3 dhr = d_normalize(hr, dh);
            sg.dwi += dhr;
            sg.dwo += dhr;
        }
    }
    float d_dw = d_dpmf / ws, d_sw = d_spmf / ws;
    float d_ws = -(d_dpmf * dw + d_spmf * sw) / (ws * ws);
    d_dw += d_ws;
    d_sw += d_ws;
    const float3 lw = f3(0.212671f, 0.715160f, 0.072169f);
    if (d_dw != 0.f) d_kd(s, m, sp.uv, lw * d_dw, g, sg.duv);
    if (d_sw != 0.f) d_ks(s, m, sp.uv, lw * d_sw, g, sg.duv);
    if (dr != 0.f) d_rough(s, m, sp.uv, dr, g, sg.duv);
}

// scatter of one triangle's vertex adjoints (global vertex ids) into the flat gradient
template <class G> DEV void scatter_tri_vertices(const DevScene &s, int tri, float3 d0, float3 d1, float3 d2, G &g) {
    int4 id = s.tri[tri];
    const DevShape &sh = s.shapes[id.w];
    int b = sh.grad_v - 3 * sh.vtx_off;
    const float3 d[3] = {d0, d1, d2};
    const int v[3] = {id.x, id.y, id.z};
    for (int k = 0; k < 3; k++) {
        g.add(b + 3 * v[k], d[k].x);
        g.add(b + 3 * v[k] + 1, d[k].y);
        g.add(b + 3 * v[k] + 2, d[k].z);
    }
}

// adjoint of next-event estimation (pathtrace.h:59-102 with eval :7-57).
// Light vertices and intensity always receive gradients; the shading point's
// adjoints (position into d_p, frame/uv/wi into sg) are meaningful only when
// the caller treats the point as differentiable.
template <class G>
DEV void d_nee(const DevScene &s, const LightSample &ls, float3 wi, int stri, const SurfacePoint &sp, float3 d_out,
               G &g, SpGrad &sg, float3 &d_p) {
    if (stri < 0 || is_zero(d_out)) return;
    LightPoint lp = sample_light_point(s, ls);
    int li = lp.light;
    const DevLight &L = s.lights[li];
    float3 ldir = normalize(lp.sp.p - sp.p);
    float lcos = fabsf(dot(ldir, lp.sp.ng));
    float lpdf = light_pdf(s, lp.tri);
    int mi = material_of_tri(s, stri);
    float bpdf = bsdf_pdf(s, mi, sp, wi, ldir) * lcos / length_sq(lp.sp.p - sp.p);
    float mis = sq(lpdf) / (sq(bpdf) + sq(lpdf));
    // eval (its shading-point checks are those of eval_light)
    float3 dv = lp.sp.p - sp.p;
    float dist = length(dv);
    if (dist == 0.f) return;
    float inv = 1.f / dist;
    float3 nd = dv * inv;
    if (occluded(s, sp.p, nd, dist)) return;
    float3 B = bsdf(s, mi, sp, wi, nd);
    float lcos2 = dot(lp.sp.f.n, -nd);
    if (lcos2 <= 0.f) return;
    float d2 = sq(dist);
    float3 I = light_intensity(s, li);
    float ratio = lcos2 / d2;
    float3 lc = I * ratio;
    float3 E = B * lc;
    float sN = mis / lpdf;
    // backward
    float3 dE = d_out * sN;
    float d_sN = dot(d_out, E);
    float d_lpdf = -d_sN * mis / (lpdf * lpdf);
    float3 dB = dE * lc;
    float3 dlc = dE * B;
    g.add(L.grad + 0, dlc.x * ratio);
    g.add(L.grad + 1, dlc.y * ratio);
    g.add(L.grad + 2, dlc.z * ratio);
    float d_ratio = dot(dlc, I);
    float d_lcos2 = d_ratio / d2;
    float d_d2 = -d_ratio * lcos2 / (d2 * d2);
    float d_dist = d_d2 * 2.f * dist;
    float3 d_lfn = d_lcos2 * (-nd);
    float3 dnd = d_lcos2 * (-lp.sp.f.n);
    SpGrad bg;
    bg.zero();
    d_bsdf(s, mi, sp, wi, nd, dB, g, bg);
    dnd += bg.dwo;
    frame_add(sg.df, bg.df);
    sg.duv.x += bg.duv.x;
    sg.duv.y += bg.duv.y;
    sg.dwi += bg.dwi;
    float3 ddv = dnd * inv;
    float d_inv = dot(dnd, dv);
    d_dist += -d_inv * inv * inv;
    ddv += dv * (d_dist / dist);
    d_p -= ddv;
    // light point p = v0 + e1 b1 + e2 b2, normal nn = normalize(e1 x e2)
    int4 id = s.tri[lp.tri];
    float3 v0 = vtx3(s.vtx, id.x), v1 = vtx3(s.vtx, id.y), v2 = vtx3(s.vtx, id.z);
    float3 e1 = v1 - v0, e2 = v2 - v0;
    float3 cr = cross(e1, e2);
    float3 dcr = d_normalize(cr, d_lfn);
    float3 de1 = ddv * lp.b1, de2 = ddv * lp.b2;
    d_cross(e1, e2, dcr, de1, de2);
    float3 dv0 = ddv - de1 - de2, dv1 = de1, dv2 = de2;
    // light pdf: lpmf * tri_pmf / area, area = 0.5 |(v1 - v0) x (v2 - v0)|
    float lpmf = luminance(I) / s.total_light_intensity;
    float clen = length(cr);
    float area = 0.5f * clen;
    float tri_pmf = area / L.area;
    float d_area = -d_lpdf * lpmf * tri_pmf / (area * area);
    float3 dcr3 = cr * (d_area * 0.5f / clen);
    float3 da = f3(0.f), db = f3(0.f);
    d_cross(e1, e2, dcr3, da, db);
    dv1 += da;
    dv2 += db;
    dv0 -= da + db;
    scatter_tri_vertices(s, lp.tri, dv0, dv1, dv2, g);
}

// adjoint of sample_primary (camera.h:48-84) w.r.t. cam_to_world
template <class G>
DEV void d_sample_primary(const DevCamera &c, float sx, float sy, float3 d_o, float3 d_d, G &g, int cam_off,
                          bool ad = true) {
    float dM[16];
    for (int i = 0; i < 16; i++) dM[i] = 0.f;
    d_xfm_point(c.c2w, f3(0.f), d_o, dM);
    float3 dir;
    if (c.fisheye) {
        float x = 2.f * (sx - 0.5f), y = 2.f * (sy - 0.5f);
        float rr = sqrtf(x * x + y * y);
        float phi = dr_atan2f(y, x);
        float theta = rr * DR_PI / 2.f;
        dir = f3(-dr_cosf(phi) * dr_sinf(theta), -dr_sinf(phi) * dr_sinf(theta), dr_cosf(theta));
    } else {
        float ndcx = (sx - 0.5f) * -2.f;
        float ndcy = ad ? ((sy - 0.5f) * -2.f) * (1.f / c.aspect) : (sy - 0.5f) * -2.f / c.aspect;
        dir = f3(c.fov * ndcx, c.fov * ndcy, 1.f);
    }
    float3 dummy = f3(0.f);
    d_xfm_vector(c.c2w, normalize(dir), d_d, dM, dummy);
    for (int i = 0; i < 16; i++) g.add(cam_off + i, dM[i]);
}
