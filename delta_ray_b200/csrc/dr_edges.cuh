// Edge sampling on the device: the boundary terms of the derivative.
//
//   is_silhouette           edge.h:59-79
//   box_cone                aabb.cpp:98-311 (GeometricTools box/cone test)
//   bsdf_bound              edge_tree.cpp:345-480
//   contains_silhouette     edge_tree.cpp:482-497
//   traverse_edges          edge_tree.cpp:511-725, recursion replaced by an
//                           explicit stack that keeps the same depth-first
//                           order (left child first), so random draws are
//                           consumed in the reference's order
//   shading_edge_sample     delta_ray.cpp:45-365 (LTC line sampling, two rays
//                           straddling the edge, dp/dv0/dv1)
//   primary_edge_sample     delta_ray.cpp:377-557 (screen-space boundary
//                           term, forward differences to world space)
#pragma once

#include "dr_shading.cuh"

DEV float3 shape_vtx(const DevScene &s, int shape, int v) { return vtx3(s.vtx, s.shapes[shape].vtx_off + v); }
DEV float3 edge_v0(const DevScene &s, const DevEdge &e) { return shape_vtx(s, e.shape, e.v0); }
DEV float3 edge_v1(const DevScene &s, const DevEdge &e) { return shape_vtx(s, e.shape, e.v1); }

DEV float3 non_shared_vertex(const DevScene &s, const DevEdge &e, int f) {
    int4 t = s.tri[s.shapes[e.shape].tri_off + f];
    int off = s.shapes[e.shape].vtx_off;
    int v[3] = {t.x - off, t.y - off, t.z - off};
    for (int i = 0; i < 3; i++)
        if (v[i] != e.v0 && v[i] != e.v1) return shape_vtx(s, e.shape, v[i]);
    return f3(0.f);
}

DEV bool is_silhouette(const DevScene &s, float3 p, const DevEdge &e) {
    if (!s.shapes[e.shape].has_n) return true;
    if (e.f0 == -1 || e.f1 == -1) return true;
    float3 v0 = edge_v0(s, e), v1 = edge_v1(s, e);
    float3 a = non_shared_vertex(s, e, e.f0), b = non_shared_vertex(s, e, e.f1);
    float3 n0 = normalize(cross(v0 - a, v1 - a)), n1 = normalize(cross(v1 - b, v0 - b));
    bool f0 = dot(p - v0, n0) > 0.f && dot(p - v1, n0) > 0.f && dot(p - a, n0) > 0.f;
    bool f1 = dot(p - v0, n1) > 0.f && dot(p - v1, n1) > 0.f && dot(p - b, n1) > 0.f;
    return (f0 && !f1) || (!f0 && f1);
}

// The silhouette test's record of an edge (see EdgeRec): the same operands
// is_silhouette computes, so that is_silhouette_rec gives its answer.
DEV EdgeRec edge_record(const DevScene &s, const DevEdge &e) {
    EdgeRec r;
    const bool always = !s.shapes[e.shape].has_n || e.f0 == -1 || e.f1 == -1;
    float3 v0 = edge_v0(s, e), v1 = edge_v1(s, e), a = v0, b = v1, n0 = f3(0.f), n1 = f3(0.f);
    if (!always) {
        a = non_shared_vertex(s, e, e.f0);
        b = non_shared_vertex(s, e, e.f1);
        n0 = normalize(cross(v0 - a, v1 - a));
        n1 = normalize(cross(v1 - b, v0 - b));
    }
    r.r[0].x = v0.x, r.r[0].y = v0.y, r.r[0].z = v0.z, r.r[0].w = n0.x;
    r.r[1].x = v1.x, r.r[1].y = v1.y, r.r[1].z = v1.z, r.r[1].w = n0.y;
    r.r[2].x = a.x, r.r[2].y = a.y, r.r[2].z = a.z, r.r[2].w = n0.z;
    r.r[3].x = b.x, r.r[3].y = b.y, r.r[3].z = b.z, r.r[3].w = n1.x;
    r.r[4].x = n1.y, r.r[4].y = n1.z, r.r[4].z = always ? 1.f : 0.f, r.r[4].w = 0.f;
    return r;
}

DEV bool is_silhouette_rec(const EdgeRec *rec, float3 p) {
    const float4 q0 = dr_ldg(&rec->r[0]), q1 = dr_ldg(&rec->r[1]), q2 = dr_ldg(&rec->r[2]), q3 = dr_ldg(&rec->r[3]),
                 q4 = dr_ldg(&rec->r[4]);
    if (q4.z != 0.f) return true;
    const float3 v0 = f3(q0.x, q0.y, q0.z), v1 = f3(q1.x, q1.y, q1.z), a = f3(q2.x, q2.y, q2.z),
                 b = f3(q3.x, q3.y, q3.z), n0 = f3(q0.w, q1.w, q2.w), n1 = f3(q3.w, q4.x, q4.y);
    bool f0 = dot(p - v0, n0) > 0.f && dot(p - v1, n0) > 0.f && dot(p - a, n0) > 0.f;
    bool f1 = dot(p - v0, n1) > 0.f && dot(p - v1, n1) > 0.f && dot(p - b, n1) > 0.f;
    return (f0 && !f1) || (!f0 && f1);
}

// ---------------------------------------------------------------------------
// Box / cone intersection.  The apex region (per axis: beyond the slab's upper
// face, inside, below its lower face) selects the silhouette polygon of the
// box seen from the apex; corner j has +extent on axis a iff bit a of j is
// set.  Same table as aabb.cpp:106-132 so that boundary cases agree.
// ---------------------------------------------------------------------------
struct ConeSpec { float3 o, d; float cos_angle; };

// packed: 4 bits per corner, count in the top nibble
DR_TABLE unsigned long long kConePoly[27] = {
    0x6000000000154623ull, 0x6000000000023154ull, 0x6000000000023754ull, 0x6000000000046231ull,
    0x4000000000000231ull, 0x6000000000023751ull, 0x6000000000046731ull, 0x6000000000026731ull,
    0x6000000000026751ull, 0x6000000000015462ull, 0x4000000000000154ull, 0x6000000000013754ull,
    0x4000000000000462ull, 0x0000000000000000ull, 0x4000000000001375ull, 0x6000000000046732ull,
    0x4000000000002673ull, 0x6000000000132675ull, 0x6000000000015762ull, 0x6000000000015764ull,
    0x6000000000013764ull, 0x6000000000045762ull, 0x4000000000004576ull, 0x6000000000137645ull,
    0x6000000000045732ull, 0x6000000000264573ull, 0x6000000000132645ull};

DEV int cone_poly(int lookup, int i) {
    unsigned long long w = kConePoly[lookup];
    if (i < 0) return (int)(w >> 60);
    int n = (int)(w >> 60);
    return (int)((w >> (4 * (n - 1 - i))) & 0xF);
}

DEV_NOINLINE bool box_cone(const float *lo, const float *hi, const ConeSpec &cone) {
    if (cone.cos_angle <= 0.f) return true;
    float3 C = f3(0.5f * (lo[0] + hi[0]), 0.5f * (lo[1] + hi[1]), 0.5f * (lo[2] + hi[2]));
    float3 E = f3(0.5f * (hi[0] - lo[0]), 0.5f * (hi[1] - lo[1]), 0.5f * (hi[2] - lo[2]));
    float3 CmV = C - cone.o;
    float DdCmV = dot(cone.d, CmV);
    float rad = E.x * fabsf(cone.d.x) + E.y * fabsf(cone.d.y) + E.z * fabsf(cone.d.z);
    if (DdCmV + rad <= 0.f) return false;
    int ix = CmV.x < -E.x ? 2 : (CmV.x > E.x ? 0 : 1);
    int iy = CmV.y < -E.y ? 2 : (CmV.y > E.y ? 0 : 1);
    int iz = CmV.z < -E.z ? 2 : (CmV.z > E.z ? 0 : 1);
    int lookup = ix + 3 * iy + 9 * iz;
    if (lookup == 13) return true;
    int np = cone_poly(lookup, -1);
    float c2 = cone.cos_angle * cone.cos_angle;
    // only the corner of largest cos^2 (jmax) is needed after this loop: keep
    // it in registers rather than per-corner arrays (local memory)
    int imax = -1, jmax = -1;
    float3 mX = f3(0.f), mP = f3(0.f);
    float mLen = 0.f, mDd = 0.f, msDd = 0.f;
    for (int i = 0; i < np; i++) {
        int j = cone_poly(lookup, i);
        float3 X = f3((j & 1) ? E.x : -E.x, (j & 2) ? E.y : -E.y, (j & 4) ? E.z : -E.z);
        float DdPmV = dot(cone.d, X) + DdCmV;
        if (DdPmV > 0.f) {
            float3 PmV = X + CmV;
            float sDd = DdPmV * DdPmV;
            float sLen = dot(PmV, PmV);
            if (sDd - c2 * sLen > 0.f) return true;
            if (imax == -1 || sDd * mLen > msDd * sLen) {
                imax = i;
                jmax = j;
                mX = X;
                mP = PmV;
                mLen = sLen;
                mDd = DdPmV;
                msDd = sDd;
            }
        }
    }
    if (imax == -1) return false;
    for (int side = 0; side < 2; side++) {
        int s, k0;
        float fder;
        if (side == 0) {
            int jn = cone_poly(lookup, imax < np - 1 ? imax + 1 : 0);
            int jd = jn - jmax;
            s = jd > 0 ? 1 : -1;
            k0 = (jd < 0 ? -jd : jd) >> 1;
            fder = s * (comp(cone.d, k0) * mLen - mDd * comp(mP, k0));
        } else {
            int jp = cone_poly(lookup, imax > 0 ? imax - 1 : np - 1);
            int jd = jmax - jp;
            s = jd > 0 ? 1 : -1;
            k0 = (jd < 0 ? -jd : jd) >> 1;
            fder = -s * (comp(cone.d, k0) * mLen - mDd * comp(mP, k0));
        }
        if (fder > 0.f) {
            int k1 = (k0 + 1) % 3, k2 = (k1 + 1) % 3;
            float numer = comp(mP, k1) * comp(mP, k1) + comp(mP, k2) * comp(mP, k2);
            float denom = comp(cone.d, k1) * comp(mP, k1) + comp(cone.d, k2) * comp(mP, k2);
            float3 M;
            comp_set(M, k0, numer * comp(cone.d, k0));
            comp_set(M, k1, denom * (comp(mX, k1) + comp(CmV, k1)));
            comp_set(M, k2, denom * (comp(mX, k2) + comp(CmV, k2)));
            float DdM = dot(cone.d, M);
            if (DdM * DdM - c2 * dot(M, M) > 0.f) return true;
            float det = s * (comp(cone.d, k1) * comp(mP, k2) - comp(cone.d, k2) * comp(mP, k1));
            return det <= 0.f;
        }
    }
    return false;
}

// ---------------------------------------------------------------------------
// Edge-tree node bounds
// ---------------------------------------------------------------------------
DEV float min_sq_bound(float lo, float hi) {
    if (lo <= 0.f && hi >= 0.f) return 0.f;
    if (lo < 0.f && hi < 0.f) return hi * hi;
    return lo * lo;
}
DEV float max_sq_bound(float lo, float hi) { return fmaxf(lo * lo, hi * hi); }

// What the BSDF bound of an edge-tree node needs of the shading point: its
// position and normal, the frame around the incoming direction wi (rows
// t, b = normalize(n x wi), n = wi) and the normal in it, the lobes'
// luminances and the lobe's exponent or GGX parameter.  Computed once per
// walk; the per-node arithmetic is that of edge_tree.cpp:345-480.
struct BoundCtx {
    float3 p, n;
    Frame hf;
    float3 ln;
    float dl, sl, rough, expo;
    int model;
};
DEV BoundCtx bound_ctx(float3 wi, const SurfacePoint &sp, float dl, float sl, float rough, int model) {
    BoundCtx c;
    c.p = sp.p;
    c.n = sp.f.n;
    c.dl = dl;
    c.sl = sl;
    c.rough = rough;
    c.model = model;
    c.expo = 0.f;
    if (sl > 0.f) {
        float3 hy = normalize(cross(sp.f.n, wi));
        c.hf.t = normalize(cross(wi, hy));
        c.hf.b = hy;
        c.hf.n = wi;
        c.ln = to_local(c.hf, sp.f.n);
        c.expo = model == DR_MICROFACET_GGX ? ggx_A(rough) : roughness_to_phong(rough);
    }
    return c;
}

// Functions of the filters that decide a node test before its exact
// evaluation: the silhouette filter's sine, cosine and reciprocal square root
// (absolute errors below 1e-6 on its arguments) and the bound filter's log2
// and exp2 (a few ulps).  The filters only ever decide with margins well above
// those errors.
#ifdef DR_HOST_BUILD
HD float filt_sin(float x) { return std::sin(x); }
HD float filt_cos(float x) { return std::cos(x); }
HD float filt_rsqrt(float x) { return 1.f / std::sqrt(x); }
HD float filt_log2(float x) { return std::log2(x); }
HD float filt_exp2(float x) { return std::exp2(x); }
#else
DEV float filt_sin(float x) { return __sinf(x); }
DEV float filt_cos(float x) { return __cosf(x); }
DEV float filt_rsqrt(float x) { return rsqrtf(x); }
DEV float filt_log2(float x) { return log2f(x); }
DEV float filt_exp2(float x) { return exp2f(x); }
#endif

// The corners' products with a direction, per axis: corner i has the hi
// coordinate on axis a iff bit a of i is set, and dot(d, corner_i - p) is
// (x[i & 1] + y[(i >> 1) & 1]) + z[i >> 2], the bits of the per-corner dot.
struct CornerDots {
    float x[2], y[2], z[2];
    DEV float at(int i) const { return (x[i & 1] + y[(i >> 1) & 1]) + z[i >> 2]; }
};
DEV CornerDots corner_dots(float3 d, const float *q) {  // q: lo - p, hi - p per axis (x0 x1 y0 y1 z0 z1)
    CornerDots c;
    c.x[0] = d.x * q[0];
    c.x[1] = d.x * q[1];
    c.y[0] = d.y * q[2];
    c.y[1] = d.y * q[3];
    c.z[0] = d.z * q[4];
    c.z[1] = d.z * q[5];
    return c;
}

// fast_m (may be null) asks for the filtered form, used where only the
// bound's side of 1 and of 0 matters: a Blinn-Phong lobe's pow(hdn, e) is then
// taken as exp2f(e log2f(hdn)), within the relative bound m = (16 + |e log2
// hdn|) 2^-22 of the reproducible pow (the float functions' few ulps, the
// rounding of the operations after it, with a wide margin).  If the bound so
// taken is within m of 1, or not clearly above 0, the reproducible pow is
// evaluated on the same hdn and *fast_m is 0; otherwise the returned bound is
// on the exact one's side of 1 and of 0, within relative m of it, and *fast_m
// is m.  Without fast_m, or for other lobes, the exact bound (*fast_m 0).
DEV_NOINLINE float bsdf_bound(const DevEdgeNode &node, const BoundCtx &c, float *fast_m = nullptr) {
    if (fast_m) *fast_m = 0.f;
    const float q[6] = {node.lo[0] - c.p.x, node.hi[0] - c.p.x, node.lo[1] - c.p.y,
                        node.hi[1] - c.p.y, node.lo[2] - c.p.z, node.hi[2] - c.p.z};
    const CornerDots cn = corner_dots(c.n, q);
    float cos_max = 0.f;
    for (int i = 0; i < 8; i++)
        if (cn.at(i) > 0.f) {
            cos_max = 1.f;
            break;
        }
    if (cos_max <= 0.f) return 0.f;
    float maxp = 0.f;
    if (c.sl > 0.f) {
        const Frame &hf = c.hf;
        const CornerDots ct = corner_dots(hf.t, q), cb = corner_dots(hf.b, q), cz = corner_dots(hf.n, q);
        float3 lo = f3(DR_INF), hi = f3(-DR_INF);
        for (int i = 0; i < 8; i++) {
            float3 v = f3(ct.at(i), cb.at(i), cz.at(i));  // to_local(hf, corner_i - p)
            lo = f3(fminf(lo.x, v.x), fminf(lo.y, v.y), fminf(lo.z, v.z));
            hi = f3(fmaxf(hi.x, v.x), fmaxf(hi.y, v.y), fmaxf(hi.z, v.z));
        }
        float cphi = 0.f;
        float hx = hi.x;
        if (hx > 0.f) cphi = hx / sqrtf(min_sq_bound(lo.y, hi.y) + hx * hx);
        else if (hx == 0.f) cphi = fmaxf(cphi, 0.f);
        else cphi = hx / sqrtf(max_sq_bound(lo.y, hi.y) + hx * hx);
        float cto_min, cto_max;
        if (lo.z > 0.f) cto_min = lo.z / (max_sq_bound(lo.x, hi.x) + max_sq_bound(lo.y, hi.y) + lo.z * lo.z);
        else cto_min = lo.z / (min_sq_bound(lo.x, hi.x) + min_sq_bound(lo.y, hi.y) + lo.z * lo.z);
        if (hi.z > 0.f) cto_max = hi.z / (min_sq_bound(lo.x, hi.x) + min_sq_bound(lo.y, hi.y) + hi.z * hi.z);
        else cto_max = hi.z / (max_sq_bound(lo.x, hi.x) + max_sq_bound(lo.y, hi.y) + hi.z * hi.z);
        float cth_min = sqrtf((cto_min + 1.f) / 2.f), cth_max = sqrtf((cto_max + 1.f) / 2.f);
        const float3 ln = c.ln;
        float chmax = cphi >= 0.f ? sqrtf(ln.z * ln.z / (ln.z * ln.z + ln.x * ln.x * cphi * cphi)) : 1.f;
        if (chmax > cth_max) chmax = cth_max;
        else if (chmax < cth_min) chmax = cth_min;
        float shmax = sqrtf(fmaxf(1.f - chmax * chmax, 0.f));
        float hdn = fminf(fabsf(ln.x * shmax * cphi) + ln.z * chmax, 1.f);
        if (c.model == DR_MICROFACET_GGX) {
            // the GGX D grows with n.h (A <= 1): its bound is the value at the bound of n.h
            maxp = ggx_D(hdn, c.expo);
        } else {
            const float e = c.expo;
            if (fast_m) {
                const float y = e * filt_log2(hdn);
                if (y < -160.f) {  // the pow underflows to 0 either way
                    maxp = 0.f;
                } else {
                    const float m = (16.f + fabsf(y)) * 2.384185791e-7f;
                    const float bf = cos_max * (c.dl / DR_PI + c.sl * (filt_exp2(y) * (e + 2.f) /
                                                                        float(2 * 3.14159265358979323846)));
                    if (m < 0.01f && bf > 1e-30f && (bf * (1.f - m) > 1.f || bf * (1.f + m) <= 1.f)) {
                        *fast_m = m;
                        return bf;
                    }
                    maxp = dr_powf(hdn, e) * (e + 2.f) / float(2 * 3.14159265358979323846);
                }
            } else {
                maxp = dr_powf(hdn, e) * (e + 2.f) / float(2 * 3.14159265358979323846);
            }
        }
    }
    return cos_max * (c.dl / DR_PI + c.sl * maxp);
}



// Whether the node's cone of normals, widened by the angle its bounding
// sphere subtends from p, reaches the directions perpendicular to p - centre:
// |pi/2 - acos(c)| <= angle + atan(vt) with c = cos(axis, centre - p).  The
// float evaluation below (reproducible atan and acos, within 3 ulp) is within
// 1.5e-6 rad of the exact comparison.  A filter decides first where the two
// sides differ by more than 1e-5 in sine space (so by more in angle, since
// |d asin| >= |d x|): for angle + atan(vt) < pi/2 the test is |c| <=
// sin(angle + atan(vt)) = (sin a + vt cos a) / sqrt(1 + vt^2), whose terms it
// takes from the fast functions; it takes the same answer as the float
// evaluation and leaves the rest to it, and also every |c| > 1 (rounding
// can give that; acos is NaN there and the float evaluation answers false).
DEV_NOINLINE bool contains_silhouette(const DevEdgeNode &node, float3 p) {
    // bounding sphere as aabb.h:266-270: center (lo + hi) / 2, radius |hi - center|
    float3 cs = f3((node.lo[0] + node.hi[0]) / 2.f, (node.lo[1] + node.hi[1]) / 2.f, (node.lo[2] + node.hi[2]) / 2.f);
    float r = length(f3(node.hi[0], node.hi[1], node.hi[2]) - cs);
    float3 d = cs - p;
    float l = length(d);
    float vt = r / l;
    if (vt >= 1.f) return true;
    d = d / l;
    const float c = dot(-d, f3(node.axis[0], node.axis[1], node.axis[2]));
    const float a = node.angle, ac = fabsf(c);
    if (a >= 0.f && a <= 1.5f && ac <= 1.f) {  // NaNs fall through to the float evaluation
        const float k = filt_rsqrt(1.f + vt * vt), sa = filt_sin(a), ca = filt_cos(a);
        const float cos_r = (ca - vt * sa) * k, sin_r = (sa + vt * ca) * k;
        const float margin = 1e-5f;
        if (cos_r < -margin) return true;  // angle + atan(vt) > pi/2
        if (cos_r > margin) {
            if (ac < sin_r - margin) return true;
            if (ac > sin_r + margin) return false;
        }
    }
    float va = dr_atanf(vt);
    float ang = dr_acosf(c);
    float range = node.angle + va;
    return ang - range <= float(3.14159265358979323846 / 2.f) && ang + range >= float(3.14159265358979323846 / 2.f);
}

// The float evaluation alone (checks of the filter).
HD bool contains_silhouette_exact(const DevEdgeNode &node, float3 p) {
    float3 cs = f3((node.lo[0] + node.hi[0]) / 2.f, (node.lo[1] + node.hi[1]) / 2.f, (node.lo[2] + node.hi[2]) / 2.f);
    float r = length(f3(node.hi[0], node.hi[1], node.hi[2]) - cs);
    float3 d = cs - p;
    float l = length(d);
    float vt = r / l;
    if (vt >= 1.f) return true;
    d = d / l;
    float va = dr_atanf(vt);
    float ang = dr_acosf(dot(-d, f3(node.axis[0], node.axis[1], node.axis[2])));
    float range = node.angle + va;
    return ang - range <= float(3.14159265358979323846 / 2.f) && ang + range >= float(3.14159265358979323846 / 2.f);
}

DEV float node_importance(const DevEdgeNode &node, float bb, float3 p) {
    float3 c = f3(0.5f * (node.lo[0] + node.hi[0]), 0.5f * (node.lo[1] + node.hi[1]), 0.5f * (node.lo[2] + node.hi[2]));
    return bb * node.total_length / length_sq(p - c);
}

DEV bool node_inside(const DevEdgeNode &n, float3 p) {
    return p.x >= n.lo[0] && p.x <= n.hi[0] && p.y >= n.lo[1] && p.y <= n.hi[1] && p.z >= n.lo[2] && p.z <= n.hi[2];
}

// The learned edge proposal of one shading point (a project addition): 32
// bf16 probabilities over directions from the point, in the shading frame:
// 4 bands of dr_cosf(theta) (split at -1/2, 0, 1/2) times 8 azimuth octants
// (dir_bin).  q == null: the reference's sampling.
struct EdgeProposal {
    const uint16_t *q;
    float alpha;  // probability of the learned descent in the defensive mixture
    bool codes;   // emit each edge's direction bin (training)
};
HD float bf16_bits_to_float(uint16_t b) { return dr_i2f((int)((uint32_t)b << 16)); }
DEV int dir_bin(const Frame &f, float3 d) {
    float x = dot(d, f.t), y = dot(d, f.b), z = dot(d, f.n);
    float z2 = z * z, r2 = x * x + y * y + z2;
    int band = z < 0.f ? (4.f * z2 > r2 ? 0 : 1) : (4.f * z2 > r2 ? 3 : 2);
    int oct = (y < 0.f ? 4 : 0) | (x < 0.f ? 2 : 0) | (fabsf(x) < fabsf(y) ? 1 : 0);
    return band * 8 + oct;
}
// The proposal's weight of a node: its probability for the direction of the box centre.
DEV float node_dir_weight(const uint16_t *q, const Frame &f, float3 p, const DevEdgeNode &n) {
    float3 c = f3(0.5f * (n.lo[0] + n.hi[0]), 0.5f * (n.lo[1] + n.hi[1]), 0.5f * (n.lo[2] + n.hi[2]));
    return bf16_bits_to_float(q[dir_bin(f, c - p)]);
}

// Stochastic traversal of one edge tree in one mode (edge_tree.cpp:511-652):
// CONE true for the cone mode, false for the all mode.
// emit(tree_edge_index, weight, slot_code) is called for every silhouette
// edge of every reached leaf, in the reference's order.  Returns false if the
// stack limit was hit (never for trees of depth < DR_EDGE_STACK).
//
// With a proposal, the "all" mode becomes a defensive mixture: `learned`
// (drawn once per traversal, probability alpha) picks the child at each
// stochastic node in proportion to the tree's importance times the
// proposal's weight of the direction towards the child, otherwise by the
// importance alone.  Every node tracks both path products (apmf plain, lpmf
// learned), so the mixture's pmf alpha lpmf + (1 - alpha) apmf takes the place
// of the all-mode pmf in the multiple-importance weights of both modes.  The
// emitted code is the direction bin of the edge's midpoint (the training
// target's slot).
#define DR_EDGE_STACK 64
// Stack entry of the traversal; with a proposal (PROP) it also carries the
// learned path product.
template <bool PROP> struct EdgeItem { int node; float bb, cpmf, apmf, lpmf; };
template <> struct EdgeItem<false> { int node; float bb, cpmf, apmf; };
template <bool PROP> HD EdgeItem<PROP> edge_item(int node, float bb, float c, float a, float l) {
    EdgeItem<PROP> it;
    it.node = node;
    it.bb = bb;
    it.cpmf = c;
    it.apmf = a;
    if constexpr (PROP) it.lpmf = l;
    return it;
}

// The children of an interior node as the traversal decides them
// (edge_tree.cpp:560-650): both when the node splits, else the one drawn in
// proportion to the importances.  Returns 0 when neither is walked (both
// importances vanish), 1 for a split, 2 for a draw; push_l / push_r say which
// children are walked (a child whose silhouette test fails or whose bound is
// 0 is not), l_leaf / r_leaf whether they are leaves.  Shared by the
// depth-first walk (EdgeWalk) and the level-by-level walk (k_edge_level).
template <bool PROP> struct ChildPick {
    EdgeItem<PROP> left, right;
    bool push_l, push_r, l_leaf, r_leaf;
};
template <bool PROP>
DEV int node_children(const DevEdgeNode *nodes, const BoundCtx &bc, const ConeSpec &cone, const NodeRng &rng,
                      const EdgeProposal &pr, const Frame &f, const bool CONE, bool dir_bounds, bool learned,
                      const EdgeItem<PROP> &it, const DevEdgeNode &node, int nid, ChildPick<PROP> &c) {
    const float3 p = bc.p;
    c.push_l = c.push_r = false;
    int li = nid + 1, ri = node.offset;
    const DevEdgeNode &L = nodes[li], &R = nodes[ri];
    bool all_split = it.bb > 1.f || node_inside(node, p);
    bool lcs = true, rcs = true;
    if (dir_bounds) {
        lcs = contains_silhouette(L, p);
        rcs = contains_silhouette(R, p);
    }
    // The children of an all-split node in the all walk, off the cone
    // walk's path (cpmf 0): their bounds only meet thresholds (above 1,
    // above 0, the importance cutoff), so they may come filtered.
    const bool filt = !CONE && all_split && it.cpmf == 0.f;
    float lm = 0.f, rm = 0.f;
    float lbb = lcs ? bsdf_bound(L, bc, filt ? &lm : nullptr) : 0.f;
    float rbb = rcs ? bsdf_bound(R, bc, filt ? &rm : nullptr) : 0.f;
    float il = lcs ? node_importance(L, lbb, p) : 0.f;
    float ir = rcs ? node_importance(R, rbb, p) : 0.f;
    if (lm > 0.f || rm > 0.f) {
        // the cutoff and the cone tests' finiteness check as the exact
        // bounds decide them: exact bounds where a filtered one could differ
        const float m = 2.f * fmaxf(lm, rm) + 1e-6f, sum = il + ir;
        if (!(sum > 1e-10f * (1.f + m) || sum < 1e-10f * (1.f - m)) || !(il < 1e30f) || !(ir < 1e30f)) {
            lbb = lcs ? bsdf_bound(L, bc) : 0.f;
            rbb = rcs ? bsdf_bound(R, bc) : 0.f;
            il = lcs ? node_importance(L, lbb, p) : 0.f;
            ir = rcs ? node_importance(R, rbb, p) : 0.f;
        }
    }
    if (il + ir <= 1e-10f) return 0;
    // a node the cone walk cannot reach (cpmf 0) gives its children cpmf
    // 0 whatever the cone tests say, as long as the importances are
    // finite: the all walk skips the tests there
    const bool cone_tests = CONE || it.cpmf != 0.f || !dr_isfinite(il) || !dr_isfinite(ir);
    bool lhc = cone_tests && box_cone(L.lo, L.hi, cone), rhc = cone_tests && box_cone(R.lo, R.hi, cone);
    bool cone_split = all_split || (lhc && rhc && lcs && rcs && cone.cos_angle > 0.95f);
    float ilc = lhc ? il : 0.f, irc = rhc ? ir : 0.f;
    if (CONE && ilc + irc <= 1e-10f) return 0;
    float plc = 0.f, prc = 0.f, pla = 0.f, pra = 0.f;
    if (cone_split) {
        plc = prc = 1.f;
    } else if (ilc + irc > 1e-10f) {
        plc = ilc / (ilc + irc);
        prc = 1.f - plc;
    }
    if (all_split) {
        pla = pra = 1.f;
    } else {
        pla = il / (il + ir);
        pra = 1.f - pla;
    }
    // the proposal's choice (both children important, no split): importance
    // times the learned weight of the direction towards each child
    float pll = pla;
    if constexpr (PROP) {
        float prl = pra;
        if (!all_split && il > 0.f && ir > 0.f) {
            float gl = il * node_dir_weight(pr.q, f, p, L), gr = ir * node_dir_weight(pr.q, f, p, R);
            if (gl + gr > 0.f) {
                pll = gl / (gl + gr);
                prl = 1.f - pll;
            }
        }
        c.left = edge_item<PROP>(li, lbb, plc * it.cpmf, pla * it.apmf, pll * it.lpmf);
        c.right = edge_item<PROP>(ri, rbb, prc * it.cpmf, pra * it.apmf, prl * it.lpmf);
    } else {
        c.left = edge_item<PROP>(li, lbb, plc * it.cpmf, pla * it.apmf, 0.f);
        c.right = edge_item<PROP>(ri, rbb, prc * it.cpmf, pra * it.apmf, 0.f);
    }
    bool split = CONE ? cone_split : all_split;
    c.l_leaf = L.nprims > 0;
    c.r_leaf = R.nprims > 0;
    if (split) {
        // a child of bound 0 would only be taken off the stack and skipped,
        // so it is not pushed
        c.push_r = rcs && !(rbb <= 0.f);
        c.push_l = lcs && !(lbb <= 0.f);
        return 1;
    }
    float u = rng.draw(CONE ? 0 : 1, nid);
    bool go_left = CONE ? u < plc : u < (learned ? pll : pla);
    if (go_left) c.push_l = !(lbb <= 0.f);
    else c.push_r = !(rbb <= 0.f);
    return 2;
}

#define DR_NODE_MASK ((1 << 27) - 1)

// The walk of one tree in one mode as a resumable state: start() pushes the
// root or a handed-on subtree, step() takes one node off the stack.  A kernel
// can interleave walks (a lane that finishes one starts the next while the
// other lanes of its warp keep stepping); the draws are keyed by node and the
// items carry their order key, so the sampled edges do not depend on it.
// CUT > 0: interior nodes at depth CUT below the start are handed to
// defer(node, bb, cpmf, apmf, lpmf) instead of being walked (inside the walk
// an item's node field carries its depth in bits 27..31).
template <bool PROP, int CUT = 0>
struct EdgeWalk {
    using Item = EdgeItem<PROP>;
    const DevScene *s;
    const DevEdgeNode *nodes;
    const DevEdge *edges;
    const EdgeRec *recs;
    BoundCtx bc;
    Frame f;  // shading frame (the proposal's direction bins)
    ConeSpec cone;
    NodeRng rng;
    EdgeProposal pr;
    int tree;
    bool cone_mode, dir_bounds, learned, ok;
    int n = 0;
    Item st[DR_EDGE_STACK];

    DEV void start(bool CONE, const DevScene &sc, const DevEdgeNode *nd, const DevEdge *ed, int tr, bool dirb,
                   float3 wi, const SurfacePoint &sp, float dl, float sl, float rough, int model, const ConeSpec &cn,
                   const EdgeTask &t, const NodeRng &r, const EdgeProposal &p, bool lrn) {
        s = &sc;
        nodes = nd;
        edges = ed;
        recs = tr ? sc.nrm_rec : sc.sil_rec;
        tree = tr;
        dir_bounds = dirb;
        cone_mode = CONE;
        learned = lrn;
        bc = bound_ctx(wi, sp, dl, sl, rough, model);
        f = sp.f;
        cone = cn;
        rng = r;
        pr = p;
        ok = true;
        n = 0;
        st[n++] = edge_item<PROP>(t.code & DR_NODE_MASK, t.bb, t.cpmf, t.apmf, t.lpmf);
    }
    DEV bool busy() const { return n > 0; }

    // Takes the shallowest pending subtree (the bottom of the stack, the
    // largest) off the walk, as a task of point `point` for another lane.
    // Only walks without a depth cut (CUT == 0) hand subtrees on.
    DEV EdgeTask take_bottom(int point) {
        const Item b = st[0];
        EdgeTask t;
        t.point = point;
        t.code = (b.node & DR_NODE_MASK) | (tree << 29) | ((cone_mode ? 0 : 1) << 30);
        t.bb = b.bb;
        t.cpmf = b.cpmf;
        t.apmf = b.apmf;
        t.lpmf = 0.f;
        if constexpr (PROP) t.lpmf = b.lpmf;
        for (int i = 1; i < n; i++) st[i - 1] = st[i];
        n--;
        return t;
    }

    template <class Emit> DEV void leaf(const Item &it, const DevEdgeNode &node, Emit &emit) {
        const bool CONE = cone_mode;
        const float3 p = bc.p;
        float apmf = it.apmf;
        if constexpr (PROP) apmf = pr.alpha * it.lpmf + (1.f - pr.alpha) * it.apmf;
        float denom = it.cpmf * it.cpmf + apmf * apmf;
        float w = CONE ? it.cpmf / denom : apmf / denom;
        for (int i = 0; i < node.nprims; i++) {
            int ei = node.offset + i;
            if (!is_silhouette_rec(recs + ei, p)) continue;
            int code = 0;
            if constexpr (PROP)
                if (pr.codes) code = dir_bin(f, 0.5f * (edge_v0(*s, edges[ei]) + edge_v1(*s, edges[ei])) - p);
            emit(ei, (CONE ? 0 : 1) << 27 | ei, w, code);
        }
    }

    // One step: the node on top of the stack.  emit(tree_edge_index, key,
    // weight, slot_code) for every silhouette edge of a reached leaf.  (Taking
    // a lane's leaves together with its next interior node in one step was
    // measured slower, with the leaf test reading scattered vertices and with
    // it reading one record per edge.)
    template <class Emit, class Defer> DEV void step(Emit &emit, Defer &defer, int *visits) {
        const bool CONE = cone_mode;
        const Item it = st[--n];
        if (it.bb <= 0.f) return;
        const int nid = it.node & DR_NODE_MASK;
        if (visits) ++*visits;
        if (nodes[nid].nprims > 0) {
            leaf(it, nodes[nid], emit);
            return;
        }
        const DevEdgeNode &node = nodes[nid];
        if (CUT > 0 && (it.node >> 27) == CUT) {  // hand the subtree on
            float lp = 0.f;
            if constexpr (PROP) lp = it.lpmf;
            defer(nid, it.bb, it.cpmf, it.apmf, lp);
            return;
        }
        const int cdepth = CUT > 0 ? ((it.node >> 27) + 1) << 27 : 0;  // the children's depth bits
        ChildPick<PROP> c;
        const int r = node_children<PROP>(nodes, bc, cone, rng, pr, f, CONE, dir_bounds, learned, it, node, nid, c);
        if (r == 0) return;
        if (n + (r == 1 ? 2 : 1) > DR_EDGE_STACK) {
            ok = false;
            return;
        }
        if (CUT > 0) {
            c.left.node |= cdepth;
            c.right.node |= cdepth;
        }
        // depth first, left subtree before right
        if (c.push_r) st[n++] = c.right;
        if (c.push_l) st[n++] = c.left;
    }
};

// Stochastic traversal of one edge tree in one mode (edge_tree.cpp:511-652),
// start to finish: CONE true for the cone mode, false for the all mode.
// Returns false if the stack limit was hit (never for trees of depth <
// DR_EDGE_STACK).
template <bool PROP, int CUT = 0, class Emit, class Defer>
DEV bool traverse_mode(const bool CONE, const DevScene &s, const DevEdgeNode *nodes, const DevEdge *edges, int tree,
                       bool dir_bounds, float3 wi, const SurfacePoint &sp, float dl, float sl, float rough, int model,
                       const ConeSpec &cone, const EdgeTask &start, const NodeRng &rng, Emit &emit,
                       const EdgeProposal &pr, bool learned, Defer &defer, int *visits = nullptr) {
    EdgeWalk<PROP, CUT> w;
    w.start(CONE, s, nodes, edges, tree, dir_bounds, wi, sp, dl, sl, rough, model, cone, start, rng, pr, learned);
    while (w.busy()) w.step(emit, defer, visits);
    return w.ok;
}

// All edges sampled for one shading point (edge_tree.cpp:654-725).
// emit(tree, edge_index, weight); tree 0 = silhouette tree, 1 = normal tree.
// emit(tree, edge_index, key, weight, code): key = mode << 27 | edge index
// (the traversal order of the reference: cone mode first, then depth first).
// `rng` draws the tree pick; `nrng` the traversal's choices.
// No subtree is handed on.
struct NoDefer {
    HD void operator()(int, float, float, float, float) {}
};

template <bool PROP, int CUT = 0, class Emit, class Defer>
DEV bool traverse_edges(const DevScene &s, float3 wi, int stri, const SurfacePoint &sp, const ConeSpec &cone, Rng &rng,
                        const NodeRng &nrng, Emit &emit, const EdgeProposal &pr, Defer &defer,
                        int *visits = nullptr) {
    if (dot(wi, sp.f.n) < 0.f) return true;
    int tree;
    float pmf = 1.f;
    if (s.num_nrm_nodes == 0 && s.num_sil_nodes == 0) return true;
    if (s.num_nrm_nodes == 0) {
        tree = 0;
    } else if (s.num_sil_nodes == 0) {
        tree = 1;
    } else {
        float ni = s.nrm_nodes[0].total_length, si = s.sil_nodes[0].total_length;
        float np = ni / (ni + si), spm = si / (ni + si);
        float u = rng.next();
        if (u < np) {
            tree = 1;
            pmf = np;
        } else {
            tree = 0;
            pmf = spm;
        }
    }
    const DevEdgeNode *nodes = tree ? s.nrm_nodes : s.sil_nodes;
    const DevEdge *edges = tree ? s.nrm_edges : s.sil_edges;
    const DevMaterial &m = s.mats[material_of_tri(s, stri)];
    float dl = luminance(get_kd(s, m, sp.uv)), sl = luminance(get_ks(s, m, sp.uv));
    float rough = get_rough(s, m, sp.uv);
    float b = bsdf_bound(nodes[0], bound_ctx(wi, sp, dl, sl, rough, m.model));
    auto em = [&](int ei, int key, float w, int code) { emit(tree, ei, key, w, code); };
    EdgeTask root;
    root.point = 0;
    root.code = 0;
    root.bb = b;
    root.cpmf = root.apmf = root.lpmf = pmf;
    // cone mode, then all mode, through one copy of the walk (a loop, not
    // unrolled: the walk's code is the kernel's hot loop)
    bool ok = true;
#pragma unroll 1
    for (int mode = 0; mode < 2; mode++) {
        bool learned = PROP && mode == 1 ? nrng.draw(1, DR_NODE_MIX_DRAW) < pr.alpha : false;
        auto dc = [&](int node, float bb, float c, float a, float l) {
            defer(node | (tree << 29) | (mode << 30), bb, c, a, l);
        };
        ok &= traverse_mode<PROP, CUT>(mode == 0, s, nodes, edges, tree, tree == 1, wi, sp, dl, sl, rough, m.model,
                                       cone, root, nrng, em, pr, learned, dc, visits);
    }
    return ok;
}

// Starts the walk of one handed-on subtree of a point's traversal (the
// point's setup is recomputed: tree and mode come with the task).
template <bool PROP>
DEV void start_subtree(EdgeWalk<PROP> &w, const DevScene &s, float3 wi, int stri, const SurfacePoint &sp,
                       const ConeSpec &cone, const NodeRng &nrng, const EdgeTask &task, const EdgeProposal &pr) {
    const int tree = (task.code >> 29) & 1, mode = (task.code >> 30) & 1;
    const DevEdgeNode *nodes = tree ? s.nrm_nodes : s.sil_nodes;
    const DevEdge *edges = tree ? s.nrm_edges : s.sil_edges;
    const DevMaterial &m = s.mats[material_of_tri(s, stri)];
    float dl = luminance(get_kd(s, m, sp.uv)), sl = luminance(get_ks(s, m, sp.uv));
    float rough = get_rough(s, m, sp.uv);
    EdgeTask start = task;
    start.code = task.code & DR_NODE_MASK;  // depth bits cleared: walked to the leaves
    bool learned = PROP && mode == 1 ? nrng.draw(1, DR_NODE_MIX_DRAW) < pr.alpha : false;
    w.start(mode == 0, s, nodes, edges, tree, tree == 1, wi, sp, dl, sl, rough, m.model, cone, start, nrng, pr,
            learned);
}

// LTC matrix lookup (material.h:464-476): nearest entry of the 128x128 table
// of the material's lobe
DEV M3 ltc_matrix(const DevScene &s, int mi, const SurfacePoint &sp, float3 wi) {
    float r = get_rough(s, s.mats[mi], sp.uv);
    float ct = dot(wi, sp.f.n);
    float th = dr_acosf(ct);
    int rid = int(r * (128 - 1));
    int tid = int(((double)th / (3.14159265358979323846 / 2.f)) * (128 - 1));
    rid = rid < 0 ? 0 : (rid > 127 ? 127 : rid);
    tid = tid < 0 ? 0 : (tid > 127 ? 127 : tid);
    M3 m;
    const float *p = (s.mats[mi].model == DR_MICROFACET_GGX ? s.ltc_ggx : s.ltc) + 9 * (rid + tid * 128);
    for (int i = 0; i < 9; i++) m.m[i] = dr_ldg(p + i);
    return m;
}

// d p / d dir of a ray hitting the plane through p with normal n (vector.h:690-716)
DEV M3 intersect_jacobian(float3 dir, float3 p, float3 n) {
    M3 m;
    float d = -dot(p, n);
    float dn = dot(dir, n);
    if (fabsf(dn) < 1e-10f) {
        for (int i = 0; i < 9; i++) m.m[i] = 0.f;
        return m;
    }
    float inv2 = 1.f / (dn * dn);
    float t = -d / dn;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) m.m[3 * i + j] = (i == j ? t : 0.f) + comp(dir, i) * d * comp(n, j) * inv2;
    return m;
}
DEV M3 normalize_jacobian(float3 x) {
    float d2 = length_sq(x);
    float d = sqrtf(d2);
    float inv = 1.f / (d * d2);
    M3 m;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) m.m[3 * i + j] = ((i == j ? d2 : 0.f) - comp(x, i) * comp(x, j)) * inv;
    return m;
}

struct EdgeResult { float3 dp, dv0, dv1; };

// Density with which a lobe's line sample (the construction of
// delta_ray.cpp:107-160 in the lobe's space minv) picks the edge point at
// offset q from the shading point, per unit of another parameterisation l of
// the same edge with dq/dl = q_l.  0 where the lobe cannot sample (below its
// horizon).  d0, d1: edge endpoints relative to the shading point.
DEV_NOINLINE float lobe_line_density(const M3 &minv, float3 d0, float3 d1, float3 q, float3 q_l) {
    float3 a = mul(minv, d0), b = mul(minv, d1);
    if (a.z <= 0.f && b.z <= 0.f) return 0.f;
    if (a.z < 0.f) a = (a * b.z - b * a.z) / (b.z - a.z);
    if (b.z < 0.f) b = (a * b.z - b * a.z) / (b.z - a.z);
    float3 vod = b - a;
    if (abs_sum(vod) < 1e-10f) return 0.f;
    float3 wt = normalize(vod);
    float l0 = dot(a, wt), l1 = dot(b, wt);
    float3 vo = a - l0 * wt;
    float d = length(vo);
    auto I = [&](float l) {
        return (l / (d * (d * d + l * l)) + dr_atanf(l / d) / (d * d)) * vo.z + (l * l / (d * (d * d + l * l))) * wt.z;
    };
    float norm = I(l1) - I(l0);
    if (norm <= 1e-10f) return 0.f;
    float3 y = mul(minv, q);
    if (y.z < 0.f) return 0.f;
    float l = dot(y, wt);
    float ds = d * d + l * l;
    float p = 2.f * d * (vo + l * wt).z / (norm * ds * ds);
    return p > 0.f ? p * length(mul(minv, q_l)) : 0.f;
}

// Line density of the lobe that was not picked, at the sampled point (out of
// line: only DR_FLAG_EDGE_LOBE_MIS needs it).
DEV_NOINLINE float other_lobe_density(const DevScene &s, int mi, const SurfacePoint &sp, float3 wi, const M3 &frame,
                                      bool sel_diffuse, float3 v0, float3 v1, float3 sample_p, float3 q_l) {
    M3 ominv = sel_diffuse ? mul(inverse(ltc_matrix(s, mi, sp, wi)), frame) : frame;
    return lobe_line_density(ominv, v0 - sp.p, v1 - sp.p, sample_p, q_l);
}

// Secondary edge sample (delta_ray.cpp:45-365), in two phases: the line
// sample on the edge (edge_line_sample: the silhouette test, the LTC lobe, the
// point on the edge and the density it was drawn with) and the shading of the
// two sides (edge_shade_sample: rays, shading, Jacobians).  The backward pass
// runs them as two kernels with the surviving line samples compacted in
// between; shading_edge_sample runs both.
struct EdgeLine {
    float3 sample_p;  // the sampled point on the edge, relative to the shading point
    float3 mwt;       // d sample_p / d l (the lobe transform times the line direction)
    float q;          // density of l: the picked lobe's pmf times its line pdf (or the lobe mixture)
};

// What a line sample needs of its shading point and of the point's edge draw
// (the same for every edge the point sampled): the picked lobe's transform
// into its LTC space (minv) and back (m) and the lobe's pick probability; for
// the lobe mixture weight also both lobes' pick probabilities, the shading
// frame and the material.  ok false: the point samples no edge (no surface,
// or a black material).
struct LineSetup {
    M3 minv, m, frame;
    float mpmf, dpmf, spmf;
    int mi;
    bool ok;
};
DEV LineSetup line_setup(const DevScene &s, const EdgeSample &es, float3 wi, int stri, const SurfacePoint &sp) {
    LineSetup ls;
    ls.ok = false;
    if (stri < 0) return ls;
    const int mi = material_of_tri(s, stri);
    const DevMaterial &mat = s.mats[mi];
    float3 kd = get_kd(s, mat, sp.uv), ks = get_ks(s, mat, sp.uv);
    float dw = luminance(kd), sw = luminance(ks), ws = dw + sw;
    if (ws <= 0.f) return ls;
    float dpmf = dw / ws, spmf = sw / ws;
    float3 n = sp.f.n;
    float3 fx = normalize(wi - n * dot(wi, n));
    float3 fy = cross(n, fx);
    M3 frame = m3_rows(fx, fy, n);
    if (es.bsdf_component <= dpmf) {
        ls.minv = frame;
        ls.m = inverse(ls.minv);
        ls.mpmf = dpmf;
    } else {
        ls.minv = mul(inverse(ltc_matrix(s, mi, sp, wi)), frame);
        ls.m = inverse(ls.minv);
        ls.mpmf = spmf;
    }
    ls.frame = frame;
    ls.dpmf = dpmf;
    ls.spmf = spmf;
    ls.mi = mi;
    ls.ok = true;
    return ls;
}

// The line sample of one edge from its point's setup (delta_ray.cpp:88-187):
// the edge clipped to the lobe's upper hemisphere in LTC space, the point on
// it drawn by inverting the line integral's CDF (Newton steps guarded by
// bisection), its density.  EXT adds the lobe mixture weight (sp and wi are
// read only then).  rec (may be null): the edge's silhouette-test record,
// which gives the answer of is_silhouette from one contiguous read.
template <bool EXT = true>
DEV bool line_sample_from(const DevScene &s, const LineSetup &ls, const EdgeSample &es, const DevEdge &edge, float3 p,
                          const SurfacePoint &sp, float3 wi, EdgeLine &out, const EdgeRec *rec) {
    const bool none = false;
    if (!(rec ? is_silhouette_rec(rec, p) : is_silhouette(s, p, edge))) return none;
    float3 v0 = edge_v0(s, edge), v1 = edge_v1(s, edge);
    if (abs_sum(v1 - v0) == 1e-10f) return none;
    const M3 &minv = ls.minv, &m = ls.m;
    float3 a = mul(minv, v0 - p), b = mul(minv, v1 - p);
    if (a.z <= 0.f && b.z <= 0.f) return none;
    if (a.z < 0.f) a = (a * b.z - b * a.z) / (b.z - a.z);
    if (b.z < 0.f) b = (a * b.z - b * a.z) / (b.z - a.z);
    float3 vod = b - a;
    if (abs_sum(vod) < 1e-10f) return none;
    float3 wt = normalize(vod);
    float l0 = dot(a, wt), l1 = dot(b, wt);
    float3 vo = a - l0 * wt;
    float d = length(vo);
    auto I = [&](float l) {
        return (l / (d * (d * d + l * l)) + dr_atanf(l / d) / (d * d)) * vo.z + (l * l / (d * (d * d + l * l))) * wt.z;
    };
    float Il0 = I(l0), Il1 = I(l1);
    float norm = Il1 - Il0;
    if (norm <= 1e-10f) return none;
    auto cdf = [&](float l) { return (I(l) - Il0) / norm; };
    auto pdf = [&](float l) {
        float ds = d * d + l * l;
        return 2.f * d * (vo + l * wt).z / (norm * ds * ds);
    };
    float lb = l0, ub = l1;
    if (lb > ub) {
        float t = lb;
        lb = ub;
        ub = t;
    }
    float l = 0.5f * (lb + ub);
    for (int it = 0; it < 20; it++) {
        if (!(l >= lb && l <= ub)) l = 0.5f * (lb + ub);
        float value = cdf(l) - es.u;
        if (fabsf(value) < 1e-5f || it == 19) break;
        if (value > 0.f) ub = l;
        else lb = l;
        l -= value / pdf(l);
    }
    if (pdf(l) <= 0.f) return none;
    float3 sample_p = mul(m, vo + l * wt);
    // DR_FLAG_EDGE_LOBE_MIS: the one-sample balance heuristic over the two
    // lobes, pmf_sel pdf_sel(l) + pmf_other pdf_other(l); the reference divides
    // by pmf_sel pdf_sel(l) alone
    float q_mix = ls.mpmf * pdf(l);
    if (EXT && s.edge_lobe_mis) {
        bool sel_diffuse = es.bsdf_component <= ls.dpmf;
        float opmf = sel_diffuse ? ls.spmf : ls.dpmf;
        if (opmf > 0.f)
            q_mix += opmf * other_lobe_density(s, ls.mi, sp, wi, ls.frame, sel_diffuse, v0, v1, sample_p, mul(m, wt));
    }
    out.sample_p = sample_p;
    out.mwt = mul(m, wt);
    out.q = q_mix;
    return true;
}

// rec (may be null): the edge's silhouette-test record.
template <bool EXT = true>
DEV bool edge_line_sample(const DevScene &s, const EdgeSample &es, const DevEdge &edge, float3 wi, int stri,
                          const SurfacePoint &sp, EdgeLine &out, const EdgeRec *rec = nullptr) {
    const LineSetup ls = line_setup(s, es, wi, stri, sp);
    if (!ls.ok) return false;
    return line_sample_from<EXT>(s, ls, es, edge, sp.p, sp, wi, out, rec);
}

// The two rays of an edge sample, one on each side of the edge: their closest
// hits and the tests that need nothing but the hits (delta_ray.cpp:223-313:
// exactly one side must hit a face of the edge, neither may hit the shading
// point's own triangle, neither hit may lie on a near-degenerate segment).
// With direct lighting only (DIRECT_ONLY), a sample neither of whose sides hits
// an emitter contributes nothing and ends here too.
struct EdgeHits {
    int r, l;  // closest-hit triangles of the "right" (+split_n) and "left" ray, -1 for none
};

DEV void edge_side_dirs(const EdgeLine &el, float3 v0, float3 v1, float3 p, float3 &sdir, float3 &rdir, float3 &ldir) {
    float3 split_n = normalize(cross(v0 - p, v1 - p));
    float delta = 1e-3f * length(el.sample_p);
    sdir = normalize(el.sample_p);
    rdir = normalize(sdir + delta * split_n);
    ldir = normalize(sdir - delta * split_n);
}

// The closest hit among the edge's faces, under the closest-hit rule and with
// the operands the LBVH's leaves hold (vertices in index order), for both
// sides' rays, which share their origin: each face's edge vectors and origin
// offset serve both rays.
DEV void hit_faces_pair(const DevScene &s, const DevEdge &edge, float3 o, float3 dr, float3 dl, float tnear, Hit &hr,
                        Hit &hl) {
    const int off = s.shapes[edge.shape].tri_off;
    const int g0 = off + edge.f0, g1 = edge.f1 >= 0 ? off + edge.f1 : -1;
    hr.tri = hl.tri = -1;
    hr.t = hl.t = DR_INF;
#pragma unroll 1
    for (int k = 0; k < 2; k++) {
        const int g = k ? g1 : g0;
        if (g < 0) continue;
        const int4 id = s.tri[g];
        float4 v[3];
        const int vi[3] = {id.x, id.y, id.z};
        for (int j = 0; j < 3; j++) {
            v[j].x = s.vtx[3 * vi[j]];
            v[j].y = s.vtx[3 * vi[j] + 1];
            v[j].z = s.vtx[3 * vi[j] + 2];
            v[j].w = 0.f;
        }
        const TriRay r = tri_ray(v[0], v[1], v[2], o);
        float t;
        if (hit_triangle(r, dr, t) && t > tnear && (t < hr.t || (t == hr.t && g < hr.tri))) {
            hr.t = t;
            hr.tri = g;
        }
        if (hit_triangle(r, dl, t) && t > tnear && (t < hl.t || (t == hl.t && g < hl.tri))) {
            hl.t = t;
            hl.tri = g;
        }
    }
}


// The connectivity test of an edge sample in an LBVH scene (most samples
// end here: edges hidden from p).  A side's closest hit is one of the edge's
// faces only if its ray hits one of them, at (ta, ida) by the closest-hit
// rule, and no triangle hits ahead of that.  True if exactly one side is
// connected: `side` (0 the right ray, 1 the left) and `face`, its closest hit.
DEV bool edge_connect_bvh(const DevScene &s, const DevEdge &edge, float3 p, float3 rdir, float3 ldir, int &side,
                          int &face) {
    Hit fr, fl;
    hit_faces_pair(s, edge, p, rdir, ldir, 1e-3f, fr, fl);
    if (fr.tri < 0 && fl.tri < 0) return false;
    const bool cr = fr.tri >= 0 && !trace_before(s, p, rdir, 1e-3f, fr.t, fr.tri);
    if (!cr && fl.tri < 0) return false;
    const bool cl = fl.tri >= 0 && !trace_before(s, p, ldir, 1e-3f, fl.t, fl.tri);
    if (cr == cl) return false;
    side = cr ? 0 : 1;
    face = cr ? fr.tri : fl.tri;
    return true;
}

// The tests on the two sides' closest hits after the connectivity test: a
// side that hits the shading point's own triangle, or a hit point nearly in
// the plane through p along its ray (degenerate), ends the sample; with
// direct lighting only, so does a sample neither of whose sides reaches an
// emitter.
DEV bool edge_hits_ok(const DevScene &s, int stri, float3 p, float3 rdir, float3 ldir, const int *hit,
                      bool direct_only) {
    if ((hit[0] >= 0 && hit[0] == stri) || (hit[1] >= 0 && hit[1] == stri)) return false;
#pragma unroll 1
    for (int k = 0; k < 2; k++) {
        if (hit[k] < 0) continue;
        SurfacePoint pp = intersect_tri(load_tri(s, hit[k]), p, k == 0 ? rdir : ldir);
        float3 dir = pp.p - p;
        if (length(dir) * fabsf(dot(normalize(dir), pp.ng)) < 1e-3f) return false;
    }
    if (direct_only && (hit[0] < 0 || light_of_tri(s, hit[0]) < 0) && (hit[1] < 0 || light_of_tri(s, hit[1]) < 0))
        return false;
    return true;
}

// The rest of an LBVH scene's sample once one side is connected: the other
// side's closest hit, then edge_hits_ok.
DEV bool edge_rays_rest(const DevScene &s, int stri, float3 p, float3 rdir, float3 ldir, int side, int face,
                        bool direct_only, EdgeHits &out) {
    int hit[2];
    hit[side] = face;
    hit[1 - side] = trace_closest(s, p, side ? rdir : ldir, 1e-3f).tri;
    if (!edge_hits_ok(s, stri, p, rdir, ldir, hit, direct_only)) return false;
    out.r = hit[0];
    out.l = hit[1];
    return true;
}

DEV bool edge_rays(const DevScene &s, const EdgeLine &el, const DevEdge &edge, int stri, float3 p, bool direct_only,
                   EdgeHits &out) {
    float3 sdir, rdir, ldir;
    edge_side_dirs(el, edge_v0(s, edge), edge_v1(s, edge), p, sdir, rdir, ldir);
    if (s.num_tris > DR_LINEAR_TRIS) {
        int side, face;
        if (!edge_connect_bvh(s, edge, p, rdir, ldir, side, face)) return false;
        return edge_rays_rest(s, stri, p, rdir, ldir, side, face, direct_only, out);
    }
    int hit[2];
    if (s.num_tris > 0) {
        Hit h0, h1;
        trace_closest_pair_linear(s.bvh_tris, s.num_tris, p, rdir, ldir, 1e-3f, h0, h1);
        hit[0] = h0.tri;
        hit[1] = h1.tri;
    } else {
        hit[0] = hit[1] = -1;
    }
    bool conn[2];
#pragma unroll 1
    for (int k = 0; k < 2; k++) {
        conn[k] = false;
        if (hit[k] >= 0) {
            int lt = s.tri_local[hit[k]];
            conn[k] = s.tri[hit[k]].w == edge.shape && (lt == edge.f0 || lt == edge.f1);
        }
    }
    if (conn[0] == conn[1] || !edge_hits_ok(s, stri, p, rdir, ldir, hit, direct_only)) return false;
    out.r = hit[0];
    out.l = hit[1];
    return true;
}

// The shading of an edge sample whose rays edge_rays kept: the emitters and
// (with more bounces) the radiance seen on each side, the BSDF toward the
// edge, and the Jacobians of the sample w.r.t. the shading point and the
// edge's end points.
// The radiance each side of an edge sample receives beyond its closest hit
// (more bounces than one), divided by the squared distance and times the
// cosine at the hit, as edge_shade_hits uses it; false (and zeros) when the
// BSDF toward the edge is negligible, where edge_shade_hits ends the sample.
DEV bool edge_side_radiance(const DevScene &s, const EdgeLine &el_, const DevEdge &edge, const LightSample &ls,
                            const Rng &rng, int nbounces, float3 wi, int stri, const SurfacePoint &sp,
                            const EdgeHits &hits, float3 &shr, float3 &shl) {
    shr = shl = f3(0.f);
    float3 v0 = edge_v0(s, edge), v1 = edge_v1(s, edge);
    float3 sdir, rdir, ldir;
    edge_side_dirs(el_, v0, v1, sp.p, sdir, rdir, ldir);
    if (sum(bsdf(s, material_of_tri(s, stri), sp, wi, sdir)) < 1e-6f) return false;
#pragma unroll 1
    for (int k = 0; k < 2; k++) {
        int tri = k == 0 ? hits.r : hits.l;
        SurfacePoint pp;
        if (tri >= 0) pp = intersect_tri(load_tri(s, tri), sp.p, k == 0 ? rdir : ldir);
        float3 sh = shade(s, -sdir, tri, pp, ls, rng, nbounces, false);
        if (tri >= 0) {
            float3 dir = pp.p - sp.p;
            float d2 = length_sq(dir);
            if (d2 > 0.f) sh = sh / fmaxf(d2, 1e-2f) * fabsf(dot(normalize(dir), pp.ng));
            else sh = f3(0.f);
        }
        if (k == 0) shr = sh;
        else shl = sh;
    }
    return true;
}

// PRE: the two sides' radiance comes from edge_side_radiance, computed by an
// earlier kernel (rad[0] right, rad[1] left), and shade() is not compiled in.
template <bool MAYBE_GI = true, bool PRE = false>
DEV EdgeResult edge_shade_hits(const DevScene &s, const EdgeLine &el_, const DevEdge &edge, const LightSample &ls,
                               const Rng &rng, int nbounces, float3 wi, int stri, const SurfacePoint &sp,
                               float3 weight, float3 d_color, bool direct_only, const EdgeHits &hits,
                               const float3 *rad = nullptr) {
    EdgeResult none;
    none.dp = none.dv0 = none.dv1 = f3(0.f);
    const float3 sample_p = el_.sample_p;
    float3 v0 = edge_v0(s, edge), v1 = edge_v1(s, edge);
    int mi = material_of_tri(s, stri);
    float3 sdir, rdir, ldir;
    edge_side_dirs(el_, v0, v1, sp.p, sdir, rdir, ldir);
    SurfacePoint pr, pl;
    if (hits.r >= 0) pr = intersect_tri(load_tri(s, hits.r), sp.p, rdir);
    if (hits.l >= 0) pl = intersect_tri(load_tri(s, hits.l), sp.p, ldir);
    float3 eb = bsdf(s, mi, sp, wi, sdir);
    if (sum(eb) < 1e-6f) return none;
    float3 shr = f3(0.f), shl = f3(0.f);
    if (PRE) {
        if (MAYBE_GI && !direct_only) {
            shr = rad[0];
            shl = rad[1];
        }
    } else if (MAYBE_GI && !direct_only) {
#pragma unroll 1
        for (int k = 0; k < 2; k++) {
            int tri = k == 0 ? hits.r : hits.l;
            SurfacePoint pp = k == 0 ? pr : pl;
            float3 sh = shade(s, -sdir, tri, pp, ls, rng, nbounces, false);
            if (tri >= 0) {
                float3 dir = pp.p - sp.p;
                float d2 = length_sq(dir);
                if (d2 > 0.f) sh = sh / fmaxf(d2, 1e-2f) * fabsf(dot(normalize(dir), pp.ng));
                else sh = f3(0.f);
            }
            if (k == 0) shr = sh;
            else shl = sh;
        }
    }
    float3 er, el;
#pragma unroll 1
    for (int k = 0; k < 2; k++) {
        float3 e = k == 0 ? eval_light(s, wi, stri, sp, hits.r, pr) + eb * shr
                          : eval_light(s, wi, stri, sp, hits.l, pl) + eb * shl;
        if (k == 0) er = e;
        else el = e;
    }
    EdgeResult res = none;
    auto accum = [&](const SurfacePoint &lp, float3 ev) {
        M3 nj = normalize_jacobian(sample_p);
        M3 ij = intersect_jacobian(sdir, lp.p, lp.ng);
        float line_j = length(mul(mul(ij, nj), el_.mwt)) / el_.q;
        float3 p = sp.p, x = lp.p;
        float3 d0 = v0 - p, d1 = v1 - p;
        float dirac_j = length(cross(d0, d1));
        float w = line_j / dirac_j;
        float3 dp = w * (cross(d1, d0) + cross(x - p, d1) + cross(d0, x - p));
        float3 dv0 = w * cross(d1, x - p);
        float3 dv1 = w * cross(x - p, d0);
        float we = dot(ev * weight, d_color);
        res.dp += dp * we;
        res.dv0 += dv0 * we;
        res.dv1 += dv1 * we;
    };
#pragma unroll 1
    for (int k = 0; k < 2; k++) {
        int tri = k == 0 ? hits.r : hits.l;
        float3 e = k == 0 ? er : el;
        if (tri >= 0 && abs_sum(e) > 0.f) accum(k == 0 ? pr : pl, k == 0 ? e : -e);
    }
    return res;
}

// The whole shading of an edge sample: edge_rays, then edge_shade_hits.
template <bool MAYBE_GI = true>
DEV EdgeResult edge_shade_sample(const DevScene &s, const EdgeLine &el, const DevEdge &edge, const LightSample &ls,
                                 const Rng &rng, int nbounces, float3 wi, int stri, const SurfacePoint &sp,
                                 float3 weight, float3 d_color, bool direct_only) {
    EdgeHits hits;
    if (!edge_rays(s, el, edge, stri, sp.p, direct_only || !MAYBE_GI, hits)) {
        EdgeResult none;
        none.dp = none.dv0 = none.dv1 = f3(0.f);
        return none;
    }
    return edge_shade_hits<MAYBE_GI>(s, el, edge, ls, rng, nbounces, wi, stri, sp, weight, d_color, direct_only, hits);
}

template <bool EXT = true, bool MAYBE_GI = true>
DEV EdgeResult shading_edge_sample(const DevScene &s, const EdgeSample &es, const DevEdge &edge, const LightSample &ls,
                                   const Rng &rng, int nbounces, float3 wi, int stri, const SurfacePoint &sp,
                                   float3 weight, float3 d_color, bool direct_only) {
    EdgeLine el;
    if (!edge_line_sample<EXT>(s, es, edge, wi, stri, sp, el)) {
        EdgeResult none;
        none.dp = none.dv0 = none.dv1 = f3(0.f);
        return none;
    }
    return edge_shade_sample<MAYBE_GI>(s, el, edge, ls, rng, nbounces, wi, stri, sp, weight, d_color, direct_only);
}

// ---------------------------------------------------------------------------
// Primary edges (camera.h:86-313, delta_ray.cpp:377-557)
// ---------------------------------------------------------------------------
// Fisheye branches out of line (rarely taken, large trigonometry).
DEV_NOINLINE float3 unproject_fisheye(float sx, float sy) {
    float x = 2.f * (sx - 0.5f), y = 2.f * (sy - 0.5f);
    float r = sqrtf(x * x + y * y), phi = dr_atan2f(y, x), theta = r * DR_PI / 2.f;
    return f3(-dr_cosf(phi) * dr_sinf(theta), -dr_sinf(phi) * dr_sinf(theta), dr_cosf(theta));
}
struct F3Pair { float3 a, b; };
DEV_NOINLINE F3Pair d_unproject_fisheye(float sx, float sy) {
    float x = 2.f * (sx - 0.5f), y = 2.f * (sy - 0.5f);
    float r = sqrtf(x * x + y * y), phi = dr_atan2f(y, x), theta = r * DR_PI / 2.f;
    float sp = dr_sinf(phi), cp = dr_cosf(phi), st = dr_sinf(theta), ct = dr_cosf(theta);
    float dxdphi = sp * st, dxdth = -cp * ct, dydphi = -cp * st, dydth = -sp * ct, dzdth = -st;
    float dphidx = -y / (r * r), dphidy = x / (r * r);
    float dthdx = (DR_PI / 2.f) * x / r, dthdy = (DR_PI / 2.f) * y / r;
    F3Pair d;
    d.a = 2.f * f3(dxdphi * dphidx + dxdth * dthdx, dydphi * dphidx + dydth * dthdx, dzdth * dthdx);
    d.b = 2.f * f3(dxdphi * dphidy + dxdth * dthdy, dydphi * dphidy + dydth * dthdy, dzdth * dthdy);
    return d;
}
DEV_NOINLINE float2 project_local_fisheye(float3 l) {
    float2 r;
    float3 d = normalize(l);
    float phi = dr_atan2f(d.y, d.x), theta = dr_acosf(d.z), rr = theta * 2.f / DR_PI;
    r.x = 0.5f * (-rr * dr_cosf(phi) + 1.f);
    r.y = 0.5f * (-rr * dr_sinf(phi) + 1.f);
    return r;
}
DEV_NOINLINE float3 d_project_local_fisheye(float3 l, float dx, float dy) {
    float3 d = normalize(l);
    float phi = dr_atan2f(d.y, d.x), theta = dr_acosf(d.z), r = theta * 2.f / DR_PI;
    float dr = -0.5f * (dr_cosf(phi) * dx + dr_sinf(phi) * dy);
    float dphi = 0.5f * r * dr_sinf(phi) * dx - 0.5f * r * dr_cosf(phi) * dy;
    float dtheta = dr * (2.f / DR_PI);
    float dcos = -dtheta / sqrtf(1.f - d.z * d.z);
    float t = d.x * d.x + d.y * d.y;
    return d_normalize(l, f3(-dphi * d.y / t, dphi * d.x / t, dcos));
}

DEV float3 unproject(const DevCamera &c, float sx, float sy) {
    if (c.fisheye) return unproject_fisheye(sx, sy);
    float ndcx = (sx - 0.5f) * -2.f, ndcy = (sy - 0.5f) * -2.f / c.aspect;
    return f3(c.fov * ndcx, c.fov * ndcy, 1.f);
}
DEV void d_unproject(const DevCamera &c, float sx, float sy, float3 &dx, float3 &dy) {
    if (c.fisheye) {
        F3Pair d = d_unproject_fisheye(sx, sy);
        dx = d.a;
        dy = d.b;
        return;
    }
    dx = f3(-2.f * c.fov, 0.f, 0.f);
    dy = f3(0.f, -2.f * c.fov / c.aspect, 0.f);
}
DEV float2 project_local(const DevCamera &c, float3 l) {
    if (c.fisheye) return project_local_fisheye(l);
    float2 r;
    r.x = (-l.x / (l.z * c.fov) + 1.f) * 0.5f;
    r.y = (-l.y / (l.z * c.fov * c.aspect) + 1.f) * 0.5f;
    return r;
}
DEV float3 d_project_local(const DevCamera &c, float3 l, float dx, float dy) {
    if (c.fisheye) return d_project_local_fisheye(l, dx, dy);
    float zf = l.z * c.fov;
    float zfy = zf * c.aspect;
    return f3(dx * (-1.f / zf), dy * (-1.f / zfy),
              dx * (c.fov * l.x / (zf * zf)) + dy * (c.fov * c.aspect * l.y / (zfy * zfy)));
}
DEV bool project(const DevCamera &c, float3 p0, float3 p1, float2 &s0, float2 &s1) {
    float3 a = xfm_point(c.w2c, p0), b = xfm_point(c.w2c, p1);
    if (a.z < c.clip_near && b.z < c.clip_near) return false;
    if (a.z < c.clip_near) {
        float3 dir = a - b;
        float t = -(b.z - c.clip_near) / dir.z;
        a = b + t * dir;
    } else if (b.z < c.clip_near) {
        float3 dir = b - a;
        float t = -(a.z - c.clip_near) / dir.z;
        b = a + t * dir;
    }
    s0 = project_local(c, a);
    s1 = project_local(c, b);
    return true;
}
// d_project (camera.h:244-313), including its +clip_near sign
DEV void d_project(const DevCamera &c, float3 p0, float3 p1, float dp0x, float dp0y, float dp1x, float dp1y, float *dw2c) {
    float3 a = xfm_point(c.w2c, p0), b = xfm_point(c.w2c, p1);
    float3 ca = a, cb = b;
    if (a.z < c.clip_near) {
        float3 dir = a - b;
        float t = -(b.z + c.clip_near) / dir.z;
        ca = b + t * dir;
    } else if (b.z < c.clip_near) {
        float3 dir = b - a;
        float t = -(a.z + c.clip_near) / dir.z;
        cb = a + t * dir;
    }
    float3 dca = d_project_local(c, ca, dp0x, dp0y), dcb = d_project_local(c, cb, dp1x, dp1y);
    float3 da = f3(0.f), db = f3(0.f);
    if (a.z < c.clip_near) {
        float3 dir = a - b;
        float t = -(b.z + c.clip_near) / dir.z;
        db += dca;
        float dt = dot(dir, dca);
        float3 ddir = t * dca;
        db.z += -dt / dir.z;
        ddir.z += dt * (b.z / (dir.z * dir.z));
        da += ddir;
        db -= ddir;
        db += dcb;
    } else if (b.z < c.clip_near) {
        float3 dir = b - a;
        float t = -(a.z + c.clip_near) / dir.z;
        da += dcb;
        float dt = dot(dir, dcb);
        float3 ddir = t * dcb;
        da.z += -dt / dir.z;
        ddir.z += dt * (a.z / (dir.z * dir.z));
        db += ddir;
        da -= ddir;
        da += dca;
    } else {
        da = dca;
        db = dcb;
    }
    d_xfm_point(c.w2c, p0, da, dw2c);
    d_xfm_point(c.w2c, p1, db, dw2c);
}
DEV bool in_screen(const DevCamera &c, float2 p) {
    if (!c.fisheye) return p.x >= 0.f && p.x < 1.f && p.y >= 0.f && p.y < 1.f;
    return (p.x - 0.5f) * (p.x - 0.5f) + (p.y - 0.5f) * (p.y - 0.5f) < 0.25f;
}

struct PrimaryEdgeResult {
    bool ok;
    DevEdge edge;
    float3 dv0, dv1;
    float dw2c[16];
};

// A primary-edge sample in three parts, so that the shading and the
// Jacobians can run as separate kernels (k_primary_shade, k_primary_grad):
// primary_edge_geom (the sample's point on the projected edge),
// primary_edge_colors (the two camera rays beside it and their shades),
// primary_edge_grad (Jacobians and the scene / camera gradients).
struct PrimaryGeom {
    float3 v0, v1, d0, d1, vd, ept3, split_n;
    float2 s0, s1, ept;
    float t, delta;
};

DEV bool primary_edge_geom(const DevCamera &cam, const DevScene &s, const EdgeSample &es, const DevEdge &edge,
                           PrimaryGeom &g) {
    g.v0 = edge_v0(s, edge);
    g.v1 = edge_v1(s, edge);
    if (!project(cam, g.v0, g.v1, g.s0, g.s1)) return false;
    g.d0 = unproject(cam, g.s0.x, g.s0.y);
    g.d1 = unproject(cam, g.s1.x, g.s1.y);
    g.vd = g.d1 - g.d0;
    g.t = es.u;
    float3 l0 = xfm_point(cam.w2c, g.v0), l1 = xfm_point(cam.w2c, g.v1);
    g.ept3 = g.d0 + g.t * g.vd;
    float3 elocal = l0 + g.t * l1;  // as written in delta_ray.cpp:403
    g.ept = project_local(cam, g.ept3);
    if (!in_screen(cam, g.ept)) return false;
    g.delta = 1e-4f * length(elocal);
    g.split_n = normalize(cross(g.d0, g.d1));
    return true;
}

// Screen point of the camera ray on side k (0: +split_n, 1: -split_n).
DEV float2 primary_side_point(const DevCamera &cam, const PrimaryGeom &g, int k) {
    float3 dir = normalize(k == 0 ? g.ept3 + g.delta * g.split_n : g.ept3 - g.delta * g.split_n);
    return project_local(cam, dir);
}

// rcol - lcol of the two sides; false if neither side's ray hits a face of the edge.
template <int BMAX = 1 << 30>
DEV bool primary_edge_colors(const DevScene &s, const PrimaryGeom &g, const DevEdge &edge, const LightSample &ls,
                             const Rng &rng, int B, float3 &diff) {
    const DevCamera &cam = s.cam;
    // right side (+split_n) then left, through one copy of the code
    Ray rray, lray;
    Hit hr, hl;
#pragma unroll 1
    for (int k = 0; k < 2; k++) {
        float2 pt = primary_side_point(cam, g, k);
        Ray ray = sample_primary(cam, pt.x, pt.y);
        Hit hh = trace_closest(s, ray.o, ray.d, 1e-3f);
        if (k == 0) {
            rray = ray;
            hr = hh;
        } else {
            lray = ray;
            hl = hh;
        }
    }
    bool rc = hr.tri >= 0 && s.tri[hr.tri].w == edge.shape &&
              (s.tri_local[hr.tri] == edge.f0 || s.tri_local[hr.tri] == edge.f1);
    bool lc = hl.tri >= 0 && s.tri[hl.tri].w == edge.shape &&
              (s.tri_local[hl.tri] == edge.f0 || s.tri_local[hl.tri] == edge.f1);
    if (!rc && !lc) return false;
    float3 rcol = f3(0.f), lcol = f3(0.f);
#pragma unroll 1
    for (int k = 0; k < 2; k++) {
        int tri = k == 0 ? hr.tri : hl.tri;
        Ray ray = k == 0 ? rray : lray;
        float3 col = f3(0.f);
        if (tri >= 0)
            col = shade<BMAX>(s, -ray.d, tri, intersect_tri(load_tri(s, tri), ray.o, ray.d), ls, rng, B, true);
        if (k == 0) rcol = col;
        else lcol = col;
    }
    diff = rcol - lcol;
    return true;
}

// Jacobians of a sample whose sides' colors differ by `cdiff` (rcol - lcol),
// scaled by `weight`; r.ok false if a perturbed end point leaves the view.
DEV void primary_edge_grad(const DevScene &s, const PrimaryGeom &g, const DevEdge &edge, float3 cdiff,
                           const float *d_image, int W, int H, float weight, PrimaryEdgeResult &r) {
    r.ok = false;
    const DevCamera &cam = s.cam;
    const float3 v0 = g.v0, v1 = g.v1, d0 = g.d0, d1 = g.d1, vd = g.vd;
    const float2 s0 = g.s0, s1 = g.s1, ept = g.ept;
    const float t = g.t, delta = g.delta;
    // the edge point is on the screen (in_screen: [0, 1)^2), but ept.x * W
    // can round up to W when W is a power of two; the reference reads past the
    // row there (delta_ray.cpp:411-416), this clamps to the last pixel
    int xi = int(ept.x * W), yi = int(ept.y * H);
    xi = xi < W ? xi : W - 1;
    yi = yi < H ? yi : H - 1;
    const float *dc = d_image + 3 * ((size_t)yi * W + xi);
    float3 d_color = f3(dr_ldg(dc), dr_ldg(dc + 1), dr_ldg(dc + 2));
    float2 rpt = primary_side_point(cam, g, 0), lpt = primary_side_point(cam, g, 1);
    float3 diff = cdiff * weight;
    float3 xdiff = diff, ydiff = diff;
    if (lpt.x > rpt.x) xdiff = -xdiff;
    if (lpt.y > rpt.y) ydiff = -ydiff;
    float3 edir = unproject(cam, ept.x, ept.y);
    float3 dv0x, dv0y, dv1x, dv1y, dex, dey;
    d_unproject(cam, s0.x, s0.y, dv0x, dv0y);
    d_unproject(cam, s1.x, s1.y, dv1x, dv1y);
    d_unproject(cam, ept.x, ept.y, dex, dey);
    float3 c01 = cross(d0, d1);
    float dadx = dot(dex, c01), dady = dot(dey, c01);
    float a0x = fabsf(dot(cross(d1, edir), dv0x)), a0y = fabsf(dot(cross(d1, edir), dv0y));
    float a1x = fabsf(dot(cross(edir, d0), dv1x)), a1y = fabsf(dot(cross(edir, d0), dv1y));
    float dirac_j = 1.f / sqrtf(dadx * dadx + dady * dady);
    float3 ept3d = d0 + (t + delta) * vd;
    float2 eptd = project_local(cam, ept3d);
    float ddx = (eptd.x - ept.x) / delta, ddy = (eptd.y - ept.y) / delta;
    float line_j = sqrtf(ddx * ddx + ddy * ddy);
    float jac = line_j * dirac_j;
    float g0x = dot(-xdiff * a0x * jac, d_color), g0y = dot(-ydiff * a0y * jac, d_color);
    float g1x = dot(-xdiff * a1x * jac, d_color), g1y = dot(-ydiff * a1y * jac, d_color);
    const float h = 1e-3f;
    float2 p0[6], p1[6];
    for (int k = 0; k < 3; k++) {
        float3 off = f3(k == 0 ? h : 0.f, k == 1 ? h : 0.f, k == 2 ? h : 0.f);
        if (!project(cam, v0 + off, v1, p0[k], p1[k])) return;
    }
    for (int k = 0; k < 3; k++) {
        float3 off = f3(k == 0 ? h : 0.f, k == 1 ? h : 0.f, k == 2 ? h : 0.f);
        if (!project(cam, v0, v1 + off, p0[3 + k], p1[3 + k])) return;
    }
    float dv0[3], dv1[3];
    for (int k = 0; k < 3; k++) {
        float a0 = (p0[k].x - s0.x) / h, a1 = (p0[k].y - s0.y) / h;
        float b0 = (p1[k].x - s1.x) / h, b1 = (p1[k].y - s1.y) / h;
        dv0[k] = g0x * a0 + g0y * a1 + g1x * b0 + g1y * b1;
        float c0 = (p0[3 + k].x - s0.x) / h, c1 = (p0[3 + k].y - s0.y) / h;
        float e0 = (p1[3 + k].x - s1.x) / h, e1 = (p1[3 + k].y - s1.y) / h;
        dv1[k] = g0x * c0 + g0y * c1 + g1x * e0 + g1y * e1;
    }
    r.ok = true;
    r.edge = edge;
    r.dv0 = f3(dv0[0], dv0[1], dv0[2]);
    r.dv1 = f3(dv1[0], dv1[1], dv1[2]);
    for (int i = 0; i < 16; i++) r.dw2c[i] = 0.f;
    d_project(cam, v0, v1, g0x, g0y, g1x, g1y, r.dw2c);
}

// The whole sample (delta_ray.cpp:377-557).
template <int BMAX = 1 << 30>
DEV void primary_edge_sample(const DevScene &s, const EdgeSample &es, const DevEdge &edge, const LightSample &ls,
                             const Rng &rng, int B, const float *d_image, int W, int H, float weight,
                             PrimaryEdgeResult &r) {
    r.ok = false;
    PrimaryGeom g;
    if (!primary_edge_geom(s.cam, s, es, edge, g)) return;
    float3 diff;
    if (!primary_edge_colors<BMAX>(s, g, edge, ls, rng, B, diff)) return;
    primary_edge_grad(s, g, edge, diff, d_image, W, H, weight, r);
}
