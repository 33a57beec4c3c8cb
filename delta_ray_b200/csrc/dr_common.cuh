// Common device math for the B200 path tracer: float3 algebra, frames, 3x3 and
// 4x4 matrices, the Philox4x32-10 counter-based generator and small helpers.
//
// Everything here is __host__ __device__ so that the per-sample kernel logic
// can also be compiled for the host by the test harness (DR_HOST_BUILD); the
// product only ever runs it on the GPU.
#pragma once

#include <stdint.h>

#ifdef DR_HOST_BUILD
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#define HD inline
#define DEV inline
#define DEV_NOINLINE inline
#define DR_RESTRICT
#define DR_TABLE static const
struct float2 { float x, y; };
struct float3 { float x, y, z; };
struct float4 { float x, y, z, w; };
struct int2 { int x, y; };
struct int4 { int x, y, z, w; };
template <typename T> inline T dr_ldg(const T *p) { return *p; }
inline void dr_atomic_add(float *p, float v) { *p += v; }
inline unsigned dr_umulhi(unsigned a, unsigned b) { return (unsigned)(((uint64_t)a * b) >> 32); }
using std::fabs; using std::sqrt; using std::pow; using std::sin; using std::cos; using std::acos;
using std::atan; using std::atan2; using std::floor; using std::log; using std::fmin; using std::fmax;
#else
#include <cuda_runtime.h>
#include <string.h>
#define HD __host__ __device__ __forceinline__
#define DEV __device__ __forceinline__
// Large routines with many call sites (BVH traversal, shading) are real calls:
// inlining every copy makes kernels of several hundred KB of code, which
// starves the instruction cache.
#define DEV_NOINLINE static __device__ __noinline__
#define DR_RESTRICT __restrict__
// small lookup tables live in constant memory, not on each thread's stack
#define DR_TABLE static __constant__ const
template <typename T> DEV T dr_ldg(const T *p) { return __ldg(p); }
// fire-and-forget reduction (RED.ADD.F32); the result is not needed
DEV void dr_atomic_add(float *p, float v) { atomicAdd(p, v); }
HD unsigned dr_umulhi(unsigned a, unsigned b) {
#ifdef __CUDA_ARCH__
    return __umulhi(a, b);
#else
    return (unsigned)(((unsigned long long)a * b) >> 32);
#endif
}
#endif

// reproducible sin, cos, atan, atan2, acos, exp, log and pow (same bits on
// the GPU and in the host builds of this code)
#include "dr_math.h"

// bit casts usable from __host__ __device__ code
HD float dr_i2f(int i) {
#ifdef __CUDA_ARCH__
    return __int_as_float(i);
#else
    float f;
    memcpy(&f, &i, 4);
    return f;
#endif
}
HD int dr_f2i(float f) {
#ifdef __CUDA_ARCH__
    return __float_as_int(f);
#else
    int i;
    memcpy(&i, &f, 4);
    return i;
#endif
}

#define DR_PI 3.14159265358979323846f

// ---------------------------------------------------------------------------
// float3 algebra
// ---------------------------------------------------------------------------
HD float3 f3(float x, float y, float z) { float3 r; r.x = x; r.y = y; r.z = z; return r; }
HD float3 f3(float s) { return f3(s, s, s); }
HD float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
HD float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
HD float3 operator-(float3 a) { return f3(-a.x, -a.y, -a.z); }
HD float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
HD float3 operator*(float s, float3 a) { return f3(s * a.x, s * a.y, s * a.z); }
HD float3 operator*(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
HD float3 operator/(float3 a, float s) { float inv = 1.f / s; return a * inv; }  // reciprocal, as vector.h:373-378
HD float3 &operator+=(float3 &a, float3 b) { a = a + b; return a; }
HD float3 &operator-=(float3 &a, float3 b) { a = a - b; return a; }
HD float3 &operator*=(float3 &a, float s) { a = a * s; return a; }
HD float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
HD float3 cross(float3 a, float3 b) {
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
HD float sq(float x) { return x * x; }
HD float length_sq(float3 a) { return sq(a.x) + sq(a.y) + sq(a.z); }
HD float length(float3 a) { return sqrtf(length_sq(a)); }
HD float3 normalize(float3 a) { return a / length(a); }
HD float sum(float3 a) { return a.x + a.y + a.z; }
HD float abs_sum(float3 a) { return fabsf(a.x) + fabsf(a.y) + fabsf(a.z); }
HD float max3(float3 a) { return fmaxf(fmaxf(a.x, a.y), a.z); }
HD bool is_zero(float3 a) { return a.x == 0.f && a.y == 0.f && a.z == 0.f; }
HD float luminance(float3 a) { return 0.212671f * a.x + 0.715160f * a.y + 0.072169f * a.z; }
HD float comp(float3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
HD void comp_set(float3 &a, int i, float v) { if (i == 0) a.x = v; else if (i == 1) a.y = v; else a.z = v; }

// Adjoint helpers: given the output adjoint, return (or accumulate) input adjoints.
// d_normalize (vector.h:453-464)
HD float3 d_normalize(float3 v, float3 d_out) {
    float l = length(v);
    float d_inv_l = dot(d_out, v);
    float d_l = -d_inv_l / (l * l);
    return (d_out + d_l * v) / l;
}
// d_length: d|v|/dv = v/|v|
HD float3 d_length(float3 v, float d_out) { return v * (d_out / length(v)); }
HD void d_cross(float3 a, float3 b, float3 d, float3 &da, float3 &db) {
    // c = a x b;  dL/da = b x d, dL/db = d x a
    da += cross(b, d);
    db += cross(d, a);
}

// ---------------------------------------------------------------------------
// Frames (vector.h:485-517): rows t, b, n
// ---------------------------------------------------------------------------
struct Frame { float3 t, b, n; };

HD Frame make_frame(float3 n) {
    Frame f;
    if (n.z < -1.f + 1e-6f) {
        f.t = f3(0.f, -1.f, 0.f);
        f.b = f3(-1.f, 0.f, 0.f);
        f.n = n;
        return f;
    }
    float a = 1.f / (1.f + n.z);
    float b = -n.x * n.y * a;
    f.t = f3(1.f - sq(n.x) * a, b, -n.x);
    f.b = f3(b, 1.f - sq(n.y) * a, -n.y);
    f.n = n;
    return f;
}
// adjoint of make_frame: accumulate dn from dt, db, dn_direct
HD float3 d_make_frame(float3 n, const Frame &df) {
    float3 dn = df.n;
    if (n.z < -1.f + 1e-6f) return dn;
    float a = 1.f / (1.f + n.z);
    // t = (1 - nx^2 a, -nx ny a, -nx); b = (-nx ny a, 1 - ny^2 a, -ny)
    float dtx = df.t.x, dty = df.t.y, dtz = df.t.z;
    float dbx = df.b.x, dby = df.b.y, dbz = df.b.z;
    float dnx = dn.x, dny = dn.y, dnz = dn.z;
    float da = 0.f;
    // t.x = 1 - nx^2 a
    dnx += dtx * (-2.f * n.x * a);
    da += dtx * (-sq(n.x));
    // t.y = b.x = -nx ny a
    float dbb = dty + dbx;
    dnx += dbb * (-n.y * a);
    dny += dbb * (-n.x * a);
    da += dbb * (-n.x * n.y);
    // t.z = -nx
    dnx -= dtz;
    // b.y = 1 - ny^2 a
    dny += dby * (-2.f * n.y * a);
    da += dby * (-sq(n.y));
    // b.z = -ny
    dny -= dbz;
    // a = 1 / (1 + nz)
    dnz += da * (-a * a);
    return f3(dnx, dny, dnz);
}
HD float3 to_local(const Frame &f, float3 v) { return f3(dot(v, f.t), dot(v, f.b), dot(v, f.n)); }
HD float3 to_world(const Frame &f, float3 v) { return f.t * v.x + f.b * v.y + f.n * v.z; }
HD Frame frame_neg(const Frame &f) { Frame r; r.t = -f.t; r.b = -f.b; r.n = -f.n; return r; }
HD Frame frame_zero() { Frame r; r.t = f3(0.f); r.b = f3(0.f); r.n = f3(0.f); return r; }
HD void frame_add(Frame &a, const Frame &b) { a.t += b.t; a.b += b.b; a.n += b.n; }
// adjoint of to_local(f, v) with output adjoint d: df += outer, dv += ...
HD void d_to_local(const Frame &f, float3 v, float3 d, Frame &df, float3 &dv) {
    df.t += v * d.x;
    df.b += v * d.y;
    df.n += v * d.z;
    dv += f.t * d.x + f.b * d.y + f.n * d.z;
}

// ---------------------------------------------------------------------------
// 3x3 and 4x4 matrices (row-major)
// ---------------------------------------------------------------------------
struct M3 { float m[9]; };
HD float3 mul(const M3 &a, float3 v) {
    return f3(a.m[0] * v.x + a.m[1] * v.y + a.m[2] * v.z, a.m[3] * v.x + a.m[4] * v.y + a.m[5] * v.z,
              a.m[6] * v.x + a.m[7] * v.y + a.m[8] * v.z);
}
HD M3 mul(const M3 &a, const M3 &b) {
    M3 r;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            float s = 0.f;
            for (int k = 0; k < 3; k++) s += a.m[3 * i + k] * b.m[3 * k + j];
            r.m[3 * i + j] = s;
        }
    return r;
}
HD M3 m3_rows(float3 a, float3 b, float3 c) {
    M3 r;
    r.m[0] = a.x; r.m[1] = a.y; r.m[2] = a.z;
    r.m[3] = b.x; r.m[4] = b.y; r.m[5] = b.z;
    r.m[6] = c.x; r.m[7] = c.y; r.m[8] = c.z;
    return r;
}
// 3x3 inverse by cofactors (the same expression order as vector.h:659-678)
HD M3 inverse(const M3 &a) {
    const float *m = a.m;
#define A(i, j) m[3 * (i) + (j)]
    float det = A(0, 0) * (A(1, 1) * A(2, 2) - A(2, 1) * A(1, 2)) - A(0, 1) * (A(1, 0) * A(2, 2) - A(1, 2) * A(2, 0)) +
                A(0, 2) * (A(1, 0) * A(2, 1) - A(1, 1) * A(2, 0));
    float id = 1 / det;
    M3 r;
    r.m[0] = (A(1, 1) * A(2, 2) - A(2, 1) * A(1, 2)) * id;
    r.m[1] = (A(0, 2) * A(2, 1) - A(0, 1) * A(2, 2)) * id;
    r.m[2] = (A(0, 1) * A(1, 2) - A(0, 2) * A(1, 1)) * id;
    r.m[3] = (A(1, 2) * A(2, 0) - A(1, 0) * A(2, 2)) * id;
    r.m[4] = (A(0, 0) * A(2, 2) - A(0, 2) * A(2, 0)) * id;
    r.m[5] = (A(1, 0) * A(0, 2) - A(0, 0) * A(1, 2)) * id;
    r.m[6] = (A(1, 0) * A(2, 1) - A(2, 0) * A(1, 1)) * id;
    r.m[7] = (A(2, 0) * A(0, 1) - A(0, 0) * A(2, 1)) * id;
    r.m[8] = (A(0, 0) * A(1, 1) - A(1, 0) * A(0, 1)) * id;
#undef A
    return r;
}

struct M4 { float m[16]; };
HD float3 xfm_point(const M4 &M, float3 p) {
    float t0 = M.m[0] * p.x + M.m[1] * p.y + M.m[2] * p.z + M.m[3];
    float t1 = M.m[4] * p.x + M.m[5] * p.y + M.m[6] * p.z + M.m[7];
    float t2 = M.m[8] * p.x + M.m[9] * p.y + M.m[10] * p.z + M.m[11];
    float t3 = M.m[12] * p.x + M.m[13] * p.y + M.m[14] * p.z + M.m[15];
    float inv_w = 1.f / t3;
    return f3(t0, t1, t2) * inv_w;
}
HD float3 xfm_vector(const M4 &M, float3 v) {
    return f3(M.m[0] * v.x + M.m[1] * v.y + M.m[2] * v.z, M.m[4] * v.x + M.m[5] * v.y + M.m[6] * v.z,
              M.m[8] * v.x + M.m[9] * v.y + M.m[10] * v.z);
}
// d_xfm_point (transform.h:21-59): accumulates d_M, returns d_p
HD float3 d_xfm_point(const M4 &M, float3 p, float3 d_out, float *dM) {
    float t[4];
    for (int r = 0; r < 4; r++) t[r] = M.m[4 * r] * p.x + M.m[4 * r + 1] * p.y + M.m[4 * r + 2] * p.z + M.m[4 * r + 3];
    float inv_w = 1.f / t[3];
    float dt[4];
    dt[0] = d_out.x * inv_w;
    dt[1] = d_out.y * inv_w;
    dt[2] = d_out.z * inv_w;
    float dinv = d_out.x * t[0] + d_out.y * t[1] + d_out.z * t[2];
    dt[3] = -dinv * inv_w * inv_w;
    float3 dp = f3(0.f);
    for (int r = 0; r < 4; r++) {
        if (dM) {
            dM[4 * r + 0] += dt[r] * p.x;
            dM[4 * r + 1] += dt[r] * p.y;
            dM[4 * r + 2] += dt[r] * p.z;
            dM[4 * r + 3] += dt[r];
        }
        dp += f3(M.m[4 * r], M.m[4 * r + 1], M.m[4 * r + 2]) * dt[r];
    }
    return dp;
}
HD void d_xfm_vector(const M4 &M, float3 v, float3 d_out, float *dM, float3 &dv) {
    for (int r = 0; r < 3; r++) {
        float d = comp(d_out, r);
        if (dM) {
            dM[4 * r + 0] += d * v.x;
            dM[4 * r + 1] += d * v.y;
            dM[4 * r + 2] += d * v.z;
        }
        dv += f3(M.m[4 * r], M.m[4 * r + 1], M.m[4 * r + 2]) * d;
    }
}

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon et al., "Parallel random numbers: as easy as 1, 2, 3",
// SC'11).  Counter = (id_lo, id_hi, sub, block), key = (seed_lo, kind ^ seed_hi).
// A stream yields 4 uniform floats per block, u = (x >> 8) * 2^-24.
// ---------------------------------------------------------------------------
HD void philox4x32_10(uint32_t &c0, uint32_t &c1, uint32_t &c2, uint32_t &c3, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        if (r > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        uint32_t lo0 = 0xD2511F53u * c0, hi0 = dr_umulhi(0xD2511F53u, c0);
        uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = dr_umulhi(0xCD9E8D57u, c2);
        uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
    }
}

enum DrStreamKind : uint32_t {
    kStreamPixel = 0,
    kStreamEdgePoint = 1,
    kStreamEdgeItem = 2,
    kStreamPrimaryEdge = 3,
    kStreamEdgeNode = 4
};

struct Rng {
    uint32_t k0, k1, id_lo, id_hi, sub, idx;
    uint32_t buf[4];
    HD void init(uint64_t seed, uint32_t kind, uint64_t id, uint32_t sub_) {
        k0 = (uint32_t)seed;
        k1 = kind ^ (uint32_t)(seed >> 32);
        id_lo = (uint32_t)id;
        id_hi = (uint32_t)(id >> 32);
        sub = sub_;
        idx = 0;
    }
    HD float next() {
        uint32_t lane = idx & 3u;
        if (lane == 0) {
            uint32_t c0 = id_lo, c1 = id_hi, c2 = sub, c3 = idx >> 2;
            philox4x32_10(c0, c1, c2, c3, k0, k1);
            buf[0] = c0;
            buf[1] = c1;
            buf[2] = c2;
            buf[3] = c3;
        }
        idx++;
        uint32_t x = lane == 0 ? buf[0] : (lane == 1 ? buf[1] : (lane == 2 ? buf[2] : buf[3]));
        return (float)(x >> 8) * (1.f / 16777216.f);
    }
};

// The draws of an edge-tree traversal are keyed by node instead of by stream
// position, so that the set of sampled edges does not depend on the order in
// which the nodes are visited (a project convention, mirrored by the oracle):
// stream kStreamEdgeNode of the point's sample id, sub = bounce << 28 |
// mode << 27 | node (mode 0 cone, 1 all).
struct NodeRng {
    uint64_t seed, sid;
    uint32_t bounce;
    HD float draw(int mode, int node) const {
        Rng r;
        r.init(seed, kStreamEdgeNode, sid, (bounce << 28) | ((uint32_t)mode << 27) | (uint32_t)node);
        return r.next();
    }
};
// Node id of the learned proposal's once-per-traversal mixture draw.
#define DR_NODE_MIX_DRAW 0x7FFFFFF

// Sample records.  Field-fill order reproduces the reference compiled by GCC,
// which evaluates function arguments right to left (light.h:46-51,
// material.h:246-250): the first of two draws lands in the second uv slot.
struct LightSample { float u0, u1, sel, tri_sel; };
struct BSDFSample { float u0, u1, w; };
struct SecondarySample { LightSample light; BSDFSample bsdf; float rr; };
struct EdgeSample { float bsdf_component, u; };

HD LightSample draw_light(Rng &r) {
    LightSample l;
    l.u1 = r.next();
    l.u0 = r.next();
    l.sel = r.next();
    l.tri_sel = r.next();
    return l;
}
HD BSDFSample draw_bsdf(Rng &r) {
    BSDFSample b;
    b.u1 = r.next();
    b.u0 = r.next();
    b.w = r.next();
    return b;
}
HD SecondarySample draw_secondary(Rng &r) {
    SecondarySample s;
    s.light = draw_light(r);
    s.bsdf = draw_bsdf(r);
    s.rr = r.next();
    return s;
}
HD EdgeSample draw_edge(Rng &r) {
    EdgeSample e;
    e.bsdf_component = r.next();
    e.u = r.next();
    return e;
}
