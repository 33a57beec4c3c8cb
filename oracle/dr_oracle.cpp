// Test infrastructure only: the ORACLE for the parity tests.  Never linked
// into, imported by or called from the product.
//
// A CPU restatement of the reference renderer's forward + backward render
// (BachiLi/delta_ray), written for this project.  Every function cites the
// reference file:line whose behaviour it restates.  Differences from the
// reference are in mechanism only:
//   * reverse-mode AD is this file's own tape (nodes with <= 2 parents)
//     instead of autodiff.h's edge list, with the same partial derivatives;
//   * ray casting uses the project's CPU BVH (oracle/ref_shim), which is also
//     what the compiled reference uses here in place of Embree;
//   * the random numbers come either from the reference's own scheme
//     (rng_mode 0: one std::mt19937 per 8x8 tile and per edge thread, seeded
//     exactly as delta_ray.cpp:1183-1191,1473) or from the Philox streams that
//     the GPU product uses (rng_mode 1), consumed in the same order.
//
// C entry point: dro_render() at the bottom; descriptors are the product's
// public structs (include/delta_ray_b200.h), gradients use its flat layout.

#include "../include/delta_ray_b200.h"
#include "ref_shim/embree3/rtcore.h"

#include <algorithm>
#include <array>
#include <cassert>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <random>
#include <tuple>
#include <vector>

#include <atomic>
#include <thread>

#include "../delta_ray_b200/csrc/dr_math.h"
#include "../delta_ray_b200/csrc/dr_edge_rules.h"

// The transcendental functions the restatement evaluates.  In the reference's
// RNG mode they are the host libm's, as in the compiled reference.  In the
// Philox mode they are the product's reproducible ones (dr_math.h), whose bits
// are the same on the GPU and here, so that a sample takes the same branches
// on both sides.
static bool g_repro_math = false;
// The edge trees' split rule.  The reference's: std::nth_element on the split
// coordinate, float normal sums in range order, std::min / std::max boxes.
// In the Philox mode, trees of more than DR_TREE_EXACT_MAX_EDGES edges follow
// the product's rule (dr_edge_rules.h), which its GPU build reproduces: a
// stable sort on the split coordinate's total-order key, exact fixed-point
// normal sums, total-order boxes.  The two rules give the same trees except
// where edges share a median coordinate (and in the last bits of cone axes);
// either is unbiased.  g_product_tree is set while such a tree is built.
static bool g_product_rule = false;
static bool g_product_tree = false;
inline float m_pow(float x, float e) { return g_repro_math ? dr_powf(x, e) : std::pow(x, e); }
inline float m_log(float x) { return g_repro_math ? dr_logf(x) : std::log(x); }
inline float m_sin(float x) { return g_repro_math ? dr_sinf(x) : std::sin(x); }
inline float m_cos(float x) { return g_repro_math ? dr_cosf(x) : std::cos(x); }
inline float m_acos(float x) { return g_repro_math ? dr_acosf(x) : std::acos(x); }
inline float m_atan(float x) { return g_repro_math ? dr_atanf(x) : std::atan(x); }
inline float m_atan2(float y, float x) { return g_repro_math ? dr_atan2f(y, x) : std::atan2(y, x); }

namespace oracle {

static const float kPi = 3.14159265358979323846f;

// ===================================================================
// Reverse-mode tape (restates autodiff.h:28-358: one node per operation,
// partial derivatives recorded at construction, one backward sweep).
// ===================================================================
struct Tape {
    struct Node { int p0, p1; float w0, w1; };
    std::vector<Node> nodes;
    std::vector<float> adj;
    void clear() { nodes.clear(); }
    int add(int p0, float w0, int p1, float w1) {
        nodes.push_back(Node{p0, p1, w0, w1});
        return (int)nodes.size() - 1;
    }
    void zero() { adj.assign(nodes.size(), 0.f); }
    void sweep() {
        for (int i = (int)nodes.size() - 1; i >= 0; i--) {
            float a = adj[i];
            if (a == 0.f) continue;
            const Node &n = nodes[i];
            if (n.p0 >= 0) adj[n.p0] += n.w0 * a;
            if (n.p1 >= 0) adj[n.p1] += n.w1 * a;
        }
    }
};
thread_local Tape *g_tape = nullptr;

struct AD {
    float v;
    int id;
    AD() : v(0.f), id(-1) {}
    AD(float x) : v(x), id(-1) {}  // constants carry no tape node
    AD(float x, int i) : v(x), id(i) {}
};

inline AD mk(float v, int p0, float w0, int p1 = -1, float w1 = 0.f) {
    if (p0 < 0 && p1 < 0) return AD(v);
    return AD(v, g_tape->add(p0, w0, p1, w1));
}
inline AD new_leaf(float v) { return AD(v, g_tape->add(-1, 0.f, -1, 0.f)); }

inline AD operator+(const AD &a, const AD &b) { return mk(a.v + b.v, a.id, 1.f, b.id, 1.f); }
inline AD operator+(const AD &a, float b) { return mk(a.v + b, a.id, 1.f); }
inline AD operator+(float a, const AD &b) { return mk(a + b.v, b.id, 1.f); }
inline AD operator-(const AD &a, const AD &b) { return mk(a.v - b.v, a.id, 1.f, b.id, -1.f); }
inline AD operator-(const AD &a, float b) { return mk(a.v - b, a.id, 1.f); }
inline AD operator-(float a, const AD &b) { return mk(a - b.v, b.id, -1.f); }
inline AD operator-(const AD &a) { return mk(-a.v, a.id, -1.f); }
inline AD operator*(const AD &a, const AD &b) { return mk(a.v * b.v, a.id, b.v, b.id, a.v); }
inline AD operator*(const AD &a, float b) { return mk(a.v * b, a.id, b); }
inline AD operator*(float a, const AD &b) { return mk(a * b.v, b.id, a); }
inline AD operator/(const AD &a, const AD &b) {
    float ib = 1.f / b.v;
    return mk(a.v * ib, a.id, ib, b.id, -a.v * ib * ib);
}
inline AD operator/(const AD &a, float b) { return a * (1.f / b); }
inline AD operator/(float a, const AD &b) {
    float ib = 1.f / b.v;
    return mk(a * ib, b.id, -a * ib * ib);
}
inline AD &operator+=(AD &a, const AD &b) { return a = a + b; }
inline AD &operator-=(AD &a, const AD &b) { return a = a - b; }
inline AD &operator*=(AD &a, const AD &b) { return a = a * b; }
inline AD &operator/=(AD &a, const AD &b) { return a = a / b; }
inline bool operator<(const AD &a, const AD &b) { return a.v < b.v; }
inline bool operator<=(const AD &a, const AD &b) { return a.v <= b.v; }
inline bool operator>(const AD &a, const AD &b) { return a.v > b.v; }
inline bool operator>=(const AD &a, const AD &b) { return a.v >= b.v; }
inline bool operator==(const AD &a, const AD &b) { return a.v == b.v; }

inline AD sqrt(const AD &x) {
    float s = std::sqrt(x.v);
    return mk(s, x.id, 0.5f / s);
}
inline AD pow(const AD &x, float e) { return mk(m_pow(x.v, e), x.id, e * m_pow(x.v, e - 1.f)); }
inline AD pow(const AD &x, const AD &e) {
    float p = m_pow(x.v, e.v);
    return mk(p, x.id, e.v * m_pow(x.v, e.v - 1.f), e.id, p * m_log(std::max(x.v, 1e-6f)));
}
inline AD pow(float x, const AD &e) { return pow(AD(x), e); }
inline AD sin(const AD &x) { return mk(m_sin(x.v), x.id, m_cos(x.v)); }
inline AD cos(const AD &x) { return mk(m_cos(x.v), x.id, -m_sin(x.v)); }
inline AD acos(const AD &x) { return mk(m_acos(x.v), x.id, -std::sqrt(1.f / (1.f - x.v * x.v))); }
inline AD atan2(const AD &y, const AD &x) {
    float t = x.v * x.v + y.v * y.v;
    return mk(m_atan2(y.v, x.v), y.id, x.v / t, x.id, -y.v / t);
}
inline AD fabs(const AD &x) { return x.v >= 0.f ? x : -x; }
// max/min keep the reference's tie conventions (autodiff.h:301-324)
inline AD max(const AD &x, const AD &y) { return x.v > y.v ? x : y; }
inline AD max(const AD &x, float y) { return x.v >= y ? x : AD(y); }
inline AD max(float x, const AD &y) { return x > y.v ? AD(x) : y; }
inline AD min(const AD &x, const AD &y) { return x.v < y.v ? x : y; }
inline AD min(const AD &x, float y) { return x.v <= y ? x : AD(y); }
inline AD min(float x, const AD &y) { return x < y.v ? AD(x) : y; }
inline float max(float x, float y) { return x > y ? x : y; }
inline float min(float x, float y) { return x < y ? x : y; }
inline float fabs(float x) { return std::fabs(x); }
inline float sqrt(float x) { return std::sqrt(x); }
inline float pow(float x, float e) { return m_pow(x, e); }
inline float sin(float x) { return m_sin(x); }
inline float cos(float x) { return m_cos(x); }
inline float acos(float x) { return m_acos(x); }
inline float atan2(float y, float x) { return m_atan2(y, x); }

inline float val(float x) { return x; }
inline float val(const AD &x) { return x.v; }

// A differentiable input: a fresh tape leaf for AD, the value for float.
template <typename T> struct Param;
template <> struct Param<float> { static float make(float x, int *id) { *id = -1; return x; } };
template <> struct Param<AD> {
    static AD make(float x, int *id) {
        AD a = new_leaf(x);
        *id = a.id;
        return a;
    }
};

// ===================================================================
// Small vector algebra (vector.h)
// ===================================================================
template <typename T> struct V2 {
    T x, y;
    T &operator[](int i) { return i == 0 ? x : y; }
    const T &operator[](int i) const { return i == 0 ? x : y; }
};
template <typename T> struct V3 {
    T x, y, z;
    T &operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    const T &operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
using V3f = V3<float>;
using V2f = V2<float>;

template <typename T> inline V3<T> v3(T x, T y, T z) { return V3<T>{x, y, z}; }
template <typename A, typename B> inline auto operator+(const V3<A> &a, const V3<B> &b) {
    return v3(a.x + b.x, a.y + b.y, a.z + b.z);
}
template <typename A, typename B> inline auto operator-(const V3<A> &a, const V3<B> &b) {
    return v3(a.x - b.x, a.y - b.y, a.z - b.z);
}
template <typename A> inline V3<A> operator-(const V3<A> &a) { return V3<A>{-a.x, -a.y, -a.z}; }
template <typename A, typename B> inline auto operator*(const V3<A> &a, const B &s) {
    return v3(a.x * s, a.y * s, a.z * s);
}
template <typename A, typename B> inline auto operator*(const B &s, const V3<A> &a) {
    return v3(s * a.x, s * a.y, s * a.z);
}
template <typename A, typename B> inline auto mul(const V3<A> &a, const V3<B> &b) {
    return v3(a.x * b.x, a.y * b.y, a.z * b.z);
}
template <typename A, typename B> inline auto div(const V3<A> &a, const V3<B> &b) {
    return v3(a.x / b.x, a.y / b.y, a.z / b.z);
}
template <typename A, typename B> inline auto operator/(const V3<A> &a, const B &s) {
    auto inv = 1.f / s;  // vector.h:373-378 multiplies by the reciprocal
    return a * inv;
}
template <typename A, typename B> inline auto dot(const V3<A> &a, const V3<B> &b) {
    return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <typename A, typename B> inline auto cross(const V3<A> &a, const V3<B> &b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <typename T> inline T sq(const T &x) { return x * x; }
template <typename T> inline T length_sq(const V3<T> &a) { return sq(a.x) + sq(a.y) + sq(a.z); }
template <typename T> inline T length(const V3<T> &a) { return sqrt(length_sq(a)); }
template <typename T> inline V3<T> normalize(const V3<T> &a) { return a / length(a); }
template <typename T> inline T sum(const V3<T> &a) { return a.x + a.y + a.z; }
template <typename T> inline T luminance(const V3<T> &a) {
    return 0.212671f * a.x + 0.715160f * a.y + 0.072169f * a.z;
}
inline float abs_sum(const V3f &a) { return std::fabs(a.x) + std::fabs(a.y) + std::fabs(a.z); }
inline bool is_zero(const V3f &a) { return a.x == 0.f && a.y == 0.f && a.z == 0.f; }
inline V3f fv(const V3<AD> &a) { return V3f{a.x.v, a.y.v, a.z.v}; }
inline V3f fv(const V3f &a) { return a; }
template <typename T> inline V3<T> tv(const V3f &a) { return V3<T>{T(a.x), T(a.y), T(a.z)}; }
inline V3f vmax3(float s) { return V3f{s, s, s}; }
inline float vmax(const V3f &a) { return std::max(std::max(a.x, a.y), a.z); }

template <typename T> using Frame = std::array<V3<T>, 3>;

// make_frame (vector.h:485-501)
template <typename T> inline Frame<T> make_frame(const V3<T> &n) {
    if (n.z < -1.f + 1e-6f) {
        return Frame<T>{V3<T>{T(0.f), T(-1.f), T(0.f)}, V3<T>{T(-1.f), T(0.f), T(0.f)}, n};
    }
    T a = 1.f / (1.f + n.z);
    T b = -n.x * n.y * a;
    return Frame<T>{V3<T>{1.f - sq(n.x) * a, b, -n.x}, V3<T>{b, 1.f - sq(n.y) * a, -n.y}, n};
}
template <typename T, typename U> inline auto to_local(const Frame<T> &f, const V3<U> &v) {
    return v3(dot(v, f[0]), dot(v, f[1]), dot(v, f[2]));
}
template <typename T, typename U> inline auto to_world(const Frame<T> &f, const V3<U> &v) {
    return f[0] * v.x + f[1] * v.y + f[2] * v.z;
}

struct M3 {
    float m[3][3];
    float &operator()(int i, int j) { return m[i][j]; }
    float operator()(int i, int j) const { return m[i][j]; }
};
inline M3 m3_rows(const V3f &a, const V3f &b, const V3f &c) {
    M3 r;
    for (int j = 0; j < 3; j++) { r.m[0][j] = a[j]; r.m[1][j] = b[j]; r.m[2][j] = c[j]; }
    return r;
}
inline M3 operator*(const M3 &a, const M3 &b) {
    M3 r;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            r.m[i][j] = 0.f;
            for (int k = 0; k < 3; k++) r.m[i][j] += a.m[i][k] * b.m[k][j];
        }
    return r;
}
inline V3f operator*(const M3 &a, const V3f &v) {
    V3f r;
    for (int i = 0; i < 3; i++) {
        r[i] = 0.f;
        for (int j = 0; j < 3; j++) r[i] += a.m[i][j] * v[j];
    }
    return r;
}
// inverse (vector.h:659-678)
inline M3 inverse(const M3 &m) {
    float det = m(0, 0) * (m(1, 1) * m(2, 2) - m(2, 1) * m(1, 2)) -
                m(0, 1) * (m(1, 0) * m(2, 2) - m(1, 2) * m(2, 0)) +
                m(0, 2) * (m(1, 0) * m(2, 1) - m(1, 1) * m(2, 0));
    float id = 1 / det;
    M3 r;
    r(0, 0) = (m(1, 1) * m(2, 2) - m(2, 1) * m(1, 2)) * id;
    r(0, 1) = (m(0, 2) * m(2, 1) - m(0, 1) * m(2, 2)) * id;
    r(0, 2) = (m(0, 1) * m(1, 2) - m(0, 2) * m(1, 1)) * id;
    r(1, 0) = (m(1, 2) * m(2, 0) - m(1, 0) * m(2, 2)) * id;
    r(1, 1) = (m(0, 0) * m(2, 2) - m(0, 2) * m(2, 0)) * id;
    r(1, 2) = (m(1, 0) * m(0, 2) - m(0, 0) * m(1, 2)) * id;
    r(2, 0) = (m(1, 0) * m(2, 1) - m(2, 0) * m(1, 1)) * id;
    r(2, 1) = (m(2, 0) * m(0, 1) - m(0, 0) * m(2, 1)) * id;
    r(2, 2) = (m(0, 0) * m(1, 1) - m(1, 0) * m(0, 1)) * id;
    return r;
}
// d(p)/d(dir) of a ray hitting the plane through p with normal n (vector.h:690-716)
inline M3 intersect_jacobian(const V3f &dir, const V3f &p, const V3f &n) {
    M3 m;
    float d = -dot(p, n);
    float dn = dot(dir, n);
    if (std::fabs(dn) < 1e-10f) {
        std::memset(&m, 0, sizeof(m));
        return m;
    }
    float inv2 = 1.f / (dn * dn);
    float t = -d / dn;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) m(i, j) = (i == j ? t : 0.f) + dir[i] * d * n[j] * inv2;
    return m;
}
// d normalize(x) / dx (vector.h:718-733)
inline M3 normalize_jacobian(const V3f &x) {
    float d2 = length_sq(x);
    float d = std::sqrt(d2);
    float inv = 1.f / (d * d2);
    M3 m;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) m(i, j) = ((i == j ? d2 : 0.f) - x[i] * x[j]) * inv;
    return m;
}

// 4x4 row-major matrices
template <typename T> struct M4 { T m[16]; };
template <typename T> inline V3<T> xfm_point(const M4<T> &M, const V3<T> &p) {
    T t0 = M.m[0] * p.x + M.m[1] * p.y + M.m[2] * p.z + M.m[3];
    T t1 = M.m[4] * p.x + M.m[5] * p.y + M.m[6] * p.z + M.m[7];
    T t2 = M.m[8] * p.x + M.m[9] * p.y + M.m[10] * p.z + M.m[11];
    T t3 = M.m[12] * p.x + M.m[13] * p.y + M.m[14] * p.z + M.m[15];
    T inv_w = 1.f / t3;
    return V3<T>{t0, t1, t2} * inv_w;
}
template <typename T> inline V3<T> xfm_vector(const M4<T> &M, const V3<T> &v) {
    return V3<T>{M.m[0] * v.x + M.m[1] * v.y + M.m[2] * v.z, M.m[4] * v.x + M.m[5] * v.y + M.m[6] * v.z,
                 M.m[8] * v.x + M.m[9] * v.y + M.m[10] * v.z};
}
// d_xfm_point (transform.h:21-59): accumulate into d_M
inline void d_xfm_point(const M4<float> &M, const V3f &p, const V3f &d_out, float *dM) {
    float t[4];
    for (int r = 0; r < 4; r++) t[r] = M.m[4 * r] * p.x + M.m[4 * r + 1] * p.y + M.m[4 * r + 2] * p.z + M.m[4 * r + 3];
    float inv_w = 1.f / t[3];
    float dt[4];
    dt[0] = d_out.x * inv_w;
    dt[1] = d_out.y * inv_w;
    dt[2] = d_out.z * inv_w;
    float dinv = d_out.x * t[0] + d_out.y * t[1] + d_out.z * t[2];
    dt[3] = -dinv * inv_w * inv_w;
    for (int r = 0; r < 4; r++) {
        dM[4 * r + 0] += dt[r] * p.x;
        dM[4 * r + 1] += dt[r] * p.y;
        dM[4 * r + 2] += dt[r] * p.z;
        dM[4 * r + 3] += dt[r];
    }
}

// ===================================================================
// RNG back-ends
// ===================================================================
struct Sampler {
    virtual float next() = 0;
    // the draw of an edge-tree traversal's stochastic choice at node nid in
    // mode (0 cone, 1 all): the next draw in the reference's scheme
    virtual float node(int mode, int nid) {
        (void)mode;
        (void)nid;
        return next();
    }
    virtual ~Sampler() {}
};

// The reference's draws: std::uniform_real_distribution<float>(0, 1) over a
// std::mt19937 (delta_ray.cpp:1170,1183-1191).
struct MtSampler : Sampler {
    std::mt19937 *g;
    std::uniform_real_distribution<float> d{0.f, 1.f};
    explicit MtSampler(std::mt19937 *g_) : g(g_) {}
    float next() override { return d(*g); }
};

// Philox4x32-10 (Salmon et al., SC'11), counter = (id_lo, id_hi, sub, block),
// key = (seed_lo, kind).  Identical arithmetic in the GPU product.
inline void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; r++) {
        if (r > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
    }
}

enum StreamKind : uint32_t { kPixel = 0, kEdgePoint = 1, kEdgeItem = 2, kPrimaryEdge = 3, kEdgeNode = 4 };

struct PhiloxSampler : Sampler {
    uint64_t seed;
    uint32_t k0, k1, id_lo, id_hi, sub, idx = 0;
    uint32_t buf[4];
    PhiloxSampler(uint64_t seed_, uint32_t kind, uint64_t id, uint32_t sub_)
        : seed(seed_), k0((uint32_t)seed_), k1(kind ^ (uint32_t)(seed_ >> 32)), id_lo((uint32_t)id),
          id_hi((uint32_t)(id >> 32)), sub(sub_) {}
    // The product's traversal draws are keyed by node, not by stream position
    // (project convention, so that a traversal's result does not depend on
    // the order of its visits): stream kEdgeNode of the same sample id,
    // sub = bounce << 28 | mode << 27 | node (this sampler's sub is the bounce).
    float node(int mode, int nid) override {
        PhiloxSampler d(seed, kEdgeNode, ((uint64_t)id_hi << 32) | id_lo,
                        (sub << 28) | ((uint32_t)mode << 27) | (uint32_t)nid);
        return d.next();
    }
    float next() override {
        uint32_t lane = idx & 3u;
        if (lane == 0) {
            buf[0] = id_lo;
            buf[1] = id_hi;
            buf[2] = sub;
            buf[3] = idx >> 2;
            philox4x32_10(buf, k0, k1);
        }
        idx++;
        return (float)(buf[lane] >> 8) * (1.f / 16777216.f);
    }
};

// ===================================================================
// Scene
// ===================================================================
struct Tex { const float *data = nullptr; int w = 0, h = 0, c = 1; };
struct Material {
    Tex diffuse, specular, roughness;
    float uv_d[2], uv_s[2], uv_r[2];
    bool two_sided;
    int model = 0;  // DR_MICROFACET_BLINN_PHONG or DR_MICROFACET_GGX
};
struct Shape {
    const float *v; int nv;
    const int *idx; int nt;
    const float *uv; const float *n;
    int mat; int light = -1;
    std::array<int, 3> ind(int t) const { return {idx[3 * t], idx[3 * t + 1], idx[3 * t + 2]}; }
    V3f vtx(int i) const { return V3f{v[3 * i], v[3 * i + 1], v[3 * i + 2]}; }
    V3f nrm(int i) const { return V3f{n[3 * i], n[3 * i + 1], n[3 * i + 2]}; }
    V3f face_normal(int t) const {  // shape.h:78-86
        auto d = ind(t);
        V3f a = vtx(d[0]), b = vtx(d[1]), c = vtx(d[2]);
        return normalize(cross(b - a, c - a));
    }
};
struct Light { int shape; float I[3]; };
struct Camera {
    M4<float> c2w, w2c, s2c, c2s;
    float fov, aspect, clip_near;
    bool fisheye;
};
struct Edge { int shape = -1, v0 = 0, v1 = 0, f0 = -1, f1 = -1; };

// pbrt's piecewise-constant 1-D distribution (distribution.h:7-61)
struct Dist1D {
    std::vector<float> func, cdf;
    float func_int = 0.f;
    int count = 0;
    Dist1D() {}
    Dist1D(const float *f, int n) {
        count = n;
        func.assign(f, f + n);
        cdf.assign(n + 1, 0.f);
        for (int i = 1; i <= n; i++) cdf[i] = cdf[i - 1] + func[i - 1] / n;
        func_int = cdf[n];
        for (int i = 1; i <= n; i++) cdf[i] = func_int == 0.f ? float(i) / float(n) : cdf[i] / func_int;
    }
    int sample_discrete(float u, float *pmf = nullptr) const {
        int off = int(std::upper_bound(cdf.begin(), cdf.end(), u) - cdf.begin()) - 1;
        off = off <= 0 ? 0 : (off >= count - 1 ? count - 1 : off);
        if (pmf) *pmf = func[off] / (func_int * count);
        return off;
    }
};

// box minima and maxima: std::min / std::max, or the total order of the
// product's tree rule (-0 below +0)
inline float box_min(float a, float b) { return g_product_tree ? (edge_ord_key(b) < edge_ord_key(a) ? b : a) : std::min(a, b); }
inline float box_max(float a, float b) { return g_product_tree ? (edge_ord_key(b) > edge_ord_key(a) ? b : a) : std::max(a, b); }
struct AABB {
    V3f lo{INFINITY, INFINITY, INFINITY}, hi{-INFINITY, -INFINITY, -INFINITY};
    void add(const V3f &p) {
        for (int a = 0; a < 3; a++) { lo[a] = box_min(lo[a], p[a]); hi[a] = box_max(hi[a], p[a]); }
    }
    void add(const AABB &b) {
        for (int a = 0; a < 3; a++) { lo[a] = box_min(lo[a], b.lo[a]); hi[a] = box_max(hi[a], b.hi[a]); }
    }
    V3f corner(int i) const { return V3f{(i & 1) ? hi.x : lo.x, (i & 2) ? hi.y : lo.y, (i & 4) ? hi.z : lo.z}; }
    V3f center() const { return 0.5f * (lo + hi); }
    bool inside(const V3f &p) const {
        return p.x >= lo.x && p.x <= hi.x && p.y >= lo.y && p.y <= hi.y && p.z >= lo.z && p.z <= hi.z;
    }
};

struct EdgeNode {
    AABB bounds;
    V3f cone_axis;
    float cone_angle;
    int offset;  // leaf: first edge; interior: second child
    int nprims;  // 0: interior
    float total_length;
};
struct EdgeTree { std::vector<EdgeNode> nodes; std::vector<Edge> edges; };

struct Scene {
    Camera cam;
    bool detached_pdf = false;
    bool edge_lobe_mis = false;  // DR_FLAG_EDGE_LOBE_MIS
    std::vector<Shape> shapes;
    std::vector<Material> mats;
    std::vector<Light> lights;
    std::vector<Dist1D> light_tri;
    Dist1D light_sel;
    std::vector<AABB> light_bounds;
    std::vector<float> light_area;
    float total_light_intensity = 0.f;
    std::vector<Edge> primary_edges;
    Dist1D primary_dist;
    EdgeTree sil_tree, nrm_tree;
    drshim::Scene bvh;
    const float *ltc = nullptr, *ltc_ggx = nullptr;
    // Sort key of each shape in the edge map.  The reference keys its edge map
    // by Shape* (scene.cpp:54-79), i.e. by heap address, so its edge order can
    // differ from the shape order; tests pass the order it used.
    std::vector<int> shape_rank;

    V3f ev0(const Edge &e) const { return shapes[e.shape].vtx(e.v0); }
    V3f ev1(const Edge &e) const { return shapes[e.shape].vtx(e.v1); }
};

// ===================================================================
// Ray casting (scene.cpp:147-202 through the shared CPU BVH)
// ===================================================================
struct Isect {
    int shape = -1, tri = -1;
    bool valid() const { return shape >= 0; }
};
template <typename T> struct Ray { V3<T> o, d; };
template <typename T> struct SPoint {
    V3<T> p, ng;
    Frame<T> f;
    V2<T> uv;
};
template <typename T> inline SPoint<float> fsp(const SPoint<T> &s) {
    SPoint<float> r;
    r.p = fv(s.p);
    r.ng = fv(s.ng);
    for (int i = 0; i < 3; i++) r.f[i] = fv(s.f[i]);
    r.uv = V2f{val(s.uv.x), val(s.uv.y)};
    return r;
}
template <typename T> inline SPoint<T> csp(const SPoint<float> &s) {
    SPoint<T> r;
    r.p = tv<T>(s.p);
    r.ng = tv<T>(s.ng);
    for (int i = 0; i < 3; i++) r.f[i] = tv<T>(s.f[i]);
    r.uv = V2<T>{T(s.uv.x), T(s.uv.y)};
    return r;
}

inline Isect nearest_hit(const Scene &sc, const Ray<float> &r) {
    float o[3] = {r.o.x, r.o.y, r.o.z}, d[3] = {r.d.x, r.d.y, r.d.z};
    float t;
    unsigned g, p;
    if (!drshim::trace(sc.bvh, o, d, 1e-3f, INFINITY, false, &t, &g, &p)) return Isect{};
    return Isect{(int)g, (int)p};
}
inline bool occluded(const Scene &sc, const Ray<float> &r, float max_t) {
    float o[3] = {r.o.x, r.o.y, r.o.z}, d[3] = {r.d.x, r.d.y, r.d.z};
    float t;
    unsigned g, p;
    return drshim::trace(sc.bvh, o, d, max_t * 1e-3f, max_t * (1.f - 1e-3f), true, &t, &g, &p);
}

// Gradient bookkeeping (IntersectParameter, MaterialParameter, LightParameter:
// intersect.h:71-76, material.h:38-53, light.h:24-27): tape ids of inputs.
struct IsectRec { int shape, tri; int v[3][3]; int n[3][3]; bool has_n; };
struct TexRec {
    int xi = -1, yi = -1;
    int t[4][3];
    bool textured = false;
    TexRec() { std::memset(t, 0xff, sizeof(t)); }  // -1: not fetched
};
struct MatRec { int mat; TexRec d, s, r; };
struct LightRec { int light; int I[3]; };
struct Records {
    std::vector<IsectRec> isect;
    std::vector<MatRec> mat;
    std::vector<LightRec> light;
};

// Analytic re-intersection of a known triangle (intersect.h:100-148)
template <typename T>
SPoint<T> intersect_tri(const Scene &sc, const Isect &is, const Ray<T> &ray, std::vector<IsectRec> *rec) {
    const Shape &sh = sc.shapes[is.shape];
    auto ind = sh.ind(is.tri);
    IsectRec ir;
    ir.shape = is.shape;
    ir.tri = is.tri;
    ir.has_n = false;
    V3<T> v[3];
    for (int k = 0; k < 3; k++) {
        V3f p = sh.vtx(ind[k]);
        for (int a = 0; a < 3; a++) v[k][a] = Param<T>::make(p[a], &ir.v[k][a]);
    }
    V2<T> uvs[3];
    if (sh.uv) {
        for (int k = 0; k < 3; k++) uvs[k] = V2<T>{T(sh.uv[2 * ind[k]]), T(sh.uv[2 * ind[k] + 1])};
    } else {
        uvs[0] = V2<T>{T(0.f), T(0.f)};
        uvs[1] = V2<T>{T(1.f), T(0.f)};
        uvs[2] = V2<T>{T(1.f), T(1.f)};
    }
    // Moller-Trumbore with the reference's zero-divisor substitution (intersect.h:71-90)
    V3<T> e1 = v[1] - v[0], e2 = v[2] - v[0];
    V3<T> pvec = cross(ray.d, e2);
    T divisor = dot(pvec, e1);
    if (divisor == T(0.f)) divisor = T(1e-8f);
    V3<T> s = ray.o - v[0];
    T u = dot(s, pvec) / divisor;
    V3<T> qvec = cross(s, e1);
    T vv = dot(ray.d, qvec) / divisor;
    T t = dot(e2, qvec) / divisor;
    T w = 1.f - (u + vv);
    V2<T> uv{w * uvs[0].x + u * uvs[1].x + vv * uvs[2].x, w * uvs[0].y + u * uvs[1].y + vv * uvs[2].y};
    V3<T> hit = ray.o + ray.d * t;
    V3<T> gn = normalize(cross(v[1] - v[0], v[2] - v[0]));
    V3<T> sn = gn;
    if (sh.n) {
        V3<T> n[3];
        ir.has_n = true;
        for (int k = 0; k < 3; k++) {
            V3f q = sh.nrm(ind[k]);
            for (int a = 0; a < 3; a++) n[k][a] = Param<T>::make(q[a], &ir.n[k][a]);
        }
        sn = normalize(w * n[0] + u * n[1] + vv * n[2]);
        if (dot(gn, sn) < T(0.f)) gn = -gn;
    }
    if (rec) rec->push_back(ir);
    SPoint<T> sp;
    sp.p = hit;
    sp.ng = gn;
    sp.f = make_frame(sn);
    sp.uv = uv;
    return sp;
}

template <typename T>
std::pair<Isect, SPoint<T>> intersect(const Scene &sc, const Ray<T> &ray, std::vector<IsectRec> *rec) {
    Ray<float> rf{fv(ray.o), fv(ray.d)};
    Isect is = nearest_hit(sc, rf);
    if (!is.valid()) return {is, SPoint<T>{}};
    return {is, intersect_tri<T>(sc, is, ray, rec)};
}

// ===================================================================
// Camera (camera.h)
// ===================================================================
template <typename T> struct TCam { M4<T> c2w; T fov, aspect; bool fisheye; };

template <typename T> inline TCam<T> make_tcam(const Camera &c, int *ids /*[16] or null*/) {
    TCam<T> tc;
    for (int i = 0; i < 16; i++) {
        int id;
        tc.c2w.m[i] = Param<T>::make(c.c2w.m[i], &id);
        if (ids) ids[i] = id;
    }
    tc.fov = T(c.fov);
    tc.aspect = T(c.aspect);
    tc.fisheye = c.fisheye;
    return tc;
}

// sample_primary (camera.h:48-84)
template <typename T> Ray<T> sample_primary(const TCam<T> &cam, const V2<T> &s) {
    V3<T> org = xfm_point(cam.c2w, V3<T>{T(0.f), T(0.f), T(0.f)});
    if (cam.fisheye) {
        T x = 2.f * (s.x - 0.5f), y = 2.f * (s.y - 0.5f);
        if (x * x + y * y > T(1.f)) return Ray<T>{org, V3<T>{T(0.f), T(0.f), T(0.f)}};
        T r = sqrt(x * x + y * y);
        T phi = atan2(y, x);
        T theta = r * kPi / 2.f;
        V3<T> dir{-cos(phi) * sin(theta), -sin(phi) * sin(theta), cos(theta)};
        return Ray<T>{org, xfm_vector(cam.c2w, normalize(dir))};
    }
    T ndcx = (s.x - 0.5f) * -2.f;
    T ndcy = (s.y - 0.5f) * -2.f / cam.aspect;
    V3<T> dir{cam.fov * ndcx, cam.fov * ndcy, T(1.f)};
    return Ray<T>{org, xfm_vector(cam.c2w, normalize(dir))};
}

// unproject / d_unproject / project_local / d_project_local (camera.h:86-214)
inline V3f unproject(const Camera &c, const V2f &s) {
    if (c.fisheye) {
        float x = 2.f * (s.x - 0.5f), y = 2.f * (s.y - 0.5f);
        float r = std::sqrt(x * x + y * y), phi = m_atan2(y, x), theta = r * kPi / 2.f;
        return V3f{-m_cos(phi) * m_sin(theta), -m_sin(phi) * m_sin(theta), m_cos(theta)};
    }
    float ndcx = (s.x - 0.5f) * -2.f, ndcy = (s.y - 0.5f) * -2.f / c.aspect;
    return V3f{c.fov * ndcx, c.fov * ndcy, 1.f};
}
inline std::pair<V3f, V3f> d_unproject(const Camera &c, const V2f &s) {
    if (c.fisheye) {
        float x = 2.f * (s.x - 0.5f), y = 2.f * (s.y - 0.5f);
        float r = std::sqrt(x * x + y * y), phi = m_atan2(y, x), theta = r * kPi / 2.f;
        float sp = m_sin(phi), cp = m_cos(phi), st = m_sin(theta), ct = m_cos(theta);
        float dxdphi = sp * st, dxdth = -cp * ct, dydphi = -cp * st, dydth = -sp * ct, dzdth = -st;
        float dphidx = -y / (r * r), dphidy = x / (r * r);
        float dthdx = (kPi / 2.f) * x / r, dthdy = (kPi / 2.f) * y / r;
        return {2.f * V3f{dxdphi * dphidx + dxdth * dthdx, dydphi * dphidx + dydth * dthdx, dzdth * dthdx},
                2.f * V3f{dxdphi * dphidy + dxdth * dthdy, dydphi * dphidy + dydth * dthdy, dzdth * dthdy}};
    }
    return {V3f{-2.f * c.fov, 0.f, 0.f}, V3f{0.f, -2.f * c.fov / c.aspect, 0.f}};
}
inline V2f project_local(const Camera &c, const V3f &l) {
    if (c.fisheye) {
        V3f d = normalize(l);
        float phi = m_atan2(d.y, d.x), theta = m_acos(d.z), r = theta * 2.f / kPi;
        return V2f{0.5f * (-r * m_cos(phi) + 1.f), 0.5f * (-r * m_sin(phi) + 1.f)};
    }
    return V2f{(-l.x / (l.z * c.fov) + 1.f) * 0.5f, (-l.y / (l.z * c.fov * c.aspect) + 1.f) * 0.5f};
}
inline V3f d_normalize(const V3f &v, const V3f &d) {
    float l = length(v);
    float dinv = dot(d, v);
    float dl = -dinv / (l * l);
    return (d + dl * v) / l;
}
inline V3f d_project_local(const Camera &c, const V3f &l, float dx, float dy) {
    if (c.fisheye) {
        V3f d = normalize(l);
        float phi = m_atan2(d.y, d.x), theta = m_acos(d.z), r = theta * 2.f / kPi;
        float dr = -0.5f * (m_cos(phi) * dx + m_sin(phi) * dy);
        float dphi = 0.5f * r * m_sin(phi) * dx - 0.5f * r * m_cos(phi) * dy;
        float dtheta = dr * (2.f / kPi);
        float dcos = -dtheta / std::sqrt(1.f - d.z * d.z);
        float t = d.x * d.x + d.y * d.y;
        return d_normalize(l, V3f{-dphi * d.y / t, dphi * d.x / t, dcos});
    }
    float zf = l.z * c.fov;
    float zfy = zf * c.aspect;
    return V3f{dx * (-1.f / zf), dy * (-1.f / zfy),
               dx * (c.fov * l.x / (zf * zf)) + dy * (c.fov * c.aspect * l.y / (zfy * zfy))};
}
// project with near-plane clipping (camera.h:216-242)
inline bool project(const Camera &c, const V3f &p0, const V3f &p1, V2f *s0, V2f *s1) {
    V3f a = xfm_point(c.w2c, p0), b = xfm_point(c.w2c, p1);
    if (a.z < c.clip_near && b.z < c.clip_near) return false;
    if (a.z < c.clip_near) {
        V3f dir = a - b;
        float t = -(b.z - c.clip_near) / dir.z;
        a = b + t * dir;
    } else if (b.z < c.clip_near) {
        V3f dir = b - a;
        float t = -(a.z - c.clip_near) / dir.z;
        b = a + t * dir;
    }
    *s0 = project_local(c, a);
    *s1 = project_local(c, b);
    return true;
}
// d_project (camera.h:244-313), including its +clip_near sign
inline void d_project(const Camera &c, const V3f &p0, const V3f &p1, float dp0x, float dp0y, float dp1x,
                      float dp1y, float *d_w2c) {
    V3f a = xfm_point(c.w2c, p0), b = xfm_point(c.w2c, p1);
    V3f ca = a, cb = b;
    if (a.z < c.clip_near) {
        V3f dir = a - b;
        float t = -(b.z + c.clip_near) / dir.z;
        ca = b + t * dir;
    } else if (b.z < c.clip_near) {
        V3f dir = b - a;
        float t = -(a.z + c.clip_near) / dir.z;
        cb = a + t * dir;
    }
    V3f dca = d_project_local(c, ca, dp0x, dp0y);
    V3f dcb = d_project_local(c, cb, dp1x, dp1y);
    V3f da{0.f, 0.f, 0.f}, db{0.f, 0.f, 0.f};
    if (a.z < c.clip_near) {
        V3f dir = a - b;
        float t = -(b.z + c.clip_near) / dir.z;
        db = db + dca;
        float dt = dot(dir, dca);
        V3f ddir = t * dca;
        db.z += -dt / dir.z;
        ddir.z += dt * (b.z / (dir.z * dir.z));
        da = da + ddir;
        db = db - ddir;
        db = db + dcb;
    } else if (b.z < c.clip_near) {
        V3f dir = b - a;
        float t = -(a.z + c.clip_near) / dir.z;
        da = da + dcb;
        float dt = dot(dir, dcb);
        V3f ddir = t * dcb;
        da.z += -dt / dir.z;
        ddir.z += dt * (a.z / (dir.z * dir.z));
        db = db + ddir;
        da = da - ddir;
        da = da + dca;
    } else {
        da = dca;
        db = dcb;
    }
    d_xfm_point(c.w2c, p0, da, d_w2c);
    d_xfm_point(c.w2c, p1, db, d_w2c);
}
inline bool in_screen(const Camera &c, const V2f &p) {
    if (!c.fisheye) return p.x >= 0.f && p.x < 1.f && p.y >= 0.f && p.y < 1.f;
    float d = (p.x - 0.5f) * (p.x - 0.5f) + (p.y - 0.5f) * (p.y - 0.5f);
    return d < 0.25f;
}

// ===================================================================
// Materials (material.h)
// ===================================================================
inline int modulo(int a, int b) {
    int r = a % b;
    return r < 0 ? r + b : r;
}

// Bilinear wrap texture or constant (material.h:84-203), recording tape ids.
template <typename T>
V3<T> tex_value(const Tex &tx, const V2<T> &uv, int ch, TexRec *rec) {
    if (tx.w == 0) {
        V3<T> r;
        for (int c = 0; c < ch; c++) {
            int id;
            r[c] = Param<T>::make(tx.data[c], &id);
            if (rec) rec->t[0][c] = id;
        }
        if (rec) { rec->xi = rec->yi = -1; rec->textured = false; }
        return r;
    }
    int xf = (int)std::floor(val(uv.x) * tx.w), yf = (int)std::floor(val(uv.y) * tx.h);
    T u = (uv.x * (float)tx.w) - (float)xf;
    T v = (uv.y * (float)tx.h) - (float)yf;
    int xfi = modulo(xf, tx.w), yfi = modulo(yf, tx.h), xci = modulo(xf + 1, tx.w), yci = modulo(yf + 1, tx.h);
    int yy[4] = {yfi, yci, yfi, yci}, xx[4] = {xfi, xfi, xci, xci};  // ff, fc, cf, cc
    V3<T> t[4];
    for (int k = 0; k < 4; k++)
        for (int c = 0; c < ch; c++) {
            int id;
            t[k][c] = Param<T>::make(tx.data[(yy[k] * tx.w + xx[k]) * ch + c], &id);
            if (rec) rec->t[k][c] = id;
        }
    if (rec) { rec->xi = xfi; rec->yi = yfi; rec->textured = true; }
    V3<T> r;
    for (int c = 0; c < ch; c++)
        r[c] = t[0][c] * (1.f - u) * (1.f - v) + t[1][c] * (1.f - u) * v + t[2][c] * u * (1.f - v) + t[3][c] * u * v;
    return r;
}

template <typename T> struct MatVals { V3<T> diffuse, specular; T roughness; };

template <typename T> V2<T> uv_scaled(const V2<T> &uv, const float *s) {
    return V2<T>{uv.x * T(s[0]), uv.y * T(s[1])};
}
template <typename T> V3<T> get_diffuse(const Material &m, const V2<T> &uv, MatRec *r) {
    return tex_value(m.diffuse, uv_scaled(uv, m.uv_d), 3, r ? &r->d : nullptr);
}
template <typename T> V3<T> get_specular(const Material &m, const V2<T> &uv, MatRec *r) {
    return tex_value(m.specular, uv_scaled(uv, m.uv_s), 3, r ? &r->s : nullptr);
}
template <typename T> T get_roughness(const Material &m, const V2<T> &uv, MatRec *r) {
    return tex_value(m.roughness, uv_scaled(uv, m.uv_r), 1, r ? &r->r : nullptr).x;
}
template <typename T> T roughness_to_phong(const T &r) { return max(2.f / r, T(0.f)); }

inline MatRec *push_mat(std::vector<MatRec> *recs, int mat) {
    if (!recs) return nullptr;
    MatRec r;
    r.mat = mat;
    recs->push_back(r);
    return &recs->back();
}

// GGX lobe (Walter et al. 2007; no counterpart in the reference):
// alpha = max(r^2, 1e-4), A = alpha^2, D = A / (pi ((n.h)^2 (A - 1) + 1)^2).
template <typename T> T ggx_A(const T &rough) {
    T a = max(rough * rough, 1e-4f);
    return a * a;
}
template <typename T> T ggx_D(const T &z, const T &A) {
    T k = z * z * (A - 1.f) + 1.f;
    return A / (kPi * k * k);
}

// Lambert + Blinn-Phong (or GGX) BSDF times cosine (material.h:257-351)
template <typename T>
V3<T> bsdf(const Scene &sc, int mi, const SPoint<T> &sp, const V3<T> &wi, const V3<T> &wo, std::vector<MatRec> *recs) {
    const Material &mat = sc.mats[mi];
    V3<T> n = sp.f[2];
    if (mat.two_sided && dot(wi, n) < T(0.f)) n = -n;
    T bcos = dot(n, wo);
    if (bcos <= T(5e-3f)) return V3<T>{T(0.f), T(0.f), T(0.f)};
    MatRec *r = push_mat(recs, mi);
    V3<T> kd = get_diffuse(mat, sp.uv, r);
    V3<T> ks = get_specular(mat, sp.uv, r);
    T rough = get_roughness(mat, sp.uv, r);
    V3<T> diff = kd * bcos / kPi;
    V3<T> spec{T(0.f), T(0.f), T(0.f)};
    if (sum(ks) > T(0.f) && dot(wi, n) > T(0.f)) {
        V3<T> m = normalize(wi + wo);
        V3<T> ml = to_local(sp.f, m);
        if (ml.z > T(0.f) && mat.model == DR_MICROFACET_GGX) {
            T A = ggx_A(rough);
            T D = ggx_D(ml.z, A);
            auto G1 = [&](const V3<T> &v) -> T {  // exact Smith G1
                T c = dot(v, n);
                if (dot(v, m) * c <= T(0.f)) return T(0.f);
                T t2 = max(1.f / (c * c) - 1.f, 0.f);
                return 2.f / (1.f + sqrt(1.f + A * t2));
            };
            T G = G1(wi) * G1(wo);
            T cd = dot(m, wo);
            T fr = pow(max(1.f - cd, 0.f), 5.f);
            V3<T> F{ks.x + (1.f - ks.x) * fr, ks.y + (1.f - ks.y) * fr, ks.z + (1.f - ks.z) * fr};
            spec = F * D * G / (4.f * dot(wi, n));
        } else if (ml.z > T(0.f)) {
            T e = roughness_to_phong(rough);
            T D = pow(max(ml.z, 0.f), e) * (e + 2.f) / float(2 * M_PI);
            auto proj_rough = [&](const V3<T> &v) -> T {
                V3<T> vl = to_local(sp.f, v);
                T c = vl.z;
                T s2 = 1.f - c * c;
                if (s2 <= T(0.f)) return sqrt(rough);
                T inv = 1.f / s2;
                T cp2 = vl.x * vl.x * inv, sp2 = vl.y * vl.y * inv;
                return sqrt(cp2 * rough + sp2 * rough);
            };
            auto G1 = [&](const V3<T> &v) -> T {
                T c = dot(v, n);
                if (dot(v, m) * c <= T(0.f)) return T(0.f);
                T tan_t = sqrt(max(1.f / (c * c) - 1.f, 0.f));
                if (tan_t == T(0.f)) return T(1.f);
                T alpha = proj_rough(v);
                T a = 1.f / (alpha * tan_t);
                if (a >= T(1.6f)) return T(1.f);
                T a2 = a * a;
                return (3.535f * a + 2.181f * a2) / (1.0f + 2.276f * a + 2.577f * a2);
            };
            T G = G1(wi) * G1(wo);
            T cd = dot(m, wo);
            T fr = pow(max(1.f - cd, 0.f), 5.f);
            V3<T> F{ks.x + (1.f - ks.x) * fr, ks.y + (1.f - ks.y) * fr, ks.z + (1.f - ks.z) * fr};
            spec = F * D * G / (4.f * dot(wi, n));
        }
    }
    return diff + spec;
}

inline V3f cos_hemisphere(const V2f &s) {  // vector.h:533-538
    float phi = 2.f * kPi * s.x;
    float tmp = std::sqrt(1.f - s.y);
    return V3f{m_cos(phi) * tmp, m_sin(phi) * tmp, std::sqrt(s.y)};
}

struct BSDFSample { V2f uv; float w; };
struct LightSample { V2f uv; float sel, tri_sel; };
struct SecondarySample { LightSample light; BSDFSample bsdf; float rr; };
struct EdgeSample { float bsdf_component, u; };

// Draw orders reproduce the reference compiled by GCC, which evaluates
// function arguments right to left: make_vector2(u(), u()) receives the first
// draw in its second slot (light.h:46-51, material.h:246-250).
inline LightSample draw_light(Sampler &s) {
    LightSample l;
    l.uv.y = s.next();
    l.uv.x = s.next();
    l.sel = s.next();
    l.tri_sel = s.next();
    return l;
}
inline BSDFSample draw_bsdf(Sampler &s) {
    BSDFSample b;
    b.uv.y = s.next();
    b.uv.x = s.next();
    b.w = s.next();
    return b;
}
inline SecondarySample draw_secondary(Sampler &s) {
    SecondarySample x;
    x.light = draw_light(s);
    x.bsdf = draw_bsdf(s);
    x.rr = s.next();
    return x;
}
inline EdgeSample draw_edge(Sampler &s) {
    EdgeSample e;
    e.bsdf_component = s.next();
    e.u = s.next();
    return e;
}

// BSDF importance sampling (material.h:353-412); returns (dir, is_specular)
template <typename T>
std::pair<V3<T>, bool> sample_bsdf_dir(const Scene &sc, int mi, const SPoint<T> &sp, const V3<T> &wi,
                                       const BSDFSample &bs, std::vector<MatRec> *recs) {
    const Material &mat = sc.mats[mi];
    MatRec *r = push_mat(recs, mi);
    V3<T> kd = get_diffuse(mat, sp.uv, r);
    V3<T> ks = get_specular(mat, sp.uv, r);
    T dw = luminance(kd), sw = luminance(ks);
    T ws = dw + sw;
    V3<T> zero{T(0.f), T(0.f), T(0.f)};
    if (ws <= T(0.f)) return {zero, false};
    T dpmf = dw / ws;
    if (T(bs.w) <= dpmf) {
        if (dpmf <= T(0.f)) return {zero, false};
        V3f l = cos_hemisphere(bs.uv);
        return {to_world(sp.f, tv<T>(l)), false};
    }
    if (sw <= T(0.f)) return {zero, false};
    T rough = get_roughness(mat, sp.uv, r);
    float phi = 2.f * kPi * bs.uv.y;
    float sphi = m_sin(phi), cphi = m_cos(phi);
    T ct;
    if (mat.model == DR_MICROFACET_GGX) {
        T A = ggx_A(rough);
        ct = sqrt((1.f - bs.uv.x) / (1.f + (A - 1.f) * bs.uv.x));
    } else {
        T e = roughness_to_phong(rough);
        ct = pow(bs.uv.x, 1.0f / (e + 2.0f));
    }
    T st = sqrt(max(1.f - ct * ct, 0.f));
    V3<T> ml{st * cphi, st * sphi, ct};
    V3<T> m = to_world(sp.f, ml);
    V3<T> dir = 2.f * dot(wi, m) * m - wi;
    return {dir, val(rough) <= 0.01f};
}

// pdf of sample_bsdf_dir in solid angle (material.h:414-462)
template <typename T>
T bsdf_pdf(const Scene &sc, int mi, const SPoint<T> &sp, const V3<T> &wi, const V3<T> &wo, std::vector<MatRec> *recs) {
    const Material &mat = sc.mats[mi];
    MatRec *r = push_mat(recs, mi);
    V3<T> kd = get_diffuse(mat, sp.uv, r);
    V3<T> ks = get_specular(mat, sp.uv, r);
    T dw = luminance(kd), sw = luminance(ks);
    T ws = dw + sw;
    if (ws <= T(0.f)) return T(0.f);
    T dpmf = dw / ws, spmf = sw / ws;
    T dpdf = T(0.f);
    if (dpmf > T(0.f)) {
        T c = dot(sp.f[2], wo);
        c = mat.two_sided ? fabs(c) : max(c, 0.f);
        dpdf = dpmf * c / kPi;
    }
    T spdf = T(0.f);
    if (spmf > T(0.f)) {
        V3<T> m = normalize(wi + wo);
        V3<T> ml = to_local(sp.f, m);
        if (ml.z > T(0.f)) {
            T rough = get_roughness(mat, sp.uv, r);
            if (mat.model == DR_MICROFACET_GGX) {  // half vectors drawn with density D (n.h)
                T D = ggx_D(ml.z, ggx_A(rough));
                spdf = spmf * D * ml.z / (4.f * fabs(dot(wo, m)));
            } else {
                T e = roughness_to_phong(rough);
                T D = pow(ml.z, e) * (e + 2.f) / float(2 * M_PI);
                spdf = spmf * D / (4.f * fabs(dot(wo, m)));
            }
        }
    }
    return dpdf + spdf;
}

// ===================================================================
// Lights (scene.h:49-108, sample.h:6-24)
// ===================================================================
template <typename T>
V3<T> get_intensity(const Scene &sc, int li, std::vector<LightRec> *recs) {
    LightRec r;
    r.light = li;
    V3<T> I;
    for (int c = 0; c < 3; c++) I[c] = Param<T>::make(sc.lights[li].I[c], &r.I[c]);
    if (recs) recs->push_back(r);
    return I;
}

template <typename T>
std::pair<Isect, SPoint<T>> sample_point_on_light(const Scene &sc, const LightSample &ls, std::vector<IsectRec> *rec) {
    int li = sc.light_sel.sample_discrete(ls.sel);
    int tri = sc.light_tri[li].sample_discrete(ls.tri_sel);
    const Shape &sh = sc.shapes[sc.lights[li].shape];
    auto ind = sh.ind(tri);
    IsectRec ir;
    ir.shape = sc.lights[li].shape;
    ir.tri = tri;
    ir.has_n = false;
    V3<T> v[3];
    for (int k = 0; k < 3; k++) {
        V3f p = sh.vtx(ind[k]);
        for (int a = 0; a < 3; a++) v[k][a] = Param<T>::make(p[a], &ir.v[k][a]);
    }
    if (rec) rec->push_back(ir);
    float a = std::sqrt(ls.uv.x);
    float b1 = 1.f - a, b2 = a * ls.uv.y;
    V3<T> e1 = v[1] - v[0], e2 = v[2] - v[0];
    V3<T> nn = normalize(cross(e1, e2));
    SPoint<T> sp;
    sp.p = v[0] + e1 * b1 + e2 * b2;
    sp.ng = nn;
    sp.f = make_frame(nn);
    sp.uv = V2<T>{T(ls.uv.x), T(ls.uv.y)};
    return {Isect{ir.shape, tri}, sp};
}

template <typename T>
T light_pdf(const Scene &sc, const Isect &is, std::vector<IsectRec> *rec) {
    if (!is.valid()) return T(0.f);
    int li = sc.shapes[is.shape].light;
    if (li < 0) return T(0.f);
    float lpmf = luminance(V3f{sc.lights[li].I[0], sc.lights[li].I[1], sc.lights[li].I[2]}) /
                 sc.total_light_intensity;
    const Shape &sh = sc.shapes[is.shape];
    auto ind = sh.ind(is.tri);
    IsectRec ir;
    ir.shape = is.shape;
    ir.tri = is.tri;
    ir.has_n = false;
    V3<T> v[3];
    for (int k = 0; k < 3; k++) {
        V3f p = sh.vtx(ind[k]);
        for (int a = 0; a < 3; a++) v[k][a] = Param<T>::make(p[a], &ir.v[k][a]);
    }
    if (rec) rec->push_back(ir);
    T area = 0.5f * length(cross(v[1] - v[0], v[2] - v[0]));
    float tri_pmf = val(area) / sc.light_area[li];
    return lpmf * tri_pmf / area;
}

// ===================================================================
// Path tracing (pathtrace.h)
// ===================================================================
template <typename T> struct SecondaryPoint {
    int bounce;
    V3f wi;
    Isect isect;
    SPoint<T> sp;
    V3f throughput;
};

// eval (pathtrace.h:7-57): contribution of a point on an emitter, shadow-tested
template <typename T>
V3<T> eval(const Scene &sc, const V3<T> &wi, const Isect &sis, const SPoint<T> &sp, const Isect &lis,
           const SPoint<T> &lp, Records *R) {
    V3<T> zero{T(0.f), T(0.f), T(0.f)};
    if (!sis.valid() || !lis.valid()) return zero;
    int li = sc.shapes[lis.shape].light;
    if (li < 0) return zero;
    V3<T> d = lp.p - sp.p;
    T dist = length(d);
    if (dist == T(0.f)) return zero;
    V3<T> nd = d / dist;
    if (occluded(sc, Ray<float>{fv(sp.p), fv(nd)}, val(dist))) return zero;
    V3<T> b = bsdf(sc, sc.shapes[sis.shape].mat, sp, wi, nd, R ? &R->mat : nullptr);
    T lcos = dot(lp.f[2], -nd);
    if (lcos <= T(0.f)) return zero;
    T d2 = sq(dist);
    V3<T> I = get_intensity<T>(sc, li, R ? &R->light : nullptr);
    V3<T> lc = I * (lcos / d2);
    return mul(b, lc);
}

// next_event_estimation (pathtrace.h:59-102); MIS weight is a constant
template <typename T>
V3<T> nee(const Scene &sc, const LightSample &ls, const V3<T> &wi, const Isect &sis, const SPoint<T> &sp, Records *R) {
    if (!sis.valid()) return V3<T>{T(0.f), T(0.f), T(0.f)};
    auto lpt = sample_point_on_light<T>(sc, ls, R ? &R->isect : nullptr);
    const SPoint<T> &lp = lpt.second;
    V3<T> ldir = normalize(lp.p - sp.p);
    T lcos = fabs(dot(ldir, lp.ng));
    T lpdf = light_pdf<T>(sc, lpt.first, R ? &R->isect : nullptr);
    float bpdf = bsdf_pdf<float>(sc, sc.shapes[sis.shape].mat, fsp(sp), fv(wi), fv(ldir), nullptr) * val(lcos) /
                 length_sq(fv(lp.p) - fv(sp.p));
    float mis = val(sq(lpdf) / (sq(T(bpdf)) + sq(lpdf)));
    V3<T> e = eval<T>(sc, wi, sis, sp, lpt.first, lp, R);
    return e * (mis / lpdf);
}

struct SampleResultBSDF { Isect isect; bool specular; };

// scene-level sample_bsdf with two-sided flip and the diffuse gradient stop
// (pathtrace.h:104-162)
template <typename T>
std::pair<SampleResultBSDF, SPoint<T>> sample_bsdf_scene(const Scene &sc, const BSDFSample &bs, const V3<T> &wi,
                                                         const Isect &sis, const SPoint<T> &sp, Records *R) {
    if (!sis.valid()) return {SampleResultBSDF{Isect{}, false}, SPoint<T>{}};
    int mi = sc.shapes[sis.shape].mat;
    if (sc.mats[mi].two_sided && dot(wi, sp.f[2]) < T(0.f)) {
        SPoint<T> fl = sp;
        fl.f[0] = -fl.f[0];
        fl.f[1] = -fl.f[1];
        fl.f[2] = -fl.f[2];
        fl.ng = -fl.ng;
        return sample_bsdf_scene<T>(sc, bs, wi, sis, fl, R);
    }
    auto dr = sample_bsdf_dir<T>(sc, mi, sp, wi, bs, R ? &R->mat : nullptr);
    if (length(dr.first) <= T(0.f)) return {SampleResultBSDF{Isect{}, false}, SPoint<T>{}};
    Ray<T> ray{sp.p, dr.first};
    auto hit = intersect<T>(sc, ray, (dr.second && R) ? &R->isect : nullptr);
    SPoint<T> hp = hit.second;
    if (!dr.second) hp = csp<T>(fsp(hit.second));
    return {SampleResultBSDF{hit.first, dr.second}, hp};
}

// shade (pathtrace.h:179-297)
template <typename T>
V3<T> shade(const Scene &sc, const V3<T> &wi, const Isect &pis, const SPoint<T> &psp, const LightSample &ls,
            const std::vector<SecondarySample> &ss, bool include_primary_light,
            std::vector<SecondaryPoint<T>> *spts, Records *R) {
    V3<T> color{T(0.f), T(0.f), T(0.f)};
    if (!pis.valid()) return color;
    if (include_primary_light && sc.shapes[pis.shape].light >= 0) {
        if (dot(psp.f[2], wi) > T(0.f)) color = color + get_intensity<T>(sc, sc.shapes[pis.shape].light, R ? &R->light : nullptr);
    }
    V3<T> thr{T(1.f), T(1.f), T(1.f)};
    V3<T> cwi = wi;
    Isect cis = pis;
    SPoint<T> csp_ = psp;
    bool hit_diffuse = false;
    for (int b = 0; b < (int)ss.size(); b++) {
        color = color + mul(thr, nee<T>(sc, ls, wi, cis, csp_, R));
        if (spts && !hit_diffuse) spts->push_back(SecondaryPoint<T>{b, fv(cwi), cis, csp_, fv(thr)});
        auto sr = sample_bsdf_scene<T>(sc, ss[b].bsdf, cwi, cis, csp_, R);
        hit_diffuse = hit_diffuse || !sr.first.specular;
        Isect nis = sr.first.isect;
        if (!nis.valid()) break;
        SPoint<T> nsp = sr.second;
        V3<T> wo = normalize(nsp.p - csp_.p);
        if (hit_diffuse) wo = tv<T>(fv(wo));
        int mi = sc.shapes[cis.shape].mat;
        T pdf = bsdf_pdf<T>(sc, mi, csp_, cwi, wo, R ? &R->mat : nullptr);
        if (sc.detached_pdf) pdf = T(val(pdf));  // DR_FLAG_DETACHED_PDF: a constant in the backward pass
        if (pdf <= T(0.f)) break;
        V3<T> be = bsdf<T>(sc, mi, csp_, cwi, wo, R ? &R->mat : nullptr);
        if (sum(be) <= T(0.f)) break;
        int nli = sc.shapes[nis.shape].light;
        if (nli >= 0 && dot(nsp.f[2], -wo) > T(0.f)) {
            V3<T> contrib = mul(be, get_intensity<T>(sc, nli, R ? &R->light : nullptr));
            float lpdf = light_pdf<float>(sc, nis, nullptr) * length_sq(fv(nsp.p) - fv(csp_.p)) /
                         std::fabs(dot(fv(wo), fv(nsp.ng)));
            float mis = val(sq(pdf) / (sq(T(lpdf)) + sq(pdf)));
            color = color + mul(thr, contrib) * (mis / pdf);
        }
        thr = mul(thr, be / pdf);
        if (b >= 5) {
            float q = std::min(vmax(fv(thr)), 0.95f);
            if (ss[b].rr >= q) break;
            thr = thr / q;
        }
        cwi = -wo;
        cis = nis;
        csp_ = nsp;
    }
    return color;
}

// ===================================================================
// Edges: extraction, silhouettes, trees (scene.cpp:54-97, edge.h, edge_tree.cpp)
// ===================================================================
inline V3f non_shared(const Scene &sc, const Edge &e, int f) {
    auto ind = sc.shapes[e.shape].ind(f);
    for (int i = 0; i < 3; i++)
        if (ind[i] != e.v0 && ind[i] != e.v1) return sc.shapes[e.shape].vtx(ind[i]);
    return V3f{0.f, 0.f, 0.f};
}
// is_silhouette (edge.h:59-79)
inline bool is_silhouette(const Scene &sc, const V3f &p, const Edge &e) {
    const Shape &sh = sc.shapes[e.shape];
    if (!sh.n) return true;
    if (e.f0 == -1 || e.f1 == -1) return true;
    V3f v0 = sc.ev0(e), v1 = sc.ev1(e);
    V3f a = non_shared(sc, e, e.f0), b = non_shared(sc, e, e.f1);
    V3f n0 = normalize(cross(v0 - a, v1 - a));
    V3f n1 = normalize(cross(v1 - b, v0 - b));
    bool ff0 = dot(p - v0, n0) > 0.f && dot(p - v1, n0) > 0.f && dot(p - a, n0) > 0.f;
    bool ff1 = dot(p - v0, n1) > 0.f && dot(p - v1, n1) > 0.f && dot(p - b, n1) > 0.f;
    return (ff0 && !ff1) || (!ff0 && ff1);
}

// Cohen-Sutherland clip to [0,1]^2 (line_clip.h:13-102)
inline bool clip_line(V2f a, V2f b, V2f *oa, V2f *ob) {
    auto code = [](const V2f &v) {
        int c = 0;
        if (v.x < 0.f) c |= 1; else if (v.x > 1.f) c |= 2;
        if (v.y < 0.f) c |= 4; else if (v.y > 1.f) c |= 8;
        return c;
    };
    int c0 = code(a), c1 = code(b);
    while (true) {
        if (!(c0 | c1)) { *oa = a; *ob = b; return true; }
        if (c0 & c1) return false;
        int out = c0 ? c0 : c1;
        V2f v{0.f, 0.f};
        if (out & 8) { v.x = a.x + (b.x - a.x) * (1.f - a.y) / (b.y - a.y); v.y = 1.f; }
        else if (out & 4) { v.x = a.x + (b.x - a.x) * (0.f - a.y) / (b.y - a.y); v.y = 0.f; }
        else if (out & 2) { v.y = a.y + (b.y - a.y) * (1.f - a.x) / (b.x - a.x); v.x = 1.f; }
        else if (out & 1) { v.y = a.y + (b.y - a.y) * (0.f - a.x) / (b.x - a.x); v.x = 0.f; }
        if (out == c0) { a = v; c0 = code(a); } else { b = v; c1 = code(b); }
    }
}

struct PrimInfo {
    int prim;
    V3f n0, n1;
    AABB sb, db;  // spatial, scaled directional
    V3f sc, dc;   // centroids
};

struct BuildNode {
    AABB sb;
    V3f axis;
    float angle;
    int first = 0, n = 0;
    std::unique_ptr<BuildNode> c[2];
};

// median-split build (edge_tree.cpp:49-173): in the reference's RNG mode
// partitioning with std::nth_element on the same comparator, so that ties
// resolve as in the reference; in the Philox mode with the product's rule
// (g_product_tree)
template <bool DIR>
std::unique_ptr<BuildNode> build_edge_node(const std::vector<Edge> &edges, std::vector<PrimInfo> &pi, int start, int end,
                                           int *total, std::vector<Edge> &ordered) {
    auto node = std::make_unique<BuildNode>();
    (*total)++;
    AABB sb, db;
    for (int i = start; i < end; i++) {
        sb.add(pi[i].sb);
        if (DIR) db.add(pi[i].db);
    }
    V3f nsum{0.f, 0.f, 0.f};
    if (g_product_tree) {
        long long fs[3] = {0, 0, 0};
        for (int i = start; i < end; i++)
            for (int a = 0; a < 3; a++) fs[a] += edge_fixed(pi[i].n0[a]) + edge_fixed(pi[i].n1[a]);
        nsum = V3f{edge_unfixed(fs[0]), edge_unfixed(fs[1]), edge_unfixed(fs[2])};
    } else {
        for (int i = start; i < end; i++) nsum = nsum + pi[i].n0 + pi[i].n1;
    }
    V3f axis = normalize(nsum);
    float cmin = 1.f;
    for (int i = start; i < end; i++) {
        cmin = std::min(cmin, dot(pi[i].n0, axis));
        cmin = std::min(cmin, dot(pi[i].n1, axis));
    }
    node->sb = sb;
    node->axis = axis;
    node->angle = m_acos(cmin);
    int n = end - start;
    auto make_leaf = [&]() {
        node->first = (int)ordered.size();
        for (int i = start; i < end; i++) ordered.push_back(edges[pi[i].prim]);
        node->n = n;
    };
    if (n == 1) {
        make_leaf();
        return node;
    }
    AABB scb, dcb;
    for (int i = start; i < end; i++) {
        scb.add(pi[i].sc);
        if (DIR) dcb.add(pi[i].dc);
    }
    int dim = -1;
    float maxe = -INFINITY;
    for (int a = 0; a < 3; a++) {
        float e = scb.hi[a] - scb.lo[a];
        if (e > maxe) { dim = a; maxe = e; }
    }
    if (DIR) {
        for (int a = 0; a < 3; a++) {
            float e = dcb.hi[a] - dcb.lo[a];
            if (e > maxe) { dim = a + 3; maxe = e; }
        }
    }
    const AABB &cb = dim < 3 ? scb : dcb;
    bool spatial = dim < 3;
    if (dim >= 3) dim -= 3;
    if (cb.hi[dim] == cb.lo[dim]) {
        make_leaf();
        return node;
    }
    int mid = (start + end) / 2;
    if (g_product_tree) {
        std::stable_sort(pi.begin() + start, pi.begin() + end, [dim, spatial](const PrimInfo &a, const PrimInfo &b) {
            return spatial ? edge_ord_key(a.sc[dim]) < edge_ord_key(b.sc[dim])
                           : edge_ord_key(a.dc[dim]) < edge_ord_key(b.dc[dim]);
        });
    } else {
        std::nth_element(&pi[start], &pi[mid], &pi[end - 1] + 1, [dim, spatial](const PrimInfo &a, const PrimInfo &b) {
            return spatial ? a.sc[dim] < b.sc[dim] : a.dc[dim] < b.dc[dim];
        });
    }
    node->c[0] = build_edge_node<DIR>(edges, pi, start, mid, total, ordered);
    node->c[1] = build_edge_node<DIR>(edges, pi, mid, end, total, ordered);
    return node;
}

// flatten_bvh (edge_tree.cpp:175-205)
inline int flatten(const Scene &sc, std::vector<EdgeNode> &nodes, const std::vector<Edge> &ordered, const BuildNode *b,
                   int *off) {
    int my = (*off)++;
    EdgeNode &ln = nodes[my];
    ln.bounds = b->sb;
    ln.cone_axis = b->axis;
    ln.cone_angle = b->angle;
    if (b->n > 0) {
        ln.offset = b->first;
        ln.nprims = b->n;
        ln.total_length = 0.f;
        for (int i = 0; i < b->n; i++) {
            const Edge &e = ordered[b->first + i];
            ln.total_length += length(sc.ev1(e) - sc.ev0(e));
        }
    } else {
        nodes[my].nprims = 0;
        flatten(sc, nodes, ordered, b->c[0].get(), off);
        int second = flatten(sc, nodes, ordered, b->c[1].get(), off);
        nodes[my].offset = second;
        nodes[my].total_length = nodes[my + 1].total_length + nodes[second].total_length;
    }
    return my;
}

template <bool DIR> EdgeTree build_edge_tree(const Scene &sc, const std::vector<Edge> &edges) {
    EdgeTree t;
    if (edges.empty()) return t;
    struct Rule {
        Rule(bool on) { g_product_tree = on; }
        ~Rule() { g_product_tree = false; }
    } rule(g_product_rule && edges.size() > (size_t)DR_TREE_EXACT_MAX_EDGES);
    std::vector<PrimInfo> pi(edges.size());
    AABB world;
    for (size_t i = 0; i < edges.size(); i++) {
        AABB b;
        b.add(sc.ev0(edges[i]));
        b.add(sc.ev1(edges[i]));
        pi[i].prim = (int)i;
        pi[i].sb = b;
        pi[i].sc = 0.5f * b.lo + 0.5f * b.hi;
        pi[i].n0 = pi[i].n1 = V3f{0.f, 0.f, 0.f};
        world.add(b);
    }
    if (DIR) {
        float factor = length(world.hi - world.lo) / 8.f;
        for (size_t i = 0; i < edges.size(); i++) {
            const Edge &e = edges[i];
            const Shape &sh = sc.shapes[e.shape];
            V3f sn = normalize(sh.nrm(e.v0) + sh.nrm(e.v1));
            V3f n0 = sh.face_normal(e.f0), n1 = sh.face_normal(e.f1);
            if (dot(n0, sn) < 0.f) n0 = -n0;
            if (dot(n1, sn) < 0.f) n1 = -n1;
            pi[i].n0 = n0;
            pi[i].n1 = n1;
            AABB d;
            d.add(n0 * factor);
            d.add(n1 * factor);
            pi[i].db = d;
            pi[i].dc = 0.5f * (d.lo + d.hi);
        }
    }
    std::vector<Edge> ordered;
    int total = 0;
    auto root = build_edge_node<DIR>(edges, pi, 0, (int)edges.size(), &total, ordered);
    t.nodes.resize(total);
    int off = 0;
    flatten(sc, t.nodes, ordered, root.get(), &off);
    t.edges = ordered;
    return t;
}

// ---- box / cone test (aabb.cpp:98-311, the GeometricTools algorithm) ----
struct ConePoly { int n; int idx[6]; };
// Silhouette polygons of a box seen from each of the 27 regions of the cone
// apex (per axis: above, inside, below the slab).  Corner j has coordinate
// +extent on axis a iff bit a of j is set.  Same table as aabb.cpp:106-132.
static const ConePoly kConePolys[27] = {
    {6, {1, 5, 4, 6, 2, 3}}, {6, {0, 2, 3, 1, 5, 4}}, {6, {0, 2, 3, 7, 5, 4}}, {6, {0, 4, 6, 2, 3, 1}},
    {4, {0, 2, 3, 1}},       {6, {0, 2, 3, 7, 5, 1}}, {6, {0, 4, 6, 7, 3, 1}}, {6, {0, 2, 6, 7, 3, 1}},
    {6, {0, 2, 6, 7, 5, 1}}, {6, {0, 1, 5, 4, 6, 2}}, {4, {0, 1, 5, 4}},       {6, {0, 1, 3, 7, 5, 4}},
    {4, {0, 4, 6, 2}},       {0, {0}},                {4, {1, 3, 7, 5}},       {6, {0, 4, 6, 7, 3, 2}},
    {4, {2, 6, 7, 3}},       {6, {1, 3, 2, 6, 7, 5}}, {6, {0, 1, 5, 7, 6, 2}}, {6, {0, 1, 5, 7, 6, 4}},
    {6, {0, 1, 3, 7, 6, 4}}, {6, {0, 4, 5, 7, 6, 2}}, {4, {4, 5, 7, 6}},       {6, {1, 3, 7, 6, 4, 5}},
    {6, {0, 4, 5, 7, 3, 2}}, {6, {2, 6, 4, 5, 7, 3}}, {6, {1, 3, 2, 6, 4, 5}}};

struct Cone { V3f o, d; float cos_angle; };

inline bool box_cone(const AABB &b, const Cone &cone) {
    if (cone.cos_angle <= 0.f) return true;
    V3f C = 0.5f * (b.lo + b.hi), E = 0.5f * (b.hi - b.lo);
    V3f CmV = C - cone.o;
    float DdCmV = dot(cone.d, CmV);
    float rad = E.x * std::fabs(cone.d.x) + E.y * std::fabs(cone.d.y) + E.z * std::fabs(cone.d.z);
    if (DdCmV + rad <= 0) return false;
    int ix[3];
    for (int a = 0; a < 3; a++) ix[a] = CmV[a] < -E[a] ? 2 : (CmV[a] > E[a] ? 0 : 1);
    int lookup = ix[0] + 3 * ix[1] + 9 * ix[2];
    if (lookup == 13) return true;
    const ConePoly &poly = kConePolys[lookup];
    float c2 = cone.cos_angle * cone.cos_angle;
    V3f X[8], PmV[8];
    float DdPmV[8], sDd[8], sLen[8];
    int imax = -1, jmax = -1;
    for (int i = 0; i < poly.n; i++) {
        int j = poly.idx[i];
        X[j] = V3f{(j & 1) ? E.x : -E.x, (j & 2) ? E.y : -E.y, (j & 4) ? E.z : -E.z};
        DdPmV[j] = dot(cone.d, X[j]) + DdCmV;
        if (DdPmV[j] > 0) {
            PmV[j] = X[j] + CmV;
            sDd[j] = DdPmV[j] * DdPmV[j];
            sLen[j] = dot(PmV[j], PmV[j]);
            if (sDd[j] - c2 * sLen[j] > 0) return true;
            if (imax == -1 || sDd[j] * sLen[jmax] > sDd[jmax] * sLen[j]) { imax = i; jmax = j; }
        }
    }
    if (imax == -1) return false;
    float mLen = sLen[jmax], mDd = DdPmV[jmax];
    const V3f &mX = X[jmax], &mP = PmV[jmax];
    for (int side = 0; side < 2; side++) {
        int jother, s, k0;
        float fder;
        if (side == 0) {
            int inext = imax < poly.n - 1 ? imax + 1 : 0;
            jother = poly.idx[inext];
            int jd = jother - jmax;
            s = jd > 0 ? 1 : -1;
            k0 = std::abs(jd) >> 1;
            fder = s * (cone.d[k0] * mLen - mDd * mP[k0]);
        } else {
            int iprev = imax > 0 ? imax - 1 : poly.n - 1;
            jother = poly.idx[iprev];
            int jd = jmax - jother;
            s = jd > 0 ? 1 : -1;
            k0 = std::abs(jd) >> 1;
            fder = -s * (cone.d[k0] * mLen - mDd * mP[k0]);
        }
        if (fder > 0) {
            int k1 = (k0 + 1) % 3, k2 = (k1 + 1) % 3;
            float numer = mP[k1] * mP[k1] + mP[k2] * mP[k2];
            float denom = cone.d[k1] * mP[k1] + cone.d[k2] * mP[k2];
            V3f M;
            M[k0] = numer * cone.d[k0];
            M[k1] = denom * (mX[k1] + CmV[k1]);
            M[k2] = denom * (mX[k2] + CmV[k2]);
            float DdM = dot(cone.d, M);
            if (DdM * DdM - c2 * dot(M, M) > 0) return true;
            float det = s * (cone.d[k1] * mP[k2] - cone.d[k2] * mP[k1]);
            return det <= 0;
        }
    }
    return false;
}

// A sampled edge with its weight and its key in the traversal order:
// mode << 27 | index of the edge in its tree (cone-mode edges first, then in
// depth-first order, which is the order of the tree's edge array).
struct EdgeW { Edge e; float w; int key; };

// bsdf_bound (edge_tree.cpp:345-480)
inline float min_sq(float lo, float hi) {
    if (lo <= 0.f && hi >= 0.f) return 0.f;
    if (lo < 0.f && hi < 0.f) return hi * hi;
    return lo * lo;
}
inline float max_sq(float lo, float hi) { return std::max(lo * lo, hi * hi); }

inline float bsdf_bound(const Scene &sc, const EdgeNode &node, const V3f &wi, const Isect &is, const SPoint<float> &sp,
                        float dl, float sl) {
    const AABB &b = node.bounds;
    const Material &mat = sc.mats[sc.shapes[is.shape].mat];
    float cos_max = 0.f;
    for (int i = 0; i < 8; i++)
        if (dot(sp.f[2], b.corner(i) - sp.p) > 0.f) { cos_max = 1.f; break; }
    if (cos_max <= 0.f) return 0.f;
    float maxp = 0.f;
    if (sl > 0.f) {
        V3f hy = normalize(cross(sp.f[2], wi));
        Frame<float> hf{normalize(cross(wi, hy)), hy, wi};
        AABB hb;
        for (int i = 0; i < 8; i++) hb.add(to_local(hf, b.corner(i) - sp.p));
        float cphi = 0.f;
        float hx = hb.hi.x;
        if (hx > 0.f) cphi = hx / std::sqrt(min_sq(hb.lo.y, hb.hi.y) + hx * hx);
        else if (hx == 0.f) cphi = std::max(cphi, 0.f);
        else cphi = hx / std::sqrt(max_sq(hb.lo.y, hb.hi.y) + hx * hx);
        float cto_min, cto_max;
        if (hb.lo.z > 0.f)
            cto_min = hb.lo.z / (max_sq(hb.lo.x, hb.hi.x) + max_sq(hb.lo.y, hb.hi.y) + hb.lo.z * hb.lo.z);
        else
            cto_min = hb.lo.z / (min_sq(hb.lo.x, hb.hi.x) + min_sq(hb.lo.y, hb.hi.y) + hb.lo.z * hb.lo.z);
        if (hb.hi.z > 0.f)
            cto_max = hb.hi.z / (min_sq(hb.lo.x, hb.hi.x) + min_sq(hb.lo.y, hb.hi.y) + hb.hi.z * hb.hi.z);
        else
            cto_max = hb.hi.z / (max_sq(hb.lo.x, hb.hi.x) + max_sq(hb.lo.y, hb.hi.y) + hb.hi.z * hb.hi.z);
        float cth_min = std::sqrt((cto_min + 1.f) / 2.f), cth_max = std::sqrt((cto_max + 1.f) / 2.f);
        V3f ln = to_local(hf, sp.f[2]);
        float chmax = cphi >= 0.f ? std::sqrt(ln.z * ln.z / (ln.z * ln.z + ln.x * ln.x * cphi * cphi)) : 1.f;
        if (chmax > cth_max) chmax = cth_max;
        else if (chmax < cth_min) chmax = cth_min;
        float shmax = std::sqrt(std::max(1.f - chmax * chmax, 0.f));
        float hdn = std::min(std::fabs(ln.x * shmax * cphi) + ln.z * chmax, 1.f);
        float rough = get_roughness<float>(mat, sp.uv, nullptr);
        if (mat.model == DR_MICROFACET_GGX) {
            maxp = ggx_D(hdn, ggx_A(rough));
        } else {
            float e = roughness_to_phong(rough);
            maxp = m_pow(hdn, e) * (e + 2.f) / float(2 * M_PI);
        }
    }
    return cos_max * (dl / kPi + sl * maxp);
}

// contains_silhouette (edge_tree.cpp:482-497)
inline bool contains_silhouette(const EdgeNode &node, const V3f &p) {
    V3f c = node.bounds.center();
    float r = length(node.bounds.hi - c);
    V3f d = c - p;
    float l = length(d);
    float vt = r / l;
    if (vt >= 1.f) return true;
    float va = m_atan(vt);
    d = d / l;
    float ang = m_acos(dot(-d, node.cone_axis));
    float range = node.cone_angle + va;
    return ang - range <= float(M_PI / 2.f) && ang + range >= float(M_PI / 2.f);
}

inline float node_importance(const EdgeNode &node, float bb, const SPoint<float> &sp) {
    return bb * node.total_length / length_sq(sp.p - node.bounds.center());
}

// stochastic two-mode traversal (edge_tree.cpp:511-652)
template <bool DIR, bool CONE>
void sample_edge(int nid, float nbb, const Scene &sc, const EdgeTree &t, const V3f &wi, const Isect &is,
                 const SPoint<float> &sp, float dl, float sl, const Cone &cone, std::vector<EdgeW> &out, float cpmf,
                 float apmf, Sampler &rng) {
    if (nbb <= 0.f) return;
    const EdgeNode &node = t.nodes[nid];
    if (node.nprims > 0) {
        float w = CONE ? cpmf / (cpmf * cpmf + apmf * apmf) : apmf / (cpmf * cpmf + apmf * apmf);
        for (int i = 0; i < node.nprims; i++) {
            const Edge &e = t.edges[node.offset + i];
            if (is_silhouette(sc, sp.p, e)) out.push_back(EdgeW{e, w, ((CONE ? 0 : 1) << 27) | (node.offset + i)});
        }
        return;
    }
    const EdgeNode &L = t.nodes[nid + 1], &Rn = t.nodes[node.offset];
    bool all_split = nbb > 1.f || node.bounds.inside(sp.p);
    bool lcs = true, rcs = true;
    if (DIR) {
        lcs = contains_silhouette(L, sp.p);
        rcs = contains_silhouette(Rn, sp.p);
    }
    float lbb = lcs ? bsdf_bound(sc, L, wi, is, sp, dl, sl) : 0.f;
    float rbb = rcs ? bsdf_bound(sc, Rn, wi, is, sp, dl, sl) : 0.f;
    float il = lcs ? node_importance(L, lbb, sp) : 0.f;
    float ir = rcs ? node_importance(Rn, rbb, sp) : 0.f;
    if (il + ir <= 1e-10f) return;
    bool lhc = box_cone(L.bounds, cone), rhc = box_cone(Rn.bounds, cone);
    bool cone_split = all_split || (lhc && rhc && lcs && rcs && cone.cos_angle > 0.95f);
    float ilc = lhc ? il : 0.f, irc = rhc ? ir : 0.f;
    if (CONE && ilc + irc <= 1e-10f) return;
    float plc = 0.f, prc = 0.f, pla = 0.f, pra = 0.f;
    if (cone_split) plc = prc = 1.f;
    else if (ilc + irc > 1e-10f) { plc = ilc / (ilc + irc); prc = 1.f - plc; }
    if (all_split) pla = pra = 1.f;
    else { pla = il / (il + ir); pra = 1.f - pla; }
    bool split = CONE ? cone_split : all_split;
    if (split) {
        if (lcs) sample_edge<DIR, CONE>(nid + 1, lbb, sc, t, wi, is, sp, dl, sl, cone, out, plc * cpmf, pla * apmf, rng);
        if (rcs) sample_edge<DIR, CONE>(node.offset, rbb, sc, t, wi, is, sp, dl, sl, cone, out, prc * cpmf, pra * apmf, rng);
    } else {
        float u = rng.node(CONE ? 0 : 1, nid);
        bool left = CONE ? u < plc : u < pla;
        if (left) sample_edge<DIR, CONE>(nid + 1, lbb, sc, t, wi, is, sp, dl, sl, cone, out, plc * cpmf, pla * apmf, rng);
        else sample_edge<DIR, CONE>(node.offset, rbb, sc, t, wi, is, sp, dl, sl, cone, out, prc * cpmf, pra * apmf, rng);
    }
}

template <bool DIR>
void sample_tree(const Scene &sc, const EdgeTree &t, const V3f &wi, const Isect &is, const SPoint<float> &sp,
                 const Cone &cone, float pmf, std::vector<EdgeW> &out, Sampler &rng) {
    if (t.nodes.empty()) return;
    const Material &mat = sc.mats[sc.shapes[is.shape].mat];
    float dl = luminance(get_diffuse<float>(mat, sp.uv, nullptr));
    float sl = luminance(get_specular<float>(mat, sp.uv, nullptr));
    float b = bsdf_bound(sc, t.nodes[0], wi, is, sp, dl, sl);
    sample_edge<DIR, true>(0, b, sc, t, wi, is, sp, dl, sl, cone, out, pmf, pmf, rng);
    sample_edge<DIR, false>(0, b, sc, t, wi, is, sp, dl, sl, cone, out, pmf, pmf, rng);
}

// edge_tree.cpp:685-725
inline void sample_shading_edges(const Scene &sc, const V3f &wi, const Isect &is, const SPoint<float> &sp,
                                 const Cone &cone, std::vector<EdgeW> &out, Sampler &rng) {
    if (dot(wi, sp.f[2]) < 0.f) return;
    if (sc.nrm_tree.nodes.empty()) {
        sample_tree<false>(sc, sc.sil_tree, wi, is, sp, cone, 1.f, out, rng);
        return;
    }
    if (sc.sil_tree.nodes.empty()) {
        sample_tree<true>(sc, sc.nrm_tree, wi, is, sp, cone, 1.f, out, rng);
        return;
    }
    float ni = sc.nrm_tree.nodes[0].total_length, si = sc.sil_tree.nodes[0].total_length;
    float np = ni / (ni + si), spm = si / (ni + si);
    float u = rng.next();
    if (u < np) sample_tree<true>(sc, sc.nrm_tree, wi, is, sp, cone, np, out, rng);
    else sample_tree<false>(sc, sc.sil_tree, wi, is, sp, cone, spm, out, rng);
}

inline M3 ltc_matrix(const Scene &sc, int mi, const SPoint<float> &sp, const V3f &wi) {
    float r = get_roughness<float>(sc.mats[mi], sp.uv, nullptr);
    float ct = dot(wi, sp.f[2]);
    float th = m_acos(ct);
    int rid = int(r * (128 - 1));
    int tid = int((th / (M_PI / 2.f)) * (128 - 1));
    rid = std::max(0, std::min(127, rid));
    tid = std::max(0, std::min(127, tid));
    const float *m = (sc.mats[mi].model == DR_MICROFACET_GGX ? sc.ltc_ggx : sc.ltc) + 9 * (rid + tid * 128);
    M3 r3;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) r3(i, j) = m[3 * i + j];
    return r3;
}

struct EdgeResult { V3f dp{0, 0, 0}, dv0{0, 0, 0}, dv1{0, 0, 0}; };

// Density with which a lobe's line sample (delta_ray.cpp:107-160, in the
// lobe's space minv) picks the edge point at offset q from the shading point,
// per unit of a parameter l of the edge with dq/dl = q_l; 0 below the lobe's
// horizon.  Project addition (DR_FLAG_EDGE_LOBE_MIS), no reference counterpart.
inline float lobe_line_density(const M3 &minv, const V3f &d0, const V3f &d1, const V3f &q, const V3f &q_l) {
    V3f a = minv * d0, b = minv * d1;
    if (a.z <= 0.f && b.z <= 0.f) return 0.f;
    if (a.z < 0.f) a = (a * b.z - b * a.z) / (b.z - a.z);
    if (b.z < 0.f) b = (a * b.z - b * a.z) / (b.z - a.z);
    V3f vod = b - a;
    if (abs_sum(vod) < 1e-10f) return 0.f;
    V3f wt = normalize(vod);
    float l0 = dot(a, wt), l1 = dot(b, wt);
    V3f vo = a - l0 * wt;
    float d = length(vo);
    auto I = [&](float l) {
        return (l / (d * (d * d + l * l)) + m_atan(l / d) / (d * d)) * vo.z + (l * l / (d * (d * d + l * l))) * wt.z;
    };
    float norm = I(l1) - I(l0);
    if (norm <= 1e-10f) return 0.f;
    V3f y = minv * q;
    if (y.z < 0.f) return 0.f;
    float l = dot(y, wt);
    float ds = d * d + l * l;
    float p = 2.f * d * (vo + l * wt).z / (norm * ds * ds);
    return p > 0.f ? p * length(minv * q_l) : 0.f;
}

// secondary edge sample (delta_ray.cpp:45-365)
inline EdgeResult shading_edge_sample(const Scene &sc, const EdgeSample &es, const Edge &edge, const LightSample &ls,
                                      const std::vector<SecondarySample> &ss, const V3f &wi, const Isect &sis,
                                      const SPoint<float> &sp, const V3f &weight, const V3f &d_color,
                                      bool direct_only) {
    EdgeResult none;
    if (!sis.valid()) return none;
    if (!is_silhouette(sc, sp.p, edge)) return none;
    V3f v0 = sc.ev0(edge), v1 = sc.ev1(edge);
    if (abs_sum(v1 - v0) == 1e-10f) return none;
    int mi = sc.shapes[sis.shape].mat;
    const Material &mat = sc.mats[mi];
    V3f kd = get_diffuse<float>(mat, sp.uv, nullptr), ks = get_specular<float>(mat, sp.uv, nullptr);
    float dw = luminance(kd), sw = luminance(ks), ws = dw + sw;
    if (ws <= 0.f) return none;
    float dpmf = dw / ws, spmf = sw / ws;
    V3f n = sp.f[2];
    V3f fx = normalize(wi - n * dot(wi, n));
    V3f fy = cross(n, fx);
    M3 frame = m3_rows(fx, fy, n);
    M3 m, minv;
    float mpmf;
    if (es.bsdf_component <= dpmf) {
        minv = frame;
        m = inverse(minv);
        mpmf = dpmf;
    } else {
        minv = inverse(ltc_matrix(sc, mi, sp, wi)) * frame;
        m = inverse(minv);
        mpmf = spmf;
    }
    V3f a = minv * (v0 - sp.p), b = minv * (v1 - sp.p);
    if (a.z <= 0.f && b.z <= 0.f) return none;
    if (a.z < 0.f) a = (a * b.z - b * a.z) / (b.z - a.z);
    if (b.z < 0.f) b = (a * b.z - b * a.z) / (b.z - a.z);
    V3f vod = b - a;
    if (abs_sum(vod) < 1e-10f) return none;
    V3f wt = normalize(vod);
    float l0 = dot(a, wt), l1 = dot(b, wt);
    V3f vo = a - l0 * wt;
    float d = length(vo);
    auto I = [&](float l) {
        return (l / (d * (d * d + l * l)) + m_atan(l / d) / (d * d)) * vo.z + (l * l / (d * (d * d + l * l))) * wt.z;
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
    if (lb > ub) std::swap(lb, ub);
    float l = 0.5f * (lb + ub);
    for (int it = 0; it < 20; it++) {
        if (!(l >= lb && l <= ub)) l = 0.5f * (lb + ub);
        float value = cdf(l) - es.u;
        if (std::fabs(value) < 1e-5f || it == 19) break;
        if (value > 0.f) ub = l; else lb = l;
        l -= value / pdf(l);
    }
    if (pdf(l) <= 0.f) return none;
    V3f sample_p = m * (vo + l * wt);
    V3f split_n = normalize(cross(v0 - sp.p, v1 - sp.p));
    float delta = 1e-3f * length(sample_p);
    V3f sdir = normalize(sample_p);
    V3f rdir = normalize(sdir + delta * split_n), ldir = normalize(sdir - delta * split_n);
    auto hr = intersect<float>(sc, Ray<float>{sp.p, rdir}, nullptr);
    auto hl = intersect<float>(sc, Ray<float>{sp.p, ldir}, nullptr);
    const Isect &ir = hr.first, &il = hl.first;
    bool rc = ir.shape == edge.shape && (ir.tri == edge.f0 || ir.tri == edge.f1);
    bool lc = il.shape == edge.shape && (il.tri == edge.f0 || il.tri == edge.f1);
    if ((!rc && !lc) || (rc && lc) || (ir.shape == sis.shape && ir.tri == sis.tri) ||
        (il.shape == sis.shape && il.tri == sis.tri))
        return none;
    V3f eb = bsdf<float>(sc, mi, sp, wi, sdir, nullptr);
    if (sum(eb) < 1e-6f) return none;
    V3f shr{0, 0, 0}, shl{0, 0, 0};
    if (!direct_only) {
        shr = shade<float>(sc, -sdir, ir, hr.second, ls, ss, false, nullptr, nullptr);
        shl = shade<float>(sc, -sdir, il, hl.second, ls, ss, false, nullptr, nullptr);
        auto clamp_gi = [&](V3f &s, const Isect &is2, const SPoint<float> &p2) {
            if (!is2.valid()) return;
            V3f dir = p2.p - sp.p;
            float d2 = length_sq(dir);
            if (d2 > 0.f) {
                s = s / std::max(d2, 1e-2f);
                s = s * std::fabs(dot(normalize(dir), p2.ng));
            } else {
                s = V3f{0, 0, 0};
            }
        };
        clamp_gi(shr, ir, hr.second);
        clamp_gi(shl, il, hl.second);
    }
    V3f er = eval<float>(sc, wi, sis, sp, ir, hr.second, nullptr) + mul(eb, shr);
    V3f el = eval<float>(sc, wi, sis, sp, il, hl.second, nullptr) + mul(eb, shl);
    auto too_close = [&](const Isect &is2, const SPoint<float> &p2) {
        if (!is2.valid()) return false;
        V3f dir = p2.p - sp.p;
        return length(dir) * std::fabs(dot(normalize(dir), p2.ng)) < 1e-3f;
    };
    if (too_close(ir, hr.second) || too_close(il, hl.second)) return none;
    EdgeResult res;
    // DR_FLAG_EDGE_LOBE_MIS: balance heuristic over the two lobes
    float q_mix = mpmf * pdf(l);
    if (sc.edge_lobe_mis) {
        bool sel_diffuse = es.bsdf_component <= dpmf;
        float opmf = sel_diffuse ? spmf : dpmf;
        if (opmf > 0.f) {
            M3 ominv = sel_diffuse ? inverse(ltc_matrix(sc, mi, sp, wi)) * frame : frame;
            q_mix += opmf * lobe_line_density(ominv, v0 - sp.p, v1 - sp.p, sample_p, m * wt);
        }
    }
    auto accum = [&](const SPoint<float> &lp, const V3f &ev) {
        M3 nj = normalize_jacobian(sample_p);
        M3 ij = intersect_jacobian(sdir, lp.p, lp.ng);
        float line_j = length(((ij * nj) * m) * wt) / q_mix;
        V3f p = sp.p, x = lp.p;
        V3f d0 = v0 - p, d1 = v1 - p;
        float dirac_j = length(cross(d0, d1));
        float w = line_j / dirac_j;
        V3f dp = w * (cross(d1, d0) + cross(x - p, d1) + cross(d0, x - p));
        V3f dv0 = w * cross(d1, x - p);
        V3f dv1 = w * cross(x - p, d0);
        float we = dot(mul(ev, weight), d_color);
        res.dp = res.dp + dp * we;
        res.dv0 = res.dv0 + dv0 * we;
        res.dv1 = res.dv1 + dv1 * we;
    };
    if (ir.valid() && abs_sum(er) > 0.f) accum(hr.second, er);
    if (il.valid() && abs_sum(el) > 0.f) accum(hl.second, -el);
    return res;
}

struct PrimaryEdgeResult {
    bool ok = false;
    float sx = -1.f, sy = -1.f;
    Edge edge;
    V3f dv0{0, 0, 0}, dv1{0, 0, 0};
    float d_w2c[16];
};

// primary edge sample (delta_ray.cpp:377-557)
inline PrimaryEdgeResult primary_edge_sample(const Scene &sc, const EdgeSample &es, const Edge &edge,
                                             const LightSample &ls, const std::vector<SecondarySample> &ss,
                                             const float *d_image, int W, int H, float weight) {
    PrimaryEdgeResult none;
    const Camera &cam = sc.cam;
    V3f v0 = sc.ev0(edge), v1 = sc.ev1(edge);
    V2f s0, s1;
    if (!project(cam, v0, v1, &s0, &s1)) return none;
    V3f d0 = unproject(cam, s0), d1 = unproject(cam, s1);
    V3f vd = d1 - d0;
    float t = es.u;
    V3f l0 = xfm_point(cam.w2c, v0), l1 = xfm_point(cam.w2c, v1);
    V3f ept3 = d0 + t * vd;
    V3f elocal = l0 + t * l1;  // as in the reference (delta_ray.cpp:403)
    V2f ept = project_local(cam, ept3);
    if (!in_screen(cam, ept)) return none;
    int xi = int(ept.x * W), yi = int(ept.y * H);
    const float *dc = d_image + 3 * (yi * W + xi);
    V3f d_color{dc[0], dc[1], dc[2]};
    float delta = 1e-4f * length(elocal);
    V3f split_n = normalize(cross(d0, d1));
    V3f rdir = normalize(ept3 + delta * split_n);
    V2f rpt = project_local(cam, rdir);
    TCam<float> tc = make_tcam<float>(cam, nullptr);
    Ray<float> rray = sample_primary(tc, rpt);
    auto hr = intersect<float>(sc, rray, nullptr);
    V3f ldir = normalize(ept3 - delta * split_n);
    V2f lpt = project_local(cam, ldir);
    Ray<float> lray = sample_primary(tc, lpt);
    auto hl = intersect<float>(sc, lray, nullptr);
    bool rc = hr.first.shape == edge.shape && (hr.first.tri == edge.f0 || hr.first.tri == edge.f1);
    bool lc = hl.first.shape == edge.shape && (hl.first.tri == edge.f0 || hl.first.tri == edge.f1);
    if (!rc && !lc) return none;
    V3f rcol = shade<float>(sc, -rray.d, hr.first, hr.second, ls, ss, true, nullptr, nullptr);
    V3f lcol = shade<float>(sc, -lray.d, hl.first, hl.second, ls, ss, true, nullptr, nullptr);
    V3f diff = (rcol - lcol) * weight;
    V3f xdiff = diff, ydiff = diff;
    if (lpt.x > rpt.x) xdiff = -xdiff;
    if (lpt.y > rpt.y) ydiff = -ydiff;
    V3f edir = unproject(cam, ept);
    auto dv0d = d_unproject(cam, s0), dv1d = d_unproject(cam, s1), ded = d_unproject(cam, ept);
    V3f c01 = cross(d0, d1);
    float dadx = dot(ded.first, c01), dady = dot(ded.second, c01);
    float a0x = std::fabs(dot(cross(d1, edir), dv0d.first));
    float a0y = std::fabs(dot(cross(d1, edir), dv0d.second));
    float a1x = std::fabs(dot(cross(edir, d0), dv1d.first));
    float a1y = std::fabs(dot(cross(edir, d0), dv1d.second));
    float dirac_j = 1.f / std::sqrt(dadx * dadx + dady * dady);
    V3f ept3d = d0 + (t + delta) * vd;
    V2f eptd = project_local(cam, ept3d);
    V2f dd{(eptd.x - ept.x) / delta, (eptd.y - ept.y) / delta};
    float line_j = std::sqrt(dd.x * dd.x + dd.y * dd.y);
    float jac = line_j * dirac_j;
    float dv0x = dot(-xdiff * a0x * jac, d_color), dv0y = dot(-ydiff * a0y * jac, d_color);
    float dv1x = dot(-xdiff * a1x * jac, d_color), dv1y = dot(-ydiff * a1y * jac, d_color);
    // screen -> world by forward differences (delta_ray.cpp:490-542)
    const float h = 1e-3f;
    V2f p0[6], p1[6];
    V3f off[3] = {V3f{h, 0, 0}, V3f{0, h, 0}, V3f{0, 0, h}};
    for (int k = 0; k < 3; k++) {
        if (!project(cam, v0 + off[k], v1, &p0[k], &p1[k])) return none;
    }
    for (int k = 0; k < 3; k++) {
        if (!project(cam, v0, v1 + off[k], &p0[3 + k], &p1[3 + k])) return none;
    }
    PrimaryEdgeResult r;
    r.ok = true;
    r.sx = ept.x;
    r.sy = ept.y;
    r.edge = edge;
    for (int k = 0; k < 3; k++) {
        V2f a0{(p0[k].x - s0.x) / h, (p0[k].y - s0.y) / h}, a1{(p1[k].x - s1.x) / h, (p1[k].y - s1.y) / h};
        r.dv0[k] = dv0x * a0.x + dv0y * a0.y + dv1x * a1.x + dv1y * a1.y;
        V2f b0{(p0[3 + k].x - s0.x) / h, (p0[3 + k].y - s0.y) / h};
        V2f b1{(p1[3 + k].x - s1.x) / h, (p1[3 + k].y - s1.y) / h};
        r.dv1[k] = dv0x * b0.x + dv0y * b0.y + dv1x * b1.x + dv1y * b1.y;
    }
    std::memset(r.d_w2c, 0, sizeof(r.d_w2c));
    d_project(cam, v0, v1, dv0x, dv0y, dv1x, dv1y, r.d_w2c);
    return r;
}

// ===================================================================
// Scene construction (scene.cpp:19-136, edge_tree.cpp:263-316)
// ===================================================================
struct GradLayout {
    size_t total = 64;
    std::vector<size_t> mat, vtx, nrm, light;
};

inline void build_scene(Scene &sc, const dr_scene_desc *d, const float *ltc_default, const int *shape_rank = nullptr) {
    if (shape_rank) sc.shape_rank.assign(shape_rank, shape_rank + d->num_shapes);
    const dr_camera_desc &c = d->camera;
    std::memcpy(sc.cam.c2w.m, c.cam_to_world, 64);
    std::memcpy(sc.cam.w2c.m, c.world_to_cam, 64);
    std::memcpy(sc.cam.s2c.m, c.sample_to_cam, 64);
    std::memcpy(sc.cam.c2s.m, c.cam_to_sample, 64);
    sc.cam.fov = c.fov_factor;
    sc.cam.aspect = c.aspect_ratio;
    sc.cam.clip_near = c.clip_near;
    sc.cam.fisheye = c.fisheye != 0;
    for (int i = 0; i < d->num_materials; i++) {
        const dr_material_desc &m = d->materials[i];
        Material mm;
        mm.diffuse = Tex{m.diffuse, m.diffuse_w, m.diffuse_h, 3};
        mm.specular = Tex{m.specular, m.specular_w, m.specular_h, 3};
        mm.roughness = Tex{m.roughness, m.roughness_w, m.roughness_h, 1};
        std::memcpy(mm.uv_d, m.diffuse_uv_scale, 8);
        std::memcpy(mm.uv_s, m.specular_uv_scale, 8);
        std::memcpy(mm.uv_r, m.roughness_uv_scale, 8);
        mm.two_sided = m.two_sided != 0;
        mm.model = m.microfacet;
        sc.mats.push_back(mm);
    }
    for (int i = 0; i < d->num_shapes; i++) {
        const dr_shape_desc &s = d->shapes[i];
        Shape sh;
        sh.v = s.vertices;
        sh.nv = s.num_vertices;
        sh.idx = s.indices;
        sh.nt = s.num_triangles;
        sh.uv = s.uvs;
        sh.n = s.normals;
        sh.mat = s.material_id;
        sc.shapes.push_back(sh);
    }
    sc.ltc = d->ltc_table ? d->ltc_table : ltc_default;
    sc.ltc_ggx = d->ltc_table_ggx ? d->ltc_table_ggx : ltc_default;
    // lights (scene.cpp:26-52)
    std::vector<float> imp;
    for (int i = 0; i < d->num_lights; i++) {
        Light L;
        L.shape = d->lights[i].shape_id;
        std::memcpy(L.I, d->lights[i].intensity, 12);
        sc.lights.push_back(L);
        sc.shapes[L.shape].light = i;
        float lum = luminance(V3f{L.I[0], L.I[1], L.I[2]});
        imp.push_back(lum);
        sc.total_light_intensity += lum;
        const Shape &sh = sc.shapes[L.shape];
        std::vector<float> areas;
        AABB b;
        float asum = 0.f;
        for (int t = 0; t < sh.nt; t++) {
            auto ind = sh.ind(t);
            V3f a = sh.vtx(ind[0]), bb = sh.vtx(ind[1]), cc = sh.vtx(ind[2]);
            float ar = 0.5f * length(cross(bb - a, cc - a));
            asum += ar;
            areas.push_back(ar);
            b.add(a);
            b.add(bb);
            b.add(cc);
        }
        sc.light_tri.emplace_back(areas.data(), (int)areas.size());
        sc.light_area.push_back(asum);
        sc.light_bounds.push_back(b);
    }
    if (!imp.empty()) sc.light_sel = Dist1D(imp.data(), (int)imp.size());
    // edges, keyed (shape, min v, max v) in map order (scene.cpp:54-97)
    std::map<std::tuple<int, int, int>, Edge> emap;
    for (int si = 0; si < (int)sc.shapes.size(); si++) {
        const Shape &sh = sc.shapes[si];
        for (int t = 0; t < sh.nt; t++) {
            auto ind = sh.ind(t);
            auto add = [&](int a, int b) {
                if (a > b) std::swap(a, b);
                auto key = std::make_tuple(sc.shape_rank.empty() ? si : sc.shape_rank[si], a, b);
                auto it = emap.find(key);
                if (it == emap.end()) emap[key] = Edge{si, a, b, t, -1};
                else it->second.f1 = t;
            };
            add(ind[0], ind[1]);
            add(ind[1], ind[2]);
            add(ind[2], ind[0]);
        }
    }
    std::vector<Edge> edges;
    for (auto &kv : emap) {
        const Edge &e = kv.second;
        if (abs_sum(sc.ev0(e) - sc.ev1(e)) < 1e-10f) continue;
        if (e.f1 != -1) {
            float ang = std::fabs(dot(sc.shapes[e.shape].face_normal(e.f0), sc.shapes[e.shape].face_normal(e.f1)));
            if (ang == 1.f || ang == -1.f) continue;
        }
        edges.push_back(e);
    }
    // primary edges: camera silhouettes with clipped screen length (edge_tree.cpp:263-294)
    std::vector<float> lens;
    V3f org = xfm_point(sc.cam.c2w, V3f{0.f, 0.f, 0.f});
    for (const Edge &e : edges) {
        V2f a, b;
        float dist = 0.f;
        if (project(sc.cam, sc.ev0(e), sc.ev1(e), &a, &b)) {
            V2f ca, cb;
            if (clip_line(a, b, &ca, &cb)) dist = std::sqrt((cb.x - ca.x) * (cb.x - ca.x) + (cb.y - ca.y) * (cb.y - ca.y));
        }
        if (!is_silhouette(sc, org, e)) dist = 0.f;
        if (dist > 0.f) {
            sc.primary_edges.push_back(e);
            lens.push_back(dist);
        }
    }
    if (!lens.empty()) sc.primary_dist = Dist1D(lens.data(), (int)lens.size());
    std::vector<Edge> sil, nrm;
    for (const Edge &e : edges) {
        if (e.f0 == -1 || e.f1 == -1 || !sc.shapes[e.shape].n) sil.push_back(e);
        else nrm.push_back(e);
    }
    sc.sil_tree = build_edge_tree<false>(sc, sil);
    sc.nrm_tree = build_edge_tree<true>(sc, nrm);
    // ray casting structure: the same CPU BVH the compiled reference uses
    for (int si = 0; si < (int)sc.shapes.size(); si++) {
        const Shape &sh = sc.shapes[si];
        for (int t = 0; t < sh.nt; t++) {
            auto ind = sh.ind(t);
            drshim::Tri tr;
            float *dst[3] = {tr.v0, tr.v1, tr.v2};
            for (int k = 0; k < 3; k++) std::memcpy(dst[k], sh.v + 3 * ind[k], 12);
            tr.geom = si;
            tr.prim = t;
            sc.bvh.tris.push_back(tr);
        }
    }
    if (!sc.bvh.tris.empty()) drshim::build_node(sc.bvh, 0, (int)sc.bvh.tris.size());
}

inline GradLayout grad_layout(const dr_scene_desc *d) {
    GradLayout g;
    size_t o = 64;
    for (int i = 0; i < d->num_materials; i++) {
        const dr_material_desc &m = d->materials[i];
        g.mat.push_back(o);
        o += m.diffuse_w ? (size_t)m.diffuse_w * m.diffuse_h * 3 : 3;
        g.mat.push_back(o);
        o += m.specular_w ? (size_t)m.specular_w * m.specular_h * 3 : 3;
        g.mat.push_back(o);
        o += m.roughness_w ? (size_t)m.roughness_w * m.roughness_h : 1;
    }
    for (int i = 0; i < d->num_shapes; i++) {
        g.vtx.push_back(o);
        o += 3 * (size_t)d->shapes[i].num_vertices;
        if (d->shapes[i].normals) {
            g.nrm.push_back(o);
            o += 3 * (size_t)d->shapes[i].num_vertices;
        } else {
            g.nrm.push_back((size_t)-1);
        }
    }
    for (int i = 0; i < d->num_lights; i++) {
        g.light.push_back(o);
        o += 3;
    }
    g.total = o;
    return g;
}

// ===================================================================
// Per-sample render with gradients (delta_ray.cpp:694-1005) and the
// scatter of its derivatives (delta_ray.cpp:1251-1323,1334-1459)
// ===================================================================
struct Accum {
    std::vector<double> g;  // flat gradient layout
    long long edges = 0, points = 0;
};

// Where a pixel sample's edge draws come from.
struct StreamPlan {
    int mode;  // 0 reference order (one sampler), 1 Philox streams
    uint64_t seed;
    uint64_t sample_id;
    Sampler *main;
};

inline void scatter_material(const Scene &sc, const GradLayout &L, const MatRec &mr, Accum &acc) {
    const Material &m = sc.mats[mr.mat];
    const Tex *tx[3] = {&m.diffuse, &m.specular, &m.roughness};
    const TexRec *tr[3] = {&mr.d, &mr.s, &mr.r};
    for (int k = 0; k < 3; k++) {
        int ch = k == 2 ? 1 : 3;
        size_t base = L.mat[3 * mr.mat + k];
        if (tx[k]->w == 0) {
            for (int c = 0; c < ch; c++) {
                int id = tr[k]->t[0][c];
                float a = id >= 0 ? g_tape->adj[id] : 0.f;
                if (k == 2 && !std::isfinite(a)) continue;  // delta_ray.cpp:849-851
                acc.g[base + c] += a;
            }
        } else if (tr[k]->textured) {
            // texel adjoints land as in delta_ray.cpp:1366-1383: t00 -> (yc, xc),
            // t01 -> (yc, xf), t10 -> (yf, xc), t11 -> (yf, xf)
            int xf = tr[k]->xi, yf = tr[k]->yi;
            int xc = modulo(xf + 1, tx[k]->w), yc = modulo(yf + 1, tx[k]->h);
            int ys[4] = {yc, yc, yf, yf}, xs[4] = {xc, xf, xc, xf};
            for (int q = 0; q < 4; q++)
                for (int c = 0; c < ch; c++) {
                    int id = tr[k]->t[q][c];
                    float a = id >= 0 ? g_tape->adj[id] : 0.f;
                    acc.g[base + (size_t)(ys[q] * tx[k]->w + xs[q]) * ch + c] += a;
                }
        }
    }
}

inline float adj_of(int id) { return id >= 0 ? g_tape->adj[id] : 0.f; }

thread_local int g_parts = 7;  // test knob: 1 continuous, 2 secondary edges, 4 primary edges

V3f render_pixel_sample(const Scene &sc, const GradLayout &L, int W, int H, int xi, int yi, float sub_x, float sub_y,
                        int spp, int B, const V3f &d_color, bool derivs, StreamPlan &sp_plan, Accum &acc,
                        int dp_mode) {
    float sw = 1.f / spp;
    Sampler &rng = *sp_plan.main;
    if (!derivs || is_zero(d_color)) {
        // render_sample_fast (delta_ray.cpp:640-692)
        TCam<float> cam = make_tcam<float>(sc.cam, nullptr);
        V2f s{float((xi + sub_x) / W), float((yi + sub_y) / H)};
        Ray<float> ray = sample_primary(cam, s);
        if (abs_sum(ray.d) == 0.f) return V3f{0, 0, 0};
        auto hit = intersect<float>(sc, ray, nullptr);
        if (!hit.first.valid()) return V3f{0, 0, 0};
        LightSample ls = draw_light(rng);
        std::vector<SecondarySample> ss;
        for (int b = 0; b < B; b++) ss.push_back(draw_secondary(rng));
        V3f c = shade<float>(sc, -ray.d, hit.first, hit.second, ls, ss, true, nullptr, nullptr);
        return c * sw;
    }
    Tape &tape = *g_tape;
    tape.clear();
    int cam_ids[16];
    TCam<AD> cam = make_tcam<AD>(sc.cam, cam_ids);
    V2<AD> s{AD(float((xi + sub_x) / W)), AD(float((yi + sub_y) / H))};
    Ray<AD> ray = sample_primary(cam, s);
    if (abs_sum(fv(ray.d)) == 0.f) return V3f{0, 0, 0};
    Records R;
    auto hit = intersect<AD>(sc, ray, &R.isect);
    if (!hit.first.valid()) return V3f{0, 0, 0};
    LightSample ls = draw_light(rng);
    std::vector<SecondarySample> ss;
    for (int b = 0; b < B; b++) ss.push_back(draw_secondary(rng));
    std::vector<SecondaryPoint<AD>> spts;
    V3<AD> col = shade<AD>(sc, -ray.d, hit.first, hit.second, ls, ss, true, &spts, &R) * sw;
    V3f color = fv(col);
    // first sweep: the image adjoint (delta_ray.cpp:771-866)
    tape.zero();
    for (int c = 0; c < 3; c++)
        if (col[c].id >= 0) tape.adj[col[c].id] = d_color[c];
    tape.sweep();
    std::vector<double> g_skip;
    if (!(g_parts & 1)) g_skip.assign(acc.g.size(), 0.0);
    double *g = (g_parts & 1) ? acc.g.data() : g_skip.data();
    for (int i = 0; i < 16; i++) g[i] += adj_of(cam_ids[i]);
    auto scatter_isect = [&](bool with_normals) {
        for (const IsectRec &ir : R.isect) {
            const Shape &sh = sc.shapes[ir.shape];
            auto ind = sh.ind(ir.tri);
            for (int k = 0; k < 3; k++)
                for (int a = 0; a < 3; a++) g[L.vtx[ir.shape] + 3 * ind[k] + a] += adj_of(ir.v[k][a]);
            if (with_normals && ir.has_n && L.nrm[ir.shape] != (size_t)-1) {
                // the reference adds the first vertex's normal adjoint to all
                // three vertices (delta_ray.cpp:1261-1269)
                for (int k = 0; k < 3; k++)
                    for (int a = 0; a < 3; a++) g[L.nrm[ir.shape] + 3 * ind[k] + a] += adj_of(ir.n[0][a]);
            }
        }
    };
    scatter_isect(true);
    if (g_parts & 1) {
        for (const MatRec &mr : R.mat) scatter_material(sc, L, mr, acc);
        for (const LightRec &lr : R.light)
            for (int c = 0; c < 3; c++) g[L.light[lr.light] + c] += adj_of(lr.I[c]);
    }
    g = acc.g.data();
    if (!(g_parts & 2)) return color;
    // secondary edges (delta_ray.cpp:868-974)
    struct DP { int id[3]; V3f dp; };
    std::vector<DP> dps;
    int li = sc.light_sel.sample_discrete(ls.sel);
    for (int k = 0; k < (int)spts.size(); k++) {
        const SecondaryPoint<AD> &P = spts[k];
        SPoint<float> psp = fsp(P.sp);
        std::unique_ptr<PhiloxSampler> pstream;
        Sampler *prng = &rng;
        if (sp_plan.mode == 1) {
            pstream.reset(new PhiloxSampler(sp_plan.seed, kEdgePoint, sp_plan.sample_id, (uint32_t)k));
            prng = pstream.get();
        }
        EdgeSample es = draw_edge(*prng);
        const AABB &lb = sc.light_bounds[li];
        V3f bc = (lb.lo + lb.hi) / 2.f;
        float br = length(lb.hi - bc);
        V3f dl = bc - psp.p;
        float tan_a = br / length(dl);
        float cos_a = tan_a <= 1.f ? 1.f / std::sqrt(tan_a * tan_a + 1.f) : 0.f;
        Cone cone{psp.p, normalize(dl), cos_a};
        std::vector<EdgeW> edges;
        sample_shading_edges(sc, P.wi, P.isect, psp, cone, edges, *prng);
        acc.points++;
        acc.edges += (long long)edges.size();
        for (int j = 0; j < (int)edges.size(); j++) {
            const EdgeW &ew = edges[j];
            if (ew.w == 0.f) continue;
            std::unique_ptr<PhiloxSampler> estream;
            Sampler *erng = &rng;
            if (sp_plan.mode == 1) {
                estream.reset(new PhiloxSampler(sp_plan.seed, kEdgeItem, sp_plan.sample_id,
                                                ((uint32_t)k << 28) | (uint32_t)ew.key));
                erng = estream.get();
            }
            LightSample els = draw_light(*erng);
            std::vector<SecondarySample> ess;
            for (int b = 0; b < B - P.bounce - 1; b++) ess.push_back(draw_secondary(*erng));
            V3f weight = P.throughput * (sw * ew.w);
            EdgeResult er = shading_edge_sample(sc, es, ew.e, els, ess, P.wi, P.isect, psp, weight, d_color, B == 1);
            if (!is_zero(er.dp)) dps.push_back(DP{{P.sp.p.x.id, P.sp.p.y.id, P.sp.p.z.id}, er.dp});
            if (!is_zero(er.dv0) || !is_zero(er.dv1)) {
                size_t base = L.vtx[ew.e.shape];
                for (int a = 0; a < 3; a++) {
                    g[base + 3 * ew.e.v0 + a] += er.dv0[a];
                    g[base + 3 * ew.e.v1 + a] += er.dv1[a];
                }
            }
        }
    }
    // second sweep: edge position derivatives pushed back along the path
    // (delta_ray.cpp:975-1002); the reference sets (not adds) each adjoint
    if (!dps.empty()) {
        tape.zero();
        for (const DP &d : dps)
            for (int a = 0; a < 3; a++)
                if (d.id[a] >= 0) {
                    if (dp_mode == DR_DP_SUM) tape.adj[d.id[a]] += d.dp[a];
                    else tape.adj[d.id[a]] = d.dp[a];
                }
        tape.sweep();
        for (int i = 0; i < 16; i++) g[i] += adj_of(cam_ids[i]);
        scatter_isect(false);
    }
    return color;
}

}  // namespace oracle

using namespace oracle;

// Runs body(i, worker) for i in [0, n) on `workers` threads (dynamic chunks of 1).
template <typename F> static void parallel_loop(long long n, int workers, long long chunk, F body) {
    std::atomic<long long> next(0);
    auto run = [&](int w) {
        while (true) {
            long long i0 = next.fetch_add(chunk);
            if (i0 >= n) break;
            long long i1 = std::min(n, i0 + chunk);
            for (long long i = i0; i < i1; i++) body(i, w);
        }
    };
    std::vector<std::thread> th;
    for (int w = 1; w < workers; w++) th.emplace_back(run, w);
    run(0);
    for (auto &t : th) t.join();
}

extern "C" {

int dro_render_parts(const dr_scene_desc *desc, const dr_render_desc *rd, int rng_mode, int cores, const float *d_image,
                     float *image, float *grad, long long *stats, int nthreads, const int *shape_rank, int parts);

// rng_mode 0: the reference's mt19937 scheme with `cores` edge threads;
// shape_rank (may be NULL) orders shapes in the edge map as the reference's
// Shape* keys did;
// rng_mode 1: the product's Philox streams and its reproducible transcendental
// functions (rng_mode 2: the same streams with the host libm).  d_image == NULL renders forward
// only.  grad (flat layout) may be NULL for forward.  stats[0..1] receive the
// number of secondary points and sampled edges.
int dro_render(const dr_scene_desc *desc, const dr_render_desc *rd, int rng_mode, int cores, const float *d_image,
               float *image, float *grad, long long *stats, int nthreads, const int *shape_rank) {
    return dro_render_parts(desc, rd, rng_mode, cores, d_image, image, grad, stats, nthreads, shape_rank, 7);
}

int dro_render_parts(const dr_scene_desc *desc, const dr_render_desc *rd, int rng_mode, int cores, const float *d_image,
                     float *image, float *grad, long long *stats, int nthreads, const int *shape_rank, int parts) {
    // rng_mode 2: the Philox streams with the host libm (a check that the
    // restatement does not depend on the libm beyond rounding)
    g_repro_math = rng_mode == 1;
    g_product_rule = rng_mode != 0;
    if (rng_mode == 2) rng_mode = 1;
    Scene sc;
    build_scene(sc, desc, nullptr, shape_rank);
    sc.detached_pdf = (rd->flags & DR_FLAG_DETACHED_PDF) != 0;
    sc.edge_lobe_mis = (rd->flags & DR_FLAG_EDGE_LOBE_MIS) != 0;
    static std::vector<float> ident;
    if (ident.empty()) {
        ident.assign(128 * 128 * 9, 0.f);
        for (int i = 0; i < 128 * 128; i++) ident[9 * i] = ident[9 * i + 4] = ident[9 * i + 8] = 1.f;
    }
    if (!sc.ltc) sc.ltc = ident.data();
    if (!sc.ltc_ggx) sc.ltc_ggx = ident.data();
    GradLayout L = grad_layout(desc);
    const int W = rd->width, H = rd->height, spp = rd->spp, B = rd->max_bounces;
    const bool derivs = d_image != nullptr;
    const int tile = 8, ntx = (W + tile - 1) / tile, nty = (H + tile - 1) / tile, ntiles = ntx * nty;
    if (cores <= 0) cores = 1;
    std::vector<int> seeds;
    {
        std::mt19937 g((int)rd->seed);
        for (int i = 0; i < ntiles + cores; i++) seeds.push_back((int)g());
    }
    int nt = nthreads > 0 ? nthreads : (int)std::max(1u, std::thread::hardware_concurrency());
    std::vector<Accum> accs(nt);
    for (auto &a : accs) a.g.assign(L.total, 0.0);
    // pass A: pixels, tile by tile (delta_ray.cpp:1190-1464)
    parallel_loop(ntiles, nt, 1, [&](long long ti_, int tid) {
        int ti = (int)ti_;
        Tape tape;
        g_tape = &tape;
        g_parts = parts;
        std::mt19937 trng(seeds[ti]);
        MtSampler mts(&trng);
        int tx = ti % ntx, ty = ti / ntx;
        int x0 = tx * tile, x1 = std::min(x0 + tile, W), y0 = ty * tile, y1 = std::min(y0 + tile, H);
        for (int y = y0; y < y1; y++)
            for (int x = x0; x < x1; x++) {
                V3f dcol{0, 0, 0};
                if (derivs) dcol = V3f{d_image[3 * (y * W + x)], d_image[3 * (y * W + x) + 1], d_image[3 * (y * W + x) + 2]};
                V3f csum{0, 0, 0};
                for (int s = 0; s < spp; s++) {
                    uint64_t sid = ((uint64_t)y * W + x) * spp + s;
                    std::unique_ptr<PhiloxSampler> ph;
                    Sampler *main = &mts;
                    if (rng_mode == 1) {
                        ph.reset(new PhiloxSampler(rd->seed, kPixel, sid, 0));
                        main = ph.get();
                    }
                    // sub-pixel offset: u / spp as the reference (delta_ray.cpp:1236-1237),
                    // or u with DR_FLAG_FULL_PIXEL_JITTER
                    float ux = main->next();
                    float uy = main->next();
                    bool full = (rd->flags & DR_FLAG_FULL_PIXEL_JITTER) != 0;
                    float sx = full ? ux : ux / spp;
                    float sy = full ? uy : uy / spp;
                    StreamPlan plan{rng_mode, rd->seed, sid, main};
                    csum = csum + render_pixel_sample(sc, L, W, H, x, y, sx, sy, spp, B, dcol, derivs, plan, accs[tid],
                                                      rd->dp_mode);
                }
                image[3 * (y * W + x)] = csum.x;
                image[3 * (y * W + x) + 1] = csum.y;
                image[3 * (y * W + x) + 2] = csum.z;
            }
        g_tape = nullptr;
    });
    // pass B: primary edges (delta_ray.cpp:1468-1550)
    if (derivs && !sc.primary_edges.empty() && (parts & 4)) {
        long long total = rd->primary_edge_samples > 0 ? rd->primary_edge_samples : (long long)spp * W * H;
        if (rng_mode == 0) {
            int per = (int)((long long)(spp * (W * H)) / cores);
            parallel_loop(cores, nt, 1, [&](long long c, int tid) {
                std::mt19937 erng(seeds[ntiles + c]);
                MtSampler ms(&erng);
                for (int i = 0; i < per; i++) {
                    float pmf = 0.f;
                    int id = sc.primary_dist.sample_discrete(ms.next(), &pmf);
                    float w = pmf > 0.f ? 1.f / pmf : 0.f;
                    if (w <= 0.f) continue;
                    EdgeSample es = draw_edge(ms);
                    LightSample ls = draw_light(ms);
                    std::vector<SecondarySample> ss;
                    for (int b = 0; b < B; b++) ss.push_back(draw_secondary(ms));
                    PrimaryEdgeResult r = primary_edge_sample(sc, es, sc.primary_edges[id], ls, ss, d_image, W, H, w / spp);
                    if (!r.ok || r.sx < 0.f || r.sy < 0.f || r.sx > 1.f || r.sy > 1.f) continue;
                    double *g = accs[tid].g.data();
                    size_t base = L.vtx[r.edge.shape];
                    for (int a = 0; a < 3; a++) {
                        g[base + 3 * r.edge.v0 + a] += r.dv0[a];
                        g[base + 3 * r.edge.v1 + a] += r.dv1[a];
                    }
                    for (int q = 0; q < 16; q++) g[16 + q] += r.d_w2c[q];
                }
            });
        } else {
            parallel_loop(total, nt, 4096, [&](long long i, int tid) {
                PhiloxSampler ps(rd->seed, kPrimaryEdge, (uint64_t)i, 0);
                float pmf = 0.f;
                int id = sc.primary_dist.sample_discrete(ps.next(), &pmf);
                float w = pmf > 0.f ? 1.f / pmf : 0.f;
                if (w <= 0.f) return;
                EdgeSample es = draw_edge(ps);
                LightSample ls = draw_light(ps);
                std::vector<SecondarySample> ss;
                for (int b = 0; b < B; b++) ss.push_back(draw_secondary(ps));
                PrimaryEdgeResult r = primary_edge_sample(sc, es, sc.primary_edges[id], ls, ss, d_image, W, H, w / spp);
                if (!r.ok || r.sx < 0.f || r.sy < 0.f || r.sx > 1.f || r.sy > 1.f) return;
                double *g = accs[tid].g.data();
                size_t base = L.vtx[r.edge.shape];
                for (int a = 0; a < 3; a++) {
                    g[base + 3 * r.edge.v0 + a] += r.dv0[a];
                    g[base + 3 * r.edge.v1 + a] += r.dv1[a];
                }
                for (int q = 0; q < 16; q++) g[16 + q] += r.d_w2c[q];
            });
        }
    }
    if (grad) {
        for (size_t i = 0; i < L.total; i++) {
            double s = 0.0;
            for (auto &a : accs) s += a.g[i];
            grad[i] = (float)s;
        }
    }
    if (stats) {
        long long p = 0, e = 0;
        for (auto &a : accs) { p += a.points; e += a.edges; }
        stats[0] = p;
        stats[1] = e;
    }
    return 0;
}

// Hit ids of a batch of rays under the shared hit rule (closest, tnear=1e-3).
int dro_trace(const dr_scene_desc *desc, const float *rays /*[n][6]*/, long long n, int *shape_out, int *tri_out,
              float *t_out) {
    Scene sc;
    build_scene(sc, desc, nullptr);
    for (long long i = 0; i < n; i++) {
        const float *r = rays + 6 * i;
        float o[3] = {r[0], r[1], r[2]}, d[3] = {r[3], r[4], r[5]};
        float t;
        unsigned g, p;
        if (drshim::trace(sc.bvh, o, d, 1e-3f, INFINITY, false, &t, &g, &p)) {
            shape_out[i] = (int)g;
            tri_out[i] = (int)p;
            t_out[i] = t;
        } else {
            shape_out[i] = -1;
            tri_out[i] = -1;
            t_out[i] = INFINITY;
        }
    }
    return 0;
}

// One raw Philox4x32-10 block (known-answer tests).
void dro_philox_raw(const uint32_t *ctr, const uint32_t *key, uint32_t *out) {
    uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
    philox4x32_10(c, key[0], key[1]);
    for (int i = 0; i < 4; i++) out[i] = c[i];
}

// Philox draws, for checking the GPU generator bit for bit.
void dro_philox(uint64_t seed, uint32_t kind, uint64_t id, uint32_t sub, int n, float *out) {
    PhiloxSampler s(seed, kind, id, sub);
    for (int i = 0; i < n; i++) out[i] = s.next();
}

// Scene statistics: counts of edges, primary edges and tree nodes.
int dro_scene_info(const dr_scene_desc *desc, int *out /*[6]*/) {
    Scene sc;
    build_scene(sc, desc, nullptr);
    out[0] = (int)sc.primary_edges.size();
    out[1] = (int)sc.sil_tree.edges.size();
    out[2] = (int)sc.sil_tree.nodes.size();
    out[3] = (int)sc.nrm_tree.edges.size();
    out[4] = (int)sc.nrm_tree.nodes.size();
    out[5] = (int)sc.bvh.tris.size();
    return 0;
}

}  // extern "C"
