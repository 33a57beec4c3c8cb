// Test infrastructure only (oracle). Not part of the product.
//
// A minimal, project-written stand-in for the subset of the Embree 3 API that
// the reference renderer calls (scene.cpp:100-135 builds the scene,
// scene.cpp:147-202 casts rays).  Embree is a third-party library that is not
// vendored with the reference and is not installed here; this header lets the
// reference sources compile unmodified so that they can serve as the oracle.
//
// Only *which* triangle a ray hits is taken from here: the reference
// re-intersects the hit triangle analytically itself (intersect.h:100-148).
// Ray conventions are the reference's: nearest_hit uses [tnear, tfar] =
// [1e-3, inf) (scene.cpp:188-189) and occluded uses [1e-3 d, (1-1e-3) d]
// (scene.cpp:159-160).
//
// Hit rule (shared with the GPU product so that hit ids agree): Moller-Trumbore
// in float, a hit is accepted when u >= 0, v >= 0, u + v <= 1 and
// tnear < t < tfar; the closest t wins and equal t is broken by the lower
// (geomID, primID).  Embree's own tie-breaking is unknown, so hits on shared
// edges are "unpinned" against real Embree.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#define RTC_INVALID_GEOMETRY_ID ((unsigned int)-1)
#define RTC_MAX_INSTANCE_LEVEL_COUNT 1

enum RTCBuildQuality { RTC_BUILD_QUALITY_LOW = 0, RTC_BUILD_QUALITY_MEDIUM = 1, RTC_BUILD_QUALITY_HIGH = 2 };
enum RTCSceneFlags { RTC_SCENE_FLAG_NONE = 0, RTC_SCENE_FLAG_DYNAMIC = 1, RTC_SCENE_FLAG_COMPACT = 2, RTC_SCENE_FLAG_ROBUST = 4 };
enum RTCGeometryType { RTC_GEOMETRY_TYPE_TRIANGLE = 0 };
enum RTCBufferType { RTC_BUFFER_TYPE_INDEX = 0, RTC_BUFFER_TYPE_VERTEX = 1 };
enum RTCFormat { RTC_FORMAT_UINT3 = 0x5003, RTC_FORMAT_FLOAT3 = 0x9003 };

struct RTCIntersectContext { unsigned int flags; };

struct RTCRay {
    float org_x, org_y, org_z, tnear;
    float dir_x, dir_y, dir_z, time;
    float tfar;
    unsigned int mask, id, flags;
};

struct RTCHit {
    float Ng_x, Ng_y, Ng_z, u, v;
    unsigned int primID, geomID;
    unsigned int instID[RTC_MAX_INSTANCE_LEVEL_COUNT];
};

struct RTCRayHit { RTCRay ray; RTCHit hit; };

namespace drshim {

struct Geometry {
    int refs = 1;
    std::vector<unsigned char> vtx, idx;
    size_t vtx_stride = 0, idx_stride = 0, nv = 0, nt = 0;
};

struct Tri { float v0[3], v1[3], v2[3]; unsigned geom, prim; };

struct Node {
    float lo[3], hi[3];
    int start, count;  // count > 0: leaf over tris[start, start+count)
    int right;         // interior: left child is this+1, right child index
};

struct Scene {
    std::vector<Geometry *> geoms;
    std::vector<Tri> tris;
    std::vector<Node> nodes;
    ~Scene() {
        for (auto *g : geoms) {
            if (--g->refs == 0) delete g;
        }
    }
};

inline void tri_bounds(const Tri &t, float lo[3], float hi[3]) {
    for (int a = 0; a < 3; a++) {
        lo[a] = std::min(std::min(t.v0[a], t.v1[a]), t.v2[a]);
        hi[a] = std::max(std::max(t.v0[a], t.v1[a]), t.v2[a]);
    }
}

inline int build_node(Scene &s, int start, int end) {
    int id = (int)s.nodes.size();
    s.nodes.push_back(Node{});
    Node nd;
    for (int a = 0; a < 3; a++) {
        nd.lo[a] = std::numeric_limits<float>::infinity();
        nd.hi[a] = -std::numeric_limits<float>::infinity();
    }
    float clo[3], chi[3];
    for (int a = 0; a < 3; a++) {
        clo[a] = std::numeric_limits<float>::infinity();
        chi[a] = -std::numeric_limits<float>::infinity();
    }
    for (int i = start; i < end; i++) {
        float lo[3], hi[3];
        tri_bounds(s.tris[i], lo, hi);
        for (int a = 0; a < 3; a++) {
            nd.lo[a] = std::min(nd.lo[a], lo[a]);
            nd.hi[a] = std::max(nd.hi[a], hi[a]);
            float c = 0.5f * (lo[a] + hi[a]);
            clo[a] = std::min(clo[a], c);
            chi[a] = std::max(chi[a], c);
        }
    }
    int axis = 0;
    for (int a = 1; a < 3; a++) {
        if (chi[a] - clo[a] > chi[axis] - clo[axis]) axis = a;
    }
    if (end - start <= 4 || chi[axis] <= clo[axis]) {
        nd.start = start;
        nd.count = end - start;
        nd.right = -1;
        s.nodes[id] = nd;
        return id;
    }
    int mid = (start + end) / 2;
    std::nth_element(s.tris.begin() + start, s.tris.begin() + mid, s.tris.begin() + end,
                     [axis](const Tri &x, const Tri &y) {
                         float cx = std::min(std::min(x.v0[axis], x.v1[axis]), x.v2[axis]) +
                                    std::max(std::max(x.v0[axis], x.v1[axis]), x.v2[axis]);
                         float cy = std::min(std::min(y.v0[axis], y.v1[axis]), y.v2[axis]) +
                                    std::max(std::max(y.v0[axis], y.v1[axis]), y.v2[axis]);
                         return cx < cy;
                     });
    nd.start = 0;
    nd.count = 0;
    build_node(s, start, mid);
    nd.right = build_node(s, mid, end);
    s.nodes[id] = nd;
    return id;
}

inline float safe_inv(float x) {
    const float big = 1e30f;
    if (x == 0.f) return big;
    float r = 1.f / x;
    return r > big ? big : (r < -big ? -big : r);
}

inline bool slab(const Node &n, const float o[3], const float inv[3], float tmax) {
    float t0 = 0.f, t1 = tmax;
    for (int a = 0; a < 3; a++) {
        float ta = (n.lo[a] - o[a]) * inv[a];
        float tb = (n.hi[a] - o[a]) * inv[a];
        if (ta > tb) std::swap(ta, tb);
        // widen slightly so that triangles lying in a box face are not culled
        tb *= 1.0000004f;
        t0 = ta > t0 ? ta : t0;
        t1 = tb < t1 ? tb : t1;
        if (t0 > t1) return false;
    }
    return true;
}

// Moller-Trumbore.  Written without NaN tests: the reference is compiled with
// -ffast-math, under which NaN comparisons are not reliable.
inline bool hit_tri(const Tri &tr, const float o[3], const float d[3], float *t_out) {
    float e1[3], e2[3], p[3], s[3], q[3];
    for (int a = 0; a < 3; a++) {
        e1[a] = tr.v1[a] - tr.v0[a];
        e2[a] = tr.v2[a] - tr.v0[a];
        s[a] = o[a] - tr.v0[a];
    }
    p[0] = d[1] * e2[2] - d[2] * e2[1];
    p[1] = d[2] * e2[0] - d[0] * e2[2];
    p[2] = d[0] * e2[1] - d[1] * e2[0];
    float det = e1[0] * p[0] + e1[1] * p[1] + e1[2] * p[2];
    if (det == 0.f) return false;
    float inv = 1.f / det;
    float u = (s[0] * p[0] + s[1] * p[1] + s[2] * p[2]) * inv;
    if (u < 0.f || u > 1.f) return false;
    q[0] = s[1] * e1[2] - s[2] * e1[1];
    q[1] = s[2] * e1[0] - s[0] * e1[2];
    q[2] = s[0] * e1[1] - s[1] * e1[0];
    float v = (d[0] * q[0] + d[1] * q[1] + d[2] * q[2]) * inv;
    if (v < 0.f || u + v > 1.f) return false;
    *t_out = (e2[0] * q[0] + e2[1] * q[1] + e2[2] * q[2]) * inv;
    return true;
}

// any == true: stop at the first hit inside (tnear, tfar).
inline bool trace(const Scene &s, const float o[3], const float d[3], float tnear, float tfar,
                  bool any, float *t_out, unsigned *geom, unsigned *prim) {
    if (s.nodes.empty()) return false;
    float inv[3] = {safe_inv(d[0]), safe_inv(d[1]), safe_inv(d[2])};
    int stack[128];
    int sp = 0;
    stack[sp++] = 0;
    bool found = false;
    float best = tfar;
    unsigned bg = RTC_INVALID_GEOMETRY_ID, bp = RTC_INVALID_GEOMETRY_ID;
    while (sp > 0) {
        const Node &n = s.nodes[stack[--sp]];
        if (!slab(n, o, inv, best)) continue;
        if (n.count > 0) {
            for (int i = n.start; i < n.start + n.count; i++) {
                const Tri &tr = s.tris[i];
                float t;
                if (!hit_tri(tr, o, d, &t)) continue;
                if (t <= tnear || t >= tfar) continue;
                if (any) {
                    *t_out = t;
                    return true;
                }
                bool closer = t < best || (t == best && (tr.geom < bg || (tr.geom == bg && tr.prim < bp)));
                if (!found || closer) {
                    found = true;
                    best = t;
                    bg = tr.geom;
                    bp = tr.prim;
                }
            }
        } else {
            int self = (int)(&n - s.nodes.data());
            stack[sp++] = n.right;
            stack[sp++] = self + 1;
        }
    }
    if (found) {
        *t_out = best;
        *geom = bg;
        *prim = bp;
    }
    return found;
}

}  // namespace drshim

typedef drshim::Scene *RTCScene;
typedef drshim::Geometry *RTCGeometry;
typedef void *RTCDevice;

inline RTCDevice rtcNewDevice(const char *) { return (RTCDevice)1; }
inline void rtcReleaseDevice(RTCDevice) {}
inline RTCScene rtcNewScene(RTCDevice) { return new drshim::Scene(); }
inline void rtcSetSceneBuildQuality(RTCScene, RTCBuildQuality) {}
inline void rtcSetSceneFlags(RTCScene, RTCSceneFlags) {}
inline RTCGeometry rtcNewGeometry(RTCDevice, RTCGeometryType) { return new drshim::Geometry(); }

inline void *rtcSetNewGeometryBuffer(RTCGeometry g, RTCBufferType type, unsigned int, RTCFormat,
                                     size_t byte_stride, size_t count) {
    if (type == RTC_BUFFER_TYPE_VERTEX) {
        g->vtx.assign(byte_stride * count + 16, 0);
        g->vtx_stride = byte_stride;
        g->nv = count;
        return g->vtx.data();
    }
    g->idx.assign(byte_stride * count + 16, 0);
    g->idx_stride = byte_stride;
    g->nt = count;
    return g->idx.data();
}

inline void rtcSetGeometryVertexAttributeCount(RTCGeometry, unsigned int) {}
inline void rtcCommitGeometry(RTCGeometry) {}

inline unsigned int rtcAttachGeometry(RTCScene s, RTCGeometry g) {
    g->refs++;
    s->geoms.push_back(g);
    return (unsigned int)(s->geoms.size() - 1);
}

inline void rtcReleaseGeometry(RTCGeometry g) {
    if (--g->refs == 0) delete g;
}

inline void rtcCommitScene(RTCScene s) {
    s->tris.clear();
    s->nodes.clear();
    for (unsigned gi = 0; gi < s->geoms.size(); gi++) {
        const drshim::Geometry *g = s->geoms[gi];
        for (size_t t = 0; t < g->nt; t++) {
            unsigned idx[3];
            std::memcpy(idx, g->idx.data() + t * g->idx_stride, sizeof(idx));
            drshim::Tri tr;
            float *dst[3] = {tr.v0, tr.v1, tr.v2};
            for (int k = 0; k < 3; k++) {
                std::memcpy(dst[k], g->vtx.data() + (size_t)idx[k] * g->vtx_stride, 3 * sizeof(float));
            }
            tr.geom = gi;
            tr.prim = (unsigned)t;
            s->tris.push_back(tr);
        }
    }
    if (!s->tris.empty()) drshim::build_node(*s, 0, (int)s->tris.size());
}

inline void rtcReleaseScene(RTCScene s) { delete s; }
inline void rtcInitIntersectContext(RTCIntersectContext *c) { c->flags = 0; }

inline void rtcOccluded1(RTCScene s, RTCIntersectContext *, RTCRay *r) {
    float o[3] = {r->org_x, r->org_y, r->org_z};
    float d[3] = {r->dir_x, r->dir_y, r->dir_z};
    float t;
    unsigned g, p;
    if (drshim::trace(*s, o, d, r->tnear, r->tfar, true, &t, &g, &p)) {
        r->tfar = -std::numeric_limits<float>::infinity();
    }
}

inline void rtcIntersect1(RTCScene s, RTCIntersectContext *, RTCRayHit *rh) {
    float o[3] = {rh->ray.org_x, rh->ray.org_y, rh->ray.org_z};
    float d[3] = {rh->ray.dir_x, rh->ray.dir_y, rh->ray.dir_z};
    float t;
    unsigned g, p;
    if (drshim::trace(*s, o, d, rh->ray.tnear, rh->ray.tfar, false, &t, &g, &p)) {
        rh->ray.tfar = t;
        rh->hit.geomID = g;
        rh->hit.primID = p;
    }
}
