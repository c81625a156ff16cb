// ORACLE shim — test infrastructure only. A project-written stand-in for
// the part of the Embree 3 API that the reference's scene.h calls
// (scene.h:275-348): one triangle geometry, committed into a CPU BVH, and
// rtcIntersect1 returning the closest hit with tnear <= t <= tfar. The
// triangle test is Moller-Trumbore (Moller & Trumbore 1997) with the same
// arithmetic and tie rule (smallest t, then smallest primID) as the
// project's device intersector, so both report the same hits. Embree's own
// source is not used or reproduced.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <limits>
#include <vector>

#define RTC_INVALID_GEOMETRY_ID ((unsigned int)-1)

enum RTCGeometryType { RTC_GEOMETRY_TYPE_TRIANGLE = 0 };
enum RTCBufferType { RTC_BUFFER_TYPE_INDEX = 0, RTC_BUFFER_TYPE_VERTEX = 1 };
enum RTCFormat { RTC_FORMAT_UINT3 = 0x5003, RTC_FORMAT_FLOAT3 = 0x9003 };

struct RTCRay {
  float org_x, org_y, org_z, tnear;
  float dir_x, dir_y, dir_z, time;
  float tfar;
  unsigned int mask, id, flags;
};
struct RTCHit {
  float Ng_x, Ng_y, Ng_z, u, v;
  unsigned int primID, geomID;
  unsigned int instID[1];
};
struct RTCRayHit {
  RTCRay ray;
  RTCHit hit;
};
struct RTCIntersectContext {
  unsigned int flags;
};

struct RTCDeviceTy {};
struct RTCGeometryTy {
  std::vector<float> vertices;
  std::vector<unsigned> indices;
  int refs = 1;
};
struct RTCSceneTy {
  RTCGeometryTy* geom = nullptr;
  // per triangle in build order: p0, e1 = p1 - p0, e2 = p2 - p0, primID
  struct Tri {
    float p0[3], e1[3], e2[3];
    unsigned prim;
  };
  std::vector<Tri> tris;
  struct Node {
    float lo[3], hi[3];
    int left, right;  // children; leaf when left < 0: tris [first, first+count)
    int first, count;
  };
  std::vector<Node> nodes;
};
typedef RTCDeviceTy* RTCDevice;
typedef RTCSceneTy* RTCScene;
typedef RTCGeometryTy* RTCGeometry;

inline RTCDevice rtcNewDevice(const char*) { return new RTCDeviceTy(); }
inline void rtcReleaseDevice(RTCDevice d) { delete d; }
inline RTCScene rtcNewScene(RTCDevice) { return new RTCSceneTy(); }
inline RTCGeometry rtcNewGeometry(RTCDevice, RTCGeometryType) { return new RTCGeometryTy(); }
inline void* rtcSetNewGeometryBuffer(RTCGeometry g, RTCBufferType type, unsigned, RTCFormat,
                                     size_t byteStride, size_t itemCount) {
  if (type == RTC_BUFFER_TYPE_VERTEX) {
    g->vertices.assign(byteStride / sizeof(float) * itemCount, 0.f);
    return g->vertices.data();
  }
  g->indices.assign(byteStride / sizeof(unsigned) * itemCount, 0u);
  return g->indices.data();
}
inline void rtcCommitGeometry(RTCGeometry) {}
inline unsigned rtcAttachGeometry(RTCScene s, RTCGeometry g) {
  s->geom = g;
  g->refs++;
  return 0;
}
inline void rtcReleaseGeometry(RTCGeometry g) {
  if (--g->refs == 0) delete g;
}
inline void rtcInitIntersectContext(RTCIntersectContext* c) { c->flags = 0; }

namespace pm_shim {
inline int build_node(RTCSceneTy* s, std::vector<unsigned>& ids, int first, int count,
                      const std::vector<float>& cen, float pad) {
  RTCSceneTy::Node n;
  for (int a = 0; a < 3; ++a) {
    n.lo[a] = std::numeric_limits<float>::max();
    n.hi[a] = -std::numeric_limits<float>::max();
  }
  for (int i = first; i < first + count; ++i) {
    const RTCSceneTy::Tri& t = s->tris[ids[i]];
    for (int a = 0; a < 3; ++a) {
      const float v0 = t.p0[a], v1 = t.p0[a] + t.e1[a], v2 = t.p0[a] + t.e2[a];
      n.lo[a] = std::min(n.lo[a], std::min(v0, std::min(v1, v2)) - pad);
      n.hi[a] = std::max(n.hi[a], std::max(v0, std::max(v1, v2)) + pad);
    }
  }
  const int me = (int)s->nodes.size();
  s->nodes.push_back(n);
  if (count <= 4) {
    s->nodes[me].left = -1;
    s->nodes[me].right = -1;
    s->nodes[me].first = first;
    s->nodes[me].count = count;
    return me;
  }
  float clo[3], chi[3];
  for (int a = 0; a < 3; ++a) {
    clo[a] = std::numeric_limits<float>::max();
    chi[a] = -std::numeric_limits<float>::max();
  }
  for (int i = first; i < first + count; ++i)
    for (int a = 0; a < 3; ++a) {
      clo[a] = std::min(clo[a], cen[3 * ids[i] + a]);
      chi[a] = std::max(chi[a], cen[3 * ids[i] + a]);
    }
  int axis = 0;
  for (int a = 1; a < 3; ++a)
    if (chi[a] - clo[a] > chi[axis] - clo[axis]) axis = a;
  const int mid = first + count / 2;
  std::nth_element(ids.begin() + first, ids.begin() + mid, ids.begin() + first + count,
                   [&](unsigned x, unsigned y) { return cen[3 * x + axis] < cen[3 * y + axis]; });
  const int l = build_node(s, ids, first, mid - first, cen, pad);
  const int r = build_node(s, ids, mid, first + count - mid, cen, pad);
  s->nodes[me].left = l;
  s->nodes[me].right = r;
  s->nodes[me].first = 0;
  s->nodes[me].count = 0;
  return me;
}
}  // namespace pm_shim

inline void rtcCommitScene(RTCScene s) {
  const RTCGeometryTy* g = s->geom;
  const size_t n = g ? g->indices.size() / 3 : 0;
  s->tris.resize(n);
  std::vector<float> cen(3 * n);
  float size = 0.f;
  for (size_t f = 0; f < n; ++f) {
    RTCSceneTy::Tri& t = s->tris[f];
    const float* p[3];
    for (int k = 0; k < 3; ++k) p[k] = &g->vertices[3 * g->indices[3 * f + k]];
    for (int a = 0; a < 3; ++a) {
      t.p0[a] = p[0][a];
      t.e1[a] = p[1][a] - p[0][a];
      t.e2[a] = p[2][a] - p[0][a];
      cen[3 * f + a] = (p[0][a] + p[1][a] + p[2][a]) / 3.0f;
      for (int k = 0; k < 3; ++k) size = std::max(size, std::fabs(p[k][a]));
    }
    t.prim = (unsigned)f;
  }
  std::vector<unsigned> ids(n);
  for (size_t i = 0; i < n; ++i) ids[i] = (unsigned)i;
  s->nodes.clear();
  if (n) pm_shim::build_node(s, ids, 0, (int)n, cen, 4e-5f * size + 1e-30f);
  std::vector<RTCSceneTy::Tri> ordered(n);
  for (size_t i = 0; i < n; ++i) ordered[i] = s->tris[ids[i]];
  s->tris.swap(ordered);
}

inline void rtcReleaseScene(RTCScene s) {
  if (s && s->geom) rtcReleaseGeometry(s->geom);
  delete s;
}

inline void rtcIntersect1(RTCScene s, RTCIntersectContext*, RTCRayHit* rh) {
  const float o[3] = {rh->ray.org_x, rh->ray.org_y, rh->ray.org_z};
  const float d[3] = {rh->ray.dir_x, rh->ray.dir_y, rh->ray.dir_z};
  const float tmin = rh->ray.tnear;
  float best = rh->ray.tfar;
  int best_prim = -1;
  float bu = 0.f, bv = 0.f;
  if (s->nodes.empty()) return;
  const float inv[3] = {1.0f / d[0], 1.0f / d[1], 1.0f / d[2]};
  int stack[128];
  int sp = 0;
  stack[sp++] = 0;
  while (sp) {
    const RTCSceneTy::Node& n = s->nodes[stack[--sp]];
    float tn = tmin, tf = best;
    for (int a = 0; a < 3; ++a) {
      const float t0 = (n.lo[a] - o[a]) * inv[a], t1 = (n.hi[a] - o[a]) * inv[a];
      const float lo = std::fmin(t0, t1), hi = std::fmax(t0, t1);
      tn = std::fmax(tn, lo);
      tf = std::fmin(tf, hi);
    }
    if (!(tn <= tf * 1.00000072f)) continue;
    if (n.left >= 0) {
      stack[sp++] = n.left;
      stack[sp++] = n.right;
      continue;
    }
    for (int i = n.first; i < n.first + n.count; ++i) {
      const RTCSceneTy::Tri& t = s->tris[i];
      const float pv[3] = {d[1] * t.e2[2] - d[2] * t.e2[1], d[2] * t.e2[0] - d[0] * t.e2[2],
                           d[0] * t.e2[1] - d[1] * t.e2[0]};
      const float det = t.e1[0] * pv[0] + t.e1[1] * pv[1] + t.e1[2] * pv[2];
      if (!(det != 0.f)) continue;
      const float invd = 1.0f / det;
      const float tv[3] = {o[0] - t.p0[0], o[1] - t.p0[1], o[2] - t.p0[2]};
      const float u = (tv[0] * pv[0] + tv[1] * pv[1] + tv[2] * pv[2]) * invd;
      if (!(u >= 0.f && u <= 1.f)) continue;
      const float qv[3] = {tv[1] * t.e1[2] - tv[2] * t.e1[1], tv[2] * t.e1[0] - tv[0] * t.e1[2],
                           tv[0] * t.e1[1] - tv[1] * t.e1[0]};
      const float v = (d[0] * qv[0] + d[1] * qv[1] + d[2] * qv[2]) * invd;
      if (!(v >= 0.f && u + v <= 1.f)) continue;
      const float tt = (t.e2[0] * qv[0] + t.e2[1] * qv[1] + t.e2[2] * qv[2]) * invd;
      if (!(tt == tt)) continue;
      if (tt >= tmin && tt <= best && (tt < best || best_prim < 0 || (int)t.prim < best_prim)) {
        best = tt;
        best_prim = (int)t.prim;
        bu = u;
        bv = v;
      }
    }
  }
  if (best_prim >= 0) {
    rh->ray.tfar = best;
    rh->hit.u = bu;
    rh->hit.v = bv;
    rh->hit.primID = (unsigned)best_prim;
    rh->hit.geomID = 0;
  }
}
