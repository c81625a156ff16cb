// Device scene: triangles, materials, area lights and the BVH that
// replaces the reference's Embree scene (scene.h:275-348).
//
// Layout in HBM (n faces, the reference's per-face unshared vertices):
//   tri    float4[3n]  p0, p1, p2 per face (face order)
//   nrm    float4[3n]  vertex normals n0, n1, n2 per face
//   geo    float4[n]   geometric normal (triangle.h:30) and area (:33)
//   mat    Material[n] per-face BxDF and emission (scene.h:21-51)
//   lights int[m]      faces with emission > 0, in face order
//   mt     float4[3n]  leaf order: {p0, face id}, {p1 - p0}, {p2 - p0}
//   nodes  float4[4(n-1)] internal nodes: {left box lo, left child},
//                      {left box hi, right child}, {right box lo},
//                      {right box hi}; a child < 0 is leaf ~child.
#pragma once

#include "pm_math.cuh"

namespace pm {

constexpr int kBvhStack = 64;

struct SceneDev {
  const float4* __restrict__ tri;
  const float4* __restrict__ nrm;
  const float4* __restrict__ geo;
  const Material* __restrict__ mat;
  const int* __restrict__ lights;
  const float4* __restrict__ mt;
  const float4* __restrict__ nodes;
  int n_faces;
  int n_lights;
  int* err;  // device error word (bit 0: traversal stack overflow)
};

struct Hit {
  float t, u, v;
  int prim;  // face id, -1 when nothing was hit
};

__device__ __forceinline__ V3 f4v3(float4 a) { return v3(a.x, a.y, a.z); }

// Moller-Trumbore ray/triangle test (Moller & Trumbore 1997), two-sided.
// The hit is valid when tmin <= t <= tmax, Embree's convention for
// [tnear, tfar]; (u, v) weight p1 and p2 like Embree's barycentrics.
__device__ __forceinline__ bool ray_triangle(V3 o, V3 d, V3 p0, V3 e1, V3 e2,
                                             float& t, float& u, float& v) {
  const V3 pvec = cross(d, e2);
  const float det = dot(e1, pvec);
  if (!(det != 0.f)) return false;
  const float inv = 1.0f / det;
  const V3 tvec = o - p0;
  u = dot(tvec, pvec) * inv;
  if (!(u >= 0.f && u <= 1.f)) return false;
  const V3 qvec = cross(tvec, e1);
  v = dot(d, qvec) * inv;
  if (!(v >= 0.f && u + v <= 1.f)) return false;
  t = dot(e2, qvec) * inv;
  return t == t;
}

// Slab test of the ray against a box; NaN products (0 * inf) impose no
// constraint. The exit distance is widened by 1 + 2*gamma(3) (Ize 2013)
// and the boxes themselves are padded at build time, so a box is never
// culled when a triangle inside it is hit.
__device__ __forceinline__ bool ray_box(V3 o, V3 inv, float tmin, float tmax,
                                        float4 lo, float4 hi, float& tnear) {
  const float tx0 = (lo.x - o.x) * inv.x, tx1 = (hi.x - o.x) * inv.x;
  const float ty0 = (lo.y - o.y) * inv.y, ty1 = (hi.y - o.y) * inv.y;
  const float tz0 = (lo.z - o.z) * inv.z, tz1 = (hi.z - o.z) * inv.z;
  const float tn = fmaxf(fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)),
                               fminf(tz0, tz1)), tmin);
  const float tf = fminf(fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)),
                               fmaxf(tz0, tz1)), tmax);
  tnear = tn;
  return tn <= tf * 1.00000072f;
}

__device__ __forceinline__ void test_leaf(const SceneDev& sc, int leaf, V3 o,
                                          V3 d, float tmin, Hit& h) {
  const float4 a = __ldg(sc.mt + 3 * leaf);
  const float4 b = __ldg(sc.mt + 3 * leaf + 1);
  const float4 c = __ldg(sc.mt + 3 * leaf + 2);
  float t, u, v;
  if (ray_triangle(o, d, f4v3(a), f4v3(b), f4v3(c), t, u, v)) {
    const int prim = __float_as_int(a.w);
    if (t >= tmin && t <= h.t &&
        (t < h.t || h.prim < 0 || prim < h.prim)) {
      h.t = t;
      h.u = u;
      h.v = v;
      h.prim = prim;
    }
  }
}

// Closest hit with tmin <= t <= tmax; ties in t go to the smaller face id,
// so the result does not depend on the traversal order. STACK entries of
// traversal stack (an overflow sets error bit 0 and loses the subtree).
template <int STACK>
__device__ __forceinline__ bool intersect_t(const SceneDev& sc, V3 o, V3 d,
                                            float tmin, float tmax, Hit& h) {
  h.t = tmax;
  h.prim = -1;
  h.u = h.v = 0.f;
  if (sc.n_faces <= 0) return false;
  if (sc.n_faces == 1) {
    test_leaf(sc, 0, o, d, tmin, h);
    return h.prim >= 0;
  }
  const V3 inv = v3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
  int stack[STACK];
  int sp = 0;
  int node = 0;
  while (true) {
    const float4 a = __ldg(sc.nodes + 4 * node);
    const float4 b = __ldg(sc.nodes + 4 * node + 1);
    const float4 c = __ldg(sc.nodes + 4 * node + 2);
    const float4 e = __ldg(sc.nodes + 4 * node + 3);
    const int left = __float_as_int(a.w), right = __float_as_int(b.w);
    float tl, tr;
    const bool hl = ray_box(o, inv, tmin, h.t, a, b, tl);
    const bool hr = ray_box(o, inv, tmin, h.t, c, e, tr);
    int next = -1, other = -1;
    if (hl) {
      if (left < 0) test_leaf(sc, ~left, o, d, tmin, h);
      else next = left;
    }
    if (hr) {
      if (right < 0) {
        test_leaf(sc, ~right, o, d, tmin, h);
      } else if (next < 0) {
        next = right;
      } else {
        other = right;
        if (tr < tl) {
          other = next;
          next = right;
        }
      }
    }
    if (other >= 0) {
      if (sp < STACK) {
        stack[sp++] = other;
      } else {
        atomicOr(sc.err, 1);
      }
    }
    if (next < 0) {
      if (sp == 0) break;
      node = stack[--sp];
    } else {
      node = next;
    }
  }
  return h.prim >= 0;
}

__device__ __forceinline__ bool intersect(const SceneDev& sc, V3 o, V3 d,
                                          float tmin, float tmax, Hit& h) {
  return intersect_t<kBvhStack>(sc, o, d, tmin, tmax, h);
}

// Surface frame at a hit (scene.h:324-337): position = ray(t), shading
// normal interpolated and not re-normalised (triangle.h:64-71), tangent
// frame from orthonormalBasis.
struct Surf {
  V3 pos, ng, ns, dpdu, dpdv;
};

__device__ __forceinline__ V3 shading_normal(const SceneDev& sc, int f,
                                             float b0, float b1) {
  const V3 n1 = f4v3(__ldg(sc.nrm + 3 * f));
  const V3 n2 = f4v3(__ldg(sc.nrm + 3 * f + 1));
  const V3 n3 = f4v3(__ldg(sc.nrm + 3 * f + 2));
  return n1 * (1.0f - b0 - b1) + n2 * b0 + n3 * b1;
}

__device__ __forceinline__ Surf surface_at(const SceneDev& sc, V3 o, V3 d,
                                           const Hit& h) {
  Surf s;
  s.pos = o + h.t * d;
  s.ng = f4v3(__ldg(sc.geo + h.prim));
  s.ns = shading_normal(sc, h.prim, h.u, h.v);
  orthonormal_basis(s.ns, s.dpdu, s.dpdv);
  return s;
}

// Triangle::samplePoint (triangle.h:84-114): uniform point, pdf = 1/area.
// Draws one getNext2D.
__device__ __forceinline__ Surf sample_triangle(const SceneDev& sc, int f,
                                                Rng& rng, float& pdf) {
  float u0, u1;
  rng.next2d(u0, u1);
  const float su0 = sqrtf(u0);
  const float b0 = 1.0f - su0, b1 = u1 * su0;
  const V3 p1 = f4v3(__ldg(sc.tri + 3 * f));
  const V3 p2 = f4v3(__ldg(sc.tri + 3 * f + 1));
  const V3 p3 = f4v3(__ldg(sc.tri + 3 * f + 2));
  Surf s;
  s.pos = (1.0f - b0 - b1) * p1 + b0 * p2 + b1 * p3;
  s.ns = shading_normal(sc, f, b0, b1);
  orthonormal_basis(s.ns, s.dpdu, s.dpdv);
  s.ng = f4v3(__ldg(sc.geo + f));
  pdf = 1.0f / __ldg(sc.geo + f).w;
  return s;
}

// Scene::sampleLight (scene.h:350-355): uniform over the light faces by
// count; getNext1D can return 1.0, clamped to the last light.
__device__ __forceinline__ int sample_light(const SceneDev& sc, Rng& rng,
                                            float& pdf) {
  unsigned idx = (unsigned)((float)sc.n_lights * rng.next1d());
  if (idx == (unsigned)sc.n_lights) idx--;
  pdf = 1.0f / (float)sc.n_lights;
  return __ldg(sc.lights + idx);
}

}  // namespace pm
