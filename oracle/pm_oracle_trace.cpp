// ORACLE — test infrastructure only. CPU restatement of the reference's
// scene intersection and photon tracing, used by tests/ as the checker of
// the device LBVH and photon tracer. Built with -ffp-contract=off.
//
// Follows yumcyaWiz/photon_mapping:
//   scene.h:307-355     intersect (closest hit) and sampleLight
//   triangle.h:25-114   geometric normal, area, shading normal, samplePoint
//   light.h:27-44       AreaLight Le and sampleDirection
//   material.h          Lambert, Mirror, Glass
//   primitive.h:32-82   world/local frames
//   integrator.h:25-46  cosTerm
//   integrator.h:265-288, 393-563  sampleRayFromLight and the two tracing loops
//   sampler.h:11-91     PCG32 (state = seed, inc = 1) and sampleCosineHemisphere
//
// Choices shared with the device code (the definition of the path, not the
// reference's): the intersector is Moller-Trumbore with tmin <= t <= tmax
// and ties in t broken by the smaller face index (Embree itself is absent);
// cos/sin(theta) of the cosine hemisphere use the closed forms sqrt(1-u),
// sqrt(u) of cos/sin(acos(1-2u)/2); sin/cos(phi) come from a double-precision
// Taylor evaluation; photon i uses the stream state
// splitmix64(seed ^ splitmix64(i)); getNext2D returns (second, first) draw,
// the argument order the reference's GCC build evaluates.
#include <cmath>
#include <cstdint>
#include <algorithm>
#include <cstring>
#include <vector>

namespace orc {

struct V {
  float x, y, z;
};
static inline V mk(float x, float y, float z) { return V{x, y, z}; }
static inline V add(V a, V b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V sub(V a, V b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V neg(V a) { return mk(-a.x, -a.y, -a.z); }
static inline V mul(V a, V b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline V muls(V a, float k) { return mk(a.x * k, a.y * k, a.z * k); }
static inline V divs(V a, float k) { return mk(a.x / k, a.y / k, a.z / k); }
static inline float dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V cross(V a, V b) {
  return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float length(V a) { return std::sqrt(dot(a, a)); }
static inline V normalize(V a) { return divs(a, length(a)); }
static inline void basis(V n, V& t, V& b) {
  if (std::fabs(n.y) < 0.9f)
    t = normalize(cross(n, mk(0, 1, 0)));
  else
    t = normalize(cross(n, mk(0, 0, -1)));
  b = normalize(cross(t, n));
}
static inline V to_local(V v, V lx, V ly, V lz) {
  return mk(dot(v, lx), dot(v, ly), dot(v, lz));
}
static inline V to_world(V v, V lx, V ly, V lz) {
  return mk(v.x * lx.x + v.y * ly.x + v.z * lz.x, v.x * lx.y + v.y * ly.y + v.z * lz.y,
            v.x * lx.z + v.y * ly.z + v.z * lz.z);
}

constexpr float PI = 3.14159265359f;
constexpr float PI_INV = 1.0f / PI;
constexpr float PI_MUL_2 = 2.0f * PI;
constexpr float RAY_EPS = 1e-5f;

struct Rng {
  uint64_t state;
  uint32_t u32() {
    const uint64_t old = state;
    state = old * 6364136223846793005ULL + 1ULL;
    const uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    const uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((0u - rot) & 31u));
  }
  float next() { return (float)u32() * (1.0f / 4294967295.0f); }
  void next2(float& u0, float& u1) {
    u1 = next();
    u0 = next();
  }
};

static inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}

// sin/cos of a float angle |x| <= 8 in float arithmetic, one rounding per
// operation (built with -ffp-contract=off): Cody-Waite reduction by pi/2
// split in three floats (21 + 21 + 24 significant bits), Taylor
// polynomials on |r| <= pi/4 (sin to r^9, cos to r^10) in Horner form with
// the coefficients 1/n! rounded to float, quadrant q mod 4.
static inline void sincos_f(float x, float& s, float& c) {
  const float q = std::rint(x * 0x1.45f306p-1f);
  float r = x - q * 0x1.921fbp+0f;
  r = r - q * 0x1.5110bp-22f;
  r = r - q * 0x1.184698p-44f;
  const float r2 = r * r;
  float ps = 1.0f / 362880.0f;
  ps = ps * r2 + -1.0f / 5040.0f;
  ps = ps * r2 + 1.0f / 120.0f;
  ps = ps * r2 + -1.0f / 6.0f;
  const float sr = r + (r * r2) * ps;
  float pc = -1.0f / 3628800.0f;
  pc = pc * r2 + 1.0f / 40320.0f;
  pc = pc * r2 + -1.0f / 720.0f;
  pc = pc * r2 + 1.0f / 24.0f;
  pc = pc * r2 + -0.5f;
  const float cr = 1.0f + r2 * pc;
  const int quad = ((int)q) & 3;
  s = quad == 0 ? sr : quad == 1 ? cr : quad == 2 ? -sr : -cr;
  c = quad == 0 ? cr : quad == 1 ? -sr : quad == 2 ? -cr : sr;
}

static inline V cos_hemisphere(float u0, float u1, float& pdf) {
  const float ct = std::sqrt(1.0f - u0);
  const float st = std::sqrt(u0);
  const float phi = PI_MUL_2 * u1;
  float sp, cp;
  sincos_f(phi, sp, cp);
  pdf = PI_INV * ct;
  return mk(cp * st, ct, sp * st);
}

struct Mat {
  int32_t type;
  float rho[3];
  float ior;
  float le[3];
};

struct Scene {
  int n = 0;
  std::vector<V> p, nrm;  // 3 per face
  std::vector<V> gn;      // geometric normal
  std::vector<float> area;
  std::vector<V> e1, e2;
  std::vector<Mat> mat;
  std::vector<int> lights;
};

struct Hit {
  float t, u, v;
  int prim;
};

static bool intersect(const Scene& s, V o, V d, float tmin, float tmax, Hit& h) {
  h.prim = -1;
  h.t = tmax;
  h.u = h.v = 0.f;
  for (int f = 0; f < s.n; ++f) {
    const V p0 = s.p[3 * f];
    const V pvec = cross(d, s.e2[f]);
    const float det = dot(s.e1[f], pvec);
    if (!(det != 0.f)) continue;
    const float inv = 1.0f / det;
    const V tvec = sub(o, p0);
    const float u = dot(tvec, pvec) * inv;
    if (!(u >= 0.f && u <= 1.f)) continue;
    const V qvec = cross(tvec, s.e1[f]);
    const float v = dot(d, qvec) * inv;
    if (!(v >= 0.f && u + v <= 1.f)) continue;
    const float t = dot(s.e2[f], qvec) * inv;
    if (!(t == t)) continue;
    if (t >= tmin && t <= h.t && (t < h.t || h.prim < 0)) {
      h.t = t;
      h.u = u;
      h.v = v;
      h.prim = f;
    }
  }
  return h.prim >= 0;
}

struct Surf {
  V pos, ng, ns, dpdu, dpdv;
};

static inline V shading_normal(const Scene& s, int f, float b0, float b1) {
  return add(add(muls(s.nrm[3 * f], 1.0f - b0 - b1), muls(s.nrm[3 * f + 1], b0)),
             muls(s.nrm[3 * f + 2], b1));
}

static Surf surface(const Scene& s, V o, V d, const Hit& h) {
  Surf r;
  r.pos = add(o, muls(d, h.t));
  r.ng = s.gn[h.prim];
  r.ns = shading_normal(s, h.prim, h.u, h.v);
  basis(r.ns, r.dpdu, r.dpdv);
  return r;
}

static inline V rho(const Mat& m) { return mk(m.rho[0], m.rho[1], m.rho[2]); }

static inline V lambert_eval(const Mat& m, V wo, V wi) {
  if (wo.y < 0 || wi.y < 0) return mk(0, 0, 0);
  return divs(rho(m), PI);
}

static inline V reflect(V v, V n) { return add(neg(v), muls(n, 2.0f * dot(v, n))); }

static inline bool refract(V v, V n, float iorI, float iorT, V& t) {
  const V th = muls(sub(v, muls(n, dot(v, n))), -iorI / iorT);
  if (dot(th, th) > 1.0f) return false;
  const V tp = muls(n, -std::sqrt(std::max(1.0f - dot(th, th), 0.0f)));
  t = add(th, tp);
  return true;
}

static inline float fresnel(float c, float iorI, float iorT) {
  const float f0 = (iorI - iorT) * (iorI - iorT) / ((iorI + iorT) * (iorI + iorT));
  const float x = std::max(1.0f - std::fabs(c), 0.0f);
  return f0 + (1.0f - f0) * (x * x * x * x * x);
}

// FROM_LIGHT = 0, FROM_CAMERA = 1
static V sample_bxdf(const Mat& m, V wo, int tdir, Rng& rng, V& wi, float& pdf) {
  if (m.type == 0) {
    float u0, u1;
    rng.next2(u0, u1);
    wi = cos_hemisphere(u0, u1, pdf);
    return lambert_eval(m, wo, wi);
  }
  if (m.type == 1) {
    wi = reflect(wo, mk(0, 1, 0));
    pdf = 1.0f;
    return divs(rho(m), std::fabs(wi.y));
  }
  float iorO, iorI;
  V n;
  if (wo.y > 0) {
    iorO = 1.0f; iorI = m.ior; n = mk(0, 1, 0);
  } else {
    iorO = m.ior; iorI = 1.0f; n = mk(0, -1, 0);
  }
  const float fr = fresnel(dot(wo, n), iorO, iorI);
  if (rng.next() < fr) {
    wi = reflect(wo, n);
    pdf = 1.0f;
    return divs(rho(m), std::fabs(wi.y));
  }
  V tr;
  if (refract(wo, n, iorO, iorI, tr)) {
    wi = tr;
    pdf = 1.0f;
    float sc = 1.0f;
    if (tdir == 1) sc = (iorO * iorO) / (iorI * iorI);
    return divs(muls(rho(m), sc), std::fabs(wi.y));
  }
  wi = reflect(wo, n);
  pdf = 1.0f;
  return divs(rho(m), std::fabs(wi.y));
}

static inline float cos_term(V wo, V wi, V ns, V ng, int tdir) {
  const float wi_ns = dot(wi, ns), wi_ng = dot(wi, ng);
  const float wo_ns = dot(wo, ns), wo_ng = dot(wo, ng);
  if (wi_ng * wi_ns <= 0 || wo_ng * wo_ns <= 0) return 0;
  if (tdir == 1) return std::fabs(wi_ns);
  return std::fabs(wo_ns) * std::fabs(wi_ng) / std::fabs(wo_ng);
}

static Surf sample_point(const Scene& s, int f, Rng& rng, float& pdf) {
  float u0, u1;
  rng.next2(u0, u1);
  const float su0 = std::sqrt(u0);
  const float b0 = 1.0f - su0, b1 = u1 * su0;
  Surf r;
  r.pos = add(add(muls(s.p[3 * f], 1.0f - b0 - b1), muls(s.p[3 * f + 1], b0)),
              muls(s.p[3 * f + 2], b1));
  r.ns = shading_normal(s, f, b0, b1);
  basis(r.ns, r.dpdu, r.dpdv);
  r.ng = s.gn[f];
  pdf = 1.0f / s.area[f];
  return r;
}

static int sample_light(const Scene& s, Rng& rng, float& pdf) {
  unsigned idx = (unsigned)((float)s.lights.size() * rng.next());
  if (idx == s.lights.size()) idx--;
  pdf = 1.0f / (float)s.lights.size();
  return s.lights[idx];
}

}  // namespace orc

using namespace orc;

extern "C" {

void* orc_scene_new(const float* verts, const float* nrms, const void* mats,
                    int64_t n) {
  Scene* s = new Scene();
  s->n = (int)n;
  const Mat* m = (const Mat*)mats;
  for (int64_t f = 0; f < n; ++f) {
    for (int k = 0; k < 3; ++k) {
      s->p.push_back(mk(verts[9 * f + 3 * k], verts[9 * f + 3 * k + 1], verts[9 * f + 3 * k + 2]));
      s->nrm.push_back(mk(nrms[9 * f + 3 * k], nrms[9 * f + 3 * k + 1], nrms[9 * f + 3 * k + 2]));
    }
    const V p1 = s->p[3 * f], p2 = s->p[3 * f + 1], p3 = s->p[3 * f + 2];
    const V c = cross(sub(p2, p1), sub(p3, p1));  // triangle.h:30-33
    s->gn.push_back(normalize(c));
    s->area.push_back(0.5f * length(c));
    s->e1.push_back(sub(p2, p1));
    s->e2.push_back(sub(p3, p1));
    s->mat.push_back(m[f]);
    if (m[f].le[0] > 0 || m[f].le[1] > 0 || m[f].le[2] > 0) s->lights.push_back((int)f);
  }
  return s;
}

void orc_scene_free(void* h) { delete (Scene*)h; }

// rays: 8 floats {origin, tmin, direction, tmax}; out: 4 words {t, u, v, prim}
void orc_intersect(void* h, const float* rays, int64_t n, float* out) {
  const Scene& s = *(const Scene*)h;
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t i = 0; i < n; ++i) {
    const float* r = rays + 8 * i;
    Hit hit;
    const bool ok = intersect(s, mk(r[0], r[1], r[2]), mk(r[4], r[5], r[6]), r[3], r[7], hit);
    float* o = out + 4 * i;
    o[0] = ok ? hit.t : 0.f;
    o[1] = ok ? hit.u : 0.f;
    o[2] = ok ? hit.v : 0.f;
    int32_t prim = ok ? hit.prim : -1;
    std::memcpy(o + 3, &prim, 4);
  }
}

// Photon tracing of integrator.h:393-563 for photons [first, first+count)
// of a trace seeded with `seed`; map 0 = global rule, 1 = caustics rule.
// Writes up to cap photons (9 floats) in (photon, bounce) order; returns the
// number stored (which may exceed cap). status[0..1]: NaN / negative stops.
int64_t orc_trace(void* h, int map, uint64_t seed, int64_t first, int64_t count,
                  int max_depth, float* out, int64_t cap, uint32_t* status) {
  const Scene& s = *(const Scene*)h;
  int64_t stored = 0;
  status[0] = status[1] = 0;
  auto store = [&](V thr, V pos, V wi) {
    if (stored < cap) {
      float* o = out + 9 * stored;
      o[0] = thr.x; o[1] = thr.y; o[2] = thr.z;
      o[3] = pos.x; o[4] = pos.y; o[5] = pos.z;
      o[6] = wi.x; o[7] = wi.y; o[8] = wi.z;
    }
    ++stored;
  };
  for (int64_t i = first; i < first + count; ++i) {
    Rng rng{splitmix64(seed ^ splitmix64((uint64_t)i))};
    float pc, pp, pd;
    const int lf = sample_light(s, rng, pc);
    const Surf ls = sample_point(s, lf, rng, pp);
    float u0, u1;
    rng.next2(u0, u1);
    V dir = to_world(cos_hemisphere(u0, u1, pd), ls.dpdu, ls.ns, ls.dpdv);
    const Mat& lm = s.mat[lf];
    V thr = muls(divs(mk(lm.le[0], lm.le[1], lm.le[2]), pc * pp * pd), std::fabs(dot(dir, ls.ns)));
    V org = ls.pos;
    bool prev_specular = false;
    for (int k = 0; k < max_depth; ++k) {
      if (std::isnan(thr.x) || std::isnan(thr.y) || std::isnan(thr.z)) {
        status[0]++;
        break;
      }
      if (thr.x < 0 || thr.y < 0 || thr.z < 0) {
        status[1]++;
        break;
      }
      Hit hit;
      if (!intersect(s, org, dir, RAY_EPS, 3.40282347e+38f, hit)) break;
      const Surf sf = surface(s, org, dir, hit);
      const Mat& m = s.mat[hit.prim];
      const bool diffuse = m.type == 0;
      if (map == 0) {
        if (diffuse) store(thr, sf.pos, neg(dir));
      } else {
        if (!prev_specular && diffuse) break;
        if (prev_specular && diffuse) {
          store(thr, sf.pos, neg(dir));
          break;
        }
        prev_specular = !diffuse;
      }
      if (k > 0) {
        const float q = std::min(std::max(thr.x, std::max(thr.y, thr.z)), 1.0f);
        if (rng.next() >= q) break;
        thr = divs(thr, q);
      }
      const V wo = neg(dir);
      V wil;
      float pdf;
      const V f = sample_bxdf(m, to_local(wo, sf.dpdu, sf.ns, sf.dpdv), 0, rng, wil, pdf);
      const V wi = to_world(wil, sf.dpdu, sf.ns, sf.dpdv);
      thr = mul(thr, divs(muls(f, cos_term(wo, wi, sf.ns, sf.ng, 0)), pdf));
      org = sf.pos;
      dir = wi;
    }
  }
  return stored;
}

// sin and cos of n float angles with the double-precision evaluation above.
void orc_sincos(const float* x, int64_t n, float* s, float* c) {
  for (int64_t i = 0; i < n; ++i) sincos_f(x[i], s[i], c[i]);
}

}  // extern "C"

// ------------------------------------------------------------ camera pass
// Restatement of examples/main.cpp:33-70 around PhotonMapping::integrate
// (integrator.h:133-377), recursive as in the reference. Photon-map
// queries are exact kNN by brute force (pairs (dist2, index)), summed in
// the reference's heap-pop order (largest pair first), in float.
namespace orc {

struct PhotonSet {
  const float* p;
  int64_t n;
  int64_t emitted;
};

struct RenderCtx {
  const Scene* s;
  PhotonSet global, caustics;
  int kg, kc, fg_depth, max_depth, n_gather;
};

static V estimate(const PhotonSet& pm, int k, const Surf& sf, V wo, const Mat& m) {
  if (pm.n == 0) return mk(0, 0, 0);
  std::vector<std::pair<float, int>> c;
  c.reserve((size_t)pm.n);
  for (int64_t i = 0; i < pm.n; ++i) {
    const float* ph = pm.p + 9 * i;
    float d2 = 0.f;
    d2 += (sf.pos.x - ph[3]) * (sf.pos.x - ph[3]);
    d2 += (sf.pos.y - ph[4]) * (sf.pos.y - ph[4]);
    d2 += (sf.pos.z - ph[5]) * (sf.pos.z - ph[5]);
    if (!std::isnan(d2)) c.push_back({d2, (int)i});
  }
  const size_t kk = std::min<size_t>((size_t)k, c.size());
  std::partial_sort(c.begin(), c.begin() + kk, c.end());
  float maxd2 = 0.f;
  for (size_t r = 0; r < kk; ++r) maxd2 = std::max(maxd2, c[r].first);
  V lo = mk(0, 0, 0);
  const V wo_l = to_local(wo, sf.dpdu, sf.ns, sf.dpdv);
  for (size_t r = kk; r-- > 0;) {
    const float* ph = pm.p + 9 * c[r].second;
    const V wi_l = to_local(mk(ph[6], ph[7], ph[8]), sf.dpdu, sf.ns, sf.dpdv);
    lo = add(lo, mul(lambert_eval(m, wo_l, wi_l), mk(ph[0], ph[1], ph[2])));
  }
  if (kk > 0) lo = divs(lo, (float)pm.emitted * PI * maxd2);
  return lo;
}

static V direct(const RenderCtx& c, const Surf& sf, V wo, const Mat& m, Rng& rng) {
  const Scene& s = *c.s;
  float pc, pp;
  const int lf = sample_light(s, rng, pc);
  const Surf ls = sample_point(s, lf, rng, pp);
  const V wi = normalize(sub(ls.pos, sf.pos));
  const float r = length(sub(ls.pos, sf.pos));
  const float pd = pp * r * r / std::fabs(dot(neg(wi), ls.ns));
  Hit h;
  if (intersect(s, sf.pos, wi, RAY_EPS, r - RAY_EPS, h)) return mk(0, 0, 0);
  const Mat& lm = s.mat[lf];
  const V f = lambert_eval(m, to_local(wo, sf.dpdu, sf.ns, sf.dpdv),
                           to_local(wi, sf.dpdu, sf.ns, sf.dpdv));
  const float cs = std::fabs(dot(wi, sf.ns));
  return divs(mul(muls(f, cs), mk(lm.le[0], lm.le[1], lm.le[2])), pc * pd);
}

static V indirect(const RenderCtx& c, V wo, const Surf& sf, const Mat& m, Rng& rng,
                  int depth) {
  if (depth >= c.max_depth) return mk(0, 0, 0);
  V wil;
  float pdf;
  const V f = sample_bxdf(m, to_local(wo, sf.dpdu, sf.ns, sf.dpdv), 1, rng, wil, pdf);
  const V dir = to_world(wil, sf.dpdu, sf.ns, sf.dpdv);
  const float cs = std::fabs(dot(sf.ns, dir));
  Hit h;
  if (!intersect(*c.s, sf.pos, dir, RAY_EPS, 3.40282347e+38f, h)) return mk(0, 0, 0);
  const Surf s2 = surface(*c.s, sf.pos, dir, h);
  const Mat& m2 = c.s->mat[h.prim];
  V x;
  if (m2.type == 0)
    x = estimate(c.global, c.kg, s2, neg(dir), m2);
  else
    x = indirect(c, neg(dir), s2, m2, rng, depth + 1);
  return divs(mul(muls(f, cs), x), pdf);
}

static V integrate(const RenderCtx& c, V o, V d, Rng& rng, int depth) {
  if (depth >= c.max_depth) return mk(0, 0, 0);
  Hit h;
  if (!intersect(*c.s, o, d, RAY_EPS, 3.40282347e+38f, h)) return mk(0, 0, 0);
  const Surf sf = surface(*c.s, o, d, h);
  const Mat& m = c.s->mat[h.prim];
  if (m.le[0] > 0 || m.le[1] > 0 || m.le[2] > 0) return mk(m.le[0], m.le[1], m.le[2]);
  const V wo = neg(d);
  if (m.type == 0) {
    if (depth >= c.fg_depth) return estimate(c.global, c.kg, sf, wo, m);
    const V ld = direct(c, sf, wo, m, rng);
    const V lc = estimate(c.caustics, c.kc, sf, wo, m);
    V li = mk(0, 0, 0);
    const float ig = 1.0f / (float)c.n_gather;
    for (int g = 0; g < c.n_gather; ++g) li = add(li, muls(indirect(c, wo, sf, m, rng, 0), ig));
    return add(add(ld, lc), li);
  }
  const V wo_l = to_local(wo, sf.dpdu, sf.ns, sf.dpdv);
  if (depth >= 3) {
    V wil;
    float pdf;
    const V f = sample_bxdf(m, wo_l, 1, rng, wil, pdf);
    const V wi = to_world(wil, sf.dpdu, sf.ns, sf.dpdv);
    const V thr = divs(muls(f, cos_term(wo, wi, sf.ns, sf.ng, 1)), pdf);
    return mul(thr, integrate(c, sf.pos, wi, rng, depth + 1));
  }
  // sampleAllBxDF
  V dirs[2], fs[2];
  int nb = 0;
  if (m.type == 1) {
    dirs[0] = reflect(wo_l, mk(0, 1, 0));
    fs[0] = divs(rho(m), std::fabs(dirs[0].y));
    nb = 1;
  } else {
    float iorO, iorI;
    V n;
    if (wo_l.y > 0) { iorO = 1.0f; iorI = m.ior; n = mk(0, 1, 0); }
    else { iorO = m.ior; iorI = 1.0f; n = mk(0, -1, 0); }
    const float fr = fresnel(dot(wo_l, n), iorO, iorI);
    dirs[0] = reflect(wo_l, n);
    fs[0] = divs(muls(rho(m), fr), std::fabs(dirs[0].y));
    nb = 1;
    V tr;
    if (refract(wo_l, n, iorO, iorI, tr)) {
      const float sc = (iorO * iorO) / (iorI * iorI);
      dirs[1] = tr;
      fs[1] = divs(muls(rho(m), (1.0f - fr) * sc), std::fabs(tr.y));
      nb = 2;
    } else {
      fs[0] = divs(rho(m), std::fabs(dirs[0].y));
    }
  }
  V lo = mk(0, 0, 0);
  for (int b = 0; b < nb; ++b) {
    const V wi = to_world(dirs[b], sf.dpdu, sf.ns, sf.dpdv);
    const V thr = muls(fs[b], std::fabs(dot(wi, sf.ns)));
    lo = add(lo, mul(thr, integrate(c, sf.pos, wi, rng, depth + 1)));
  }
  return lo;
}

}  // namespace orc

extern "C" {

// cam: 13 floats {position, forward, right, up, focal_length};
// iprm: {width, height, spp, k_global, k_caustics, fg_depth, max_depth,
// n_gather}; out: height x width x 3; dropped[0..1]: NaN / negative.
void orc_render(void* h, const float* gph, int64_t gn, int64_t g_emitted,
                const float* cph, int64_t cn, int64_t c_emitted, const float* cam,
                const int32_t* iprm, float* out, int64_t* dropped) {
  RenderCtx c;
  c.s = (const Scene*)h;
  c.global = PhotonSet{gph, gn, g_emitted};
  c.caustics = PhotonSet{cph, cn, c_emitted};
  const int W = iprm[0], H = iprm[1], spp = iprm[2];
  c.kg = iprm[3];
  c.kc = iprm[4];
  c.fg_depth = iprm[5];
  c.max_depth = iprm[6];
  c.n_gather = iprm[7];
  const V pos = mk(cam[0], cam[1], cam[2]), fwd = mk(cam[3], cam[4], cam[5]);
  const V right = mk(cam[6], cam[7], cam[8]), up = mk(cam[9], cam[10], cam[11]);
  const float focal = cam[12];
  int64_t dn = 0, dneg = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : dn, dneg)
  for (int p = 0; p < W * H; ++p) {
    const int i = p / W, j = p % W;
    Rng rng{(uint64_t)(j + W * i)};
    V acc = mk(0, 0, 0);
    for (int k = 0; k < spp; ++k) {
      const float u = (2.0f * (j + rng.next()) - W) / H;
      const float v = (2.0f * (i + rng.next()) - H) / H;
      const V pinhole = add(pos, muls(fwd, focal));
      const V sensor = add(add(pos, muls(right, u)), muls(up, v));
      const V rad = integrate(c, sensor, normalize(sub(pinhole, sensor)), rng, 0);
      if (std::isnan(rad.x) || std::isnan(rad.y) || std::isnan(rad.z)) { ++dn; continue; }
      if (rad.x < 0 || rad.y < 0 || rad.z < 0) { ++dneg; continue; }
      acc = add(acc, rad);
    }
    const float k = (float)spp;
    out[3 * p] = acc.x / k;
    out[3 * p + 1] = acc.y / k;
    out[3 * p + 2] = acc.z / k;
  }
  dropped[0] = dn;
  dropped[1] = dneg;
}

}  // extern "C"

extern "C" {

// PathTracing::integrate (integrator.h:60-105) in the loop of
// tests/test_path_tracing.cpp:25-52.
void orc_render_pt(void* h, const float* cam, int W, int H, int spp, int max_depth,
                   float* out, int64_t* dropped) {
  const Scene& s = *(const Scene*)h;
  const V pos = mk(cam[0], cam[1], cam[2]), fwd = mk(cam[3], cam[4], cam[5]);
  const V right = mk(cam[6], cam[7], cam[8]), up = mk(cam[9], cam[10], cam[11]);
  const float focal = cam[12];
  int64_t dn = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : dn)
  for (int p = 0; p < W * H; ++p) {
    const int i = p / W, j = p % W;
    Rng rng{(uint64_t)(j + W * i)};
    V acc = mk(0, 0, 0);
    for (int smp = 0; smp < spp; ++smp) {
      const float u = (2.0f * (j + rng.next()) - W) / H;
      const float v = (2.0f * (i + rng.next()) - H) / H;
      const V pinhole = add(pos, muls(fwd, focal));
      const V sensor = add(add(pos, muls(right, u)), muls(up, v));
      V o = sensor, d = normalize(sub(pinhole, sensor));
      V rad = mk(0, 0, 0), thr = mk(1, 1, 1);
      for (int k = 0; k < max_depth; ++k) {
        Hit hit;
        if (!intersect(s, o, d, RAY_EPS, 3.40282347e+38f, hit)) break;
        const Surf sf = surface(s, o, d, hit);
        const Mat& m = s.mat[hit.prim];
        if (k > 0) {
          const float q = std::min(std::max(thr.x, std::max(thr.y, thr.z)), 1.0f);
          if (rng.next() >= q) break;
          thr = divs(thr, q);
        }
        if (m.le[0] > 0 || m.le[1] > 0 || m.le[2] > 0)
          rad = add(rad, mul(thr, mk(m.le[0], m.le[1], m.le[2])));
        const V wo = neg(d);
        V wil;
        float pdf;
        const V f = sample_bxdf(m, to_local(wo, sf.dpdu, sf.ns, sf.dpdv), 1, rng, wil, pdf);
        const V wi = to_world(wil, sf.dpdu, sf.ns, sf.dpdv);
        thr = mul(thr, divs(muls(f, cos_term(wo, wi, sf.ns, sf.ng, 1)), pdf));
        o = sf.pos;
        d = wi;
      }
      if (std::isnan(rad.x) || std::isnan(rad.y) || std::isnan(rad.z)) {
        ++dn;
        continue;
      }
      acc = add(acc, rad);
    }
    const float k = (float)(spp > 0 ? spp : 1);
    out[3 * p] = acc.x / k;
    out[3 * p + 1] = acc.y / k;
    out[3 * p + 2] = acc.z / k;
  }
  *dropped = dn;
}

}  // extern "C"

extern "C" {

// PhotonMapping::integrate for n given rays (6 floats each) and sampler
// states (advanced in place); iprm as in orc_render from k_global on:
// {k_global, k_caustics, fg_depth, max_depth, n_gather}.
void orc_integrate(void* h, const float* gph, int64_t gn, int64_t g_emitted,
                   const float* cph, int64_t cn, int64_t c_emitted, const float* rays,
                   int64_t n, uint64_t* states, const int32_t* iprm, float* out) {
  RenderCtx c;
  c.s = (const Scene*)h;
  c.global = PhotonSet{gph, gn, g_emitted};
  c.caustics = PhotonSet{cph, cn, c_emitted};
  c.kg = iprm[0];
  c.kc = iprm[1];
  c.fg_depth = iprm[2];
  c.max_depth = iprm[3];
  c.n_gather = iprm[4];
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t i = 0; i < n; ++i) {
    Rng rng{states[i]};
    const float* r = rays + 6 * i;
    const V rad = integrate(c, mk(r[0], r[1], r[2]), mk(r[3], r[4], r[5]), rng, 0);
    out[3 * i] = rad.x;
    out[3 * i + 1] = rad.y;
    out[3 * i + 2] = rad.z;
    states[i] = rng.state;
  }
}

}  // extern "C"

// ------------------------------------------------ gradient (forward mode)
// FP64 CPU derivative of the image loss of the camera pass above with
// respect to per-face albedo parameters and the light emission, by forward
// differentiation: every throughput and radiance value carries, in double,
// its derivative with respect to each parameter channel (albedos only
// affect their own colour channel, so one derivative per parameter and
// channel). Values themselves are computed in float exactly as above, so
// the paths, the kNN sets and the dropped samples are the render's.
// Russian-roulette decisions use the values (the derivative is that of the
// estimator with these decisions held).
namespace orc {

constexpr int kGMax = 33;  // albedo parameters + emission

struct DV {
  V v;
  double d[kGMax][3];
};

struct GradCtx {
  RenderCtx rc;
  const int* pid;  // per face
  int np;          // albedo parameters; slot np is the emission
  int nd;          // np + 1
  const double* gtan;  // global photons' tangents, nd * 3 per photon
  const double* ctan;  // caustics photons' tangents
};

static inline void dv_zero(DV& a, int nd) {
  a.v = mk(0, 0, 0);
  for (int x = 0; x < nd; ++x) a.d[x][0] = a.d[x][1] = a.d[x][2] = 0.0;
}

// a.d += s (per channel) * b.d
static inline void dv_axpy(DV& a, const double s[3], const DV& b, int nd) {
  for (int x = 0; x < nd; ++x)
    for (int c = 0; c < 3; ++c) a.d[x][c] += s[c] * b.d[x][c];
}

static inline double comp(V v, int c) { return c == 0 ? v.x : (c == 1 ? v.y : v.z); }

// Photon tracing with tangents (both rules), photons stored in (photon,
// bounce) order with nd * 3 doubles each.
static void trace_tan(const Scene& s, const int* pid, int nd, int map, uint64_t seed,
                      int64_t n_emit, int max_depth, std::vector<float>& ph,
                      std::vector<double>& tan) {
  const int np = nd - 1;
  std::vector<double> t((size_t)nd * 3);
  for (int64_t i = 0; i < n_emit; ++i) {
    Rng rng{splitmix64(seed ^ splitmix64((uint64_t)i))};
    float pc, pp, pd;
    const int lf = sample_light(s, rng, pc);
    const Surf ls = sample_point(s, lf, rng, pp);
    float u0, u1;
    rng.next2(u0, u1);
    V dir = to_world(cos_hemisphere(u0, u1, pd), ls.dpdu, ls.ns, ls.dpdv);
    const Mat& lm = s.mat[lf];
    V thr = muls(divs(mk(lm.le[0], lm.le[1], lm.le[2]), pc * pp * pd), std::fabs(dot(dir, ls.ns)));
    std::fill(t.begin(), t.end(), 0.0);
    const double dle = 1.0 / ((double)pc * pp * pd) * std::fabs((double)dot(dir, ls.ns));
    for (int c = 0; c < 3; ++c) t[3 * np + c] = dle;
    V org = ls.pos;
    bool prev_specular = false;
    for (int k = 0; k < max_depth; ++k) {
      if (std::isnan(thr.x) || std::isnan(thr.y) || std::isnan(thr.z)) break;
      if (thr.x < 0 || thr.y < 0 || thr.z < 0) break;
      Hit hit;
      if (!intersect(s, org, dir, RAY_EPS, 3.40282347e+38f, hit)) break;
      const Surf sf = surface(s, org, dir, hit);
      const Mat& m = s.mat[hit.prim];
      const bool diffuse = m.type == 0;
      bool store = false, stop = false;
      if (map == 0) {
        store = diffuse;
      } else {
        if (!prev_specular && diffuse) break;
        if (prev_specular && diffuse) store = stop = true;
        prev_specular = !diffuse;
      }
      if (store) {
        const V wi = neg(dir);
        const float rec[9] = {thr.x, thr.y, thr.z, sf.pos.x, sf.pos.y, sf.pos.z, wi.x, wi.y, wi.z};
        ph.insert(ph.end(), rec, rec + 9);
        tan.insert(tan.end(), t.begin(), t.end());
      }
      if (stop) break;
      double qinv = 1.0;
      if (k > 0) {
        const float q = std::min(std::max(thr.x, std::max(thr.y, thr.z)), 1.0f);
        if (rng.next() >= q) break;
        thr = divs(thr, q);
        qinv = 1.0 / (double)q;
      }
      const V wo = neg(dir);
      V wil;
      float pdf;
      const V wol = to_local(wo, sf.dpdu, sf.ns, sf.dpdv);
      const V f = sample_bxdf(m, wol, 0, rng, wil, pdf);
      const V wi = to_world(wil, sf.dpdu, sf.ns, sf.dpdv);
      const float ct = cos_term(wo, wi, sf.ns, sf.ng, 0);
      // thr' = (thr / q) f ct / pdf: the tangent t (not yet divided by q)
      // becomes t f ct / (pdf q) + (thr / q) (d f / d albedo) ct / pdf
      const int p = pid[hit.prim];
      const bool valid = diffuse && !(wol.y < 0 || wil.y < 0);
      for (int x = 0; x < nd; ++x)
        for (int c = 0; c < 3; ++c) t[3 * x + c] *= comp(f, c) * (double)ct / (double)pdf * qinv;
      if (p >= 0 && valid)
        for (int c = 0; c < 3; ++c)
          t[3 * p + c] += comp(thr, c) * (1.0 / (double)PI) * (double)ct / (double)pdf;
      thr = mul(thr, divs(muls(f, ct), pdf));
      org = sf.pos;
      dir = wi;
    }
  }
}

// Lambert f at a surface of material m with parameter p: value (float, as
// lambert_eval) and d f_c / d albedo_c = 1/pi when the directions pass.
static DV estimate_d(const GradCtx& g, const PhotonSet& pm, const double* tan, int k,
                     const Surf& sf, V wo, const Mat& m, int p) {
  DV r;
  dv_zero(r, g.nd);
  if (pm.n == 0) return r;
  std::vector<std::pair<float, int>> c;
  c.reserve((size_t)pm.n);
  for (int64_t i = 0; i < pm.n; ++i) {
    const float* ph = pm.p + 9 * i;
    float d2 = 0.f;
    d2 += (sf.pos.x - ph[3]) * (sf.pos.x - ph[3]);
    d2 += (sf.pos.y - ph[4]) * (sf.pos.y - ph[4]);
    d2 += (sf.pos.z - ph[5]) * (sf.pos.z - ph[5]);
    if (!std::isnan(d2)) c.push_back({d2, (int)i});
  }
  const size_t kk = std::min<size_t>((size_t)k, c.size());
  std::partial_sort(c.begin(), c.begin() + kk, c.end());
  float maxd2 = 0.f;
  for (size_t q = 0; q < kk; ++q) maxd2 = std::max(maxd2, c[q].first);
  V lo = mk(0, 0, 0);
  const V wo_l = to_local(wo, sf.dpdu, sf.ns, sf.dpdv);
  for (size_t q = kk; q-- > 0;) {
    const int idx = c[q].second;
    const float* ph = pm.p + 9 * idx;
    const V wi_l = to_local(mk(ph[6], ph[7], ph[8]), sf.dpdu, sf.ns, sf.dpdv);
    const V f = lambert_eval(m, wo_l, wi_l);
    lo = add(lo, mul(f, mk(ph[0], ph[1], ph[2])));
    const bool valid = !(wo_l.y < 0 || wi_l.y < 0);
    if (!valid) continue;
    const double* t = tan + (size_t)idx * 3 * g.nd;
    for (int x = 0; x < g.nd; ++x)
      for (int ch = 0; ch < 3; ++ch) r.d[x][ch] += comp(f, ch) * t[3 * x + ch];
    if (p >= 0)
      for (int ch = 0; ch < 3; ++ch) r.d[p][ch] += (1.0 / (double)PI) * (double)ph[ch];
  }
  if (kk > 0) {
    const float den = (float)pm.emitted * PI * maxd2;
    lo = divs(lo, den);
    for (int x = 0; x < g.nd; ++x)
      for (int ch = 0; ch < 3; ++ch) r.d[x][ch] /= (double)den;
  }
  r.v = lo;
  return r;
}

static DV direct_d(const GradCtx& g, const Surf& sf, V wo, const Mat& m, int p, Rng& rng) {
  const Scene& s = *g.rc.s;
  DV r;
  dv_zero(r, g.nd);
  float pc, pp;
  const int lf = sample_light(s, rng, pc);
  const Surf ls = sample_point(s, lf, rng, pp);
  const V wi = normalize(sub(ls.pos, sf.pos));
  const float rr = length(sub(ls.pos, sf.pos));
  const float pd = pp * rr * rr / std::fabs(dot(neg(wi), ls.ns));
  Hit h;
  if (intersect(s, sf.pos, wi, RAY_EPS, rr - RAY_EPS, h)) return r;
  const Mat& lm = s.mat[lf];
  const V wol = to_local(wo, sf.dpdu, sf.ns, sf.dpdv), wil = to_local(wi, sf.dpdu, sf.ns, sf.dpdv);
  const V f = lambert_eval(m, wol, wil);
  const float cs = std::fabs(dot(wi, sf.ns));
  const V le = mk(lm.le[0], lm.le[1], lm.le[2]);
  r.v = divs(mul(muls(f, cs), le), pc * pd);
  const double k = (double)cs / ((double)pc * (double)pd);
  for (int c = 0; c < 3; ++c) r.d[g.np][c] = comp(f, c) * k;  // d / d Le_c
  if (p >= 0 && !(wol.y < 0 || wil.y < 0))
    for (int c = 0; c < 3; ++c) r.d[p][c] += (1.0 / (double)PI) * k * comp(le, c);
  return r;
}

static DV indirect_d(const GradCtx& g, V wo, const Surf& sf, const Mat& m, int p, Rng& rng,
                     int depth) {
  DV r;
  dv_zero(r, g.nd);
  const RenderCtx& c = g.rc;
  if (depth >= c.max_depth) return r;
  V wil;
  float pdf;
  const V wol = to_local(wo, sf.dpdu, sf.ns, sf.dpdv);
  const V f = sample_bxdf(m, wol, 1, rng, wil, pdf);
  const V dir = to_world(wil, sf.dpdu, sf.ns, sf.dpdv);
  const float cs = std::fabs(dot(sf.ns, dir));
  Hit h;
  if (!intersect(*c.s, sf.pos, dir, RAY_EPS, 3.40282347e+38f, h)) return r;
  const Surf s2 = surface(*c.s, sf.pos, dir, h);
  const Mat& m2 = c.s->mat[h.prim];
  DV x;
  if (m2.type == 0)
    x = estimate_d(g, c.global, g.gtan, c.kg, s2, neg(dir), m2, g.pid[h.prim]);
  else
    x = indirect_d(g, neg(dir), s2, m2, g.pid[h.prim], rng, depth + 1);
  r.v = divs(mul(muls(f, cs), x.v), pdf);
  double s3[3];
  for (int ch = 0; ch < 3; ++ch) s3[ch] = comp(f, ch) * (double)cs / (double)pdf;
  dv_axpy(r, s3, x, g.nd);
  if (p >= 0 && m.type == 0 && !(wol.y < 0 || wil.y < 0))
    for (int ch = 0; ch < 3; ++ch)
      r.d[p][ch] += (1.0 / (double)PI) * (double)cs / (double)pdf * comp(x.v, ch);
  return r;
}

static DV integrate_d(const GradCtx& g, V o, V d, Rng& rng, int depth) {
  DV r;
  dv_zero(r, g.nd);
  const RenderCtx& c = g.rc;
  if (depth >= c.max_depth) return r;
  Hit h;
  if (!intersect(*c.s, o, d, RAY_EPS, 3.40282347e+38f, h)) return r;
  const Surf sf = surface(*c.s, o, d, h);
  const Mat& m = c.s->mat[h.prim];
  const int p = g.pid[h.prim];
  if (m.le[0] > 0 || m.le[1] > 0 || m.le[2] > 0) {
    r.v = mk(m.le[0], m.le[1], m.le[2]);
    for (int ch = 0; ch < 3; ++ch) r.d[g.np][ch] = 1.0;
    return r;
  }
  const V wo = neg(d);
  if (m.type == 0) {
    if (depth >= c.fg_depth) return estimate_d(g, c.global, g.gtan, c.kg, sf, wo, m, p);
    const DV ld = direct_d(g, sf, wo, m, p, rng);
    const DV lc = estimate_d(g, c.caustics, g.ctan, c.kc, sf, wo, m, p);
    DV li;
    dv_zero(li, g.nd);
    const float ig = 1.0f / (float)c.n_gather;
    const double one[3] = {1.0, 1.0, 1.0}, igd[3] = {ig, ig, ig};
    for (int gi = 0; gi < c.n_gather; ++gi) {
      const DV x = indirect_d(g, wo, sf, m, p, rng, 0);
      li.v = add(li.v, muls(x.v, ig));
      dv_axpy(li, igd, x, g.nd);
    }
    r.v = add(add(ld.v, lc.v), li.v);
    dv_axpy(r, one, ld, g.nd);
    dv_axpy(r, one, lc, g.nd);
    dv_axpy(r, one, li, g.nd);
    return r;
  }
  const V wo_l = to_local(wo, sf.dpdu, sf.ns, sf.dpdv);
  if (depth >= 3) {
    V wil;
    float pdf;
    const V f = sample_bxdf(m, wo_l, 1, rng, wil, pdf);
    const V wi = to_world(wil, sf.dpdu, sf.ns, sf.dpdv);
    const V thr = divs(muls(f, cos_term(wo, wi, sf.ns, sf.ng, 1)), pdf);
    const DV x = integrate_d(g, sf.pos, wi, rng, depth + 1);
    r.v = mul(thr, x.v);
    const double s3[3] = {thr.x, thr.y, thr.z};
    dv_axpy(r, s3, x, g.nd);
    return r;
  }
  V dirs[2], fs[2];
  int nb = 0;
  if (m.type == 1) {
    dirs[0] = reflect(wo_l, mk(0, 1, 0));
    fs[0] = divs(rho(m), std::fabs(dirs[0].y));
    nb = 1;
  } else {
    float iorO, iorI;
    V n;
    if (wo_l.y > 0) { iorO = 1.0f; iorI = m.ior; n = mk(0, 1, 0); }
    else { iorO = m.ior; iorI = 1.0f; n = mk(0, -1, 0); }
    const float fr = fresnel(dot(wo_l, n), iorO, iorI);
    dirs[0] = reflect(wo_l, n);
    fs[0] = divs(muls(rho(m), fr), std::fabs(dirs[0].y));
    nb = 1;
    V tr;
    if (refract(wo_l, n, iorO, iorI, tr)) {
      const float sc = (iorO * iorO) / (iorI * iorI);
      dirs[1] = tr;
      fs[1] = divs(muls(rho(m), (1.0f - fr) * sc), std::fabs(tr.y));
      nb = 2;
    } else {
      fs[0] = divs(rho(m), std::fabs(dirs[0].y));
    }
  }
  for (int b = 0; b < nb; ++b) {
    const V wi = to_world(dirs[b], sf.dpdu, sf.ns, sf.dpdv);
    const V thr = muls(fs[b], std::fabs(dot(wi, sf.ns)));
    const DV x = integrate_d(g, sf.pos, wi, rng, depth + 1);
    r.v = add(r.v, mul(thr, x.v));
    const double s3[3] = {thr.x, thr.y, thr.z};
    dv_axpy(r, s3, x, g.nd);
  }
  return r;
}

}  // namespace orc

extern "C" {

// Traces both maps (global: seed; caustics, with final gathering: seed + 1)
// and renders like orc_render, and returns out_grad[(np + 1) * 3]: d loss /
// d albedo parameter (np x 3) then d loss / d emission (3), for
// d loss / d image = grad_img (height x width x 3). pid: parameter of each
// face (-1: none). out_img receives the image.
// iprm: {width, height, spp, k, fg_depth, max_depth, n_gather}.
void orc_grad(void* h, const int32_t* pid, int np, uint64_t seed, int64_t n_global,
              int64_t n_caustic, const float* cam, const int32_t* iprm,
              const float* grad_img, double* out_grad, float* out_img) {
  const Scene& s = *(const Scene*)h;
  const int nd = np + 1;
  const int W = iprm[0], H = iprm[1], spp = iprm[2];
  std::vector<float> gph, cph;
  std::vector<double> gtan, ctan;
  trace_tan(s, pid, nd, 0, seed, n_global, iprm[5], gph, gtan);
  if (iprm[4] > 0) trace_tan(s, pid, nd, 1, seed + 1, n_caustic, iprm[5], cph, ctan);
  GradCtx g;
  g.rc.s = &s;
  g.rc.global = PhotonSet{gph.data(), (int64_t)(gph.size() / 9), n_global};
  g.rc.caustics = PhotonSet{cph.data(), (int64_t)(cph.size() / 9), n_caustic};
  g.rc.kg = g.rc.kc = iprm[3];
  g.rc.fg_depth = iprm[4];
  g.rc.max_depth = iprm[5];
  g.rc.n_gather = iprm[6];
  g.pid = pid;
  g.np = np;
  g.nd = nd;
  g.gtan = gtan.data();
  g.ctan = ctan.data();
  const V pos = mk(cam[0], cam[1], cam[2]), fwd = mk(cam[3], cam[4], cam[5]);
  const V right = mk(cam[6], cam[7], cam[8]), up = mk(cam[9], cam[10], cam[11]);
  const float focal = cam[12];
  std::vector<double> acc((size_t)nd * 3, 0.0);
#pragma omp parallel
  {
    std::vector<double> mine((size_t)nd * 3, 0.0);
#pragma omp for schedule(dynamic, 1)
    for (int p = 0; p < W * H; ++p) {
      const int i = p / W, j = p % W;
      Rng rng{(uint64_t)(j + W * i)};
      V a = mk(0, 0, 0);
      for (int k = 0; k < spp; ++k) {
        const float u = (2.0f * (j + rng.next()) - W) / H;
        const float v = (2.0f * (i + rng.next()) - H) / H;
        const V pinhole = add(pos, muls(fwd, focal));
        const V sensor = add(add(pos, muls(right, u)), muls(up, v));
        const DV rad = integrate_d(g, sensor, normalize(sub(pinhole, sensor)), rng, 0);
        const V rv = rad.v;
        if (std::isnan(rv.x) || std::isnan(rv.y) || std::isnan(rv.z)) continue;
        if (rv.x < 0 || rv.y < 0 || rv.z < 0) continue;
        a = add(a, rv);
        for (int x = 0; x < nd; ++x)
          for (int c = 0; c < 3; ++c)
            mine[3 * x + c] += (double)grad_img[3 * p + c] / (double)spp * rad.d[x][c];
      }
      out_img[3 * p] = a.x / (float)spp;
      out_img[3 * p + 1] = a.y / (float)spp;
      out_img[3 * p + 2] = a.z / (float)spp;
    }
#pragma omp critical
    for (size_t t = 0; t < acc.size(); ++t) acc[t] += mine[t];
  }
  for (size_t t = 0; t < acc.size(); ++t) out_grad[t] = acc[t];
}

}  // extern "C"
