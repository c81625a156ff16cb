// Device math of the renderer, written to round exactly like the
// reference's float code (compiled here with -fmad=false): every helper
// evaluates its expression in the reference's order.
//
//   core.h:193-247   Vec3 ops, dot, cross, normalize, orthonormalBasis,
//                    worldToLocal, localToWorld
//   sampler.h:11-91  PCG32 RNG and sampleCosineHemisphere
//   material.h       Lambert / Mirror / Glass
//   integrator.h:25-46  cosTerm
#pragma once

#include "pm_common.cuh"

namespace pm {

struct V3 {
  float x, y, z;
};

__host__ __device__ __forceinline__ V3 v3(float x, float y, float z) {
  return V3{x, y, z};
}
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ V3 operator*(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ V3 operator*(V3 a, float k) { return v3(a.x * k, a.y * k, a.z * k); }
__device__ __forceinline__ V3 operator*(float k, V3 a) { return v3(a.x * k, a.y * k, a.z * k); }
__device__ __forceinline__ V3 operator/(V3 a, float k) { return v3(a.x / k, a.y / k, a.z / k); }
__device__ __forceinline__ V3 operator/(V3 a, V3 b) { return v3(a.x / b.x, a.y / b.y, a.z / b.z); }
__device__ __forceinline__ float comp(V3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

// core.h:200-203
__device__ __forceinline__ float dot(V3 a, V3 b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}
// core.h:206-209
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
  return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
// core.h:214-216
__device__ __forceinline__ float length(V3 v) { return sqrtf(dot(v, v)); }
__device__ __forceinline__ float length2(V3 v) { return dot(v, v); }
__device__ __forceinline__ V3 normalize(V3 v) { return v / length(v); }

// core.h:224-231
__device__ __forceinline__ void orthonormal_basis(V3 n, V3& t, V3& b) {
  if (fabsf(n.y) < 0.9f)
    t = normalize(cross(n, v3(0.f, 1.f, 0.f)));
  else
    t = normalize(cross(n, v3(0.f, 0.f, -1.f)));
  b = normalize(cross(t, n));
}
// core.h:234-237
__device__ __forceinline__ V3 world_to_local(V3 v, V3 lx, V3 ly, V3 lz) {
  return v3(dot(v, lx), dot(v, ly), dot(v, lz));
}
// core.h:240-247: ret[i] = v0*lx[i] + v1*ly[i] + v2*lz[i]
__device__ __forceinline__ V3 local_to_world(V3 v, V3 lx, V3 ly, V3 lz) {
  return v3(v.x * lx.x + v.y * ly.x + v.z * lz.x,
            v.x * lx.y + v.y * ly.y + v.z * lz.y,
            v.x * lx.z + v.y * ly.z + v.z * lz.z);
}

__device__ __forceinline__ bool has_nan(V3 a) {
  return isnan(a.x) || isnan(a.y) || isnan(a.z);
}

// ------------------------------------------------------------------ RNG
// sampler.h:11-47: PCG32 XSH-RR with state = seed, inc = 1; getNext =
// u32 * (1.0f / UINT32_MAX) in float, so 1.0 is reachable.
struct Rng {
  unsigned long long state;
  __device__ __forceinline__ uint32_t next_u32() {
    const unsigned long long old = state;
    state = old * 6364136223846793005ull + 1ull;
    const uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    const uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((0u - rot) & 31u));
  }
  __device__ __forceinline__ float next1d() {
    return (float)next_u32() * (1.0f / 4294967295.0f);
  }
  // UniformSampler::getNext2D builds Vec2f(rng.getNext(), rng.getNext());
  // the reference's compiler (GCC, x86-64) evaluates those two arguments
  // right to left, so the first draw lands in v[1] and the second in v[0].
  __device__ __forceinline__ void next2d(float& u0, float& u1) {
    u1 = next1d();
    u0 = next1d();
  }
};

// ------------------------------------------------------ sin/cos, float
// sin and cos of a float angle |x| <= 8 in float arithmetic only, each
// operation rounded on its own (the CPU oracle runs the same sequence):
//   * Cody-Waite reduction: q = rint(x 2/pi), r = x - q pi/2 with pi/2
//     split in three floats (21 + 21 + 24 significant bits), so q*hi and
//     q*mid are exact for |q| <= 7 and x - q*hi is exact (Sterbenz);
//   * Taylor polynomials on |r| <= pi/4, Horner form: sin to r^9, cos to
//     r^10 (truncation below 3e-9 relative), coefficients 1/n! rounded to
//     float;
//   * the quadrant q mod 4 picks +-sin r / +-cos r.
// Measured against double-precision sin/cos over [-8, 8]: at most 1.5 ulp.
constexpr float kTwoOverPiF = 0x1.45f306p-1f;
constexpr float kPio2Hi = 0x1.921fbp+0f;
constexpr float kPio2Mid = 0x1.5110bp-22f;
constexpr float kPio2Lo = 0x1.184698p-44f;
__device__ __forceinline__ void sincos_f32(float x, float& s, float& c) {
  const float q = rintf(__fmul_rn(x, kTwoOverPiF));
  float r = __fsub_rn(x, __fmul_rn(q, kPio2Hi));
  r = __fsub_rn(r, __fmul_rn(q, kPio2Mid));
  r = __fsub_rn(r, __fmul_rn(q, kPio2Lo));
  const float r2 = __fmul_rn(r, r);
  float ps = 1.0f / 362880.0f;
  ps = __fadd_rn(__fmul_rn(ps, r2), -1.0f / 5040.0f);
  ps = __fadd_rn(__fmul_rn(ps, r2), 1.0f / 120.0f);
  ps = __fadd_rn(__fmul_rn(ps, r2), -1.0f / 6.0f);
  const float sr = __fadd_rn(r, __fmul_rn(__fmul_rn(r, r2), ps));
  float pc = -1.0f / 3628800.0f;
  pc = __fadd_rn(__fmul_rn(pc, r2), 1.0f / 40320.0f);
  pc = __fadd_rn(__fmul_rn(pc, r2), -1.0f / 720.0f);
  pc = __fadd_rn(__fmul_rn(pc, r2), 1.0f / 24.0f);
  pc = __fadd_rn(__fmul_rn(pc, r2), -0.5f);
  const float cr = __fadd_rn(1.0f, __fmul_rn(r2, pc));
  const int quad = ((int)q) & 3;
  s = quad == 0 ? sr : quad == 1 ? cr : quad == 2 ? -sr : -cr;
  c = quad == 0 ? cr : quad == 1 ? -sr : quad == 2 ? -cr : sr;
}

// constants of core.h:7-17
constexpr float kPI_INV = 1.0f / kPI;
constexpr float kPI_MUL_2 = 2.0f * kPI;

// sampler.h:84-91, sampleCosineHemisphere. theta = acos(1 - 2u)/2 gives
// cos(theta) = sqrt(1 - u) and sin(theta) = sqrt(u) exactly; the closed
// forms are used (they need no inverse trigonometry), phi = 2 PI u1.
__device__ __forceinline__ V3 sample_cos_hemisphere(float u0, float u1,
                                                    float& pdf) {
  const float ct = sqrtf(1.0f - u0);
  const float st = sqrtf(u0);
  const float phi = kPI_MUL_2 * u1;
  float sp, cp;
  sincos_f32(phi, sp, cp);
  pdf = kPI_INV * ct;
  // core.h:250-253 sphericalToCartesian
  return v3(cp * st, ct, sp * st);
}

// ------------------------------------------------------------- materials
enum MatType { kLambert = 0, kMirror = 1, kGlass = 2 };
enum TransportDir { kFromLight = 0, kFromCamera = 1 };

struct Material {
  int type;
  float rho[3];
  float ior;
  float le[3];
};

__device__ __forceinline__ V3 mat_rho(const Material& m) {
  return v3(m.rho[0], m.rho[1], m.rho[2]);
}

// material.h:27-29 with n = (0, +-1, 0)
__device__ __forceinline__ V3 reflect(V3 v, V3 n) {
  return -v + 2.0f * dot(v, n) * n;
}
// material.h:32-42
__device__ __forceinline__ bool refract(V3 v, V3 n, float iorI, float iorT,
                                        V3& t) {
  const V3 th = -iorI / iorT * (v - dot(v, n) * n);
  if (length2(th) > 1.0f) return false;
  const V3 tp = -sqrtf(fmaxf(1.0f - length2(th), 0.0f)) * n;
  t = th + tp;
  return true;
}
// material.h:45-50
__device__ __forceinline__ float fresnel(float cosThetaI, float iorI,
                                         float iorT) {
  const float f0 =
      (iorI - iorT) * (iorI - iorT) / ((iorI + iorT) * (iorI + iorT));
  const float x = fmaxf(1.0f - fabsf(cosThetaI), 0.0f);
  return f0 + (1.0f - f0) * (x * x * x * x * x);
}
__device__ __forceinline__ float abs_cos_theta(V3 v) { return fabsf(v.y); }

// Lambert::evaluate (material.h:80-88)
__device__ __forceinline__ V3 lambert_eval(const Material& m, V3 wo, V3 wi) {
  if (wo.y < 0.f || wi.y < 0.f) return v3(0.f, 0.f, 0.f);
  return mat_rho(m) / kPI;
}

// BxDF::sampleDirection in the local frame (material.h:90-98, 120-128,
// 146-204). Draws: Lambert 2 (getNext2D), Mirror 0, Glass 1 (getNext1D).
__device__ __forceinline__ V3 bxdf_sample(const Material& m, V3 wo, int tdir,
                                          Rng& rng, V3& wi, float& pdf) {
  if (m.type == kLambert) {
    float u0, u1;
    rng.next2d(u0, u1);
    wi = sample_cos_hemisphere(u0, u1, pdf);
    return lambert_eval(m, wo, wi);
  }
  if (m.type == kMirror) {
    wi = reflect(wo, v3(0.f, 1.f, 0.f));
    pdf = 1.0f;
    return mat_rho(m) / abs_cos_theta(wi);
  }
  // Glass
  float iorO, iorI;
  V3 n;
  if (wo.y > 0.f) {
    iorO = 1.0f;
    iorI = m.ior;
    n = v3(0.f, 1.f, 0.f);
  } else {
    iorO = m.ior;
    iorI = 1.0f;
    n = v3(0.f, -1.f, 0.f);
  }
  const float fr = fresnel(dot(wo, n), iorO, iorI);
  if (rng.next1d() < fr) {
    wi = reflect(wo, n);
    pdf = 1.0f;
    return mat_rho(m) / abs_cos_theta(wi);
  }
  V3 tr;
  if (refract(wo, n, iorO, iorI, tr)) {
    wi = tr;
    pdf = 1.0f;
    float scaling = 1.0f;
    if (tdir == kFromCamera) scaling = (iorO * iorO) / (iorI * iorI);
    return scaling * mat_rho(m) / abs_cos_theta(wi);
  }
  wi = reflect(wo, n);
  pdf = 1.0f;
  return mat_rho(m) / abs_cos_theta(wi);
}

// Integrator::cosTerm (integrator.h:25-46)
__device__ __forceinline__ float cos_term(V3 wo, V3 wi, V3 ns, V3 ng,
                                          int tdir) {
  const float wi_ns = dot(wi, ns);
  const float wi_ng = dot(wi, ng);
  const float wo_ns = dot(wo, ns);
  const float wo_ng = dot(wo, ng);
  if (wi_ng * wi_ns <= 0.f || wo_ng * wo_ns <= 0.f) return 0.f;
  if (tdir == kFromCamera) return fabsf(wi_ns);
  return fabsf(wo_ns) * fabsf(wi_ng) / fabsf(wo_ng);
}

}  // namespace pm
