// Shared device helpers of libpm_cuda.
//
// All device code of this library is compiled with -fmad=false: every
// float expression rounds after each operation, exactly like the
// reference's x86-64 build (SSE scalar math, no FMA contraction), so
// distances, dot products and normalisations are bit-identical to the
// reference arithmetic written in the same order.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace pm {

constexpr int kWarp = 32;
constexpr unsigned kFull = 0xffffffffu;

// core.h:7 — PI is the double literal 3.14159265359 rounded to float.
constexpr float kPI = 3.14159265359f;
// core.h:19
constexpr float kRayEps = 1e-5f;

// Lane id and lane masks (not volatile: the compiler may keep one read for
// a whole loop instead of reading the special register at every use).
__device__ __forceinline__ unsigned lane_id() {
  unsigned l;
  asm("mov.u32 %0, %%laneid;" : "=r"(l));
  return l;
}
__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}
// lanemask_lt from a lane number already in a register (two integer
// instructions instead of a special-register read).
__device__ __forceinline__ unsigned lt_mask(int lane) { return (1u << lane) - 1u; }
__device__ __forceinline__ unsigned lanemask_le() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_le;" : "=r"(m));
  return m;
}

// Squared distance in the reference order: ((dx*dx) + dy*dy) + dz*dz with
// d = q - p (photon_map.h:33-41; 0 + a == a exactly).
__device__ __forceinline__ float dist2_ref(float qx, float qy, float qz,
                                           float px, float py, float pz) {
  const float dx = qx - px, dy = qy - py, dz = qz - pz;
  return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)),
                   __fmul_rn(dz, dz));
}

// dot() of core.h:200-203: (a0*b0 + a1*b1) + a2*b2, rounded per operation.
__device__ __forceinline__ float dot_ref(float a0, float a1, float a2,
                                         float b0, float b1, float b2) {
  return __fadd_rn(__fadd_rn(__fmul_rn(a0, b0), __fmul_rn(a1, b1)),
                   __fmul_rn(a2, b2));
}

// Lower bound of dist2_ref(q, p) over every p inside the box [lo, hi]:
// each axis term uses the same subtraction and rounding as dist2_ref, and
// IEEE rounding is monotone, so the result never exceeds the distance the
// kernel computes for any photon inside the box. Per axis at most one of
// lo - q and q - hi is positive (lo <= hi), so max(lo - q, q - hi, 0) is the
// gap outside the slab without branches (5 % of the kNN time against an
// if/else chain; same values).
__device__ __forceinline__ float box_dist2(float qx, float qy, float qz,
                                           const float4& lo,
                                           const float4& hi) {
  const float dx = fmaxf(fmaxf(lo.x - qx, qx - hi.x), 0.f);
  const float dy = fmaxf(fmaxf(lo.y - qy, qy - hi.y), 0.f);
  const float dz = fmaxf(fmaxf(lo.z - qz, qz - hi.z), 0.f);
  return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)),
                   __fmul_rn(dz, dz));
}

// Low 10 bits of x spread to every third bit (one axis of a 30-bit Morton
// code).
__device__ __forceinline__ uint32_t spread10(uint32_t x) {
  x &= 0x3ffu;
  x = (x | (x << 16)) & 0x030000ffu;
  x = (x | (x << 8)) & 0x0300f00fu;
  x = (x | (x << 4)) & 0x030c30c3u;
  x = (x | (x << 2)) & 0x09249249u;
  return x;
}

// Cell (0..1023) of coordinate v along an axis of the box [lo, lo + ext]
// (NaN and values below lo: cell 0).
__device__ __forceinline__ uint32_t cell10(float v, float lo, float ext) {
  if (!(ext > 0.f)) return 0;
  const float t = (v - lo) / ext * 1024.f;
  if (!(t > 0.f)) return 0;
  return t >= 1023.f ? 1023u : (uint32_t)t;
}

// Float <-> unsigned with the same order (negative floats reversed), for
// atomicMin / atomicMax on floats.
__device__ __forceinline__ uint32_t ordered_bits(float f) {
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float from_ordered(uint32_t u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

}  // namespace pm
