// Photon emission and tracing on the device (PhotonMapping::build,
// integrator.h:393-563), one thread per emitted photon.
//
// Random numbers: photon i draws from its own UniformSampler-style PCG32
// stream whose state starts at photon_stream_state(seed, i); the draws
// follow the reference's order exactly (sampleLight 1, samplePoint 2,
// sampleDirection 2, then per bounce: Russian roulette 1 when k > 0, BxDF
// sample 2 / 0 / 1). The reference gives each OpenMP thread one stream, so
// its photon set depends on the thread count; keying the stream by the
// photon index makes the set reproducible and lets a photon be replayed
// on its own.
//
// Stored photons are appended with an atomic counter and tagged with the
// key (photon index << 8 | bounce); sorting by that key afterwards gives
// the order a sequential trace produces.
#include "pm_scene.cuh"
#include "pm_sort.cuh"
#include "pm_trace.cuh"

namespace pm {

__host__ __device__ __forceinline__ unsigned long long splitmix64(
    unsigned long long x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

__host__ __device__ unsigned long long photon_stream_state(
    unsigned long long seed, unsigned long long i) {
  return splitmix64(seed ^ splitmix64(i));
}

__device__ __forceinline__ void store_photon(const TraceArgs& a, int photon,
                                             int bounce, V3 thr, V3 pos,
                                             V3 wi) {
  const unsigned long long slot = atomicAdd(a.counter, 1ull);
  if (slot >= a.cap) return;
  float* o = a.out + 9 * slot;
  o[0] = thr.x; o[1] = thr.y; o[2] = thr.z;
  o[3] = pos.x; o[4] = pos.y; o[5] = pos.z;
  o[6] = wi.x; o[7] = wi.y; o[8] = wi.z;
  a.keys[slot] = ((unsigned long long)photon << 8) | (unsigned)bounce;
}

__global__ void __launch_bounds__(128)
    trace_kernel(SceneDev sc, TraceArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n_emit) return;
  Rng rng{photon_stream_state(a.seed, (unsigned long long)i)};

  // sampleRayFromLight (integrator.h:265-288)
  float pdf_choose, pdf_pos, pdf_dir;
  const int lf = sample_light(sc, rng, pdf_choose);
  const Surf ls = sample_triangle(sc, lf, rng, pdf_pos);
  float u0, u1;
  rng.next2d(u0, u1);
  const V3 dl = sample_cos_hemisphere(u0, u1, pdf_dir);
  V3 dir = local_to_world(dl, ls.dpdu, ls.ns, ls.dpdv);
  const Material& lm = sc.mat[lf];
  V3 thr = v3(lm.le[0], lm.le[1], lm.le[2]) /
           (pdf_choose * pdf_pos * pdf_dir) * fabsf(dot(dir, ls.ns));
  V3 org = ls.pos;

  bool prev_specular = false;
  for (int k = 0; k < a.max_depth; ++k) {
    if (has_nan(thr)) {
      atomicAdd(a.status + 0, 1u);
      break;
    }
    if (thr.x < 0.f || thr.y < 0.f || thr.z < 0.f) {
      atomicAdd(a.status + 1, 1u);
      break;
    }
    Hit h;
    if (!intersect(sc, org, dir, kRayEps, __int_as_float(0x7f7fffff), h))
      break;  // photon goes to the sky
    const Surf s = surface_at(sc, org, dir, h);
    const Material& m = sc.mat[h.prim];
    const bool diffuse = m.type == kLambert;
    if (!a.caustic) {
      if (diffuse) store_photon(a, i, k, thr, s.pos, -dir);
    } else {
      // integrator.h:510-523
      if (!prev_specular && diffuse) break;
      if (prev_specular && diffuse) {
        store_photon(a, i, k, thr, s.pos, -dir);
        break;
      }
      prev_specular = !diffuse;
    }
    // Russian roulette (integrator.h:441-449)
    if (k > 0) {
      const float q =
          fminf(fmaxf(thr.x, fmaxf(thr.y, thr.z)), 1.0f);
      if (rng.next1d() >= q) break;
      thr = thr / q;
    }
    // Primitive::sampleBxDF FROM_LIGHT (primitive.h:46-62)
    const V3 wo = -dir;
    const V3 wo_l = world_to_local(wo, s.dpdu, s.ns, s.dpdv);
    V3 wi_l;
    float pdf;
    const V3 f = bxdf_sample(m, wo_l, kFromLight, rng, wi_l, pdf);
    const V3 wi = local_to_world(wi_l, s.dpdu, s.ns, s.dpdv);
    thr = thr * (f * cos_term(wo, wi, s.ns, s.ng, kFromLight) / pdf);
    org = s.pos;
    dir = wi;
  }
}

__global__ void gather_photons_kernel(const float* __restrict__ raw,
                                      const uint32_t* __restrict__ order,
                                      int n, float* __restrict__ out) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const float* r = raw + 9 * (size_t)order[s];
  float* o = out + 9 * (size_t)s;
#pragma unroll
  for (int j = 0; j < 9; ++j) o[j] = r[j];
}

__global__ void iota_kernel(uint32_t* v, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = (uint32_t)i;
}

void trace_launch(const SceneDev& sc, const TraceArgs& a, cudaStream_t st) {
  if (a.n_emit <= 0) return;
  const int tb = 128;
  trace_kernel<<<(a.n_emit + tb - 1) / tb, tb, 0, st>>>(sc, a);
}

size_t order_scratch_bytes(int64_t n) {
  const size_t nn = (size_t)(n > 1 ? n : 2);
  return 2 * nn * 8 + 2 * nn * 4 + sort_hist_words(nn) * 4 + 64;
}

void order_photons_launch(unsigned long long* keys, const float* raw, int n,
                          int key_bits, float* out, void* scratch,
                          cudaStream_t st) {
  if (n <= 0) return;
  unsigned long long* kb = (unsigned long long*)scratch;
  uint32_t* va = (uint32_t*)(kb + n);
  uint32_t* vb = va + n;
  uint32_t* hist = vb + n;
  const int tb = 256;
  const int gb = (n + tb - 1) / tb;
  iota_kernel<<<gb, tb, 0, st>>>(va, n);
  const bool in_b = radix_sort_pairs<unsigned long long>(keys, va, kb, vb, n,
                                                          key_bits, hist, st);
  gather_photons_kernel<<<gb, tb, 0, st>>>(raw, in_b ? vb : va, n, out);
}

}  // namespace pm
