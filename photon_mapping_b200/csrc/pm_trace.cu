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
#include "pm_batch.cuh"
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

enum { kTracePlain = 0, kTraceFrozen = 1, kTraceReplay = 2 };

// Shared accumulators of the replay: per block, the parameter sums and, per
// thread, how many times each parameter has scaled the throughput so far.
struct ReplaySmem {
  float g[kMaxDiffParams * 3];
  unsigned char cnt[kMaxDiffParams][128];
};

// One emitted photon of PhotonMapping::build (integrator.h:406-469 global,
// :483-558 caustics).
template <int MODE, int STACK>
__device__ __forceinline__ void trace_one(const SceneDev& sc, const TraceArgs& a, int i,
                                          ReplaySmem* rs) {
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
  // decision throughput: the same arithmetic over the decision materials
  V3 td = thr;
  if (MODE != kTracePlain) {
    const Material& dm = a.dmat[lf];
    td = v3(dm.le[0], dm.le[1], dm.le[2]) /
         (pdf_choose * pdf_pos * pdf_dir) * fabsf(dot(dir, ls.ns));
  }
  V3 org = ls.pos;
  int nst = 0;  // replay: photons this path has stored so far

  bool prev_specular = false;
  for (int k = 0; k < a.max_depth; ++k) {
    const V3 dec = MODE != kTracePlain ? td : thr;
    if (has_nan(dec)) {
      if (MODE != kTraceReplay) atomicAdd(a.status + 0, 1u);
      break;
    }
    if (dec.x < 0.f || dec.y < 0.f || dec.z < 0.f) {
      if (MODE != kTraceReplay) atomicAdd(a.status + 1, 1u);
      break;
    }
    Hit h;
    if (!intersect_t<STACK>(sc, org, dir, kRayEps, __int_as_float(0x7f7fffff), h))
      break;  // photon goes to the sky
    const Surf s = surface_at(sc, org, dir, h);
    const Material& m = sc.mat[h.prim];
    const bool diffuse = m.type == kLambert;
    bool store = false, stop = false;
    if (!a.caustic) {
      store = diffuse;
    } else {
      // integrator.h:510-523
      if (!prev_specular && diffuse) break;
      if (prev_specular && diffuse) store = stop = true;
      prev_specular = !diffuse;
    }
    if (store) {
      if (MODE == kTraceReplay) {
        // the replay stores where the trace stored; cap = photons stored
        const unsigned long long si = (unsigned long long)a.first[i] + (unsigned)nst;
        if (si >= a.cap) {
          atomicOr(sc.err, 8);
          break;
        }
        const float4 g = a.adj[si];
        const V3 w = v3(g.x, g.y, g.z) * thr;
        for (int j = 0; j < a.n_params; ++j) {
          const unsigned c = rs->cnt[j][threadIdx.x];
          if (c) {
            atomicAdd(&rs->g[3 * j + 0], (float)c * w.x);
            atomicAdd(&rs->g[3 * j + 1], (float)c * w.y);
            atomicAdd(&rs->g[3 * j + 2], (float)c * w.z);
          }
        }
      } else {
        store_photon(a, i, k, thr, s.pos, -dir);
      }
      ++nst;
    }
    if (stop) break;
    // Russian roulette (integrator.h:441-449)
    if (k > 0) {
      const float q =
          fminf(fmaxf(dec.x, fmaxf(dec.y, dec.z)), 1.0f);
      if (rng.next1d() >= q) break;
      thr = thr / q;
      if (MODE != kTracePlain) td = td / q;
    }
    // Primitive::sampleBxDF FROM_LIGHT (primitive.h:46-62)
    const V3 wo = -dir;
    const V3 wo_l = world_to_local(wo, s.dpdu, s.ns, s.dpdv);
    V3 wi_l;
    float pdf;
    const V3 f = bxdf_sample(m, wo_l, kFromLight, rng, wi_l, pdf);
    const V3 wi = local_to_world(wi_l, s.dpdu, s.ns, s.dpdv);
    const float ct = cos_term(wo, wi, s.ns, s.ng, kFromLight);
    thr = thr * (f * ct / pdf);
    if (MODE != kTracePlain) {
      // albedo parameters sit on Lambert faces only; the direction drawn
      // does not depend on the albedo
      const V3 fd = diffuse ? lambert_eval(a.dmat[h.prim], wo_l, wi_l) : f;
      td = td * (fd * ct / pdf);
    }
    if (MODE == kTraceReplay) {
      const int pid = a.face_pid[h.prim];
      if (pid >= 0) ++rs->cnt[pid][threadIdx.x];
    }
    org = s.pos;
    dir = wi;
  }
}

template <int MODE>
__global__ void __launch_bounds__(128)
    trace_kernel(SceneDev sc, TraceArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (MODE == kTraceReplay) {
    __shared__ ReplaySmem rs;
    for (int t = threadIdx.x; t < 3 * a.n_params; t += blockDim.x) rs.g[t] = 0.f;
    for (int j = 0; j < a.n_params; ++j) rs.cnt[j][threadIdx.x] = 0;
    __syncthreads();
    if (i < a.n_emit) trace_one<MODE, kBvhStack>(sc, a, i, &rs);
    __syncthreads();
    for (int t = threadIdx.x; t < 3 * a.n_params; t += blockDim.x)
      if (rs.g[t] != 0.f) atomicAdd(a.grad + t, (double)rs.g[t]);
    return;
  }
  if (i >= a.n_emit) return;
  trace_one<MODE, kBvhStack>(sc, a, i, nullptr);
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

// Every emitted photon of every scene of a batch, one thread each: the
// global map rule, appended to the scene's own region.
template <int STACK>
__global__ void __launch_bounds__(256)
    batch_trace_kernel(BatchTables t, int64_t total) {
  __shared__ int64_t off[kMaxBatchScenes + 1];
  batch_load_offsets(off, t.emit_off, t.n_scenes);
  __syncthreads();
  const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (g >= total) return;
  const int s = batch_find(off, t.n_scenes, g);
  const BatchScene& bs = t.scenes[s];
  TraceArgs a{};
  a.seed = bs.seed;
  a.n_emit = bs.n_emit;
  a.max_depth = bs.max_depth;
  a.caustic = 0;
  a.out = bs.raw;
  a.keys = bs.keys;
  a.counter = bs.counter;
  a.cap = bs.cap;
  a.status = t.status;
  trace_one<kTracePlain, STACK>(bs.sc, a, (int)(g - off[s]), nullptr);
}

void batch_trace_launch(const BatchTables& t, int64_t total_emit, int block, int stack,
                        cudaStream_t st) {
  if (total_emit <= 0) return;
  const unsigned gb = (unsigned)((total_emit + block - 1) / block);
  if (stack <= 32)
    batch_trace_kernel<32><<<gb, block, 0, st>>>(t, total_emit);
  else
    batch_trace_kernel<64><<<gb, block, 0, st>>>(t, total_emit);
}

// first[p] = sorted index of the first stored photon of emitted photon p.
__global__ void first_of_photon_kernel(const unsigned long long* __restrict__ keys,
                                       int n, uint32_t* __restrict__ first) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const unsigned long long p = keys[s] >> 8;
  if (s == 0 || (keys[s - 1] >> 8) != p) first[p] = (uint32_t)s;
}

__global__ void iota_kernel(uint32_t* v, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = (uint32_t)i;
}

void trace_launch(const SceneDev& sc, const TraceArgs& a, cudaStream_t st) {
  if (a.n_emit <= 0) return;
  const int tb = 128;  // ReplaySmem holds 128 threads' counters
  const int gb = (a.n_emit + tb - 1) / tb;
  if (a.adj)
    trace_kernel<kTraceReplay><<<gb, tb, 0, st>>>(sc, a);
  else if (a.dmat)
    trace_kernel<kTraceFrozen><<<gb, tb, 0, st>>>(sc, a);
  else
    trace_kernel<kTracePlain><<<gb, tb, 0, st>>>(sc, a);
}

size_t order_scratch_bytes(int64_t n) {
  const size_t nn = (size_t)(n > 1 ? n : 2);
  return 2 * nn * 8 + 2 * nn * 4 + sort_hist_words(nn) * 4 + 64;
}

void order_photons_launch(unsigned long long* keys, const float* raw, int n,
                          int key_bits, float* out, void* scratch,
                          cudaStream_t st, uint32_t* first) {
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
  if (first) first_of_photon_kernel<<<gb, tb, 0, st>>>(in_b ? kb : keys, n, first);
}

}  // namespace pm
