// Camera pass of the photon mapper on the device: the render loop of
// examples/main.cpp:33-70 around PhotonMapping::integrate
// (integrator.h:290-377, 566-569), as a wavefront.
//
//   1. camera_kernel, one thread per pixel: the pixel's sampler is seeded
//      j + width*i and draws exactly as the reference does (u and v jitter,
//      then the integrator's draws), so sample s of a pixel sees the same
//      random numbers as the reference's loop. The path is followed with an
//      explicit stack (specular surfaces expand every branch at depth < 3,
//      integrator.h:347-366, one sampled branch deeper, :326-343); light hits
//      and next-event estimation are summed at once, every photon-map
//      estimate the path needs (integrator.h:306-307, 310-318, 239-243) is
//      written as a query with its path weight into the sample's slots.
//   2. The queries of each map are sorted by the Morton code of their
//      position and answered by the warp-per-query kNN kernel.
//   3. resolve_kernel, one thread per pixel: per sample in order, direct +
//      sum(weight * estimate); NaN or negative samples are dropped
//      (main.cpp:49-56) and the rest added to the pixel.
#include "pm_batch.cuh"
#include "pm_photonmap.cuh"
#include "pm_render.cuh"
#include "pm_scene.cuh"
#include "pm_sort.cuh"

namespace pm {

constexpr int kPathStack = 8;

struct Frame {
  V3 o, d, w;
  int depth;
};

template <bool D>
__device__ __forceinline__ void emit_query(const RenderArgs& a, int64_t base,
                                           int& nq, int map, const Surf& s,
                                           V3 wo, V3 rho, V3 w, int pid_w,
                                           int pid_q) {
  if (nq >= a.q_per_sample) {
    atomicOr(a.err, 2);
    return;
  }
  if (D) a.slot_pid[base + nq] = make_int2(pid_w, pid_q);
  float4* r = a.slots + 4 * (base + nq);
  r[0] = make_float4(s.pos.x, s.pos.y, s.pos.z, rho.x);
  r[1] = make_float4(wo.x, wo.y, wo.z, rho.y);
  r[2] = make_float4(s.ns.x, s.ns.y, s.ns.z, rho.z);
  r[3] = make_float4(w.x, w.y, w.z, __int_as_float(map));
  ++nq;
}

// PhotonMapping::computeDirectIllumination (integrator.h:178-213).
template <int STACK>
__device__ V3 direct_light(const SceneDev& sc, const Surf& s, V3 wo,
                           const Material& m, Rng& rng) {
  float pc, pp;
  const int lf = sample_light(sc, rng, pc);
  const Surf ls = sample_triangle(sc, lf, rng, pp);
  const V3 wi = normalize(ls.pos - s.pos);
  const float r = length(ls.pos - s.pos);
  const float pd = pp * r * r / fabsf(dot(-wi, ls.ns));
  Hit h;
  if (intersect_t<STACK>(sc, s.pos, wi, kRayEps, r - kRayEps, h)) return v3(0.f, 0.f, 0.f);
  const Material& lm = sc.mat[lf];
  const V3 le = v3(lm.le[0], lm.le[1], lm.le[2]);
  const V3 f = lambert_eval(m, world_to_local(wo, s.dpdu, s.ns, s.dpdv),
                            world_to_local(wi, s.dpdu, s.ns, s.dpdv));
  const float c = fabsf(dot(wi, s.ns));
  return f * c * le / (pc * pd);
}

// PhotonMapping::computeIndirectIlluminationRecursive (integrator.h:
// 215-262) for one gather ray: a diffuse hit becomes a global-map query
// with the accumulated weight, a specular hit continues the path. pid_w is
// the albedo parameter of the surface the gather starts from.
template <bool D, int STACK>
__device__ void gather(const RenderArgs& a, const SceneDev& sc, Surf s, V3 wo,
                       const Material* m, V3 w, Rng& rng, int64_t base,
                       int& nq, int pid_w, unsigned& nr) {
  for (int depth = 0; depth < a.max_depth; ++depth) {
    ++nr;
    V3 wi_l;
    float pdf;
    const V3 f = bxdf_sample(*m, world_to_local(wo, s.dpdu, s.ns, s.dpdv),
                             kFromCamera, rng, wi_l, pdf);
    const V3 dir = local_to_world(wi_l, s.dpdu, s.ns, s.dpdv);
    const float c = fabsf(dot(s.ns, dir));
    Hit h;
    if (!intersect_t<STACK>(sc, s.pos, dir, kRayEps, __int_as_float(0x7f7fffff), h)) return;
    const Surf s2 = surface_at(sc, s.pos, dir, h);
    const Material* m2 = sc.mat + h.prim;
    w = w * (f * c / pdf);
    if (m2->type == kLambert) {
      emit_query<D>(a, base, nq, kQueryGlobal, s2, -dir, mat_rho(*m2), w, pid_w,
                    D ? a.face_pid[h.prim] : -1);
      return;
    }
    s = s2;
    wo = -dir;
    m = m2;
  }
}

// One pixel's samples of the camera pass (all a.batch of them).
template <bool D, int STACK>
__device__ __forceinline__ void camera_pixel(const SceneDev& sc, const RenderArgs& a, int p,
                                             unsigned& nr) {
  const int i = p / a.width, j = p % a.width;
  Rng rng{a.rng_state[p]};
  for (int sidx = 0; sidx < a.batch; ++sidx) {
    const int64_t srec = (int64_t)p * a.batch + sidx;
    const int64_t base = srec * a.q_per_sample;
    int nq = 0, nn = 0;
    V3 direct = v3(0.f, 0.f, 0.f);
    V3 ro, rd;
    if (a.in_rays) {
      // caller's ray (PhotonMapping::integrate): no camera draws
      const float* r = a.in_rays + 6 * (int64_t)p;
      ro = v3(r[0], r[1], r[2]);
      rd = v3(r[3], r[4], r[5]);
    } else {
      // examples/main.cpp:40-41 and Camera::sampleRay (camera.h:41-47)
      const float u = (2.0f * ((float)j + rng.next1d()) - (float)a.width) / (float)a.height;
      const float v = (2.0f * ((float)i + rng.next1d()) - (float)a.height) / (float)a.height;
      const V3 pinhole = a.cam_pos + a.focal * a.cam_fwd;
      const V3 sensor = a.cam_pos + u * a.cam_right + v * a.cam_up;
      ro = sensor;
      rd = normalize(pinhole - sensor);
    }
    Frame st[kPathStack];
    int sp = 0;
    st[sp++] = Frame{ro, rd, v3(1.f, 1.f, 1.f), 0};
    while (sp > 0) {
      const Frame f = st[--sp];
      if (f.depth >= a.max_depth) continue;
      Hit h;
      ++nr;
      if (!intersect_t<STACK>(sc, f.o, f.d, kRayEps, __int_as_float(0x7f7fffff), h)) continue;
      const Surf s = surface_at(sc, f.o, f.d, h);
      const Material& m = sc.mat[h.prim];
      const V3 wo = -f.d;
      if (m.le[0] > 0.f || m.le[1] > 0.f || m.le[2] > 0.f) {
        direct = direct + f.w * v3(m.le[0], m.le[1], m.le[2]);
        continue;
      }
      if (m.type == kLambert) {
        const int pid = D ? a.face_pid[h.prim] : -1;
        if (f.depth >= a.fg_depth) {
          emit_query<D>(a, base, nq, kQueryGlobal, s, wo, mat_rho(m), f.w, -1, pid);
        } else {
          ++nr;  // the shadow ray
          const V3 ld = f.w * direct_light<STACK>(sc, s, wo, m, rng);
          direct = direct + ld;
          if (D && nn < a.q_per_sample)
            a.nee[base + nn++] = make_float4(ld.x, ld.y, ld.z, __int_as_float(pid));
          emit_query<D>(a, base, nq, kQueryCaustics, s, wo, mat_rho(m), f.w, -1, pid);
          const V3 wg = f.w * a.inv_gather;
          for (int g = 0; g < a.n_gather; ++g)
            gather<D, STACK>(a, sc, s, wo, &m, wg, rng, base, nq, pid, nr);
        }
        continue;
      }
      const V3 wo_l = world_to_local(wo, s.dpdu, s.ns, s.dpdv);
      if (f.depth >= 3) {
        V3 wi_l;
        float pdf;
        const V3 fb = bxdf_sample(m, wo_l, kFromCamera, rng, wi_l, pdf);
        const V3 wi = local_to_world(wi_l, s.dpdu, s.ns, s.dpdv);
        const V3 thr = fb * cos_term(wo, wi, s.ns, s.ng, kFromCamera) / pdf;
        st[sp++] = Frame{s.pos, wi, f.w * thr, f.depth + 1};
        continue;
      }
      // sampleAllDirection (material.h:111-118, 206-244): every branch,
      // pushed last-first so the first one is followed first
      V3 dir[2], fv[2];
      int nb = 0;
      if (m.type == kMirror) {
        dir[0] = reflect(wo_l, v3(0.f, 1.f, 0.f));
        fv[0] = mat_rho(m) / abs_cos_theta(dir[0]);
        nb = 1;
      } else {
        float iorO, iorI;
        V3 n;
        if (wo_l.y > 0.f) { iorO = 1.0f; iorI = m.ior; n = v3(0.f, 1.f, 0.f); }
        else { iorO = m.ior; iorI = 1.0f; n = v3(0.f, -1.f, 0.f); }
        const float fr = fresnel(dot(wo_l, n), iorO, iorI);
        dir[0] = reflect(wo_l, n);
        fv[0] = fr * mat_rho(m) / abs_cos_theta(dir[0]);
        nb = 1;
        V3 tr;
        if (refract(wo_l, n, iorO, iorI, tr)) {
          const float scaling = (iorO * iorO) / (iorI * iorI);
          dir[1] = tr;
          fv[1] = (1.0f - fr) * scaling * mat_rho(m) / abs_cos_theta(tr);
          nb = 2;
        } else {
          fv[0] = mat_rho(m) / abs_cos_theta(dir[0]);
        }
      }
      for (int b = nb - 1; b >= 0; --b) {
        const V3 wi = local_to_world(dir[b], s.dpdu, s.ns, s.dpdv);
        const V3 thr = fv[b] * fabsf(dot(wi, s.ns));
        if (sp < kPathStack) st[sp++] = Frame{s.pos, wi, f.w * thr, f.depth + 1};
        else atomicOr(a.err, 4);
      }
    }
    a.sample_rec[srec] = make_float4(direct.x, direct.y, direct.z, __int_as_float(nq));
    if (D) a.nee_count[srec] = nn;
  }
  a.rng_state[p] = rng.state;
}

template <bool D>
__global__ void __launch_bounds__(128)
    camera_kernel(SceneDev sc, RenderArgs a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned nr = 0;
  if (p < a.width * a.height) camera_pixel<D, kBvhStack>(sc, a, p, nr);
  if (a.rays) {
    const unsigned tot = __reduce_add_sync(kFull, nr);
    if ((threadIdx.x & 31) == 0 && tot) atomicAdd(a.rays, (unsigned long long)tot);
  }
}

__global__ void rng_init_kernel(unsigned long long* st, int w, int n) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int i = p / w, j = p % w;
  st[p] = (unsigned long long)(j + w * i);  // UniformSampler(j + width * i)
}

// Lists the slots holding a query of `map`, with the Morton code of the
// query position (in the scene box) as the sort key.
__global__ void list_queries_kernel(const float4* __restrict__ slots,
                                    const float4* __restrict__ srec,
                                    int64_t n_samples, int q_per_sample, int map,
                                    float3 lo, float3 inv_ext,
                                    uint32_t* __restrict__ keys,
                                    uint32_t* __restrict__ vals,
                                    unsigned* __restrict__ count) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  // every lane reaches the ballot and the shuffle (no early exit)
  bool mine = false;
  float4 r0 = make_float4(0.f, 0.f, 0.f, 0.f);
  if (t < n_samples * q_per_sample) {
    const int64_t sidx = t / q_per_sample;
    const int q = (int)(t % q_per_sample);
    if (q < __float_as_int(srec[sidx].w)) {
      mine = __float_as_int(slots[4 * t + 3].w) == map;
      r0 = slots[4 * t];
    }
  }
  const unsigned bal = __ballot_sync(kFull, mine);
  unsigned base = 0;
  const int leader = bal ? __ffs(bal) - 1 : 0;
  if (bal && (int)lane_id() == leader)
    base = atomicAdd(count, (unsigned)__popc(bal));
  base = __shfl_sync(kFull, base, leader);
  if (!mine) return;
  const unsigned o = base + __popc(bal & lanemask_lt());
  auto cell = [](float v, float l, float ie) -> uint32_t {
    const float c = (v - l) * ie * 1024.f;
    if (!(c > 0.f)) return 0u;
    return c >= 1023.f ? 1023u : (uint32_t)c;
  };
  keys[o] = (spread10(cell(r0.x, lo.x, inv_ext.x)) << 2) |
            (spread10(cell(r0.y, lo.y, inv_ext.y)) << 1) |
            spread10(cell(r0.z, lo.z, inv_ext.z));
  vals[o] = (uint32_t)t;
}

// Radiance of sample sidx: direct + sum(weight * estimate) over its slots.
__device__ __forceinline__ V3 sample_radiance(const float4* __restrict__ slots,
                                              const float4* __restrict__ srec,
                                              const float* __restrict__ res, int64_t sidx,
                                              int q_per_sample) {
  const float4 d = srec[sidx];
  V3 rad = v3(d.x, d.y, d.z);
  const int nq = __float_as_int(d.w);
  for (int q = 0; q < nq; ++q) {
    const int64_t t = sidx * q_per_sample + q;
    const float4 w = slots[4 * t + 3];
    const V3 l = v3(res[3 * t], res[3 * t + 1], res[3 * t + 2]);
    rad = rad + v3(w.x, w.y, w.z) * l;
  }
  return rad;
}

__global__ void resolve_kernel(const float4* __restrict__ slots,
                               const float4* __restrict__ srec,
                               const float* __restrict__ res, int npix,
                               int batch, int q_per_sample,
                               float4* __restrict__ accum,
                               unsigned long long* __restrict__ dropped,
                               float* __restrict__ raw, double* __restrict__ shadow) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npix) return;
  float4 acc = raw ? make_float4(0.f, 0.f, 0.f, 0.f) : accum[p];
  unsigned nan_n = 0, neg_n = 0;
  for (int s = 0; s < batch; ++s) {
    const int64_t sidx = (int64_t)p * batch + s;
    const V3 rad = sample_radiance(slots, srec, res, sidx, q_per_sample);
    if (raw) {  // integrate(): the radiance itself, no filtering
      raw[3 * sidx] = rad.x;
      raw[3 * sidx + 1] = rad.y;
      raw[3 * sidx + 2] = rad.z;
      continue;
    }
    if (has_nan(rad)) { ++nan_n; continue; }
    if (rad.x < 0.f || rad.y < 0.f || rad.z < 0.f) { ++neg_n; continue; }
    acc.x += rad.x;
    acc.y += rad.y;
    acc.z += rad.z;
    if (shadow) {
      shadow[3 * p] += (double)rad.x;
      shadow[3 * p + 1] += (double)rad.y;
      shadow[3 * p + 2] += (double)rad.z;
    }
  }
  if (raw) return;
  accum[p] = acc;
  if (nan_n) atomicAdd(dropped, (unsigned long long)nan_n);
  if (neg_n) atomicAdd(dropped + 1, (unsigned long long)neg_n);
}

__global__ void finish_kernel(const float4* __restrict__ accum, int npix,
                              float spp, float* __restrict__ out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npix) return;
  const float4 a = accum[p];
  // Image::divide (image.h:49-56)
  out[3 * p] = a.x / spp;
  out[3 * p + 1] = a.y / spp;
  out[3 * p + 2] = a.z / spp;
}

void render_rng_init(unsigned long long* st, int w, int h, cudaStream_t s) {
  const int n = w * h;
  rng_init_kernel<<<(n + 255) / 256, 256, 0, s>>>(st, w, n);
}

void render_camera(const SceneDev& sc, const RenderArgs& a, cudaStream_t s) {
  const int n = a.width * a.height;
  if (a.slot_pid)
    camera_kernel<true><<<(n + 127) / 128, 128, 0, s>>>(sc, a);
  else
    camera_kernel<false><<<(n + 127) / 128, 128, 0, s>>>(sc, a);
}

void render_list_queries(const float4* slots, const float4* srec,
                         int64_t n_samples, int q_per_sample, int map,
                         const float* scene_lo, const float* scene_hi,
                         uint32_t* keys, uint32_t* vals, unsigned* count,
                         cudaStream_t s) {
  const int64_t n = n_samples * q_per_sample;
  if (n <= 0) return;
  float3 lo = make_float3(scene_lo[0], scene_lo[1], scene_lo[2]);
  float3 ie;
  ie.x = scene_hi[0] > scene_lo[0] ? 1.0f / (scene_hi[0] - scene_lo[0]) : 0.f;
  ie.y = scene_hi[1] > scene_lo[1] ? 1.0f / (scene_hi[1] - scene_lo[1]) : 0.f;
  ie.z = scene_hi[2] > scene_lo[2] ? 1.0f / (scene_hi[2] - scene_lo[2]) : 0.f;
  list_queries_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(
      slots, srec, n_samples, q_per_sample, map, lo, ie, keys, vals, count);
}

void render_resolve(const float4* slots, const float4* srec, const float* res,
                    int npix, int batch, int q_per_sample, float4* accum,
                    unsigned long long* dropped, cudaStream_t s, float* raw,
                    double* shadow) {
  resolve_kernel<<<(npix + 127) / 128, 128, 0, s>>>(
      slots, srec, res, npix, batch, q_per_sample, accum, dropped, raw, shadow);
}

__global__ void shadow_compare_kernel(const float* __restrict__ out,
                                      const double* __restrict__ shadow, int n, double spp,
                                      unsigned* __restrict__ max_bits) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  float rel = 0.f;
  if (i < n) {
    const double want = shadow[i] / spp;
    const double d = fabs((double)out[i] - want);
    const double sc = fabs(want);
    rel = (float)(sc > 0.0 ? d / sc : d);
    if (!(rel >= 0.f)) rel = 0.f;  // NaN: pixels of NaN samples are not summed
  }
  for (int o = 16; o > 0; o >>= 1) rel = fmaxf(rel, __shfl_xor_sync(kFull, rel, o));
  if ((threadIdx.x & 31) == 0 && rel > 0.f) atomicMax(max_bits, __float_as_uint(rel));
}

void render_shadow_compare(const float* out, const double* shadow, int npix, int spp,
                           unsigned* max_bits, cudaStream_t s) {
  const int n = 3 * npix;
  shadow_compare_kernel<<<(n + 255) / 256, 256, 0, s>>>(out, shadow, n,
                                                        (double)(spp > 0 ? spp : 1), max_bits);
}

void render_finish(const float4* accum, int npix, int spp, float* out,
                   cudaStream_t s) {
  finish_kernel<<<(npix + 255) / 256, 256, 0, s>>>(accum, npix, (float)spp, out);
}

}  // namespace pm

namespace pm {

// PathTracing::integrate (integrator.h:60-105) inside the render loop of
// tests/test_path_tracing.cpp:25-52 (NaN samples dropped, counted in the
// average), one thread per pixel, the pixel's sampler seeded j + width*i.
__global__ void __launch_bounds__(128)
    path_trace_kernel(SceneDev sc, PathArgs a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.width * a.height) return;
  const int i = p / a.width, j = p % a.width;
  Rng rng{a.in_rays ? a.rng_states[p] : (unsigned long long)(j + a.width * i)};
  float ax = 0.f, ay = 0.f, az = 0.f;
  unsigned dropped = 0;
  const int spp = a.in_rays ? 1 : a.spp;
  for (int sidx = 0; sidx < spp; ++sidx) {
    V3 o, d;
    if (a.in_rays) {  // caller's ray and sampler (PathTracing::integrate)
      const float* r = a.in_rays + 6 * (int64_t)p;
      o = v3(r[0], r[1], r[2]);
      d = v3(r[3], r[4], r[5]);
    } else {
      const float u = (2.0f * ((float)j + rng.next1d()) - (float)a.width) / (float)a.height;
      const float v = (2.0f * ((float)i + rng.next1d()) - (float)a.height) / (float)a.height;
      const V3 pinhole = a.cam_pos + a.focal * a.cam_fwd;
      const V3 sensor = a.cam_pos + u * a.cam_right + v * a.cam_up;
      o = sensor;
      d = normalize(pinhole - sensor);
    }
    V3 rad = v3(0.f, 0.f, 0.f), thr = v3(1.f, 1.f, 1.f);
    for (int k = 0; k < a.max_depth; ++k) {
      Hit h;
      if (!intersect(sc, o, d, kRayEps, __int_as_float(0x7f7fffff), h)) break;
      const Surf s = surface_at(sc, o, d, h);
      const Material& m = sc.mat[h.prim];
      if (k > 0) {  // Russian roulette (integrator.h:70-78)
        const float q = fminf(fmaxf(thr.x, fmaxf(thr.y, thr.z)), 1.0f);
        if (rng.next1d() >= q) break;
        thr = thr / q;
      }
      if (m.le[0] > 0.f || m.le[1] > 0.f || m.le[2] > 0.f)
        rad = rad + thr * v3(m.le[0], m.le[1], m.le[2]);
      const V3 wo = -d;
      V3 wi_l;
      float pdf;
      const V3 f = bxdf_sample(m, world_to_local(wo, s.dpdu, s.ns, s.dpdv),
                               kFromCamera, rng, wi_l, pdf);
      const V3 wi = local_to_world(wi_l, s.dpdu, s.ns, s.dpdv);
      thr = thr * (f * cos_term(wo, wi, s.ns, s.ng, kFromCamera) / pdf);
      o = s.pos;
      d = wi;
    }
    if (a.in_rays) {  // the radiance itself, unfiltered
      ax = rad.x;
      ay = rad.y;
      az = rad.z;
      break;
    }
    if (has_nan(rad)) {
      ++dropped;
      continue;
    }
    ax += rad.x;
    ay += rad.y;
    az += rad.z;
  }
  if (a.in_rays) a.rng_states[p] = rng.state;
  const float k = (float)(a.in_rays ? 1 : (a.spp > 0 ? a.spp : 1));
  a.out[3 * p] = ax / k;
  a.out[3 * p + 1] = ay / k;
  a.out[3 * p + 2] = az / k;
  if (dropped) atomicAdd(a.dropped, (unsigned long long)dropped);
}

void render_path_tracing(const SceneDev& sc, const PathArgs& a, cudaStream_t s) {
  const int n = a.width * a.height;
  path_trace_kernel<<<(n + 127) / 128, 128, 0, s>>>(sc, a);
}

}  // namespace pm

// ------------------------------------------------------------ batched pass
namespace pm {

// Sampler seeds and the camera pass of every pixel of every scene.
template <int STACK>
__global__ void __launch_bounds__(256)
    batch_camera_kernel(BatchTables t, int64_t total) {
  __shared__ int64_t off[kMaxBatchScenes + 1];
  batch_load_offsets(off, t.pix_off, t.n_scenes);
  __syncthreads();
  const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (g >= total) return;
  const int s = batch_find(off, t.n_scenes, g);
  const BatchScene& bs = t.scenes[s];
  const int p = (int)(g - off[s]);
  const int i = p / bs.ra.width, j = p % bs.ra.width;
  bs.ra.rng_state[p] = (unsigned long long)(j + bs.ra.width * i);  // UniformSampler(j + w*i)
  unsigned nr = 0;
  camera_pixel<false, STACK>(bs.sc, bs.ra, p, nr);
}

void batch_camera_launch(const BatchTables& t, int64_t total_pix, int block, int stack,
                         cudaStream_t st) {
  if (total_pix <= 0) return;
  const unsigned gb = (unsigned)((total_pix + block - 1) / block);
  if (stack <= 16)
    batch_camera_kernel<16><<<gb, block, 0, st>>>(t, total_pix);
  else if (stack <= 32)
    batch_camera_kernel<32><<<gb, block, 0, st>>>(t, total_pix);
  else
    batch_camera_kernel<64><<<gb, block, 0, st>>>(t, total_pix);
}

__global__ void __launch_bounds__(256)
    batch_list_queries_kernel(BatchTables t, int64_t total, const float4* __restrict__ slots,
                              unsigned long long* __restrict__ keys,
                              uint32_t* __restrict__ vals, unsigned* __restrict__ count) {
  __shared__ int64_t off[kMaxBatchScenes + 1];
  batch_load_offsets(off, t.slot_off, t.n_scenes);
  __syncthreads();
  const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  // every lane reaches the ballot and the shuffle (no early exit)
  bool mine = false;
  int s = 0;
  float4 r0 = make_float4(0.f, 0.f, 0.f, 0.f);
  if (g < total) {
    s = batch_find(off, t.n_scenes, g);
    const BatchScene& bs = t.scenes[s];
    const int64_t tl = g - off[s];
    const int64_t sidx = tl / bs.ra.q_per_sample;
    const int q = (int)(tl % bs.ra.q_per_sample);
    if (q < __float_as_int(bs.ra.sample_rec[sidx].w)) {
      mine = __float_as_int(slots[4 * g + 3].w) == kQueryGlobal;
      r0 = slots[4 * g];
    }
  }
  const unsigned bal = __ballot_sync(kFull, mine);
  unsigned base = 0;
  const int leader = bal ? __ffs(bal) - 1 : 0;
  if (bal && (int)lane_id() == leader) base = atomicAdd(count, (unsigned)__popc(bal));
  base = __shfl_sync(kFull, base, leader);
  if (!mine) return;
  const unsigned o = base + __popc(bal & lanemask_lt());
  const BatchScene& bs = t.scenes[s];
  auto cell = [](float v, float l, float ie) -> uint32_t {
    const float c = (v - l) * ie * 1024.f;
    if (!(c > 0.f)) return 0u;
    return c >= 1023.f ? 1023u : (uint32_t)c;
  };
  const uint32_t mc = (spread10(cell(r0.x, bs.qlo.x, bs.qinv.x)) << 2) |
                      (spread10(cell(r0.y, bs.qlo.y, bs.qinv.y)) << 1) |
                      spread10(cell(r0.z, bs.qlo.z, bs.qinv.z));
  keys[o] = ((unsigned long long)s << 30) | mc;
  vals[o] = (uint32_t)g;
}

void batch_list_queries_launch(const BatchTables& t, int64_t total_slots,
                               unsigned long long* keys, uint32_t* vals, unsigned* count,
                               cudaStream_t st) {
  if (total_slots <= 0) return;
  batch_list_queries_kernel<<<(unsigned)((total_slots + 255) / 256), 256, 0, st>>>(
      t, total_slots, t.slots, keys, vals, count);
}

// Keys past the listed queries are all ones (the list buffer is cleared
// before listing), so they sort last and name no scene.
__global__ void batch_query_start_kernel(const unsigned long long* __restrict__ keys, int64_t nq,
                                         int n, int64_t* __restrict__ qstart) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nq) return;
  const unsigned long long s = keys[i] >> 30;
  if (s >= (unsigned long long)n) return;
  if (i == 0 || (keys[i - 1] >> 30) != s) qstart[s] = i;
}

__global__ void batch_query_prefix_kernel(const int64_t* __restrict__ qstart, int64_t nq,
                                          const unsigned* __restrict__ listed, int n, int chunk,
                                          int64_t* __restrict__ qoff,
                                          int64_t* __restrict__ item_off) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  qoff[n] = min(nq, (int64_t)*listed);
  for (int s = n - 1; s >= 0; --s) qoff[s] = qstart[s] >= 0 ? qstart[s] : qoff[s + 1];
  item_off[0] = 0;
  for (int s = 0; s < n; ++s)
    item_off[s + 1] = item_off[s] + (qoff[s + 1] - qoff[s] + chunk - 1) / chunk;
}

void batch_query_ranges_launch(const unsigned long long* sorted_keys, int64_t nq,
                               const unsigned* listed, int n_scenes, int chunk, int64_t* qstart,
                               int64_t* qoff, int64_t* item_off, cudaStream_t st) {
  cudaMemsetAsync(qstart, 0xff, (size_t)n_scenes * sizeof(int64_t), st);
  if (nq > 0)
    batch_query_start_kernel<<<(unsigned)((nq + 255) / 256), 256, 0, st>>>(sorted_keys, nq,
                                                                          n_scenes, qstart);
  batch_query_prefix_kernel<<<1, 32, 0, st>>>(qstart, nq, listed, n_scenes, chunk, qoff,
                                              item_off);
}

__global__ void __launch_bounds__(256) batch_resolve_kernel(BatchTables t, int64_t total) {
  __shared__ int64_t off[kMaxBatchScenes + 1];
  batch_load_offsets(off, t.pix_off, t.n_scenes);
  __syncthreads();
  const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (g >= total) return;
  const int s = batch_find(off, t.n_scenes, g);
  const BatchScene& bs = t.scenes[s];
  const int p = (int)(g - off[s]);
  const int batch = bs.ra.batch;
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  unsigned nan_n = 0, neg_n = 0;
  for (int k = 0; k < batch; ++k) {
    const V3 rad = sample_radiance(bs.ra.slots, bs.ra.sample_rec, bs.res,
                                   (int64_t)p * batch + k, bs.ra.q_per_sample);
    if (has_nan(rad)) { ++nan_n; continue; }
    if (rad.x < 0.f || rad.y < 0.f || rad.z < 0.f) { ++neg_n; continue; }
    acc.x += rad.x;
    acc.y += rad.y;
    acc.z += rad.z;
  }
  // Image::divide (image.h:49-56)
  const float spp = (float)(batch > 0 ? batch : 1);
  bs.image[3 * p] = acc.x / spp;
  bs.image[3 * p + 1] = acc.y / spp;
  bs.image[3 * p + 2] = acc.z / spp;
  if (nan_n) atomicAdd(t.dropped, (unsigned long long)nan_n);
  if (neg_n) atomicAdd(t.dropped + 1, (unsigned long long)neg_n);
}

void batch_resolve_launch(const BatchTables& t, int64_t total_pix, cudaStream_t st) {
  if (total_pix <= 0) return;
  batch_resolve_kernel<<<(unsigned)((total_pix + 255) / 256), 256, 0, st>>>(t, total_pix);
}

}  // namespace pm
