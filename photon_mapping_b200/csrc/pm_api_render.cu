// C ABI of the camera pass: pm_render, pm_integrate, pm_render_path_tracing.
#include <cstring>

#include "../../include/pm_cuda.h"
#include "pm_api_internal.cuh"
#include "pm_api_render.cuh"
#include "pm_render.cuh"
#include "pm_sort.cuh"

using namespace pm;

static_assert(sizeof(pm_camera) == 13 * 4, "camera layout");

namespace pm {

// Buffers of the camera pipeline: npix pixel (or ray) slots, n_samples
// samples per pass, n_slots query slots per pass.
int render_buffers(pm_ctx* c, int npix, int64_t n_samples, int64_t n_slots) {
  c->diff.ready = false;  // the camera buffers are about to be reused
  int s;
  if ((s = c->r_rng.ensure((size_t)npix * 8)) || (s = c->r_accum.ensure((size_t)npix * 16)) ||
      (s = c->r_slots.ensure((size_t)n_slots * 64)) ||
      (s = c->r_srec.ensure((size_t)n_samples * 16)) ||
      (s = c->r_res.ensure((size_t)n_slots * 12)) ||
      (s = c->r_sort.ensure((size_t)n_slots * 16 + sort_hist_words(n_slots) * 4 + 64)) ||
      (s = c->r_misc.ensure(64)) || (s = c->dev_err.ensure(64)) ||
      (s = c->q_out.ensure((size_t)npix * 12)))
    return set_err(c, s, "render buffers (%lld query slots)", (long long)n_slots);
  return PM_OK;
}

// Answers the photon-map queries a camera pass wrote: per map, list the
// slots holding one, sort them by Morton code, run the radiance kernel.
// With slot_adj, runs the adjoint instead: the neighbours of each slot
// receive slot_adj times d estimate / d throughput in photon_adj[map].
int answer_queries(pm_ctx* c, const RenderArgs& a, int64_t ns, int64_t n_slots,
                   bool need_caustics, int kg, int kc, int64_t* q_tot,
                   const float* slot_adj, float4* const* photon_adj) {
  cudaStream_t st = c->stream;
  uint32_t* ka = (uint32_t*)c->r_sort.ptr;
  uint32_t* kb = ka + n_slots;
  uint32_t* va = kb + n_slots;
  uint32_t* vb = va + n_slots;
  uint32_t* hist = vb + n_slots;
  unsigned* qcount = (unsigned*)((char*)c->r_misc.ptr + 16);
  cudaError_t e;
  for (int map = 0; map < 2; ++map) {
    if (map == 1 && !need_caustics) continue;
    if ((e = cudaMemsetAsync(qcount, 0, 4, st)) != cudaSuccess)
      return cuda_status(c, e, "render");
    render_list_queries(a.slots, a.sample_rec, ns, a.q_per_sample, map, c->scene.lo,
                        c->scene.hi, ka, va, qcount, st);
    unsigned nq = 0;
    if ((e = cudaMemcpyAsync(&nq, qcount, 4, cudaMemcpyDeviceToHost, st)) ||
        (e = cudaStreamSynchronize(st)))
      return cuda_status(c, e, "render queries");
    q_tot[map] += nq;
    if (nq == 0) continue;
    const bool in_b = radix_sort_pairs<uint32_t>(ka, va, kb, vb, (int)nq, 30, hist, st);
    KnnOut o{};
    o.rgb = (float*)c->r_res.ptr;
    o.stats = c->stats_ptr();
    o.adj_in = slot_adj;
    o.photon_adj = slot_adj ? photon_adj[map] : nullptr;
    e = knn_launch(map_view(c->maps[map]), a.slots, nq, map == 0 ? kg : kc,
                   slot_adj ? kModeAdjoint : kModeRadiance, (float)c->map_emitted[map], o,
                   c->next_counter(), c->num_sms, st, in_b ? vb : va, 4);
    if (e != cudaSuccess) return cuda_status(c, e, "render estimates");
  }
  return PM_OK;
}

RenderArgs base_args(pm_ctx* c, int width, int height, int q_per_sample, int fg_depth,
                     int max_depth, int n_gather) {
  RenderArgs a{};
  a.width = width;
  a.height = height;
  a.q_per_sample = q_per_sample;
  a.fg_depth = fg_depth;
  a.max_depth = max_depth;
  a.n_gather = n_gather;
  const float ig = 1.0f / (float)n_gather;
  a.inv_gather = v3(ig, ig, ig);
  a.rng_state = (unsigned long long*)c->r_rng.ptr;
  a.slots = (float4*)c->r_slots.ptr;
  a.sample_rec = (float4*)c->r_srec.ptr;
  a.err = (int*)c->dev_err.ptr;
  a.in_rays = nullptr;
  return a;
}

// Query slots per sample: every diffuse leaf of the path tree (at most 8
// with specular branching) needs 1 estimate, or 1 + n_gather with final
// gathering.
int slots_per_sample(const pm_ctx* c, bool need_caustics, int n_gather) {
  const int per_leaf = need_caustics ? 1 + n_gather : 1;
  return (c->scene.has_specular ? 8 : 1) * per_leaf;
}

}  // namespace pm

extern "C" int pm_render(pm_ctx* c, const pm_camera* cam,
                         const pm_render_params* prm, float* out_rgb,
                         pm_render_stats* stats) {
  if (!c) return PM_ERR_INVALID_ARGUMENT;
  if (!cam || !prm || !out_rgb)
    return set_err(c, PM_ERR_INVALID_ARGUMENT, "camera / params / output");
  const pm_render_params p = *prm;
  if (p.width <= 0 || p.height <= 0 || (int64_t)p.width * p.height > (1 << 26) ||
      p.spp < 0 || p.max_depth < 0 || p.n_gather < 1 || p.n_gather > 64 ||
      p.k_global < 1 || p.k_global > PM_MAX_K || p.k_caustics < 1 ||
      p.k_caustics > PM_MAX_K || p.spp_batch < 0)
    return set_err(c, PM_ERR_INVALID_ARGUMENT, "render parameters");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  if (!c->scene.built) return set_err(c, PM_ERR_NOT_BUILT, "scene not built");
  if (!c->maps[0].built) return set_err(c, PM_ERR_NOT_BUILT, "global photon map not built");
  const bool need_caustics = p.final_gathering_depth > 0;
  if (need_caustics && !c->maps[1].built)
    return set_err(c, PM_ERR_NOT_BUILT, "caustics photon map not built");
  cudaStream_t st = c->stream;
  const int npix = p.width * p.height;
  const int q_per_sample = slots_per_sample(c, need_caustics, p.n_gather);
  int batch = p.spp_batch;
  if (batch <= 0) {
    const int64_t budget = (int64_t)32 << 20;  // query slots per pass
    batch = (int)std::max<int64_t>(1, budget / ((int64_t)npix * q_per_sample));
  }
  batch = std::max(1, std::min(batch, std::max(p.spp, 1)));
  const int64_t n_samples = (int64_t)npix * batch;
  const int64_t n_slots = n_samples * q_per_sample;
  if (n_slots > 0x7fffffffLL)
    return set_err(c, PM_ERR_INVALID_ARGUMENT, "too many query slots per pass");
  int s;
  if ((s = render_buffers(c, npix, n_samples, n_slots)) != PM_OK) return s;
  cudaError_t e;
  unsigned long long* dropped = (unsigned long long*)c->r_misc.ptr;
  if ((e = cudaMemsetAsync(c->r_accum.ptr, 0, (size_t)npix * 16, st)) ||
      (e = cudaMemsetAsync(c->r_misc.ptr, 0, 64, st)) ||
      (e = cudaMemsetAsync(c->dev_err.ptr, 0, 64, st)))
    return cuda_status(c, e, "render init");
  render_rng_init((unsigned long long*)c->r_rng.ptr, p.width, p.height, st);
  double* shadow = nullptr;
  if (p.flags & PM_RENDER_FP64_CHECK) {
    if ((s = c->r_shadow.ensure((size_t)npix * 24)) != PM_OK)
      return set_err(c, s, "FP64 sums");
    shadow = (double*)c->r_shadow.ptr;
    if ((e = cudaMemsetAsync(shadow, 0, (size_t)npix * 24, st)) != cudaSuccess)
      return cuda_status(c, e, "render init");
  }
  RenderArgs a = base_args(c, p.width, p.height, q_per_sample, p.final_gathering_depth,
                           p.max_depth, p.n_gather);
  a.cam_pos = v3(cam->position[0], cam->position[1], cam->position[2]);
  a.cam_fwd = v3(cam->forward[0], cam->forward[1], cam->forward[2]);
  a.cam_right = v3(cam->right[0], cam->right[1], cam->right[2]);
  a.cam_up = v3(cam->up[0], cam->up[1], cam->up[2]);
  a.focal = cam->focal_length;
  const SceneDev sv = c->scene_view();
  a.rays = (unsigned long long*)((char*)c->r_misc.ptr + 48);
  int64_t q_tot[2] = {0, 0};
  int passes = 0;
  // device time of the camera pass and of the estimates, summed over passes
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
  for (auto& x : ev)
    if ((e = cudaEventCreate(&x)) != cudaSuccess) {
      for (auto& y : ev)
        if (y) cudaEventDestroy(y);
      return cuda_status(c, e, "render events");
    }
  struct EvGuard {
    cudaEvent_t* ev;
    ~EvGuard() {
      for (int i = 0; i < 3; ++i) cudaEventDestroy(ev[i]);
    }
  } guard{ev};
  float cam_ms = 0.f, est_ms = 0.f;
  for (int done = 0; done < p.spp; done += batch) {
    const int b = std::min(batch, p.spp - done);
    a.batch = b;
    const int64_t ns = (int64_t)npix * b;
    cudaEventRecord(ev[0], st);
    render_camera(sv, a, st);
    cudaEventRecord(ev[1], st);
    if ((s = answer_queries(c, a, ns, n_slots, need_caustics, p.k_global, p.k_caustics,
                            q_tot, nullptr, nullptr)) != PM_OK)
      return s;
    cudaEventRecord(ev[2], st);
    if ((e = cudaEventSynchronize(ev[2])) != cudaSuccess) return cuda_status(c, e, "render");
    float t1 = 0.f, t2 = 0.f;
    cudaEventElapsedTime(&t1, ev[0], ev[1]);
    cudaEventElapsedTime(&t2, ev[1], ev[2]);
    cam_ms += t1;
    est_ms += t2;
    render_resolve(a.slots, a.sample_rec, (const float*)c->r_res.ptr, npix, b, q_per_sample,
                   (float4*)c->r_accum.ptr, dropped, st, nullptr, shadow);
    ++passes;
  }
  render_finish((const float4*)c->r_accum.ptr, npix, std::max(p.spp, 1), (float*)c->q_out.ptr,
                st);
  unsigned* max_bits = (unsigned*)((char*)c->r_misc.ptr + 32);
  if (shadow)
    render_shadow_compare((const float*)c->q_out.ptr, shadow, npix, std::max(p.spp, 1),
                          max_bits, st);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_status(c, e, "render");
  unsigned long long hd[2] = {0, 0}, hrays = 0;
  int herr = 0;
  unsigned hmax = 0;
  if ((e = cudaMemcpyAsync(out_rgb, c->q_out.ptr, (size_t)npix * 12, cudaMemcpyDeviceToHost,
                           st)) ||
      (e = cudaMemcpyAsync(hd, dropped, 16, cudaMemcpyDeviceToHost, st)) ||
      (e = cudaMemcpyAsync(&hrays, a.rays, 8, cudaMemcpyDeviceToHost, st)) ||
      (e = cudaMemcpyAsync(&hmax, max_bits, 4, cudaMemcpyDeviceToHost, st)) ||
      (e = cudaMemcpyAsync(&herr, c->dev_err.ptr, 4, cudaMemcpyDeviceToHost, st)) ||
      (e = cudaStreamSynchronize(st)))
    return cuda_status(c, e, "render output");
  if (herr) {
    cudaMemsetAsync(c->dev_err.ptr, 0, 4, st);
    return set_err(c, PM_ERR_DEVICE_STATUS, "render: device error bits 0x%x", herr);
  }
  if (stats) {
    stats->samples = (int64_t)npix * p.spp;
    stats->dropped_nan = (int64_t)hd[0];
    stats->dropped_negative = (int64_t)hd[1];
    stats->queries_global = q_tot[0];
    stats->queries_caustics = q_tot[1];
    stats->passes = passes;
    stats->reserved = 0;
    float mx = 0.f;
    memcpy(&mx, &hmax, 4);
    stats->accum_rel_err = shadow ? (double)mx : 0.0;
    stats->rays = (int64_t)hrays;
    stats->camera_ms = cam_ms;
    stats->estimate_ms = est_ms;
  }
  return PM_OK;
}

extern "C" int pm_integrate(pm_ctx* c, const float* rays, int64_t n,
                            uint64_t* rng_states, const pm_integrate_params* prm,
                            float* out_rgb) {
  if (!c) return PM_ERR_INVALID_ARGUMENT;
  if (!prm || n < 0 || (n > 0 && (!rays || !rng_states || !out_rgb)) || n > (1 << 26))
    return set_err(c, PM_ERR_INVALID_ARGUMENT, "integrate arguments");
  const pm_integrate_params p = *prm;
  if (p.max_depth < 0 || p.n_gather < 1 || p.n_gather > 64 || p.k_global < 1 ||
      p.k_global > PM_MAX_K || p.k_caustics < 1 || p.k_caustics > PM_MAX_K)
    return set_err(c, PM_ERR_INVALID_ARGUMENT, "integrate parameters");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  if (!c->scene.built) return set_err(c, PM_ERR_NOT_BUILT, "scene not built");
  if (!c->maps[0].built) return set_err(c, PM_ERR_NOT_BUILT, "global photon map not built");
  const bool need_caustics = p.final_gathering_depth > 0;
  if (need_caustics && !c->maps[1].built)
    return set_err(c, PM_ERR_NOT_BUILT, "caustics photon map not built");
  if (n == 0) return PM_OK;
  const int npix = (int)n;
  const int q_per_sample = slots_per_sample(c, need_caustics, p.n_gather);
  const int64_t n_slots = (int64_t)npix * q_per_sample;
  int s;
  if ((s = render_buffers(c, npix, npix, n_slots)) != PM_OK) return s;
  if ((s = c->q_in.ensure((size_t)npix * 24)) != PM_OK)
    return set_err(c, s, "integrate buffers");
  cudaStream_t st = c->stream;
  cudaError_t e;
  if ((e = cudaMemcpyAsync(c->q_in.ptr, rays, (size_t)npix * 24, cudaMemcpyHostToDevice, st)) ||
      (e = cudaMemcpyAsync(c->r_rng.ptr, rng_states, (size_t)npix * 8, cudaMemcpyHostToDevice,
                           st)) ||
      (e = cudaMemsetAsync(c->dev_err.ptr, 0, 64, st)))
    return cuda_status(c, e, "integrate upload");
  RenderArgs a = base_args(c, npix, 1, q_per_sample, p.final_gathering_depth, p.max_depth,
                           p.n_gather);
  a.batch = 1;
  a.in_rays = (const float*)c->q_in.ptr;
  render_camera(c->scene_view(), a, st);
  int64_t q_tot[2] = {0, 0};
  if ((s = answer_queries(c, a, npix, n_slots, need_caustics, p.k_global, p.k_caustics,
                          q_tot, nullptr, nullptr)) != PM_OK)
    return s;
  render_resolve(a.slots, a.sample_rec, (const float*)c->r_res.ptr, npix, 1, q_per_sample,
                 (float4*)c->r_accum.ptr, (unsigned long long*)c->r_misc.ptr, st,
                 (float*)c->q_out.ptr);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_status(c, e, "integrate");
  int herr = 0;
  if ((e = cudaMemcpyAsync(out_rgb, c->q_out.ptr, (size_t)npix * 12, cudaMemcpyDeviceToHost,
                           st)) ||
      (e = cudaMemcpyAsync(rng_states, c->r_rng.ptr, (size_t)npix * 8, cudaMemcpyDeviceToHost,
                           st)) ||
      (e = cudaMemcpyAsync(&herr, c->dev_err.ptr, 4, cudaMemcpyDeviceToHost, st)) ||
      (e = cudaStreamSynchronize(st)))
    return cuda_status(c, e, "integrate output");
  if (herr) return set_err(c, PM_ERR_DEVICE_STATUS, "integrate: device error bits 0x%x", herr);
  return PM_OK;
}

extern "C" int pm_render_path_tracing(pm_ctx* c, const pm_camera* cam,
                                      int32_t width, int32_t height,
                                      int32_t spp, int32_t max_depth,
                                      float* out_rgb, int64_t* dropped_nan) {
  if (!c) return PM_ERR_INVALID_ARGUMENT;
  if (!cam || !out_rgb || width <= 0 || height <= 0 ||
      (int64_t)width * height > (1 << 26) || spp < 0 || max_depth < 0)
    return set_err(c, PM_ERR_INVALID_ARGUMENT, "path tracing parameters");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  if (!c->scene.built) return set_err(c, PM_ERR_NOT_BUILT, "scene not built");
  const int npix = width * height;
  int s;
  if ((s = c->q_out.ensure((size_t)npix * 12)) || (s = c->r_misc.ensure(64)) ||
      (s = c->dev_err.ensure(64)))
    return set_err(c, s, "path tracing buffers");
  cudaStream_t st = c->stream;
  cudaError_t e;
  if ((e = cudaMemsetAsync(c->r_misc.ptr, 0, 64, st)) ||
      (e = cudaMemsetAsync(c->dev_err.ptr, 0, 64, st)))
    return cuda_status(c, e, "path tracing init");
  PathArgs a;
  a.cam_pos = v3(cam->position[0], cam->position[1], cam->position[2]);
  a.cam_fwd = v3(cam->forward[0], cam->forward[1], cam->forward[2]);
  a.cam_right = v3(cam->right[0], cam->right[1], cam->right[2]);
  a.cam_up = v3(cam->up[0], cam->up[1], cam->up[2]);
  a.focal = cam->focal_length;
  a.width = width;
  a.height = height;
  a.spp = spp;
  a.max_depth = max_depth;
  a.out = (float*)c->q_out.ptr;
  a.dropped = (unsigned long long*)c->r_misc.ptr;
  a.in_rays = nullptr;
  a.rng_states = nullptr;
  render_path_tracing(c->scene_view(), a, st);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_status(c, e, "path tracing");
  unsigned long long hd = 0;
  int herr = 0;
  if ((e = cudaMemcpyAsync(out_rgb, c->q_out.ptr, (size_t)npix * 12,
                           cudaMemcpyDeviceToHost, st)) ||
      (e = cudaMemcpyAsync(&hd, a.dropped, 8, cudaMemcpyDeviceToHost, st)) ||
      (e = cudaMemcpyAsync(&herr, c->dev_err.ptr, 4, cudaMemcpyDeviceToHost, st)) ||
      (e = cudaStreamSynchronize(st)))
    return cuda_status(c, e, "path tracing output");
  if (herr) return set_err(c, PM_ERR_DEVICE_STATUS, "path tracing: device error bits 0x%x", herr);
  if (dropped_nan) *dropped_nan = (int64_t)hd;
  return PM_OK;
}

extern "C" int pm_path_trace_rays(pm_ctx* c, const float* rays, int64_t n,
                                  uint64_t* rng_states, int32_t max_depth,
                                  float* out_rgb) {
  if (!c) return PM_ERR_INVALID_ARGUMENT;
  if (n < 0 || n > (1 << 26) || max_depth < 0 || (n > 0 && (!rays || !rng_states || !out_rgb)))
    return set_err(c, PM_ERR_INVALID_ARGUMENT, "path tracing arguments");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  if (!c->scene.built) return set_err(c, PM_ERR_NOT_BUILT, "scene not built");
  if (n == 0) return PM_OK;
  int s;
  if ((s = c->q_in.ensure((size_t)n * 24)) || (s = c->q_out.ensure((size_t)n * 12)) ||
      (s = c->r_rng.ensure((size_t)n * 8)) || (s = c->r_misc.ensure(64)) ||
      (s = c->dev_err.ensure(64)))
    return set_err(c, s, "path tracing buffers");
  cudaStream_t st = c->stream;
  cudaError_t e;
  if ((e = cudaMemcpyAsync(c->q_in.ptr, rays, (size_t)n * 24, cudaMemcpyHostToDevice, st)) ||
      (e = cudaMemcpyAsync(c->r_rng.ptr, rng_states, (size_t)n * 8, cudaMemcpyHostToDevice, st)) ||
      (e = cudaMemsetAsync(c->r_misc.ptr, 0, 64, st)) ||
      (e = cudaMemsetAsync(c->dev_err.ptr, 0, 64, st)))
    return cuda_status(c, e, "path tracing upload");
  PathArgs a{};
  a.width = (int)n;
  a.height = 1;
  a.spp = 1;
  a.max_depth = max_depth;
  a.out = (float*)c->q_out.ptr;
  a.dropped = (unsigned long long*)c->r_misc.ptr;
  a.in_rays = (const float*)c->q_in.ptr;
  a.rng_states = (unsigned long long*)c->r_rng.ptr;
  render_path_tracing(c->scene_view(), a, st);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_status(c, e, "path tracing");
  int herr = 0;
  if ((e = cudaMemcpyAsync(out_rgb, c->q_out.ptr, (size_t)n * 12, cudaMemcpyDeviceToHost, st)) ||
      (e = cudaMemcpyAsync(rng_states, c->r_rng.ptr, (size_t)n * 8, cudaMemcpyDeviceToHost, st)) ||
      (e = cudaMemcpyAsync(&herr, c->dev_err.ptr, 4, cudaMemcpyDeviceToHost, st)) ||
      (e = cudaStreamSynchronize(st)))
    return cuda_status(c, e, "path tracing output");
  if (herr) return set_err(c, PM_ERR_DEVICE_STATUS, "path tracing: device error bits 0x%x", herr);
  return PM_OK;
}
