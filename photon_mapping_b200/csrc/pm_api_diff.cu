// C ABI of the differentiable render: pm_diff_set_parameters,
// pm_diff_forward, pm_diff_backward.
//
// Forward: the parameters are written into the scene's materials, both
// photon maps are traced with frozen Russian-roulette decisions (pm_trace.cu,
// frozen mode; the first stored photon of every emitted photon is kept for
// the replay), and the camera pass runs in one batch of all spp with its
// per-slot parameter ids and next-event records (pm_render.cu).
//
// Backward, from d loss / d image:
//   1. pm_diff.cu: per sample, the terms of the camera pass; the adjoint of
//      every slot's estimate.
//   2. pm_photonmap.cu, adjoint mode: the same kNN queries scatter each
//      slot's adjoint onto its neighbours' throughputs.
//   3. pm_trace.cu, replay mode: every emitted photon's path is replayed
//      from its seed; each stored photon's adjoint x throughput goes to the
//      parameters its path met.
//   4. d loss / d theta = G / theta (see pm_diff.cu).
#include <cmath>
#include <vector>

#include "../../include/pm_cuda.h"
#include "pm_api_internal.cuh"
#include "pm_api_render.cuh"
#include "pm_diff.cuh"
#include "pm_trace.cuh"

using namespace pm;

static_assert(PM_DIFF_MAX_PARAMS == kMaxDiffParams, "parameter limit");

namespace {

bool positive_finite(const float* v, int n) {
  for (int i = 0; i < n; ++i)
    if (!(v[i] > 0.f) || !std::isfinite(v[i])) return false;
  return true;
}

}  // namespace

extern "C" int pm_diff_set_parameters(pm_ctx* c, const int32_t* face_param, int64_t n_faces,
                                      int32_t n_params) {
  if (!c) return PM_ERR_INVALID_ARGUMENT;
  if (n_params < 0 || n_params > PM_DIFF_MAX_PARAMS || n_faces < 0 ||
      (n_faces > 0 && !face_param))
    return set_err(c, PM_ERR_INVALID_ARGUMENT, "n_params %d / face_param", n_params);
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  DiffState& d = c->diff;
  d.ready = false;
  d.scene_generation = ~0ull;
  if (!c->scene.built) return set_err(c, PM_ERR_NOT_BUILT, "scene not built");
  if (n_faces != c->scene.n_faces)
    return set_err(c, PM_ERR_INVALID_ARGUMENT, "%lld face parameters for %lld faces",
                   (long long)n_faces, (long long)c->scene.n_faces);
  const size_t nf = (size_t)(n_faces > 0 ? n_faces : 1);
  std::vector<Material> mats((size_t)n_faces);
  cudaStream_t st = c->stream;
  cudaError_t e;
  if (n_faces > 0 &&
      ((e = cudaMemcpyAsync(mats.data(), c->scene.mat.ptr, (size_t)n_faces * sizeof(Material),
                            cudaMemcpyDeviceToHost, st)) ||
       (e = cudaStreamSynchronize(st))))
    return cuda_status(c, e, "materials");
  for (int64_t f = 0; f < n_faces; ++f) {
    const int pid = face_param[f];
    if (pid < -1 || pid >= n_params)
      return set_err(c, PM_ERR_INVALID_ARGUMENT, "face %lld: parameter %d of %d",
                     (long long)f, pid, n_params);
    if (pid >= 0 && mats[(size_t)f].type != PM_LAMBERT)
      return set_err(c, PM_ERR_INVALID_ARGUMENT,
                     "face %lld: an albedo parameter needs a Lambert material", (long long)f);
  }
  int s;
  if ((s = d.face_pid.ensure(nf * 4)) || (s = d.base_mat.ensure(nf * sizeof(Material))) ||
      (s = d.dec_mat.ensure(nf * sizeof(Material))) ||
      (s = d.theta.ensure(2 * 3 * (kMaxDiffParams + 1) * 4)) ||
      (s = d.grad.ensure(3 * (kMaxDiffParams + 1) * 8)))
    return set_err(c, s, "parameter buffers");
  if (n_faces > 0 &&
      ((e = cudaMemcpyAsync(d.face_pid.ptr, face_param, (size_t)n_faces * 4,
                            cudaMemcpyHostToDevice, st)) ||
       (e = cudaMemcpyAsync(d.base_mat.ptr, mats.data(), (size_t)n_faces * sizeof(Material),
                            cudaMemcpyHostToDevice, st)) ||
       (e = cudaStreamSynchronize(st))))
    return cuda_status(c, e, "parameter upload");
  d.n_params = n_params;
  d.scene_generation = c->scene.generation;
  return PM_OK;
}

extern "C" int pm_diff_forward(pm_ctx* c, const pm_camera* cam, const pm_diff_params* prm,
                               const float* albedo, const float* emission,
                               const float* decision_albedo, const float* decision_emission,
                               float* out_rgb, pm_render_stats* stats) {
  if (!c) return PM_ERR_INVALID_ARGUMENT;
  if (!cam || !prm || !emission || !out_rgb)
    return set_err(c, PM_ERR_INVALID_ARGUMENT, "camera / params / emission / output");
  const pm_diff_params p = *prm;
  if (p.width <= 0 || p.height <= 0 || (int64_t)p.width * p.height > (1 << 26) || p.spp < 1 ||
      p.max_depth < 0 || p.max_depth > 255 || p.n_gather < 1 || p.n_gather > 64 || p.k < 1 ||
      p.k > PM_MAX_K || p.final_gathering_depth < 0 || p.n_photons < 0 ||
      p.n_photons > (int64_t)0x7fffffff || p.n_photons_caustics < 0 ||
      p.n_photons_caustics > (int64_t)0x7fffffff)
    return set_err(c, PM_ERR_INVALID_ARGUMENT, "differentiable render parameters");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  DiffState& d = c->diff;
  d.ready = false;
  if (!c->scene.built) return set_err(c, PM_ERR_NOT_BUILT, "scene not built");
  if (d.scene_generation != c->scene.generation)
    return set_err(c, PM_ERR_NOT_BUILT, "pm_diff_set_parameters not called for this scene");
  const int np = d.n_params;
  if ((np > 0 && !albedo) || !positive_finite(albedo, 3 * np) || !positive_finite(emission, 3))
    return set_err(c, PM_ERR_INVALID_ARGUMENT, "parameters must be positive and finite");
  const float* dalb = decision_albedo ? decision_albedo : albedo;
  const float* dem = decision_emission ? decision_emission : emission;
  if (!positive_finite(dalb, 3 * np) || !positive_finite(dem, 3))
    return set_err(c, PM_ERR_INVALID_ARGUMENT, "decision parameters must be positive and finite");
  const bool need_caustics = p.final_gathering_depth > 0;
  const int npix = p.width * p.height;
  const int q_per_sample = slots_per_sample(c, need_caustics, p.n_gather);
  const int64_t n_samples = (int64_t)npix * p.spp;
  const int64_t n_slots = n_samples * q_per_sample;
  if (n_slots > ((int64_t)1 << 28))
    return set_err(c, PM_ERR_INVALID_ARGUMENT,
                   "%lld query slots: the differentiable render keeps every sample of one "
                   "image (at most 2^28 slots)", (long long)n_slots);
  cudaStream_t st = c->stream;
  cudaError_t e;
  int s;
  // parameters: [albedo | emission] then the decision copy
  const int nt = 3 * (np + 1);
  std::vector<float> th(2 * (size_t)nt);
  for (int i = 0; i < 3 * np; ++i) {
    th[i] = albedo[i];
    th[nt + i] = dalb[i];
  }
  for (int i = 0; i < 3; ++i) {
    th[3 * np + i] = emission[i];
    th[nt + 3 * np + i] = dem[i];
  }
  float* dth = (float*)d.theta.ptr;
  if ((e = cudaMemcpyAsync(dth, th.data(), th.size() * 4, cudaMemcpyHostToDevice, st)))
    return cuda_status(c, e, "parameter upload");
  const int nf = (int)c->scene.n_faces;
  diff_apply_launch((const Material*)d.base_mat.ptr, (const int*)d.face_pid.ptr, nf, dth,
                    dth + 3 * np, (Material*)c->scene.mat.ptr, st);
  diff_apply_launch((const Material*)d.base_mat.ptr, (const int*)d.face_pid.ptr, nf, dth + nt,
                    dth + nt + 3 * np, (Material*)d.dec_mat.ptr, st);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_status(c, e, "parameters");
  // photon maps (integrator.h:393-563) with frozen decisions
  if ((s = trace_map(c, PM_MAP_GLOBAL, p.seed, p.n_photons, p.max_depth,
                     (const Material*)d.dec_mat.ptr, &d.first[0], nullptr)) != PM_OK)
    return s;
  if (need_caustics &&
      (s = trace_map(c, PM_MAP_CAUSTICS, p.seed + 1, p.n_photons_caustics, p.max_depth,
                     (const Material*)d.dec_mat.ptr, &d.first[1], nullptr)) != PM_OK)
    return s;
  // camera pass, one batch of all samples
  if ((s = render_buffers(c, npix, n_samples, n_slots)) != PM_OK) return s;
  if ((s = d.slot_pid.ensure((size_t)n_slots * 8)) || (s = d.nee.ensure((size_t)n_slots * 16)) ||
      (s = d.nee_count.ensure((size_t)n_samples * 4)) ||
      (s = d.slot_adj.ensure((size_t)n_slots * 12)))
    return set_err(c, s, "differentiable render buffers");
  unsigned long long* dropped = (unsigned long long*)c->r_misc.ptr;
  if ((e = cudaMemsetAsync(c->r_accum.ptr, 0, (size_t)npix * 16, st)) ||
      (e = cudaMemsetAsync(c->r_misc.ptr, 0, 64, st)) ||
      (e = cudaMemsetAsync(c->dev_err.ptr, 0, 64, st)))
    return cuda_status(c, e, "render init");
  render_rng_init((unsigned long long*)c->r_rng.ptr, p.width, p.height, st);
  RenderArgs a = base_args(c, p.width, p.height, q_per_sample, p.final_gathering_depth,
                           p.max_depth, p.n_gather);
  a.cam_pos = v3(cam->position[0], cam->position[1], cam->position[2]);
  a.cam_fwd = v3(cam->forward[0], cam->forward[1], cam->forward[2]);
  a.cam_right = v3(cam->right[0], cam->right[1], cam->right[2]);
  a.cam_up = v3(cam->up[0], cam->up[1], cam->up[2]);
  a.focal = cam->focal_length;
  a.batch = p.spp;
  a.face_pid = (const int*)d.face_pid.ptr;
  a.slot_pid = (int2*)d.slot_pid.ptr;
  a.nee = (float4*)d.nee.ptr;
  a.nee_count = (int*)d.nee_count.ptr;
  render_camera(c->scene_view(), a, st);
  int64_t q_tot[2] = {0, 0};
  if ((s = answer_queries(c, a, n_samples, n_slots, need_caustics, p.k, p.k, q_tot, nullptr,
                          nullptr)) != PM_OK)
    return s;
  render_resolve(a.slots, a.sample_rec, (const float*)c->r_res.ptr, npix, p.spp, q_per_sample,
                 (float4*)c->r_accum.ptr, dropped, st);
  render_finish((const float4*)c->r_accum.ptr, npix, p.spp, (float*)c->q_out.ptr, st);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_status(c, e, "render");
  unsigned long long hd[2] = {0, 0};
  int herr = 0;
  if ((e = cudaMemcpyAsync(out_rgb, c->q_out.ptr, (size_t)npix * 12, cudaMemcpyDeviceToHost,
                           st)) ||
      (e = cudaMemcpyAsync(hd, dropped, 16, cudaMemcpyDeviceToHost, st)) ||
      (e = cudaMemcpyAsync(&herr, c->dev_err.ptr, 4, cudaMemcpyDeviceToHost, st)) ||
      (e = cudaStreamSynchronize(st)))
    return cuda_status(c, e, "render output");
  if (herr) {
    cudaMemsetAsync(c->dev_err.ptr, 0, 4, st);
    return set_err(c, PM_ERR_DEVICE_STATUS, "differentiable render: device error bits 0x%x",
                   herr);
  }
  d.width = p.width;
  d.height = p.height;
  d.spp = p.spp;
  d.q_per_sample = q_per_sample;
  d.k = p.k;
  d.max_depth = p.max_depth;
  d.fg_depth = p.final_gathering_depth;
  d.seed = p.seed;
  d.emitted[0] = p.n_photons;
  d.emitted[1] = need_caustics ? p.n_photons_caustics : 0;
  for (int i = 0; i < nt; ++i) d.theta_host[i] = th[i];
  d.ready = true;
  if (stats) {
    stats->samples = n_samples;
    stats->dropped_nan = (int64_t)hd[0];
    stats->dropped_negative = (int64_t)hd[1];
    stats->queries_global = q_tot[0];
    stats->queries_caustics = q_tot[1];
    stats->passes = 1;
    stats->reserved = 0;
    stats->accum_rel_err = 0.0;
  }
  return PM_OK;
}

extern "C" int pm_diff_backward(pm_ctx* c, const float* grad_rgb, float* grad_albedo,
                                float* grad_emission) {
  if (!c) return PM_ERR_INVALID_ARGUMENT;
  if (!grad_rgb || !grad_emission)
    return set_err(c, PM_ERR_INVALID_ARGUMENT, "gradient arrays");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  DiffState& d = c->diff;
  if (!d.ready || d.scene_generation != c->scene.generation)
    return set_err(c, PM_ERR_NOT_BUILT, "no pm_diff_forward to differentiate");
  const int np = d.n_params;
  if (np > 0 && !grad_albedo) return set_err(c, PM_ERR_INVALID_ARGUMENT, "grad_albedo");
  const bool need_caustics = d.fg_depth > 0;
  const int npix = d.width * d.height;
  const int64_t n_samples = (int64_t)npix * d.spp;
  const int64_t n_slots = n_samples * d.q_per_sample;
  cudaStream_t st = c->stream;
  cudaError_t e;
  int s;
  if ((s = c->q_in.ensure((size_t)npix * 12)) != PM_OK) return set_err(c, s, "gradient input");
  const int ng = 3 * (np + 1);
  double* dg = (double*)d.grad.ptr;
  if ((e = cudaMemcpyAsync(c->q_in.ptr, grad_rgb, (size_t)npix * 12, cudaMemcpyHostToDevice,
                           st)) ||
      (e = cudaMemsetAsync(dg, 0, (size_t)ng * 8, st)))
    return cuda_status(c, e, "gradient upload");
  // 1. the camera pass's terms
  DiffAdjointArgs g{};
  g.slots = (const float4*)c->r_slots.ptr;
  g.srec = (const float4*)c->r_srec.ptr;
  g.res = (const float*)c->r_res.ptr;
  g.slot_pid = (const int2*)d.slot_pid.ptr;
  g.nee = (const float4*)d.nee.ptr;
  g.nee_count = (const int*)d.nee_count.ptr;
  g.grad_img = (const float*)c->q_in.ptr;
  g.npix = npix;
  g.spp = d.spp;
  g.q_per_sample = d.q_per_sample;
  g.n_params = np;
  g.slot_adj = (float*)d.slot_adj.ptr;
  g.grad = dg;
  diff_adjoint_samples_launch(g, st);
  // 2. estimates -> photon throughputs
  float4* padj[2] = {nullptr, nullptr};
  for (int map = 0; map < 2; ++map) {
    if (map == 1 && !need_caustics) continue;
    const int64_t n = c->maps[map].n;
    if ((s = d.photon_adj[map].ensure((size_t)(n > 0 ? n : 1) * 16)) != PM_OK)
      return set_err(c, s, "photon adjoints");
    padj[map] = (float4*)d.photon_adj[map].ptr;
    if (n > 0 && (e = cudaMemsetAsync(padj[map], 0, (size_t)n * 16, st)))
      return cuda_status(c, e, "photon adjoints");
  }
  RenderArgs a = base_args(c, d.width, d.height, d.q_per_sample, d.fg_depth, d.max_depth, 1);
  a.batch = d.spp;
  int64_t q_tot[2] = {0, 0};
  if ((s = answer_queries(c, a, n_samples, n_slots, need_caustics, d.k, d.k, q_tot,
                          (const float*)d.slot_adj.ptr, padj)) != PM_OK)
    return s;
  // 3. photon throughputs -> parameters, paths replayed from the seeds
  for (int map = 0; map < 2; ++map) {
    if (map == 1 && !need_caustics) continue;
    if (c->maps[map].n == 0 || np == 0) continue;
    TraceArgs t{};
    t.seed = map == 0 ? d.seed : d.seed + 1;
    t.n_emit = (int)d.emitted[map];
    t.max_depth = d.max_depth;
    t.caustic = map;
    t.cap = (unsigned long long)c->maps[map].n;
    t.next = (unsigned long long*)((char*)c->trace_misc.ptr + 32);
    t.dmat = (const Material*)d.dec_mat.ptr;
    t.first = (const uint32_t*)d.first[map].ptr;
    t.adj = padj[map];
    t.face_pid = (const int*)d.face_pid.ptr;
    t.n_params = np;
    t.grad = dg;
    trace_launch(c->scene_view(), t, st);
  }
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_status(c, e, "adjoint");
  std::vector<double> hg((size_t)ng);
  if ((e = cudaMemcpyAsync(hg.data(), dg, (size_t)ng * 8, cudaMemcpyDeviceToHost, st)) ||
      (e = cudaStreamSynchronize(st)))
    return cuda_status(c, e, "adjoint output");
  if ((s = take_device_error(c, "adjoint")) != PM_OK) return s;
  // 4. d loss / d theta = G / theta
  for (int i = 0; i < 3 * np; ++i) grad_albedo[i] = (float)(hg[i] / d.theta_host[i]);
  for (int i = 0; i < 3; ++i)
    grad_emission[i] = (float)(hg[3 * np + i] / d.theta_host[3 * np + i]);
  return PM_OK;
}
