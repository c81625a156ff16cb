// Drop-in for the reference's integrator.h (integrator.h:11-570):
// Integrator, PathTracing and PhotonMapping with the same constructors and
// build / integrate calls, running on the device through libpm_cuda.
//
// integrate() keeps the reference's per-ray contract: it is const, may be
// called from many host threads at once (calls on one context are
// serialised by the library) and advances the caller's sampler by exactly
// the draws the reference makes. A per-ray call is one device round trip;
// render() is the batched form of the reference's render loop
// (examples/main.cpp:33-70) for throughput.
#ifndef PM_DROPIN_INTEGRATOR_H
#define PM_DROPIN_INTEGRATOR_H
#include <cstdint>
#include <vector>

#include "camera.h"
#include "core.h"
#include "image.h"
#include "photon_map.h"
#include "pm_cuda.h"
#include "sampler.h"
#include "scene.h"
#include "spdlog/spdlog.h"

class Integrator {
 public:
  virtual ~Integrator() {}
  virtual void build(const Scene& scene, Sampler& sampler) = 0;
  virtual Vec3f integrate(const Ray& ray, const Scene& scene, Sampler& sampler) const = 0;
};

class PathTracing : public Integrator {
  const int maxDepth;

 public:
  PathTracing(int maxDepth = 100) : maxDepth(maxDepth) {}
  void build(const Scene&, Sampler&) override {}

  Vec3f integrate(const Ray& ray, const Scene& scene, Sampler& sampler) const override {
    const float r[6] = {ray.origin[0],    ray.origin[1],    ray.origin[2],
                        ray.direction[0], ray.direction[1], ray.direction[2]};
    uint64_t state = sampler.getSeed();
    float rgb[3];
    pm_dropin::check(scene.context(),
                     pm_path_trace_rays(scene.context(), r, 1, &state, maxDepth, rgb),
                     "pm_path_trace_rays");
    sampler.setSeed(state);
    return Vec3f(rgb[0], rgb[1], rgb[2]);
  }

  // tests/test_path_tracing.cpp:25-58 in one call: image = average of
  // n_samples samples per pixel (before gamma correction).
  void render(const Scene& scene, const Camera& camera, Image& image, int n_samples) const {
    const pm_camera cam = camera.toDevice();
    pm_dropin::check(scene.context(),
                     pm_render_path_tracing(scene.context(), &cam, (int32_t)image.getWidth(),
                                            (int32_t)image.getHeight(), n_samples, maxDepth,
                                            image.data(), nullptr),
                     "pm_render_path_tracing");
  }
};

class PhotonMapping : public Integrator {
  const int nPhotonsGlobal;
  const int nEstimationGlobal;
  const int nPhotonsCaustics;
  const int nEstimationCaustics;
  const int finalGatheringDepth;
  const int maxDepth;
  PhotonMap globalPhotonMap;
  PhotonMap causticsPhotonMap;

  pm_integrate_params params(int n_gather) const {
    pm_integrate_params p{};
    p.k_global = nEstimationGlobal;
    p.k_caustics = nEstimationGlobal;  // the reference's caustics estimate uses
                                       // nEstimationGlobal (integrator.h:161)
    p.final_gathering_depth = finalGatheringDepth;
    p.max_depth = maxDepth;
    p.n_gather = n_gather;
    return p;
  }

 public:
  PhotonMapping(int nPhotonsGlobal, int nEstimationGlobal, float nPhotonsCausticsMultiplier,
                int nEstimationCaustics, int strictCalcDepth, int maxDepth)
      : nPhotonsGlobal(nPhotonsGlobal),
        nEstimationGlobal(nEstimationGlobal),
        nPhotonsCaustics(nPhotonsGlobal * nPhotonsCausticsMultiplier),
        nEstimationCaustics(nEstimationCaustics),
        finalGatheringDepth(strictCalcDepth),
        maxDepth(maxDepth) {}

  const PhotonMap* getPhotonMapPtr() const { return &globalPhotonMap; }

  // integrator.h:393-563 on the device. The trace seed is the sampler's
  // current state; photon i uses its own stream derived from it.
  void build(const Scene& scene, Sampler& sampler) override {
    pm_ctx* ctx = scene.context();
    const uint64_t seed = sampler.getSeed();
    pm_trace_stats st;
    spdlog::info("[PhotonMapping] tracing photons to build global photon map");
    pm_dropin::check(ctx, pm_photons_trace(ctx, PM_MAP_GLOBAL, seed, nPhotonsGlobal, maxDepth, &st),
                     "pm_photons_trace");
    globalPhotonMap.bind(ctx, PM_MAP_GLOBAL);
    globalPhotonMap.pull();
    causticsPhotonMap.bind(ctx, PM_MAP_CAUSTICS);
    if (finalGatheringDepth > 0) {
      spdlog::info("[PhotonMapping] tracing photons to build caustics photon map");
      pm_dropin::check(ctx,
                       pm_photons_trace(ctx, PM_MAP_CAUSTICS, seed + 1, nPhotonsCaustics, maxDepth,
                                        &st),
                       "pm_photons_trace");
    } else {
      pm_dropin::check(ctx, pm_photonmap_build(ctx, PM_MAP_CAUSTICS, nullptr, 0),
                       "pm_photonmap_build");
    }
    causticsPhotonMap.pull();
  }

  // integrator.h:566-569
  Vec3f integrate(const Ray& ray, const Scene& scene, Sampler& sampler) const override {
    const float r[6] = {ray.origin[0],    ray.origin[1],    ray.origin[2],
                        ray.direction[0], ray.direction[1], ray.direction[2]};
    uint64_t state = sampler.getSeed();
    float rgb[3];
    const pm_integrate_params p = params(1);
    pm_dropin::check(scene.context(), pm_integrate(scene.context(), r, 1, &state, &p, rgb),
                     "pm_integrate");
    sampler.setSeed(state);
    return Vec3f(rgb[0], rgb[1], rgb[2]);
  }

  // The render loop of examples/main.cpp:33-67 in one call: every pixel's
  // sampler seeded j + width*i, NaN and negative samples dropped, image =
  // average of n_samples samples (before gamma correction). n_gather > 1
  // averages that many gather rays per diffuse hit.
  void render(const Scene& scene, const Camera& camera, Image& image, int n_samples,
              int n_gather = 1) const {
    const pm_camera cam = camera.toDevice();
    pm_render_params p{};
    p.width = (int32_t)image.getWidth();
    p.height = (int32_t)image.getHeight();
    p.spp = n_samples;
    p.k_global = nEstimationGlobal;
    p.k_caustics = nEstimationGlobal;
    p.final_gathering_depth = finalGatheringDepth;
    p.max_depth = maxDepth;
    p.n_gather = n_gather;
    pm_render_stats st;
    pm_dropin::check(scene.context(), pm_render(scene.context(), &cam, &p, image.data(), &st),
                     "pm_render");
  }
};

#endif
