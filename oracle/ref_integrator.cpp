// ORACLE — test infrastructure only. Compiles the reference's own Scene,
// PhotonMapping and PathTracing (include/scene.h and include/integrator.h
// of yumcyaWiz/photon_mapping, unchanged, read from the reference tree at
// build time) into oracle/_ref/libpmref_integrator.so. Embree 3 and
// tinyobjloader are not in this image: oracle/shim holds project-written
// stand-ins for the calls scene.h makes (a CPU BVH with the project's
// Moller-Trumbore arithmetic, and an OBJ/MTL reader). The library times the
// reference's CPU renderer and checks the GPU renderer against it
// statistically (both are Monte Carlo estimators of the same image; their
// random streams differ).
#include <omp.h>
#include <unistd.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <concepts>
#include <cstdint>
#include <filesystem>
#include <fstream>
#include <functional>
#include <iostream>
#include <limits>
#include <memory>
#include <numeric>
#include <optional>
#include <queue>
#include <string>
#include <vector>

#include <embree3/rtcore.h>

#include "spdlog/spdlog.h"
#include "tiny_obj_loader.h"
// Reference headers. Their photon maps are private members; the harness
// replaces them with given photon sets (ref_int_set_maps) so the camera pass
// can be compared per pixel, so members are made reachable while these
// headers are read. Every standard header they use is included above.
#define private public
#include "camera.h"
#include "integrator.h"
#include "scene.h"
#undef private

namespace {

struct RefRenderer {
  Scene scene;
  std::unique_ptr<PhotonMapping> pm;
  int64_t n_global = 0, n_caustics = 0;
};

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// The reference's loader reads the MTL file from "./" (scene.h:116), so the
// OBJ is parsed with its own directory as the working directory.
bool load_scene(Scene& scene, const char* dir, const char* obj) {
  char prev[4096];
  if (!getcwd(prev, sizeof(prev))) return false;
  if (chdir(dir) != 0) return false;
  scene.loadModel(obj);
  const bool ok = chdir(prev) == 0;
  if (ok) scene.build();
  return ok && scene.nFaces() > 0;
}

// The per-pixel loop of examples/main.cpp:33-66 over rows [row0, row1):
// `integrate` returns one camera sample's radiance; NaN and negative
// samples are dropped as there. out holds the raw per-pixel mean over spp.
template <class F>
void pixel_loop(const float* cam, int width, int height, int spp, int row0, int row1,
                float* out, F&& integrate) {
  const Camera camera(Vec3f(cam[0], cam[1], cam[2]), Vec3f(cam[3], cam[4], cam[5]), cam[6]);
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
  for (int i = row0; i < row1; ++i) {
    for (int j = 0; j < width; ++j) {
      UniformSampler sampler(j + width * i);
      Vec3f sum(0);
      for (int k = 0; k < spp; ++k) {
        const float u = (2.0f * (j + sampler.getNext1D()) - width) / height;
        const float v = (2.0f * (i + sampler.getNext1D()) - height) / height;
        Ray ray;
        float pdf;
        if (camera.sampleRay(Vec2f(u, v), ray, pdf)) {
          const Vec3f radiance = integrate(ray, sampler) / pdf;
          if (std::isnan(radiance[0]) || std::isnan(radiance[1]) || std::isnan(radiance[2]))
            continue;
          if (radiance[0] < 0 || radiance[1] < 0 || radiance[2] < 0) continue;
          sum += radiance;
        }
      }
      float* o = out + 3 * ((int64_t)(i - row0) * width + j);
      o[0] = sum[0] / spp;
      o[1] = sum[1] / spp;
      o[2] = sum[2] / spp;
    }
  }
}

}  // namespace

extern "C" {

int ref_int_max_threads() { return omp_get_max_threads(); }

// Scene::loadModel + Scene::build (scene.h:108-304).
void* ref_int_new(const char* dir, const char* obj) {
  RefRenderer* r = new RefRenderer();
  if (!load_scene(r->scene, dir, obj)) {
    delete r;
    return nullptr;
  }
  return r;
}

void ref_int_free(void* h) { delete (RefRenderer*)h; }

// PhotonMapping constructor + build (integrator.h:380-563), with the
// UniformSampler the example passes. Returns the build's seconds.
double ref_int_build(void* h, int n_photons, int n_est_global, float caustics_multiplier,
                     int n_est_caustics, int fg_depth, int max_depth) {
  RefRenderer* r = (RefRenderer*)h;
  r->pm.reset(new PhotonMapping(n_photons, n_est_global, caustics_multiplier, n_est_caustics,
                                fg_depth, max_depth));
  UniformSampler sampler;
  const double t0 = now_s();
  r->pm->build(r->scene, sampler);
  const double t1 = now_s();
  r->n_global = r->pm->getPhotonMapPtr()->getNPhotons();
  return t1 - t0;
}

// A PhotonMapping whose global and caustics maps hold the given photons
// (9 floats each: throughput, position, wi — photon_map.h Photon) instead
// of traced ones: the constructor as integrator.h:380-389, then
// PhotonMap::setPhotons + build (photon_map.h:198-206) on each map.
void ref_int_set_maps(void* h, const float* global, int64_t n_global, const float* caustics,
                      int64_t n_caustics, int n_photons, int n_est_global,
                      float caustics_multiplier, int n_est_caustics, int fg_depth,
                      int max_depth) {
  RefRenderer* r = (RefRenderer*)h;
  r->pm.reset(new PhotonMapping(n_photons, n_est_global, caustics_multiplier, n_est_caustics,
                                fg_depth, max_depth));
  auto fill = [](PhotonMap& m, const float* ph, int64_t n) {
    std::vector<Photon> v((size_t)n);
    for (int64_t i = 0; i < n; ++i) {
      const float* q = ph + 9 * i;
      v[i] = Photon(Vec3f(q[0], q[1], q[2]), Vec3f(q[3], q[4], q[5]), Vec3f(q[6], q[7], q[8]));
    }
    m.setPhotons(v);
    m.build();
  };
  fill(r->pm->globalPhotonMap, global, n_global);
  fill(r->pm->causticsPhotonMap, caustics, n_caustics);
  r->n_global = n_global;
}

int64_t ref_int_n_photons(void* h) { return ((RefRenderer*)h)->n_global; }

// PhotonMapping::integrate over rows [row0, row1) of a width x height image
// (cam = position xyz, forward xyz, fov). Returns the seconds taken.
double ref_int_render(void* h, const float* cam, int width, int height, int spp, int row0,
                      int row1, float* out) {
  RefRenderer* r = (RefRenderer*)h;
  const double t0 = now_s();
  pixel_loop(cam, width, height, spp, row0, row1, out,
             [&](const Ray& ray, Sampler& s) { return r->pm->integrate(ray, r->scene, s); });
  return now_s() - t0;
}

// PathTracing::integrate (integrator.h:60-105), the loop of
// tests/test_path_tracing.cpp:25-58 over rows [row0, row1).
double ref_int_render_pt(void* h, const float* cam, int width, int height, int spp, int max_depth,
                         int row0, int row1, float* out) {
  RefRenderer* r = (RefRenderer*)h;
  const PathTracing pt(max_depth);
  const double t0 = now_s();
  pixel_loop(cam, width, height, spp, row0, row1, out,
             [&](const Ray& ray, Sampler& s) { return pt.integrate(ray, r->scene, s); });
  return now_s() - t0;
}

}  // extern "C"
