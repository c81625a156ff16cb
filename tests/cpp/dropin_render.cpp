// Exercises the drop-in C++ API (photon_mapping_b200/cpp/include) the way
// the reference's examples/main.cpp and tests/*.cpp use it: loads an OBJ
// from the working directory, builds the scene and the photon maps, renders
// a small image ray by ray (integrate) and in one call (render), queries
// the photon map per pixel, and writes raw float images for the test.
//   dropin_render <scene.obj> <width> <height> <spp> <out prefix>
#include <omp.h>

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

#include "camera.h"
#include "image.h"
#include "integrator.h"
#include "photon_map.h"
#include "scene.h"

static void dump(const std::string& path, Image& img) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char*>(img.data()),
          sizeof(float) * 3 * img.getWidth() * img.getHeight());
}

int main(int argc, char** argv) {
  if (argc < 6) return 2;
  const std::string obj = argv[1];
  const int width = std::atoi(argv[2]), height = std::atoi(argv[3]), n_samples = std::atoi(argv[4]);
  const std::string out = argv[5];

  Scene scene;
  scene.loadModel(obj);
  scene.build();
  Camera camera(Vec3f(0.5f, 0.5f, 4.7f), Vec3f(0, 0, -1), 0.25 * PI);

  PhotonMapping integrator(20000, 30, 1.0f, 30, 1, 12);
  UniformSampler sampler;
  integrator.build(scene, sampler);

  // the reference's render loop, one integrate() per camera ray
  Image image(width, height);
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
  for (int i = 0; i < height; ++i) {
    for (int j = 0; j < width; ++j) {
      UniformSampler px(j + width * i);
      for (int k = 0; k < n_samples; ++k) {
        const float u = (2.0f * (j + px.getNext1D()) - width) / height;
        const float v = (2.0f * (i + px.getNext1D()) - height) / height;
        Ray ray;
        float pdf;
        if (camera.sampleRay(Vec2f(u, v), ray, pdf)) {
          const Vec3f radiance = integrator.integrate(ray, scene, px) / pdf;
          if (std::isnan(radiance[0]) || std::isnan(radiance[1]) || std::isnan(radiance[2])) continue;
          if (radiance[0] < 0 || radiance[1] < 0 || radiance[2] < 0) continue;
          image.addPixel(i, j, radiance);
        }
      }
    }
  }
  image.divide(n_samples);
  dump(out + "_perray.f32", image);

  Image batched(width, height);
  integrator.render(scene, camera, batched, n_samples);
  dump(out + "_batched.f32", batched);

  // tests/visualize_photon_map.cpp: k = 1 per primary hit
  const PhotonMap* pm = integrator.getPhotonMapPtr();
  Image nearest(width, height);
  std::vector<int> idx(width * height, -1);
  for (int i = 0; i < height; ++i)
    for (int j = 0; j < width; ++j) {
      Ray ray;
      float pdf;
      camera.sampleRay(Vec2f((2.0f * j - width) / height, (2.0f * i - height) / height), ray, pdf);
      IntersectInfo info;
      if (scene.intersect(ray, info)) {
        float r2;
        const std::vector<int> ids = pm->queryKNearestPhotons(info.surfaceInfo.position, 1, r2);
        if (!ids.empty()) {
          idx[i * width + j] = ids[0];
          nearest.setPixel(i, j, pm->getIthPhoton(ids[0]).throughput);
        }
      }
    }
  dump(out + "_nearest.f32", nearest);
  std::ofstream(out + "_nearest_idx.i32", std::ios::binary)
      .write(reinterpret_cast<const char*>(idx.data()), sizeof(int) * idx.size());

  // PathTracing, per ray and batched
  PathTracing pt(12);
  Image ptimg(width, height);
  for (int i = 0; i < height; ++i)
    for (int j = 0; j < width; ++j) {
      UniformSampler px(j + width * i);
      for (int k = 0; k < n_samples; ++k) {
        const float u = (2.0f * (j + px.getNext1D()) - width) / height;
        const float v = (2.0f * (i + px.getNext1D()) - height) / height;
        Ray ray;
        float pdf;
        camera.sampleRay(Vec2f(u, v), ray, pdf);
        const Vec3f radiance = pt.integrate(ray, scene, px) / pdf;
        if (std::isnan(radiance[0]) || std::isnan(radiance[1]) || std::isnan(radiance[2])) continue;
        ptimg.addPixel(i, j, radiance);
      }
    }
  ptimg.divide(n_samples);
  dump(out + "_pt_perray.f32", ptimg);
  Image ptb(width, height);
  pt.render(scene, camera, ptb, n_samples);
  dump(out + "_pt_batched.f32", ptb);
  std::printf("photons %d\n", pm->getNPhotons());
  return 0;
}
