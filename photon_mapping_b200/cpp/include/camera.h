// Drop-in for the reference's camera.h (camera.h:10-48): pinhole camera.
#ifndef PM_DROPIN_CAMERA_H
#define PM_DROPIN_CAMERA_H
#include <cmath>

#include "core.h"
#include "pm_cuda.h"
#include "spdlog/spdlog.h"

class Camera {
  Vec3f position, forward, right, up;
  float FOV;
  float focal_length;

 public:
  Camera(const Vec3f& position, const Vec3f& forward, float FOV = 0.5f * PI)
      : position(position), forward(forward), FOV(FOV) {
    right = normalize(cross(forward, Vec3f(0, 1, 0)));
    up = normalize(cross(right, forward));
    focal_length = 1.0f / std::tan(0.5f * FOV);
    spdlog::info("[Camera] focal_length: {}", focal_length);
  }

  // uv in [-1, 1]^2 on the sensor (camera.h:41-47)
  bool sampleRay(const Vec2f& uv, Ray& ray, float& pdf) const {
    const Vec3f pinhole = position + focal_length * forward;
    const Vec3f sensor = position + uv[0] * right + uv[1] * up;
    ray = Ray(sensor, normalize(pinhole - sensor));
    pdf = 1.0f;
    return true;
  }

  // the constructed camera, for pm_render
  pm_camera toDevice() const {
    pm_camera c;
    for (int i = 0; i < 3; ++i) {
      c.position[i] = position[i];
      c.forward[i] = forward[i];
      c.right[i] = right[i];
      c.up[i] = up[i];
    }
    c.focal_length = focal_length;
    return c;
  }
};

#endif
