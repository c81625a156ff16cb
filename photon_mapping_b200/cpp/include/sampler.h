// Drop-in for the reference's sampler.h (sampler.h:9-91): the PCG32 RNG
// with state = seed and inc = 1, Sampler / UniformSampler and
// sampleCosineHemisphere. getSeed() returns the generator's current state,
// which is how the device entry points continue a caller's stream.
#ifndef PM_DROPIN_SAMPLER_H
#define PM_DROPIN_SAMPLER_H
#include <algorithm>
#include <cstdint>
#include <limits>
#include <memory>

#include "core.h"

class RNG {
  uint64_t state_ = 1;

 public:
  RNG() {}
  RNG(uint64_t seed) : state_(seed) {}
  uint64_t getSeed() const { return state_; }
  void setSeed(uint64_t seed) { state_ = seed; }
  uint32_t next_u32() {
    const uint64_t old = state_;
    state_ = old * 6364136223846793005ULL + 1ULL;
    const uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    const uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((0u - rot) & 31u));
  }
  float getNext() {
    constexpr float divider = 1.0f / std::numeric_limits<uint32_t>::max();
    return next_u32() * divider;
  }
};

class Sampler {
 protected:
  RNG rng;

 public:
  Sampler() {}
  Sampler(uint64_t seed) : rng(seed) {}
  virtual ~Sampler() {}
  uint64_t getSeed() const { return rng.getSeed(); }
  void setSeed(uint64_t seed) { rng.setSeed(seed); }
  virtual std::unique_ptr<Sampler> clone() const = 0;
  virtual float getNext1D() = 0;
  virtual Vec2f getNext2D() = 0;
};

class UniformSampler : public Sampler {
 public:
  UniformSampler() : Sampler() {}
  UniformSampler(uint64_t seed) : Sampler(seed) {}
  std::unique_ptr<Sampler> clone() const override { return std::make_unique<UniformSampler>(); }
  float getNext1D() override { return rng.getNext(); }
  // the reference's Vec2f(getNext(), getNext()): its GCC build evaluates
  // the second argument first, so the first draw lands in v[1]
  Vec2f getNext2D() override {
    const float draw1 = rng.getNext();
    const float draw2 = rng.getNext();
    return Vec2f(draw2, draw1);
  }
};

inline Vec3f sampleCosineHemisphere(const Vec2f& uv, float& pdf) {
  const float theta = 0.5f * std::acos(std::clamp(1.0f - 2.0f * uv[0], -1.0f, 1.0f));
  const float phi = PI_MUL_2 * uv[1];
  pdf = PI_INV * std::cos(theta);
  return sphericalToCartesian(theta, phi);
}

#endif
