// Drop-in for the reference's core.h: vector types, rays and hit records
// with the same names, members and operators (core.h:1-287 of
// yumcyaWiz/photon_mapping). Header-only, host side.
#ifndef PM_DROPIN_CORE_H
#define PM_DROPIN_CORE_H
#include <cmath>
#include <cstdint>
#include <iostream>
#include <limits>

constexpr float PI = 3.14159265359;
constexpr float PI_MUL_2 = 2.0f * PI;
constexpr float PI_MUL_4 = 4.0f * PI;
constexpr float PI_DIV_2 = 0.5f * PI;
constexpr float PI_DIV_4 = 0.25f * PI;
constexpr float PI_INV = 1.0f / PI;
constexpr float PI_MUL_2_INV = 1.0f / PI_MUL_2;
constexpr float PI_MUL_4_INV = 1.0f / PI_MUL_4;
constexpr float RAY_EPS = 1e-5f;

inline float rad2deg(float rad) { return 180.0f * rad / PI; }
inline float deg2rad(float deg) { return deg / 180.0f * PI; }

template <typename T, int N>
struct VecN {
  T v[N];
  static constexpr int dim = N;
  T operator[](int i) const { return v[i]; }
  T& operator[](int i) { return v[i]; }
};

template <typename T>
struct Vec2 : VecN<T, 2> {
  Vec2() { this->v[0] = this->v[1] = 0; }
  Vec2(T x) { this->v[0] = this->v[1] = x; }
  Vec2(T x, T y) {
    this->v[0] = x;
    this->v[1] = y;
  }
  Vec2 operator-() const { return Vec2(-this->v[0], -this->v[1]); }
  Vec2& operator+=(const Vec2& o) { for (int i = 0; i < 2; ++i) this->v[i] += o.v[i]; return *this; }
  Vec2& operator*=(const Vec2& o) { for (int i = 0; i < 2; ++i) this->v[i] *= o.v[i]; return *this; }
  Vec2& operator/=(const Vec2& o) { for (int i = 0; i < 2; ++i) this->v[i] /= o.v[i]; return *this; }
};

template <typename T>
struct Vec3 : VecN<T, 3> {
  Vec3() { this->v[0] = this->v[1] = this->v[2] = 0; }
  Vec3(T x) { this->v[0] = this->v[1] = this->v[2] = x; }
  Vec3(T x, T y, T z) {
    this->v[0] = x;
    this->v[1] = y;
    this->v[2] = z;
  }
  Vec3 operator-() const { return Vec3(-this->v[0], -this->v[1], -this->v[2]); }
  Vec3& operator+=(const Vec3& o) { for (int i = 0; i < 3; ++i) this->v[i] += o.v[i]; return *this; }
  Vec3& operator*=(const Vec3& o) { for (int i = 0; i < 3; ++i) this->v[i] *= o.v[i]; return *this; }
  Vec3& operator/=(const Vec3& o) { for (int i = 0; i < 3; ++i) this->v[i] /= o.v[i]; return *this; }
};

// element-wise arithmetic, vector (op) vector and vector (op) scalar, in
// component order
#define PM_DROPIN_OPS(V, N)                                                              \
  template <typename T> inline V<T> operator+(const V<T>& a, const V<T>& b) { V<T> r; for (int i = 0; i < N; ++i) r[i] = a[i] + b[i]; return r; } \
  template <typename T> inline V<T> operator-(const V<T>& a, const V<T>& b) { V<T> r; for (int i = 0; i < N; ++i) r[i] = a[i] - b[i]; return r; } \
  template <typename T> inline V<T> operator*(const V<T>& a, const V<T>& b) { V<T> r; for (int i = 0; i < N; ++i) r[i] = a[i] * b[i]; return r; } \
  template <typename T> inline V<T> operator/(const V<T>& a, const V<T>& b) { V<T> r; for (int i = 0; i < N; ++i) r[i] = a[i] / b[i]; return r; } \
  template <typename T> inline V<T> operator+(const V<T>& a, float k) { V<T> r; for (int i = 0; i < N; ++i) r[i] = a[i] + k; return r; } \
  template <typename T> inline V<T> operator-(const V<T>& a, float k) { V<T> r; for (int i = 0; i < N; ++i) r[i] = a[i] - k; return r; } \
  template <typename T> inline V<T> operator*(const V<T>& a, float k) { V<T> r; for (int i = 0; i < N; ++i) r[i] = a[i] * k; return r; } \
  template <typename T> inline V<T> operator/(const V<T>& a, float k) { V<T> r; for (int i = 0; i < N; ++i) r[i] = a[i] / k; return r; } \
  template <typename T> inline V<T> operator+(float k, const V<T>& a) { return a + k; }  \
  template <typename T> inline V<T> operator-(float k, const V<T>& a) { V<T> r; for (int i = 0; i < N; ++i) r[i] = k - a[i]; return r; } \
  template <typename T> inline V<T> operator*(float k, const V<T>& a) { return a * k; }  \
  template <typename T> inline V<T> operator/(float k, const V<T>& a) { V<T> r; for (int i = 0; i < N; ++i) r[i] = k / a[i]; return r; }
PM_DROPIN_OPS(Vec2, 2)
PM_DROPIN_OPS(Vec3, 3)
#undef PM_DROPIN_OPS

using Vec2f = Vec2<float>;
using Vec3f = Vec3<float>;
using Vec3ui = Vec3<uint32_t>;

template <typename T>
inline T dot(const Vec3<T>& a, const Vec3<T>& b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
template <typename T>
inline Vec3<T> cross(const Vec3<T>& a, const Vec3<T>& b) {
  return Vec3<T>(a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]);
}
inline float length(const Vec3f& v) { return std::sqrt(dot(v, v)); }
inline float length2(const Vec3f& v) { return dot(v, v); }
inline Vec3f normalize(const Vec3f& v) { return v / length(v); }

inline void orthonormalBasis(const Vec3f& n, Vec3f& t, Vec3f& b) {
  t = std::abs(n[1]) < 0.9f ? normalize(cross(n, Vec3f(0, 1, 0)))
                            : normalize(cross(n, Vec3f(0, 0, -1)));
  b = normalize(cross(t, n));
}
inline Vec3f worldToLocal(const Vec3f& v, const Vec3f& lx, const Vec3f& ly, const Vec3f& lz) {
  return Vec3f(dot(v, lx), dot(v, ly), dot(v, lz));
}
inline Vec3f localToWorld(const Vec3f& v, const Vec3f& lx, const Vec3f& ly, const Vec3f& lz) {
  Vec3f r;
  for (int i = 0; i < 3; ++i) r[i] = v[0] * lx[i] + v[1] * ly[i] + v[2] * lz[i];
  return r;
}
inline Vec3f sphericalToCartesian(float theta, float phi) {
  return Vec3f(std::cos(phi) * std::sin(theta), std::cos(theta), std::sin(phi) * std::sin(theta));
}

struct Ray {
  Vec3f origin;
  Vec3f direction;
  static constexpr float tmin = RAY_EPS;
  mutable float tmax = std::numeric_limits<float>::max();
  Ray() {}
  Ray(const Vec3f& o, const Vec3f& d) : origin(o), direction(d) {}
  Vec3f operator()(float t) const { return origin + t * direction; }
};

struct SurfaceInfo {
  Vec3f position;
  Vec3f geometricNormal;
  Vec3f shadingNormal;
  Vec3f dpdu;
  Vec3f dpdv;
  Vec2f texcoords;
  Vec2f barycentric;
};

class Primitive;

struct IntersectInfo {
  float t;
  SurfaceInfo surfaceInfo;
  const Primitive* hitPrimitive;
};

#endif
