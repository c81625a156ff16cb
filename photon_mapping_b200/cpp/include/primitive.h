// Drop-in for the reference's primitive.h: a face with its material and
// area light (primitive.h:12-83). Shading runs on the device; the host
// object answers the questions user code asks about a hit.
#ifndef PM_DROPIN_PRIMITIVE_H
#define PM_DROPIN_PRIMITIVE_H
#include <cstdint>

#include "core.h"
#include "material.h"
#include "pm_cuda.h"

class Primitive {
  uint32_t faceID;
  pm_material mat;

 public:
  Primitive(uint32_t faceID, const pm_material& m) : faceID(faceID), mat(m) {}
  uint32_t getFaceID() const { return faceID; }
  const pm_material& getMaterial() const { return mat; }
  bool hasAreaLight() const { return mat.le[0] > 0 || mat.le[1] > 0 || mat.le[2] > 0; }
  Vec3f Le(const SurfaceInfo&, const Vec3f&) const { return Vec3f(mat.le[0], mat.le[1], mat.le[2]); }
  BxDFType getBxDFType() const {
    return mat.type == PM_LAMBERT ? BxDFType::DIFFUSE : BxDFType::SPECULAR;
  }
  // Lambert::evaluate (material.h:80-88) in the hit's shading frame
  Vec3f evaluateBxDF(const Vec3f& wo, const Vec3f& wi, const SurfaceInfo& s,
                     const TransportDirection&) const {
    if (mat.type != PM_LAMBERT) return Vec3f(0);
    if (dot(wo, s.shadingNormal) < 0 || dot(wi, s.shadingNormal) < 0) return Vec3f(0);
    return Vec3f(mat.rho[0], mat.rho[1], mat.rho[2]) / PI;
  }
};

#endif
