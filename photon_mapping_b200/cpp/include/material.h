// Drop-in for the reference's material.h: the BxDF kinds and transport
// directions (material.h:8-10). The BxDFs themselves run on the device
// (photon_mapping_b200/csrc/pm_math.cuh); a face's material is the
// pm_material record Scene::loadModel derives from the MTL file.
#ifndef PM_DROPIN_MATERIAL_H
#define PM_DROPIN_MATERIAL_H
#include <utility>

#include "core.h"

enum class BxDFType { DIFFUSE, SPECULAR };
enum class TransportDirection { FROM_LIGHT, FROM_CAMERA };
using DirectionPair = std::pair<Vec3f, Vec3f>;

#endif
