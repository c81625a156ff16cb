// Drop-in for the reference's light.h: area lights and triangles are part of
// the device scene (photon_mapping_b200/csrc/pm_scene.cuh); see scene.h.
#ifndef PM_DROPIN_LIGHT_H
#define PM_DROPIN_LIGHT_H
#include "core.h"
#include "sampler.h"
#endif
