// Host-side launchers of the scene build and of the batched intersection.
#pragma once

#include "pm_scene.cuh"

namespace pm {

// Scratch bytes scene_build_launch needs for n faces.
size_t scene_build_scratch_bytes(int n);

// verts / nrms: device, 9 floats per face. Fills tri, nrm, geo (face
// order), mt (leaf order) and nodes (n - 1 internal nodes). Synchronises st
// once per clustering pass (it reads the clusters left).
cudaError_t scene_build_launch(const float* verts, const float* nrms, int n, float4* tri,
                               float4* nrm, float4* geo, float4* mt, float4* nodes,
                               void* scratch, cudaStream_t st);

// rays: 2 float4 per ray {origin, tmin}, {direction, tmax}; out: one float4
// per ray {t, u, v, face id bits (-1: miss)}.
void intersect_launch(const SceneDev& sc, const float4* rays, int64_t n,
                      float4* out, cudaStream_t st);

}  // namespace pm
