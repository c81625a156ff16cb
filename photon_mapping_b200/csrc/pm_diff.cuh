// Kernels of the differentiable render (see pm_diff.cu).
#pragma once

#include "pm_scene.cuh"
#include "pm_trace.cuh"

namespace pm {

// Writes the albedo and emission parameters into the materials:
// out[f] = base[f], with rho = albedo[face_pid[f]] where face_pid[f] >= 0
// and le = emission where base[f] emits.
void diff_apply_launch(const Material* base, const int* face_pid, int n_faces,
                       const float* albedo, const float* emission, Material* out,
                       cudaStream_t st);

struct DiffAdjointArgs {
  const float4* slots;     // query slots of the forward camera pass
  const float4* srec;      // per sample {direct, query count}
  const float* res;        // estimate of each slot (3 floats)
  const int2* slot_pid;    // per slot {pid of the weight, pid of the query}
  const float4* nee;       // per sample, q_per_sample records
  const int* nee_count;    // per sample
  const float* grad_img;   // d loss / d image, height x width x 3
  int npix, spp, q_per_sample, n_params;
  float* slot_adj;         // out: d loss / d estimate per slot (3 floats)
  double* grad;            // out, accumulated: n_params x 3 sums, then 3 for
                           // the emission (d loss / d log parameter)
};

// One thread per pixel: the reverse of resolve + finish. Samples that the
// forward pass dropped (NaN or negative radiance) get no adjoint.
void diff_adjoint_samples_launch(const DiffAdjointArgs& a, cudaStream_t st);

}  // namespace pm
