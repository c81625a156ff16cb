// Camera-pipeline helpers shared by the render entry points
// (pm_api_render.cu) and the differentiable render (pm_api_diff.cu).
#pragma once

#include "pm_api_internal.cuh"
#include "pm_render.cuh"

namespace pm {

// Buffers of the camera pipeline: npix pixel (or ray) slots, n_samples
// samples per pass, n_slots query slots per pass.
int render_buffers(pm_ctx* c, int npix, int64_t n_samples, int64_t n_slots);

int answer_queries(pm_ctx* c, const RenderArgs& a, int64_t ns, int64_t n_slots,
                   bool need_caustics, int kg, int kc, int64_t* q_tot,
                   const float* slot_adj, float4* const* photon_adj);

RenderArgs base_args(pm_ctx* c, int width, int height, int q_per_sample, int fg_depth,
                     int max_depth, int n_gather);

// Query slots per sample.
int slots_per_sample(const pm_ctx* c, bool need_caustics, int n_gather);

}  // namespace pm
