// Camera-pass launchers (see pm_render.cu).
#pragma once

#include "pm_scene.cuh"

namespace pm {

enum { kQueryGlobal = 0, kQueryCaustics = 1 };

struct RenderArgs {
  V3 cam_pos, cam_fwd, cam_right, cam_up;
  float focal;
  int width, height;
  int batch;         // samples per pixel in this pass
  int q_per_sample;  // query slots per sample
  int fg_depth;      // finalGatheringDepth
  int max_depth;
  int n_gather;      // gather rays per diffuse hit (1 in the reference)
  V3 inv_gather;     // 1 / n_gather
  unsigned long long* rng_state;  // per pixel, kept across passes
  float4* slots;       // 4 float4 per query slot
  float4* sample_rec;  // per sample {direct radiance, query count bits}
  const float* in_rays;  // null: camera rays; else 6 floats per pixel slot
  int* err;            // bit 1: slots exhausted, bit 2: path stack full
  // Differentiable render (null otherwise): what the adjoint pass needs to
  // split each sample's radiance by albedo parameter.
  const int* face_pid;  // albedo parameter of each face, -1 for none
  int2* slot_pid;       // per slot {parameter whose BSDF scaled the weight,
                        //           parameter of the query surface}
  float4* nee;          // per sample, q_per_sample records {next-event
                        // radiance, parameter of the surface (int bits)}
  int* nee_count;       // per sample
  unsigned long long* rays;  // closest-hit queries of the pass (added to), or null
};

struct PathArgs {
  V3 cam_pos, cam_fwd, cam_right, cam_up;
  float focal;
  int width, height, spp, max_depth;
  float* out;                    // height x width x 3, averaged
  unsigned long long* dropped;   // NaN samples
  const float* in_rays;          // null: camera rays; else 6 floats per ray
  unsigned long long* rng_states;  // with in_rays: per-ray sampler states
};

void render_path_tracing(const SceneDev& sc, const PathArgs& a, cudaStream_t s);

void render_rng_init(unsigned long long* st, int w, int h, cudaStream_t s);
void render_camera(const SceneDev& sc, const RenderArgs& a, cudaStream_t s);
void render_list_queries(const float4* slots, const float4* srec,
                         int64_t n_samples, int q_per_sample, int map,
                         const float* scene_lo, const float* scene_hi,
                         uint32_t* keys, uint32_t* vals, unsigned* count,
                         cudaStream_t s);
// raw != null: write each sample's radiance there instead of accumulating.
// shadow != null: also add every kept sample to the pixel's FP64 sums
// (3 doubles per pixel).
void render_resolve(const float4* slots, const float4* srec, const float* res,
                    int npix, int batch, int q_per_sample, float4* accum,
                    unsigned long long* dropped, cudaStream_t s,
                    float* raw = nullptr, double* shadow = nullptr);
// Largest relative difference between out (the image, height x width x 3)
// and shadow / spp, as float bits in *max_bits (atomicMax; start it at 0).
void render_shadow_compare(const float* out, const double* shadow, int npix, int spp,
                           unsigned* max_bits, cudaStream_t s);
void render_finish(const float4* accum, int npix, int spp, float* out,
                   cudaStream_t s);

}  // namespace pm
