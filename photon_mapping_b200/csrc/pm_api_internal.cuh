// Internal state behind the C ABI: the context, its device buffers and the
// device photon maps.
#pragma once

#include <cstdarg>
#include <mutex>
#include <string>

#include "../../include/pm_cuda.h"
#include "pm_photonmap.cuh"
#include "pm_scene.cuh"

namespace pm {

// Grow-only device allocation owned by a context.
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  int ensure(size_t n);  // PM_OK or PM_ERR_OUT_OF_MEMORY
  void release();
};

struct DevMap {
  int64_t n = 0;
  int nlevels = 0;
  int lvl_off[kMaxLevels] = {};
  int lvl_cnt[kMaxLevels] = {};
  DevBuf aos, pos4, thr4, wi2, boxes;
  bool built = false;
  void release() {
    aos.release();
    pos4.release();
    thr4.release();
    wi2.release();
    boxes.release();
    built = false;
    n = 0;
  }
};

struct DevScene {
  uint64_t generation = 0;  // bumped by every upload
  int64_t n_faces = 0;
  int n_lights = 0;
  bool has_specular = false;
  float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};  // bounds of the vertices
  DevBuf tri, nrm, geo, mat, lights, mt, nodes, verts_in, nrms_in;
  bool built = false;
  void release() {
    tri.release(); nrm.release(); geo.release(); mat.release();
    lights.release(); mt.release(); nodes.release();
    verts_in.release(); nrms_in.release();
    built = false;
    n_faces = 0;
  }
};

// State of the differentiable render between pm_diff_forward and
// pm_diff_backward.
struct DiffState {
  uint64_t scene_generation = ~0ull;  // scene the parameters were set for
  int n_params = 0;
  DevBuf face_pid, base_mat, dec_mat, theta, grad;
  DevBuf first[2];      // first stored photon of each emitted photon, per map
  DevBuf photon_adj[2]; // d loss / d throughput per stored photon, per map
  DevBuf slot_pid, nee, nee_count, slot_adj;
  // the last forward pass
  bool ready = false;
  int width = 0, height = 0, spp = 0, q_per_sample = 0, k = 0, max_depth = 0;
  int fg_depth = 0;
  uint64_t seed = 0;
  int64_t emitted[2] = {0, 0};
  float theta_host[3 * 33] = {};  // albedos then emission of the last forward
  void release() {
    face_pid.release(); base_mat.release(); dec_mat.release(); theta.release();
    grad.release(); first[0].release(); first[1].release();
    photon_adj[0].release(); photon_adj[1].release();
    slot_pid.release(); nee.release(); nee_count.release(); slot_adj.release();
    ready = false;
    scene_generation = ~0ull;
  }
};

inline SceneDev scene_view(const DevScene& scene, int* err) {
  SceneDev v;
  v.tri = (const float4*)scene.tri.ptr;
  v.nrm = (const float4*)scene.nrm.ptr;
  v.geo = (const float4*)scene.geo.ptr;
  v.mat = (const Material*)scene.mat.ptr;
  v.lights = (const int*)scene.lights.ptr;
  v.mt = (const float4*)scene.mt.ptr;
  v.nodes = (const float4*)scene.nodes.ptr;
  v.n_faces = (int)scene.n_faces;
  v.n_lights = scene.n_lights;
  v.err = err;
  return v;
}

// Work counters: each kNN launch takes the next slot of a ring, so launches
// in flight on different streams do not share a counter (up to kCounterRing
// launches in flight at once).
constexpr int kCounterRing = 64;

}  // namespace pm

struct pm_ctx {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  std::mutex mu;
  std::string err;
  pm::DevMap maps[2];
  int64_t map_emitted[2] = {0, 0};  // photons emitted for each traced map
  pm::DevScene scene;
  pm::DevBuf dev_err;   // device error word of the kernels (int)
  pm::DevBuf trace_raw, trace_keys, trace_misc;  // photon tracing buffers
  pm::DevBuf trace_count, trace_first;  // per emitted photon: stores, first index
  pm::DevBuf r_rng, r_accum, r_slots, r_srec, r_res, r_sort, r_misc;  // render
  pm::DevBuf r_shadow;  // FP64 per-pixel sums of PM_RENDER_FP64_CHECK
  pm::DevBuf scratch;  // map build scratch
  pm::DevBuf q_in, q_out;  // staging of the host-pointer entry points
  pm::DevBuf counter;      // kCounterRing work counters
  unsigned counter_next = 0;
  pm::DevBuf stats;        // pm_knn_stats counters (device)
  pm::DiffState diff;      // differentiable render
  bool stats_on = false;
  unsigned long long* stats_ptr() {
    return stats_on ? (unsigned long long*)stats.ptr : nullptr;
  }

  unsigned long long* next_counter() {
    unsigned long long* base = (unsigned long long*)counter.ptr;
    return base + (counter_next++ % pm::kCounterRing);
  }
  void release_all() {
    maps[0].release();
    maps[1].release();
    scratch.release();
    q_in.release();
    q_out.release();
    counter.release();
    stats.release();
    scene.release();
    dev_err.release();
    trace_raw.release();
    trace_keys.release();
    trace_misc.release();
    trace_count.release();
    trace_first.release();
    r_rng.release(); r_accum.release(); r_slots.release(); r_srec.release();
    r_res.release(); r_sort.release(); r_misc.release(); r_shadow.release();
    diff.release();
  }
  pm::SceneDev scene_view() const { return pm::scene_view(scene, (int*)dev_err.ptr); }
};

namespace pm {
int set_err(pm_ctx* c, int status, const char* fmt, ...);
int cuda_status(pm_ctx* c, cudaError_t e, const char* where);
MapDev map_view(const DevMap& dm);
int build_map(pm_ctx* c, DevMap& dm, const float* d_aos, int64_t n,
              cudaStream_t st);
int take_device_error(pm_ctx* c, const char* where);
// Uploads a scene and builds its BVH on stream st (synchronises st). On
// failure returns the status and names the step in *what.
int upload_scene(DevScene& sc, DevBuf& scratch, cudaStream_t st, const float* vertices,
                 const float* normals, const pm_material* materials, int64_t n,
                 const char** what);
// Traces `map` (the body of pm_photons_trace; the caller holds the lock).
// dmat: decision materials (frozen decisions) or null; first: receives the
// first stored photon of each emitted photon, or null.
int trace_map(pm_ctx* c, int map, uint64_t seed, int64_t n_emit, int max_depth,
              const Material* dmat, DevBuf* first, pm_trace_stats* stats);
}  // namespace pm
