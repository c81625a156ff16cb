// Batched rendering of many scenes: the per-scene tables the batched
// kernels read and their launchers (pm_trace.cu, pm_render.cu,
// pm_photonmap.cu, pm_batch_maps.cu). Each batched kernel covers every scene of the batch in
// one launch; a thread or warp finds its scene by binary search in a prefix
// array (pixels, emitted photons, query work items) held in shared memory.
#pragma once

#include "pm_photonmap.cuh"
#include "pm_render.cuh"
#include "pm_trace.cuh"

namespace pm {

constexpr int kMaxBatchScenes = 256;

// One scene of a batch as the batched kernels see it (device memory).
struct BatchScene {
  SceneDev sc;
  RenderArgs ra;       // camera pass; pointers into the batch's buffers
  MapDev map;          // its photon map
  int k;               // nEstimationGlobal
  float n_emitted;     // photons emitted for the map
  float3 qlo, qinv;    // box of the query Morton codes (vertex bounds)
  TraceArgs ta;         // photon trace into this scene's append region
  // resolve
  float* res;          // the estimates of this scene's slots
  float4* accum;
  float* image;        // height x width x 3
};

// s with off[s] <= i < off[s + 1], for 0 <= i < off[n] (off non-decreasing
// from off[0] = 0; empty ranges are skipped).
__device__ __forceinline__ int batch_find(const int64_t* off, int n, int64_t i) {
  int lo = 0, hi = n;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (off[mid] <= i) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Copies off[0 .. n] into shared memory (call from every thread of the
// block, followed by __syncthreads).
__device__ __forceinline__ void batch_load_offsets(int64_t* dst, const int64_t* off, int n) {
  for (int i = threadIdx.x; i <= n; i += blockDim.x) dst[i] = off[i];
}

struct BatchTables {
  const BatchScene* scenes;  // n_scenes records
  const int64_t* emit_off;   // n_scenes + 1 prefix of emitted photons
  const int64_t* pix_off;    // n_scenes + 1 prefix of pixels
  const int64_t* slot_off;   // n_scenes + 1 prefix of query slots
  const float4* slots;       // the query slots of all scenes (4 float4 each)
  int n_scenes;
  unsigned* status;             // trace NaN / negative stops (2 words)
  unsigned long long* next_photon;  // work counter of the batched trace
  unsigned long long* dropped;  // NaN / negative samples (2 words)
};

// Photon emission and tracing of every scene (pm_trace.cu).
void batch_trace_launch(const BatchTables& t, int64_t total_emit, int block, int stack,
                        cudaStream_t st);

// The photon maps of every scene of a batch (pm_batch_maps.cu). The trace
// wrote scene s's stored photons and their keys (photon << 8 | ordinal) to
// records [stored_off[s], stored_off[s + 1]) of raw / keys_a, and the store
// count of the photon with work index emit_off[s] + p to count. order
// receives, for each scene's index-order places (at the same offsets), the
// trace record there; the map goes to pos4 / thr4 / wi2 at the same
// offsets and the boxes from box 2 * box_base[s] on. All device arrays.
struct BatchMapBuild {
  const float* raw;                 // total records of 9 floats
  unsigned long long* keys_a;       // total: the trace's keys, then sort scratch
  unsigned long long* keys_b;       // total: map keys
  uint32_t* va;                     // total each: sort values
  uint32_t* vb;
  uint32_t* hist;                   // sort_hist_words(total)
  const uint32_t* count;            // total_emit
  uint32_t* first;                  // total_emit: first index of each photon's stores
  uint32_t* sums;                   // scan_tiles(total_emit)
  uint32_t* order;                  // total
  uint32_t* bb;                     // 6 n: the scenes' position boxes
  int* err;                         // device error word
  const int64_t* stored_off;        // n + 1
  const int64_t* emit_off;          // n + 1
  const int64_t* group_off;         // n + 1: prefix of the 8-photon groups
  const int64_t* box_base;          // n
  const int64_t* level_off;         // kMaxLevels rows of n + 1: prefix of level-l boxes
  const int* lvl;                   // n x (kMaxLevels level offsets, kMaxLevels counts)
  float4* pos4;
  float4* thr4;
  float2* wi2;
  float4* boxes;
  int64_t total;                    // stored photons of all scenes (< 2^31)
  int64_t total_emit;
  int64_t total_groups;
  int64_t level_total[kMaxLevels];  // boxes of level l over all scenes
  int n_scenes;
  int scene_bits;   // bits of a scene number
  int max_levels;   // most tree levels of any scene
  int num_sms;      // streaming multiprocessors of the device (grid sizes)
};

void batch_maps_launch(const BatchMapBuild& a, cudaStream_t st);

// out[j] = raw record order[j], j < m (9 floats each).
void batch_photons_launch(const float* raw, const uint32_t* order, int64_t m, float* out,
                          cudaStream_t st);

// Camera pass of every pixel of every scene (pm_render.cu): sampler seeds,
// then the camera kernel.
void batch_camera_launch(const BatchTables& t, int64_t total_pix, int block, int stack,
                         cudaStream_t st);

// Lists the slots holding a query with key (scene << 30 | Morton code of
// the position in the scene's box); count = queries listed.
void batch_list_queries_launch(const BatchTables& t, int64_t total_slots,
                               unsigned long long* keys, uint32_t* vals, unsigned* count,
                               cudaStream_t st);

// From the sorted keys of nq queries: qoff[s] = first query of scene s
// (qoff[n_scenes] = min(nq, *listed), the queries actually listed) and
// item_off = prefix of ceil(queries / chunk). qstart: n_scenes words of
// scratch.
void batch_query_ranges_launch(const unsigned long long* sorted_keys, int64_t nq,
                               const unsigned* listed, int n_scenes, int chunk, int64_t* qstart,
                               int64_t* qoff, int64_t* item_off, cudaStream_t st);

// The radiance estimate of every query of every scene in one persistent
// launch (pm_photonmap.cu): warps take work items of `chunk` consecutive
// queries (one scene each) from `counter`. warps: per block (1..8);
// buffer: candidate entries per warp (512, which needs k <= 224, or 2048).
// batch_knn_prepare sets the kernel's shared-memory limit and gives its
// resident blocks per SM; call it before capturing a launch in a graph.
cudaError_t batch_knn_prepare(int warps, int buffer, int* blocks_per_sm);
cudaError_t batch_knn_launch(const BatchTables& t, const float4* slots, const uint32_t* order,
                             const int64_t* qoff, const int64_t* item_off, int64_t max_items,
                             float* res, int warps, int chunk, int buffer, int blocks_per_sm,
                             unsigned long long* counter, int num_sms, cudaStream_t st);

// Per pixel of every scene: the samples' radiance summed (NaN and negative
// samples dropped), divided by spp into the scene's image (pm_render.cu).
void batch_resolve_launch(const BatchTables& t, int64_t total_pix, cudaStream_t st);

}  // namespace pm
