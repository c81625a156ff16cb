// Device photon map: layout and the launch functions of its kernels.
//
// Layout in HBM (n photons):
//   aos    float[9n]   photons in index order, {throughput, position, wi}
//                      (the Photon record of photon_map.h:10-22), kept for
//                      getIthPhoton and for rebuilding.
//   pos4   float4[n]   sorted by 30-bit Morton code of the position, ties by
//                      index: {x, y, z, index bits}. The kNN scan reads only
//                      this array (16 B per photon, one coalesced 512 B
//                      line per 32-photon leaf).
//   thr4   float4[n]   same order: {throughput.rgb, wi.x}
//   wi2    float2[n]   same order: {wi.y, wi.z}
//   boxes  float4[2m]  32-ary box tree over the sorted array: level 0 has
//                      one box per group of 8 consecutive photons, level
//                      l+1 one box per 32 level-l boxes; node j of all
//                      levels is {lo, hi} at boxes[2j], boxes[2j+1].
#pragma once

#include "pm_common.cuh"

namespace pm {

constexpr int kMaxLevels = 8;
constexpr int kGroup = 8;  // photons per bottom-level box

struct MapDev {
  const float4* __restrict__ pos4;
  const float4* __restrict__ thr4;
  const float2* __restrict__ wi2;
  const float4* __restrict__ boxes;
  int n;
  int nlevels;
  int lvl_off[kMaxLevels];
  int lvl_cnt[kMaxLevels];
};

// Tree shape for n photons (host side). Returns the total number of boxes.
int map_levels(int64_t n, int* nlevels, int* lvl_off, int* lvl_cnt);

// Bytes of scratch the build needs for n photons.
size_t map_build_scratch_bytes(int64_t n);

// Builds pos4/thr4/wi2/boxes from `aos` (device, 9 floats per photon).
void map_build_launch(const float* aos, int n, float4* pos4, float4* thr4,
                      float2* wi2, float4* boxes, const int* lvl_off,
                      const int* lvl_cnt, int nlevels, void* scratch,
                      cudaStream_t st);

enum KnnMode { kModeRadiance = 0, kModeKnn = 1, kModeAdjoint = 2 };

struct KnnOut {
  float* rgb;          // radiance mode: 3 floats per record
  int32_t* idx;        // knn mode: k per query
  int32_t* count;      // knn mode
  float* maxd2;        // knn mode
  unsigned long long* stats;  // 6 counters (pm_knn_stats) or null
  const float* adj_in;  // adjoint mode: d loss / d estimate, 3 floats per record
  float4* photon_adj;   // adjoint mode: d loss / d throughput per photon
                        // (index order, .xyz), accumulated atomically
};

// Launches the warp-per-query k-nearest-neighbour kernel.
//   radiance mode: query i reads the record r = order ? order[i] : i, a
//                  pm_radiance_query at queries + stride4 * r float4s, and
//                  writes rgb[3r .. 3r+3)
//   knn mode:      queries = 3 floats per query (order and stride unused)
//   adjoint mode:  the records of radiance mode; the neighbours of record r
//                  receive adj_in[3r .. 3r+3) times d estimate / d
//                  throughput in photon_adj
// `counter` is one device word of scratch (reset by this call).
cudaError_t knn_launch(const MapDev& m, const void* queries, int64_t nq,
                       int k, int mode, float n_emitted, KnnOut out,
                       unsigned long long* counter, int num_sms,
                       cudaStream_t st, const uint32_t* order = nullptr,
                       int stride4 = 3);

}  // namespace pm
