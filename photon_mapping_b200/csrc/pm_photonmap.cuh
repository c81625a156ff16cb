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
//   grid   uint32[]    cell tables over the same order: 8 header words (the
//                      box of the photon positions, order-preserving bits,
//                      as the Morton codes were made), then for each level L
//                      in [kGridMinLevel, grid_lmax] the first sorted photon
//                      of every level-L cell (8^L cells, the cell code being
//                      the Morton key's top 3L bits) and a final word n, so
//                      cell c holds photons [tab[c], tab[c+1]).
#pragma once

#include "pm_common.cuh"

namespace pm {

constexpr int kMaxLevels = 8;
constexpr int kGroup = 8;  // photons per bottom-level box

// Cell grids: levels kGridMinLevel..grid_lmax (at most kGridMaxLevel; a
// level-L cell is 1/2^L of the photons' box along each axis).
constexpr int kGridMinLevel = 3;
constexpr int kGridMaxLevel = 7;
constexpr int kGridLevels = kGridMaxLevel - kGridMinLevel + 1;
constexpr int kGridHeader = 8;

struct MapDev {
  const float4* __restrict__ pos4;
  const float4* __restrict__ thr4;
  const float2* __restrict__ wi2;
  const float4* __restrict__ boxes;
  int n;
  int nlevels;
  int lvl_off[kMaxLevels];
  int lvl_cnt[kMaxLevels];
  const uint32_t* __restrict__ grid;  // null: no cell grid
  int grid_lmax;                      // finest level with a table
  int grid_off[kGridLevels];          // word offset of level kGridMinLevel + i
};

// Tree shape for n photons (host side). Returns the total number of boxes.
int map_levels(int64_t n, int* nlevels, int* lvl_off, int* lvl_cnt);

// Cell-grid shape for n photons (host side): finest level *lmax (0: no
// grid) and the word offset of every level's table. Returns the words of
// the grid buffer (0 without a grid).
size_t grid_words(int64_t n, int* lmax, int* off);

// Bytes of scratch the build needs for n photons.
size_t map_build_scratch_bytes(int64_t n);

// Builds pos4/thr4/wi2/boxes from `aos` (device, 9 floats per photon), and
// the cell grid into `grid` when grid_lmax > 0 (offsets from grid_words).
void map_build_launch(const float* aos, int n, float4* pos4, float4* thr4,
                      float2* wi2, float4* boxes, const int* lvl_off,
                      const int* lvl_cnt, int nlevels, void* scratch,
                      cudaStream_t st, uint32_t* grid = nullptr, int grid_lmax = 0,
                      const int* grid_off = nullptr);

enum KnnMode { kModeRadiance = 0, kModeKnn = 1, kModeAdjoint = 2 };

struct KnnOut {
  float* rgb;          // radiance mode: 3 floats per record
  int32_t* idx;        // knn mode: k per query
  int32_t* count;      // knn mode
  float* maxd2;        // knn mode
  unsigned long long* stats;  // the pm_knn_stats counters or null
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
// `counter` is one device word of scratch (reset by this call). `grid`
// lets the searches list their candidates from the map's cell grid (when
// it has one) instead of walking the box tree; the results are the same
// either way.
cudaError_t knn_launch(const MapDev& m, const void* queries, int64_t nq,
                       int k, int mode, float n_emitted, KnnOut out,
                       unsigned long long* counter, int num_sms,
                       cudaStream_t st, const uint32_t* order = nullptr,
                       int stride4 = 3, bool grid = true);

}  // namespace pm
