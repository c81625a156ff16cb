// Photon maps of a batch, built for every scene at once. The reference
// rebuilds each scene's map after its trace (PhotonMapping::build,
// integrator.h:470-474 for the global map, :560-562 for the caustics map);
// here one step's maps are one sequence of launches over all scenes:
//   1. one exclusive scan of the store counts of every scene's emitted
//      photons gives each photon's first index, so each stored photon's
//      place in the reference's append order (the index order of its
//      scene's photon vector); one pass takes every scene's box of stored
//      positions;
//   2. one pass writes each photon's map key (scene, 30-bit Morton code)
//      and trace record to its index-order place, and one radix sort,
//      stable from index order, gives every scene's map order;
//   3. one gather writes pos4 / thr4 / wi2 of every scene;
//   4. one launch per tree level builds that level's boxes in every scene.
// Each scene's map is bit-identical to what map_build_launch
// (pm_photonmap.cu) builds from the same photons: the same Morton codes
// from the same box, the same stable order, the same box arithmetic.
#include "pm_batch.cuh"
#include "pm_sort.cuh"

#include <float.h>

#include <algorithm>

namespace pm {

namespace {

constexpr int kSegThreads = 256;
constexpr int kBoxTile = 8192;  // photons per block of the box reduction

// Blocks for n threads, at most `per_sm` blocks per SM (grid-stride loops).
unsigned grid_for(int64_t n, int threads, int num_sms, int per_sm = 16) {
  const int64_t g = (n + threads - 1) / threads;
  return (unsigned)std::min<int64_t>(std::max<int64_t>(g, 1), (int64_t)num_sms * per_sm);
}

// Box of each scene's stored positions, in the ordered-bits form of
// bbox_kernel: bb[3s + a] = min, bb[3n + 3s + a] = max along axis a. Every
// contribution is clamped to +-FLT_MAX first like bbox_kernel's running
// fminf / fmaxf from +-FLT_MAX (NaN contributes the clamp value), so the
// box is the same. A block reduces kBoxTile consecutive trace records (the
// box does not depend on their order); a tile inside one scene ends in 6
// atomics, a tile across scenes uses per-record ones.
__global__ void __launch_bounds__(kSegThreads)
    seg_bbox_kernel(const float* __restrict__ raw, int64_t total,
                    const int64_t* __restrict__ stored_off, int n, uint32_t* __restrict__ bb) {
  __shared__ int64_t off[kMaxBatchScenes + 1];
  __shared__ float part[6][kSegThreads / 32];
  batch_load_offsets(off, stored_off, n);
  __syncthreads();
  const int64_t t0 = (int64_t)blockIdx.x * kBoxTile;
  const int64_t t1 = t0 + kBoxTile < total ? t0 + kBoxTile : total;
  if (t0 >= t1) return;
  const int s0 = batch_find(off, n, t0);
  const int s1 = batch_find(off, n, t1 - 1);
  if (s0 != s1) {  // block-uniform
    for (int64_t i = t0 + threadIdx.x; i < t1; i += blockDim.x) {
      const int s = batch_find(off, n, i);
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const float v = raw[9 * i + 3 + a];
        atomicMin(&bb[3 * s + a], ordered_bits(fminf(FLT_MAX, v)));
        atomicMax(&bb[3 * n + 3 * s + a], ordered_bits(fmaxf(-FLT_MAX, v)));
      }
    }
    return;
  }
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
  float hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  for (int64_t i = t0 + threadIdx.x; i < t1; i += blockDim.x) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float v = raw[9 * i + 3 + a];
      lo[a] = fminf(lo[a], v);
      hi[a] = fmaxf(hi[a], v);
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo[a] = fminf(lo[a], __shfl_xor_sync(kFull, lo[a], o));
      hi[a] = fmaxf(hi[a], __shfl_xor_sync(kFull, hi[a], o));
    }
    if (lane == 0) {
      part[a][warp] = lo[a];
      part[3 + a][warp] = hi[a];
    }
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    const int c = threadIdx.x;
    float v = part[c][0];
    for (int w = 1; w < kSegThreads / 32; ++w)
      v = c < 3 ? fminf(v, part[c][w]) : fmaxf(v, part[c][w]);
    if (c < 3) atomicMin(&bb[3 * s0 + c], ordered_bits(v));
    else atomicMax(&bb[3 * n + 3 * s0 + (c - 3)], ordered_bits(v));
  }
}

// Trace record r of scene s, key p << 8 | j, has index-order place
// d = first[emit_off[s] + p] + j, which must lie in the scene's range (bit
// 5 of *err otherwise). Writes its map key (scene << 30 | Morton code of
// the position in the scene's box, morton_kernel per scene) to mkeys[d]
// and r to order[d]; vals[r] = r (index-order places, the sort's values).
__global__ void __launch_bounds__(kSegThreads)
    seg_place_kernel(const unsigned long long* __restrict__ keys, const float* __restrict__ raw,
                     int64_t total, const int64_t* __restrict__ stored_off,
                     const int64_t* __restrict__ emit_off, int n,
                     const uint32_t* __restrict__ first, const uint32_t* __restrict__ bb,
                     unsigned long long* __restrict__ mkeys, uint32_t* __restrict__ order,
                     uint32_t* __restrict__ vals, int* __restrict__ err) {
  __shared__ int64_t off[kMaxBatchScenes + 1];
  __shared__ int64_t eoff[kMaxBatchScenes + 1];
  batch_load_offsets(off, stored_off, n);
  batch_load_offsets(eoff, emit_off, n);
  __syncthreads();
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < total;
       r += (int64_t)gridDim.x * blockDim.x) {
    const int s = batch_find(off, n, r);
    const unsigned long long key = keys[r];
    const int64_t d = (int64_t)first[eoff[s] + (int64_t)(key >> 8)] + (int64_t)(key & 255u);
    vals[r] = (uint32_t)r;
    if (d < off[s] || d >= off[s + 1]) {
      atomicOr(err, 32);
      continue;
    }
    const float* p = raw + 9 * r + 3;
    uint32_t c[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float lo = from_ordered(bb[3 * s + a]);
      const float ext = from_ordered(bb[3 * n + 3 * s + a]) - lo;
      c[a] = cell10(p[a], lo, ext);
    }
    const uint32_t m = (spread10(c[0]) << 2) | (spread10(c[1]) << 1) | spread10(c[2]);
    mkeys[d] = ((unsigned long long)s << 30) | m;
    order[d] = (uint32_t)r;
  }
}

// Map position j of the batch: perm[j] = index-order place c, whose trace
// record is order[c]; its index within the scene goes into pos4.w
// (gather_kernel per scene).
__global__ void __launch_bounds__(kSegThreads)
    seg_gather_kernel(const float* __restrict__ raw, const uint32_t* __restrict__ order,
                      const uint32_t* __restrict__ perm, int64_t total,
                      const int64_t* __restrict__ stored_off, int n, float4* __restrict__ pos4,
                      float4* __restrict__ thr4, float2* __restrict__ wi2) {
  __shared__ int64_t off[kMaxBatchScenes + 1];
  batch_load_offsets(off, stored_off, n);
  __syncthreads();
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < total;
       j += (int64_t)gridDim.x * blockDim.x) {
    const int s = batch_find(off, n, j);
    const uint32_t c = perm[j];
    const uint32_t i = (uint32_t)(c - off[s]);
    const float* r = raw + 9 * (size_t)order[c];
    pos4[j] = make_float4(r[3], r[4], r[5], __uint_as_float(i));
    thr4[j] = make_float4(r[0], r[1], r[2], r[6]);
    wi2[j] = make_float2(r[7], r[8]);
  }
}

// Level-0 boxes (8-photon groups) of every scene: 8 lanes per group
// (group_box_kernel per scene). Groups never straddle scenes.
__global__ void __launch_bounds__(kSegThreads)
    seg_group_box_kernel(const float4* __restrict__ pos4, const int64_t* __restrict__ stored_off,
                         const int64_t* __restrict__ group_off,
                         const int64_t* __restrict__ box_base, int n, int64_t total_groups,
                         float4* __restrict__ boxes) {
  __shared__ int64_t goff[kMaxBatchScenes + 1];
  batch_load_offsets(goff, group_off, n);
  __syncthreads();
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t g = t >> 3;
  const bool has = g < total_groups;
  int s = 0;
  int64_t lg = 0;
  float4 lo = make_float4(FLT_MAX, FLT_MAX, FLT_MAX, 0.f);
  float4 hi = make_float4(-FLT_MAX, -FLT_MAX, -FLT_MAX, 0.f);
  if (has) {
    s = batch_find(goff, n, g);
    lg = g - goff[s];
    const int64_t li = lg * kGroup + (t & 7);
    if (li < stored_off[s + 1] - stored_off[s]) {
      const float4 p = pos4[stored_off[s] + li];
      lo.x = fminf(lo.x, p.x); lo.y = fminf(lo.y, p.y); lo.z = fminf(lo.z, p.z);
      hi.x = fmaxf(hi.x, p.x); hi.y = fmaxf(hi.y, p.y); hi.z = fmaxf(hi.z, p.z);
    }
  }
#pragma unroll
  for (int o = 4; o > 0; o >>= 1) {
    lo.x = fminf(lo.x, __shfl_xor_sync(kFull, lo.x, o));
    lo.y = fminf(lo.y, __shfl_xor_sync(kFull, lo.y, o));
    lo.z = fminf(lo.z, __shfl_xor_sync(kFull, lo.z, o));
    hi.x = fmaxf(hi.x, __shfl_xor_sync(kFull, hi.x, o));
    hi.y = fmaxf(hi.y, __shfl_xor_sync(kFull, hi.y, o));
    hi.z = fmaxf(hi.z, __shfl_xor_sync(kFull, hi.z, o));
  }
  if (has && (t & 7) == 0) {
    float4* bx = boxes + 2 * box_base[s];
    bx[2 * lg] = lo;
    bx[2 * lg + 1] = hi;
  }
}

// Level-l boxes of every scene, one warp per box over its 32 children
// (node_box_kernel per scene). row: prefix over scenes of the level-l box
// counts; lvl: per scene, kMaxLevels level offsets then kMaxLevels counts.
__global__ void __launch_bounds__(kSegThreads)
    seg_node_box_kernel(float4* __restrict__ boxes, const int64_t* __restrict__ row,
                        const int64_t* __restrict__ box_base, const int* __restrict__ lvl,
                        int n, int l, int64_t total_nodes) {
  __shared__ int64_t off[kMaxBatchScenes + 1];
  batch_load_offsets(off, row, n);
  __syncthreads();
  const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= total_nodes) return;  // whole warps
  const int s = batch_find(off, n, w);
  const int node = (int)(w - off[s]);
  const int* lv = lvl + 2 * kMaxLevels * s;
  const int child_off = lv[l - 1], child_cnt = lv[kMaxLevels + l - 1], node_off = lv[l];
  float4* bx = boxes + 2 * box_base[s];
  const int c = node * 32 + lane;
  float4 lo = make_float4(FLT_MAX, FLT_MAX, FLT_MAX, 0.f);
  float4 hi = make_float4(-FLT_MAX, -FLT_MAX, -FLT_MAX, 0.f);
  if (c < child_cnt) {
    const float4 a = bx[2 * (child_off + c)];
    const float4 b = bx[2 * (child_off + c) + 1];
    lo.x = a.x; lo.y = a.y; lo.z = a.z;
    hi.x = b.x; hi.y = b.y; hi.z = b.z;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo.x = fminf(lo.x, __shfl_xor_sync(kFull, lo.x, o));
    lo.y = fminf(lo.y, __shfl_xor_sync(kFull, lo.y, o));
    lo.z = fminf(lo.z, __shfl_xor_sync(kFull, lo.z, o));
    hi.x = fmaxf(hi.x, __shfl_xor_sync(kFull, hi.x, o));
    hi.y = fmaxf(hi.y, __shfl_xor_sync(kFull, hi.y, o));
    hi.z = fmaxf(hi.z, __shfl_xor_sync(kFull, hi.z, o));
  }
  if (lane == 0) {
    bx[2 * (node_off + node)] = lo;
    bx[2 * (node_off + node) + 1] = hi;
  }
}

// out[j] = trace record order[j] (one scene's photon vector, on demand).
__global__ void __launch_bounds__(kSegThreads)
    seg_photons_kernel(const float* __restrict__ raw, const uint32_t* __restrict__ order,
                       int64_t m, float* __restrict__ out) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < m;
       j += (int64_t)gridDim.x * blockDim.x) {
    const float* r = raw + 9 * (size_t)order[j];
    float* o = out + 9 * j;
#pragma unroll
    for (int q = 0; q < 9; ++q) o[q] = r[q];
  }
}

}  // namespace

void batch_photons_launch(const float* raw, const uint32_t* order, int64_t m, float* out,
                          cudaStream_t st) {
  if (m <= 0) return;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  seg_photons_kernel<<<grid_for(m, kSegThreads, sms), kSegThreads, 0, st>>>(raw, order, m, out);
}

void batch_maps_launch(const BatchMapBuild& a, cudaStream_t st) {
  const int64_t total = a.total;
  if (total <= 0) return;
  const int n = a.n_scenes;
  const int tb = kSegThreads;
  const unsigned gb = grid_for(total, tb, a.num_sms);
  // 1. index-order places and the scenes' boxes
  exclusive_scan_u32(a.count, a.first, a.total_emit, a.sums, st);
  cudaMemsetAsync(a.bb, 0xff, 3 * sizeof(uint32_t) * (size_t)n, st);
  cudaMemsetAsync(a.bb + 3 * n, 0x00, 3 * sizeof(uint32_t) * (size_t)n, st);
  const unsigned tiles = (unsigned)((total + kBoxTile - 1) / kBoxTile);
  seg_bbox_kernel<<<tiles, tb, 0, st>>>(a.raw, total, a.stored_off, n, a.bb);
  // 2. map order
  // a small grid (4 blocks per SM): the records in flight at once span a
  // narrow window of index-order places, so the scattered 12-B writes fill
  // their sectors in L2 before eviction (48.2 -> 37.5 ms for the maps of 211M
  // photons against 16 blocks per SM)
  seg_place_kernel<<<grid_for(total, tb, a.num_sms, 4), tb, 0, st>>>(
      a.keys_a, a.raw, total, a.stored_off, a.emit_off, n, a.first, a.bb, a.keys_b, a.order,
      a.va, a.err);
  // sorted pairs end in (keys_a, vb) or back in (keys_b, va)
  const bool in_second = radix_sort_pairs<unsigned long long>(
      a.keys_b, a.va, a.keys_a, a.vb, (int)total, 30 + a.scene_bits, a.hist, st);
  const uint32_t* perm = in_second ? a.vb : a.va;
  // 3. the map arrays
  seg_gather_kernel<<<gb, tb, 0, st>>>(a.raw, a.order, perm, total, a.stored_off, n, a.pos4,
                                       a.thr4, a.wi2);
  // 4. the box tree, level by level
  if (a.total_groups > 0)
    seg_group_box_kernel<<<(unsigned)((a.total_groups * kGroup + tb - 1) / tb), tb, 0, st>>>(
        a.pos4, a.stored_off, a.group_off, a.box_base, n, a.total_groups, a.boxes);
  for (int l = 1; l < a.max_levels; ++l) {
    const int64_t nodes = a.level_total[l];
    if (nodes <= 0) continue;
    seg_node_box_kernel<<<(unsigned)((nodes * 32 + tb - 1) / tb), tb, 0, st>>>(
        a.boxes, a.level_off + (size_t)l * (n + 1), a.box_base, a.lvl, n, l, nodes);
  }
}

}  // namespace pm
