// Stable LSD radix sort of (key, uint32 value) pairs, 8-bit digits.
//
// Per digit pass: rs_hist counts digits per tile, rs_scan_rows scans the
// digit-major table of tile counts row by row (one block per digit),
// rs_scatter adds the digit offsets and moves every pair to its place,
// ranking equal digits in input order so the sort is stable (needed for
// deterministic photon indices and Morton order ties).
#pragma once

#include "pm_common.cuh"

namespace pm {

constexpr int kSortThreads = 256;
constexpr int kSortTile = 4096;  // pairs per tile (16 rounds of 256)

constexpr int sort_tiles(int64_t n) {
  return (int)((n + kSortTile - 1) / kSortTile);
}

// Words of the count table: 256 digits x tiles, then the 256 digit totals.
constexpr size_t sort_hist_words(int64_t n) {
  return 256 * (size_t)sort_tiles(n) + 256;
}

template <typename K>
__global__ void __launch_bounds__(kSortThreads)
    rs_hist(const K* __restrict__ kin, int n, int shift,
            uint32_t* __restrict__ hist, int ntiles) {
  __shared__ uint32_t h[256];
  const int tid = threadIdx.x;
  h[tid] = 0;
  __syncthreads();
  const int t0 = blockIdx.x * kSortTile;
#pragma unroll 4
  for (int r = 0; r < kSortTile / kSortThreads; ++r) {
    const int i = t0 + r * kSortThreads + tid;
    if (i < n) atomicAdd(&h[(uint32_t)(kin[i] >> shift) & 255u], 1u);
  }
  __syncthreads();
  hist[tid * ntiles + blockIdx.x] = h[tid];
}

// Block d: exclusive scan, in place, of row d of the digit-major table of
// tile counts (coalesced, 256 tiles per round), and the row's total into
// totals[d]. The digit offsets (the scan of the 256 totals) are added by
// rs_scatter.
static __global__ void __launch_bounds__(kSortThreads)
    rs_scan_rows(uint32_t* __restrict__ hist, int ntiles, uint32_t* __restrict__ totals) {
  __shared__ uint32_t wsum[kSortThreads / 32];
  uint32_t* row = hist + (size_t)blockIdx.x * ntiles;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  uint32_t carry = 0;
  for (int c0 = 0; c0 < ntiles; c0 += kSortThreads) {
    const int i = c0 + tid;
    const uint32_t v = i < ntiles ? row[i] : 0u;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(kFull, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    uint32_t before = 0, total = 0;
#pragma unroll
    for (int w = 0; w < kSortThreads / 32; ++w) {
      const uint32_t ws = wsum[w];
      before += w < warp ? ws : 0u;
      total += ws;
    }
    if (i < ntiles) row[i] = carry + before + x - v;
    carry += total;
    __syncthreads();
  }
  if (tid == 0) totals[blockIdx.x] = carry;
}

template <typename K>
__global__ void __launch_bounds__(kSortThreads)
    rs_scatter(const K* __restrict__ kin, const uint32_t* __restrict__ vin,
               K* __restrict__ kout, uint32_t* __restrict__ vout, int n,
               int shift, const uint32_t* __restrict__ offs, int ntiles,
               const uint32_t* __restrict__ totals) {
  constexpr int kWarps = kSortThreads / 32;
  __shared__ uint32_t base[256];
  __shared__ uint32_t wcnt[kWarps][256];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // digit offset = exclusive scan of the 256 digit totals
  {
    const uint32_t v = totals[tid];
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(kFull, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wcnt[0][warp] = x;
    __syncthreads();
    uint32_t before = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) before += w < warp ? wcnt[0][w] : 0u;
    base[tid] = before + x - v + offs[tid * ntiles + blockIdx.x];
    __syncthreads();
  }
#pragma unroll
  for (int w = 0; w < kWarps; ++w) wcnt[w][tid] = 0;
  __syncthreads();
  const int t0 = blockIdx.x * kSortTile;
  for (int r = 0; r < kSortTile / kSortThreads; ++r) {
    const int i = t0 + r * kSortThreads + tid;
    const bool ok = i < n;
    K key = 0;
    uint32_t val = 0;
    if (ok) {
      key = kin[i];
      val = vin[i];
    }
    const uint32_t d = ok ? ((uint32_t)(key >> shift) & 255u) : 0xffffffffu;
    const unsigned peers = __match_any_sync(kFull, d);
    const unsigned rank = __popc(peers & lanemask_lt());
    if (ok && rank == 0) wcnt[warp][d] = __popc(peers);
    __syncthreads();
    if (ok) {
      uint32_t off = base[d] + rank;
      for (int w = 0; w < warp; ++w) off += wcnt[w][d];
      kout[off] = key;
      vout[off] = val;
    }
    __syncthreads();
    uint32_t tot = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
      tot += wcnt[w][tid];
      wcnt[w][tid] = 0;
    }
    base[tid] += tot;
    __syncthreads();
  }
}

// Sorts n pairs on bits [0, key_bits) of the keys. Buffers a (input) and b
// are ping-ponged; the return value says where the sorted pairs are
// (false: ka/va, true: kb/vb). `hist` needs sort_hist_words(n) words.
template <typename K>
bool radix_sort_pairs(K* ka, uint32_t* va, K* kb, uint32_t* vb, int n,
                      int key_bits, uint32_t* hist, cudaStream_t st) {
  if (n <= 1) return false;
  const int nt = sort_tiles(n);
  bool in_b = false;
  for (int shift = 0; shift < key_bits; shift += 8) {
    const K* kin = in_b ? kb : ka;
    const uint32_t* vin = in_b ? vb : va;
    K* kout = in_b ? ka : kb;
    uint32_t* vout = in_b ? va : vb;
    rs_hist<K><<<nt, kSortThreads, 0, st>>>(kin, n, shift, hist, nt);
    rs_scan_rows<<<256, kSortThreads, 0, st>>>(hist, nt, hist + 256 * (size_t)nt);
    rs_scatter<K><<<nt, kSortThreads, 0, st>>>(kin, vin, kout, vout, n, shift,
                                               hist, nt, hist + 256 * (size_t)nt);
    in_b = !in_b;
  }
  return in_b;
}

}  // namespace pm
