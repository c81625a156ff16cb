// Stable LSD radix sort of (key, uint32 value) pairs, 8-bit digits.
//
// Per digit pass: rs_hist counts digits per tile, rs_scan turns the
// digit-major table of tile counts into scatter offsets, rs_scatter moves
// every pair to its place, ranking equal digits in input order so the sort
// is stable (needed for deterministic photon indices and Morton order ties).
#pragma once

#include "pm_common.cuh"

namespace pm {

constexpr int kSortThreads = 256;
constexpr int kSortTile = 4096;  // pairs per tile (16 rounds of 256)

inline int sort_tiles(int64_t n) {
  return (int)((n + kSortTile - 1) / kSortTile);
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

// Exclusive scan of m counts in place, one block of 1024 threads.
static __global__ void __launch_bounds__(1024) rs_scan(uint32_t* a, int m) {
  __shared__ uint32_t sums[1024];
  const int tid = threadIdx.x;
  const int per = (m + 1023) / 1024;
  const int s = tid * per;
  const int e = min(m, s + per);
  uint32_t acc = 0;
  for (int i = s; i < e; ++i) acc += a[i];
  sums[tid] = acc;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    const uint32_t v = tid >= off ? sums[tid - off] : 0u;
    __syncthreads();
    sums[tid] += v;
    __syncthreads();
  }
  uint32_t run = sums[tid] - acc;
  for (int i = s; i < e; ++i) {
    const uint32_t v = a[i];
    a[i] = run;
    run += v;
  }
}

template <typename K>
__global__ void __launch_bounds__(kSortThreads)
    rs_scatter(const K* __restrict__ kin, const uint32_t* __restrict__ vin,
               K* __restrict__ kout, uint32_t* __restrict__ vout, int n,
               int shift, const uint32_t* __restrict__ offs, int ntiles) {
  constexpr int kWarps = kSortThreads / 32;
  __shared__ uint32_t base[256];
  __shared__ uint32_t wcnt[kWarps][256];
  const int tid = threadIdx.x, warp = tid >> 5;
  base[tid] = offs[tid * ntiles + blockIdx.x];
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
// (false: ka/va, true: kb/vb). `hist` needs 256 * sort_tiles(n) words.
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
    rs_scan<<<1, 1024, 0, st>>>(hist, 256 * nt);
    rs_scatter<K><<<nt, kSortThreads, 0, st>>>(kin, vin, kout, vout, n, shift,
                                               hist, nt);
    in_b = !in_b;
  }
  return in_b;
}

}  // namespace pm
