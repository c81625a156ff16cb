// Stable LSD radix sort of (key, uint32 value) pairs, 8-bit digits.
//
// Per digit pass: rs_hist counts digits per tile, rs_scan_rows scans the
// digit-major table of tile counts row by row (one block per digit),
// rs_scatter ranks the tile's pairs by digit in shared memory, equal digits
// in input order so the sort is stable (deterministic photon indices and
// Morton order ties), and writes each digit's run of the tile to its place
// in one contiguous stretch.
#pragma once

#include "pm_common.cuh"

namespace pm {

constexpr int kSortThreads = 256;

// Pairs per tile: the tile's keys and values fit the block's shared memory
// (36 KB for 64-bit keys, 43 KB for 32-bit keys).
template <typename K>
__host__ __device__ constexpr int sort_tile() {
  return sizeof(K) == 8 ? 2048 : 4096;
}

template <typename K>
__host__ __device__ constexpr int sort_tiles(int64_t n) {
  return (int)((n + sort_tile<K>() - 1) / sort_tile<K>());
}

// Words of the count table for either key type: 256 digits x tiles, then
// the 256 digit totals.
constexpr size_t sort_hist_words(int64_t n) {
  return 256 * (size_t)sort_tiles<unsigned long long>(n) + 256;
}

// Exclusive scan of one value per thread of a kSortThreads block (ws:
// kSortThreads / 32 words of shared memory; ends synchronised).
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* ws,
                                                         uint32_t* total = nullptr) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(kFull, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) ws[warp] = x;
  __syncthreads();
  uint32_t before = 0, all = 0;
#pragma unroll
  for (int w = 0; w < kSortThreads / 32; ++w) {
    before += w < warp ? ws[w] : 0u;
    all += ws[w];
  }
  __syncthreads();
  if (total) *total = all;
  return before + x - v;
}

template <typename K>
__global__ void __launch_bounds__(kSortThreads)
    rs_hist(const K* __restrict__ kin, int n, int shift,
            uint32_t* __restrict__ hist, int ntiles) {
  __shared__ uint32_t h[256];
  const int tid = threadIdx.x;
  h[tid] = 0;
  __syncthreads();
  const int t0 = blockIdx.x * sort_tile<K>();
#pragma unroll 4
  for (int r = 0; r < sort_tile<K>() / kSortThreads; ++r) {
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
  constexpr int kTile = sort_tile<K>();
  constexpr int kWarps = kSortThreads / 32;
  __shared__ K sk[kTile];
  __shared__ uint32_t sv[kTile];
  __shared__ uint32_t wcnt[kWarps][256];
  __shared__ uint32_t tstart[256];  // first slot of digit d in the tile
  __shared__ uint32_t gbase[256];   // output place of that slot
  __shared__ uint32_t run[256];     // pairs of digit d placed so far
  __shared__ uint32_t ws[kWarps];
  const int tid = threadIdx.x, warp = tid >> 5;
  const int tile = blockIdx.x;
  const int t0 = tile * kTile;
  const int cnt = n - t0 < kTile ? n - t0 : kTile;
  {
    // digit offset = exclusive scan of the digit totals, plus this tile's
    // exclusive prefix over the tiles; the tile's own count of digit tid is
    // the step to the next tile's prefix
    const uint32_t doff = block_exclusive_scan(totals[tid], ws);
    const uint32_t pre = offs[tid * ntiles + tile];
    const uint32_t next = tile + 1 < ntiles ? offs[tid * ntiles + tile + 1] : totals[tid];
    const uint32_t mine = next - pre;
    gbase[tid] = doff + pre;
    tstart[tid] = block_exclusive_scan(mine, ws);
    run[tid] = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) wcnt[w][tid] = 0;
    __syncthreads();
  }
  // rank: round r holds pairs t0 + r * kSortThreads + tid; equal digits
  // keep input order (earlier rounds, then earlier warps, then lanes)
  for (int r = 0; r < kTile / kSortThreads; ++r) {
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
    const unsigned rank = __popc(peers & lt_mask(tid & 31));
    if (ok && rank == 0) wcnt[warp][d] = __popc(peers);
    __syncthreads();
    if (ok) {
      uint32_t pos = tstart[d] + run[d] + rank;
      for (int w = 0; w < warp; ++w) pos += wcnt[w][d];
      sk[pos] = key;
      sv[pos] = val;
    }
    __syncthreads();
    uint32_t tot = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
      tot += wcnt[w][tid];
      wcnt[w][tid] = 0;
    }
    run[tid] += tot;
    __syncthreads();
  }
  // write: consecutive slots of one digit go to consecutive places
  for (int q = tid; q < cnt; q += kSortThreads) {
    const K key = sk[q];
    const uint32_t d = (uint32_t)(key >> shift) & 255u;
    const uint32_t o = gbase[d] + (uint32_t)q - tstart[d];
    kout[o] = key;
    vout[o] = sv[q];
  }
}

// ------------------------------------------------- exclusive scan (uint32)
//
// out[i] = in[0] + ... + in[i - 1] for n values whose total fits in 32
// bits: tile sums, one block scanning the tile sums, then each tile scanned
// from its base (a thread holds kScanPer consecutive values).

constexpr int kScanPer = 16;
constexpr int kScanTile = kSortThreads * kScanPer;

constexpr int64_t scan_tiles(int64_t n) { return (n + kScanTile - 1) / kScanTile; }

static __global__ void __launch_bounds__(kSortThreads)
    scan_tile_sums(const uint32_t* __restrict__ in, int64_t n, uint32_t* __restrict__ sums) {
  __shared__ uint32_t ws[kSortThreads / 32];
  const int64_t t0 = (int64_t)blockIdx.x * kScanTile;
  uint32_t v = 0;
  for (int r = 0; r < kScanPer; ++r) {
    const int64_t i = t0 + (int64_t)r * kSortThreads + threadIdx.x;
    if (i < n) v += in[i];
  }
  v = __reduce_add_sync(kFull, v);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int w = 0; w < kSortThreads / 32; ++w) t += ws[w];
    sums[blockIdx.x] = t;
  }
}

// One block: exclusive scan of the m tile sums, in place.
static __global__ void __launch_bounds__(1024) scan_sums(uint32_t* __restrict__ sums, int64_t m) {
  __shared__ uint32_t ws[32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  uint32_t carry = 0;
  for (int64_t c0 = 0; c0 < m; c0 += 1024) {
    const int64_t i = c0 + tid;
    const uint32_t v = i < m ? sums[i] : 0u;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(kFull, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) ws[warp] = x;
    __syncthreads();
    uint32_t before = 0, total = 0;
    for (int w = 0; w < 32; ++w) {
      before += w < warp ? ws[w] : 0u;
      total += ws[w];
    }
    if (i < m) sums[i] = carry + before + x - v;
    carry += total;
    __syncthreads();
  }
}

static __global__ void __launch_bounds__(kSortThreads)
    scan_tiles_kernel(const uint32_t* __restrict__ in, int64_t n,
                      const uint32_t* __restrict__ base, uint32_t* __restrict__ out) {
  __shared__ uint32_t ws[kSortThreads / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t i0 = (int64_t)blockIdx.x * kScanTile + (int64_t)tid * kScanPer;
  uint32_t v[kScanPer];
  uint32_t sum = 0;
#pragma unroll
  for (int r = 0; r < kScanPer; ++r) {
    v[r] = i0 + r < n ? in[i0 + r] : 0u;
    sum += v[r];
  }
  uint32_t x = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(kFull, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) ws[warp] = x;
  __syncthreads();
  uint32_t run = base[blockIdx.x] + x - sum;
#pragma unroll
  for (int w = 0; w < kSortThreads / 32; ++w) run += w < warp ? ws[w] : 0u;
#pragma unroll
  for (int r = 0; r < kScanPer; ++r) {
    if (i0 + r < n) out[i0 + r] = run;
    run += v[r];
  }
}

// `sums` needs scan_tiles(n) words. in and out may not alias.
inline void exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t n, uint32_t* sums,
                               cudaStream_t st) {
  if (n <= 0) return;
  const unsigned nt = (unsigned)scan_tiles(n);
  scan_tile_sums<<<nt, kSortThreads, 0, st>>>(in, n, sums);
  scan_sums<<<1, 1024, 0, st>>>(sums, nt);
  scan_tiles_kernel<<<nt, kSortThreads, 0, st>>>(in, n, sums, out);
}

// Sorts n pairs on bits [0, key_bits) of the keys. Buffers a (input) and b
// are ping-ponged; the return value says where the sorted pairs are
// (false: ka/va, true: kb/vb). `hist` needs sort_hist_words(n) words.
template <typename K>
bool radix_sort_pairs(K* ka, uint32_t* va, K* kb, uint32_t* vb, int n,
                      int key_bits, uint32_t* hist, cudaStream_t st) {
  if (n <= 1) return false;
  const int nt = sort_tiles<K>(n);
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
