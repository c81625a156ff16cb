// Photon map on the device: build (Morton order + 32-ary box tree) and the
// warp-per-query k-nearest-neighbour search with the radiance estimate.
//
// Reference behaviour followed here (yumcyaWiz/photon_mapping):
//   photon_map.h:33-41    distance2: float sum of squared differences x,y,z
//   photon_map.h:107-147  kNN search keeping the k smallest (dist2, index)
//                         pairs (std::priority_queue of pair<float,int>,
//                         so among equal distances the smaller index wins)
//   photon_map.h:166-183  result order (heap pops: largest pair first) and
//                         maxDist2 = largest kept dist2
//   integrator.h:133-152  radiance estimate with the Lambert BRDF
//   material.h:80-88      Lambert::evaluate
#include "pm_batch.cuh"
#include "pm_photonmap.cuh"
#include "pm_sort.cuh"

#include <float.h>

namespace pm {

// ------------------------------------------------------------------ build

int map_levels(int64_t n, int* nlevels, int* lvl_off, int* lvl_cnt) {
  if (n <= 0) {
    *nlevels = 0;
    return 0;
  }
  int64_t cnt = (n + kGroup - 1) / kGroup;
  int lv = 0, off = 0;
  while (true) {
    lvl_off[lv] = off;
    lvl_cnt[lv] = (int)cnt;
    off += (int)cnt;
    ++lv;
    if (cnt == 1) break;
    cnt = (cnt + 31) / 32;
  }
  *nlevels = lv;
  return off;
}

size_t map_build_scratch_bytes(int64_t n) {
  const size_t nn = (size_t)(n > 0 ? n : 1);
  // keys a/b, values a/b, tile histogram, bbox words
  return 4 * nn * sizeof(uint32_t) + sort_hist_words(nn) * 4 + 64;
}

__device__ __forceinline__ uint32_t ordered_bits(float f) {
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float from_ordered(uint32_t u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__global__ void bbox_kernel(const float* __restrict__ aos, int n,
                            uint32_t* __restrict__ bb) {
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
  float hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float v = aos[9 * (size_t)i + 3 + a];
      lo[a] = fminf(lo[a], v);  // fminf ignores NaN
      hi[a] = fmaxf(hi[a], v);
    }
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo[a] = fminf(lo[a], __shfl_xor_sync(kFull, lo[a], o));
      hi[a] = fmaxf(hi[a], __shfl_xor_sync(kFull, hi[a], o));
    }
  }
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      atomicMin(&bb[a], ordered_bits(lo[a]));
      atomicMax(&bb[3 + a], ordered_bits(hi[a]));
    }
  }
}

__device__ __forceinline__ uint32_t spread10(uint32_t x) {
  x &= 0x3ffu;
  x = (x | (x << 16)) & 0x030000ffu;
  x = (x | (x << 8)) & 0x0300f00fu;
  x = (x | (x << 4)) & 0x030c30c3u;
  x = (x | (x << 2)) & 0x09249249u;
  return x;
}

__device__ __forceinline__ uint32_t cell10(float v, float lo, float ext) {
  if (!(ext > 0.f)) return 0;
  float t = (v - lo) / ext * 1024.f;
  if (!(t > 0.f)) return 0;  // also NaN
  return t >= 1023.f ? 1023u : (uint32_t)t;
}

__global__ void morton_kernel(const float* __restrict__ aos, int n,
                              const uint32_t* __restrict__ bb,
                              uint32_t* __restrict__ keys,
                              uint32_t* __restrict__ vals) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float lo[3], ext[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    lo[a] = from_ordered(bb[a]);
    ext[a] = from_ordered(bb[3 + a]) - lo[a];
  }
  const float* p = aos + 9 * (size_t)i + 3;
  const uint32_t cx = cell10(p[0], lo[0], ext[0]);
  const uint32_t cy = cell10(p[1], lo[1], ext[1]);
  const uint32_t cz = cell10(p[2], lo[2], ext[2]);
  keys[i] = (spread10(cx) << 2) | (spread10(cy) << 1) | spread10(cz);
  vals[i] = (uint32_t)i;
}

__global__ void gather_kernel(const float* __restrict__ aos, int n,
                              const uint32_t* __restrict__ order,
                              float4* __restrict__ pos4,
                              float4* __restrict__ thr4,
                              float2* __restrict__ wi2) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const uint32_t i = order[s];
  const float* r = aos + 9 * (size_t)i;
  pos4[s] = make_float4(r[3], r[4], r[5], __uint_as_float(i));
  thr4[s] = make_float4(r[0], r[1], r[2], r[6]);
  wi2[s] = make_float2(r[7], r[8]);
}

// Box of each 8-photon group: 8 lanes per group, 4 groups per warp.
__global__ void group_box_kernel(const float4* __restrict__ pos4, int n,
                                 int ngroups, float4* __restrict__ boxes) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int g = t >> 3;
  const int i = g * kGroup + (threadIdx.x & 7);
  float4 lo = make_float4(FLT_MAX, FLT_MAX, FLT_MAX, 0.f);
  float4 hi = make_float4(-FLT_MAX, -FLT_MAX, -FLT_MAX, 0.f);
  if (g < ngroups && i < n) {
    const float4 p = pos4[i];
    lo.x = fminf(lo.x, p.x); lo.y = fminf(lo.y, p.y); lo.z = fminf(lo.z, p.z);
    hi.x = fmaxf(hi.x, p.x); hi.y = fmaxf(hi.y, p.y); hi.z = fmaxf(hi.z, p.z);
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
  if (g < ngroups && (threadIdx.x & 7) == 0) {
    boxes[2 * g] = lo;
    boxes[2 * g + 1] = hi;
  }
}

__global__ void node_box_kernel(float4* __restrict__ boxes, int child_off,
                                int child_cnt, int node_off, int node_cnt) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= node_cnt) return;
  const int c = warp * 32 + lane;
  float4 lo = make_float4(FLT_MAX, FLT_MAX, FLT_MAX, 0.f);
  float4 hi = make_float4(-FLT_MAX, -FLT_MAX, -FLT_MAX, 0.f);
  if (c < child_cnt) {
    const float4 a = boxes[2 * (child_off + c)];
    const float4 b = boxes[2 * (child_off + c) + 1];
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
    boxes[2 * (node_off + warp)] = lo;
    boxes[2 * (node_off + warp) + 1] = hi;
  }
}

void map_build_launch(const float* aos, int n, float4* pos4, float4* thr4,
                      float2* wi2, float4* boxes, const int* lvl_off,
                      const int* lvl_cnt, int nlevels, void* scratch,
                      cudaStream_t st) {
  if (n <= 0) return;
  uint32_t* ka = (uint32_t*)scratch;
  uint32_t* kb = ka + n;
  uint32_t* va = kb + n;
  uint32_t* vb = va + n;
  uint32_t* hist = vb + n;
  uint32_t* bb = hist + sort_hist_words(n);
  cudaMemsetAsync(bb, 0xff, 3 * sizeof(uint32_t), st);
  cudaMemsetAsync(bb + 3, 0x00, 3 * sizeof(uint32_t), st);
  const int tb = 256;
  const int gb = (n + tb - 1) / tb;
  bbox_kernel<<<min(gb, 1184), tb, 0, st>>>(aos, n, bb);
  morton_kernel<<<gb, tb, 0, st>>>(aos, n, bb, ka, va);
  const bool in_b = radix_sort_pairs<uint32_t>(ka, va, kb, vb, n, 30, hist, st);
  gather_kernel<<<gb, tb, 0, st>>>(aos, n, in_b ? vb : va, pos4, thr4, wi2);
  const int ngroups = lvl_cnt[0];
  group_box_kernel<<<(int)(((int64_t)ngroups * kGroup + tb - 1) / tb), tb, 0,
                     st>>>(pos4, n, ngroups, boxes);
  for (int l = 1; l < nlevels; ++l) {
    node_box_kernel<<<(lvl_cnt[l] * 32 + tb - 1) / tb, tb, 0, st>>>(
        boxes, lvl_off[l - 1], lvl_cnt[l - 1], lvl_off[l], lvl_cnt[l]);
  }
}

// -------------------------------------------------------------- kNN query
//
// One warp answers the queries of a work item (16 consecutive queries, 8 at
// the end of a launch; the batched kernel takes `chunk`), 32 at a time in a
// window whose query records sit in the lanes' registers (lane i holds
// query i of the window).
//
// Neighbourhood pools (k <= kPoolMaxK). Queries close to each other share
// most of their neighbours, so one tree walk serves a group of them. A
// group is every pending query of the window within kPoolGroup x r of the
// first pending one (r: the last exact k-th distance the warp found). The
// walk collects every photon within R = kPoolFactor x r + rc of the
// group's centre (rc: the largest distance of a member from it) into a pool
// in shared memory: position and sorted position, at most P photons. A
// member at distance rq from the centre needs no photon outside the pool
// when its k-th distance is at most R - rq (triangle inequality, with
// rounding margins): it computes its distance to every pool photon (one
// register per 32 photons), finds the exact k-th (dist2, index) pair with
// a 256-bin histogram of the distances over [0, (R - rq)^2] and a rank of
// the critical bin, and keeps the pool photons below it. A member that
// fails the test (fewer than k pool photons within R - rq, or a critical
// bin of more than 32 photons), and every member of a group whose pool
// overflowed, is answered by the per-query search afterwards.
//
// Per-query search:
//   1. bound: an upper bound tau of the k-th distance. From the previous
//      query answered this way by the triangle inequality when it is close
//      ((r_prev + delta)^2, inflated for rounding; first tried at the
//      smaller (1.06 r_prev)^2, kept when it holds k photons), else from
//      the photons Morton-adjacent to the group nearest the query.
//   2. collect: depth-first walk of the 32-ary box tree; the passing
//      8-photon groups of a node are scanned packed, 4 groups per round,
//      every photon with dist2 <= tau appended to the warp's buffer. A
//      nearly full buffer is cut to the k best, lowering tau.
//   3. select: exact k-th (dist2, index) pair (histogram, else radix).
// Both ways give the kept photons in the order of the tree's depth-first
// walk: a fixed total order of the photons that no bound changes (a pool
// and a search buffer list the photons they hold in that order, and the
// cuts keep it). The radiance sum over them (Lambert, integrator.h:141-150)
// therefore does not depend on how a query was answered, nor on the order
// queries come in.

constexpr int kStack = 32 * kMaxLevels;

// First radius tried for a query near the previous one: kWarmGuess times
// the previous k-th distance (below the sure bound, the previous k-th
// distance plus the distance between the queries). Any value gives the
// same exact result; this one sets the work (measured on primary-hit
// queries: 123 candidates per query at k = 100 against 181 with the sure
// bound alone).
constexpr float kWarmGuess = 1.06f;
// Work items of the persistent launch: kChunk consecutive queries per
// work-counter bump, then kTail queries per bump for the last
// kTailItems x (resident warps) x kTail queries, so that the warps run out
// of work at nearly the same time.
constexpr int kChunk = 16;
constexpr int kTail = 8;
constexpr int kTailItems = 2;
static_assert(kChunk % 8 == 0 && kTail % 8 == 0, "items start at multiples of 8");
static_assert(kChunk <= 32 && kTail <= kChunk, "an item fits one window");

// Pools: k up to kPoolMaxK (the kept list of a pool query, keys and sorted
// positions, lives in the 256 words of the histogram); group radius and
// pool radius in units of the last k-th distance.
constexpr int kPoolMaxK = 128;
constexpr float kPoolGroup = 0.6f;
constexpr float kPoolFactor = 1.15f;
// Photons held by a pool in the kernels that pool (16 B each, in the space
// of the search buffer), and that search buffer's size.
constexpr int kPoolSize = 512;
constexpr int kPoolBuf = 1024;
static_assert(kPoolSize * 16 <= kPoolBuf * 8, "the pool fits the search buffer");

// Entries of the search buffer kept free for the next append round and the
// cut: a buffer holding more than C - kCutSlack candidates is cut.
constexpr int kCutSlack = 56;

template <int C>
struct WarpBuf {
  uint32_t key[C];  // float bits of dist2 (non-negative: order == uint order);
                    // with id[], also the pool (float4 {position, sorted position})
  uint32_t id[C];   // sorted position of the photon
  uint32_t hist[256];  // selection histogram; the kept list of a pool query
  uint32_t stack[kStack];
  uint32_t list[64];   // passing groups waiting to be scanned, in walk order
  uint32_t sel[32];    // entries of the critical bin of a selection
  uint32_t stat[8];    // per-warp counters, same order as pm_knn_stats
  float stage[3 * kChunk];  // radiance of the current work item (host path)
};

struct Levels {
  int2 oc[kMaxLevels];  // {offset of the level's boxes, boxes in the level}
};

enum {
  kStatQueries = 0, kStatCold, kStatCand, kStatLeaves, kStatNodes, kStatSelects, kStatWalks,
  kStatPoolQueries, kNumStats
};
static_assert(kNumStats <= 8, "stat[] holds the counters");

// Counters are compiled in only for the kernels launched with statistics.
template <bool S, int C>
__device__ __forceinline__ void stat_add(WarpBuf<C>& s, int lane, int which,
                                         uint32_t v) {
  if (S && lane == 0) s.stat[which] += v;
}

__device__ __forceinline__ uint32_t orig_index(const float4* pos4, uint32_t s) {
  return __float_as_uint(pos4[s].w);
}

// k-th smallest (1-based) value among the valid entries i in [0, cnt),
// `get(i, v)` giving validity and value. Radix select over 8-bit digits
// (MSB first) with a 256-bin shared histogram; digits common to all values
// are skipped. Returns the value; *rank_eq = rank still needed among the
// entries equal to it (>= 1), *n_eq = how many entries equal it.
// Precondition: 1 <= kk <= number of valid entries.
template <class Get>
__device__ uint32_t warp_select(uint32_t* hist, int cnt, uint32_t kk, Get get,
                                int lane, uint32_t* rank_eq, uint32_t* n_eq) {
  uint32_t vor = 0, vand = 0xffffffffu, nvalid = 0;
  for (int i = lane; i < cnt; i += 32) {
    uint32_t v;
    if (get(i, v)) {
      vor |= v;
      vand &= v;
      ++nvalid;
    }
  }
  vor = __reduce_or_sync(kFull, vor);
  vand = __reduce_and_sync(kFull, vand);
  const uint32_t diff = vor ^ vand;
  if (diff == 0) {
    *rank_eq = kk;
    *n_eq = __reduce_add_sync(kFull, nvalid);
    return vand;
  }
  const int top = 31 - __clz(diff);
  int shift = (top / 8) * 8;
  const uint64_t above = ~((1ull << (shift + 8)) - 1ull);
  uint32_t pmask = (uint32_t)above;
  uint32_t prefix = vand & pmask;
  uint32_t last = 0;
#pragma unroll 1
  for (; shift >= 0; shift -= 8) {
    for (int b = lane; b < 256; b += 32) hist[b] = 0;
    __syncwarp();
    for (int i = lane; i < cnt; i += 32) {
      uint32_t v;
      if (get(i, v) && (v & pmask) == prefix)
        atomicAdd(&hist[(v >> shift) & 255u], 1u);
    }
    __syncwarp();
    uint32_t h[8];
    uint32_t sum = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      h[j] = hist[lane * 8 + j];
      sum += h[j];
    }
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += t;
    }
    const uint32_t excl = incl - sum;
    const unsigned owner = __ballot_sync(kFull, excl < kk && kk <= incl);
    const int ol = __ffs(owner) - 1;
    uint32_t digit = 0, nk = 0, cd = 0;
    if (lane == ol) {
      uint32_t run = excl;
      bool found = false;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        if (!found) {
          if (run + h[j] >= kk) {
            digit = (uint32_t)(lane * 8 + j);
            nk = kk - run;
            cd = h[j];
            found = true;
          } else {
            run += h[j];
          }
        }
      }
    }
    digit = __shfl_sync(kFull, digit, ol);
    kk = __shfl_sync(kFull, nk, ol);
    last = __shfl_sync(kFull, cd, ol);
    prefix |= digit << shift;
    pmask |= 255u << shift;
    __syncwarp();
  }
  *rank_eq = kk;
  *n_eq = last;
  return prefix;
}

// Finds the bin holding the kk-th smallest entry of a 256-bin histogram
// already filled: returns the bin; *kk_in = rank inside it (1-based),
// *n_bin = entries in it, *total = entries in all bins. When *total < kk
// the other outputs are 0.
__device__ __forceinline__ uint32_t hist_find(const uint32_t* hist, uint32_t kk,
                                              int lane, uint32_t* kk_in,
                                              uint32_t* n_bin, uint32_t* total) {
  uint32_t h[8];
  uint32_t sum = 0;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    h[j] = hist[lane * 8 + j];
    sum += h[j];
  }
  uint32_t incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += t;
  }
  *total = __shfl_sync(kFull, incl, 31);
  if (*total < kk) {
    *kk_in = 0;
    *n_bin = 0;
    return 0;
  }
  const uint32_t excl = incl - sum;
  const unsigned owner = __ballot_sync(kFull, excl < kk && kk <= incl);
  const int ol = __ffs(owner) - 1;
  uint32_t bin = 0, nk = 0, cd = 0;
  if (lane == ol) {
    uint32_t run = excl;
    bool found = false;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      if (!found) {
        if (run + h[j] >= kk) {
          bin = (uint32_t)(lane * 8 + j);
          nk = kk - run;
          cd = h[j];
          found = true;
        } else {
          run += h[j];
        }
      }
    }
  }
  *kk_in = __shfl_sync(kFull, nk, ol);
  *n_bin = __shfl_sync(kFull, cd, ol);
  return __shfl_sync(kFull, bin, ol);
}

// The k-th (key, original index) pair among the nb <= 32 entries of a
// critical bin held by lanes 0..nb-1 (kj, oj; other lanes ~0): rank kk
// (1-based) among them. Returns kth_key; *kth_oid = the pair's index, or
// 0xffffffff when no other entry of the bin has that key (every entry with
// the key is then kept).
__device__ __forceinline__ uint32_t rank_critical(uint32_t kj, uint32_t oj, int nb, uint32_t kk,
                                                  int lane, uint32_t* kth_oid) {
  int rank = 0;
  for (int t = 0; t < nb; ++t) {
    const uint32_t kt = __shfl_sync(kFull, kj, t);
    const uint32_t ot = __shfl_sync(kFull, oj, t);
    rank += (kt < kj) || (kt == kj && ot < oj);
  }
  const unsigned who = __ballot_sync(kFull, lane < nb && rank == (int)kk - 1);
  const int wl = __ffs(who) - 1;
  const uint32_t kth_key = __shfl_sync(kFull, kj, wl);
  uint32_t oid = __shfl_sync(kFull, oj, wl);
  const unsigned same = __ballot_sync(kFull, lane < nb && kj == kth_key);
  if (__popc(same) == 1) oid = 0xffffffffu;
  *kth_oid = oid;
  return kth_key;
}

// Fast exact selection for a buffer whose dist2 all lie in [0, tau]:
// one histogram of dist2 over 256 equal bins of [0, tau] (bin = floor(d2 *
// 256/tau) is monotone in d2, so every entry of a lower bin is smaller),
// then the critical bin is ranked exactly by (dist2, index) across lanes.
// Photons on surfaces give dist2 close to uniform on [0, tau], so the
// critical bin holds one or two entries. Returns false (caller falls back
// to the radix select) when tau is not a positive finite bound or the
// critical bin holds more than 32 entries.
template <int C>
__device__ __forceinline__ bool select_kth_hist(const float4* pos4,
                                                WarpBuf<C>& s, int cnt, int k,
                                                float tau, int lane,
                                                uint32_t& kth_key,
                                                uint32_t& kth_oid) {
  const float sc = __fdiv_rn(256.f, tau);
  if (!(tau > 0.f) || !(sc < __int_as_float(0x7f800000))) return false;
  for (int b = lane; b < 256; b += 32) s.hist[b] = 0;
  __syncwarp();
  for (int i = lane; i < cnt; i += 32) {
    const float d2 = __uint_as_float(s.key[i]);
    const int b = min(255, __float2int_rz(__fmul_rz(d2, sc)));
    atomicAdd(&s.hist[b], 1u);
  }
  __syncwarp();
  uint32_t kk, nb, total;
  const int bin = (int)hist_find(s.hist, (uint32_t)k, lane, &kk, &nb, &total);
  if (total < (uint32_t)k || nb > 32) return false;
  int pos = 0;
  for (int base = 0; base < cnt; base += 32) {
    const int i = base + lane;
    bool in = false;
    if (i < cnt)
      in = min(255, __float2int_rz(__fmul_rz(__uint_as_float(s.key[i]), sc))) ==
           bin;
    const unsigned bal = __ballot_sync(kFull, in);
    if (in) s.sel[pos + __popc(bal & lanemask_lt())] = (uint32_t)i;
    pos += __popc(bal);
  }
  __syncwarp();
  uint32_t kj = 0xffffffffu, oj = 0xffffffffu;
  if (lane < (int)nb) {
    const uint32_t i = s.sel[lane];
    kj = s.key[i];
    oj = orig_index(pos4, s.id[i]);
  }
  kth_key = rank_critical(kj, oj, (int)nb, kk, lane, &kth_oid);
  __syncwarp();
  return true;
}

// Exact k-th smallest (dist2, index) pair of the buffer: kth_key, and
// kth_oid = largest original index kept among entries with key == kth_key
// (0xffffffff when all of them are kept). Every entry has dist2 <= tau.
template <int C, bool S>
__device__ __forceinline__ void select_kth(const float4* pos4, WarpBuf<C>& s,
                                           int cnt, int k, float tau, int lane,
                                           uint32_t& kth_key,
                                           uint32_t& kth_oid) {
  uint32_t rank_eq, n_eq;
  stat_add<S>(s, lane, kStatSelects, 1);
  if (select_kth_hist(pos4, s, cnt, k, tau, lane, kth_key, kth_oid)) return;
  kth_key = warp_select(
      s.hist, cnt, (uint32_t)k,
      [&](int i, uint32_t& v) {
        v = s.key[i];
        return true;
      },
      lane, &rank_eq, &n_eq);
  kth_oid = 0xffffffffu;
  if (rank_eq != n_eq) {
    uint32_t r2, n2;
    const uint32_t kk = kth_key;
    kth_oid = warp_select(
        s.hist, cnt, rank_eq,
        [&](int i, uint32_t& v) {
          if (s.key[i] != kk) return false;
          v = orig_index(pos4, s.id[i]);
          return true;
        },
        lane, &r2, &n2);
  }
}

__device__ __forceinline__ bool keep_entry(const float4* pos4, uint32_t key,
                                           uint32_t id, uint32_t kth_key,
                                           uint32_t kth_oid) {
  if (key < kth_key) return true;
  if (key != kth_key) return false;
  return kth_oid == 0xffffffffu || orig_index(pos4, id) <= kth_oid;
}

template <int C>
__device__ __forceinline__ int compact_kept(const float4* pos4, WarpBuf<C>& s,
                                            int cnt, uint32_t kth_key,
                                            uint32_t kth_oid, int lane) {
  int dst = 0;
  for (int b = 0; b < cnt; b += 32) {
    const int i = b + lane;
    const bool v = i < cnt;
    const uint32_t key = v ? s.key[i] : 0u;
    const uint32_t id = v ? s.id[i] : 0u;
    const bool kp = v && keep_entry(pos4, key, id, kth_key, kth_oid);
    const unsigned bal = __ballot_sync(kFull, kp);
    __syncwarp();
    if (kp) {
      const int o = dst + __popc(bal & lanemask_lt());
      s.key[o] = key;
      s.id[o] = id;
    }
    dst += __popc(bal);
  }
  __syncwarp();
  return dst;
}

// State of a search walk.
struct Query {
  float x, y, z;
  float tau;  // every photon with dist2 <= tau is collected
  int cnt;    // entries in the warp buffer (or the pool)
  int k;
};

// Rare path, kept out of line: the buffer is nearly full. Keeps the k best
// entries; returns {new count, float bits of the k-th distance}.
template <int C, bool S>
__device__ __forceinline__ uint2 tighten(const float4* pos4, WarpBuf<C>* sp,
                                         int cnt, int k, float tau, int lane) {
  WarpBuf<C>& s = *sp;
  uint32_t kth_key, kth_oid;
  select_kth<C, S>(pos4, s, cnt, k, tau, lane, kth_key, kth_oid);
  const int n2 = compact_kept(pos4, s, cnt, kth_key, kth_oid, lane);
  return make_uint2((uint32_t)n2, kth_key);
}

// Appends photon i (position p) when valid and dist2 <= tau.
// P == 0: to the search buffer ({dist2, sorted position}); when the buffer
//         is nearly full, keeps the k best and lowers tau to the k-th.
// P > 0:  to the pool ({position, sorted position} as float4); entries past
//         P are counted but not written (the caller sees q.cnt > P).
template <int C, int P, bool S>
__device__ __forceinline__ void offer(const MapDev& m, Query& q, WarpBuf<C>& s,
                                      int lane, const float4& p, int i,
                                      bool valid) {
  const float d2 = dist2_ref(q.x, q.y, q.z, p.x, p.y, p.z);
  const bool pass = valid && d2 <= q.tau;
  const unsigned bal = __ballot_sync(kFull, pass);
  if (P > 0) {
    if (pass) {
      const int o = q.cnt + __popc(bal & lanemask_lt());
      if (o < P)
        reinterpret_cast<float4*>(s.key)[o] = make_float4(p.x, p.y, p.z, __uint_as_float((uint32_t)i));
    }
    q.cnt += __popc(bal);
    return;
  }
  if (pass) {
    const int o = q.cnt + __popc(bal & lanemask_lt());
    s.key[o] = __float_as_uint(d2);
    s.id[o] = (uint32_t)i;
  }
  q.cnt += __popc(bal);
  if (q.cnt > C - kCutSlack) {
    __syncwarp();
    const uint2 r = tighten<C, S>(m.pos4, &s, q.cnt, q.k, q.tau, lane);
    q.cnt = (int)r.x;
    q.tau = __uint_as_float(r.y);
  }
}

// Scans the photons of the ng groups listed in s.list: lane l handles
// photon (l & 7) of group 4r + (l >> 3) in round r; two rounds are loaded
// before either is used.
template <int C, int P, bool S>
__device__ __forceinline__ void scan_groups(const MapDev& m, Query& q,
                                            WarpBuf<C>& s, int lane, int ng) {
  const int sub = lane >> 3, j = lane & 7;
  stat_add<S>(s, lane, kStatLeaves, (uint32_t)ng);
  for (int r = 0; r < ng; r += 8) {
    const int ga = r + sub, gb = r + 4 + sub;
    int ia = 0, ib = 0;
    bool va = ga < ng, vb = gb < ng;
    if (va) ia = (int)s.list[ga] * kGroup + j;
    if (vb) ib = (int)s.list[gb] * kGroup + j;
    va = va && ia < m.n;
    vb = vb && ib < m.n;
    float4 pa = make_float4(0.f, 0.f, 0.f, 0.f), pb = pa;
    if (va) pa = __ldg(m.pos4 + ia);
    if (vb) pb = __ldg(m.pos4 + ib);
    offer<C, P, S>(m, q, s, lane, pa, ia, va);
    if (r + 4 < ng) offer<C, P, S>(m, q, s, lane, pb, ib, vb);
  }
  __syncwarp();
}

// Scans the contiguous photon range [lo, hi), 32 photons per round.
template <int C, int P, bool S>
__device__ __forceinline__ void scan_range(const MapDev& m, Query& q,
                                           WarpBuf<C>& s, int lane, int lo,
                                           int hi) {
  for (int b = lo; b < hi; b += 64) {
    const int ia = b + lane, ib = b + 32 + lane;
    const bool va = ia < hi, vb = ib < hi;
    float4 pa = make_float4(0.f, 0.f, 0.f, 0.f), pb = pa;
    if (va) pa = __ldg(m.pos4 + ia);
    if (vb) pb = __ldg(m.pos4 + ib);
    offer<C, P, S>(m, q, s, lane, pa, ia, va);
    if (b + 32 < hi) offer<C, P, S>(m, q, s, lane, pb, ib, vb);
  }
}

// Depth-first walk of the box tree collecting all photons with
// dist2 <= q.tau into the warp buffer (P == 0) or the pool (P > 0; the walk
// stops once more than P photons were found). Passing 8-photon groups join
// a waiting list, scanned in full rounds of 8 as they accumulate and in
// full once the walk ends. Both go through one scan site: the scan inlines
// the candidate appends and the rare buffer cut, and a second copy of it
// made the kernel 1.9 % slower (same scan order, same results).
template <int C, int P, bool S>
__device__ __forceinline__ void collect(const MapDev& m, const Levels& L,
                                        Query& q, WarpBuf<C>& s, int lane) {
  q.cnt = 0;
  stat_add<S>(s, lane, kStatWalks, 1);
  if (m.nlevels == 1) {  // a single 8-photon group
    scan_range<C, P, S>(m, q, s, lane, 0, m.n);
    return;
  }
  if (lane == 0) s.stack[0] = ((uint32_t)(m.nlevels - 1) << 28);
  int sp = 1, pending = 0;
  __syncwarp();
  while (true) {
    --sp;
    const uint32_t e = s.stack[sp];
    __syncwarp();
    const int cl = (int)(e >> 28) - 1;  // level of the children
    const int c = (int)(e & 0x0fffffffu) * 32 + lane;
    stat_add<S>(s, lane, kStatNodes, 1);
    bool pass = false;
    const int2 oc = L.oc[cl];
    if (c < oc.y) {
      const int jb = oc.x + c;
      const float4 lo = __ldg(m.boxes + 2 * jb);
      const float4 hi = __ldg(m.boxes + 2 * jb + 1);
      pass = box_dist2(q.x, q.y, q.z, lo, hi) <= q.tau;
    }
    const unsigned bal = __ballot_sync(kFull, pass);
    const int off = __popc(bal & lanemask_lt());
    if (cl == 0) {
      // the passing groups join the waiting list
      if (pass) s.list[pending + off] = (uint32_t)c;
      pending += __popc(bal);
    } else {
      if (pass) s.stack[sp + off] = ((uint32_t)cl << 28) | c;
      sp += __popc(bal);
    }
    __syncwarp();
    const bool done = sp == 0;
    // full rounds of 8 groups after a bottom-level node, the rest at the end
    const int take = done ? pending : (cl == 0 ? (pending & ~7) : 0);
    if (take > 0) {
      scan_groups<C, P, S>(m, q, s, lane, take);
      const int rest = pending - take;
      uint32_t keep = 0;
      if (lane < rest) keep = s.list[take + lane];
      __syncwarp();
      if (lane < rest) s.list[lane] = keep;
      __syncwarp();
      pending = rest;
      if (P > 0 && q.cnt > P) break;  // the pool overflowed
    }
    if (done) break;
  }
}

__device__ __forceinline__ unsigned long long warp_min_u64(
    unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long t = __shfl_xor_sync(kFull, v, o);
    v = t < v ? t : v;
  }
  return v;
}

// Upper bound of the k-th distance from scratch: walk down to a group
// greedily (nearest box at each level), then take the k-th distance among
// the photons of the Morton-adjacent groups around it (real photons, so
// the bound holds).
template <int C, bool S>
__device__ __forceinline__ float cold_tau(const float4* pos4, const float4* boxes,
                                       int n, int nlevels, const Levels* Lp,
                                       float qx, float qy, float qz, int k,
                                       WarpBuf<C>* sp, int lane) {
  const Levels& L = *Lp;
  WarpBuf<C>& s = *sp;
  int node = 0;
  for (int cl = nlevels - 2; cl >= 0; --cl) {
    const int c = node * 32 + lane;
    unsigned long long key = ~0ull;
    const int2 oc = L.oc[cl];
    if (c < oc.y) {
      const int jb = oc.x + c;
      const float d = box_dist2(qx, qy, qz, __ldg(boxes + 2 * jb),
                                __ldg(boxes + 2 * jb + 1));
      key = ((unsigned long long)__float_as_uint(d) << 32) | (unsigned)c;
    }
    key = warp_min_u64(key);
    node = (int)(key & 0xffffffffu);
  }
  MapDev m;
  m.pos4 = pos4;
  m.n = n;
  Query q;
  q.x = qx; q.y = qy; q.z = qz;
  q.k = k;
  q.tau = __int_as_float(0x7f800000);  // +inf
  q.cnt = 0;
  // the photons of the 32 groups sharing the nearest group's parent (a
  // compact patch of 256 Morton-adjacent photons), or more groups around
  // it when k needs them
  const int ngroups = L.oc[0].y;
  const int want = min(ngroups, max(32, (k + kGroup - 1) / kGroup + 8));
  const int first =
      max(0, min(want == 32 ? (node & ~31) : node - want / 2, ngroups - want));
  scan_range<C, 0, S>(m, q, s, lane, first * kGroup, min(n, (first + want) * kGroup));
  __syncwarp();
  if (q.cnt < k) return __int_as_float(0x7f800000);
  uint32_t mx = 0;
  for (int i = lane; i < q.cnt; i += 32) mx = max(mx, s.key[i]);
  mx = __reduce_max_sync(kFull, mx);  // every entry lies in [0, mx]
  uint32_t kth_key, kth_oid;
  select_kth<C, S>(pos4, s, q.cnt, k, __uint_as_float(mx), lane, kth_key, kth_oid);
  return __uint_as_float(kth_key);
}

// Warm state of the per-query search: the previous query answered this way
// and its exact k-th distance.
struct Warm {
  bool have;
  float x, y, z, kth;
};

// Per-query search of query (qx, qy, qz): the kept photons (the k nearest,
// or all photons when fewer), compacted in s.key / s.id in walk order.
// Returns their number; *maxd2 = the largest kept dist2 (0 when none).
// r_hint: the last exact k-th distance this warp found (in/out).
template <int C, bool S>
__device__ __forceinline__ int search_one(const MapDev& m, const Levels& L, WarpBuf<C>& s,
                                          int lane, float qx, float qy, float qz, int k,
                                          Warm& w, float& r_hint, float* maxd2) {
  const float kInf = __int_as_float(0x7f800000);
  Query q;
  q.x = qx; q.y = qy; q.z = qz;
  q.k = k;
  q.cnt = 0;
  q.tau = kInf;
  const bool bad = m.n == 0 || isnan(qx) || isnan(qy) || isnan(qz);
  if (!bad) {
    bool warm = false, warm_guess = false;
    float tau_sure = 0.f;
    if (w.have) {
      const float d2 = dist2_ref(qx, qy, qz, w.x, w.y, w.z);
      if (d2 <= w.kth) {
        const float rp = sqrtf(w.kth);
        const float r = rp + sqrtf(d2);
        const float rr = r * 1.00001f;
        tau_sure = fmaxf(rr * rr * 1.00001f, 1e-37f);
        q.tau = tau_sure;
        warm = true;
        // the k-th distance changes little between neighbours: collect
        // within a radius a little above the previous one first; fewer
        // than k photons inside it falls back to the sure bound
        const float rg = kWarmGuess * rp;
        if (rg * rg < tau_sure) {
          q.tau = rg * rg;
          warm_guess = true;
        }
      }
    }
    // Guess and verify when no bound is known: collect with a radius a
    // little above the last k-th distance this warp found; k photons or
    // more inside it make the result exact, otherwise the radius doubles
    // (twice), then the patch bound of cold_tau is used.
    bool guess = false, need_cold = false;
    float rg = 0.f;
    if (!warm) {
      stat_add<S>(s, lane, kStatCold, 1);
      if (r_hint > 0.f) {
        guess = true;
        rg = 1.3f * r_hint;
        q.tau = fmaxf(rg * rg, 1e-37f);
      } else {
        need_cold = true;
      }
    }
    for (int attempt = 0;; ++attempt) {
      if (need_cold) {
        q.tau = cold_tau<C, S>(m.pos4, m.boxes, m.n, m.nlevels, &L, qx, qy, qz, k, &s, lane);
        need_cold = false;
        guess = false;
      }
      collect<C, 0, S>(m, L, q, s, lane);
      if (warm_guess) {
        if (q.cnt >= k) break;
        warm_guess = false;
        q.tau = tau_sure;
        continue;
      }
      if (!guess || q.cnt >= k) break;
      if (attempt < 2) {
        rg *= 2.0f;
        q.tau = fmaxf(rg * rg, 1e-37f);
      } else {
        need_cold = true;
      }
    }
  }
  __syncwarp();
  stat_add<S>(s, lane, kStatQueries, 1);
  stat_add<S>(s, lane, kStatCand, (uint32_t)q.cnt);
  const int cnt = q.cnt;
  const bool all = cnt <= k;
  uint32_t kth_key = 0, kth_oid = 0xffffffffu;
  if (all) {
    uint32_t mx = 0;
    for (int i = lane; i < cnt; i += 32) mx = max(mx, s.key[i]);
    kth_key = __reduce_max_sync(kFull, mx);
  } else {
    select_kth<C, S>(m.pos4, s, cnt, k, q.tau, lane, kth_key, kth_oid);
  }
  const int kept = all ? cnt : k;
  *maxd2 = kept > 0 ? __uint_as_float(kth_key) : 0.f;
  const int nk = all ? cnt : compact_kept(m.pos4, s, cnt, kth_key, kth_oid, lane);
  if (!bad && kept >= k) {
    w.have = true;
    w.x = qx; w.y = qy; w.z = qz;
    w.kth = *maxd2;
    r_hint = sqrtf(*maxd2);
  } else {
    w.have = false;
  }
  return nk;
}

// A query answered from a pool of np photons collected within radius
// sqrt(tau) of (cx, cy, cz); rp = sqrt(tau) shrunk for rounding. On success
// the kept photons (exactly k) are in kkey / kid (the histogram's words) in
// pool order, and *maxd2 is the k-th distance; false when the pool cannot
// prove the result (the query is then searched on its own).
template <int C, int P, bool S>
__device__ __forceinline__ bool pool_query(const MapDev& m, WarpBuf<C>& s, int lane, int np,
                                           float qx, float qy, float qz, float cx, float cy,
                                           float cz, float rp, int k, float* maxd2) {
  const float4* pool = reinterpret_cast<const float4*>(s.key);
  // every photon within a of the query lies in the pool: |p - c| <=
  // |p - q| + |q - c| <= a + rq <= rp, with margins of 1e-5 relative for
  // the rounding of the distances (a few units of 2^-24 each)
  const float rq = sqrtf(dist2_ref(qx, qy, qz, cx, cy, cz)) * 1.00001f;
  const float a = rp - rq;
  if (!(a > 0.f)) return false;
  const float a2 = a * a * 0.99999f;
  const float sc = __fdiv_rn(256.f, a2);
  if (!(sc < __int_as_float(0x7f800000))) return false;
  constexpr int NS = P > 0 ? P / 32 : 1;
  float d[NS];
#pragma unroll
  for (int j = 0; j < NS; ++j) {
    d[j] = __int_as_float(0x7f800000);
    if (j * 32 < np) {
      const int e = j * 32 + lane;
      if (e < np) {
        const float4 p = pool[e];
        d[j] = dist2_ref(qx, qy, qz, p.x, p.y, p.z);
      }
    }
  }
  // histogram of the distances within a, over 256 bins of [0, a2]
  for (int b = lane; b < 256; b += 32) s.hist[b] = 0;
  __syncwarp();
#pragma unroll
  for (int j = 0; j < NS; ++j)
    if (d[j] <= a2) atomicAdd(&s.hist[min(255, __float2int_rz(__fmul_rz(d[j], sc)))], 1u);
  __syncwarp();
  uint32_t kk, nb, total;
  const int bin = (int)hist_find(s.hist, (uint32_t)k, lane, &kk, &nb, &total);
  stat_add<S>(s, lane, kStatCand, total);
  if (total < (uint32_t)k || nb > 32) return false;
  // the critical bin's entries (key, pool index) in sel / list
  int pos = 0;
#pragma unroll
  for (int j = 0; j < NS; ++j) {
    const bool in = d[j] <= a2 && min(255, __float2int_rz(__fmul_rz(d[j], sc))) == bin;
    const unsigned bal = __ballot_sync(kFull, in);
    if (in) {
      const int o = pos + __popc(bal & lanemask_lt());
      s.sel[o] = __float_as_uint(d[j]);
      s.list[o] = (uint32_t)(j * 32 + lane);
    }
    pos += __popc(bal);
  }
  __syncwarp();
  uint32_t kj = 0xffffffffu, oj = 0xffffffffu;
  if (lane < (int)nb) {
    kj = s.sel[lane];
    oj = orig_index(m.pos4, __float_as_uint(pool[s.list[lane]].w));
  }
  uint32_t kth_oid;
  const uint32_t kth_key = rank_critical(kj, oj, (int)nb, kk, lane, &kth_oid);
  __syncwarp();  // the histogram is read: its words take the kept list
  uint32_t* kkey = s.hist;
  uint32_t* kid = s.hist + 128;
  int nk = 0;
#pragma unroll
  for (int j = 0; j < NS; ++j) {
    if (j * 32 < np) {
      const uint32_t kb = __float_as_uint(d[j]);  // +inf past the pool: never kept
      const int e = j * 32 + lane;
      uint32_t sid = 0;
      if (e < np) sid = __float_as_uint(pool[e].w);
      bool kp = kb < kth_key;
      if (kb == kth_key)
        kp = kth_oid == 0xffffffffu || orig_index(m.pos4, sid) <= kth_oid;
      const unsigned bal = __ballot_sync(kFull, kp);
      const int o = nk + __popc(bal & lanemask_lt());
      if (kp && o < kPoolMaxK) {
        kkey[o] = kb;
        kid[o] = sid;
      }
      nk += __popc(bal);
    }
  }
  __syncwarp();
  if (nk != k) return false;  // (the selection keeps exactly k)
  stat_add<S>(s, lane, kStatQueries, 1);
  stat_add<S>(s, lane, kStatPoolQueries, 1);
  *maxd2 = __uint_as_float(kth_key);
  return true;
}

// Output of one query from its kept photons (key[], id[] hold nk entries in
// walk order; id = sorted positions, rewritten in place in knn mode).
//   radiance: the estimate of integrator.h:141-150 into stage[0..3) when
//             stage is set, else out.rgb[3 rec ..]
//   knn:      the index list in the reference's order (photon_map.h:166-
//             183), count and maxDist2 at row qi
//   adjoint:  adj_in[3 rec ..] times d estimate / d throughput onto every
//             kept photon of photon_adj
// r0 = {pos, rho.r}, r1 = {wo, rho.g}, r2 = {ns, rho.b} (radiance records).
template <int MODE>
__device__ __forceinline__ void emit(const MapDev& m, int lane, const uint32_t* key, uint32_t* id,
                                     int nk, float maxd2, int k, float n_emitted,
                                     const float4& r0, const float4& r1, const float4& r2,
                                     int64_t qi, int64_t rec, const KnnOut& out, float* stage) {
  if (MODE == kModeAdjoint) {
    // d estimate / d throughput_i = f(wo, wi_i) / (n_emitted pi maxd2)
    // for the kept photons (integrator.h:141-150)
    const float ax = out.adj_in[3 * rec], ay = out.adj_in[3 * rec + 1],
                az = out.adj_in[3 * rec + 2];
    if (nk > 0 && (ax != 0.f || ay != 0.f || az != 0.f)) {
      const float cos_o = dot_ref(r1.x, r1.y, r1.z, r2.x, r2.y, r2.z);
      const float den = __fmul_rn(__fmul_rn(n_emitted, kPI), maxd2);
      const float cr = __fdiv_rn(__fmul_rn(ax, __fdiv_rn(r0.w, kPI)), den);
      const float cg = __fdiv_rn(__fmul_rn(ay, __fdiv_rn(r1.w, kPI)), den);
      const float cb = __fdiv_rn(__fmul_rn(az, __fdiv_rn(r2.w, kPI)), den);
      for (int i = lane; i < nk; i += 32) {
        const uint32_t sid = id[i];
        const float4 t = __ldg(m.thr4 + sid);
        const float2 wv = __ldg(m.wi2 + sid);
        const float cos_i = dot_ref(t.w, wv.x, wv.y, r2.x, r2.y, r2.z);
        if (!(cos_o < 0.f) && !(cos_i < 0.f))
          atomicAdd(out.photon_adj + orig_index(m.pos4, sid), make_float4(cr, cg, cb, 0.f));
      }
    }
  } else if (MODE == kModeRadiance) {
    const float cos_o = dot_ref(r1.x, r1.y, r1.z, r2.x, r2.y, r2.z);
    const float fr = __fdiv_rn(r0.w, kPI);
    const float fg = __fdiv_rn(r1.w, kPI);
    const float fb = __fdiv_rn(r2.w, kPI);
    float lr = 0.f, lg = 0.f, lb = 0.f;
    for (int i = lane; i < nk; i += 32) {
      const uint32_t sid = id[i];
      const float4 t = __ldg(m.thr4 + sid);
      const float2 wv = __ldg(m.wi2 + sid);
      const float cos_i = dot_ref(t.w, wv.x, wv.y, r2.x, r2.y, r2.z);
      // Lambert::evaluate returns 0 when either cosine is < 0
      if (!(cos_o < 0.f) && !(cos_i < 0.f)) {
        lr = __fadd_rn(lr, __fmul_rn(fr, t.x));
        lg = __fadd_rn(lg, __fmul_rn(fg, t.y));
        lb = __fadd_rn(lb, __fmul_rn(fb, t.z));
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lr = __fadd_rn(lr, __shfl_xor_sync(kFull, lr, o));
      lg = __fadd_rn(lg, __shfl_xor_sync(kFull, lg, o));
      lb = __fadd_rn(lb, __shfl_xor_sync(kFull, lb, o));
    }
    if (lane == 0) {
      float3 o3 = make_float3(0.f, 0.f, 0.f);
      if (nk > 0) {
        const float den = __fmul_rn(__fmul_rn(n_emitted, kPI), maxd2);
        o3 = make_float3(__fdiv_rn(lr, den), __fdiv_rn(lg, den), __fdiv_rn(lb, den));
      }
      float* dst = stage ? stage : out.rgb + 3 * rec;
      dst[0] = o3.x;
      dst[1] = o3.y;
      dst[2] = o3.z;
    }
  } else {
    for (int i = lane; i < nk; i += 32) id[i] = orig_index(m.pos4, id[i]);
    __syncwarp();
    int32_t* orow = out.idx + qi * (int64_t)k;
    for (int i = lane; i < nk; i += 32) {
      const uint32_t ki = key[i], oi = id[i];
      int rank = 0;
      for (int j = 0; j < nk; ++j) {
        const uint32_t kj = key[j], oj = id[j];
        rank += (kj > ki) || (kj == ki && oj > oi);
      }
      orow[rank] = (int32_t)oi;
    }
    for (int r = nk + lane; r < k; r += 32) orow[r] = -1;
    if (lane == 0) {
      out.count[qi] = nk;
      out.maxd2[qi] = maxd2;
    }
  }
  __syncwarp();
}

// Answers queries [qb, qb + nw) (nw <= 32) on map m. Lane i loads the
// record of query qb + i (record order[qb + i] when `order` is set). When
// `stage` is set (radiance mode), query qb + i's radiance goes to
// stage[3 i ..] instead of the output. P > 0: neighbourhood pools first
// (when `pool` and k <= kPoolMaxK), the per-query search for the rest.
template <int C, int P, int MODE, bool S>
__device__ __forceinline__ void knn_window(const MapDev& m, const Levels& L, WarpBuf<C>& s,
                                           int lane, const void* __restrict__ queries,
                                           int64_t qb, int nw, int k, float n_emitted,
                                           const KnnOut& out, const uint32_t* __restrict__ order,
                                           int stride4, bool pool, float& r_hint,
                                           float* stage) {
  const float kInf = __int_as_float(0x7f800000);
  float4 a0 = make_float4(0.f, 0.f, 0.f, 0.f), a1 = a0, a2 = a0;
  int64_t rec = qb + lane;
  if (lane < nw) {
    if (MODE == kModeKnn) {
      const float* q3 = reinterpret_cast<const float*>(queries) + 3 * rec;
      a0 = make_float4(__ldcg(q3), __ldcg(q3 + 1), __ldcg(q3 + 2), 0.f);
    } else {
      if (order) rec = (int64_t)__ldg(order + qb + lane);
      const float4* q4 = reinterpret_cast<const float4*>(queries) + stride4 * rec;
      a0 = __ldcg(q4);
      a1 = __ldcg(q4 + 1);
      a2 = __ldcg(q4 + 2);
    }
  }
  const bool mine = lane < nw;
  const bool badq = mine && (m.n == 0 || isnan(a0.x) || isnan(a0.y) || isnan(a0.z));
  unsigned fb = __ballot_sync(kFull, badq);  // answered by the per-query search
  unsigned todo = __ballot_sync(kFull, mine) & ~fb;
  Warm w;
  w.have = false;
  w.x = w.y = w.z = w.kth = 0.f;

  auto emit_i = [&](int i, const uint32_t* key, uint32_t* id, int nk, float maxd2) {
    float4 r0, r1, r2;
    r0.x = __shfl_sync(kFull, a0.x, i); r0.y = __shfl_sync(kFull, a0.y, i);
    r0.z = __shfl_sync(kFull, a0.z, i); r0.w = __shfl_sync(kFull, a0.w, i);
    r1.x = __shfl_sync(kFull, a1.x, i); r1.y = __shfl_sync(kFull, a1.y, i);
    r1.z = __shfl_sync(kFull, a1.z, i); r1.w = __shfl_sync(kFull, a1.w, i);
    r2.x = __shfl_sync(kFull, a2.x, i); r2.y = __shfl_sync(kFull, a2.y, i);
    r2.z = __shfl_sync(kFull, a2.z, i); r2.w = __shfl_sync(kFull, a2.w, i);
    const int64_t ri = __shfl_sync(kFull, rec, i);
    emit<MODE>(m, lane, key, id, nk, maxd2, k, n_emitted, r0, r1, r2, qb + i, ri, out,
               stage ? stage + 3 * i : nullptr);
  };
  auto answer = [&](int i) {  // the per-query search
    const float qx = __shfl_sync(kFull, a0.x, i), qy = __shfl_sync(kFull, a0.y, i),
                qz = __shfl_sync(kFull, a0.z, i);
    float maxd2;
    const int nk = search_one<C, S>(m, L, s, lane, qx, qy, qz, k, w, r_hint, &maxd2);
    emit_i(i, s.key, s.id, nk, maxd2);
  };

  if constexpr (P > 0) {
   if (pool && k <= kPoolMaxK && m.nlevels > 1) {
    if (!(r_hint > 0.f) && todo) {  // a warp without a k-th distance yet
      const int i = __ffs(todo) - 1;
      todo &= todo - 1;
      answer(i);
    }
    while (todo && r_hint > 0.f) {
      const int lead = __ffs(todo) - 1;
      const float lx = __shfl_sync(kFull, a0.x, lead), ly = __shfl_sync(kFull, a0.y, lead),
                  lz = __shfl_sync(kFull, a0.z, lead);
      const float gr = kPoolGroup * r_hint;
      const bool mem = lane == lead || (((todo >> lane) & 1u) &&
                                        dist2_ref(a0.x, a0.y, a0.z, lx, ly, lz) <= gr * gr);
      const unsigned mset = __ballot_sync(kFull, mem);
      todo &= ~mset;
      // centre: the middle of the members' bounding box
      float lo_x = mem ? a0.x : kInf, lo_y = mem ? a0.y : kInf, lo_z = mem ? a0.z : kInf;
      float hi_x = mem ? a0.x : -kInf, hi_y = mem ? a0.y : -kInf, hi_z = mem ? a0.z : -kInf;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        lo_x = fminf(lo_x, __shfl_xor_sync(kFull, lo_x, o));
        lo_y = fminf(lo_y, __shfl_xor_sync(kFull, lo_y, o));
        lo_z = fminf(lo_z, __shfl_xor_sync(kFull, lo_z, o));
        hi_x = fmaxf(hi_x, __shfl_xor_sync(kFull, hi_x, o));
        hi_y = fmaxf(hi_y, __shfl_xor_sync(kFull, hi_y, o));
        hi_z = fmaxf(hi_z, __shfl_xor_sync(kFull, hi_z, o));
      }
      Query pq;
      pq.x = 0.5f * (lo_x + hi_x);
      pq.y = 0.5f * (lo_y + hi_y);
      pq.z = 0.5f * (lo_z + hi_z);
      const float rc2 = mem ? dist2_ref(a0.x, a0.y, a0.z, pq.x, pq.y, pq.z) : 0.f;
      const float rc = sqrtf(__uint_as_float(__reduce_max_sync(kFull, __float_as_uint(rc2))));
      const float R = (kPoolFactor * r_hint + rc) * 1.00002f;
      pq.tau = R * R;
      pq.k = k;
      pq.cnt = 0;
      collect<C, P, S>(m, L, pq, s, lane);
      const int np = pq.cnt;
      if (np > P) {
        fb |= mset;
        continue;
      }
      const float rp = sqrtf(pq.tau) * 0.99999f;
      unsigned mm = mset;
      while (mm) {
        const int i = __ffs(mm) - 1;
        mm &= mm - 1;
        const float qx = __shfl_sync(kFull, a0.x, i), qy = __shfl_sync(kFull, a0.y, i),
                    qz = __shfl_sync(kFull, a0.z, i);
        float maxd2;
        if (pool_query<C, P, S>(m, s, lane, np, qx, qy, qz, pq.x, pq.y, pq.z, rp, k, &maxd2)) {
          emit_i(i, s.hist, s.hist + 128, k, maxd2);
          r_hint = sqrtf(maxd2);
        } else {
          fb |= 1u << i;
        }
      }
    }
   }
  }
  fb |= todo;
  // the per-query search for the rest, in query order
  while (fb) {
    const int i = __ffs(fb) - 1;
    fb &= fb - 1;
    answer(i);
  }
}

// Answers the work item [qb, qe) in windows of up to 32 queries; in
// radiance mode without `order` the radiance of the item (at most kChunk
// queries, qb a multiple of 8) is staged and stored together (16-byte
// words when the output allows: few, wide stores into mapped host memory).
template <int C, int P, int MODE, bool S>
__device__ __forceinline__ void knn_item(const MapDev& m, const Levels& L, WarpBuf<C>& s,
                                         int lane, const void* __restrict__ queries, int64_t qb,
                                         int64_t qe, int k, float n_emitted, const KnnOut& out,
                                         const uint32_t* __restrict__ order, int stride4,
                                         bool pool, float& r_hint) {
  const bool staged = MODE == kModeRadiance && !order && qe - qb <= kChunk;
  for (int64_t wb = qb; wb < qe; wb += 32) {
    const int nw = (int)min((int64_t)32, qe - wb);
    knn_window<C, P, MODE, S>(m, L, s, lane, queries, wb, nw, k, n_emitted, out, order, stride4,
                              pool, r_hint, staged ? s.stage : nullptr);
  }
  if (staged) {
    __syncwarp();
    const int nf = 3 * (int)(qe - qb);
    float* dst = out.rgb + 3 * qb;
    if (nf % 4 == 0 && (reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
      if (lane < nf / 4)
        reinterpret_cast<float4*>(dst)[lane] = reinterpret_cast<const float4*>(s.stage)[lane];
    } else {
      for (int i = lane; i < nf; i += 32) dst[i] = s.stage[i];
    }
    __syncwarp();
  }
}

// Threads per block and minimum resident blocks of a kernel with search
// buffer C and pool P.
constexpr int knn_threads(int C, int P) { return P > 0 ? 128 : (C <= 512 ? 256 : 128); }
constexpr int knn_min_blocks(int C, int P) { return P > 0 ? 5 : (C <= 512 ? 4 : 2); }

template <int C, int P, int MODE, bool S>
__global__ void __launch_bounds__(knn_threads(C, P), knn_min_blocks(C, P))
    knn_kernel(MapDev m, const void* __restrict__ queries, int64_t nq, int k,
               float n_emitted, KnnOut out,
               unsigned long long* __restrict__ counter,
               const uint32_t* __restrict__ order, int stride4, int64_t head_items,
               int pool) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ Levels L;
  WarpBuf<C>& s = reinterpret_cast<WarpBuf<C>*>(smem_raw)[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < kMaxLevels; ++i) {  // constant indices: m stays in
      L.oc[i] = make_int2(m.lvl_off[i], m.lvl_cnt[i]);  // the parameter bank
    }
  }
  if (lane < 8) s.stat[lane] = 0;
  __syncthreads();
  float r_hint = -1.f;  // last exact k-th distance this warp found

  while (true) {
    unsigned long long c0 = 0;
    if (lane == 0) c0 = atomicAdd(counter, 1ull);
    c0 = __shfl_sync(kFull, c0, 0);
    const int64_t item = (int64_t)c0;  // items [0, head_items) hold kChunk queries
    const bool head = item < head_items;
    const int64_t qb = head ? item * kChunk : head_items * kChunk + (item - head_items) * kTail;
    if (qb >= nq) break;
    const int64_t qe = min(nq, qb + (head ? kChunk : kTail));

    knn_item<C, P, MODE, S>(m, L, s, lane, queries, qb, qe, k, n_emitted, out, order, stride4,
                            pool != 0, r_hint);
    if (S) {
      __syncwarp();
      if (lane < kNumStats) {
        atomicAdd(out.stats + lane, (unsigned long long)s.stat[lane]);
        s.stat[lane] = 0;
      }
      __syncwarp();
    }
  }
}

template <int C, int P, int MODE>
static cudaError_t launch_one(const MapDev& m, const void* queries,
                              int64_t nq, int k, float n_emitted, KnnOut out,
                              unsigned long long* counter, int num_sms,
                              cudaStream_t st, const uint32_t* order,
                              int stride4, bool pool) {
  constexpr int kThreads = knn_threads(C, P);
  const size_t smem = (kThreads / 32) * sizeof(WarpBuf<C>);
  auto kern = out.stats ? knn_kernel<C, P, MODE, true> : knn_kernel<C, P, MODE, false>;
  cudaError_t e = cudaFuncSetAttribute(
      kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads,
                                                    smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) per_sm = 1;
  const int64_t chunks = (nq + kTail - 1) / kTail;
  const int64_t warps_per_block = kThreads / 32;
  int64_t blocks = (int64_t)num_sms * per_sm;
  const int64_t need = (chunks + warps_per_block - 1) / warps_per_block;
  if (blocks > need) blocks = need;
  if (blocks < 1) blocks = 1;
  const int64_t tail = blocks * warps_per_block * kTail * kTailItems;
  const int64_t head_items = nq > tail ? (nq - tail) / kChunk : 0;
  e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st);
  if (e != cudaSuccess) return e;
  kern<<<(unsigned)blocks, kThreads, smem, st>>>(m, queries, nq, k, n_emitted,
                                                 out, counter, order, stride4, head_items,
                                                 pool ? 1 : 0);
  return cudaGetLastError();
}

template <int MODE>
static cudaError_t launch_mode(const MapDev& m, const void* queries, int64_t nq, int k,
                               float n_emitted, KnnOut out, unsigned long long* counter,
                               int num_sms, cudaStream_t st, const uint32_t* order, int stride4,
                               bool pool) {
  if (k <= kPoolMaxK)
    return launch_one<kPoolBuf, kPoolSize, MODE>(m, queries, nq, k, n_emitted, out, counter,
                                                 num_sms, st, order, stride4, pool);
  if (k <= 224)
    return launch_one<512, 0, MODE>(m, queries, nq, k, n_emitted, out, counter, num_sms, st,
                                    order, stride4, false);
  return launch_one<2048, 0, MODE>(m, queries, nq, k, n_emitted, out, counter, num_sms, st,
                                   order, stride4, false);
}

cudaError_t knn_launch(const MapDev& m, const void* queries, int64_t nq,
                       int k, int mode, float n_emitted, KnnOut out,
                       unsigned long long* counter, int num_sms,
                       cudaStream_t st, const uint32_t* order, int stride4, bool pool) {
  if (nq <= 0) return cudaSuccess;
  if (mode == kModeAdjoint)
    return launch_mode<kModeAdjoint>(m, queries, nq, k, n_emitted, out, counter, num_sms, st,
                                     order, stride4, pool);
  if (mode == kModeRadiance)
    return launch_mode<kModeRadiance>(m, queries, nq, k, n_emitted, out, counter, num_sms, st,
                                      order, stride4, pool);
  return launch_mode<kModeKnn>(m, queries, nq, k, n_emitted, out, counter, num_sms, st, order,
                               stride4, pool);
}

}  // namespace pm

// ------------------------------------------------------------ batched kNN
namespace pm {

// The radiance estimate of every query of every scene of a batch in one
// persistent launch. A work item is `chunk` consecutive queries of one
// scene (in the order of the sorted keys: scene, then Morton code); a warp
// takes items from `counter` until none are left, switching its copy of the
// photon map (map pointers, tree shape) when the scene changes. The
// kernel with search buffer kPoolBuf pools neighbourhoods for scenes with
// k <= kPoolMaxK.
template <int C, int P>
__global__ void __launch_bounds__(256, 2)
    knn_batch_kernel(BatchTables t, const float4* __restrict__ slots,
                     const uint32_t* __restrict__ order, const int64_t* __restrict__ qoff,
                     const int64_t* __restrict__ item_off, int chunk, KnnOut out,
                     unsigned long long* __restrict__ counter) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int64_t ioff[kMaxBatchScenes + 1];
  __shared__ MapDev wmap[8];
  __shared__ Levels wlev[8];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WarpBuf<C>& s = reinterpret_cast<WarpBuf<C>*>(smem_raw)[warp];
  batch_load_offsets(ioff, item_off, t.n_scenes);
  __syncthreads();
  const int64_t total = ioff[t.n_scenes];
  float r_hint = -1.f;
  int cur = -1, k = 0;
  float n_emitted = 0.f;
  while (true) {
    unsigned long long c0 = 0;
    if (lane == 0) c0 = atomicAdd(counter, 1ull);
    c0 = __shfl_sync(kFull, c0, 0);
    if ((int64_t)c0 >= total) break;
    const int sc = batch_find(ioff, t.n_scenes, (int64_t)c0);
    if (sc != cur) {
      __syncwarp();
      if (lane == 0) {
        const BatchScene& bs = t.scenes[sc];
        wmap[warp] = bs.map;
        for (int i = 0; i < kMaxLevels; ++i) {
          wlev[warp].oc[i] = make_int2(bs.map.lvl_off[i], bs.map.lvl_cnt[i]);
        }
      }
      __syncwarp();
      cur = sc;
      k = t.scenes[sc].k;
      n_emitted = t.scenes[sc].n_emitted;
      r_hint = -1.f;
    }
    const int64_t qb = qoff[sc] + ((int64_t)c0 - ioff[sc]) * chunk;
    const int64_t qe = min(qoff[sc + 1], qb + chunk);
    knn_item<C, P, kModeRadiance, false>(wmap[warp], wlev[warp], s, lane, slots, qb, qe, k,
                                         n_emitted, out, order, 4, true, r_hint);
  }
}

// The kernel behind a tuning's candidate-buffer size: 512 selects the
// pooling kernel (search buffer kPoolBuf), 2048 the large-k one.
template <class F>
static cudaError_t with_batch_kernel(int buffer, F f) {
  if (buffer <= 512) return f(knn_batch_kernel<kPoolBuf, kPoolSize>, sizeof(WarpBuf<kPoolBuf>));
  return f(knn_batch_kernel<2048, 0>, sizeof(WarpBuf<2048>));
}

cudaError_t batch_knn_prepare(int warps, int buffer, int* blocks_per_sm) {
  if (warps < 1 || warps > 8) return cudaErrorInvalidValue;
  return with_batch_kernel(buffer, [&](auto kern, size_t wb) {
    const size_t smem = (size_t)warps * wb;
    cudaError_t e =
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * warps, smem);
    if (e != cudaSuccess) return e;
    *blocks_per_sm = per_sm < 1 ? 1 : per_sm;
    return cudaSuccess;
  });
}

cudaError_t batch_knn_launch(const BatchTables& t, const float4* slots, const uint32_t* order,
                             const int64_t* qoff, const int64_t* item_off, int64_t max_items,
                             float* res, int warps, int chunk, int buffer, int blocks_per_sm,
                             unsigned long long* counter, int num_sms, cudaStream_t st) {
  if (warps < 1 || warps > 8 || chunk < 1) return cudaErrorInvalidValue;
  const int threads = 32 * warps;
  int64_t blocks = (int64_t)num_sms * blocks_per_sm;
  const int64_t need = (max_items + warps - 1) / warps;
  if (blocks > need) blocks = need;
  if (blocks < 1) blocks = 1;
  cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st);
  if (e != cudaSuccess) return e;
  KnnOut out{};
  out.rgb = res;
  return with_batch_kernel(buffer, [&](auto kern, size_t wb) {
    const size_t smem = (size_t)warps * wb;
    kern<<<(unsigned)blocks, threads, smem, st>>>(t, slots, order, qoff, item_off, chunk, out,
                                                  counter);
    return cudaGetLastError();
  });
}

}  // namespace pm
