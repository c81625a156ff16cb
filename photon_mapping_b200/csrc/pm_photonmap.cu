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
// One warp answers one query at a time, walking a chunk of consecutive
// queries. Per query:
//   1. bound: an upper bound tau of the k-th distance. From the previous
//      query of the chunk by the triangle inequality when it is close
//      ((r_prev + delta)^2, inflated for rounding; first tried at the
//      smaller (1.06 r_prev)^2, kept when it holds k photons), else from
//      the photons Morton-adjacent to the group nearest the query.
//   2. collect: depth-first walk of the 32-ary box tree; the passing
//      8-photon groups of a node are scanned packed, 4 groups per round,
//      every photon with dist2 <= tau appended to the warp's buffer. A
//      nearly full buffer is cut to the k best, lowering tau.
//   3. select: radix select of the exact k-th (dist2, index) pair.
//   4. output: the radiance sum (Lambert, integrator.h:141-150) or the
//      index list in the reference's order.

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
// of work at nearly the same time (measured on 1M primary-hit queries at
// k = 100: 3.68 ms against 3.96 ms with items of 32 throughout; larger
// items keep more warm starts but leave a longer tail).
constexpr int kChunk = 16;
constexpr int kTail = 8;
constexpr int kTailItems = 2;
static_assert(kChunk % 8 == 0 && kTail % 8 == 0, "items start at multiples of 8");

// The last kStageWords entries of WarpBuf::id hold the radiance of up to 8
// consecutive queries (an aligned group of 8) until the warp stores them
// together: 96 bytes in six 16-byte stores instead of 24 scattered words,
// which matters when the output is mapped host memory.
constexpr int kStageWords = 24;

template <int C>
struct WarpBuf {
  uint32_t key[C];  // float bits of dist2 (non-negative: order == uint order)
  uint32_t id[C];   // sorted position of the photon
  uint32_t hist[256];
  uint32_t stack[kStack];
  uint32_t list[64];  // passing groups waiting to be scanned, in walk order
  uint32_t sel[32];   // entries of the critical bin of a selection
  uint32_t stat[8];   // per-warp counters, same order as pm_knn_stats
  float4 rec[2][3];   // radiance records of this query and the next (cp.async)
};

// 16-byte asynchronous copy global -> shared (the source may be mapped host
// memory), and the waits on it (per thread).
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

struct Levels {
  int2 oc[kMaxLevels];  // {offset of the level's boxes, boxes in the level}
};

enum {
  kStatQueries = 0, kStatCold, kStatCand, kStatLeaves, kStatNodes, kStatSelects, kStatWalks,
  kNumStats
};

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
// already filled (sum >= kk): returns the bin; *kk_in = rank inside it
// (1-based), *n_bin = entries in it.
__device__ __forceinline__ uint32_t hist_find(const uint32_t* hist, uint32_t kk,
                                              int lane, uint32_t* kk_in,
                                              uint32_t* n_bin) {
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
  uint32_t kk, nb;
  const int bin = (int)hist_find(s.hist, (uint32_t)k, lane, &kk, &nb);
  if (nb > 32) return false;
  int pos = 0;
  for (int base = 0; base < cnt; base += 32) {
    const int i = base + lane;
    bool in = false;
    if (i < cnt)
      in = min(255, __float2int_rz(__fmul_rz(__uint_as_float(s.key[i]), sc))) ==
           bin;
    const unsigned bal = __ballot_sync(kFull, in);
    if (in) s.sel[pos + __popc(bal & lt_mask(lane))] = (uint32_t)i;
    pos += __popc(bal);
  }
  __syncwarp();
  uint32_t kj = 0xffffffffu, oj = 0xffffffffu;
  if (lane < (int)nb) {
    const uint32_t i = s.sel[lane];
    kj = s.key[i];
    oj = orig_index(pos4, s.id[i]);
  }
  int rank = 0;
  for (int t = 0; t < (int)nb; ++t) {
    const uint32_t kt = __shfl_sync(kFull, kj, t);
    const uint32_t ot = __shfl_sync(kFull, oj, t);
    rank += (kt < kj) || (kt == kj && ot < oj);
  }
  const unsigned who = __ballot_sync(kFull, lane < (int)nb && rank == (int)kk - 1);
  const int wl = __ffs(who) - 1;
  kth_key = __shfl_sync(kFull, kj, wl);
  kth_oid = __shfl_sync(kFull, oj, wl);
  // a key held by one entry only: keep every entry with that key
  const unsigned same = __ballot_sync(kFull, lane < (int)nb && kj == kth_key);
  if (__popc(same) == 1) kth_oid = 0xffffffffu;
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
      const int o = dst + __popc(bal & lt_mask(lane));
      s.key[o] = key;
      s.id[o] = id;
    }
    dst += __popc(bal);
  }
  __syncwarp();
  return dst;
}

// Per-query state of the search.
struct Query {
  float x, y, z;
  float tau;  // every photon with dist2 <= tau is collected
  int cnt;    // entries in the warp buffer
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

// Appends photon i (position p) when valid and dist2 <= tau. When the
// buffer is nearly full, keeps the k best and lowers tau to the k-th.
template <int C, bool S>
__device__ __forceinline__ void offer(const MapDev& m, Query& q, WarpBuf<C>& s,
                                      int lane, const float4& p, int i,
                                      bool valid) {
  const float d2 = dist2_ref(q.x, q.y, q.z, p.x, p.y, p.z);
  const bool pass = valid && d2 <= q.tau;
  const unsigned bal = __ballot_sync(kFull, pass);
  if (pass) {
    const int o = q.cnt + __popc(bal & lt_mask(lane));
    s.key[o] = __float_as_uint(d2);
    s.id[o] = (uint32_t)i;
  }
  q.cnt += __popc(bal);
  if (q.cnt > C - 32 - kStageWords) {
    __syncwarp();
    const uint2 r = tighten<C, S>(m.pos4, &s, q.cnt, q.k, q.tau, lane);
    q.cnt = (int)r.x;
    q.tau = __uint_as_float(r.y);
  }
}

// Scans the photons of the ng groups listed in s.list: lane l handles
// photon (l & 7) of group 4r + (l >> 3) in round r; two rounds are loaded
// before either is used.
template <int C, bool S>
__device__ __forceinline__ void scan_groups(const MapDev& m, Query& q,
                                            WarpBuf<C>& s, int lane, int ng) {
  const int sub = lane >> 3, j = lane & 7;
  stat_add<S>(s, lane, kStatLeaves, (uint32_t)ng);
  for (int r = 0; r < ng; r += 8) {
    // invalid lanes read group 0 / photon 0 and offer nothing (no divergent
    // branch around the loads)
    const int ga = r + sub, gb = r + 4 + sub;
    const int ia = (int)s.list[ga < ng ? ga : 0] * kGroup + j;
    const int ib = (int)s.list[gb < ng ? gb : 0] * kGroup + j;
    const bool va = ga < ng && ia < m.n, vb = gb < ng && ib < m.n;
    const float4 pa = __ldg(m.pos4 + (va ? ia : 0));
    const float4 pb = __ldg(m.pos4 + (vb ? ib : 0));
    offer<C, S>(m, q, s, lane, pa, ia, va);
    if (r + 4 < ng) offer<C, S>(m, q, s, lane, pb, ib, vb);
  }
  __syncwarp();
}

// Scans the contiguous photon range [lo, hi), 32 photons per round.
template <int C, bool S>
__device__ __forceinline__ void scan_range(const MapDev& m, Query& q,
                                           WarpBuf<C>& s, int lane, int lo,
                                           int hi) {
  for (int b = lo; b < hi; b += 64) {
    const int ia = b + lane, ib = b + 32 + lane;
    const bool va = ia < hi, vb = ib < hi;
    const float4 pa = __ldg(m.pos4 + (va ? ia : lo));
    const float4 pb = __ldg(m.pos4 + (vb ? ib : lo));
    offer<C, S>(m, q, s, lane, pa, ia, va);
    if (b + 32 < hi) offer<C, S>(m, q, s, lane, pb, ib, vb);
  }
}

// Depth-first walk of the box tree collecting all photons with
// dist2 <= q.tau into the warp buffer. Passing 8-photon groups join a
// waiting list, scanned in full rounds of 8 as they accumulate and in full
// once the walk ends. Both go through one scan site: the scan inlines the
// candidate appends and the rare buffer cut, and a second copy of it made
// the kernel 1.9 % slower (3.387 against 3.324 ms on 1M primary-hit queries
// at k = 100; same scan order, same results).
template <int C, bool S>
__device__ __forceinline__ void collect(const MapDev& m, const Levels& L,
                                        Query& q, WarpBuf<C>& s, int lane) {
  q.cnt = 0;
  stat_add<S>(s, lane, kStatWalks, 1);
  if (m.nlevels == 1) {  // a single 8-photon group
    scan_range<C, S>(m, q, s, lane, 0, m.n);
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
    // lanes past the level's end read its first box and do not pass (no
    // divergent branch around the loads: 3 % of the kNN time)
    const int2 oc = L.oc[cl];
    const bool in = c < oc.y;
    const int jb = oc.x + (in ? c : 0);
    const float4 lo = __ldg(m.boxes + 2 * jb);
    const float4 hi = __ldg(m.boxes + 2 * jb + 1);
    const bool pass = in && box_dist2(q.x, q.y, q.z, lo, hi) <= q.tau;
    const unsigned bal = __ballot_sync(kFull, pass);
    const int off = __popc(bal & lt_mask(lane));
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
      scan_groups<C, S>(m, q, s, lane, take);
      const int rest = pending - take;
      uint32_t keep = 0;
      if (lane < rest) keep = s.list[take + lane];
      __syncwarp();
      if (lane < rest) s.list[lane] = keep;
      __syncwarp();
      pending = rest;
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
  scan_range<C, S>(m, q, s, lane, first * kGroup, min(n, (first + want) * kGroup));
  __syncwarp();
  if (q.cnt < k) return __int_as_float(0x7f800000);
  uint32_t mx = 0;
  for (int i = lane; i < q.cnt; i += 32) mx = max(mx, s.key[i]);
  mx = __reduce_max_sync(kFull, mx);  // every entry lies in [0, mx]
  uint32_t kth_key, kth_oid;
  select_kth<C, S>(pos4, s, q.cnt, k, __uint_as_float(mx), lane, kth_key, kth_oid);
  return __uint_as_float(kth_key);
}

// Answers queries [qb, qe) of a work item on map m, one at a time (one warp).
// r_hint: the last exact k-th distance this warp found (in/out).
// HIO (the single-map kernel, whose queries and output may be mapped host
// memory): radiance records are prefetched one query ahead with cp.async,
// and without `order` the radiance goes out in aligned groups of 8 queries.
// Without HIO (the batched kernel, device-resident slots) records are read
// with plain loads: measured on the 64-scene batch, the prefetch and the
// staging code together cost it 13 % through register allocation.
template <int C, int MODE, bool S, bool HIO>
__device__ __forceinline__ void knn_chunk(const MapDev& m, const Levels& L, WarpBuf<C>& s,
                                          int lane, const void* __restrict__ queries,
                                          int64_t qb, int64_t qe, int k, float n_emitted,
                                          const KnnOut& out, const uint32_t* __restrict__ order,
                                          int stride4, float& r_hint) {
  const float kInf = __int_as_float(0x7f800000);
  bool have_prev = false;
  float pqx = 0.f, pqy = 0.f, pqz = 0.f, pkth = 0.f;
  // HIO: the three float4 of a radiance record are staged in s.rec by lanes
  // 0-2 one query ahead, so the load (from device or mapped host memory)
  // overlaps the previous query's search.
  auto fetch = [&](int64_t qn, int b) {
    if (lane < 3) {
      const int64_t rn = order ? (int64_t)__ldg(order + qn) : qn;
      cp_async16(&s.rec[b][lane], reinterpret_cast<const float4*>(queries) + stride4 * rn + lane);
    }
    cp_async_commit();
  };
  int buf = 0;
  if (MODE != kModeKnn && HIO) fetch(qb, 0);
  for (int64_t qi = qb; qi < qe; ++qi, buf ^= 1) {
    Query q;
    q.k = k;
    q.cnt = 0;
    q.tau = kInf;
    const int64_t rec = (MODE != kModeKnn && order) ? (int64_t)__ldg(order + qi) : qi;
    if (MODE != kModeKnn && !HIO) {
      const float4 r0 = __ldg(reinterpret_cast<const float4*>(queries) + stride4 * rec);
      q.x = r0.x; q.y = r0.y; q.z = r0.z;
    } else if (MODE != kModeKnn) {
      cp_async_wait_all();
      __syncwarp();  // this record is visible; every lane is done with the other buffer
      if (qi + 1 < qe) fetch(qi + 1, buf ^ 1);
      // r0 = {pos, rho.r}; wo, ns and the other albedo channels are read
      // after the search
      const float4 r0 = s.rec[buf][0];
      q.x = r0.x; q.y = r0.y; q.z = r0.z;
    } else {
      const float* q3 = reinterpret_cast<const float*>(queries) + 3 * qi;
      q.x = __ldg(q3);
      q.y = __ldg(q3 + 1);
      q.z = __ldg(q3 + 2);
    }

    const bool bad = m.n == 0 || isnan(q.x) || isnan(q.y) || isnan(q.z);
    if (!bad) {
      bool warm = false, warm_guess = false;
      float tau_sure = 0.f;
      if (have_prev) {
        const float d2 = dist2_ref(q.x, q.y, q.z, pqx, pqy, pqz);
        if (d2 <= pkth) {
          const float rp = sqrtf(pkth);
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
      // more inside it make the result exact, otherwise the radius
      // doubles (twice), then the patch bound of cold_tau is used.
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
          q.tau = cold_tau<C, S>(m.pos4, m.boxes, m.n, m.nlevels, &L, q.x, q.y,
                                 q.z, k, &s, lane);
          need_cold = false;
          guess = false;
        }
        collect<C, S>(m, L, q, s, lane);
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

    // final selection
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
    const float maxd2 = kept > 0 ? __uint_as_float(kth_key) : 0.f;

    if (MODE == kModeAdjoint) {
      // d estimate / d throughput_i = f(wo, wi_i) / (n_emitted pi maxd2)
      // for the kept photons (integrator.h:141-150)
      const float4* q4 = reinterpret_cast<const float4*>(queries) + stride4 * rec;
      const float4 r0 = HIO ? s.rec[buf][0] : __ldg(q4);
      const float4 r1 = HIO ? s.rec[buf][1] : __ldg(q4 + 1);
      const float4 r2 = HIO ? s.rec[buf][2] : __ldg(q4 + 2);
      const float ax = out.adj_in[3 * rec], ay = out.adj_in[3 * rec + 1],
                  az = out.adj_in[3 * rec + 2];
      const int nk = all ? cnt : compact_kept(m.pos4, s, cnt, kth_key, kth_oid, lane);
      if (kept > 0 && (ax != 0.f || ay != 0.f || az != 0.f)) {
        const float cos_o = dot_ref(r1.x, r1.y, r1.z, r2.x, r2.y, r2.z);
        const float den = __fmul_rn(__fmul_rn(n_emitted, kPI), maxd2);
        const float cr = __fdiv_rn(__fmul_rn(ax, __fdiv_rn(r0.w, kPI)), den);
        const float cg = __fdiv_rn(__fmul_rn(ay, __fdiv_rn(r1.w, kPI)), den);
        const float cb = __fdiv_rn(__fmul_rn(az, __fdiv_rn(r2.w, kPI)), den);
        for (int i = lane; i < nk; i += 32) {
          const uint32_t id = s.id[i];
          const float4 t = __ldg(m.thr4 + id);
          const float2 w = __ldg(m.wi2 + id);
          const float cos_i = dot_ref(t.w, w.x, w.y, r2.x, r2.y, r2.z);
          if (!(cos_o < 0.f) && !(cos_i < 0.f))
            atomicAdd(out.photon_adj + orig_index(m.pos4, id), make_float4(cr, cg, cb, 0.f));
        }
      }
    } else if (MODE == kModeRadiance) {
      // r0 = {pos, rho.r}, r1 = {wo, rho.g}, r2 = {ns, rho.b}
      const float4* q4 = reinterpret_cast<const float4*>(queries) + stride4 * rec;
      const float4 r0 = HIO ? s.rec[buf][0] : __ldg(q4);
      const float4 r1 = HIO ? s.rec[buf][1] : __ldg(q4 + 1);
      const float4 r2 = HIO ? s.rec[buf][2] : __ldg(q4 + 2);
      const float cos_o = dot_ref(r1.x, r1.y, r1.z, r2.x, r2.y, r2.z);
      const float fr = __fdiv_rn(r0.w, kPI);
      const float fg = __fdiv_rn(r1.w, kPI);
      const float fb = __fdiv_rn(r2.w, kPI);
      // the kept entries, in the walk's order whatever the bound was, so
      // the sum below does not depend on the order queries are answered
      const int nk = all ? cnt : compact_kept(m.pos4, s, cnt, kth_key, kth_oid, lane);
      float lr = 0.f, lg = 0.f, lb = 0.f;
      for (int i = lane; i < nk; i += 32) {
        const uint32_t id = s.id[i];
        {
          const float4 t = __ldg(m.thr4 + id);
          const float2 w = __ldg(m.wi2 + id);
          const float cos_i = dot_ref(t.w, w.x, w.y, r2.x, r2.y, r2.z);
          // Lambert::evaluate returns 0 when either cosine is < 0
          if (!(cos_o < 0.f) && !(cos_i < 0.f)) {
            lr = __fadd_rn(lr, __fmul_rn(fr, t.x));
            lg = __fadd_rn(lg, __fmul_rn(fg, t.y));
            lb = __fadd_rn(lb, __fmul_rn(fb, t.z));
          }
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
        if (kept > 0) {
          const float den = __fmul_rn(__fmul_rn(n_emitted, kPI), maxd2);
          o3 = make_float3(__fdiv_rn(lr, den), __fdiv_rn(lg, den),
                           __fdiv_rn(lb, den));
        }
        if (HIO && !order) {
          float* r = reinterpret_cast<float*>(s.id + C - kStageWords) + 3 * (qi & 7);
          r[0] = o3.x; r[1] = o3.y; r[2] = o3.z;
        } else {
          out.rgb[3 * rec + 0] = o3.x;
          out.rgb[3 * rec + 1] = o3.y;
          out.rgb[3 * rec + 2] = o3.z;
        }
      }
      // work items without `order` start at multiples of 8: a group of 8 is
      // complete at qi % 8 == 7 or cut by the end of the queries
      if (HIO && !order && ((qi & 7) == 7 || qi + 1 == qe)) {
        __syncwarp();
        const int64_t g0 = qi & ~(int64_t)7;
        const int nf = 3 * (int)(qi + 1 - g0);
        float* dst = out.rgb + 3 * g0;
        const float* src = reinterpret_cast<const float*>(s.id + C - kStageWords);
        if (nf == kStageWords && (reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
          if (lane < kStageWords / 4)
            reinterpret_cast<float4*>(dst)[lane] = reinterpret_cast<const float4*>(src)[lane];
        } else if (lane < nf) {
          dst[lane] = src[lane];
        }
      }
    } else {
      int n2 = cnt;
      if (!all) n2 = compact_kept(m.pos4, s, cnt, kth_key, kth_oid, lane);
      for (int i = lane; i < n2; i += 32)
        s.id[i] = orig_index(m.pos4, s.id[i]);
      __syncwarp();
      int32_t* orow = out.idx + qi * (int64_t)k;
      for (int i = lane; i < n2; i += 32) {
        const uint32_t ki = s.key[i], oi = s.id[i];
        int rank = 0;
        for (int j = 0; j < n2; ++j) {
          const uint32_t kj = s.key[j], oj = s.id[j];
          rank += (kj > ki) || (kj == ki && oj > oi);
        }
        orow[rank] = (int32_t)oi;
      }
      for (int r = n2 + lane; r < k; r += 32) orow[r] = -1;
      if (lane == 0) {
        out.count[qi] = n2;
        out.maxd2[qi] = maxd2;
      }
    }
    __syncwarp();

    if (!bad && kept >= k) {
      have_prev = true;
      pqx = q.x; pqy = q.y; pqz = q.z;
      pkth = maxd2;
      r_hint = sqrtf(maxd2);
    } else {
      have_prev = false;
    }
  }
}

template <int C, int MODE, bool S>
__global__ void __launch_bounds__(256, 4)
    knn_kernel(MapDev m, const void* __restrict__ queries, int64_t nq, int k,
               float n_emitted, KnnOut out,
               unsigned long long* __restrict__ counter,
               const uint32_t* __restrict__ order, int stride4, int64_t head_items) {
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

    knn_chunk<C, MODE, S, true>(m, L, s, lane, queries, qb, qe, k, n_emitted, out, order, stride4,
                          r_hint);
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

template <int C, int MODE>
static cudaError_t launch_one(const MapDev& m, const void* queries,
                              int64_t nq, int k, float n_emitted, KnnOut out,
                              unsigned long long* counter, int num_sms,
                              cudaStream_t st, const uint32_t* order,
                              int stride4) {
  constexpr int kThreads = (C <= 512) ? 256 : 128;
  const size_t smem = (kThreads / 32) * sizeof(WarpBuf<C>);
  auto kern = out.stats ? knn_kernel<C, MODE, true> : knn_kernel<C, MODE, false>;
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
                                                 out, counter, order, stride4, head_items);
  return cudaGetLastError();
}

cudaError_t knn_launch(const MapDev& m, const void* queries, int64_t nq,
                       int k, int mode, float n_emitted, KnnOut out,
                       unsigned long long* counter, int num_sms,
                       cudaStream_t st, const uint32_t* order, int stride4) {
  if (nq <= 0) return cudaSuccess;
  if (mode == kModeAdjoint) {
    return k <= 224 ? launch_one<512, kModeAdjoint>(m, queries, nq, k, n_emitted, out, counter,
                                                   num_sms, st, order, stride4)
                    : launch_one<2048, kModeAdjoint>(m, queries, nq, k, n_emitted, out, counter,
                                                    num_sms, st, order, stride4);
  }
  if (k <= 224) {
    return mode == kModeRadiance
               ? launch_one<512, kModeRadiance>(m, queries, nq, k, n_emitted,
                                                out, counter, num_sms, st, order, stride4)
               : launch_one<512, kModeKnn>(m, queries, nq, k, n_emitted, out,
                                           counter, num_sms, st, order, stride4);
  }
  return mode == kModeRadiance
             ? launch_one<2048, kModeRadiance>(m, queries, nq, k, n_emitted,
                                               out, counter, num_sms, st, order, stride4)
             : launch_one<2048, kModeKnn>(m, queries, nq, k, n_emitted, out,
                                          counter, num_sms, st, order, stride4);
}

}  // namespace pm

// ------------------------------------------------------------ batched kNN
namespace pm {

// The radiance estimate of every query of every scene of a batch in one
// persistent launch. A work item is `chunk` consecutive queries of one
// scene (in the order of the sorted keys: scene, then Morton code); a warp
// takes items from `counter` until none are left, switching its copy of the
// photon map (map pointers, tree shape) when the scene changes.
template <int C>
__global__ void __launch_bounds__(256, 4)
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
    knn_chunk<C, kModeRadiance, false, false>(wmap[warp], wlev[warp], s, lane, slots, qb, qe, k,
                                       n_emitted, out, order, 4, r_hint);
  }
}

cudaError_t batch_knn_prepare(int warps, int buffer, int* blocks_per_sm) {
  if (warps < 1 || warps > 8) return cudaErrorInvalidValue;
  auto kern = buffer <= 512 ? knn_batch_kernel<512> : knn_batch_kernel<2048>;
  const size_t smem =
      (size_t)warps * (buffer <= 512 ? sizeof(WarpBuf<512>) : sizeof(WarpBuf<2048>));
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * warps, smem);
  if (e != cudaSuccess) return e;
  *blocks_per_sm = per_sm < 1 ? 1 : per_sm;
  return cudaSuccess;
}

cudaError_t batch_knn_launch(const BatchTables& t, const float4* slots, const uint32_t* order,
                             const int64_t* qoff, const int64_t* item_off, int64_t max_items,
                             float* res, int warps, int chunk, int buffer, int blocks_per_sm,
                             unsigned long long* counter, int num_sms, cudaStream_t st) {
  if (warps < 1 || warps > 8 || chunk < 1) return cudaErrorInvalidValue;
  const int threads = 32 * warps;
  auto kern = buffer <= 512 ? knn_batch_kernel<512> : knn_batch_kernel<2048>;
  const size_t smem =
      (size_t)warps * (buffer <= 512 ? sizeof(WarpBuf<512>) : sizeof(WarpBuf<2048>));
  int64_t blocks = (int64_t)num_sms * blocks_per_sm;
  const int64_t need = (max_items + warps - 1) / warps;
  if (blocks > need) blocks = need;
  if (blocks < 1) blocks = 1;
  cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st);
  if (e != cudaSuccess) return e;
  KnnOut out{};
  out.rgb = res;
  kern<<<(unsigned)blocks, threads, smem, st>>>(t, slots, order, qoff, item_off, chunk, out,
                                                counter);
  return cudaGetLastError();
}

}  // namespace pm
