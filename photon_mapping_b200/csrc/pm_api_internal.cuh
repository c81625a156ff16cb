// Internal state behind the C ABI: the context, its device buffers and the
// device photon maps.
#pragma once

#include <cstdarg>
#include <mutex>
#include <string>

#include "pm_photonmap.cuh"

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
  pm::DevBuf scratch;  // map build scratch
  pm::DevBuf q_in, q_out;  // staging of the host-pointer entry points
  pm::DevBuf counter;      // kCounterRing work counters
  unsigned counter_next = 0;
  pm::DevBuf stats;        // pm_knn_stats counters (device)
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
  }
};

namespace pm {
int set_err(pm_ctx* c, int status, const char* fmt, ...);
int cuda_status(pm_ctx* c, cudaError_t e, const char* where);
MapDev map_view(const DevMap& dm);
int build_map(pm_ctx* c, DevMap& dm, const float* d_aos, int64_t n,
              cudaStream_t st);
}  // namespace pm
