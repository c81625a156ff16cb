// Allocation-free radiance estimate: pm_photonmap_radiance_noalloc.
//
// Some callers cannot call cudaMalloc: a plug-in whose host application
// owns all device memory and forbids allocations inside its callbacks, or a
// real-time loop that cannot afford the device-wide synchronisation
// cudaMalloc and cudaFree imply. This entry point allocates nothing: the
// caller passes the photons, the queries and the output in device memory,
// and every intermediate buffer (the sorted photon arrays, the box tree,
// the radix-sort buffers and the work counter) lives in one file-scope
// __device__ array sized for kNoAllocMaxPhotons photons (about 3.9 MiB,
// held by every GPU that loads the library until the process exits).
//
// Set-up: every call looks the array's device address up with
// cudaGetSymbolAddress in the CUDA context current at the call. The address
// belongs to that context (a plug-in may run in a context that is not the
// device's primary one, and cudaDeviceReset makes a new one), so it is not
// cached across calls; the lookup is cheap once the library's module is
// loaded in the context. The first call in a context loads that module and
// should come before any stream capture.
// Every call reuses the same array: calls that overlap on the GPU (on two
// streams, or from two host threads) race on it and must be serialised by
// the caller. Words that must start at zero (the box of the photon set, the
// work counter) are cleared by each call.
#include "../../include/pm_cuda.h"
#include "pm_photonmap.cuh"
#include "pm_sort.cuh"

namespace pm {

constexpr int kNoAllocMaxPhotons = PM_NOALLOC_MAX_PHOTONS;

constexpr size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// Boxes of the tree for n photons (level 0: groups of 8, then /32).
constexpr size_t noalloc_boxes(size_t n) {
  size_t cnt = (n + kGroup - 1) / kGroup, total = 0;
  while (true) {
    total += cnt;
    if (cnt <= 1) break;
    cnt = (cnt + 31) / 32;
  }
  return total;
}

constexpr size_t kNaPos4 = align256((size_t)kNoAllocMaxPhotons * 16);
constexpr size_t kNaThr4 = align256((size_t)kNoAllocMaxPhotons * 16);
constexpr size_t kNaWi2 = align256((size_t)kNoAllocMaxPhotons * 8);
constexpr size_t kNaBoxes = align256(noalloc_boxes(kNoAllocMaxPhotons) * 32);
// map_build_scratch_bytes(n): keys/values a/b, tile histogram, box words
constexpr size_t kNaSort =
    align256(4 * (size_t)kNoAllocMaxPhotons * 4 +
             sort_hist_words(kNoAllocMaxPhotons) * 4 + 64);
constexpr size_t kNaCounter = 256;
constexpr size_t kNaBytes = kNaPos4 + kNaThr4 + kNaWi2 + kNaBoxes + kNaSort + kNaCounter;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

// Device address of g_noalloc_scratch in the context current at the call.
static int noalloc_scratch(unsigned char** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p) {
    cudaGetLastError();
    return PM_ERR_CUDA;
  }
  *out = (unsigned char*)p;
  return PM_OK;
}

}  // namespace pm

using namespace pm;

extern "C" int pm_photonmap_radiance_noalloc(const float* d_photons,
                                             int64_t n_photons,
                                             const pm_radiance_query* d_queries,
                                             int64_t nq, int k,
                                             int64_t n_emitted, float* d_out_rgb,
                                             void* stream) {
  // sizes are checked before any CUDA call
  if (n_photons < 0 || n_photons > kNoAllocMaxPhotons) return PM_ERR_INVALID_ARGUMENT;
  if (k < 1 || k > PM_MAX_K || nq < 0) return PM_ERR_INVALID_ARGUMENT;
  if ((n_photons > 0 && !d_photons) || (nq > 0 && (!d_queries || !d_out_rgb)))
    return PM_ERR_INVALID_ARGUMENT;
  if (((uintptr_t)d_queries & 15) != 0) return PM_ERR_INVALID_ARGUMENT;
  if (nq == 0) return PM_OK;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) {
    cudaGetLastError();
    return PM_ERR_CUDA;
  }
  unsigned char* base = nullptr;
  int s = noalloc_scratch(&base);
  if (s != PM_OK) return s;
  int num_sms = 148;
  cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device);
  const cudaStream_t st = (cudaStream_t)stream;

  float4* pos4 = (float4*)base;
  float4* thr4 = (float4*)(base + kNaPos4);
  float2* wi2 = (float2*)(base + kNaPos4 + kNaThr4);
  float4* boxes = (float4*)(base + kNaPos4 + kNaThr4 + kNaWi2);
  void* sort = base + kNaPos4 + kNaThr4 + kNaWi2 + kNaBoxes;
  unsigned long long* counter =
      (unsigned long long*)(base + kNaPos4 + kNaThr4 + kNaWi2 + kNaBoxes + kNaSort);

  MapDev m;
  int lvl_off[kMaxLevels] = {}, lvl_cnt[kMaxLevels] = {};
  map_levels(n_photons, &m.nlevels, lvl_off, lvl_cnt);
  for (int i = 0; i < kMaxLevels; ++i) {
    m.lvl_off[i] = lvl_off[i];
    m.lvl_cnt[i] = lvl_cnt[i];
  }
  m.pos4 = pos4;
  m.thr4 = thr4;
  m.wi2 = wi2;
  m.boxes = boxes;
  m.n = (int)n_photons;
  map_build_launch(d_photons, (int)n_photons, pos4, thr4, wi2, boxes, lvl_off,
                   lvl_cnt, m.nlevels, sort, st);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return PM_ERR_CUDA;
  KnnOut o{};
  o.rgb = d_out_rgb;
  e = knn_launch(m, d_queries, nq, k, kModeRadiance, (float)n_emitted, o,
                 counter, num_sms, st);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return PM_ERR_CUDA;
  }
  return PM_OK;
}
