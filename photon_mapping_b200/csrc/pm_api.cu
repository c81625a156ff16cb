// C ABI of libpm_cuda.so: contexts, device buffers and the entry points
// declared in include/pm_cuda.h.
#include "../../include/pm_cuda.h"
#include "pm_api_internal.cuh"
#include "pm_hostio.cuh"

#include <cstdio>
#include <cstring>

using namespace pm;

// ------------------------------------------------------------ utilities

namespace pm {

int DevBuf::ensure(size_t n) {
  if (n <= bytes) return PM_OK;
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  bytes = 0;
  size_t want = n < 256 ? 256 : n;
  if (cudaMalloc(&ptr, want) != cudaSuccess) {
    cudaGetLastError();
    ptr = nullptr;
    return PM_ERR_OUT_OF_MEMORY;
  }
  bytes = want;
  return PM_OK;
}

void DevBuf::release() {
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  bytes = 0;
}

int set_err(pm_ctx* c, int status, const char* fmt, ...) {
  if (c) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    c->err = buf;
  }
  return status;
}

int cuda_status(pm_ctx* c, cudaError_t e, const char* where) {
  if (e == cudaSuccess) return PM_OK;
  cudaGetLastError();
  if (e == cudaErrorMemoryAllocation)
    return set_err(c, PM_ERR_OUT_OF_MEMORY, "%s: %s", where,
                   cudaGetErrorString(e));
  return set_err(c, PM_ERR_CUDA, "%s: %s", where, cudaGetErrorString(e));
}

MapDev map_view(const DevMap& dm) {
  MapDev m;
  m.pos4 = (const float4*)dm.pos4.ptr;
  m.thr4 = (const float4*)dm.thr4.ptr;
  m.wi2 = (const float2*)dm.wi2.ptr;
  m.boxes = (const float4*)dm.boxes.ptr;
  m.n = (int)dm.n;
  m.nlevels = dm.nlevels;
  for (int i = 0; i < kMaxLevels; ++i) {
    m.lvl_off[i] = i < dm.nlevels ? dm.lvl_off[i] : 0;
    m.lvl_cnt[i] = i < dm.nlevels ? dm.lvl_cnt[i] : 0;
  }
  return m;
}

// Builds map `dm` from `d_aos` (device, 9 floats per photon). When d_aos is
// not dm.aos it is copied there first.
int build_map(pm_ctx* c, DevMap& dm, const float* d_aos, int64_t n,
              cudaStream_t st) {
  if (n < 0 || n > (int64_t)0x7fffffff)
    return set_err(c, PM_ERR_INVALID_ARGUMENT, "photon count %lld",
                   (long long)n);
  int st_ok;
  dm.built = false;
  c->diff.ready = false;
  dm.n = n;
  int total = map_levels(n, &dm.nlevels, dm.lvl_off, dm.lvl_cnt);
  if (n == 0) {
    dm.built = true;
    return PM_OK;
  }
  if ((st_ok = dm.aos.ensure((size_t)n * 9 * sizeof(float))) ||
      (st_ok = dm.pos4.ensure((size_t)n * sizeof(float4))) ||
      (st_ok = dm.thr4.ensure((size_t)n * sizeof(float4))) ||
      (st_ok = dm.wi2.ensure((size_t)n * sizeof(float2))) ||
      (st_ok = dm.boxes.ensure((size_t)total * 2 * sizeof(float4))) ||
      (st_ok = c->scratch.ensure(map_build_scratch_bytes(n))))
    return set_err(c, st_ok, "photon map allocation (%lld photons)",
                   (long long)n);
  if (d_aos != (const float*)dm.aos.ptr) {
    cudaError_t e = cudaMemcpyAsync(dm.aos.ptr, d_aos,
                                    (size_t)n * 9 * sizeof(float),
                                    cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return cuda_status(c, e, "photon copy");
  }
  map_build_launch((const float*)dm.aos.ptr, (int)n, (float4*)dm.pos4.ptr,
                   (float4*)dm.thr4.ptr, (float2*)dm.wi2.ptr,
                   (float4*)dm.boxes.ptr, dm.lvl_off, dm.lvl_cnt, dm.nlevels,
                   c->scratch.ptr, st);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_status(c, e, "photon map build");
  dm.built = true;
  return PM_OK;
}

}  // namespace pm

// Streams passed through the C ABI follow CUDA's convention: NULL is the
// legacy default stream.
static inline cudaStream_t as_stream(void* s) { return (cudaStream_t)s; }

#define PM_CHECK_CTX(c)                                   \
  do {                                                    \
    if (!(c)) return PM_ERR_INVALID_ARGUMENT;             \
  } while (0)

#define PM_CHECK_MAP(c, map)                                               \
  do {                                                                     \
    if ((map) != PM_MAP_GLOBAL && (map) != PM_MAP_CAUSTICS)                \
      return set_err((c), PM_ERR_INVALID_ARGUMENT, "map id %d", (int)(map)); \
  } while (0)

// ----------------------------------------------------------------- C ABI

extern "C" {

const char* pm_status_string(int status) {
  switch (status) {
    case PM_OK: return "PM_OK";
    case PM_ERR_INVALID_ARGUMENT: return "PM_ERR_INVALID_ARGUMENT";
    case PM_ERR_CUDA: return "PM_ERR_CUDA";
    case PM_ERR_OUT_OF_MEMORY: return "PM_ERR_OUT_OF_MEMORY";
    case PM_ERR_NOT_BUILT: return "PM_ERR_NOT_BUILT";
    case PM_ERR_DEVICE_STATUS: return "PM_ERR_DEVICE_STATUS";
    default: return "PM_ERR_UNKNOWN";
  }
}

int pm_ctx_create(int device, pm_ctx** out) {
  if (!out) return PM_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return PM_ERR_CUDA;
  }
  if (device < 0 || device >= ndev) return PM_ERR_INVALID_ARGUMENT;
  if ((e = cudaSetDevice(device)) != cudaSuccess) return PM_ERR_CUDA;
  pm_ctx* c = new pm_ctx();
  c->device = device;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) !=
      cudaSuccess) {
    delete c;
    return PM_ERR_CUDA;
  }
  cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
  if (c->counter.ensure(pm::kCounterRing * sizeof(unsigned long long)) != PM_OK) {
    cudaStreamDestroy(c->stream);
    delete c;
    return PM_ERR_OUT_OF_MEMORY;
  }
  *out = c;
  return PM_OK;
}

int pm_ctx_destroy(pm_ctx* c) {
  PM_CHECK_CTX(c);
  {
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    c->release_all();
    cudaStreamDestroy(c->stream);
  }
  delete c;
  return PM_OK;
}

int pm_ctx_synchronize(pm_ctx* c) {
  PM_CHECK_CTX(c);
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  return cuda_status(c, cudaStreamSynchronize(c->stream), "synchronize");
}

int pm_ctx_set_stats(pm_ctx* c, int enable) {
  PM_CHECK_CTX(c);
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  if (enable && !c->stats.ptr) {
    int s = c->stats.ensure(8 * sizeof(unsigned long long));
    if (s != PM_OK) return set_err(c, s, "stats counters");
    cudaError_t e = cudaMemsetAsync(c->stats.ptr, 0, c->stats.bytes, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_status(c, e, "stats counters");
  }
  c->stats_on = enable != 0;
  return PM_OK;
}

int pm_ctx_get_stats(pm_ctx* c, pm_knn_stats* out, int reset) {
  PM_CHECK_CTX(c);
  if (!out) return PM_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  memset(out, 0, sizeof(*out));
  if (!c->stats.ptr) return PM_OK;
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess)
    e = cudaMemcpy(out, c->stats.ptr, sizeof(*out), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && reset) e = cudaMemset(c->stats.ptr, 0, c->stats.bytes);
  return cuda_status(c, e, "stats read");
}

const char* pm_ctx_last_error(const pm_ctx* c) {
  return c ? c->err.c_str() : "null context";
}

int pm_photonmap_build(pm_ctx* c, int map, const float* photons, int64_t n) {
  PM_CHECK_CTX(c);
  PM_CHECK_MAP(c, map);
  if (n < 0 || (n > 0 && !photons))
    return set_err(c, PM_ERR_INVALID_ARGUMENT, "photons/n");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  DevMap& dm = c->maps[map];
  int s;
  if (n > 0) {
    if ((s = dm.aos.ensure((size_t)n * 9 * sizeof(float))) != PM_OK)
      return set_err(c, s, "photon upload (%lld photons)", (long long)n);
    cudaError_t e = cudaMemcpyAsync(dm.aos.ptr, photons,
                                    (size_t)n * 9 * sizeof(float),
                                    cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return cuda_status(c, e, "photon upload");
  }
  if ((s = build_map(c, dm, (const float*)dm.aos.ptr, n, c->stream)) != PM_OK)
    return s;
  return cuda_status(c, cudaStreamSynchronize(c->stream), "photon map build");
}

int pm_photonmap_build_device(pm_ctx* c, int map, const void* d_photons,
                              int64_t n, void* stream) {
  PM_CHECK_CTX(c);
  PM_CHECK_MAP(c, map);
  if (n < 0 || (n > 0 && !d_photons))
    return set_err(c, PM_ERR_INVALID_ARGUMENT, "photons/n");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  return build_map(c, c->maps[map], (const float*)d_photons, n,
                   as_stream(stream));
}

int pm_photonmap_set_emitted(pm_ctx* c, int map, int64_t n_emitted) {
  PM_CHECK_CTX(c);
  PM_CHECK_MAP(c, map);
  if (n_emitted < 0)
    return set_err(c, PM_ERR_INVALID_ARGUMENT, "n_emitted %lld", (long long)n_emitted);
  std::lock_guard<std::mutex> lk(c->mu);
  c->map_emitted[map] = n_emitted;
  return PM_OK;
}

int pm_photonmap_size(pm_ctx* c, int map, int64_t* n) {
  PM_CHECK_CTX(c);
  PM_CHECK_MAP(c, map);
  if (!n) return PM_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(c->mu);
  *n = c->maps[map].built ? c->maps[map].n : 0;
  return PM_OK;
}

int pm_photonmap_get_photons(pm_ctx* c, int map, int64_t first, int64_t count,
                             float* out) {
  PM_CHECK_CTX(c);
  PM_CHECK_MAP(c, map);
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  DevMap& dm = c->maps[map];
  if (!dm.built) return set_err(c, PM_ERR_NOT_BUILT, "map %d not built", map);
  if (first < 0 || count < 0 || first + count > dm.n || (count > 0 && !out))
    return set_err(c, PM_ERR_INVALID_ARGUMENT, "range [%lld, %lld) of %lld",
                   (long long)first, (long long)(first + count),
                   (long long)dm.n);
  if (count == 0) return PM_OK;
  cudaError_t e = cudaMemcpyAsync(out, (const float*)dm.aos.ptr + 9 * first,
                                  (size_t)count * 9 * sizeof(float),
                                  cudaMemcpyDeviceToHost, c->stream);
  if (e != cudaSuccess) return cuda_status(c, e, "photon download");
  return cuda_status(c, cudaStreamSynchronize(c->stream), "photon download");
}

int pm_photonmap_knn(pm_ctx* c, int map, const float* queries, int64_t nq,
                     int k, int32_t* out_idx, int32_t* out_count,
                     float* out_maxdist2) {
  PM_CHECK_CTX(c);
  PM_CHECK_MAP(c, map);
  if (k < 1 || k > PM_MAX_K)
    return set_err(c, PM_ERR_INVALID_ARGUMENT, "k=%d not in [1, %d]", k,
                   PM_MAX_K);
  if (nq < 0 || (nq > 0 && (!queries || !out_idx || !out_count ||
                            !out_maxdist2)))
    return set_err(c, PM_ERR_INVALID_ARGUMENT, "queries/outputs");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  DevMap& dm = c->maps[map];
  if (!dm.built) return set_err(c, PM_ERR_NOT_BUILT, "map %d not built", map);
  if (nq == 0) return PM_OK;
  const size_t qb = (size_t)nq * 3 * sizeof(float);
  const size_t ib = (size_t)nq * k * sizeof(int32_t);
  const size_t cb = (size_t)nq * sizeof(int32_t);
  const size_t mb = (size_t)nq * sizeof(float);
  int s;
  if ((s = c->q_in.ensure(qb)) || (s = c->q_out.ensure(ib + cb + mb)))
    return set_err(c, s, "query buffers");
  cudaStream_t st = c->stream;
  cudaError_t e = copy_in(c->q_in.ptr, queries, qb, c->num_sms, st);
  if (e != cudaSuccess) return cuda_status(c, e, "query upload");
  // mapped output buffers are written by the kernel itself
  int32_t* m_idx = (int32_t*)mapped_host(out_idx);
  int32_t* m_cnt = (int32_t*)mapped_host(out_count);
  float* m_md2 = (float*)mapped_host(out_maxdist2);
  KnnOut o{};
  o.stats = c->stats_ptr();
  o.idx = m_idx ? m_idx : (int32_t*)c->q_out.ptr;
  o.count = m_cnt ? m_cnt : (int32_t*)((char*)c->q_out.ptr + ib);
  o.maxd2 = m_md2 ? m_md2 : (float*)((char*)c->q_out.ptr + ib + cb);
  e = knn_launch(map_view(dm), c->q_in.ptr, nq, k, kModeKnn, 0.f, o,
                 c->next_counter(), c->num_sms, st);
  if (e != cudaSuccess) return cuda_status(c, e, "knn launch");
  if ((!m_idx && (e = cudaMemcpyAsync(out_idx, o.idx, ib, cudaMemcpyDeviceToHost, st))) ||
      (!m_cnt && (e = cudaMemcpyAsync(out_count, o.count, cb, cudaMemcpyDeviceToHost, st))) ||
      (!m_md2 && (e = cudaMemcpyAsync(out_maxdist2, o.maxd2, mb, cudaMemcpyDeviceToHost, st))))
    return cuda_status(c, e, "knn download");
  return cuda_status(c, cudaStreamSynchronize(st), "knn");
}

int pm_photonmap_radiance(pm_ctx* c, int map, const pm_radiance_query* q,
                          int64_t nq, int k, int64_t n_emitted,
                          float* out_rgb) {
  PM_CHECK_CTX(c);
  PM_CHECK_MAP(c, map);
  if (k < 1 || k > PM_MAX_K)
    return set_err(c, PM_ERR_INVALID_ARGUMENT, "k=%d not in [1, %d]", k,
                   PM_MAX_K);
  if (nq < 0 || (nq > 0 && (!q || !out_rgb)))
    return set_err(c, PM_ERR_INVALID_ARGUMENT, "queries/outputs");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  DevMap& dm = c->maps[map];
  if (!dm.built) return set_err(c, PM_ERR_NOT_BUILT, "map %d not built", map);
  if (nq == 0) return PM_OK;
  const size_t qb = (size_t)nq * sizeof(pm_radiance_query);
  const size_t ob = (size_t)nq * 3 * sizeof(float);
  cudaStream_t st = c->stream;
  cudaError_t e;
  // A mapped, 16-byte aligned query buffer is read in place by the kernel
  // (each record is fetched one query ahead, so the host-memory latency
  // overlaps the previous query's search); others are copied first.
  const void* d_q = mapped_host(q);
  if (d_q && ((uintptr_t)d_q & 15) != 0) d_q = nullptr;
  // a mapped output buffer is written by the kernel itself
  float* mapped_out = (float*)mapped_host(out_rgb);
  int s = PM_OK;
  if ((!d_q && (s = c->q_in.ensure(qb))) || (!mapped_out && (s = c->q_out.ensure(ob))))
    return set_err(c, s, "query buffers");
  if (!d_q) {
    e = copy_in(c->q_in.ptr, q, qb, c->num_sms, st);
    if (e != cudaSuccess) return cuda_status(c, e, "query upload");
    d_q = c->q_in.ptr;
  }
  KnnOut o{};
  o.stats = c->stats_ptr();
  o.rgb = mapped_out ? mapped_out : (float*)c->q_out.ptr;
  e = knn_launch(map_view(dm), d_q, nq, k, kModeRadiance,
                 (float)n_emitted, o, c->next_counter(), c->num_sms, st);
  if (e != cudaSuccess) return cuda_status(c, e, "radiance launch");
  if (!mapped_out) {
    e = cudaMemcpyAsync(out_rgb, o.rgb, ob, cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return cuda_status(c, e, "radiance download");
  }
  return cuda_status(c, cudaStreamSynchronize(st), "radiance");
}

int pm_photonmap_radiance_device(pm_ctx* c, int map, const void* d_queries,
                                 int64_t nq, int k, int64_t n_emitted,
                                 void* d_out_rgb, void* stream) {
  PM_CHECK_CTX(c);
  PM_CHECK_MAP(c, map);
  if (k < 1 || k > PM_MAX_K)
    return set_err(c, PM_ERR_INVALID_ARGUMENT, "k=%d not in [1, %d]", k,
                   PM_MAX_K);
  if (nq < 0 || (nq > 0 && (!d_queries || !d_out_rgb)))
    return set_err(c, PM_ERR_INVALID_ARGUMENT, "queries/outputs");
  if (((uintptr_t)d_queries & 15) != 0)
    return set_err(c, PM_ERR_INVALID_ARGUMENT,
                   "queries must be 16-byte aligned");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  DevMap& dm = c->maps[map];
  if (!dm.built) return set_err(c, PM_ERR_NOT_BUILT, "map %d not built", map);
  KnnOut o{};
  o.stats = c->stats_ptr();
  o.rgb = (float*)d_out_rgb;
  cudaError_t e = knn_launch(map_view(dm), d_queries, nq, k, kModeRadiance,
                             (float)n_emitted, o, c->next_counter(),
                             c->num_sms, as_stream(stream));
  return cuda_status(c, e, "radiance launch");
}

}  // extern "C"
