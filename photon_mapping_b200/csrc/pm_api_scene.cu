// C ABI of the scene, the batched intersection and photon tracing.
#include "../../include/pm_cuda.h"
#include "pm_api_internal.cuh"
#include "pm_scene_build.cuh"
#include "pm_trace.cuh"

#include <cstring>
#include <vector>

using namespace pm;

static_assert(sizeof(pm_material) == sizeof(Material), "material layout");
static_assert(sizeof(pm_hit) == 16, "hit layout");

#define CHECK_CTX(c) \
  do {               \
    if (!(c)) return PM_ERR_INVALID_ARGUMENT; \
  } while (0)

namespace pm {

// Ensures the context's error word exists (zeroed at creation).
static int ensure_err(pm_ctx* c) {
  if (c->dev_err.ptr) return PM_OK;
  int s = c->dev_err.ensure(64);
  if (s != PM_OK) return s;
  return cudaMemset(c->dev_err.ptr, 0, 64) == cudaSuccess ? PM_OK : PM_ERR_CUDA;
}

// Reads and clears the device error word; a set bit is a kernel-reported
// failure (bit 0: BVH traversal stack overflow).
int take_device_error(pm_ctx* c, const char* where) {
  int e = 0;
  cudaError_t ce = cudaMemcpyAsync(&e, c->dev_err.ptr, sizeof(int),
                                   cudaMemcpyDeviceToHost, c->stream);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(c->stream);
  if (ce != cudaSuccess) return cuda_status(c, ce, where);
  if (e) {
    cudaMemsetAsync(c->dev_err.ptr, 0, sizeof(int), c->stream);
    return set_err(c, PM_ERR_DEVICE_STATUS, "%s: device error bits 0x%x",
                   where, e);
  }
  return PM_OK;
}

}  // namespace pm

namespace pm {

int upload_scene(DevScene& sc, DevBuf& scratch, cudaStream_t st, const float* vertices,
                 const float* normals, const pm_material* materials, int64_t n,
                 const char** what) {
  sc.built = false;
  ++sc.generation;
  // area lights in face order (scene.h:41-51, :245-252)
  std::vector<int> lights;
  for (int64_t f = 0; f < n; ++f)
    if (materials[f].le[0] > 0.f || materials[f].le[1] > 0.f ||
        materials[f].le[2] > 0.f)
      lights.push_back((int)f);
  sc.n_faces = n;
  sc.n_lights = (int)lights.size();
  sc.has_specular = false;
  for (int a = 0; a < 3; ++a) {
    sc.lo[a] = n > 0 ? vertices[a] : 0.f;
    sc.hi[a] = sc.lo[a];
  }
  for (int64_t f = 0; f < n; ++f) {
    sc.has_specular |= materials[f].type != PM_LAMBERT;
    for (int k = 0; k < 3; ++k)
      for (int a = 0; a < 3; ++a) {
        const float x = vertices[9 * f + 3 * k + a];
        if (x < sc.lo[a]) sc.lo[a] = x;
        if (x > sc.hi[a]) sc.hi[a] = x;
      }
  }
  if (n == 0) {
    sc.built = true;
    return PM_OK;
  }
  const size_t nf = (size_t)n;
  int s;
  *what = "scene allocation";
  if ((s = sc.verts_in.ensure(nf * 9 * 4)) || (s = sc.nrms_in.ensure(nf * 9 * 4)) ||
      (s = sc.tri.ensure(nf * 3 * 16)) || (s = sc.nrm.ensure(nf * 3 * 16)) ||
      (s = sc.geo.ensure(nf * 16)) || (s = sc.mat.ensure(nf * sizeof(Material))) ||
      (s = sc.lights.ensure((lights.size() + 1) * 4)) ||
      (s = sc.mt.ensure(nf * 3 * 16)) ||
      (s = sc.nodes.ensure((nf > 1 ? nf - 1 : 1) * 4 * 16)) ||
      (s = scratch.ensure(scene_build_scratch_bytes((int)n))))
    return s;
  cudaError_t e;
  *what = "scene upload";
  if ((e = cudaMemcpyAsync(sc.verts_in.ptr, vertices, nf * 9 * 4,
                           cudaMemcpyHostToDevice, st)) ||
      (e = cudaMemcpyAsync(sc.nrms_in.ptr, normals, nf * 9 * 4,
                           cudaMemcpyHostToDevice, st)) ||
      (e = cudaMemcpyAsync(sc.mat.ptr, materials, nf * sizeof(Material),
                           cudaMemcpyHostToDevice, st)) ||
      (!lights.empty() &&
       (e = cudaMemcpyAsync(sc.lights.ptr, lights.data(), lights.size() * 4,
                            cudaMemcpyHostToDevice, st))))
    return e == cudaErrorMemoryAllocation ? PM_ERR_OUT_OF_MEMORY : PM_ERR_CUDA;
  *what = "scene build";
  if ((e = scene_build_launch((const float*)sc.verts_in.ptr, (const float*)sc.nrms_in.ptr,
                              (int)n, (float4*)sc.tri.ptr, (float4*)sc.nrm.ptr,
                              (float4*)sc.geo.ptr, (float4*)sc.mt.ptr, (float4*)sc.nodes.ptr,
                              scratch.ptr, st)) != cudaSuccess) {
    cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? PM_ERR_OUT_OF_MEMORY : PM_ERR_CUDA;
  }
  if ((e = cudaGetLastError()) != cudaSuccess) return PM_ERR_CUDA;
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return PM_ERR_CUDA;
  sc.built = true;
  return PM_OK;
}

int trace_map(pm_ctx* c, int map, uint64_t seed, int64_t n_emit, int max_depth,
              const Material* dmat, DevBuf* first, pm_trace_stats* stats) {
  c->diff.ready = false;  // the photon maps are about to change
  if (!c->scene.built) return set_err(c, PM_ERR_NOT_BUILT, "scene not built");
  if (n_emit > 0 && c->scene.n_lights == 0)
    return set_err(c, PM_ERR_INVALID_ARGUMENT, "scene has no area light");
  cudaStream_t st = c->stream;
  cudaError_t e;
  int s;
  if ((s = c->trace_misc.ensure(64)) != PM_OK)
    return set_err(c, s, "trace counters");
  unsigned long long* counter = (unsigned long long*)c->trace_misc.ptr;
  unsigned* status = (unsigned*)((char*)c->trace_misc.ptr + 16);
  // capacity guess: 4 stored photons per emitted one; retried when short
  unsigned long long cap = (unsigned long long)(n_emit > 0 ? n_emit : 1) * 4;
  unsigned long long stored = 0, hrays = 0;
  unsigned hstatus[2] = {0, 0};
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
  for (auto& x : ev)
    if ((e = cudaEventCreate(&x)) != cudaSuccess) {
      for (auto& y : ev)
        if (y) cudaEventDestroy(y);
      return cuda_status(c, e, "trace events");
    }
  struct EvGuard {
    cudaEvent_t* ev;
    ~EvGuard() {
      for (int i = 0; i < 3; ++i) cudaEventDestroy(ev[i]);
    }
  } guard{ev};
  const size_t ne = (size_t)(n_emit > 0 ? n_emit : 1);
  if ((s = c->trace_count.ensure(ne * 4)) != PM_OK)
    return set_err(c, s, "trace buffers (%lld photons)", (long long)n_emit);
  for (int attempt = 0; attempt < 2; ++attempt) {
    if ((s = c->trace_raw.ensure(cap * 36)) || (s = c->trace_keys.ensure(cap * 8)))
      return set_err(c, s, "trace buffers (%llu photons)", cap);
    if ((e = cudaMemsetAsync(c->trace_misc.ptr, 0, 64, st)) != cudaSuccess)
      return cuda_status(c, e, "trace counters");
    TraceArgs a{};
    a.seed = seed;
    a.n_emit = (int)n_emit;
    a.max_depth = max_depth;
    a.caustic = map == PM_MAP_CAUSTICS;
    a.out = (float*)c->trace_raw.ptr;
    a.keys = (unsigned long long*)c->trace_keys.ptr;
    a.store_count = (uint32_t*)c->trace_count.ptr;
    a.counter = counter;
    a.cap = cap;
    a.status = status;
    a.next = (unsigned long long*)((char*)c->trace_misc.ptr + 32);
    a.rays = (unsigned long long*)((char*)c->trace_misc.ptr + 48);
    a.dmat = dmat;
    cudaEventRecord(ev[0], st);
    trace_launch(c->scene_view(), a, st);
    cudaEventRecord(ev[1], st);
    if ((e = cudaGetLastError()) != cudaSuccess)
      return cuda_status(c, e, "trace launch");
    if ((e = cudaMemcpyAsync(&stored, counter, 8, cudaMemcpyDeviceToHost, st)) ||
        (e = cudaMemcpyAsync(hstatus, status, 8, cudaMemcpyDeviceToHost, st)) ||
        (e = cudaMemcpyAsync(&hrays, a.rays, 8, cudaMemcpyDeviceToHost, st)) ||
        (e = cudaStreamSynchronize(st)))
      return cuda_status(c, e, "trace");
    if ((s = take_device_error(c, "trace")) != PM_OK) return s;
    if (stored <= cap) break;
    cap = stored;  // the trace is deterministic: rerun with room for all
  }
  if (stored > (unsigned long long)0x7fffffff)
    return set_err(c, PM_ERR_INVALID_ARGUMENT, "%llu photons stored", stored);
  DevMap& dm = c->maps[map];
  const int n = (int)stored;
  DevBuf* fb = first ? first : &c->trace_first;
  if ((s = fb->ensure(ne * 4)) != PM_OK) return set_err(c, s, "photon offsets");
  if (n > 0) {
    if ((s = dm.aos.ensure((size_t)n * 36)) ||
        (s = c->scratch.ensure(order_scratch_bytes(n_emit))))
      return set_err(c, s, "photon order buffers");
    order_photons_launch((const unsigned long long*)c->trace_keys.ptr,
                         (const float*)c->trace_raw.ptr, n, (const uint32_t*)c->trace_count.ptr,
                         n_emit, (uint32_t*)fb->ptr, (float*)dm.aos.ptr, c->scratch.ptr,
                         (int*)c->dev_err.ptr, st);
    if ((e = cudaGetLastError()) != cudaSuccess)
      return cuda_status(c, e, "photon order");
  }
  if ((s = build_map(c, dm, (const float*)dm.aos.ptr, n, st)) != PM_OK) return s;
  cudaEventRecord(ev[2], st);
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess)
    return cuda_status(c, e, "photon map build");
  if ((s = take_device_error(c, "photon order")) != PM_OK) return s;
  c->map_emitted[map] = n_emit;
  if (stats) {
    stats->emitted = n_emit;
    stats->stored = (int64_t)stored;
    stats->nan_throughput = hstatus[0];
    stats->negative_throughput = hstatus[1];
    stats->rays = (int64_t)hrays;
    stats->trace_ms = 0.f;
    stats->build_ms = 0.f;
    cudaEventElapsedTime(&stats->trace_ms, ev[0], ev[1]);
    cudaEventElapsedTime(&stats->build_ms, ev[1], ev[2]);
  }
  return PM_OK;
}

}  // namespace pm

extern "C" {

int pm_scene_upload(pm_ctx* c, const float* vertices, const float* normals,
                    const pm_material* materials, int64_t n) {
  CHECK_CTX(c);
  if (n < 0 || n > (int64_t)0x3fffffff ||
      (n > 0 && (!vertices || !normals || !materials)))
    return set_err(c, PM_ERR_INVALID_ARGUMENT, "scene arrays / n_faces");
  for (int64_t f = 0; f < n; ++f)
    if (materials[f].type < PM_LAMBERT || materials[f].type > PM_GLASS)
      return set_err(c, PM_ERR_INVALID_ARGUMENT, "face %lld: material type %d",
                     (long long)f, materials[f].type);
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  int s;
  if ((s = ensure_err(c)) != PM_OK) return set_err(c, s, "error word");
  const char* what = "";
  if ((s = upload_scene(c->scene, c->scratch, c->stream, vertices, normals, materials, n,
                        &what)) != PM_OK) {
    if (s == PM_ERR_CUDA || s == PM_ERR_OUT_OF_MEMORY)
      cudaGetLastError();
    return set_err(c, s, "%s (%lld faces)", what, (long long)n);
  }
  return PM_OK;
}

int pm_scene_intersect(pm_ctx* c, const float* rays, int64_t n, pm_hit* out) {
  CHECK_CTX(c);
  if (n < 0 || (n > 0 && (!rays || !out)))
    return set_err(c, PM_ERR_INVALID_ARGUMENT, "rays / out");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  if (!c->scene.built) return set_err(c, PM_ERR_NOT_BUILT, "scene not built");
  if (n == 0) return PM_OK;
  int s;
  if ((s = c->q_in.ensure((size_t)n * 32)) || (s = c->q_out.ensure((size_t)n * 16)))
    return set_err(c, s, "ray buffers");
  cudaStream_t st = c->stream;
  cudaError_t e = cudaMemcpyAsync(c->q_in.ptr, rays, (size_t)n * 32,
                                  cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return cuda_status(c, e, "ray upload");
  intersect_launch(c->scene_view(), (const float4*)c->q_in.ptr, n,
                   (float4*)c->q_out.ptr, st);
  if ((e = cudaGetLastError()) != cudaSuccess)
    return cuda_status(c, e, "intersect launch");
  e = cudaMemcpyAsync(out, c->q_out.ptr, (size_t)n * 16,
                      cudaMemcpyDeviceToHost, st);
  if (e != cudaSuccess) return cuda_status(c, e, "hit download");
  return take_device_error(c, "intersect");
}

int pm_photons_trace(pm_ctx* c, int map, uint64_t seed, int64_t n_emit,
                     int max_depth, pm_trace_stats* stats) {
  CHECK_CTX(c);
  if (map != PM_MAP_GLOBAL && map != PM_MAP_CAUSTICS)
    return set_err(c, PM_ERR_INVALID_ARGUMENT, "map id %d", map);
  if (n_emit < 0 || n_emit > (int64_t)0x7fffffff || max_depth < 0 ||
      max_depth > 255)
    return set_err(c, PM_ERR_INVALID_ARGUMENT, "n_emit %lld / max_depth %d",
                   (long long)n_emit, max_depth);
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  return trace_map(c, map, seed, n_emit, max_depth, nullptr, nullptr, stats);
}

}  // extern "C"
