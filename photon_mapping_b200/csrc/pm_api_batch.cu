// C ABI of the batched render: pm_batch_create / _render / _autotune /
// _image / _counts / _destroy.
//
// Planning (pm_batch_create) uploads every scene and runs the step once with
// host read-backs: photons stored per scene (the trace is deterministic, so
// a short capacity is rerun exactly), then the number of queries. From then
// on every size is fixed, so the step needs no host synchronisation and is
// captured in a CUDA graph as it is; each step checks its counts against the
// plan afterwards.
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/pm_cuda.h"
#include "pm_api_internal.cuh"
#include "pm_batch.cuh"
#include "pm_scene_build.cuh"
#include "pm_sort.cuh"
#include "pm_trace.cuh"

using namespace pm;

static_assert(PM_BATCH_MAX_SCENES == kMaxBatchScenes, "batch limit");

struct pm_batch {
  std::mutex mu;  // calls on one batch are serialised
  int device = 0, num_sms = 148;
  cudaStream_t st = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::string err;
  int n = 0;
  std::vector<DevScene> scenes;
  std::vector<pm_batch_scene> desc;
  std::vector<int> qps;
  std::vector<int64_t> cap, stored, queries;
  std::vector<int64_t> emit_off, pix_off, slot_off, sample_off, cap_off;
  DevBuf raw, keys, counters, status, dropped, rng, slots, srec, res, images;
  DevBuf qka, qkb, qva, qvb, qhist, qcount, qstart, qoff, item_off, knn_counter;
  DevBuf table, offs, err_word, scene_scratch;
  // the photon maps of all scenes, built together (batch_maps_launch)
  struct Shape {
    int nlevels = 0;
    int lvl_off[kMaxLevels] = {};
    int lvl_cnt[kMaxLevels] = {};
  };
  std::vector<Shape> shape;
  std::vector<int64_t> box_base;
  DevBuf m_pos4, m_thr4, m_wi2, m_boxes, m_keys_b, m_va, m_vb, m_hist, m_bb, m_tab, m_lvl;
  DevBuf m_order, m_count, m_first, m_sums;
  BatchMapBuild mb{};
  int64_t total_emit = 0, total_pix = 0, total_slots = 0, total_samples = 0, nq = 0;
  int max_k = 1;
  pm_batch_tuning tune{8, 32, 512, 64, 128, 0};
  int knn_per_sm = 1;
  bool sorted_in_b = false;  // where the last query sort left its output
  cudaGraphExec_t exec = nullptr;
  BatchTables tables{};

  ~pm_batch() {
    if (exec) cudaGraphExecDestroy(exec);
    for (auto& s : scenes) s.release();
    DevBuf* bufs[] = {&raw,    &keys,    &counters, &status, &dropped,  &rng,
                      &slots,  &srec,    &res,      &images, &qka,      &qkb,
                      &qva,    &qvb,     &qhist,    &qcount, &qstart,   &qoff,
                      &item_off, &knn_counter, &table, &offs, &err_word, &scene_scratch,
                      &m_pos4, &m_thr4,  &m_wi2,    &m_boxes, &m_keys_b, &m_va,
                      &m_vb,   &m_hist,  &m_bb,     &m_tab,  &m_lvl,    &m_order,
                      &m_count, &m_first, &m_sums};
    for (DevBuf* b : bufs) b->release();
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (st) cudaStreamDestroy(st);
  }
};

namespace {

int berr(pm_batch* b, int status, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  b->err = buf;
  return status;
}

int bcuda(pm_batch* b, cudaError_t e, const char* where) {
  if (e == cudaSuccess) return PM_OK;
  cudaGetLastError();
  return berr(b, e == cudaErrorMemoryAllocation ? PM_ERR_OUT_OF_MEMORY : PM_ERR_CUDA, "%s: %s",
              where, cudaGetErrorString(e));
}

int key_bits(int n_scenes) {
  int b = 0;
  while ((1 << b) < n_scenes) ++b;
  return 30 + b;
}

bool tuning_ok(const pm_batch* b, const pm_batch_tuning& t) {
  return t.knn_warps >= 1 && t.knn_warps <= 8 && t.knn_chunk >= 1 && t.knn_chunk <= 1024 &&
         (t.knn_buffer == 2048 || (t.knn_buffer == 512 && b->max_k <= 224)) &&
         (t.bvh_stack == 16 || t.bvh_stack == 32 || t.bvh_stack == 64) && t.block >= 64 && t.block <= 256 &&
         t.block % 32 == 0;
}

// Writes the per-scene table (pointers into the batch's buffers, maps as
// built) and the prefix arrays to the device.
int upload_tables(pm_batch* b) {
  const int n = b->n;
  std::vector<BatchScene> t((size_t)n);
  int* errw = (int*)b->err_word.ptr;
  for (int s = 0; s < n; ++s) {
    const pm_batch_scene& d = b->desc[s];
    BatchScene& x = t[s];
    memset(&x, 0, sizeof(x));
    x.sc = scene_view(b->scenes[s], errw);
    RenderArgs& a = x.ra;
    a.cam_pos = v3(d.camera.position[0], d.camera.position[1], d.camera.position[2]);
    a.cam_fwd = v3(d.camera.forward[0], d.camera.forward[1], d.camera.forward[2]);
    a.cam_right = v3(d.camera.right[0], d.camera.right[1], d.camera.right[2]);
    a.cam_up = v3(d.camera.up[0], d.camera.up[1], d.camera.up[2]);
    a.focal = d.camera.focal_length;
    a.width = d.width;
    a.height = d.height;
    a.batch = d.spp;
    a.q_per_sample = b->qps[s];
    a.fg_depth = 0;
    a.max_depth = d.max_depth;
    a.n_gather = 1;
    a.inv_gather = v3(1.f, 1.f, 1.f);
    a.rng_state = (unsigned long long*)b->rng.ptr + b->pix_off[s];
    a.slots = (float4*)b->slots.ptr + 4 * b->slot_off[s];
    a.sample_rec = (float4*)b->srec.ptr + b->sample_off[s];
    a.in_rays = nullptr;
    a.err = errw;
    MapDev& mv = x.map;
    const pm_batch::Shape& sh = b->shape.empty() ? pm_batch::Shape{} : b->shape[s];
    mv.pos4 = (const float4*)b->m_pos4.ptr + b->cap_off[s];
    mv.thr4 = (const float4*)b->m_thr4.ptr + b->cap_off[s];
    mv.wi2 = (const float2*)b->m_wi2.ptr + b->cap_off[s];
    mv.boxes = b->box_base.empty() ? nullptr : (const float4*)b->m_boxes.ptr + 2 * b->box_base[s];
    mv.n = b->shape.empty() ? 0 : (int)b->stored[s];
    mv.nlevels = sh.nlevels;
    for (int l = 0; l < kMaxLevels; ++l) {
      mv.lvl_off[l] = l < sh.nlevels ? sh.lvl_off[l] : 0;
      mv.lvl_cnt[l] = l < sh.nlevels ? sh.lvl_cnt[l] : 0;
    }
    x.k = d.k;
    x.n_emitted = (float)d.n_photons;
    const DevScene& sc = b->scenes[s];
    x.qlo = make_float3(sc.lo[0], sc.lo[1], sc.lo[2]);
    x.qinv = make_float3(sc.hi[0] > sc.lo[0] ? 1.0f / (sc.hi[0] - sc.lo[0]) : 0.f,
                         sc.hi[1] > sc.lo[1] ? 1.0f / (sc.hi[1] - sc.lo[1]) : 0.f,
                         sc.hi[2] > sc.lo[2] ? 1.0f / (sc.hi[2] - sc.lo[2]) : 0.f);
    TraceArgs& ta = x.ta;
    ta = TraceArgs{};
    ta.seed = d.seed;
    ta.n_emit = (int)d.n_photons;
    ta.max_depth = d.max_depth;
    ta.caustic = 0;
    ta.out = (float*)b->raw.ptr + 9 * b->cap_off[s];
    ta.keys = (unsigned long long*)b->keys.ptr + b->cap_off[s];
    ta.store_count = (uint32_t*)b->m_count.ptr;  // by the batch's work index
    ta.counter = (unsigned long long*)b->counters.ptr + s;
    ta.cap = (unsigned long long)b->cap[s];
    ta.status = (unsigned*)b->status.ptr;
    x.res = (float*)b->res.ptr + 3 * b->slot_off[s];
    x.accum = nullptr;
    x.image = (float*)b->images.ptr + 3 * b->pix_off[s];
  }
  int s;
  if ((s = b->table.ensure(sizeof(BatchScene) * (size_t)n)) ||
      (s = b->offs.ensure(sizeof(int64_t) * 3 * (size_t)(n + 1))))
    return berr(b, s, "batch tables");
  std::vector<int64_t> o;
  o.insert(o.end(), b->emit_off.begin(), b->emit_off.end());
  o.insert(o.end(), b->pix_off.begin(), b->pix_off.end());
  o.insert(o.end(), b->slot_off.begin(), b->slot_off.end());
  cudaError_t e;
  if ((e = cudaMemcpyAsync(b->table.ptr, t.data(), sizeof(BatchScene) * (size_t)n,
                           cudaMemcpyHostToDevice, b->st)) ||
      (e = cudaMemcpyAsync(b->offs.ptr, o.data(), o.size() * sizeof(int64_t),
                           cudaMemcpyHostToDevice, b->st)) ||
      (e = cudaStreamSynchronize(b->st)))
    return bcuda(b, e, "batch tables");
  BatchTables& bt = b->tables;
  bt.scenes = (const BatchScene*)b->table.ptr;
  bt.emit_off = (const int64_t*)b->offs.ptr;
  bt.pix_off = bt.emit_off + (n + 1);
  bt.slot_off = bt.pix_off + (n + 1);
  bt.slots = (const float4*)b->slots.ptr;
  bt.n_scenes = n;
  bt.status = (unsigned*)b->status.ptr;
  bt.next_photon = (unsigned long long*)((char*)b->status.ptr + 16);
  bt.dropped = (unsigned long long*)b->dropped.ptr;
  return PM_OK;
}

// Trace buffers for the capacities in b->cap.
int size_trace(pm_batch* b) {
  const int n = b->n;
  b->cap_off.assign((size_t)n + 1, 0);
  for (int s = 0; s < n; ++s) b->cap_off[s + 1] = b->cap_off[s] + b->cap[s];
  const size_t tot = (size_t)std::max<int64_t>(b->cap_off[n], 1);
  int s;
  if ((s = b->raw.ensure(tot * 36)) || (s = b->keys.ensure(tot * 8)))
    return berr(b, s, "trace buffers (%zu photons)", tot);
  return PM_OK;
}

// Enqueues the trace (counters reset first).
void enqueue_trace(pm_batch* b, int block, int stack) {
  cudaMemsetAsync(b->counters.ptr, 0, 8 * (size_t)b->n, b->st);
  cudaMemsetAsync(b->status.ptr, 0, 8, b->st);
  batch_trace_launch(b->tables, b->total_emit, block, stack, b->st);
}

// Orders every scene's photons and builds every scene's map, all scenes
// in each launch.
void enqueue_maps(pm_batch* b) { batch_maps_launch(b->mb, b->st); }

int bits_for(int64_t v) {  // smallest b with 2^b >= v
  int r = 0;
  while (r < 62 && ((int64_t)1 << r) < v) ++r;
  return r;
}

// After the stored counts are known (cap = stored): the map shapes, their
// device tables and buffers, and the build's arguments.
int plan_maps(pm_batch* b) {
  const int n = b->n;
  const int64_t total = b->cap_off[n];
  if (total > 0x7fffffffLL)
    return berr(b, PM_ERR_INVALID_ARGUMENT, "%lld photons stored in the batch (at most 2^31 - 1)",
                (long long)total);
  b->shape.assign((size_t)n, pm_batch::Shape{});
  b->box_base.assign((size_t)n + 1, 0);
  std::vector<int64_t> group_off((size_t)n + 1, 0), level_off((size_t)kMaxLevels * (n + 1), 0);
  std::vector<int> lvl((size_t)n * 2 * kMaxLevels, 0);
  int max_levels = 0;
  for (int s = 0; s < n; ++s) {
    pm_batch::Shape& sh = b->shape[s];
    const int boxes = map_levels(b->stored[s], &sh.nlevels, sh.lvl_off, sh.lvl_cnt);
    b->box_base[s + 1] = b->box_base[s] + boxes;
    group_off[s + 1] = group_off[s] + (sh.nlevels > 0 ? sh.lvl_cnt[0] : 0);
    for (int l = 0; l < kMaxLevels; ++l) {
      const int cnt = l < sh.nlevels ? sh.lvl_cnt[l] : 0;
      level_off[(size_t)l * (n + 1) + s + 1] = level_off[(size_t)l * (n + 1) + s] + cnt;
      lvl[(size_t)s * 2 * kMaxLevels + l] = l < sh.nlevels ? sh.lvl_off[l] : 0;
      lvl[(size_t)s * 2 * kMaxLevels + kMaxLevels + l] = cnt;
    }
    max_levels = std::max(max_levels, sh.nlevels);
  }
  const size_t tn = (size_t)std::max<int64_t>(total, 1);
  const size_t nb = (size_t)std::max<int64_t>(b->box_base[n], 1);
  std::vector<int64_t> tab;
  tab.insert(tab.end(), b->cap_off.begin(), b->cap_off.end());
  tab.insert(tab.end(), group_off.begin(), group_off.end());
  tab.insert(tab.end(), b->box_base.begin(), b->box_base.end());
  tab.insert(tab.end(), level_off.begin(), level_off.end());
  tab.insert(tab.end(), b->emit_off.begin(), b->emit_off.end());
  const size_t te = (size_t)std::max<int64_t>(b->total_emit, 1);
  int s;
  if ((s = b->m_pos4.ensure(tn * 16)) || (s = b->m_thr4.ensure(tn * 16)) ||
      (s = b->m_wi2.ensure(tn * 8)) || (s = b->m_boxes.ensure(nb * 32)) ||
      (s = b->m_keys_b.ensure(tn * 8)) || (s = b->m_va.ensure(tn * 4)) ||
      (s = b->m_vb.ensure(tn * 4)) || (s = b->m_order.ensure(tn * 4)) ||
      (s = b->m_count.ensure(te * 4)) || (s = b->m_first.ensure(te * 4)) ||
      (s = b->m_sums.ensure((size_t)scan_tiles((int64_t)te) * 4 + 64)) ||
      (s = b->m_hist.ensure(sort_hist_words((int64_t)tn) * 4)) ||
      (s = b->m_bb.ensure(24 * (size_t)n)) || (s = b->m_tab.ensure(tab.size() * 8)) ||
      (s = b->m_lvl.ensure(lvl.size() * 4)))
    return berr(b, s, "photon maps (%lld photons)", (long long)total);
  cudaError_t e;
  if ((e = cudaMemcpyAsync(b->m_tab.ptr, tab.data(), tab.size() * 8, cudaMemcpyHostToDevice,
                           b->st)) ||
      (e = cudaMemcpyAsync(b->m_lvl.ptr, lvl.data(), lvl.size() * 4, cudaMemcpyHostToDevice,
                           b->st)) ||
      (e = cudaStreamSynchronize(b->st)))
    return bcuda(b, e, "photon map tables");
  BatchMapBuild& a = b->mb;
  a = BatchMapBuild{};
  const int64_t* t = (const int64_t*)b->m_tab.ptr;
  a.raw = (const float*)b->raw.ptr;
  a.keys_a = (unsigned long long*)b->keys.ptr;
  a.keys_b = (unsigned long long*)b->m_keys_b.ptr;
  a.va = (uint32_t*)b->m_va.ptr;
  a.vb = (uint32_t*)b->m_vb.ptr;
  a.hist = (uint32_t*)b->m_hist.ptr;
  a.count = (const uint32_t*)b->m_count.ptr;
  a.first = (uint32_t*)b->m_first.ptr;
  a.sums = (uint32_t*)b->m_sums.ptr;
  a.order = (uint32_t*)b->m_order.ptr;
  a.err = (int*)b->err_word.ptr;
  a.bb = (uint32_t*)b->m_bb.ptr;
  a.stored_off = t;
  a.group_off = t + (n + 1);
  a.box_base = t + 2 * (n + 1);
  a.level_off = t + 3 * (n + 1);
  a.emit_off = t + 3 * (n + 1) + (size_t)kMaxLevels * (n + 1);
  a.lvl = (const int*)b->m_lvl.ptr;
  a.pos4 = (float4*)b->m_pos4.ptr;
  a.thr4 = (float4*)b->m_thr4.ptr;
  a.wi2 = (float2*)b->m_wi2.ptr;
  a.boxes = (float4*)b->m_boxes.ptr;
  a.total = total;
  a.total_emit = b->total_emit;
  a.total_groups = group_off[n];
  for (int l = 0; l < kMaxLevels; ++l) a.level_total[l] = level_off[(size_t)l * (n + 1) + n];
  a.n_scenes = n;
  a.scene_bits = bits_for(n);
  a.max_levels = max_levels;
  a.num_sms = b->num_sms;
  return PM_OK;
}

void enqueue_camera_and_list(pm_batch* b, int block, int stack) {
  cudaMemsetAsync(b->dropped.ptr, 0, 16, b->st);
  batch_camera_launch(b->tables, b->total_pix, block, stack, b->st);
  cudaMemsetAsync(b->qcount.ptr, 0, 4, b->st);
  // unlisted entries: keys sort last and name no scene, values name slot 0
  cudaMemsetAsync(b->qka.ptr, 0xff, (size_t)b->total_slots * 8, b->st);
  cudaMemsetAsync(b->qva.ptr, 0, (size_t)b->total_slots * 4, b->st);
  batch_list_queries_launch(b->tables, b->total_slots, (unsigned long long*)b->qka.ptr,
                            (uint32_t*)b->qva.ptr, (unsigned*)b->qcount.ptr, b->st);
}

// Sorts the listed queries (scene, Morton code); returns the order array.
const uint32_t* enqueue_sort(pm_batch* b) {
  b->sorted_in_b = radix_sort_pairs<unsigned long long>(
      (unsigned long long*)b->qka.ptr, (uint32_t*)b->qva.ptr, (unsigned long long*)b->qkb.ptr,
      (uint32_t*)b->qvb.ptr, (int)b->nq, key_bits(b->n), (uint32_t*)b->qhist.ptr, b->st);
  return (const uint32_t*)(b->sorted_in_b ? b->qvb.ptr : b->qva.ptr);
}

const unsigned long long* sorted_keys(const pm_batch* b) {
  return (const unsigned long long*)(b->sorted_in_b ? b->qkb.ptr : b->qka.ptr);
}

cudaError_t enqueue_knn(pm_batch* b, const uint32_t* order, const pm_batch_tuning& t,
                        int per_sm) {
  batch_query_ranges_launch(sorted_keys(b), b->nq, (const unsigned*)b->qcount.ptr, b->n,
                            t.knn_chunk, (int64_t*)b->qstart.ptr, (int64_t*)b->qoff.ptr,
                            (int64_t*)b->item_off.ptr, b->st);
  const int64_t max_items = b->nq / t.knn_chunk + b->n;
  return batch_knn_launch(b->tables, (const float4*)b->slots.ptr, order,
                          (const int64_t*)b->qoff.ptr, (const int64_t*)b->item_off.ptr,
                          max_items, (float*)b->res.ptr, t.knn_warps, t.knn_chunk, t.knn_buffer,
                          per_sm, (unsigned long long*)b->knn_counter.ptr, b->num_sms, b->st);
}

// The whole step with the current tuning (no host synchronisation).
cudaError_t enqueue_step(pm_batch* b) {
  const pm_batch_tuning& t = b->tune;
  cudaMemsetAsync(b->err_word.ptr, 0, 4, b->st);
  enqueue_trace(b, t.block, t.bvh_stack);
  enqueue_maps(b);
  enqueue_camera_and_list(b, t.block, t.bvh_stack);
  const uint32_t* order = enqueue_sort(b);
  cudaError_t e = enqueue_knn(b, order, t, b->knn_per_sm);
  if (e != cudaSuccess) return e;
  batch_resolve_launch(b->tables, b->total_pix, b->st);
  return cudaGetLastError();
}

// After a step: counts against the plan, and the device error word.
int check_step(pm_batch* b, const char* where) {
  std::vector<unsigned long long> cnt((size_t)b->n);
  unsigned nq = 0;
  int errw = 0;
  cudaError_t e;
  if ((e = cudaMemcpyAsync(cnt.data(), b->counters.ptr, 8 * (size_t)b->n,
                           cudaMemcpyDeviceToHost, b->st)) ||
      (e = cudaMemcpyAsync(&nq, b->qcount.ptr, 4, cudaMemcpyDeviceToHost, b->st)) ||
      (e = cudaMemcpyAsync(&errw, b->err_word.ptr, 4, cudaMemcpyDeviceToHost, b->st)) ||
      (e = cudaStreamSynchronize(b->st)))
    return bcuda(b, e, where);
  if (errw) return berr(b, PM_ERR_DEVICE_STATUS, "%s: device error bits 0x%x", where, errw);
  for (int s = 0; s < b->n; ++s)
    if ((int64_t)cnt[s] != b->stored[s])
      return berr(b, PM_ERR_DEVICE_STATUS, "%s: scene %d stored %llu photons, planned %lld",
                  where, s, cnt[s], (long long)b->stored[s]);
  if ((int64_t)nq != b->nq)
    return berr(b, PM_ERR_DEVICE_STATUS, "%s: %u queries, planned %lld", where, nq,
                (long long)b->nq);
  return PM_OK;
}

int plan(pm_batch* b) {
  const int n = b->n;
  cudaError_t e;
  int s;
  // 1. photons stored per scene
  b->cap.assign((size_t)n, 0);
  for (int i = 0; i < n; ++i) b->cap[i] = std::max<int64_t>(4 * b->desc[i].n_photons, 16);
  b->stored.assign((size_t)n, 0);
  for (int attempt = 0; attempt < 2; ++attempt) {
    if ((s = size_trace(b)) != PM_OK) return s;
    if ((s = upload_tables(b)) != PM_OK) return s;
    cudaMemsetAsync(b->err_word.ptr, 0, 4, b->st);
    enqueue_trace(b, b->tune.block, 64);
    std::vector<unsigned long long> cnt((size_t)n);
    int errw = 0;
    if ((e = cudaGetLastError()) ||
        (e = cudaMemcpyAsync(cnt.data(), b->counters.ptr, 8 * (size_t)n, cudaMemcpyDeviceToHost,
                             b->st)) ||
        (e = cudaMemcpyAsync(&errw, b->err_word.ptr, 4, cudaMemcpyDeviceToHost, b->st)) ||
        (e = cudaStreamSynchronize(b->st)))
      return bcuda(b, e, "batch trace");
    if (errw) return berr(b, PM_ERR_DEVICE_STATUS, "batch trace: device error bits 0x%x", errw);
    bool short_cap = false;
    for (int i = 0; i < n; ++i) {
      if (cnt[i] > 0x7fffffffull)
        return berr(b, PM_ERR_INVALID_ARGUMENT, "scene %d: %llu photons stored", i, cnt[i]);
      b->stored[i] = (int64_t)cnt[i];
      if (b->stored[i] > b->cap[i]) {
        b->cap[i] = b->stored[i];  // the trace is deterministic: rerun with room for all
        short_cap = true;
      }
    }
    if (!short_cap) break;
    if (attempt == 1) return berr(b, PM_ERR_DEVICE_STATUS, "batch trace: capacity");
  }
  // 2. photon maps: the trace regions shrink to the stored counts (the trace
  // is deterministic), so the stored photons of all scenes lie back to back
  b->cap = b->stored;
  if ((s = size_trace(b)) != PM_OK) return s;
  if ((s = plan_maps(b)) != PM_OK) return s;
  // 3. camera-pass buffers
  const size_t ts = (size_t)std::max<int64_t>(b->total_slots, 2);
  if ((s = b->rng.ensure((size_t)b->total_pix * 8)) ||
      (s = b->slots.ensure(ts * 64)) || (s = b->srec.ensure((size_t)b->total_samples * 16)) ||
      (s = b->res.ensure(ts * 12)) || (s = b->images.ensure((size_t)b->total_pix * 12)) ||
      (s = b->qka.ensure(ts * 8)) || (s = b->qkb.ensure(ts * 8)) ||
      (s = b->qva.ensure(ts * 4)) || (s = b->qvb.ensure(ts * 4)) ||
      (s = b->qhist.ensure(sort_hist_words((int64_t)ts) * 4)) || (s = b->qcount.ensure(16)) ||
      (s = b->qstart.ensure(8 * (size_t)n)) || (s = b->qoff.ensure(8 * (size_t)(n + 1))) ||
      (s = b->item_off.ensure(8 * (size_t)(n + 1))) || (s = b->knn_counter.ensure(16)))
    return berr(b, s, "camera buffers (%lld query slots)", (long long)b->total_slots);
  if ((s = upload_tables(b)) != PM_OK) return s;
  // 4. queries: the step up to the listing
  cudaMemsetAsync(b->err_word.ptr, 0, 4, b->st);
  enqueue_trace(b, b->tune.block, 64);
  enqueue_maps(b);
  enqueue_camera_and_list(b, b->tune.block, 64);
  unsigned nq = 0;
  if ((e = cudaGetLastError()) ||
      (e = cudaMemcpyAsync(&nq, b->qcount.ptr, 4, cudaMemcpyDeviceToHost, b->st)) ||
      (e = cudaStreamSynchronize(b->st)))
    return bcuda(b, e, "batch plan");
  b->nq = nq;
  if ((e = batch_knn_prepare(b->tune.knn_warps, b->tune.knn_buffer, &b->knn_per_sm)))
    return bcuda(b, e, "kNN set-up");
  // 5. one full step, checked
  if ((e = enqueue_step(b)) != cudaSuccess) return bcuda(b, e, "batch step");
  if ((s = check_step(b, "batch plan")) != PM_OK) return s;
  std::vector<int64_t> qo((size_t)n + 1);
  if ((e = cudaMemcpy(qo.data(), b->qoff.ptr, 8 * (size_t)(n + 1), cudaMemcpyDeviceToHost)))
    return bcuda(b, e, "batch plan");
  b->queries.assign((size_t)n, 0);
  for (int i = 0; i < n; ++i) b->queries[i] = qo[i + 1] - qo[i];
  return PM_OK;
}

int set_tuning(pm_batch* b, const pm_batch_tuning* t);

}  // namespace

extern "C" {

int pm_batch_create(int device, const pm_batch_scene* scenes, int32_t n, pm_batch** out) {
  if (!out) return PM_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (!scenes || n < 1 || n > PM_BATCH_MAX_SCENES) return PM_ERR_INVALID_ARGUMENT;
  for (int s = 0; s < n; ++s) {
    const pm_batch_scene& d = scenes[s];
    if (d.n_faces < 1 || d.n_faces > (int64_t)0x3fffffff || !d.vertices || !d.normals ||
        !d.materials || d.width <= 0 || d.height <= 0 ||
        (int64_t)d.width * d.height > (1 << 26) || d.spp < 1 || d.k < 1 || d.k > PM_MAX_K ||
        d.max_depth < 0 || d.max_depth > 255 || d.n_photons < 0 ||
        d.n_photons > (int64_t)0x7fffffff)
      return PM_ERR_INVALID_ARGUMENT;
    for (int64_t f = 0; f < d.n_faces; ++f)
      if (d.materials[f].type < PM_LAMBERT || d.materials[f].type > PM_GLASS)
        return PM_ERR_INVALID_ARGUMENT;
  }
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return PM_ERR_CUDA;
  }
  pm_batch* b = new pm_batch();
  b->device = device;
  cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, device);
  if (cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess) {
    delete b;
    cudaGetLastError();
    return PM_ERR_CUDA;
  }
  b->n = n;
  b->scenes.resize((size_t)n);
  b->desc.assign(scenes, scenes + n);
  b->qps.assign((size_t)n, 1);
  b->emit_off.assign((size_t)n + 1, 0);
  b->pix_off.assign((size_t)n + 1, 0);
  b->slot_off.assign((size_t)n + 1, 0);
  b->sample_off.assign((size_t)n + 1, 0);
  *out = b;
  int s;
  if ((s = b->err_word.ensure(64)) != PM_OK) return berr(b, s, "error word");
  cudaMemset(b->err_word.ptr, 0, 64);
  if ((s = b->counters.ensure(8 * (size_t)n)) || (s = b->status.ensure(64)) ||
      (s = b->dropped.ensure(64)))
    return berr(b, s, "counters");
  for (int i = 0; i < n; ++i) {
    const pm_batch_scene& d = scenes[i];
    const char* what = "";
    if ((s = upload_scene(b->scenes[i], b->scene_scratch, b->st, d.vertices, d.normals,
                          d.materials, d.n_faces, &what)) != PM_OK)
      return berr(b, s, "scene %d: %s", i, what);
    if (d.n_photons > 0 && b->scenes[i].n_lights == 0)
      return berr(b, PM_ERR_INVALID_ARGUMENT, "scene %d has no area light", i);
    b->qps[i] = b->scenes[i].has_specular ? 8 : 1;
    b->desc[i].vertices = nullptr;
    b->desc[i].normals = nullptr;
    b->desc[i].materials = nullptr;
    const int64_t px = (int64_t)d.width * d.height;
    b->emit_off[i + 1] = b->emit_off[i] + d.n_photons;
    b->pix_off[i + 1] = b->pix_off[i] + px;
    b->sample_off[i + 1] = b->sample_off[i] + px * d.spp;
    b->slot_off[i + 1] = b->slot_off[i] + px * d.spp * b->qps[i];
    b->max_k = std::max(b->max_k, d.k);
  }
  b->scene_scratch.release();
  b->total_emit = b->emit_off[n];
  b->total_pix = b->pix_off[n];
  b->total_samples = b->sample_off[n];
  b->total_slots = b->slot_off[n];
  if (b->total_slots > 0x7fffffffLL)
    return berr(b, PM_ERR_INVALID_ARGUMENT, "%lld query slots (at most 2^31 - 1)",
                (long long)b->total_slots);
  if (b->max_k > 224) b->tune.knn_buffer = 2048;
  return plan(b);
}

int pm_batch_destroy(pm_batch* b) {
  if (!b) return PM_ERR_INVALID_ARGUMENT;
  cudaSetDevice(b->device);
  if (b->st) cudaStreamSynchronize(b->st);
  delete b;
  return PM_OK;
}

const char* pm_batch_last_error(const pm_batch* b) { return b ? b->err.c_str() : ""; }

int pm_batch_set_tuning(pm_batch* b, const pm_batch_tuning* t) {
  if (!b) return PM_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(b->mu);
  return set_tuning(b, t);
}

}  // extern "C"

namespace {

// pm_batch_set_tuning with the batch's lock held.
int set_tuning(pm_batch* b, const pm_batch_tuning* t) {
  if (!t || !tuning_ok(b, *t)) return berr(b, PM_ERR_INVALID_ARGUMENT, "tuning out of range");
  cudaSetDevice(b->device);
  cudaError_t e;
  int per_sm = 1;
  if ((e = batch_knn_prepare(t->knn_warps, t->knn_buffer, &per_sm)))
    return bcuda(b, e, "kNN set-up");
  b->tune = *t;
  b->knn_per_sm = per_sm;
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  return PM_OK;
}

}  // namespace

extern "C" {

int pm_batch_get_tuning(pm_batch* b, pm_batch_tuning* t) {
  if (!b || !t) return PM_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(b->mu);
  *t = b->tune;
  return PM_OK;
}

int pm_batch_render(pm_batch* b, int32_t use_graph, float* ms) {
  if (!b) return PM_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(b->mu);
  cudaSetDevice(b->device);
  cudaError_t e;
  if (use_graph && !b->exec) {
    cudaGraph_t g = nullptr;
    if ((e = cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal)))
      return bcuda(b, e, "graph capture");
    const cudaError_t es = enqueue_step(b);
    e = cudaStreamEndCapture(b->st, &g);
    if (es != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return bcuda(b, es, "graph capture");
    }
    if (e != cudaSuccess) return bcuda(b, e, "graph capture");
    e = cudaGraphInstantiate(&b->exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      b->exec = nullptr;
      return bcuda(b, e, "graph instantiate");
    }
  }
  if ((e = cudaEventRecord(b->ev0, b->st))) return bcuda(b, e, "batch step");
  e = use_graph ? cudaGraphLaunch(b->exec, b->st) : enqueue_step(b);
  if (e != cudaSuccess) return bcuda(b, e, "batch step");
  if ((e = cudaEventRecord(b->ev1, b->st))) return bcuda(b, e, "batch step");
  int s;
  if ((s = check_step(b, "batch step")) != PM_OK) return s;
  if (ms) {
    float t = 0.f;
    cudaEventElapsedTime(&t, b->ev0, b->ev1);
    *ms = t;
  }
  return PM_OK;
}

int pm_batch_autotune(pm_batch* b, pm_batch_tuning* best, float* ms_stage) {
  if (!b) return PM_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(b->mu);
  cudaSetDevice(b->device);
  cudaError_t e;
  int s;
  auto timed = [&](auto&& fn, float* t) -> int {
    cudaMemsetAsync(b->err_word.ptr, 0, 4, b->st);
    cudaEventRecord(b->ev0, b->st);
    const cudaError_t fe = fn();
    cudaEventRecord(b->ev1, b->st);
    int errw = 0;
    cudaError_t ce;
    if (fe != cudaSuccess) return bcuda(b, fe, "autotune");
    if ((ce = cudaMemcpyAsync(&errw, b->err_word.ptr, 4, cudaMemcpyDeviceToHost, b->st)) ||
        (ce = cudaStreamSynchronize(b->st)))
      return bcuda(b, ce, "autotune");
    cudaEventElapsedTime(t, b->ev0, b->ev1);
    return errw ? -1 : PM_OK;  // -1: the candidate reported an error (rejected)
  };
  pm_batch_tuning t = b->tune;
  // trace and camera: block x stack
  float best_tc = 3.4e38f, best_trace = 0.f, best_cam = 0.f;
  const int blocks[] = {64, 128, 256};
  const int stacks[] = {16, 32, 64};
  for (int bl : blocks)
    for (int sk : stacks) {
      float tt = 0.f, tc = 0.f;
      int r1 = timed([&] { enqueue_trace(b, bl, sk); return cudaGetLastError(); }, &tt);
      if (r1 > 0) return r1;
      int r2 = timed([&] {
        batch_camera_launch(b->tables, b->total_pix, bl, sk, b->st);
        return cudaGetLastError();
      }, &tc);
      if (r2 > 0) return r2;
      if (r1 == 0 && r2 == 0 && tt + tc < best_tc) {
        best_tc = tt + tc;
        best_trace = tt;
        best_cam = tc;
        t.block = bl;
        t.bvh_stack = sk;
      }
    }
  if (best_tc > 3e38f) return berr(b, PM_ERR_DEVICE_STATUS, "autotune: no trace setting ran");
  // the queries of the current step, listed and sorted once
  cudaMemsetAsync(b->err_word.ptr, 0, 4, b->st);
  enqueue_trace(b, t.block, t.bvh_stack);
  enqueue_maps(b);
  enqueue_camera_and_list(b, t.block, t.bvh_stack);
  const uint32_t* order = enqueue_sort(b);
  if ((e = cudaGetLastError())) return bcuda(b, e, "autotune");
  // kNN: warps x chunk x buffer
  float best_knn = 3.4e38f;
  const int warps[] = {4, 8};
  const int chunks[] = {8, 16, 32, 64, 128, 256, 512, 1024};
  const int bufs[] = {512, 2048};
  for (int w : warps)
    for (int c : chunks)
      for (int bf : bufs) {
        pm_batch_tuning cand = t;
        cand.knn_warps = w;
        cand.knn_chunk = c;
        cand.knn_buffer = bf;
        if (!tuning_ok(b, cand)) continue;
        int per_sm = 1;
        if ((e = batch_knn_prepare(w, bf, &per_sm))) return bcuda(b, e, "autotune");
        float tk = 0.f;
        const int r = timed([&] { return enqueue_knn(b, order, cand, per_sm); }, &tk);
        if (r > 0) return r;
        if (r == 0 && tk < best_knn) {
          best_knn = tk;
          t.knn_warps = w;
          t.knn_chunk = c;
          t.knn_buffer = bf;
        }
      }
  if ((s = set_tuning(b, &t)) != PM_OK) return s;
  if (best) *best = t;
  if (ms_stage) {
    ms_stage[0] = best_trace;
    ms_stage[1] = best_cam;
    ms_stage[2] = best_knn;
  }
  // leave the batch as after a full step with the chosen tuning
  if ((e = enqueue_step(b)) != cudaSuccess) return bcuda(b, e, "autotune");
  return check_step(b, "autotune");
}

int pm_batch_stage_times(pm_batch* b, float* ms, int32_t n) {
  if (!b || !ms || n < 1) return PM_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(b->mu);
  cudaSetDevice(b->device);
  cudaEvent_t ev[PM_BATCH_STAGES + 1] = {};
  struct Guard {
    cudaEvent_t* e;
    ~Guard() {
      for (int i = 0; i <= PM_BATCH_STAGES; ++i)
        if (e[i]) cudaEventDestroy(e[i]);
    }
  } guard{ev};
  cudaError_t e;
  for (int i = 0; i <= PM_BATCH_STAGES; ++i)
    if ((e = cudaEventCreate(&ev[i]))) return bcuda(b, e, "stage events");
  const pm_batch_tuning& t = b->tune;
  cudaMemsetAsync(b->err_word.ptr, 0, 4, b->st);
  cudaEventRecord(ev[0], b->st);
  enqueue_trace(b, t.block, t.bvh_stack);
  cudaEventRecord(ev[1], b->st);
  enqueue_maps(b);
  cudaEventRecord(ev[2], b->st);
  enqueue_camera_and_list(b, t.block, t.bvh_stack);
  cudaEventRecord(ev[3], b->st);
  const uint32_t* order = enqueue_sort(b);
  cudaEventRecord(ev[4], b->st);
  if ((e = enqueue_knn(b, order, t, b->knn_per_sm))) return bcuda(b, e, "stage times");
  cudaEventRecord(ev[5], b->st);
  batch_resolve_launch(b->tables, b->total_pix, b->st);
  cudaEventRecord(ev[6], b->st);
  if ((e = cudaGetLastError())) return bcuda(b, e, "stage times");
  int s;
  if ((s = check_step(b, "stage times")) != PM_OK) return s;
  for (int i = 0; i < std::min<int>(n, PM_BATCH_STAGES); ++i) {
    float x = 0.f;
    cudaEventElapsedTime(&x, ev[i], ev[i + 1]);
    ms[i] = x;
  }
  return PM_OK;
}

int pm_batch_image(pm_batch* b, int32_t scene, float* out) {
  if (!b) return PM_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(b->mu);
  if (scene < 0 || scene >= b->n || !out) return berr(b, PM_ERR_INVALID_ARGUMENT, "scene / out");
  cudaSetDevice(b->device);
  const int64_t px = b->pix_off[scene + 1] - b->pix_off[scene];
  cudaError_t e;
  if ((e = cudaMemcpyAsync(out, (float*)b->images.ptr + 3 * b->pix_off[scene], (size_t)px * 12,
                           cudaMemcpyDeviceToHost, b->st)) ||
      (e = cudaStreamSynchronize(b->st)))
    return bcuda(b, e, "batch image");
  return PM_OK;
}

int pm_batch_photons(pm_batch* b, int32_t scene, float* out) {
  if (!b) return PM_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(b->mu);
  if (scene < 0 || scene >= b->n || !out) return berr(b, PM_ERR_INVALID_ARGUMENT, "scene / out");
  cudaSetDevice(b->device);
  const int64_t m = b->stored[scene];
  if (m == 0) return PM_OK;
  DevBuf tmp;
  int s;
  if ((s = tmp.ensure((size_t)m * 36)) != PM_OK) return berr(b, s, "batch photons");
  batch_photons_launch((const float*)b->raw.ptr, (const uint32_t*)b->m_order.ptr + b->cap_off[scene],
                       m, (float*)tmp.ptr, b->st);
  cudaError_t e;
  if ((e = cudaGetLastError()) ||
      (e = cudaMemcpyAsync(out, tmp.ptr, (size_t)m * 36, cudaMemcpyDeviceToHost, b->st)) ||
      (e = cudaStreamSynchronize(b->st))) {
    tmp.release();
    return bcuda(b, e, "batch photons");
  }
  tmp.release();
  return PM_OK;
}

int pm_batch_counts(pm_batch* b, int64_t* stored, int64_t* queries) {
  if (!b) return PM_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(b->mu);
  for (int s = 0; s < b->n; ++s) {
    if (stored) stored[s] = b->stored[s];
    if (queries) queries[s] = b->queries[s];
  }
  return PM_OK;
}

}  // extern "C"
