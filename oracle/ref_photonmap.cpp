// ORACLE — test infrastructure only. Compiles the reference's own
// PhotonMap / KdTree (include/photon_map.h of yumcyaWiz/photon_mapping,
// unchanged, read from the reference tree at build time) into
// oracle/_ref/libpmref_photonmap.so, to pin the oracle and to time the
// reference CPU path. spdlog comes from the shim in oracle/shim.
#include <algorithm>
#include <cstdint>
#include <memory>
#include <vector>

#include <omp.h>

#include "spdlog/spdlog.h"
// reference headers
#include "photon_map.h"
#include "primitive.h"

namespace {

struct RefMap {
  PhotonMap map;
  int64_t n = 0;
};

// One Lambert primitive per distinct albedo (scenes have a handful), built
// before any timed call so the estimate does not allocate per query.
struct LambertCache {
  std::vector<Vec3f> rho;
  std::vector<std::unique_ptr<Primitive>> prim;
  const Primitive* get(const Vec3f& r) const {
    for (size_t i = 0; i < rho.size(); ++i)
      if (rho[i][0] == r[0] && rho[i][1] == r[1] && rho[i][2] == r[2])
        return prim[i].get();
    return nullptr;
  }
  void add(const Vec3f& r) {
    if (get(r)) return;
    rho.push_back(r);
    prim.emplace_back(new Primitive(nullptr, std::make_shared<Lambert>(r)));
  }
};

}  // namespace

extern "C" {

// PhotonMap::setPhotons + build (photon_map.h:198-206).
void* ref_pm_build(const float* ph, int64_t n) {
  RefMap* m = new RefMap();
  std::vector<Photon> v((size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    const float* r = ph + 9 * i;
    v[i] = Photon(Vec3f(r[0], r[1], r[2]), Vec3f(r[3], r[4], r[5]),
                  Vec3f(r[6], r[7], r[8]));
  }
  m->map.setPhotons(v);
  m->map.build();
  m->n = n;
  return m;
}

void ref_pm_free(void* h) { delete static_cast<RefMap*>(h); }

int ref_max_threads() { return omp_get_max_threads(); }

// PhotonMap::queryKNearestPhotons (photon_map.h:208-211) per query, OpenMP
// over queries; output as in orc_knn.
void ref_pm_knn(void* h, const float* q, int64_t nq, int k, int32_t* out_idx,
                int32_t* out_cnt, float* out_maxd2) {
  const RefMap* m = static_cast<const RefMap*>(h);
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < nq; ++i) {
    float md2 = 0.f;
    const std::vector<int> r = m->map.queryKNearestPhotons(
        Vec3f(q[3 * i], q[3 * i + 1], q[3 * i + 2]), k, md2);
    int32_t* row = out_idx + i * (int64_t)k;
    for (int j = 0; j < k; ++j) row[j] = j < (int)r.size() ? r[j] : -1;
    out_cnt[i] = (int32_t)r.size();
    out_maxd2[i] = md2;
  }
}

// The loop of PhotonMapping::computeRadianceWithPhotonMap
// (integrator.h:133-152) on the reference's own PhotonMap, Primitive and
// Lambert, with the hit's shading frame built as Scene::intersect builds it
// (scene.h:334-337). queries: nq x 12 {pos, rho.r, wo, rho.g, ns, rho.b}.
void ref_pm_radiance(void* h, const float* q, int64_t nq, int k,
                     int n_emitted, float* out) {
  const RefMap* m = static_cast<const RefMap*>(h);
  LambertCache cache;
  for (int64_t i = 0; i < nq; ++i) {
    const float* r = q + 12 * i;
    cache.add(Vec3f(r[3], r[7], r[11]));
  }
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < nq; ++i) {
    const float* r = q + 12 * i;
    IntersectInfo info;
    info.surfaceInfo.position = Vec3f(r[0], r[1], r[2]);
    info.surfaceInfo.shadingNormal = Vec3f(r[8], r[9], r[10]);
    orthonormalBasis(info.surfaceInfo.shadingNormal, info.surfaceInfo.dpdu,
                     info.surfaceInfo.dpdv);
    info.hitPrimitive = cache.get(Vec3f(r[3], r[7], r[11]));
    const Vec3f wo(r[4], r[5], r[6]);

    float max_dist2;
    const std::vector<int> photon_indices =
        m->map.queryKNearestPhotons(info.surfaceInfo.position, k, max_dist2);
    Vec3f Lo;
    for (const int photon_idx : photon_indices) {
      const Photon& photon = m->map.getIthPhoton(photon_idx);
      const Vec3f f = info.hitPrimitive->evaluateBxDF(
          wo, photon.wi, info.surfaceInfo, TransportDirection::FROM_CAMERA);
      Lo += f * photon.throughput;
    }
    if (photon_indices.size() > 0) {
      Lo /= (n_emitted * PI * max_dist2);
    }
    out[3 * i] = Lo[0];
    out[3 * i + 1] = Lo[1];
    out[3 * i + 2] = Lo[2];
  }
}

}  // extern "C"
