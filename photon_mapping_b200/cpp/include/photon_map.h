// Drop-in for the reference's photon_map.h (photon_map.h:10-212): Photon
// and PhotonMap with the same members and methods. The map itself is built
// and queried on the device through libpm_cuda (pm_photonmap_*); the host
// keeps the photon array for getIthPhoton.
#ifndef PM_DROPIN_PHOTON_MAP_H
#define PM_DROPIN_PHOTON_MAP_H
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

#include "core.h"
#include "pm_cuda.h"
#include "spdlog/spdlog.h"

struct Photon {
  Vec3f throughput;
  Vec3f position;
  Vec3f wi;
  static constexpr int dim = 3;
  float operator[](int i) const { return position[i]; }
  Photon() {}
  Photon(const Vec3f& throughput, const Vec3f& position, const Vec3f& wi)
      : throughput(throughput), position(position), wi(wi) {}
};
static_assert(sizeof(Photon) == 36, "Photon is the 9-float record of the C ABI");

namespace pm_dropin {
inline int device_index() {
  const char* e = std::getenv("PM_DEVICE");
  return e ? std::atoi(e) : 0;
}
inline void check(pm_ctx* ctx, int status, const char* what) {
  if (status != PM_OK) {
    const std::string msg = std::string(what) + ": " + pm_status_string(status) + " " +
                            (ctx ? pm_ctx_last_error(ctx) : "");
    spdlog::error("{}", msg);
    throw std::runtime_error(msg);
  }
}
}  // namespace pm_dropin

class PhotonMap {
  std::vector<Photon> photons;
  pm_ctx* ctx = nullptr;
  bool own_ctx = false;
  int map_id = PM_MAP_GLOBAL;

  void ensure_ctx() {
    if (!ctx) {
      pm_dropin::check(nullptr, pm_ctx_create(pm_dropin::device_index(), &ctx), "pm_ctx_create");
      own_ctx = true;
    }
  }

 public:
  PhotonMap() {}
  PhotonMap(const PhotonMap&) = delete;
  PhotonMap& operator=(const PhotonMap&) = delete;
  ~PhotonMap() {
    if (own_ctx && ctx) pm_ctx_destroy(ctx);
  }

  // Binds the map to slot `map` of an existing context (PhotonMapping's).
  void bind(pm_ctx* shared, int map) {
    if (own_ctx && ctx) pm_ctx_destroy(ctx);
    ctx = shared;
    own_ctx = false;
    map_id = map;
  }
  // Refreshes the host copy from a map traced on the device.
  void pull() {
    int64_t n = 0;
    pm_dropin::check(ctx, pm_photonmap_size(ctx, map_id, &n), "pm_photonmap_size");
    photons.resize((size_t)n);
    if (n)
      pm_dropin::check(ctx,
                       pm_photonmap_get_photons(ctx, map_id, 0, n,
                                                reinterpret_cast<float*>(photons.data())),
                       "pm_photonmap_get_photons");
  }

  const int getNPhotons() const { return (int)photons.size(); }
  const Photon& getIthPhoton(int i) const { return photons[i]; }
  void addPhoton(const Photon& photon) { photons.push_back(photon); }
  void setPhotons(const std::vector<Photon>& p) { photons = p; }

  void build() {
    spdlog::info("[PhotonMap] photons: {}", photons.size());
    ensure_ctx();
    pm_dropin::check(ctx,
                     pm_photonmap_build(ctx, map_id, reinterpret_cast<const float*>(photons.data()),
                                        (int64_t)photons.size()),
                     "pm_photonmap_build");
  }

  // photon_map.h:208-211: indices largest distance first, maxDist2
  std::vector<int> queryKNearestPhotons(const Vec3f& p, int k, float& max_dist2) const {
    std::vector<int32_t> idx((size_t)k);
    int32_t cnt = 0;
    const float q[3] = {p[0], p[1], p[2]};
    pm_dropin::check(ctx, pm_photonmap_knn(ctx, map_id, q, 1, k, idx.data(), &cnt, &max_dist2),
                     "pm_photonmap_knn");
    return std::vector<int>(idx.begin(), idx.begin() + cnt);
  }

  // Batched queries: points n x 3, idx n x k (padded with -1).
  void queryKNearestPhotons(const float* points, int64_t n, int k, int32_t* idx, int32_t* count,
                            float* max_dist2) const {
    pm_dropin::check(ctx, pm_photonmap_knn(ctx, map_id, points, n, k, idx, count, max_dist2),
                     "pm_photonmap_knn");
  }
};

#endif
