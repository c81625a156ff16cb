/*
 * pm_cuda.h — C ABI of the B200 photon-mapping hot path (libpm_cuda.so).
 *
 * Every entry point replaces one call of the reference renderer
 * (yumcyaWiz/photon_mapping, a header-only C++ library); the reference
 * function each one stands in for is cited as file:line of that project.
 *
 * Conventions
 *   - Every function returns an int status (PM_OK == 0); nothing throws
 *     across this boundary. pm_ctx_last_error() gives a message for the last
 *     failing call on a context.
 *   - Host pointers are copied before the call returns ("host" API). The
 *     *_device variants take device pointers and a cudaStream_t (as void*;
 *     NULL is CUDA's legacy default stream), enqueue asynchronously on that
 *     stream and return immediately.
 *   - All device allocations are owned by the context and released by
 *     pm_ctx_destroy(). Calls on one context are serialised by a mutex, so a
 *     context may be shared by host threads (the reference calls integrate()
 *     and the photon-map query from OpenMP threads).
 *   - Float arrays use the reference's own layouts: a photon is 9 floats
 *     {throughput.rgb, position.xyz, wi.xyz} (photon_map.h:10-22); a
 *     position or direction is 3 floats.
 */
#ifndef PM_CUDA_H
#define PM_CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
enum pm_status {
  PM_OK = 0,
  PM_ERR_INVALID_ARGUMENT = 1, /* bad size, k, map id or null pointer       */
  PM_ERR_CUDA = 2,             /* a CUDA runtime call failed                 */
  PM_ERR_OUT_OF_MEMORY = 3,    /* device allocation failed                   */
  PM_ERR_NOT_BUILT = 4,        /* query on a map / scene that was not built  */
  PM_ERR_DEVICE_STATUS = 5     /* a kernel reported an error in its status   */
};

/* Photon map ids. The reference keeps two maps in PhotonMapping
 * (integrator.h:129-130): the global map and the caustics map. */
enum pm_map_id { PM_MAP_GLOBAL = 0, PM_MAP_CAUSTICS = 1 };

/* Largest k accepted by the k-nearest-neighbour entry points. */
#define PM_MAX_K 1024

typedef struct pm_ctx pm_ctx;

/* Query record of the radiance estimate, 48 bytes, laid out for float4
 * loads. pos = hit point, wo = direction towards the viewer (-ray.direction),
 * ns = shading normal as the intersector returns it (not re-normalised),
 * rho = Lambert albedo of the hit primitive (material.h:73-88). */
typedef struct pm_radiance_query {
  float px, py, pz, rho_r;
  float wox, woy, woz, rho_g;
  float nsx, nsy, nsz, rho_b;
} pm_radiance_query;

/* ------------------------------------------------------------- context */
/* Creates a context on CUDA device `device` with its own stream. */
int pm_ctx_create(int device, pm_ctx** out);
/* Frees every device allocation of the context. */
int pm_ctx_destroy(pm_ctx* ctx);
/* Waits for all work enqueued on the context's stream. */
int pm_ctx_synchronize(pm_ctx* ctx);
/* Message of the last failing call on `ctx` ("" if none). */
const char* pm_ctx_last_error(const pm_ctx* ctx);
/* Static name of a status code. */
const char* pm_status_string(int status);

/* Counters of the k-nearest-neighbour kernels (diagnostics; no reference
 * counterpart). Collected only while enabled with pm_ctx_set_stats. */
typedef struct pm_knn_stats {
  uint64_t queries;     /* queries answered                                  */
  uint64_t cold_starts; /* queries whose search radius was bounded afresh    */
  uint64_t candidates;  /* photons found within the search radius            */
  uint64_t leaves;      /* 8-photon groups scanned                           */
  uint64_t nodes;       /* inner tree nodes expanded                         */
  uint64_t selects;     /* k-th distance selections                          */
} pm_knn_stats;

/* Turns the kNN counters on (1) or off (0) for later launches. */
int pm_ctx_set_stats(pm_ctx* ctx, int enable);
/* Copies the counters (waits for the context's stream); reset != 0 zeroes
 * them afterwards. */
int pm_ctx_get_stats(pm_ctx* ctx, pm_knn_stats* out, int reset);

/* ---------------------------------------------------------- photon map */
/* Replaces PhotonMap::setPhotons + PhotonMap::build
 * (photon_map.h:198-206, KdTree::buildTree photon_map.h:157-164).
 * `photons` holds n records of 9 floats (see above); n == 0 gives an empty
 * map, which every query answers with no neighbours. The map is rebuilt on
 * the device: Morton codes, radix sort, boxes over 8-photon groups, 32-ary
 * box tree above them. */
int pm_photonmap_build(pm_ctx* ctx, int map, const float* photons, int64_t n);

/* Same as pm_photonmap_build with `d_photons` in device memory. */
int pm_photonmap_build_device(pm_ctx* ctx, int map, const void* d_photons,
                              int64_t n, void* stream);

/* PhotonMap::getNPhotons (photon_map.h:194). */
int pm_photonmap_size(pm_ctx* ctx, int map, int64_t* n);

/* PhotonMap::getIthPhoton (photon_map.h:195) for i in [first, first+count):
 * copies count records of 9 floats, in the map's index order. */
int pm_photonmap_get_photons(pm_ctx* ctx, int map, int64_t first,
                             int64_t count, float* out);

/* PhotonMap::queryKNearestPhotons (photon_map.h:208-211, search in
 * photon_map.h:107-147 and :166-183), batched over nq query points.
 * queries: nq x 3 floats. For query i, out_idx[i*k .. i*k+k) receives the
 * photon indices in the reference's return order (largest distance first;
 * among equal distances the larger index first), padded with -1 when the
 * map holds fewer than k photons; out_count[i] is the number returned and
 * out_maxdist2[i] the largest squared distance kept (0 when none).
 * The neighbour set is the exact k smallest (dist2, index) pairs, dist2
 * being the float sum of squared differences in x, y, z order
 * (photon_map.h:33-41). Requires 1 <= k <= PM_MAX_K. */
int pm_photonmap_knn(pm_ctx* ctx, int map, const float* queries, int64_t nq,
                     int k, int32_t* out_idx, int32_t* out_count,
                     float* out_maxdist2);

/* PhotonMapping::computeRadianceWithPhotonMap (integrator.h:133-152) for a
 * Lambert hit, batched: out_rgb[3*i..3*i+3) =
 *   sum over the k nearest photons of f(wo, wi) * throughput
 *   / (n_emitted * PI * maxDist2),
 * with f = rho/PI when both cosines in the shading frame are >= 0 and 0
 * otherwise (material.h:80-88). n_emitted is the number of photons emitted
 * when the map was traced (nPhotonsGlobal, integrator.h:149). */
int pm_photonmap_radiance(pm_ctx* ctx, int map, const pm_radiance_query* q,
                          int64_t nq, int k, int64_t n_emitted,
                          float* out_rgb);

/* Same as pm_photonmap_radiance with device pointers, asynchronous. */
int pm_photonmap_radiance_device(pm_ctx* ctx, int map, const void* d_queries,
                                 int64_t nq, int k, int64_t n_emitted,
                                 void* d_out_rgb, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* PM_CUDA_H */
