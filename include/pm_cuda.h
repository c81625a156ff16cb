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
  uint64_t walks;       /* tree walks: more than one per query when a guessed
                           radius held fewer than k photons                  */
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

/* Sets how many photons were emitted to make `map` (nPhotonsGlobal,
 * nPhotonsCaustics: the normalisation of integrator.h:149 and :171) for
 * pm_render; pm_photons_trace sets it itself. */
int pm_photonmap_set_emitted(pm_ctx* ctx, int map, int64_t n_emitted);

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

/* ------------------------------------------- allocation-free estimate */
/* No counterpart in the reference. For callers that cannot call cudaMalloc
 * (a plug-in whose host application owns all device memory and forbids
 * allocations in its callbacks; a real-time loop that cannot afford the
 * device-wide synchronisation of cudaMalloc/cudaFree): the radiance
 * estimate of pm_photonmap_radiance over a photon set of at most
 * PM_NOALLOC_MAX_PHOTONS photons, with no context and no allocation. The
 * caller passes d_photons (n_photons x 9 floats), d_queries (16-byte
 * aligned pm_radiance_query records) and d_out_rgb (nq x 3 floats) in
 * device memory of the current device; the call enqueues the map build
 * and the queries on `stream` (NULL: legacy default stream) and returns.
 * Intermediate buffers live in one static device array (about 3.9 MiB per
 * GPU that loads the library, kept until exit). Every call looks that
 * array's address up (cudaGetSymbolAddress) in the CUDA context current at
 * the call, so a non-primary context or a context made after
 * cudaDeviceReset gets its own address; the first call in a context loads
 * the library's device code and should come before any stream capture.
 * Calls share the array: calls that overlap on
 * the GPU race and must be serialised by the caller. Larger photon sets
 * are rejected with PM_ERR_INVALID_ARGUMENT. */
#define PM_NOALLOC_MAX_PHOTONS 65536
int pm_photonmap_radiance_noalloc(const float* d_photons, int64_t n_photons,
                                  const pm_radiance_query* d_queries,
                                  int64_t nq, int k, int64_t n_emitted,
                                  float* d_out_rgb, void* stream);

/* --------------------------------------------------------------- scene */
/* Per-face material, as Scene::loadModel derives it from the OBJ/MTL
 * (scene.h:15-51): illum 5 -> Mirror, illum 7 -> Glass(Ni), otherwise
 * Lambert(Kd); Ke > 0 makes the face an area light (AreaLight, light.h). */
enum pm_material_type { PM_LAMBERT = 0, PM_MIRROR = 1, PM_GLASS = 2 };
typedef struct pm_material {
  int32_t type;   /* pm_material_type                                      */
  float rho[3];   /* albedo; Mirror and Glass use (1, 1, 1) (scene.h:26-33) */
  float ior;      /* Glass index of refraction                             */
  float le[3];    /* emitted radiance; light when any component > 0        */
} pm_material;

/* Replaces Scene::build (scene.h:275-304): uploads the faces and builds the
 * device BVH. vertices and normals hold 9 floats per face (the reference's
 * per-face unshared vertices, scene.h:199-212; a face without normals
 * carries its geometric normal three times, scene.h:182-189). */
int pm_scene_upload(pm_ctx* ctx, const float* vertices, const float* normals,
                    const pm_material* materials, int64_t n_faces);

/* Closest hit of a ray (Scene::intersect, scene.h:307-348). */
typedef struct pm_hit {
  float t;        /* hit distance; hit point = origin + t * direction      */
  float u, v;     /* barycentrics of vertices 1 and 2 (Embree's u, v)      */
  int32_t prim;   /* face index, -1 when nothing was hit                   */
} pm_hit;

/* Batched Scene::intersect. rays: 8 floats each {origin.xyz, tmin,
 * direction.xyz, tmax}; a hit needs tmin <= t <= tmax. Among hits at the
 * same distance the smallest face index is returned. */
int pm_scene_intersect(pm_ctx* ctx, const float* rays, int64_t n,
                       pm_hit* out);

/* ------------------------------------------------------ photon tracing */
typedef struct pm_trace_stats {
  int64_t emitted;              /* photons emitted                       */
  int64_t stored;               /* photons stored in the map             */
  uint32_t nan_throughput;      /* paths stopped on a NaN throughput     */
  uint32_t negative_throughput; /* paths stopped on a negative one       */
  int64_t rays;                 /* closest-hit queries traced            */
  float trace_ms;               /* device time of the tracing kernel     */
  float build_ms;               /* device time of ordering the photons
                                   and building the map                  */
} pm_trace_stats;

/* Replaces the photon-tracing half of PhotonMapping::build
 * (integrator.h:393-563): emits n_emit photons from the scene's area lights
 * and traces them for at most max_depth (<= 255) bounces with the storage
 * rule of `map` (PM_MAP_GLOBAL: every diffuse hit, integrator.h:406-469;
 * PM_MAP_CAUSTICS: the first diffuse hit after a specular one,
 * integrator.h:483-558), then builds that photon map. Photon i draws from
 * its own PCG32 stream (state derived from seed and i), so the stored set
 * and its order (by photon, then bounce) are reproducible. */
int pm_photons_trace(pm_ctx* ctx, int map, uint64_t seed, int64_t n_emit,
                     int max_depth, pm_trace_stats* stats);

/* -------------------------------------------------------------- render */
/* A constructed pinhole Camera (camera.h:21-37): right = normalize(forward
 * x (0,1,0)), up = normalize(right x forward), focal_length = 1/tan(FOV/2),
 * computed by the caller exactly as the reference's constructor does. */
typedef struct pm_camera {
  float position[3];
  float forward[3];
  float right[3];
  float up[3];
  float focal_length;
} pm_camera;

typedef struct pm_render_params {
  int32_t width, height;
  int32_t spp;                   /* samples per pixel (n_samples)           */
  int32_t k_global;              /* nEstimationGlobal                       */
  int32_t k_caustics;            /* k of the caustics-map estimate; the
                                    reference uses nEstimationGlobal there
                                    (integrator.h:161)                       */
  int32_t final_gathering_depth; /* strictCalcDepth                         */
  int32_t max_depth;             /* maxDepth                                */
  int32_t n_gather;              /* gather rays per diffuse hit at depth <
                                    final_gathering_depth, averaged; 1 is the
                                    reference (integrator.h:224-235)         */
  int32_t spp_batch;             /* samples per pixel per pass, 0 = auto    */
  int32_t flags;                 /* PM_RENDER_FP64_CHECK or 0               */
} pm_render_params;

/* pm_render_params.flags: also sum every pixel's kept samples in FP64 and
 * report how far the FP32 image is from those sums (accum_rel_err). */
#define PM_RENDER_FP64_CHECK 1

typedef struct pm_render_stats {
  int64_t samples;            /* camera samples taken                      */
  int64_t dropped_nan;        /* samples dropped as NaN (main.cpp:49-52)   */
  int64_t dropped_negative;   /* samples dropped as negative (:53-56)      */
  int64_t queries_global;     /* global-map estimates                      */
  int64_t queries_caustics;   /* caustics-map estimates                    */
  int32_t passes;             /* sample batches                            */
  int32_t reserved;
  double accum_rel_err;       /* with PM_RENDER_FP64_CHECK: the largest
                                 relative difference, over pixels and
                                 channels, between the image and the FP64
                                 sums of the same samples; 0 otherwise     */
  int64_t rays;               /* closest-hit queries of the camera pass
                                 (camera and specular rays, shadow rays,
                                 gather rays)                              */
  float camera_ms;            /* device time of the camera-pass kernels    */
  float estimate_ms;          /* device time of listing, sorting and
                                 answering the photon-map queries          */
} pm_render_stats;

/* The render loop of examples/main.cpp:33-70 with
 * PhotonMapping::integrate (integrator.h:290-377): for every pixel (i, j)
 * a sampler seeded j + width*i takes spp samples, each a camera ray
 * through (2(j+u)-width)/height, (2(i+v)-height)/height; NaN and negative
 * samples are dropped but counted in the average. out_rgb receives
 * height x width x 3 floats, row-major, divided by spp (Image::divide),
 * before gamma correction. Uses the scene and the traced photon maps of
 * the context; the estimates divide by the photons emitted for each map
 * (integrator.h:149, :171). */
int pm_render(pm_ctx* ctx, const pm_camera* camera,
              const pm_render_params* params, float* out_rgb,
              pm_render_stats* stats);

typedef struct pm_integrate_params {
  int32_t k_global, k_caustics;  /* as in pm_render_params                */
  int32_t final_gathering_depth;
  int32_t max_depth;
  int32_t n_gather;              /* 1 = the reference                      */
  int32_t reserved;
} pm_integrate_params;

/* PhotonMapping::integrate (integrator.h:566-569), batched over n rays:
 * rays holds 6 floats each {origin, direction}; rng_states[i] is the state
 * of the caller's sampler for ray i (the reference's RNG: PCG32 with
 * inc = 1, sampler.h:11-47) and comes back advanced by exactly the draws
 * integrate makes. out_rgb[3i..3i+3) receives the radiance, unfiltered
 * (the caller drops NaN or negative samples, examples/main.cpp:49-56). */
int pm_integrate(pm_ctx* ctx, const float* rays, int64_t n,
                 uint64_t* rng_states, const pm_integrate_params* params,
                 float* out_rgb);

/* PathTracing::integrate (integrator.h:51-106) inside the render loop of
 * tests/test_path_tracing.cpp:25-52: spp samples per pixel from a sampler
 * seeded j + width*i, NaN samples dropped but counted in the average.
 * out_rgb: height x width x 3 floats, divided by spp. dropped_nan may be
 * NULL. */
int pm_render_path_tracing(pm_ctx* ctx, const pm_camera* camera,
                           int32_t width, int32_t height, int32_t spp,
                           int32_t max_depth, float* out_rgb,
                           int64_t* dropped_nan);

/* PathTracing::integrate (integrator.h:60-105) for n given rays (6 floats
 * each {origin, direction}) with their samplers' PCG32 states, advanced in
 * place by the draws made; out_rgb receives each ray's radiance. */
int pm_path_trace_rays(pm_ctx* ctx, const float* rays, int64_t n,
                       uint64_t* rng_states, int32_t max_depth,
                       float* out_rgb);

/* ------------------------------------------------- differentiable render
 * The reference computes no gradients; these entry points extend its
 * PhotonMapping::build + render loop (integrator.h:393-563, 290-377,
 * examples/main.cpp:33-70) with the derivative of an image loss with
 * respect to per-material Lambert albedos and the light emission.
 *
 * The parameters: n_params albedo parameters (RGB each), face f using
 * parameter face_param[f] (-1: its material stays as uploaded), and one
 * emission RGB that replaces Le of every emitting face. Parameter faces
 * must be Lambertian. All parameters must be positive and finite.
 *
 * Photon paths are replayed from their per-photon seeds, never stored. The
 * Russian-roulette decisions of the photon trace (integrator.h:441-449)
 * depend on the throughput, hence on the albedos; the forward pass makes
 * them with the "decision" parameters, so that a change of the albedos
 * alone moves no path (frozen decisions) and the image is a smooth
 * function of the parameters. With decision parameters equal to the
 * parameters the forward pass is the plain render. */

#define PM_DIFF_MAX_PARAMS 32

/* Sets the albedo parameter of every face of the uploaded scene (n_faces
 * entries in [-1, n_params)). Uploading a scene clears it. */
int pm_diff_set_parameters(pm_ctx* ctx, const int32_t* face_param,
                           int64_t n_faces, int32_t n_params);

typedef struct pm_diff_params {
  int32_t width, height, spp;
  int32_t k;                     /* nEstimationGlobal, both maps
                                    (integrator.h:139, :161)                 */
  int32_t final_gathering_depth;
  int32_t max_depth;
  int32_t n_gather;              /* 1 = the reference                      */
  int32_t reserved;
  int64_t n_photons;             /* nPhotonsGlobal                         */
  int64_t n_photons_caustics;    /* caustics map (final gathering only)    */
  uint64_t seed;                 /* global map; the caustics map: seed + 1 */
} pm_diff_params;

/* Forward pass: writes albedo (n_params x 3) and emission (3) into the
 * scene's materials, traces both photon maps with Russian-roulette
 * decisions taken on decision_albedo / decision_emission (NULL: the
 * parameters themselves), renders the image (as pm_render, all spp in one
 * pass) into out_rgb (height x width x 3) and keeps what pm_diff_backward
 * needs. stats may be NULL. */
int pm_diff_forward(pm_ctx* ctx, const pm_camera* camera,
                    const pm_diff_params* params, const float* albedo,
                    const float* emission, const float* decision_albedo,
                    const float* decision_emission, float* out_rgb,
                    pm_render_stats* stats);

/* Backward pass of the last pm_diff_forward on this context: given
 * grad_rgb = d loss / d image (height x width x 3), writes d loss / d
 * albedo (n_params x 3) and d loss / d emission (3). The hand-written
 * adjoint runs the camera pass in reverse, scatters each estimate's adjoint
 * onto its k nearest photons, and replays the photon paths from their
 * seeds. */
int pm_diff_backward(pm_ctx* ctx, const float* grad_rgb, float* grad_albedo,
                     float* grad_emission);

/* ------------------------------------------------------- batched render
 * Many scenes, views and query sets of uneven size rendered together. The
 * reference renders one scene per process (examples/main.cpp:7-71:
 * Scene::loadModel, PhotonMapping::build, the OpenMP pixel loop over
 * integrate); a batch runs that for every scene at once. One step traces
 * the global photon map of every scene (one launch), orders and builds each
 * map (per scene, on 8 streams), runs the camera pass of every pixel of
 * every scene (one launch), and answers every photon-map query of every
 * scene in one persistent kNN launch, then resolves every image (one
 * launch). The step can be captured once in a CUDA graph and replayed.
 *
 * The render of scene s is the one pm_photons_trace + pm_render give on
 * its own context for the same scene, seed, camera and parameters, with
 * finalGatheringDepth 0 (the estimate at the first diffuse hit) and spp
 * samples per pixel: the images are identical. */

#define PM_BATCH_MAX_SCENES 256

typedef struct pm_batch pm_batch;

typedef struct pm_batch_scene {
  const float* vertices;          /* as pm_scene_upload; read during create */
  const float* normals;
  const pm_material* materials;
  int64_t n_faces;
  pm_camera camera;
  int32_t width, height, spp;
  int32_t k;                      /* nEstimationGlobal                     */
  int32_t max_depth;              /* maxDepth                              */
  int32_t reserved;
  int64_t n_photons;              /* nPhotonsGlobal                        */
  uint64_t seed;                  /* pm_photons_trace seed                 */
} pm_batch_scene;

/* Launch shapes of the batched kernels (pm_batch_autotune picks them). */
typedef struct pm_batch_tuning {
  int32_t knn_warps;   /* warps per block of the persistent kNN kernel, 1..8 */
  int32_t knn_chunk;   /* consecutive queries per warp work item, 1..1024    */
  int32_t knn_buffer;  /* candidate buffer per warp: 512 (k <= 224) or 2048  */
  int32_t bvh_stack;   /* BVH traversal stack entries: 16, 32 or 64          */
  int32_t block;       /* threads per block of trace and camera: 64..256     */
  int32_t reserved;
} pm_batch_tuning;

/* Uploads every scene (its own BVH), sizes every buffer by running the
 * step once (photons stored and queries per scene), and keeps the scenes'
 * parameters. */
int pm_batch_create(int device, const pm_batch_scene* scenes, int32_t n_scenes,
                    pm_batch** out);
int pm_batch_destroy(pm_batch* batch);
const char* pm_batch_last_error(const pm_batch* batch);
int pm_batch_set_tuning(pm_batch* batch, const pm_batch_tuning* tuning);
int pm_batch_get_tuning(pm_batch* batch, pm_batch_tuning* tuning);
/* Times candidate launch shapes on this batch's own work (trace and camera
 * kernels: block x stack depth; kNN: warps x chunk x buffer), keeps the
 * fastest that reported no error, and returns it. ms_per_stage (may be
 * NULL) receives the best times of {trace, camera, kNN} in ms. */
int pm_batch_autotune(pm_batch* batch, pm_batch_tuning* best, float* ms_per_stage);
/* One step over every scene. use_graph != 0: the step is captured in a
 * CUDA graph on first use (and after a tuning change) and replayed. ms
 * (may be NULL) receives the step's device time. */
int pm_batch_render(pm_batch* batch, int32_t use_graph, float* ms);
/* Image of scene s after the last step: height x width x 3 floats. */
int pm_batch_image(pm_batch* batch, int32_t scene, float* out_rgb);
/* Photons stored and photon-map queries answered per scene (n_scenes each;
 * either may be NULL). */
int pm_batch_counts(pm_batch* batch, int64_t* photons_stored, int64_t* queries);
/* The photon map of scene s after the last step: photons_stored[s] records
 * of 9 floats in index order, as PhotonMapping::build stores them for that
 * scene (integrator.h:406-469; the counterpart of pm_photonmap_get_photons). */
int pm_batch_photons(pm_batch* batch, int32_t scene, float* out_photons);

/* Stages of one batched step, in order, for pm_batch_stage_times. */
#define PM_BATCH_STAGE_TRACE 0   /* photon emission and tracing, every scene   */
#define PM_BATCH_STAGE_MAPS 1    /* photon order and map build, every scene    */
#define PM_BATCH_STAGE_CAMERA 2  /* camera pass and the listing of the queries */
#define PM_BATCH_STAGE_SORT 3    /* sort of the queries by (scene, Morton)     */
#define PM_BATCH_STAGE_KNN 4     /* query ranges and the radiance estimates    */
#define PM_BATCH_STAGE_RESOLVE 5 /* samples into the images                    */
#define PM_BATCH_STAGES 6
/* Runs one step without a graph, timing each stage with CUDA events, and
 * writes min(n, PM_BATCH_STAGES) times in ms. The step's results are those
 * of pm_batch_render. */
int pm_batch_stage_times(pm_batch* batch, float* ms, int32_t n);

#ifdef __cplusplus
}
#endif
#endif /* PM_CUDA_H */
