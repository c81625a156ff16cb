// Photon tracing launchers.
#pragma once

#include "pm_scene.cuh"

namespace pm {

// Albedo parameters of the differentiable render (per context).
constexpr int kMaxDiffParams = 32;

struct TraceArgs {
  unsigned long long seed;
  int n_emit;     // photons emitted
  int max_depth;  // bounces (<= 255)
  int caustic;    // 0: global map rule, 1: caustics map rule
  float* out;     // 9 floats per stored photon (append order)
  unsigned long long* keys;     // (photon index << 8 | j) per stored photon, j its
                                // ordinal among its photon's stores (< 255)
  uint32_t* store_count;        // per work index of the launch (the photon index
                                // of a single trace): photons its path stored,
                                // written when the path ends; or null
  unsigned long long* counter;  // photons stored (keeps counting past cap)
  unsigned long long cap;       // capacity of out / keys
  unsigned* status;  // [0] NaN throughput, [1] negative throughput
  unsigned long long* next;  // work counter of the persistent kernel (reset by the launch)
  unsigned long long* rays;  // closest-hit queries traced (added to), or null
  // Differentiable render; all null in a plain trace.
  //   dmat != null: Russian roulette and the NaN / negative stops are
  //     decided on a second throughput carried with these materials, so the
  //     paths do not move when the albedos in sc.mat change (frozen
  //     decisions).
  //   adj != null (replay): nothing is stored; at each point where a photon
  //     would be stored, s = first[photon] + (stores so far) (< cap, the
//     photons stored; error bit 8 otherwise), and
  //     adj[s].xyz * throughput * (times face parameter j scaled the
  //     throughput) is added to grad[3j .. 3j+3).
  const Material* dmat;
  const uint32_t* first;
  const float4* adj;
  const int* face_pid;  // albedo parameter of each face, -1 for none
  int n_params;         // <= kMaxDiffParams
  double* grad;
};

// State of the PCG32 stream of photon i for a trace seeded with `seed`.
__host__ __device__ unsigned long long photon_stream_state(
    unsigned long long seed, unsigned long long i);

void trace_launch(const SceneDev& sc, const TraceArgs& a, cudaStream_t st);

// The n appended photons of a trace of n_emit photons, in index order (the
// order PhotonMapping::build appends them to its photon vector,
// integrator.h:406-469): photon p's stores come after every store of the
// photons before it, in path order. With the store counts the trace wrote,
// first[p] = count[0] + ... + count[p - 1] (an exclusive scan) is the index
// of p's first stored photon, and the record with key p << 8 | j goes to
// out[first[p] + j]: no sort. A key whose index falls outside [0, n) sets
// bit 5 (32) of *err and is dropped. scratch: order_scratch_bytes(n_emit).
size_t order_scratch_bytes(int64_t n_emit);
void order_photons_launch(const unsigned long long* keys, const float* raw, int64_t n,
                          const uint32_t* count, int64_t n_emit, uint32_t* first, float* out,
                          void* scratch, int* err, cudaStream_t st);

}  // namespace pm
