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
  unsigned long long* keys;     // (photon index << 8 | bounce) per photon
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

size_t order_scratch_bytes(int64_t n);

// Sorts the n appended photons by key (key_bits wide) into `out`. With
// first != null, first[p] receives the sorted index of the first stored
// photon of emitted photon p (entries of photons that stored none are left
// as they were).
void order_photons_launch(unsigned long long* keys, const float* raw, int n,
                          int key_bits, float* out, void* scratch,
                          cudaStream_t st, uint32_t* first = nullptr);

}  // namespace pm
