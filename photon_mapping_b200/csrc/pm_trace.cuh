// Photon tracing launchers.
#pragma once

#include "pm_scene.cuh"

namespace pm {

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
};

// State of the PCG32 stream of photon i for a trace seeded with `seed`.
__host__ __device__ unsigned long long photon_stream_state(
    unsigned long long seed, unsigned long long i);

void trace_launch(const SceneDev& sc, const TraceArgs& a, cudaStream_t st);

size_t order_scratch_bytes(int64_t n);

// Sorts the n appended photons by key (key_bits wide) into `out`.
void order_photons_launch(unsigned long long* keys, const float* raw, int n,
                          int key_bits, float* out, void* scratch,
                          cudaStream_t st);

}  // namespace pm
