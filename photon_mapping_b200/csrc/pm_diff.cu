// Differentiable render: the adjoint of the camera pass's resolve step.
//
// Every radiance term the photon mapper sums is a product of one emission
// factor and of albedo factors, times quantities that do not depend on the
// parameters once the paths are fixed (photon paths replayed from their
// seeds with frozen Russian-roulette decisions, camera paths drawn from the
// per-pixel streams):
//   light seen along a camera path          Le
//   next-event estimation at diffuse x      rho(x) Le ...
//   photon-map estimate at diffuse x        rho(x) sum_i Phi_i / (N pi r^2)
//   the same behind a gather ray from y     rho(y) rho(x) sum_i Phi_i ...
//   photon throughput Phi_i                 Le prod_j rho(hit j) ...
// so d term / d log theta_j = (times theta_j appears in it) * term. The
// adjoint accumulates G_j = sum over terms of (d loss / d term) * count *
// term; d loss / d theta_j = G_j / theta_j (the parameters are positive).
//
// This file handles the terms of the camera pass: per sample, its
// next-event records and, per query slot, weight * estimate, and writes the
// adjoint of each slot's estimate for the photon-map pass (pm_photonmap.cu,
// adjoint mode) and the photon replay (pm_trace.cu, replay mode).
#include "pm_diff.cuh"

namespace pm {

__global__ void diff_apply_kernel(const Material* __restrict__ base,
                                  const int* __restrict__ face_pid, int n,
                                  const float* __restrict__ albedo,
                                  const float* __restrict__ emission,
                                  Material* __restrict__ out) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= n) return;
  Material m = base[f];
  const int pid = face_pid[f];
  if (pid >= 0) {
    m.rho[0] = albedo[3 * pid];
    m.rho[1] = albedo[3 * pid + 1];
    m.rho[2] = albedo[3 * pid + 2];
  }
  if (m.le[0] > 0.f || m.le[1] > 0.f || m.le[2] > 0.f) {
    m.le[0] = emission[0];
    m.le[1] = emission[1];
    m.le[2] = emission[2];
  }
  out[f] = m;
}

void diff_apply_launch(const Material* base, const int* face_pid, int n_faces,
                       const float* albedo, const float* emission, Material* out,
                       cudaStream_t st) {
  if (n_faces <= 0) return;
  diff_apply_kernel<<<(n_faces + 127) / 128, 128, 0, st>>>(base, face_pid, n_faces, albedo,
                                                           emission, out);
}

__device__ __forceinline__ void acc3(float* g, int pid, V3 v) {
  atomicAdd(g + 3 * pid + 0, v.x);
  atomicAdd(g + 3 * pid + 1, v.y);
  atomicAdd(g + 3 * pid + 2, v.z);
}

__global__ void __launch_bounds__(128)
    diff_adjoint_samples_kernel(DiffAdjointArgs a) {
  // parameter sums of this block; slot n_params holds the emission
  __shared__ float g[3 * (kMaxDiffParams + 1)];
  const int ng = 3 * (a.n_params + 1);
  for (int t = threadIdx.x; t < ng; t += blockDim.x) g[t] = 0.f;
  __syncthreads();
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < a.npix) {
    // image = sum of kept samples / spp (Image::divide, image.h:49-56)
    const float ispp = 1.0f / (float)a.spp;
    const V3 gp = v3(a.grad_img[3 * p] * ispp, a.grad_img[3 * p + 1] * ispp,
                     a.grad_img[3 * p + 2] * ispp);
    for (int s = 0; s < a.spp; ++s) {
      const int64_t sidx = (int64_t)p * a.spp + s;
      const float4 d = a.srec[sidx];
      const int nq = __float_as_int(d.w);
      // the forward's resolve arithmetic, to drop the same samples
      V3 rad = v3(d.x, d.y, d.z);
      for (int q = 0; q < nq; ++q) {
        const int64_t t = sidx * a.q_per_sample + q;
        const float4 w = a.slots[4 * t + 3];
        rad = rad + v3(w.x, w.y, w.z) *
                        v3(a.res[3 * t], a.res[3 * t + 1], a.res[3 * t + 2]);
      }
      const bool kept = !has_nan(rad) && !(rad.x < 0.f || rad.y < 0.f || rad.z < 0.f);
      if (!kept) {
        for (int q = 0; q < nq; ++q) {
          const int64_t t = sidx * a.q_per_sample + q;
          a.slot_adj[3 * t] = a.slot_adj[3 * t + 1] = a.slot_adj[3 * t + 2] = 0.f;
        }
        continue;
      }
      // every term carries the emission once
      acc3(g, a.n_params, gp * rad);
      const int nn = a.nee_count[sidx];
      for (int r = 0; r < nn; ++r) {
        const float4 e = a.nee[sidx * a.q_per_sample + r];
        const int pid = __float_as_int(e.w);
        if (pid >= 0) acc3(g, pid, gp * v3(e.x, e.y, e.z));
      }
      for (int q = 0; q < nq; ++q) {
        const int64_t t = sidx * a.q_per_sample + q;
        const float4 w4 = a.slots[4 * t + 3];
        const V3 w = v3(w4.x, w4.y, w4.z);
        const V3 term = gp * w * v3(a.res[3 * t], a.res[3 * t + 1], a.res[3 * t + 2]);
        const int2 pp = a.slot_pid[t];
        if (pp.x >= 0) acc3(g, pp.x, term);
        if (pp.y >= 0) acc3(g, pp.y, term);
        const V3 adj = gp * w;
        a.slot_adj[3 * t] = adj.x;
        a.slot_adj[3 * t + 1] = adj.y;
        a.slot_adj[3 * t + 2] = adj.z;
      }
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < ng; t += blockDim.x)
    if (g[t] != 0.f) atomicAdd(a.grad + t, (double)g[t]);
}

void diff_adjoint_samples_launch(const DiffAdjointArgs& a, cudaStream_t st) {
  if (a.npix <= 0) return;
  diff_adjoint_samples_kernel<<<(a.npix + 127) / 128, 128, 0, st>>>(a);
}

}  // namespace pm
