// ORACLE — test infrastructure only. CPU restatement of the reference's
// photon-map query and radiance estimate, used by tests/ and by bench.py's
// CPU-baseline leg as the checker. Nothing in the product links it.
//
// Built with -ffp-contract=off: float expressions round per operation, as
// the reference's x86-64 build does (SSE scalar, no FMA).
//
// Parity pins: the neighbour sets are checked against the reference's own
// KdTree compiled unchanged from its headers (oracle/_ref, built by
// oracle/Makefile), see tests/test_oracle.py.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

namespace {

constexpr float kPI = 3.14159265359f;  // core.h:7

// photon_map.h:33-41 — dist2 = 0; dist2 += (p1[i]-p2[i])^2 for i = x, y, z,
// p1 = query point, p2 = photon.
inline float distance2(const float* q, const float* p) {
  float d2 = 0.f;
  for (int i = 0; i < 3; ++i) d2 += (q[i] - p[i]) * (q[i] - p[i]);
  return d2;
}

// core.h:200-203
inline float dot3(const float* a, const float* b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

struct Cand {
  float d2;
  int32_t idx;
};
// std::priority_queue<std::pair<float,int>> (photon_map.h:107) orders by
// (dist2, index) lexicographically; the k smallest pairs are kept.
inline bool pair_less(const Cand& a, const Cand& b) {
  return a.d2 < b.d2 || (a.d2 == b.d2 && a.idx < b.idx);
}

}  // namespace

extern "C" {

// Exact k nearest neighbours by brute force over all n photons.
// photons: n x 9 floats {throughput, position, wi}; queries: nq x 3.
// Output per query, like KdTree::searchKNearest (photon_map.h:166-183):
// indices in heap-pop order (largest (dist2, index) first), padded with -1,
// the number returned and maxDist2 (largest kept dist2, 0 when none).
// Photons whose distance is NaN are never returned. Every photon is tested;
// a max-heap of the k smallest (dist2, index) pairs seen so far (the
// bounded queue of photon_map.h:120-126) keeps the scan linear.
void orc_knn(const float* photons, int64_t n, const float* queries,
             int64_t nq, int k, int32_t* out_idx, int32_t* out_cnt,
             float* out_maxd2) {
#pragma omp parallel
  {
    std::vector<Cand> h;
    h.reserve((size_t)k + 1);
#pragma omp for schedule(dynamic, 4)
    for (int64_t qi = 0; qi < nq; ++qi) {
      const float* q = queries + 3 * qi;
      h.clear();
      for (int64_t i = 0; i < n; ++i) {
        const float d2 = distance2(q, photons + 9 * i + 3);
        if (std::isnan(d2)) continue;
        const Cand c{d2, (int32_t)i};
        if ((int)h.size() < k) {
          h.push_back(c);
          std::push_heap(h.begin(), h.end(), pair_less);
        } else if (pair_less(c, h.front())) {
          std::pop_heap(h.begin(), h.end(), pair_less);
          h.back() = c;
          std::push_heap(h.begin(), h.end(), pair_less);
        }
      }
      std::sort_heap(h.begin(), h.end(), pair_less);  // ascending
      const size_t kk = h.size();
      int32_t* row = out_idx + qi * (int64_t)k;
      float maxd2 = 0.f;
      for (size_t r = 0; r < kk; ++r) {
        row[r] = h[kk - 1 - r].idx;  // descending
        maxd2 = std::max(maxd2, h[r].d2);
      }
      for (size_t r = kk; r < (size_t)k; ++r) row[r] = -1;
      out_cnt[qi] = (int32_t)kk;
      out_maxd2[qi] = maxd2;
    }
  }
}

// Radiance estimate of integrator.h:133-152 for a Lambert hit, accumulated
// in FP64 over the given neighbour sets. The BRDF selection (material.h:
// 80-88: zero when cos(wo) < 0 or cos(wi) < 0 in the shading frame, whose
// y axis is the shading normal, primitive.h:32-44) is taken in FP32 exactly
// as the reference decides it; only the sum and the normalisation are FP64.
// queries: nq x 12 floats {pos, rho.r, wo, rho.g, ns, rho.b}.
void orc_radiance_fp64(const float* photons, const int32_t* nbr_idx,
                       const int32_t* nbr_cnt, const float* maxd2, int k,
                       const float* queries, int64_t nq, int64_t n_emitted,
                       double* out) {
#pragma omp parallel for schedule(static)
  for (int64_t qi = 0; qi < nq; ++qi) {
    const float* r = queries + 12 * qi;
    const float wo[3] = {r[4], r[5], r[6]};
    const float ns[3] = {r[8], r[9], r[10]};
    const float rho[3] = {r[3], r[7], r[11]};
    const float cos_o = dot3(wo, ns);
    double lo[3] = {0, 0, 0};
    const int cnt = nbr_cnt[qi];
    for (int j = 0; j < cnt; ++j) {
      const float* p = photons + 9 * (int64_t)nbr_idx[qi * (int64_t)k + j];
      const float wi[3] = {p[6], p[7], p[8]};
      const float cos_i = dot3(wi, ns);
      if (cos_o < 0.f || cos_i < 0.f) continue;
      for (int c = 0; c < 3; ++c)
        lo[c] += ((double)rho[c] / (double)kPI) * (double)p[c];
    }
    for (int c = 0; c < 3; ++c) {
      double v = lo[c];
      if (cnt > 0) v /= ((double)n_emitted * (double)kPI * (double)maxd2[qi]);
      out[3 * qi + c] = v;
    }
  }
}

// The same estimate in FP32 in the reference's own order: photons summed in
// heap-pop order (the order of nbr_idx), f = rho/PI per channel, then one
// division by float(n_emitted) * PI * maxDist2 (integrator.h:141-150).
void orc_radiance_fp32(const float* photons, const int32_t* nbr_idx,
                       const int32_t* nbr_cnt, const float* maxd2, int k,
                       const float* queries, int64_t nq, int64_t n_emitted,
                       float* out) {
#pragma omp parallel for schedule(static)
  for (int64_t qi = 0; qi < nq; ++qi) {
    const float* r = queries + 12 * qi;
    const float wo[3] = {r[4], r[5], r[6]};
    const float ns[3] = {r[8], r[9], r[10]};
    const float rho[3] = {r[3], r[7], r[11]};
    const float cos_o = dot3(wo, ns);
    float lo[3] = {0.f, 0.f, 0.f};
    const int cnt = nbr_cnt[qi];
    for (int j = 0; j < cnt; ++j) {
      const float* p = photons + 9 * (int64_t)nbr_idx[qi * (int64_t)k + j];
      const float wi[3] = {p[6], p[7], p[8]};
      const float cos_i = dot3(wi, ns);
      if (cos_o < 0.f || cos_i < 0.f) continue;
      for (int c = 0; c < 3; ++c) lo[c] += (rho[c] / kPI) * p[c];
    }
    if (cnt > 0) {
      const float den = (float)n_emitted * kPI * maxd2[qi];
      for (int c = 0; c < 3; ++c) lo[c] /= den;
    }
    for (int c = 0; c < 3; ++c) out[3 * qi + c] = lo[c];
  }
}

}  // extern "C"
