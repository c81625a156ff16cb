// Scene upload and BVH build on the device (replaces the Embree BVH of
// scene.h:275-304): per-face constants, Morton codes of the triangle
// centroids, radix sort, then the tree built by parallel locally-ordered
// clustering over the sorted leaves (PLOC, below).
#include "pm_scene.cuh"
#include "pm_scene_build.cuh"
#include "pm_sort.cuh"

#include <float.h>

#include <utility>

namespace pm {

// Per-face constants (triangle.h:25-34) and the leaf records.
__global__ void face_setup_kernel(const float* __restrict__ verts,
                                  const float* __restrict__ nrms, int n,
                                  float4* __restrict__ tri,
                                  float4* __restrict__ nrm,
                                  float4* __restrict__ geo) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= n) return;
  const float* v = verts + 9 * (size_t)f;
  const float* nn = nrms + 9 * (size_t)f;
  const V3 p1 = v3(v[0], v[1], v[2]);
  const V3 p2 = v3(v[3], v[4], v[5]);
  const V3 p3 = v3(v[6], v[7], v[8]);
  tri[3 * f] = make_float4(p1.x, p1.y, p1.z, 0.f);
  tri[3 * f + 1] = make_float4(p2.x, p2.y, p2.z, 0.f);
  tri[3 * f + 2] = make_float4(p3.x, p3.y, p3.z, 0.f);
  nrm[3 * f] = make_float4(nn[0], nn[1], nn[2], 0.f);
  nrm[3 * f + 1] = make_float4(nn[3], nn[4], nn[5], 0.f);
  nrm[3 * f + 2] = make_float4(nn[6], nn[7], nn[8], 0.f);
  const V3 c = cross(p2 - p1, p3 - p1);
  const V3 g = normalize(c);
  geo[f] = make_float4(g.x, g.y, g.z, 0.5f * length(c));
}

__global__ void scene_bbox_kernel(const float4* __restrict__ tri, int n,
                                  uint32_t* __restrict__ bb) {
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
  float hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < n;
       f += gridDim.x * blockDim.x) {
    for (int k = 0; k < 3; ++k) {
      const float4 p = tri[3 * f + k];
      lo[0] = fminf(lo[0], p.x); lo[1] = fminf(lo[1], p.y); lo[2] = fminf(lo[2], p.z);
      hi[0] = fmaxf(hi[0], p.x); hi[1] = fmaxf(hi[1], p.y); hi[2] = fmaxf(hi[2], p.z);
    }
  }
  for (int a = 0; a < 3; ++a) {
    for (int o = 16; o > 0; o >>= 1) {
      lo[a] = fminf(lo[a], __shfl_xor_sync(kFull, lo[a], o));
      hi[a] = fmaxf(hi[a], __shfl_xor_sync(kFull, hi[a], o));
    }
  }
  if ((threadIdx.x & 31) == 0) {
    for (int a = 0; a < 3; ++a) {
      atomicMin(&bb[a], ordered_bits(lo[a]));
      atomicMax(&bb[3 + a], ordered_bits(hi[a]));
    }
  }
}

__global__ void tri_morton_kernel(const float4* __restrict__ tri, int n,
                                  const uint32_t* __restrict__ bb,
                                  uint32_t* __restrict__ keys,
                                  uint32_t* __restrict__ vals) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= n) return;
  float lo[3], ext[3];
  for (int a = 0; a < 3; ++a) {
    lo[a] = from_ordered(bb[a]);
    ext[a] = from_ordered(bb[3 + a]) - lo[a];
  }
  const float4 a = tri[3 * f], b = tri[3 * f + 1], c = tri[3 * f + 2];
  const float cx = (a.x + b.x + c.x) * (1.0f / 3.0f);
  const float cy = (a.y + b.y + c.y) * (1.0f / 3.0f);
  const float cz = (a.z + b.z + c.z) * (1.0f / 3.0f);
  keys[f] = (spread10(cell10(cx, lo[0], ext[0])) << 2) |
            (spread10(cell10(cy, lo[1], ext[1])) << 1) |
            spread10(cell10(cz, lo[2], ext[2]));
  vals[f] = (uint32_t)f;
}

// Leaf records in sorted order: {p0, face id}, {p1 - p0}, {p2 - p0}.
__global__ void leaf_setup_kernel(const float4* __restrict__ tri, int n,
                                  const uint32_t* __restrict__ order,
                                  float4* __restrict__ mt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int f = (int)order[i];
  const V3 p0 = f4v3(tri[3 * f]), p1 = f4v3(tri[3 * f + 1]),
           p2 = f4v3(tri[3 * f + 2]);
  const V3 e1 = p1 - p0, e2 = p2 - p0;
  mt[3 * i] = make_float4(p0.x, p0.y, p0.z, __int_as_float(f));
  mt[3 * i + 1] = make_float4(e1.x, e1.y, e1.z, 0.f);
  mt[3 * i + 2] = make_float4(e2.x, e2.y, e2.z, 0.f);
}

// ------------------------------------------------------------ BVH (PLOC)
//
// Parallel locally-ordered clustering (Meister & Bittner, IEEE TVCG 2018):
// the clusters start as the leaves in Morton order; each pass finds every
// cluster's nearest neighbour among the kPlocRadius clusters on either side
// (the distance is the surface area of the two boxes' union), merges every
// mutual pair into a new internal node and compacts the clusters in order.
// Pairs are ordered by (union area, index distance, parity of the smaller
// index, smaller index): a total order on pairs, so the globally first pair
// is mutual and every pass merges at least one pair, and clusters with
// equal boxes pair up as (2k, 2k + 1), a balanced tree, instead of all
// choosing one neighbour (a chain one merge per pass). Internal nodes are
// numbered from the top down in creation order (the last merge, the root,
// is node 0). Leaf boxes are padded by `pad`, so ray/box rounding never
// culls a hit triangle; a parent's box is the union of its children's.

constexpr int kPlocRadius = 16;
constexpr int kPlocBlock = 256;

__device__ __forceinline__ float union_area(float4 alo, float4 ahi, float4 blo, float4 bhi) {
  const float dx = fmaxf(ahi.x, bhi.x) - fminf(alo.x, blo.x);
  const float dy = fmaxf(ahi.y, bhi.y) - fminf(alo.y, blo.y);
  const float dz = fmaxf(ahi.z, bhi.z) - fminf(alo.z, blo.z);
  const float a = dx * dy + dy * dz + dz * dx;
  return a <= FLT_MAX ? a : FLT_MAX;  // NaN and infinity order last
}

// Leaf clusters: id ~leaf, box of the leaf triangle padded by 4e-5 of the
// scene's size (largest extent or coordinate).
__global__ void ploc_leaf_kernel(const float4* __restrict__ mt, int n,
                                 const uint32_t* __restrict__ bb, int* __restrict__ cid,
                                 float4* __restrict__ blo, float4* __restrict__ bhi) {
  const int leaf = blockIdx.x * blockDim.x + threadIdx.x;
  if (leaf >= n) return;
  float size = 0.f;
  for (int a = 0; a < 3; ++a) {
    const float lo = from_ordered(bb[a]), hi = from_ordered(bb[3 + a]);
    size = fmaxf(size, fmaxf(hi - lo, fmaxf(fabsf(lo), fabsf(hi))));
  }
  const float pad = 4e-5f * size + 1e-30f;
  const V3 p0 = f4v3(mt[3 * leaf]);
  const V3 p1 = p0 + f4v3(mt[3 * leaf + 1]);
  const V3 p2 = p0 + f4v3(mt[3 * leaf + 2]);
  blo[leaf] = make_float4(fminf(fminf(p0.x, p1.x), p2.x) - pad,
                          fminf(fminf(p0.y, p1.y), p2.y) - pad,
                          fminf(fminf(p0.z, p1.z), p2.z) - pad, 0.f);
  bhi[leaf] = make_float4(fmaxf(fmaxf(p0.x, p1.x), p2.x) + pad,
                          fmaxf(fmaxf(p0.y, p1.y), p2.y) + pad,
                          fmaxf(fmaxf(p0.z, p1.z), p2.z) + pad, 0.f);
  cid[leaf] = ~leaf;
}

// nn[i] = the cluster j != i, |i - j| <= kPlocRadius, whose pair with i
// comes first in the pair order. m >= 2.
__global__ void __launch_bounds__(kPlocBlock)
    ploc_nn_kernel(const float4* __restrict__ blo, const float4* __restrict__ bhi, int m,
                   int* __restrict__ nn) {
  __shared__ float4 slo[kPlocBlock + 2 * kPlocRadius];
  __shared__ float4 shi[kPlocBlock + 2 * kPlocRadius];
  const int base = blockIdx.x * kPlocBlock - kPlocRadius;
  for (int t = threadIdx.x; t < kPlocBlock + 2 * kPlocRadius; t += blockDim.x) {
    const int k = base + t;
    if (k >= 0 && k < m) {
      slo[t] = blo[k];
      shi[t] = bhi[k];
    }
  }
  __syncthreads();
  const int i = blockIdx.x * kPlocBlock + threadIdx.x;
  if (i >= m) return;
  const float4 lo = slo[threadIdx.x + kPlocRadius], hi = shi[threadIdx.x + kPlocRadius];
  float best = INFINITY;
  int bj = -1, bkey = 0;
  for (int o = -kPlocRadius; o <= kPlocRadius; ++o) {
    const int j = i + o;
    if (o == 0 || j < 0 || j >= m) continue;
    const int t = threadIdx.x + kPlocRadius + o;
    const float c = union_area(lo, hi, slo[t], shi[t]);
    // ties: nearer first, then an even smaller index, then the smaller one
    const int mn = min(i, j);
    const int key = (abs(o) << 2) | ((mn & 1) << 1) | (o > 0 ? 1 : 0);
    if (c < best || (c == best && key < bkey)) {
      best = c;
      bj = j;
      bkey = key;
    }
  }
  nn[i] = bj;
}

// mflag[i]: i merges with nn[i] and owns the new node (mutual, i < nn[i]);
// keep[i]: cluster i survives the pass (not absorbed by a smaller owner).
__global__ void ploc_flags_kernel(const int* __restrict__ nn, int m, uint32_t* __restrict__ mflag,
                                  uint32_t* __restrict__ keep) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int j = nn[i];
  const bool mutual = nn[j] == i;
  mflag[i] = mutual && i < j;
  keep[i] = !(mutual && j < i);
}

// The pass's merges and the compacted clusters. Merge owner i gets node
// top - 1 - mrank[i]; out[0] = clusters left, out[1] = merges.
__global__ void ploc_merge_kernel(const int* __restrict__ cid, const float4* __restrict__ blo,
                                  const float4* __restrict__ bhi, const int* __restrict__ nn,
                                  int m, const uint32_t* __restrict__ mflag,
                                  const uint32_t* __restrict__ mrank,
                                  const uint32_t* __restrict__ keep,
                                  const uint32_t* __restrict__ kpos, int top,
                                  int* __restrict__ cid2, float4* __restrict__ blo2,
                                  float4* __restrict__ bhi2, float4* __restrict__ nodes,
                                  int* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  if (i == m - 1) {
    out[0] = (int)(kpos[i] + keep[i]);
    out[1] = (int)(mrank[i] + mflag[i]);
  }
  if (!keep[i]) return;
  const float4 alo = blo[i], ahi = bhi[i];
  const int o = (int)kpos[i];
  if (!mflag[i]) {
    cid2[o] = cid[i];
    blo2[o] = alo;
    bhi2[o] = ahi;
    return;
  }
  const int j = nn[i];
  const float4 clo = blo[j], chi = bhi[j];
  const int idx = top - 1 - (int)mrank[i];
  float4* nd = nodes + 4 * (size_t)idx;
  nd[0] = make_float4(alo.x, alo.y, alo.z, __int_as_float(cid[i]));
  nd[1] = make_float4(ahi.x, ahi.y, ahi.z, __int_as_float(cid[j]));
  nd[2] = make_float4(clo.x, clo.y, clo.z, 0.f);
  nd[3] = make_float4(chi.x, chi.y, chi.z, 0.f);
  cid2[o] = idx;
  blo2[o] = make_float4(fminf(alo.x, clo.x), fminf(alo.y, clo.y), fminf(alo.z, clo.z), 0.f);
  bhi2[o] = make_float4(fmaxf(ahi.x, chi.x), fmaxf(ahi.y, chi.y), fmaxf(ahi.z, chi.z), 0.f);
}

size_t scene_build_scratch_bytes(int n) {
  const size_t nn = (size_t)(n > 1 ? n : 2);
  // cluster boxes a/b (4n float4), sort keys / values a/b (4n), histogram,
  // scene box, cluster ids a/b and neighbours (3n), pass flags and ranks
  // (4n), scan tile sums, pass counts
  return 4 * nn * 16 + 4 * nn * 4 + sort_hist_words(nn) * 4 + 64 + 3 * nn * 4 + 4 * nn * 4 +
         (size_t)scan_tiles((int64_t)nn) * 4 + 64;
}

cudaError_t scene_build_launch(const float* verts, const float* nrms, int n, float4* tri,
                               float4* nrm, float4* geo, float4* mt, float4* nodes,
                               void* scratch, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  float4* blo_a = (float4*)scratch;
  float4* bhi_a = blo_a + n;
  float4* blo_b = bhi_a + n;
  float4* bhi_b = blo_b + n;
  uint32_t* ka = (uint32_t*)(bhi_b + n);
  uint32_t* kb = ka + n;
  uint32_t* va = kb + n;
  uint32_t* vb = va + n;
  uint32_t* hist = vb + n;
  uint32_t* bb = hist + sort_hist_words(n);
  int* cid_a = (int*)(bb + 16);
  int* cid_b = cid_a + n;
  int* nn = cid_b + n;
  uint32_t* mflag = (uint32_t*)(nn + n);
  uint32_t* keep = mflag + n;
  uint32_t* mrank = keep + n;
  uint32_t* kpos = mrank + n;
  uint32_t* sums = kpos + n;
  int* out = (int*)(sums + scan_tiles(n));
  const int tb = 256;
  const int gb = (n + tb - 1) / tb;
  face_setup_kernel<<<gb, tb, 0, st>>>(verts, nrms, n, tri, nrm, geo);
  cudaMemsetAsync(bb, 0xff, 3 * sizeof(uint32_t), st);
  cudaMemsetAsync(bb + 3, 0x00, 3 * sizeof(uint32_t), st);
  scene_bbox_kernel<<<min(gb, 1184), tb, 0, st>>>(tri, n, bb);
  tri_morton_kernel<<<gb, tb, 0, st>>>(tri, n, bb, ka, va);
  const bool in_b = radix_sort_pairs<uint32_t>(ka, va, kb, vb, n, 30, hist, st);
  const uint32_t* order = in_b ? vb : va;
  leaf_setup_kernel<<<gb, tb, 0, st>>>(tri, n, order, mt);
  if (n == 1) return cudaGetLastError();
  ploc_leaf_kernel<<<gb, tb, 0, st>>>(mt, n, bb, cid_a, blo_a, bhi_a);
  int m = n, top = n - 1;
  int counts[2] = {0, 0};
  cudaError_t e;
  // every pass merges at least one pair: at most n - 1 passes
  for (int pass = 0; m > 1 && pass < n; ++pass) {
    const int g = (m + tb - 1) / tb;
    ploc_nn_kernel<<<(m + kPlocBlock - 1) / kPlocBlock, kPlocBlock, 0, st>>>(blo_a, bhi_a, m,
                                                                             nn);
    ploc_flags_kernel<<<g, tb, 0, st>>>(nn, m, mflag, keep);
    exclusive_scan_u32(mflag, mrank, m, sums, st);
    exclusive_scan_u32(keep, kpos, m, sums, st);
    ploc_merge_kernel<<<g, tb, 0, st>>>(cid_a, blo_a, bhi_a, nn, m, mflag, mrank, keep, kpos, top,
                                        cid_b, blo_b, bhi_b, nodes, out);
    if ((e = cudaMemcpyAsync(counts, out, sizeof(counts), cudaMemcpyDeviceToHost, st)) ||
        (e = cudaStreamSynchronize(st)))
      return e;
    if (counts[1] < 1 || counts[1] > top || counts[0] != m - counts[1])
      return cudaErrorUnknown;  // no progress: cannot happen with the tie rule
    m = counts[0];
    top -= counts[1];
    std::swap(cid_a, cid_b);
    std::swap(blo_a, blo_b);
    std::swap(bhi_a, bhi_b);
  }
  if (m != 1 || top != 0) return cudaErrorUnknown;
  return cudaGetLastError();
}

// Batched closest-hit queries (Scene::intersect, scene.h:307-348).
// rays: 8 floats each {origin, tmin, direction, tmax}.
__global__ void intersect_kernel(SceneDev sc, const float4* __restrict__ rays,
                                 int64_t n, float4* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 a = rays[2 * i], b = rays[2 * i + 1];
  Hit h;
  const bool hit = intersect(sc, v3(a.x, a.y, a.z), v3(b.x, b.y, b.z), a.w,
                             b.w, h);
  out[i] = hit ? make_float4(h.t, h.u, h.v, __int_as_float(h.prim))
               : make_float4(0.f, 0.f, 0.f, __int_as_float(-1));
}

void intersect_launch(const SceneDev& sc, const float4* rays, int64_t n,
                      float4* out, cudaStream_t st) {
  if (n <= 0) return;
  const int tb = 128;
  intersect_kernel<<<(unsigned)((n + tb - 1) / tb), tb, 0, st>>>(sc, rays, n,
                                                                 out);
}

}  // namespace pm
