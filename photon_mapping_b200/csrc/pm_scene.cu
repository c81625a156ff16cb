// Scene upload and LBVH build on the device (replaces the Embree BVH of
// scene.h:275-304): per-face constants, Morton codes of the triangle
// centroids, radix sort, the binary radix tree of Karras (2012) over the
// sorted codes, and a bottom-up refit of padded child boxes.
#include "pm_scene.cuh"
#include "pm_scene_build.cuh"
#include "pm_sort.cuh"

#include <float.h>

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

// Length of the common prefix of (code, index) pairs i and j; -1 outside.
__device__ __forceinline__ int delta(const uint32_t* __restrict__ codes, int n,
                                     int i, int j) {
  if (j < 0 || j >= n) return -1;
  const uint32_t a = codes[i], b = codes[j];
  if (a != b) return __clz(a ^ b);
  return 32 + __clz((uint32_t)i ^ (uint32_t)j);
}

// Karras 2012: internal node i of the binary radix tree over n sorted
// codes. Children: >= 0 internal node, < 0 leaf ~index.
__global__ void radix_tree_kernel(const uint32_t* __restrict__ codes, int n,
                                  int* __restrict__ child,
                                  int* __restrict__ parent) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  const int d = (delta(codes, n, i, i + 1) - delta(codes, n, i, i - 1)) >= 0 ? 1 : -1;
  const int dmin = delta(codes, n, i, i - d);
  int lmax = 2;
  while (delta(codes, n, i, i + lmax * d) > dmin) lmax *= 2;
  int l = 0;
  for (int t = lmax / 2; t >= 1; t /= 2)
    if (delta(codes, n, i, i + (l + t) * d) > dmin) l += t;
  const int j = i + l * d;
  const int dnode = delta(codes, n, i, j);
  int s = 0;
  for (int div = 2;; div *= 2) {
    const int t = (l + div - 1) / div;
    if (delta(codes, n, i, i + (s + t) * d) > dnode) s += t;
    if (t == 1) break;
  }
  const int g = i + s * d + min(d, 0);
  const int left = (min(i, j) == g) ? ~g : g;
  const int right = (max(i, j) == g + 1) ? ~(g + 1) : g + 1;
  child[2 * i] = left;
  child[2 * i + 1] = right;
  // parents: internal nodes in [0, n-1), leaves at n-1 + leaf
  parent[left < 0 ? (n - 1 + ~left) : left] = i;
  parent[right < 0 ? (n - 1 + ~right) : right] = i;
}

// Bottom-up refit: each leaf walks towards the root; the second child to
// arrive at a node merges both child boxes and continues. Boxes are padded
// by `pad` so ray/box rounding never culls a hit triangle.
__global__ void refit_kernel(const float4* __restrict__ mt, int n,
                             const int* __restrict__ child,
                             const int* __restrict__ parent,
                             unsigned* __restrict__ flags,
                             float4* __restrict__ nodes,
                             const uint32_t* __restrict__ bb) {
  const int leaf = blockIdx.x * blockDim.x + threadIdx.x;
  if (leaf >= n) return;
  // padding: 4e-5 of the scene's size (largest extent or coordinate)
  float size = 0.f;
  for (int a = 0; a < 3; ++a) {
    const float lo = from_ordered(bb[a]), hi = from_ordered(bb[3 + a]);
    size = fmaxf(size, fmaxf(hi - lo, fmaxf(fabsf(lo), fabsf(hi))));
  }
  const float pad = 4e-5f * size + 1e-30f;
  const V3 p0 = f4v3(mt[3 * leaf]);
  const V3 p1 = p0 + f4v3(mt[3 * leaf + 1]);
  const V3 p2 = p0 + f4v3(mt[3 * leaf + 2]);
  float4 lo = make_float4(fminf(fminf(p0.x, p1.x), p2.x) - pad,
                          fminf(fminf(p0.y, p1.y), p2.y) - pad,
                          fminf(fminf(p0.z, p1.z), p2.z) - pad, 0.f);
  float4 hi = make_float4(fmaxf(fmaxf(p0.x, p1.x), p2.x) + pad,
                          fmaxf(fmaxf(p0.y, p1.y), p2.y) + pad,
                          fmaxf(fmaxf(p0.z, p1.z), p2.z) + pad, 0.f);
  int me = ~leaf;
  int node = parent[n - 1 + leaf];
  // at most n - 1 steps up
  for (int step = 0; step < n; ++step) {
    const bool is_left = child[2 * node] == me;
    float4* slot = nodes + 4 * node + (is_left ? 0 : 2);
    slot[0] = make_float4(lo.x, lo.y, lo.z, __int_as_float(child[2 * node]));
    slot[1] = make_float4(hi.x, hi.y, hi.z, __int_as_float(child[2 * node + 1]));
    if (!is_left) {
      // keep the child ids in the node's first two words
      nodes[4 * node].w = __int_as_float(child[2 * node]);
      nodes[4 * node + 1].w = __int_as_float(child[2 * node + 1]);
    }
    __threadfence();
    if (atomicAdd(&flags[node], 1u) == 0) return;
    __threadfence();
    const volatile float4* vn = nodes + 4 * node;
    const float4 a = make_float4(vn[0].x, vn[0].y, vn[0].z, 0.f);
    const float4 b = make_float4(vn[1].x, vn[1].y, vn[1].z, 0.f);
    const float4 c = make_float4(vn[2].x, vn[2].y, vn[2].z, 0.f);
    const float4 e = make_float4(vn[3].x, vn[3].y, vn[3].z, 0.f);
    lo = make_float4(fminf(a.x, c.x), fminf(a.y, c.y), fminf(a.z, c.z), 0.f);
    hi = make_float4(fmaxf(b.x, e.x), fmaxf(b.y, e.y), fmaxf(b.z, e.z), 0.f);
    if (node == 0) return;
    me = node;
    node = parent[node];
  }
}

size_t scene_build_scratch_bytes(int n) {
  const size_t nn = (size_t)(n > 1 ? n : 2);
  // keys a/b, vals a/b, hist, bbox, child (2n), parent (2n), flags (n)
  return 4 * nn * 4 + sort_hist_words(nn) * 4 + 64 + 2 * nn * 4 +
         2 * nn * 4 + nn * 4;
}

void scene_build_launch(const float* verts, const float* nrms, int n,
                        float4* tri, float4* nrm, float4* geo, float4* mt,
                        float4* nodes, void* scratch, cudaStream_t st) {
  if (n <= 0) return;
  uint32_t* ka = (uint32_t*)scratch;
  uint32_t* kb = ka + n;
  uint32_t* va = kb + n;
  uint32_t* vb = va + n;
  uint32_t* hist = vb + n;
  uint32_t* bb = hist + sort_hist_words(n);
  int* child = (int*)(bb + 16);
  int* parent = child + 2 * (size_t)n;
  unsigned* flags = (unsigned*)(parent + 2 * (size_t)n);
  const int tb = 256;
  const int gb = (n + tb - 1) / tb;
  face_setup_kernel<<<gb, tb, 0, st>>>(verts, nrms, n, tri, nrm, geo);
  cudaMemsetAsync(bb, 0xff, 3 * sizeof(uint32_t), st);
  cudaMemsetAsync(bb + 3, 0x00, 3 * sizeof(uint32_t), st);
  scene_bbox_kernel<<<min(gb, 1184), tb, 0, st>>>(tri, n, bb);
  tri_morton_kernel<<<gb, tb, 0, st>>>(tri, n, bb, ka, va);
  const bool in_b = radix_sort_pairs<uint32_t>(ka, va, kb, vb, n, 30, hist, st);
  const uint32_t* codes = in_b ? kb : ka;
  const uint32_t* order = in_b ? vb : va;
  leaf_setup_kernel<<<gb, tb, 0, st>>>(tri, n, order, mt);
  if (n == 1) return;
  radix_tree_kernel<<<(n - 1 + tb - 1) / tb, tb, 0, st>>>(codes, n, child,
                                                          parent);
  cudaMemsetAsync(flags, 0, (size_t)(n - 1) * sizeof(unsigned), st);
  refit_kernel<<<gb, tb, 0, st>>>(mt, n, child, parent, flags, nodes, bb);
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
