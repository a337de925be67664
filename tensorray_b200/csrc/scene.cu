// Scene construction, the differentiable geometry chain, the LBVH build and
// the geometry-chain adjoint.
//
// Reference counterparts:
//   Scene::ExtractGeometry / ConfigureLight / Configure   Scene.cpp:46-124, 471-533
//   Primitive::Configure (translation parameter)          Primitive.cpp:134-210
//   TriangleMesh::ComputeFaceNormalAndDistrib             Primitive.cpp:299-321
//   TriangleMesh::ComputeVertexNormal                     Primitive.cpp:323-340
//   ObjMesh::processEdges                                 ObjMesh.cpp:584-632
//   ConstructSecEdgeList                                  Edge.cpp:42-88
//   Distribution1D::SetFunction                           Distribution.cpp:45-58
//   Scene::ConstructAccelerationStructure (OptiX GAS)     Scene.cpp:171-366
#include <cub/cub.cuh>
#include <algorithm>
#include <cstring>
#include <atomic>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "../../include/trn.h"
#include "scene_impl.cuh"

namespace trn {

static thread_local std::string g_err;
void set_error(const std::string& msg) { g_err = msg; }
static std::atomic<unsigned long long> g_launches{0};
void count_launch(int n) { g_launches.fetch_add((unsigned long long)n, std::memory_order_relaxed); }

static_assert(sizeof(trn_camera) == sizeof(CameraDesc), "camera layout");
static_assert(sizeof(trn_bsdf) == sizeof(BsdfDesc), "bsdf layout");

// ---------------------------------------------------------------------------
// geometry chain kernels
// ---------------------------------------------------------------------------
__global__ void k_transform(int nv, const float* raw, const int* vmesh, const float* trans, float* pos) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  const int m = vmesh[v];
  // TransformPoints with (I + T) (Primitive.cpp:172-176, 193): x + t exactly
  pos[3 * v + 0] = raw[3 * v + 0] + trans[3 * m + 0];
  pos[3 * v + 1] = raw[3 * v + 1] + trans[3 * m + 1];
  pos[3 * v + 2] = raw[3 * v + 2] + trans[3 * m + 2];
}

__global__ void k_face(int nt, const float* pos, const int* idx, float* fn, float* area) {
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nt) return;
  const F3 p0 = make_f3(pos + 3 * idx[3 * f]), p1 = make_f3(pos + 3 * idx[3 * f + 1]),
           p2 = make_f3(pos + 3 * idx[3 * f + 2]);
  const F3 c = cross(p1 - p0, p2 - p0);
  const float len = length(c);
  fn[3 * f + 0] = c.x / len; fn[3 * f + 1] = c.y / len; fn[3 * f + 2] = c.z / len;
  area[f] = len * 0.5f;
}

// averaged face normals, normalised (Primitive.cpp:323-340); faces are summed
// in increasing face order for determinism.
__global__ void k_vnormal(int nv, const int* off, const int* list, const float* fn, float* vn) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  F3 s(0.f, 0.f, 0.f);
  const int a = off[v], b = off[v + 1];
  for (int k = a; k < b; k++) s = s + make_f3(fn + 3 * list[k]);
  const float cnt = (float)(b - a);
  s = s / cnt;
  const F3 n = normalize(s);
  vn[3 * v + 0] = n.x; vn[3 * v + 1] = n.y; vn[3 * v + 2] = n.z;
}

__global__ void k_light_func(int n, const int* tris, const int* emitter_id, const float* lum,
                             const float* area, float* func) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const int t = tris[e];
  func[e] = lum[emitter_id[t]] * area[t];
}

// Secondary edges (Edge.cpp:42-88): boundary, or non-coplanar and convex.
__global__ void k_sec_edges(int ne, const int* edges, const float* pos, const float* fn, float* func) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  const int v0 = edges[5 * e], v1 = edges[5 * e + 1], f0 = edges[5 * e + 2], f1 = edges[5 * e + 3],
            v2 = edges[5 * e + 4];
  const F3 p0 = make_f3(pos + 3 * v0), p1 = make_f3(pos + 3 * v1), p2 = make_f3(pos + 3 * v2);
  bool valid;
  if (f1 < 0) {
    valid = true;
  } else {
    const F3 n0 = make_f3(fn + 3 * f0), n1 = make_f3(fn + 3 * f1);
    const bool valid0 = dot(n0, n1) < 1.0f - 1e-6f;
    const F3 e2 = normalize(p2 - p0);
    const bool valid1 = dot(n1, e2) < -kEdgeEps;
    valid = valid0 && valid1;
  }
  func[e] = valid ? length(p1 - p0) : 0.f;
}

// Distribution1D::SetFunction over n weights: cdf_i = (S_i / n) / (S_n / n),
// prefix sums accumulated in double in a fixed order.
__global__ void k_cdf(int n, const float* func, float* cdf, float* integral_out) {
  __shared__ double part[1024];
  const int T = blockDim.x;
  const int tid = threadIdx.x;
  const int chunk = (n + T - 1) / T;
  const int a = min(n, tid * chunk), b = min(n, a + chunk);
  double s = 0.0;
  for (int i = a; i < b; i++) s += (double)func[i];
  part[tid] = s;
  __syncthreads();
  if (tid == 0) {
    double run = 0.0;
    for (int i = 0; i < T; i++) { double x = part[i]; part[i] = run; run += x; }
  }
  __syncthreads();
  const float inv_size = 1.0f / (float)n;
  double run = part[tid];
  for (int i = a; i < b; i++) {
    run += (double)func[i];
    cdf[i] = (float)run * inv_size;
  }
  __syncthreads();
  __shared__ float integral;
  if (tid == 0) { integral = n > 0 ? cdf[n - 1] : 0.f; if (integral_out) *integral_out = integral; }
  __syncthreads();
  if (integral > 0.f)
    for (int i = a; i < b; i++) cdf[i] = cdf[i] / integral;
}

// ---------------------------------------------------------------------------
// LBVH (Karras, "Maximizing Parallelism in the Construction of BVHs,
// Octrees, and k-d Trees", HPG 2012)
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned int ordered(float f) {
  unsigned int u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float unordered(unsigned int u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__global__ void k_bounds_init(unsigned int* b) {
  if (threadIdx.x < 3) { b[threadIdx.x] = 0xffffffffu; b[3 + threadIdx.x] = 0u; }
}
__global__ void k_bounds(int nt, const float* pos, const int* idx, unsigned int* b) {
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  F3 c(0.f, 0.f, 0.f);
  bool ok = f < nt;
  if (ok) {
    const F3 p0 = make_f3(pos + 3 * idx[3 * f]), p1 = make_f3(pos + 3 * idx[3 * f + 1]),
             p2 = make_f3(pos + 3 * idx[3 * f + 2]);
    c = (p0 + p1 + p2) * (1.f / 3.f);
  }
  for (int k = 0; k < 3; k++) {
    unsigned int lo = ok ? ordered(c[k]) : 0xffffffffu, hi = ok ? ordered(c[k]) : 0u;
    for (int o = 16; o > 0; o >>= 1) {
      lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
      hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if ((threadIdx.x & 31) == 0) { atomicMin(&b[k], lo); atomicMax(&b[3 + k], hi); }
  }
}

__device__ __forceinline__ unsigned int expand_bits(unsigned int v) {
  v = (v * 0x00010001u) & 0xFF0000FFu;
  v = (v * 0x00000101u) & 0x0F00F00Fu;
  v = (v * 0x00000011u) & 0xC30C30C3u;
  v = (v * 0x00000005u) & 0x49249249u;
  return v;
}

#ifndef TRN_LARGE_SPLIT
#define TRN_LARGE_SPLIT 1
#endif
__global__ void k_morton(int nt, const float* pos, const int* idx, const unsigned int* b,
                         unsigned long long* keys) {
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nt) return;
  const F3 p0 = make_f3(pos + 3 * idx[3 * f]), p1 = make_f3(pos + 3 * idx[3 * f + 1]),
           p2 = make_f3(pos + 3 * idx[3 * f + 2]);
  const F3 c = (p0 + p1 + p2) * (1.f / 3.f);
  unsigned int m[3];
  for (int k = 0; k < 3; k++) {
    const float lo = unordered(b[k]), hi = unordered(b[3 + k]);
    const float ext = hi - lo;
    float x = ext > 0.f ? (c[k] - lo) / ext : 0.5f;
    x = fminf(fmaxf(x * 1024.f, 0.f), 1023.f);
    m[k] = expand_bits((unsigned int)x);
  }
  unsigned int code = (m[0] << 2) | (m[1] << 1) | m[2];
  // Oversized triangles (box diagonal above 1/16 of the scene's, e.g. a ground
  // plane) get a code above the 30-bit Morton range: they sort last and the
  // root split puts them in their own subtree instead of inflating the boxes
  // of every ancestor among the small triangles near their centroids.
  float sd2 = 0.f, td2 = 0.f;
  for (int k = 0; k < 3; k++) {
    const float e = unordered(b[3 + k]) - unordered(b[k]);
    const float t = fmaxf(fmaxf(p0[k], p1[k]), p2[k]) - fminf(fminf(p0[k], p1[k]), p2[k]);
    sd2 += e * e;
    td2 += t * t;
  }
  if (TRN_LARGE_SPLIT && td2 * 256.f > sd2) code = 1u << 30;
  keys[f] = ((unsigned long long)code << 32) | (unsigned int)f;
}

__device__ __forceinline__ int delta(const unsigned long long* k, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  return __clzll(k[i] ^ k[j]);
}

// internal node i covers sorted leaves [first, last]; children are encoded as
// internal index (>= 0) or ~leaf (< 0). parent[] indexes internal nodes for
// slots 0..n-2 and leaves at n-1+leaf.
__global__ void k_karras(int n, const unsigned long long* keys, BvhNode* nodes, int* parent) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  const int d = (delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
  const int dmin = delta(keys, n, i, i - d);
  int lmax = 2;
  while (delta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
  int l = 0;
  for (int t = lmax >> 1; t >= 1; t >>= 1)
    if (delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
  const int j = i + l * d;
  const int dnode = delta(keys, n, i, j);
  int s = 0;
  int t = l;
  do {
    t = (t + 1) >> 1;
    if (delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
  } while (t > 1);
  const int gamma = i + s * d + min(d, 0);
  const int first = min(i, j), last = max(i, j);
  int c0, c1;
  if (first == gamma) { c0 = ~gamma; parent[n - 1 + gamma] = i; }
  else { c0 = gamma; parent[gamma] = i; }
  if (last == gamma + 1) { c1 = ~(gamma + 1); parent[n - 1 + gamma + 1] = i; }
  else { c1 = gamma + 1; parent[gamma + 1] = i; }
  nodes[i].d = make_int4(c0, c1, 0, 0);
  if (i == 0) parent[0] = -1;
}

// ---------------------------------------------------------------------------
// PLOC build (Meister and Bittner 2018, "Parallel Locally-Ordered Clustering
// for Bounding Volume Construction"): clusters start as the Morton-ordered
// leaves; each round every cluster finds, within +-kPlocR positions, the
// neighbour whose union box has the smallest surface area, mutual nearest
// neighbours merge into a new internal node, and the survivors are compacted
// in order. The output has the LBVH's layout (internal nodes [0, T-1) with the
// root at 0, parent links for k_refit), so traversal and refit are unchanged.
// ---------------------------------------------------------------------------
#ifndef TRN_PLOC
#define TRN_PLOC 1
#endif
constexpr int kPlocR = 16;
constexpr int kPlocBlock = 256;

__global__ void k_ploc_init(int n, const unsigned long long* keys, const float* pos, const int* idx, int* cnode,
                            float* cbox) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int f = (int)(keys[i] & 0xffffffffull);
  const F3 p0 = make_f3(pos + 3 * idx[3 * f]), p1 = make_f3(pos + 3 * idx[3 * f + 1]),
           p2 = make_f3(pos + 3 * idx[3 * f + 2]);
  for (int k = 0; k < 3; k++) {
    cbox[6 * i + k] = fminf(fminf(p0[k], p1[k]), p2[k]);
    cbox[6 * i + 3 + k] = fmaxf(fmaxf(p0[k], p1[k]), p2[k]);
  }
  cnode[i] = ~i;
}

__device__ __forceinline__ float union_area(const float* a, const float* b) {
  const float dx = fmaxf(a[3], b[3]) - fminf(a[0], b[0]);
  const float dy = fmaxf(a[4], b[4]) - fminf(a[1], b[1]);
  const float dz = fmaxf(a[5], b[5]) - fminf(a[2], b[2]);
  return dx * dy + dy * dz + dz * dx;
}

// Nearest neighbour in the window; ties go to the smaller index, which keeps
// at least one mutual pair (the smallest index among the closest pairs).
__global__ void k_ploc_nn(int* count, const float* cbox, int* nn) {
  __shared__ float sb[(kPlocBlock + 2 * kPlocR) * 6];
  const int n = count[1];  // clusters of this round (the launch covers an upper bound)
  if (blockIdx.x == 0 && threadIdx.x == 0 && n > 1) count[2] += 1;  // rounds that merge
  if ((int)(blockIdx.x * kPlocBlock) >= n) return;
  const int start = blockIdx.x * kPlocBlock - kPlocR;
  for (int t = threadIdx.x; t < (kPlocBlock + 2 * kPlocR) * 6; t += blockDim.x) {
    const int c = start + t / 6;
    sb[t] = (c >= 0 && c < n) ? cbox[(size_t)6 * c + t % 6] : 0.f;
  }
  __syncthreads();
  const int i = blockIdx.x * kPlocBlock + threadIdx.x;
  if (i >= n) return;
  const float* bi = sb + 6 * (threadIdx.x + kPlocR);
  float best = 3.402823466e+38f;
  int bj = -1;
  const int j0 = max(0, i - kPlocR), j1 = min(n - 1, i + kPlocR);
  for (int j = j0; j <= j1; j++) {
    if (j == i) continue;
    const float a = union_area(bi, sb + 6 * (j - start));
    if (a < best) { best = a; bj = j; }
  }
  nn[i] = bj;
}

__global__ void k_ploc_merge(int nleaf, int nmax, const int* nn, const int* cnode, const float* cbox, int* onode,
                             float* obox, int* flag, BvhNode* nodes, int* parent, int* counter) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nmax) return;
  const int n = counter[1];
  if (i >= n) { flag[i] = 0; return; }
  const int j = nn[i];
  const float* bi = cbox + (size_t)6 * i;
  if (j >= 0 && nn[j] == i) {
    if (i > j) { flag[i] = 0; return; }
    const int id = nleaf - 2 - atomicAdd(counter, 1);
    const int a = cnode[i], b = cnode[j];
    nodes[id].d = make_int4(a, b, 0, 0);
    parent[a < 0 ? nleaf - 1 + ~a : a] = id;
    parent[b < 0 ? nleaf - 1 + ~b : b] = id;
    const float* bj = cbox + (size_t)6 * j;
    for (int k = 0; k < 3; k++) {
      obox[6 * i + k] = fminf(bi[k], bj[k]);
      obox[6 * i + 3 + k] = fmaxf(bi[3 + k], bj[3 + k]);
    }
    onode[i] = id;
  } else {
    for (int k = 0; k < 6; k++) obox[6 * i + k] = bi[k];
    onode[i] = cnode[i];
  }
  flag[i] = 1;
}

__global__ void k_ploc_compact(int nmax, const int* flag, const int* pos, const int* onode, const float* obox,
                               int* cnode, float* cbox, int* count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nmax) return;
  if (flag[i]) {
    const int d = pos[i];
    cnode[d] = onode[i];
    for (int k = 0; k < 6; k++) cbox[6 * d + k] = obox[6 * i + k];
  }
  if (i == nmax - 1) count[1] = pos[i] + flag[i];
}

__device__ __forceinline__ void write_child_box(BvhNode* nd, int side, const float lo[3], const float hi[3]) {
  float* a = reinterpret_cast<float*>(nd);
  if (side == 0) {
    a[0] = lo[0]; a[1] = lo[1]; a[2] = lo[2]; a[3] = hi[0]; a[4] = hi[1]; a[5] = hi[2];
  } else {
    a[6] = lo[0]; a[7] = lo[1]; a[8] = lo[2]; a[9] = hi[0]; a[10] = hi[1]; a[11] = hi[2];
  }
}

// Leaves write their (padded) boxes into the parent; the second thread to
// arrive at an internal node merges both child boxes and moves up.
__global__ void k_refit(int n, const unsigned long long* keys, const float* pos, const int* idx,
                        BvhNode* nodes, const int* parent, int* flags, float4* tri_verts) {
  int leaf = blockIdx.x * blockDim.x + threadIdx.x;
  if (leaf >= n) return;
  const int f = (int)(keys[leaf] & 0xffffffffull);
  const F3 p0 = make_f3(pos + 3 * idx[3 * f]), p1 = make_f3(pos + 3 * idx[3 * f + 1]),
           p2 = make_f3(pos + 3 * idx[3 * f + 2]);
  tri_verts[3 * leaf + 0] = make_float4(p0.x, p0.y, p0.z, __int_as_float(f));
  tri_verts[3 * leaf + 1] = make_float4(p1.x, p1.y, p1.z, 0.f);
  tri_verts[3 * leaf + 2] = make_float4(p2.x, p2.y, p2.z, 0.f);
  float lo[3], hi[3];
  for (int k = 0; k < 3; k++) {
    lo[k] = fminf(fminf(p0[k], p1[k]), p2[k]);
    hi[k] = fmaxf(fmaxf(p0[k], p1[k]), p2[k]);
    const float pad = 1e-6f * fmaxf(fabsf(lo[k]), fabsf(hi[k])) + 1e-30f;
    lo[k] -= pad; hi[k] += pad;
  }
  if (n == 1) {
    write_child_box(&nodes[0], 0, lo, hi);
    return;
  }
  int child = ~leaf;
  int p = parent[n - 1 + leaf];
  while (p >= 0) {
    BvhNode* nd = &nodes[p];
    const int side = (nd->d.x == child) ? 0 : 1;
    write_child_box(nd, side, lo, hi);
    __threadfence();
    if (atomicAdd(&flags[p], 1) == 0) return;
    __threadfence();
    const float* a = reinterpret_cast<const float*>(nd);
    // read both child boxes (volatile: the sibling wrote one of them)
    const volatile float* va = a;
    for (int k = 0; k < 3; k++) {
      lo[k] = fminf(va[k], va[6 + k]);
      hi[k] = fmaxf(va[3 + k], va[9 + k]);
    }
    child = p;
    p = parent[p];
  }
}


// ---------------------------------------------------------------------------
// Multi-triangle leaves: every subtree of the binary LBVH with at most
// TRN_LEAF_MAX triangles becomes one leaf whose triangles are contiguous in
// ctri. cnodes keeps the binary nodes (same indices and child boxes) with
// such children re-encoded as leaves: ~(first | (count - 1) << 29). Nodes
// inside a collapsed subtree are not reached. A ray meets the same triangles
// or fewer node boxes; its result (closest (t, triangle id), or any hit)
// does not depend on the tree.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int leaf_code(int first, int count) { return ~(first | ((count - 1) << 29)); }

// subtree triangle counts, bottom-up from the leaves (the second child to
// arrive at a node continues, as in k_refit)
__global__ void k_leaf_counts(int n, const BvhNode* nodes, const int* parent, int* flags, int* cnt) {
  const int leaf = blockIdx.x * blockDim.x + threadIdx.x;
  if (leaf >= n) return;
  int p = parent[n - 1 + leaf];
  while (p >= 0) {
    __threadfence();
    if (atomicAdd(&flags[p], 1) == 0) return;
    __threadfence();
    const int4 d = nodes[p].d;
    const volatile int* vc = cnt;
    const int c = (d.x < 0 ? 1 : vc[d.x]) + (d.y < 0 ? 1 : vc[d.y]);
    cnt[p] = c;
    p = parent[p];
  }
}

// triangles each reachable node's leaf children hold (0 inside a collapsed
// subtree): the scan of this gives each node its first ctri slot
__global__ void k_leaf_slots(int ninner, const BvhNode* nodes, const int* cnt, int* slots) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ninner) return;
  if (cnt[i] <= TRN_LEAF_MAX) { slots[i] = 0; return; }
  const int4 d = nodes[i].d;
  int k = 0;
  for (int side = 0; side < 2; side++) {
    const int c = side ? d.y : d.x;
    k += c < 0 ? 1 : (cnt[c] <= TRN_LEAF_MAX ? cnt[c] : 0);
  }
  slots[i] = k;
}

__device__ __forceinline__ void copy_tri(const float4* src, int leaf, float4* dst, int slot) {
  dst[3 * slot + 0] = src[3 * leaf + 0];
  dst[3 * slot + 1] = src[3 * leaf + 1];
  dst[3 * slot + 2] = src[3 * leaf + 2];
}

__global__ void k_leaf_collapse(int ninner, const BvhNode* nodes, const int* cnt, const int* base,
                                const float4* tri_verts, BvhNode* cnodes, float4* ctri) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ninner || cnt[i] <= TRN_LEAF_MAX) return;
  BvhNode o = nodes[i];
  int slot = base[i];
  int child[2];
  for (int side = 0; side < 2; side++) {
    const int c = side ? o.d.y : o.d.x;
    if (c < 0) {
      copy_tri(tri_verts, ~c, ctri, slot);
      child[side] = leaf_code(slot, 1);
      slot += 1;
    } else if (cnt[c] <= TRN_LEAF_MAX) {
      // gather the subtree's triangles (at most TRN_LEAF_MAX leaves)
      const int first = slot;
      int stack[TRN_LEAF_MAX];
      int sp = 0;
      stack[sp++] = c;
      while (sp > 0) {
        const int4 d = nodes[stack[--sp]].d;
        for (int k = 0; k < 2; k++) {  // (the order within a leaf is immaterial)
          const int g = k ? d.y : d.x;
          if (g < 0) {
            copy_tri(tri_verts, ~g, ctri, slot++);
          } else if (sp < TRN_LEAF_MAX) {
            stack[sp++] = g;
          }
        }
      }
      child[side] = leaf_code(first, cnt[c]);
    } else {
      child[side] = c;
    }
  }
  o.d = make_int4(child[0], child[1], 0, 0);
  cnodes[i] = o;
}

// ---------------------------------------------------------------------------
// collapse the binary LBVH into the 8-wide quantised BVH (top-down, one
// level of wide nodes per launch). Each wide node takes the two children of
// its binary node and repeatedly opens the internal child with the largest
// surface area until it holds 8 children or only leaves.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float box_area(const float* lo, const float* hi) {
  const float dx = fmaxf(hi[0] - lo[0], 0.f), dy = fmaxf(hi[1] - lo[1], 0.f), dz = fmaxf(hi[2] - lo[2], 0.f);
  return dx * dy + dy * dz + dz * dx;
}

__device__ __forceinline__ void child_box(const BvhNode& n, int side, float* lo, float* hi) {
  const float* a = reinterpret_cast<const float*>(&n);
  const int o = side ? 6 : 0;
  lo[0] = a[o]; lo[1] = a[o + 1]; lo[2] = a[o + 2];
  hi[0] = a[o + 3]; hi[1] = a[o + 4]; hi[2] = a[o + 5];
}

__device__ __forceinline__ float qdecode(int q, float scale, float origin) {
  return __fmaf_rn((float)q, scale, origin);
}

__global__ void k_collapse(int n_in, const int2* in, int2* out, int* counters, const BvhNode* nodes,
                           const float4* tri_verts, WNode* wnodes, float4* wtri) {
  const int item = blockIdx.x * blockDim.x + threadIdx.x;
  if (item >= n_in) return;
  const int b = in[item].x, w = in[item].y;
  int cid[8];
  float clo[8][3], chi[8][3];
  const BvhNode nb = nodes[b];
  cid[0] = nb.d.x; child_box(nb, 0, clo[0], chi[0]);
  cid[1] = nb.d.y; child_box(nb, 1, clo[1], chi[1]);
  int n = 2;
  while (n < 8) {
    int best = -1;
    float best_a = -1.f;
    for (int i = 0; i < n; i++)
      if (cid[i] >= 0) {
        const float a = box_area(clo[i], chi[i]);
        if (a > best_a) { best_a = a; best = i; }
      }
    if (best < 0) break;
    const BvhNode c = nodes[cid[best]];
    cid[best] = c.d.x; child_box(c, 0, clo[best], chi[best]);
    cid[n] = c.d.y; child_box(c, 1, clo[n], chi[n]);
    n++;
  }
  int ni = 0, nl = 0;
  for (int i = 0; i < n; i++) (cid[i] >= 0 ? ni : nl)++;
  const int child_base = ni ? atomicAdd(&counters[0], ni) : 0;
  const int tri_base = nl ? atomicAdd(&counters[1], nl) : 0;
  const int qbase = ni ? atomicAdd(&counters[2], ni) : 0;
  WNode wn;
  float lo[3] = {3.4e38f, 3.4e38f, 3.4e38f}, hi[3] = {-3.4e38f, -3.4e38f, -3.4e38f};
  for (int i = 0; i < n; i++)
    for (int k = 0; k < 3; k++) { lo[k] = fminf(lo[k], clo[i][k]); hi[k] = fmaxf(hi[k], chi[i][k]); }
  float scale[3];
  unsigned char ebias[3];
  for (int k = 0; k < 3; k++) {
    const float ext = hi[k] - lo[k];
    int e = -100;
    if (ext > 0.f) {
      int ee;
      const float m = frexpf(ext / 255.f, &ee);
      e = (m == 0.5f) ? ee - 1 : ee;
      while (ldexpf(255.f, e) < ext) e++;
    }
    e = max(-126, min(127, e));
    ebias[k] = (unsigned char)(e + 127);
    scale[k] = __uint_as_float((unsigned)(e + 127) << 23);
  }
  wn.ox = lo[0]; wn.oy = lo[1]; wn.oz = lo[2];
  wn.ex = ebias[0]; wn.ey = ebias[1]; wn.ez = ebias[2];
  wn.nchild = (unsigned char)n;
  wn.child_base = child_base;
  wn.tri_base = tri_base;
  int ii = 0, il = 0;
  for (int i = 0; i < 8; i++) {
    if (i >= n) {
      wn.meta[i] = 0;
      for (int k = 0; k < 3; k++) { wn.qlo[k][i] = 255; wn.qhi[k][i] = 0; }
      continue;
    }
    for (int k = 0; k < 3; k++) {
      int ql = (int)floorf((clo[i][k] - lo[k]) / scale[k]);
      int qh = (int)ceilf((chi[i][k] - lo[k]) / scale[k]);
      ql = max(0, min(255, ql));
      qh = max(0, min(255, qh));
      while (ql > 0 && qdecode(ql, scale[k], lo[k]) > clo[i][k]) ql--;
      while (qh < 255 && qdecode(qh, scale[k], lo[k]) < chi[i][k]) qh++;
      wn.qlo[k][i] = (unsigned char)ql;
      wn.qhi[k][i] = (unsigned char)qh;
    }
    if (cid[i] >= 0) {
      wn.meta[i] = (unsigned char)(0x80 | ii);
      out[qbase + ii] = make_int2(cid[i], child_base + ii);
      ii++;
    } else {
      const int leaf = ~cid[i];
      wn.meta[i] = (unsigned char)(0xC0 | il);
      const int slot = tri_base + il;
      wtri[3 * slot + 0] = tri_verts[3 * leaf + 0];
      wtri[3 * slot + 1] = tri_verts[3 * leaf + 1];
      wtri[3 * slot + 2] = tri_verts[3 * leaf + 2];
      il++;
    }
  }
  wnodes[w] = wn;
}

// ---------------------------------------------------------------------------
// geometry-chain adjoint
// ---------------------------------------------------------------------------
// vertex normal n_v = normalize(s_v / c_v), s_v = sum of incident face normals
// -> dL/d(face normal) for every incident face, then the face normal
// n_f = c / |c| with c = cross(p1 - p0, p2 - p0) -> dL/d(positions).
__global__ void k_vnormal_adj(int nv, const int* off, const int* list, const float* fn, const float* g_vn,
                              float* g_sum) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  F3 s(0.f, 0.f, 0.f);
  const int a = off[v], b = off[v + 1];
  for (int k = a; k < b; k++) s = s + make_f3(fn + 3 * list[k]);
  const float cnt = (float)(b - a);
  const F3 m = s / cnt;
  const float len = length(m);
  const F3 n = m / len;
  const F3 g = make_f3(g_vn + 3 * v);
  // d normalize(m)/dm^T g = (g - n (n.g)) / |m|
  const F3 gm = (g - n * dot(n, g)) / len;
  const F3 gs = gm / cnt;
  g_sum[3 * v + 0] = gs.x; g_sum[3 * v + 1] = gs.y; g_sum[3 * v + 2] = gs.z;
}

__device__ __forceinline__ void atomic_add3(float* a, const F3& g) {
  atomicAdd(a, g.x); atomicAdd(a + 1, g.y); atomicAdd(a + 2, g.z);
}

__global__ void k_face_adj(int nt, const float* pos, const int* idx, const float* g_sum, float* g_pos) {
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nt) return;
  const int i0 = idx[3 * f], i1 = idx[3 * f + 1], i2 = idx[3 * f + 2];
  const F3 gn = make_f3(g_sum + 3 * i0) + make_f3(g_sum + 3 * i1) + make_f3(g_sum + 3 * i2);
  if (gn.x == 0.f && gn.y == 0.f && gn.z == 0.f) return;
  const F3 p0 = make_f3(pos + 3 * i0), p1 = make_f3(pos + 3 * i1), p2 = make_f3(pos + 3 * i2);
  const F3 e1 = p1 - p0, e2 = p2 - p0;
  const F3 c = cross(e1, e2);
  const float len = length(c);
  const F3 n = c / len;
  const F3 gc = (gn - n * dot(n, gn)) / len;
  const F3 ge1 = cross(e2, gc), ge2 = cross(gc, e1);
  atomic_add3(g_pos + 3 * i1, ge1);
  atomic_add3(g_pos + 3 * i2, ge2);
  atomic_add3(g_pos + 3 * i0, -(ge1 + ge2));
}

// dL/d translation_m = sum of dL/dP over the vertices of mesh m
__global__ void k_translation_adj(int nv, const int* vmesh, const float* g_pos, float* g_trans) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  const bool ok = v < nv;
  const int m = ok ? vmesh[v] : -1;
  F3 g = ok ? make_f3(g_pos + 3 * v) : F3(0.f, 0.f, 0.f);
  // warp-aggregate runs of the same mesh id
  const unsigned mask = __match_any_sync(0xffffffffu, m);
  const int leader = __ffs(mask) - 1;
  for (int k = 0; k < 3; k++) {
    float x = g[k];
    float sum = 0.f;
    for (int l = 0; l < 32; l++) {
      float y = __shfl_sync(0xffffffffu, x, l);
      if (mask & (1u << l)) sum += y;
    }
    g[k] = sum;
  }
  if (ok && (int)(threadIdx.x & 31) == leader) atomic_add3(g_trans + 3 * m, g);
}

static inline int nblk(long long n, int b = 256) { return (int)((n + b - 1) / b); }

}  // namespace trn

using namespace trn;

// ---------------------------------------------------------------------------
// host helpers
// ---------------------------------------------------------------------------
namespace {

template <class T>
int dev_alloc_copy(T** dst, const T* src, size_t n) {
  *dst = nullptr;
  if (n == 0) return 0;
  TRN_CUDA_TRY(cudaMalloc((void**)dst, n * sizeof(T)));
  if (src) TRN_CUDA_TRY(cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice));
  else TRN_CUDA_TRY(cudaMemset(*dst, 0, n * sizeof(T)));
  return 0;
}

// ObjMesh::processEdges (ObjMesh.cpp:584-632): unique undirected edges in
// (min vertex, max vertex) order; face0/face1 are the first two faces using
// the edge in face order, v2 the vertex opposite the edge in face0; an edge
// with other than exactly two faces is a boundary edge (face1 = -1).
void build_edges(int nt, const int* idx, std::vector<int>& out) {
  struct HE { unsigned long long key; int face; int third; };
  std::vector<HE> he;
  he.reserve((size_t)nt * 3);
  for (int i = 0; i < nt; i++)
    for (int j = 0; j < 3; j++) {
      int a = idx[3 * i + j], b = idx[3 * i + (j + 1) % 3], c = idx[3 * i + (j + 2) % 3];
      unsigned lo = (unsigned)std::min(a, b), hi = (unsigned)std::max(a, b);
      he.push_back({((unsigned long long)lo << 32) | hi, i, c});
    }
  std::stable_sort(he.begin(), he.end(), [](const HE& x, const HE& y) { return x.key < y.key; });
  out.clear();
  for (size_t s = 0; s < he.size();) {
    size_t e = s;
    while (e < he.size() && he[e].key == he[s].key) e++;
    const int cnt = (int)(e - s);
    const int v0 = (int)(he[s].key >> 32), v1 = (int)(he[s].key & 0xffffffffu);
    out.push_back(v0);
    out.push_back(v1);
    out.push_back(he[s].face);
    out.push_back(cnt == 2 ? he[s + 1].face : -1);
    out.push_back(he[s].third);
    s = e;
  }
}

// ---- 4x4 double matrices for the camera (EDXUtil/Math/Matrix.cpp) --------
struct M4 { double m[4][4]; };
M4 mat_id() { M4 r{}; for (int i = 0; i < 4; i++) r.m[i][i] = 1.0; return r; }
M4 mat_mul(const M4& a, const M4& b) {
  M4 r{};
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      double s = 0.0;
      for (int k = 0; k < 4; k++) s += a.m[i][k] * b.m[k][j];
      r.m[i][j] = s;
    }
  return r;
}
M4 mat_scale(double x, double y, double z) { M4 r = mat_id(); r.m[0][0] = x; r.m[1][1] = y; r.m[2][2] = z; return r; }
M4 mat_translate(double x, double y, double z) { M4 r = mat_id(); r.m[0][3] = x; r.m[1][3] = y; r.m[2][3] = z; return r; }
M4 mat_inv(const M4& a) {
  double m[4][8];
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 8; j++) m[i][j] = j < 4 ? a.m[i][j] : (j - 4 == i ? 1.0 : 0.0);
  for (int c = 0; c < 4; c++) {
    int piv = c;
    for (int r = c + 1; r < 4; r++) if (fabs(m[r][c]) > fabs(m[piv][c])) piv = r;
    if (piv != c) for (int j = 0; j < 8; j++) std::swap(m[c][j], m[piv][j]);
    const double d = m[c][c];
    for (int j = 0; j < 8; j++) m[c][j] /= d;
    for (int r = 0; r < 4; r++) {
      if (r == c) continue;
      const double f = m[r][c];
      for (int j = 0; j < 8; j++) m[r][j] -= f * m[c][j];
    }
  }
  M4 r;
  for (int i = 0; i < 4; i++) for (int j = 0; j < 4; j++) r.m[i][j] = m[i][4 + j];
  return r;
}
void mat_store(const M4& a, float* out) {
  for (int i = 0; i < 4; i++) for (int j = 0; j < 4; j++) out[4 * i + j] = (float)a.m[i][j];
}
void xform_h(const M4& a, const double p[4], double out[3]) {
  double r[4];
  for (int i = 0; i < 4; i++) r[i] = a.m[i][0] * p[0] + a.m[i][1] * p[1] + a.m[i][2] * p[2] + a.m[i][3] * p[3];
  out[0] = r[0] / r[3]; out[1] = r[1] / r[3]; out[2] = r[2] / r[3];
}

}  // namespace

// ---------------------------------------------------------------------------
// C-ABI
// ---------------------------------------------------------------------------
extern "C" {

const char* trn_last_error(void) { return g_err.c_str(); }
const char* trn_version(void) { return "trn 0.1 sm_100a"; }

int trn_camera_init(trn_camera* out, const float pos[3], const float target[3], const float up[3], int width,
                    int height, float fov_deg) {
  if (!out || !pos || !target || !up || width <= 0 || height <= 0) {
    set_error("trn_camera_init: invalid arguments");
    return -1;
  }
  // BaseCamera::Init (BaseCamera.cpp:45-72) + Matrix::LookAt (Matrix.cpp:181-209)
  double P[3] = {pos[0], pos[1], pos[2]}, Tg[3] = {target[0], target[1], target[2]}, U[3] = {up[0], up[1], up[2]};
  auto norm3 = [](double* v) { double l = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); v[0] /= l; v[1] /= l; v[2] /= l; };
  auto cross3 = [](const double* a, const double* b, double* o) {
    o[0] = a[1] * b[2] - a[2] * b[1]; o[1] = a[2] * b[0] - a[0] * b[2]; o[2] = a[0] * b[1] - a[1] * b[0];
  };
  double dir[3] = {Tg[0] - P[0], Tg[1] - P[1], Tg[2] - P[2]};
  norm3(dir);
  double upn[3] = {U[0], U[1], U[2]};
  norm3(upn);
  double right[3]; cross3(upn, dir, right); norm3(right);
  double nup[3]; cross3(dir, right, nup);
  M4 cam2world = mat_id();
  for (int i = 0; i < 3; i++) { cam2world.m[i][0] = right[i]; cam2world.m[i][1] = nup[i]; cam2world.m[i][2] = dir[i]; cam2world.m[i][3] = P[i]; }
  const M4 view = mat_inv(cam2world);
  const M4 view_inv = cam2world;
  // BaseCamera::Resize (BaseCamera.cpp:74-88) + Matrix::Perspective (Matrix.cpp:211-220)
  const double near_clip = 1.0, far_clip = 1000.0;  // Camera::Init defaults (Camera.h)
  const double ratio = (double)width / (double)height;
  M4 persp = mat_id();
  persp.m[2][2] = far_clip / (far_clip - near_clip);
  persp.m[2][3] = -far_clip * near_clip / (far_clip - near_clip);
  persp.m[3][2] = 1.0; persp.m[3][3] = 0.0;
  const double inv_tan = 1.0 / tan(fov_deg * M_PI / 180.0 / 2.0);
  const M4 proj = mat_mul(mat_scale(inv_tan / ratio, inv_tan, 1.0), persp);
  const M4 screen_to_raster = mat_mul(mat_mul(mat_scale(width, height, 1.0), mat_scale(-0.5, -0.5, 1.0)),
                                      mat_translate(-1.0, -1.0, 0.0));
  const M4 raster_to_camera = mat_mul(mat_inv(proj), mat_inv(screen_to_raster));
  const M4 camera_to_raster = mat_inv(raster_to_camera);
  const M4 raster_to_world = mat_mul(view_inv, raster_to_camera);
  // Camera::Resize (Camera.cpp:105-137)
  const M4 camera_to_sample = mat_mul(mat_scale(1.0 / width, 1.0 / height, 1.0), camera_to_raster);
  const M4 sample_to_camera_img = mat_mul(raster_to_camera, mat_scale(width, height, 1.0));
  double v00[3], v10[3], v11[3], vc[3];
  const double q00[4] = {0, 0, 0, 1}, q10[4] = {1, 0, 0, 1}, q11[4] = {1, 1, 0, 1}, qc[4] = {0.5, 0.5, 0, 1};
  xform_h(sample_to_camera_img, q00, v00); xform_h(sample_to_camera_img, q10, v10);
  xform_h(sample_to_camera_img, q11, v11); xform_h(sample_to_camera_img, qc, vc);
  double hz[3] = {v00[0] - v10[0], v00[1] - v10[1], v00[2] - v10[2]};
  double vt[3] = {v11[0] - v10[0], v11[1] - v10[1], v11[2] - v10[2]};
  const double lx = sqrt(hz[0] * hz[0] + hz[1] * hz[1] + hz[2] * hz[2]);
  const double ly = sqrt(vt[0] * vt[0] + vt[1] * vt[1] + vt[2] * vt[2]);
  const double inv_area = 1.0 / (lx * ly) * (vc[0] * vc[0] + vc[1] * vc[1] + vc[2] * vc[2]);
  out->width = width; out->height = height;
  for (int i = 0; i < 3; i++) { out->pos[i] = pos[i]; out->dir[i] = (float)dir[i]; }
  mat_store(raster_to_camera, out->raster_to_camera);
  mat_store(view_inv, out->view_inv);
  mat_store(mat_mul(camera_to_sample, view), out->world_to_sample);
  mat_store(mat_inv(camera_to_sample), out->sample_to_camera);
  mat_store(raster_to_world, out->raster_to_world);
  out->inv_area = (float)inv_area;
  out->plane_len_x = (float)lx;
  out->plane_len_y = (float)ly;
  return 0;
}

long long trn_mesh_edges(int num_triangles, const int* indices, int* out, long long cap) {
  if (num_triangles < 0 || (num_triangles > 0 && !indices) || cap < 0 || (cap > 0 && !out)) {
    set_error("trn_mesh_edges: invalid arguments");
    return -1;
  }
  std::vector<int> rows;
  build_edges(num_triangles, indices, rows);
  const long long n = (long long)(rows.size() / 5);
  if (cap > 0) std::copy(rows.begin(), rows.begin() + 5 * std::min(n, cap), out);
  return n;
}

int trn_scene_create(const trn_scene_desc* d, trn_scene** out) {
  if (!d || !out) { set_error("trn_scene_create: null argument"); return -1; }
  *out = nullptr;
  if (d->num_vertices <= 0 || d->num_triangles <= 0 || !d->positions || !d->indices || !d->vertex_mesh ||
      !d->triangle_mesh || d->num_meshes <= 0 || !d->mesh_bsdf || !d->mesh_light || !d->mesh_smooth ||
      d->num_bsdfs <= 0 || !d->bsdfs) {
    set_error("trn_scene_create: incomplete scene description");
    return -1;
  }
  const int nv = d->num_vertices, nt = d->num_triangles, nm = d->num_meshes;
  for (int i = 0; i < 3 * nt; i++)
    if (d->indices[i] < 0 || d->indices[i] >= nv) { set_error("trn_scene_create: index out of range"); return -1; }
  for (int i = 0; i < nv; i++)
    if (d->vertex_mesh[i] < 0 || d->vertex_mesh[i] >= nm) { set_error("trn_scene_create: vertex_mesh out of range"); return -1; }
  for (int i = 0; i < nt; i++)
    if (d->triangle_mesh[i] < 0 || d->triangle_mesh[i] >= nm) { set_error("trn_scene_create: triangle_mesh out of range"); return -1; }
  for (int m = 0; m < nm; m++) {
    if (d->mesh_bsdf[m] < 0 || d->mesh_bsdf[m] >= d->num_bsdfs) { set_error("trn_scene_create: mesh_bsdf out of range"); return -1; }
    if (d->mesh_light[m] >= d->num_lights) { set_error("trn_scene_create: mesh_light out of range"); return -1; }
  }
  if (d->num_lights > 64) { set_error("trn_scene_create: at most 64 lights"); return -1; }
  if (d->uv_indices) {
    for (int i = 0; i < 3 * nt; i++)
      if (d->uv_indices[i] < 0 || d->uv_indices[i] >= d->num_uvs) { set_error("trn_scene_create: uv index out of range"); return -1; }
  }
  for (int b = 0; b < d->num_bsdfs; b++) {
    const trn_bsdf& x = d->bsdfs[b];
    if (x.type != 0 && x.type != 1) { set_error("trn_scene_create: unknown bsdf type"); return -1; }
    if (x.texture >= d->num_textures) { set_error("trn_scene_create: bsdf texture out of range"); return -1; }
  }
  trn_scene* s = new trn_scene();
  auto fail = [&]() { trn_scene_destroy(s); return -1; };
  s->nv = nv; s->nt = nt; s->nmesh = nm; s->nlight = d->num_lights; s->nbsdf = d->num_bsdfs;
  s->ntex = d->num_textures;
  // per-triangle attributes
  std::vector<unsigned char> smooth(nt);
  std::vector<int> bsdf(nt), emitter(nt), tri_to_emit(nt, -1), emit_tris;
  for (int i = 0; i < nt; i++) {
    const int m = d->triangle_mesh[i];
    smooth[i] = d->mesh_smooth[m];
    bsdf[i] = d->mesh_bsdf[m];
    emitter[i] = d->mesh_light[m];
    if (emitter[i] >= 0) { tri_to_emit[i] = (int)emit_tris.size(); emit_tris.push_back(i); }
  }
  s->n_emit = (int)emit_tris.size();
  // luminance per light (Scene.cpp:484-486)
  s->h_light_radiance.assign(d->light_radiance ? d->light_radiance : nullptr,
                             d->light_radiance ? d->light_radiance + 3 * d->num_lights : nullptr);
  std::vector<float> lum(std::max(1, d->num_lights), 0.f);
  for (int l = 0; l < d->num_lights; l++)
    lum[l] = 0.212671f * d->light_radiance[3 * l] + 0.715160f * d->light_radiance[3 * l + 1] +
             0.072169f * d->light_radiance[3 * l + 2];
  // vertex -> faces CSR in face order
  std::vector<int> off(nv + 1, 0), list(3 * (size_t)nt);
  for (int i = 0; i < 3 * nt; i++) off[d->indices[i] + 1]++;
  for (int v = 0; v < nv; v++) off[v + 1] += off[v];
  {
    std::vector<int> fill(off.begin(), off.end() - 1);
    for (int f = 0; f < nt; f++)
      for (int j = 0; j < 3; j++) list[fill[d->indices[3 * f + j]]++] = f;
  }
  std::vector<int> edges;
  build_edges(nt, d->indices, edges);
  s->ne = (int)edges.size() / 5;
  // textures
  std::vector<TexDesc> texs;
  long long ntexel = 0;
  for (int t = 0; t < d->num_textures; t++) {
    texs.push_back({d->textures[t].width, d->textures[t].height, ntexel});
    ntexel += (long long)d->textures[t].width * d->textures[t].height;
  }
  s->ntexel = ntexel;
  std::vector<float> texel_data((size_t)ntexel * 3);
  for (int t = 0; t < d->num_textures; t++)
    std::memcpy(texel_data.data() + 3 * texs[t].offset, d->textures[t].data,
                sizeof(float) * 3 * (size_t)d->textures[t].width * d->textures[t].height);
  s->h_bsdfs.resize(d->num_bsdfs);
  std::memcpy(s->h_bsdfs.data(), d->bsdfs, sizeof(BsdfDesc) * d->num_bsdfs);
  s->h_texs = texs;
  std::vector<float> trans(3 * nm, 0.f);
  if (d->mesh_translation) std::memcpy(trans.data(), d->mesh_translation, sizeof(float) * 3 * nm);
  std::vector<int> idx(d->indices, d->indices + 3 * nt);
  if (dev_alloc_copy(&s->raw_pos, d->positions, 3 * (size_t)nv) ||
      dev_alloc_copy(&s->translation, trans.data(), trans.size()) ||
      dev_alloc_copy(&s->texels, texel_data.data(), texel_data.size()) ||
      dev_alloc_copy(&s->pos, (const float*)nullptr, 3 * (size_t)nv) ||
      dev_alloc_copy(&s->idx, idx.data(), idx.size()) ||
      dev_alloc_copy(&s->fnormal, (const float*)nullptr, 3 * (size_t)nt) ||
      dev_alloc_copy(&s->area, (const float*)nullptr, (size_t)nt) ||
      dev_alloc_copy(&s->vnormal, (const float*)nullptr, 3 * (size_t)nv) ||
      dev_alloc_copy(&s->smooth, smooth.data(), smooth.size()) ||
      dev_alloc_copy(&s->bsdf_id, bsdf.data(), bsdf.size()) ||
      dev_alloc_copy(&s->emitter_id, emitter.data(), emitter.size()) ||
      dev_alloc_copy(&s->vert_mesh, d->vertex_mesh, (size_t)nv) ||
      dev_alloc_copy(&s->vf_off, off.data(), off.size()) ||
      dev_alloc_copy(&s->vf_list, list.data(), list.size()) ||
      dev_alloc_copy(&s->tri_to_emit, tri_to_emit.data(), tri_to_emit.size()) ||
      dev_alloc_copy(&s->emit_tris, emit_tris.data(), emit_tris.size()) ||
      dev_alloc_copy(&s->light_func, (const float*)nullptr, std::max<size_t>(1, emit_tris.size())) ||
      dev_alloc_copy(&s->light_cdf, (const float*)nullptr, std::max<size_t>(1, emit_tris.size())) ||
      dev_alloc_copy(&s->light_radiance, s->h_light_radiance.data(), s->h_light_radiance.size()) ||
      dev_alloc_copy(&s->light_integral_dev, (const float*)nullptr, 1) ||
      dev_alloc_copy(&s->bsdfs, s->h_bsdfs.data(), s->h_bsdfs.size()) ||
      dev_alloc_copy(&s->texs, texs.data(), std::max<size_t>(texs.size(), 0)) ||
      dev_alloc_copy(&s->edges, edges.data(), edges.size()) ||
      dev_alloc_copy(&s->sec_func, (const float*)nullptr, std::max<size_t>(1, (size_t)s->ne)) ||
      dev_alloc_copy(&s->sec_cdf, (const float*)nullptr, std::max<size_t>(1, (size_t)s->ne)) ||
      dev_alloc_copy(&s->sec_integral_dev, (const float*)nullptr, 1) ||
      dev_alloc_copy(&s->aq_poly, (const float*)nullptr, std::max<size_t>(1, (size_t)s->ne)) ||
      dev_alloc_copy(&s->aq_func, (const float*)nullptr, std::max<size_t>(1, (size_t)s->ne)) ||
      dev_alloc_copy(&s->aq_cdf, (const float*)nullptr, std::max<size_t>(1, (size_t)s->ne)) ||
      dev_alloc_copy(&s->aq_int, (const float*)nullptr, 2) ||
      dev_alloc_copy(&s->aq_box, (const float*)nullptr, 6 * std::max<size_t>(1, (size_t)s->ne)) ||
      dev_alloc_copy(&s->aq_edge, (const int*)nullptr, std::max<size_t>(1, (size_t)s->ne)) ||
      dev_alloc_copy(&s->aq_count, (const int*)nullptr, 4) ||
      dev_alloc_copy(&s->nodes, (const BvhNode*)nullptr, std::max(1, nt - 1)) ||
      dev_alloc_copy(&s->tri_verts, (const float4*)nullptr, 3 * (size_t)nt) ||
      dev_alloc_copy(&s->parent, (const int*)nullptr, 2 * (size_t)nt) ||
      dev_alloc_copy(&s->flags, (const int*)nullptr, std::max(1, nt - 1)) ||
      (TRN_LEAF_MAX > 1 && nt > TRN_LEAF_MAX &&
       (dev_alloc_copy(&s->cnodes, (const BvhNode*)nullptr, (size_t)nt - 1) ||
        dev_alloc_copy(&s->ctri, (const float4*)nullptr, 3 * (size_t)nt) ||
        dev_alloc_copy(&s->leaf_cnt, (const int*)nullptr, 3 * ((size_t)nt - 1)))) ||
      dev_alloc_copy(&s->keys, (const unsigned long long*)nullptr, (size_t)nt) ||
      dev_alloc_copy(&s->keys_alt, (const unsigned long long*)nullptr, (size_t)nt) ||
      dev_alloc_copy(&s->bounds, (const float*)nullptr, 6) ||
      dev_alloc_copy(&s->wnodes, (const WNode*)nullptr, std::max(1, nt)) ||
      dev_alloc_copy(&s->wtri, (const float4*)nullptr, 3 * (size_t)nt) ||
      dev_alloc_copy(&s->wqueue, (const int*)nullptr, 4 * (size_t)std::max(1, nt)) ||
      dev_alloc_copy(&s->wcount, (const int*)nullptr, 4) ||
      dev_alloc_copy(&s->g_pos, (const float*)nullptr, 3 * (size_t)nv) ||
      dev_alloc_copy(&s->g_vnormal, (const float*)nullptr, 3 * (size_t)nv) ||
      dev_alloc_copy(&s->g_texels, (const float*)nullptr, std::max<size_t>(3, 3 * (size_t)ntexel)) ||
      dev_alloc_copy(&s->g_translation, (const float*)nullptr, 3 * (size_t)nm) ||
      dev_alloc_copy(&s->err, (const int*)nullptr, 1) ||
      dev_alloc_copy(&s->stats, (const unsigned long long*)nullptr, 16))
    return fail();
  s->aq_cap = std::max<long long>(1, s->ne);
  if (d->uvs && d->uv_indices && d->num_uvs > 0) {
    s->nuv = d->num_uvs;
    if (dev_alloc_copy(&s->uv, d->uvs, 2 * (size_t)d->num_uvs) ||
        dev_alloc_copy(&s->uvidx, d->uv_indices, 3 * (size_t)nt))
      return fail();
  }
  for (int l = 0; l < 64; l++) s->light_lum[l] = l < d->num_lights ? lum[l] : 0.f;
  // radix sort scratch
  size_t bytes = 0;
  cub::DeviceRadixSort::SortKeys(nullptr, bytes, s->keys, s->keys_alt, nt);
  s->sort_tmp_bytes = bytes;
  if (cudaMalloc(&s->sort_tmp, bytes) != cudaSuccess) { set_error("trn_scene_create: out of memory"); return fail(); }
  if (s->cnodes) {
    size_t sb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, sb, s->leaf_cnt, s->leaf_cnt, nt - 1);
    s->leaf_scan_bytes = std::max<size_t>(sb, 16);
    if (cudaMalloc(&s->leaf_scan_tmp, s->leaf_scan_bytes) != cudaSuccess) {
      set_error("trn_scene_create: out of memory");
      return fail();
    }
  }
  if (TRN_PLOC) {
    size_t sb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, sb, s->ploc_flag, s->ploc_pos, nt);
    s->scan_tmp_bytes = sb;
    if (dev_alloc_copy(&s->ploc_node, (const int*)nullptr, 2 * (size_t)nt) ||
        dev_alloc_copy(&s->ploc_box, (const float*)nullptr, 12 * (size_t)nt) ||
        dev_alloc_copy(&s->ploc_nn, (const int*)nullptr, (size_t)nt) ||
        dev_alloc_copy(&s->ploc_flag, (const int*)nullptr, (size_t)nt) ||
        dev_alloc_copy(&s->ploc_pos, (const int*)nullptr, (size_t)nt) ||
        dev_alloc_copy(&s->ploc_count, (const int*)nullptr, 3) ||
        cudaMalloc(&s->scan_tmp, std::max<size_t>(sb, 16)) != cudaSuccess) {
      set_error("trn_scene_create: out of memory");
      return fail();
    }
  }
  *out = s;
  return 0;
}

int trn_scene_destroy(trn_scene* s) {
  if (!s) return 0;
  if (s->single) trn_viewset_destroy(s->single);
  s->single = nullptr;
  void* ptrs[] = {s->raw_pos, s->translation, s->texels, s->pos, s->idx, s->fnormal, s->area, s->vnormal,
                  s->smooth, s->uv, s->uvidx, s->bsdf_id, s->emitter_id, s->vert_mesh, s->vf_off, s->vf_list,
                  s->emit_tris, s->tri_to_emit, s->light_func, s->light_cdf, s->light_radiance,
                  s->light_integral_dev, s->bsdfs, s->texs, s->edges, s->sec_func, s->sec_cdf,
                  s->sec_integral_dev, s->nodes, s->tri_verts, s->parent, s->flags, s->keys, s->keys_alt,
                  s->sort_tmp, s->bounds, s->g_pos, s->g_vnormal, s->g_texels, s->g_translation, s->err,
                  s->stats, s->wnodes, s->wtri, s->wqueue, s->wcount, s->aq_poly, s->aq_func, s->aq_cdf,
                  s->aq_int, s->aq_box, s->aq_edge, s->aq_count, s->aq_eval, s->aq_flag, s->aq_prefix, s->ploc_node, s->ploc_box, s->ploc_nn, s->ploc_flag, s->ploc_pos, s->ploc_count,
                  s->scan_tmp, s->cnodes, s->ctri, s->leaf_cnt, s->leaf_scan_tmp};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  delete s;
  return 0;
}

}  // extern "C"

namespace {
// Primitive::Configure + ComputeFaceNormalAndDistrib + ComputeVertexNormal +
// ConfigureLight + ConstructSecEdgeList (everything but the acceleration structure)
int configure_geometry(trn_scene* s, cudaStream_t st) {
  const int nv = s->nv, nt = s->nt;
  k_transform<<<nblk(nv), 256, 0, st>>>(nv, s->raw_pos, s->vert_mesh, s->translation, s->pos);
  k_face<<<nblk(nt), 256, 0, st>>>(nt, s->pos, s->idx, s->fnormal, s->area);
  k_vnormal<<<nblk(nv), 256, 0, st>>>(nv, s->vf_off, s->vf_list, s->fnormal, s->vnormal);
  count_launch(3);
  // merged light distribution
  if (s->n_emit > 0) {
    float* lum_dev = nullptr;
    TRN_CUDA_TRY(cudaMallocAsync((void**)&lum_dev, sizeof(float) * 64, st));
    TRN_CUDA_TRY(cudaMemcpyAsync(lum_dev, s->light_lum, sizeof(float) * 64, cudaMemcpyHostToDevice, st));
    k_light_func<<<nblk(s->n_emit), 256, 0, st>>>(s->n_emit, s->emit_tris, s->emitter_id, lum_dev, s->area,
                                                   s->light_func);
    k_cdf<<<1, 1024, 0, st>>>(s->n_emit, s->light_func, s->light_cdf, s->light_integral_dev);
    count_launch(2);
    TRN_CUDA_TRY(cudaFreeAsync(lum_dev, st));
  }
  // secondary edge list
  if (s->ne > 0) {
    k_sec_edges<<<nblk(s->ne), 256, 0, st>>>(s->ne, s->edges, s->pos, s->fnormal, s->sec_func);
    k_cdf<<<1, 1024, 0, st>>>(s->ne, s->sec_func, s->sec_cdf, s->sec_integral_dev);
    count_launch(2);
  }
  return 0;
}
// Rebuild the collapsed arrays from the binary LBVH (after a build or refit).
int leaf_collapse(trn_scene* s, cudaStream_t st) {
  s->collapsed = false;
  if (!s->cnodes) return 0;
  const int nt = s->nt, ninner = nt - 1;
  int* cnt = s->leaf_cnt;
  int* slots = s->leaf_cnt + ninner;
  int* base = s->leaf_cnt + 2 * ninner;
  TRN_CUDA_TRY(cudaMemsetAsync(s->flags, 0, sizeof(int) * ninner, st));
  k_leaf_counts<<<nblk(nt), 256, 0, st>>>(nt, s->nodes, s->parent, s->flags, cnt);
  k_leaf_slots<<<nblk(ninner), 256, 0, st>>>(ninner, s->nodes, cnt, slots);
  size_t sb = s->leaf_scan_bytes;
  if (cub::DeviceScan::ExclusiveSum(s->leaf_scan_tmp, sb, slots, base, ninner, st) != cudaSuccess) {
    set_error("trn_scene_configure: leaf scan failed");
    return -1;
  }
  k_leaf_collapse<<<nblk(ninner), 256, 0, st>>>(ninner, s->nodes, cnt, base, s->tri_verts, s->cnodes, s->ctri);
  count_launch(4);
  TRN_CUDA_TRY(cudaGetLastError());
  s->collapsed = true;
  return 0;
}

// PLOC rounds until one cluster is left. The kernels read the round's cluster
// count from the device (count[1]); the host launches for an upper bound and
// reads the count back only every kPlocBatch rounds, so the GPU does not wait
// on the host between rounds (rounds after convergence are no-ops).
constexpr int kPlocBatch = 32;

__global__ void k_ploc_count_init(int* count, int n) {
  if (threadIdx.x == 0) { count[0] = 0; count[1] = n; count[2] = 0; }
}

__global__ void k_set_root_parent(int* parent) {
  if (threadIdx.x == 0) parent[0] = -1;
}
int ploc_build(trn_scene* s, cudaStream_t st) {
  const int nt = s->nt;
  int* cur_node = s->ploc_node;
  int* tmp_node = s->ploc_node + nt;
  float* cur_box = s->ploc_box;
  float* tmp_box = s->ploc_box + 6 * (size_t)nt;
  k_ploc_count_init<<<1, 32, 0, st>>>(s->ploc_count, nt);
  k_ploc_init<<<nblk(nt), 256, 0, st>>>(nt, s->keys_alt, s->pos, s->idx, cur_node, cur_box);
  count_launch(1);
  int n = nt;  // upper bound of the device-side count
  // The previous build of this scene needed s->ploc_rounds rounds: the first
  // batch runs that many and a few more (over the full upper bound), so that
  // a rebuild of similar geometry reads the count back once.
  for (int batch = 0; n > 1; batch++) {
    if (batch * kPlocBatch > 4 * nt + 64) { set_error("trn_scene_configure: PLOC did not converge"); return -1; }
    const int rounds = batch == 0 && s->ploc_rounds > 0 ? s->ploc_rounds + 4 : kPlocBatch;
    for (int r = 0; r < rounds; r++) {
      k_ploc_nn<<<(n + kPlocBlock - 1) / kPlocBlock, kPlocBlock, 0, st>>>(s->ploc_count, cur_box, s->ploc_nn);
      k_ploc_merge<<<nblk(n), 256, 0, st>>>(nt, n, s->ploc_nn, cur_node, cur_box, tmp_node, tmp_box, s->ploc_flag,
                                            s->nodes, s->parent, s->ploc_count);
      size_t sb = s->scan_tmp_bytes;
      if (cub::DeviceScan::ExclusiveSum(s->scan_tmp, sb, s->ploc_flag, s->ploc_pos, n, st) != cudaSuccess) {
        set_error("trn_scene_configure: scan failed");
        return -1;
      }
      k_ploc_compact<<<nblk(n), 256, 0, st>>>(n, s->ploc_flag, s->ploc_pos, tmp_node, tmp_box, cur_node, cur_box,
                                              s->ploc_count);
      count_launch(4);
    }
    int counts[3];
    TRN_CUDA_TRY(cudaMemcpyAsync(counts, s->ploc_count, sizeof(counts), cudaMemcpyDeviceToHost, st));
    TRN_CUDA_TRY(cudaStreamSynchronize(st));
    if (counts[1] >= n && n > 1) { set_error("trn_scene_configure: PLOC rounds merged nothing"); return -1; }
    n = counts[1];
    s->ploc_rounds = counts[2];
  }
  k_set_root_parent<<<1, 32, 0, st>>>(s->parent);
  count_launch(1);
  TRN_CUDA_TRY(cudaGetLastError());
  return 0;
}

}  // namespace

extern "C" {

int trn_scene_configure(trn_scene* s, cudaStream_t st) {
  if (!s) { set_error("trn_scene_configure: null scene"); return -1; }
  const int nt = s->nt;
  if (configure_geometry(s, st)) return -1;
  // LBVH
  k_bounds_init<<<1, 32, 0, st>>>((unsigned int*)s->bounds);
  k_bounds<<<nblk(nt), 256, 0, st>>>(nt, s->pos, s->idx, (unsigned int*)s->bounds);
  k_morton<<<nblk(nt), 256, 0, st>>>(nt, s->pos, s->idx, (const unsigned int*)s->bounds, s->keys);
  count_launch(4);  // bounds init, bounds, morton, and the radix sort counted as one
  size_t bytes = s->sort_tmp_bytes;
  if (cub::DeviceRadixSort::SortKeys(s->sort_tmp, bytes, s->keys, s->keys_alt, nt, 0, 64, st) != cudaSuccess) {
    set_error("trn_scene_configure: radix sort failed");
    return -1;
  }
  if (nt > 1) {
    TRN_CUDA_TRY(cudaMemsetAsync(s->flags, 0, sizeof(int) * (nt - 1), st));
    if (TRN_PLOC) {
      if (ploc_build(s, st)) return -1;
    } else {
      k_karras<<<nblk(nt - 1), 256, 0, st>>>(nt, s->keys_alt, s->nodes, s->parent);
      count_launch(1);
    }
  }
  k_refit<<<nblk(nt), 256, 0, st>>>(nt, s->keys_alt, s->pos, s->idx, s->nodes, s->parent, s->flags, s->tri_verts);
  count_launch(1);
  if (!TRN_WIDE_BVH && leaf_collapse(s, st)) return -1;
  // 8-wide quantised BVH
  s->n_wnodes = 0;
  if (TRN_WIDE_BVH && nt > 1) {
    int2* qa = reinterpret_cast<int2*>(s->wqueue);
    int2* qb = qa + nt;
    const int init[4] = {1, 0, 0, 0};
    const int2 root = make_int2(0, 0);
    TRN_CUDA_TRY(cudaMemcpyAsync(s->wcount, init, sizeof(init), cudaMemcpyHostToDevice, st));
    TRN_CUDA_TRY(cudaMemcpyAsync(qa, &root, sizeof(int2), cudaMemcpyHostToDevice, st));
    int n_in = 1;
    int levels = 0;
    while (n_in > 0) {
      TRN_CUDA_TRY(cudaMemsetAsync(s->wcount + 2, 0, sizeof(int), st));
      k_collapse<<<nblk(n_in, 128), 128, 0, st>>>(n_in, qa, qb, s->wcount, s->nodes, s->tri_verts, s->wnodes, s->wtri);
      count_launch(1);
      int c[4];
      TRN_CUDA_TRY(cudaMemcpyAsync(c, s->wcount, sizeof(c), cudaMemcpyDeviceToHost, st));
      TRN_CUDA_TRY(cudaStreamSynchronize(st));
      n_in = c[2];
      s->n_wnodes = c[0];
      std::swap(qa, qb);
      if (++levels > 64) { set_error("trn_scene_configure: wide BVH collapse did not terminate"); return -1; }
    }
  }
  TRN_CUDA_TRY(cudaGetLastError());
  s->configured = true;
  s->built = true;
  s->version++;
  return 0;
}

// Scene::UpdateAccelerationStructure (Scene.cpp:368-469): new positions, same
// BVH topology; leaf boxes and node boxes are recomputed bottom-up.
int trn_scene_refit(trn_scene* s, cudaStream_t st) {
  if (!s) { set_error("trn_scene_refit: null scene"); return -1; }
  if (!s->built || TRN_WIDE_BVH) return trn_scene_configure(s, st);  // the wide BVH is re-collapsed
  const int nt = s->nt;
  if (configure_geometry(s, st)) return -1;
  if (nt > 1) TRN_CUDA_TRY(cudaMemsetAsync(s->flags, 0, sizeof(int) * (nt - 1), st));
  k_refit<<<nblk(nt), 256, 0, st>>>(nt, s->keys_alt, s->pos, s->idx, s->nodes, s->parent, s->flags, s->tri_verts);
  count_launch(1);
  if (leaf_collapse(s, st)) return -1;
  TRN_CUDA_TRY(cudaGetLastError());
  s->configured = true;
  s->version++;
  return 0;
}

int trn_scene_set_translation(trn_scene* s, const float* t, cudaStream_t st) {
  if (!s || !t) { set_error("trn_scene_set_translation: null argument"); return -1; }
  TRN_CUDA_TRY(cudaMemcpyAsync(s->translation, t, sizeof(float) * 3 * s->nmesh, cudaMemcpyDeviceToDevice, st));
  s->configured = false;
  s->version++;
  return 0;
}
int trn_scene_set_positions(trn_scene* s, const float* p, cudaStream_t st) {
  if (!s || !p) { set_error("trn_scene_set_positions: null argument"); return -1; }
  TRN_CUDA_TRY(cudaMemcpyAsync(s->raw_pos, p, sizeof(float) * 3 * s->nv, cudaMemcpyDeviceToDevice, st));
  s->configured = false;
  s->version++;
  return 0;
}
int trn_scene_set_texels(trn_scene* s, const float* p, cudaStream_t st) {
  if (!s || !p) { set_error("trn_scene_set_texels: null argument"); return -1; }
  if (s->ntexel == 0) return 0;
  TRN_CUDA_TRY(cudaMemcpyAsync(s->texels, p, sizeof(float) * 3 * s->ntexel, cudaMemcpyDeviceToDevice, st));
  s->version++;
  return 0;
}

int trn_scene_get_geometry(trn_scene* s, float* pos, float* fn, float* area, float* vn, cudaStream_t st) {
  if (!s) { set_error("trn_scene_get_geometry: null scene"); return -1; }
  if (pos) TRN_CUDA_TRY(cudaMemcpyAsync(pos, s->pos, sizeof(float) * 3 * s->nv, cudaMemcpyDeviceToDevice, st));
  if (fn) TRN_CUDA_TRY(cudaMemcpyAsync(fn, s->fnormal, sizeof(float) * 3 * s->nt, cudaMemcpyDeviceToDevice, st));
  if (area) TRN_CUDA_TRY(cudaMemcpyAsync(area, s->area, sizeof(float) * s->nt, cudaMemcpyDeviceToDevice, st));
  if (vn) TRN_CUDA_TRY(cudaMemcpyAsync(vn, s->vnormal, sizeof(float) * 3 * s->nv, cudaMemcpyDeviceToDevice, st));
  return 0;
}

int trn_scene_counts(const trn_scene* s, int* nv, int* nt, int* ne, long long* ntexel, int* nm) {
  if (!s) { set_error("trn_scene_counts: null scene"); return -1; }
  if (nv) *nv = s->nv;
  if (nt) *nt = s->nt;
  if (ne) *ne = s->ne;
  if (ntexel) *ntexel = s->ntexel;
  if (nm) *nm = s->nmesh;
  return 0;
}

unsigned long long trn_kernel_launches(void) { return g_launches.load(); }

int trn_scene_finalize_grads(trn_scene* s, float* gpos, float* gvn, float* d_translation, cudaStream_t st) {
  if (!s || !gpos || !gvn) { set_error("trn_scene_finalize_grads: null argument"); return -1; }
  const int nv = s->nv, nt = s->nt;
  float* g_sum = nullptr;
  TRN_CUDA_TRY(cudaMallocAsync((void**)&g_sum, sizeof(float) * 3 * nv, st));
  k_vnormal_adj<<<nblk(nv), 256, 0, st>>>(nv, s->vf_off, s->vf_list, s->fnormal, gvn, g_sum);
  k_face_adj<<<nblk(nt), 256, 0, st>>>(nt, s->pos, s->idx, g_sum, gpos);
  count_launch(2);
  TRN_CUDA_TRY(cudaFreeAsync(g_sum, st));
  TRN_CUDA_TRY(cudaMemsetAsync(gvn, 0, sizeof(float) * 3 * nv, st));
  if (d_translation) {
    TRN_CUDA_TRY(cudaMemsetAsync(d_translation, 0, sizeof(float) * 3 * s->nmesh, st));
    k_translation_adj<<<nblk(nv), 256, 0, st>>>(nv, s->vert_mesh, gpos, d_translation);
    count_launch(1);
  }
  TRN_CUDA_TRY(cudaGetLastError());
  return 0;
}

int trn_stats_enable(trn_scene* s, int on) {
  if (!s) { set_error("trn_stats_enable: null scene"); return -1; }
  s->stats_on = on != 0;
  return 0;
}

int trn_stats_read(trn_scene* s, unsigned long long* out, int reset, cudaStream_t st) {
  if (!s || !out) { set_error("trn_stats_read: null argument"); return -1; }
  TRN_CUDA_TRY(cudaMemcpyAsync(out, s->stats, sizeof(unsigned long long) * 16, cudaMemcpyDeviceToHost, st));
  TRN_CUDA_TRY(cudaStreamSynchronize(st));
  if (reset) TRN_CUDA_TRY(cudaMemsetAsync(s->stats, 0, sizeof(unsigned long long) * 16, st));
  return 0;
}

int trn_scene_clear_grads(trn_scene* s, cudaStream_t st) {
  if (!s) { set_error("trn_scene_clear_grads: null scene"); return -1; }
  TRN_CUDA_TRY(cudaMemsetAsync(s->g_pos, 0, sizeof(float) * 3 * s->nv, st));
  TRN_CUDA_TRY(cudaMemsetAsync(s->g_vnormal, 0, sizeof(float) * 3 * s->nv, st));
  if (s->ntexel) TRN_CUDA_TRY(cudaMemsetAsync(s->g_texels, 0, sizeof(float) * 3 * s->ntexel, st));
  TRN_CUDA_TRY(cudaMemsetAsync(s->g_translation, 0, sizeof(float) * 3 * s->nmesh, st));
  s->grads_finalized = true;
  return 0;
}

int trn_scene_get_grads(trn_scene* s, float* d_translation, float* d_positions, float* d_texels, int clear,
                        cudaStream_t st) {
  if (!s) { set_error("trn_scene_get_grads: null scene"); return -1; }
  const int nv = s->nv, nt = s->nt;
  if (!s->grads_finalized) {
    // vertex-normal gradients -> face normals -> positions
    float* g_sum = nullptr;
    TRN_CUDA_TRY(cudaMallocAsync((void**)&g_sum, sizeof(float) * 3 * nv, st));
    k_vnormal_adj<<<nblk(nv), 256, 0, st>>>(nv, s->vf_off, s->vf_list, s->fnormal, s->g_vnormal, g_sum);
    k_face_adj<<<nblk(nt), 256, 0, st>>>(nt, s->pos, s->idx, g_sum, s->g_pos);
    TRN_CUDA_TRY(cudaFreeAsync(g_sum, st));
    TRN_CUDA_TRY(cudaMemsetAsync(s->g_vnormal, 0, sizeof(float) * 3 * nv, st));
    TRN_CUDA_TRY(cudaMemsetAsync(s->g_translation, 0, sizeof(float) * 3 * s->nmesh, st));
    k_translation_adj<<<nblk(nv), 256, 0, st>>>(nv, s->vert_mesh, s->g_pos, s->g_translation);
    count_launch(3);
    TRN_CUDA_TRY(cudaGetLastError());
    s->grads_finalized = true;
  }
  if (d_translation)
    TRN_CUDA_TRY(cudaMemcpyAsync(d_translation, s->g_translation, sizeof(float) * 3 * s->nmesh,
                                 cudaMemcpyDeviceToDevice, st));
  if (d_positions)
    TRN_CUDA_TRY(cudaMemcpyAsync(d_positions, s->g_pos, sizeof(float) * 3 * nv, cudaMemcpyDeviceToDevice, st));
  if (d_texels && s->ntexel)
    TRN_CUDA_TRY(cudaMemcpyAsync(d_texels, s->g_texels, sizeof(float) * 3 * s->ntexel, cudaMemcpyDeviceToDevice, st));
  if (clear) return trn_scene_clear_grads(s, st);
  return 0;
}

}  // extern "C"
