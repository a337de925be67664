// Ray queries against the project LBVH: closest hit and occlusion.
//
// Replaces the OptiX ray-query seam RayIntersectOptix (LibTensorRay/Renderer/
// Optix.cpp:252-305) and its programs (ptx.cu:61-113). Hit semantics:
//   * a hit is a triangle whose watertight intersection (Woop, Benthin and
//     Wald, "Watertight Ray/Triangle Intersection", JCGT 2013) has
//     tmin < t < tmax, both faces count (no culling, like OptiX's default);
//   * the closest hit is the lexicographic minimum of (t, triangle id), so the
//     result does not depend on traversal order;
//   * a miss returns triangle -1 (ptx.cu:61-113 writes -1 on a miss);
//   * Scene::Occluded (Scene.cpp:548-562) is "no hit inside (tmin, tmax)".
// The triangle test is written with explicitly rounded float operations so it
// is bit-identical to the CPU restatement of the same formula.
#pragma once
#include "scene_types.cuh"

namespace trn {

struct Hit {
  int tri;
  float u, v, t;  // u weights P1, v weights P2 (Scene.cpp:677-684)
};

struct RayPre {
  F3 o, d, inv;
  int kx, ky, kz;
  float sx, sy, sz;
};

TRN_D RayPre ray_setup(const F3& o, const F3& d) {
  RayPre r;
  r.o = o; r.d = d;
  float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
  int kz = 0; float m = ax;
  if (ay > m) { kz = 1; m = ay; }
  if (az > m) { kz = 2; }
  int kx = kz + 1; if (kx == 3) kx = 0;
  int ky = kx + 1; if (ky == 3) ky = 0;
  if (d[kz] < 0.f) { int t = kx; kx = ky; ky = t; }
  r.kx = kx; r.ky = ky; r.kz = kz;
  r.sx = __fdiv_rn(d[kx], d[kz]);
  r.sy = __fdiv_rn(d[ky], d[kz]);
  r.sz = __fdiv_rn(1.f, d[kz]);
  // reciprocal direction for the box slabs (culling only)
  auto safe = [](float x) { return fabsf(x) < 1e-20f ? copysignf(1e-20f, x) : x; };
  r.inv = F3(1.f / safe(d.x), 1.f / safe(d.y), 1.f / safe(d.z));
  return r;
}

// Woop et al. 2013, section 3 (algorithm of figure 1), with the double
// precision fallback when an edge function is exactly zero.
TRN_D bool intersect_tri(const RayPre& r, const F3& p0, const F3& p1, const F3& p2,
                         float tmin, float tmax, float& t_out, float& u_out, float& v_out) {
  F3 A(__fsub_rn(p0.x, r.o.x), __fsub_rn(p0.y, r.o.y), __fsub_rn(p0.z, r.o.z));
  F3 B(__fsub_rn(p1.x, r.o.x), __fsub_rn(p1.y, r.o.y), __fsub_rn(p1.z, r.o.z));
  F3 C(__fsub_rn(p2.x, r.o.x), __fsub_rn(p2.y, r.o.y), __fsub_rn(p2.z, r.o.z));
  const float Akz = A[r.kz], Bkz = B[r.kz], Ckz = C[r.kz];
  const float Ax = __fsub_rn(A[r.kx], __fmul_rn(r.sx, Akz));
  const float Ay = __fsub_rn(A[r.ky], __fmul_rn(r.sy, Akz));
  const float Bx = __fsub_rn(B[r.kx], __fmul_rn(r.sx, Bkz));
  const float By = __fsub_rn(B[r.ky], __fmul_rn(r.sy, Bkz));
  const float Cx = __fsub_rn(C[r.kx], __fmul_rn(r.sx, Ckz));
  const float Cy = __fsub_rn(C[r.ky], __fmul_rn(r.sy, Ckz));
  float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
  float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
  float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
  if (U == 0.f || V == 0.f || W == 0.f) {
    U = (float)__dsub_rn(__dmul_rn((double)Cx, (double)By), __dmul_rn((double)Cy, (double)Bx));
    V = (float)__dsub_rn(__dmul_rn((double)Ax, (double)Cy), __dmul_rn((double)Ay, (double)Cx));
    W = (float)__dsub_rn(__dmul_rn((double)Bx, (double)Ay), __dmul_rn((double)By, (double)Ax));
  }
  if ((U < 0.f || V < 0.f || W < 0.f) && (U > 0.f || V > 0.f || W > 0.f)) return false;
  const float det = __fadd_rn(__fadd_rn(U, V), W);
  if (det == 0.f) return false;
  const float Az = __fmul_rn(r.sz, Akz);
  const float Bz = __fmul_rn(r.sz, Bkz);
  const float Cz = __fmul_rn(r.sz, Ckz);
  const float T = __fadd_rn(__fadd_rn(__fmul_rn(U, Az), __fmul_rn(V, Bz)), __fmul_rn(W, Cz));
  const float rcp = __fdiv_rn(1.f, det);
  const float t = __fmul_rn(T, rcp);
  if (!(t > tmin && t < tmax)) return false;
  t_out = t;
  u_out = __fmul_rn(V, rcp);
  v_out = __fmul_rn(W, rcp);
  return true;
}

// Slab test of one child box; boxes are padded at build time and the far
// distance gets a relative slack so culling stays conservative w.r.t. the
// exactly rounded triangle test.
TRN_D bool slab(const RayPre& r, float lx, float ly, float lz, float hx, float hy, float hz,
                float tmin, float tmax, float& tnear) {
  float tx0 = (lx - r.o.x) * r.inv.x, tx1 = (hx - r.o.x) * r.inv.x;
  float ty0 = (ly - r.o.y) * r.inv.y, ty1 = (hy - r.o.y) * r.inv.y;
  float tz0 = (lz - r.o.z) * r.inv.z, tz1 = (hz - r.o.z) * r.inv.z;
  float tn = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), tmin));
  float tf = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fminf(fmaxf(tz0, tz1), tmax));
  tnear = tn;
  return tn <= tf * 1.0000004f;
}

constexpr int kStackSize = 64;

TRN_D void leaf_tri(const DeviceScene& s, int leaf, F3& p0, F3& p1, F3& p2, int& tri) {
  const float4 a = __ldg(&s.tri_verts[3 * leaf + 0]);
  const float4 b = __ldg(&s.tri_verts[3 * leaf + 1]);
  const float4 c = __ldg(&s.tri_verts[3 * leaf + 2]);
  p0 = F3(a.x, a.y, a.z); p1 = F3(b.x, b.y, b.z); p2 = F3(c.x, c.y, c.z);
  tri = __float_as_int(a.w);
}


// ---- 8-wide quantised BVH -------------------------------------------------
// Top levels (root, its children, grandchildren: kTopNodes nodes) are staged
// in shared memory once per block by stage_top(); deeper nodes are read with
// 16-byte read-only loads.
TRN_D WNode* top_nodes() {
  __shared__ WNode top[kTopNodes];
  return top;
}

// every kernel that traces rays calls this once before its work loop
TRN_D void stage_top(const DeviceScene& s) {
  if (!TRN_WIDE_BVH) return;
  const int n = min(s.n_wnodes, kTopNodes);
  const uint4* src = reinterpret_cast<const uint4*>(s.wnodes);
  uint4* dst = reinterpret_cast<uint4*>(top_nodes());
  for (int i = threadIdx.x; i < n * 5; i += blockDim.x) dst[i] = __ldg(src + i);
  __syncthreads();
}

TRN_D void load_wnode(const DeviceScene& s, int idx, WNode& n) {
  uint4* d = reinterpret_cast<uint4*>(&n);
  if (idx < kTopNodes) {
    const uint4* src = reinterpret_cast<const uint4*>(top_nodes() + idx);
#pragma unroll
    for (int i = 0; i < 5; i++) d[i] = src[i];
  } else {
    const uint4* src = reinterpret_cast<const uint4*>(s.wnodes + idx);
#pragma unroll
    for (int i = 0; i < 5; i++) d[i] = __ldg(src + i);
  }
}

template <bool ANY>
__device__ __noinline__ bool trace_wide(const DeviceScene& s, const RayPre& r, float tmin, float tmax, Hit& hit,
                                        int* err) {
  float best_t = tmax;
  int best_tri = 0x7fffffff;
  bool found = false;
  int2 stack[kStackSize];  // (node, tnear bits)
  int sp = 0;
  int cur = 0;
  for (;;) {
    WNode n;
    load_wnode(s, cur, n);
    const float sx = __uint_as_float((unsigned)n.ex << 23);
    const float sy = __uint_as_float((unsigned)n.ey << 23);
    const float sz = __uint_as_float((unsigned)n.ez << 23);
    // box tests of all children first; hits go to two bit masks
    unsigned leaf_mask = 0u, node_mask = 0u;
    float tnear[8];
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const unsigned m = n.meta[i];
      tnear[i] = 0.f;
      if (!(m & 0x80u)) continue;
      const float lx = __fmaf_rn((float)n.qlo[0][i], sx, n.ox), hx = __fmaf_rn((float)n.qhi[0][i], sx, n.ox);
      const float ly = __fmaf_rn((float)n.qlo[1][i], sy, n.oy), hy = __fmaf_rn((float)n.qhi[1][i], sy, n.oy);
      const float lz = __fmaf_rn((float)n.qlo[2][i], sz, n.oz), hz = __fmaf_rn((float)n.qhi[2][i], sz, n.oz);
      float tn;
      if (slab(r, lx, ly, lz, hx, hy, hz, tmin, best_t, tn)) {
        tnear[i] = tn;
        if (m & 0x40u) leaf_mask |= 1u << i; else node_mask |= 1u << i;
      }
    }
    // leaf triangles
    while (leaf_mask) {
      const int i = __ffs(leaf_mask) - 1;
      leaf_mask &= leaf_mask - 1u;
      const int slot = n.tri_base + (int)(n.meta[i] & 0x3fu);
      const float4 a = __ldg(&s.wtri[3 * slot + 0]);
      const float4 b = __ldg(&s.wtri[3 * slot + 1]);
      const float4 c = __ldg(&s.wtri[3 * slot + 2]);
      const int tri = __float_as_int(a.w);
      float t, u, v;
      if (intersect_tri(r, F3(a.x, a.y, a.z), F3(b.x, b.y, b.z), F3(c.x, c.y, c.z), tmin, tmax, t, u, v)) {
        if (ANY) { hit.tri = tri; hit.t = t; hit.u = u; hit.v = v; return true; }
        if (t < best_t || (t == best_t && tri < best_tri)) {
          best_t = t; best_tri = tri; hit.u = u; hit.v = v; found = true;
        }
      }
    }
    // internal children: descend into the nearest, push the rest far-to-near
    int next = -1;
    if (node_mask) {
      float nt = 3.4e38f;
      int ni = 0;
      for (unsigned mm = node_mask; mm; mm &= mm - 1u) {
        const int i = __ffs(mm) - 1;
        if (tnear[i] < nt) { nt = tnear[i]; ni = i; }
      }
      node_mask &= ~(1u << ni);
      next = n.child_base + (int)(n.meta[ni] & 0x3fu);
      while (node_mask) {
        // push the farthest remaining first so nearer ones pop earlier
        float ft = -1.f;
        int fi = 0;
        for (unsigned mm = node_mask; mm; mm &= mm - 1u) {
          const int i = __ffs(mm) - 1;
          if (tnear[i] >= ft) { ft = tnear[i]; fi = i; }
        }
        node_mask &= ~(1u << fi);
        if (sp < kStackSize) stack[sp++] = make_int2(n.child_base + (int)(n.meta[fi] & 0x3fu), __float_as_int(ft));
        else if (err) atomicExch(err, 1);
      }
    }
    if (next >= 0) { cur = next; continue; }
    // pop the next node whose box is still in front of the closest hit
    bool got = false;
    while (sp > 0) {
      const int2 e = stack[--sp];
      if (__int_as_float(e.y) <= best_t * 1.0000004f) { cur = e.x; got = true; break; }
    }
    if (!got) break;
  }
  if (ANY) return false;
  if (found) { hit.tri = best_tri; hit.t = best_t; }
  return found;
}

// Closest hit (ANY == false) or occlusion (ANY == true). Returns true on hit.
#ifndef TRN_ONE_LEAF_SITE
#define TRN_ONE_LEAF_SITE 1
#endif
static_assert(TRN_ONE_LEAF_SITE || TRN_LEAF_MAX == 1, "multi-triangle leaves need the one-leaf-site traversal");

template <bool ANY>
TRN_D bool trace(const DeviceScene& s, const F3& o, const F3& d, float tmin, float tmax, Hit& hit,
                 int* err = nullptr) {
  hit.tri = -1; hit.u = 0.f; hit.v = 0.f; hit.t = -1.f;
  if (s.nt <= 0) return false;
  const RayPre r = ray_setup(o, d);
  if (TRN_WIDE_BVH && s.n_wnodes > 0) return trace_wide<ANY>(s, r, tmin, tmax, hit, err);
  float best_t = tmax;
  int best_tri = 0x7fffffff;
  bool found = false;
  auto test_leaf = [&](int leaf) -> bool {
    F3 p0, p1, p2; int tri;
    leaf_tri(s, leaf, p0, p1, p2, tri);
    float t, u, v;
    if (intersect_tri(r, p0, p1, p2, tmin, tmax, t, u, v)) {
      if (ANY) { hit.tri = tri; hit.t = t; hit.u = u; hit.v = v; return true; }
      if (t < best_t || (t == best_t && tri < best_tri)) {
        best_t = t; best_tri = tri; hit.u = u; hit.v = v; found = true;
      }
    }
    return false;
  };
  if (s.root_is_leaf) {
    if (test_leaf(0)) return true;
  } else if (TRN_ONE_LEAF_SITE) {
    // leaves are visited through the loop like inner nodes, so the triangle
    // test is instantiated once per traversal (smaller code)
    int stack[kStackSize];
    int sp = 0;
    int cur = 0;
    for (;;) {
      if (cur < 0) {
        if (TRN_LEAF_MAX == 1) {
          if (test_leaf(~cur)) return true;
        } else {
          // leaf: ~(first | (count - 1) << 29), count triangles from first
          const int v = ~cur;
          const int first = v & 0x1fffffff, count = (v >> 29) + 1;
          for (int k = 0; k < count; k++)
            if (test_leaf(first + k)) return true;
        }
        if (sp == 0) break;
        cur = stack[--sp];
        continue;
      }
      const BvhNode* n = &s.nodes[cur];
      const float4 a = __ldg(&n->a), b = __ldg(&n->b), c = __ldg(&n->c);
      const int4 dd = __ldg(&n->d);
      float tn0, tn1;
      const bool h0 = slab(r, a.x, a.y, a.z, a.w, b.x, b.y, tmin, best_t, tn0);
      const bool h1 = slab(r, b.z, b.w, c.x, c.y, c.z, c.w, tmin, best_t, tn1);
      if (h0 && h1) {
        int nearc = dd.x, farc = dd.y;
        if (tn1 < tn0) { nearc = dd.y; farc = dd.x; }
        if (sp < kStackSize) stack[sp++] = farc;
        else if (err) atomicExch(err, 1);
        cur = nearc;
      } else if (h0) {
        cur = dd.x;
      } else if (h1) {
        cur = dd.y;
      } else {
        if (sp == 0) break;
        cur = stack[--sp];
      }
    }
  } else {
    int stack[kStackSize];
    int sp = 0;
    int cur = 0;
    for (;;) {
      const BvhNode* n = &s.nodes[cur];
      const float4 a = __ldg(&n->a), b = __ldg(&n->b), c = __ldg(&n->c);
      const int4 dd = __ldg(&n->d);
      float tn0, tn1;
      bool h0 = slab(r, a.x, a.y, a.z, a.w, b.x, b.y, tmin, best_t, tn0);
      bool h1 = slab(r, b.z, b.w, c.x, c.y, c.z, c.w, tmin, best_t, tn1);
      int c0 = dd.x, c1 = dd.y;
      if (h0 && c0 < 0) { if (test_leaf(~c0)) return true; h0 = false; }
      if (h1 && c1 < 0) { if (test_leaf(~c1)) return true; h1 = false; }
      if (h0 && h1) {
        int nearc = c0, farc = c1;
        if (tn1 < tn0) { nearc = c1; farc = c0; }
        if (sp < kStackSize) stack[sp++] = farc;
        else if (err) atomicExch(err, 1);
        cur = nearc;
      } else if (h0) {
        cur = c0;
      } else if (h1) {
        cur = c1;
      } else {
        if (sp == 0) break;
        cur = stack[--sp];
      }
    }
  }
  if (ANY) return false;
  if (found) { hit.tri = best_tri; hit.t = best_t; }
  return found;
}

TRN_D bool occluded(const DeviceScene& s, const F3& o, const F3& d, float tmin, float tmax) {
  Hit h;
  return trace<true>(s, o, d, tmin, tmax, h);
}

// One shared, non-inlined copy of the traversal. Kernels with many ray-query
// sites (the indirect boundary term traces on both sides of the edge, with
// NEE and importance rays on each) call this one (NI = true): inlined copies
// would inflate them past the instruction cache. Kernels with few sites keep
// the inlined form (NI = false), which avoids the call's register traffic.
template <bool ANY>
__device__ __noinline__ bool trace_shared(const DeviceScene& s, const F3& o, const F3& d, float tmin, float tmax,
                                          Hit& hit, int* err) {
  return trace<ANY>(s, o, d, tmin, tmax, hit, err);
}

template <bool NI, bool ANY>
TRN_D bool trace_k(const DeviceScene& s, const F3& o, const F3& d, float tmin, float tmax, Hit& hit,
                   int* err = nullptr) {
  if constexpr (NI) return trace_shared<ANY>(s, o, d, tmin, tmax, hit, err);
  else return trace<ANY>(s, o, d, tmin, tmax, hit, err);
}

template <bool NI>
TRN_D bool occluded_k(const DeviceScene& s, const F3& o, const F3& d, float tmin, float tmax) {
  Hit h;
  return trace_k<NI, true>(s, o, d, tmin, tmax, h);
}

}  // namespace trn
