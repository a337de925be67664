// Integrator kernels: the interior path tracer (forward and replaying
// adjoint) and the primary / direct / indirect / pixel boundary terms.
//
// One thread owns one sample slot (one path) end to end. Where the reference
// builds a tensor expression per stage and compacts surviving rays between
// stages (Integrator.cpp:178-303, Ray.cpp:65-116), a path here keeps its
// state in registers and simply stops; the per-slot sample layout replaces
// the reference's per-call RandomFloat tensors (see SampleSource).
#include <algorithm>
#include <atomic>
#include <cstring>
#include <string>
#include <vector>
#include <cub/cub.cuh>
#include "../../include/trn.h"
#include "scene_impl.cuh"
#include "shading.cuh"

namespace trn {

struct Params {
  DeviceScene s;
  const ViewDesc* views;     // [nviews] cameras, slot ranges, pixel offsets
  const long long* vbegin;   // [nviews] first path slot of each view
  int nviews;
  long long total;           // path slots of this launch (all views)
  unsigned long long* work;  // work-distribution counter (zeroed before launch)
  int chunk;                 // slots per lane per work fetch
  const float* table;        // sample table [dim][total-slot] or nullptr (hash)
  long long stride;
  uint32_t term;             // integrator id (hash stream)
  uint32_t seed;             // RenderOptions::mRndSeed
  float* image;              // call image buffer (views without their own)
  const float* dLdI;         // call dL/dI buffer (views without their own)
  int D;                     // max bounces
  float* g_pos;              // [V*3]
  float* g_vn;               // [V*3]
  float* g_tex;              // [texels*3]
  int diff_tex;              // accumulate texture gradients
  // secondary edge sampling table (per scene); primary tables live in the views
  const int* edges;
  const float* ecdf;
  const float* efunc;
  const float* eint;
  int ne;
  int* err;
  unsigned long long* stats;  // optional work counters (see Cnt), nullptr = off
  // AQ guiding of the direct boundary term (nullptr = unguided)
  const float* aq_poly;       // [leaves] leaf weights
  const float* aq_cdf;        // [leaves] leaf distribution
  const float* aq_int;        // [2] integral, sum of weight x volume
  const float* aq_box;        // [6][aq_cap] leaf boxes (x0, y0, z0, x1, y1, z1)
  const int* aq_edge;         // [leaves] the secondary edge a leaf lies on
  const int* aq_n;            // leaf count
  long long aq_cap;
  // queues of the split kernels (nullptr = fused kernel): q_count[0] counts
  // `queue`, q_count[1] counts `queue2` (the indirect term's second stage),
  // q_count[2] hands out the items of `queue` to a regenerating stage
  void* queue;
  void* queue2;
  unsigned long long* q_count;
  long long q_cap;
  // run order of a split set-up round (nullptr = slot order): the i-th slot
  // of the round [order_first, total) is order_first + order[i - order_first]
  const unsigned* order;
  long long order_first;
};

// Slot that runs at position i of the current round.
TRN_D long long slot_at(const Params& P, long long i) {
  if (!P.order || i >= P.total) return i;
  return P.order_first + (long long)__ldg(P.order + (i - P.order_first));
}

constexpr int kMaxDepth = 16;

// The integrator kernels' parameter block. Its members (the scene above all)
// are passed by reference into non-inlined functions; a plain by-value
// kernel parameter whose address is taken is first copied into every
// thread's local memory, a __grid_constant__ one is addressed in place.
#ifndef TRN_GRID_CONSTANT
#define TRN_GRID_CONSTANT 1
#endif
#if TRN_GRID_CONSTANT
#define TRN_KPARAMS const __grid_constant__ Params P
#else
#define TRN_KPARAMS Params P
#endif

// Minimum resident 256-thread blocks per SM the integrator kernels are
// compiled for (caps registers per thread at 65536 / (256 * minimum)); the
// values below are the measured best per kernel family.
#ifndef TRN_MINB
#define TRN_MINB 4
#endif
#ifndef TRN_MINB_PATHADJ
#define TRN_MINB_PATHADJ 4
#endif
#ifndef TRN_MINB_REVERSE
#define TRN_MINB_REVERSE 2
#endif
#ifndef TRN_MINB_FWDREC
#define TRN_MINB_FWDREC 4
#endif
#ifndef TRN_MINB_INDIRECT
#define TRN_MINB_INDIRECT 4
#endif
// the split forms' set-up kernels are latency-bound with little state: four
// blocks per SM (64 registers) hide more of it (measured)
#ifndef TRN_MINB_SETUP
#define TRN_MINB_SETUP 4
#endif
#ifndef TRN_MINB_BODY
#define TRN_MINB_BODY 4
#endif
// the indirect set-up traces the sensor-side ray first (1) or the
// emitter-side ray first (0); a miss of the first skips the second
#ifndef TRN_INDIRECT_SENSOR_FIRST
#define TRN_INDIRECT_SENSOR_FIRST 0
#endif
// the indirect kernel's two set-up rays use the shared traversal
#ifndef TRN_INDIRECT_SETUP_SHARED
#define TRN_INDIRECT_SETUP_SHARED 1
#endif
// set-up rays of the other kernels: shared or inlined traversal (measured)
#ifndef TRN_SETUP_SHARED_FWD
#define TRN_SETUP_SHARED_FWD 0
#endif
#ifndef TRN_SETUP_SHARED_PATHADJ
#define TRN_SETUP_SHARED_PATHADJ 0
#endif
#ifndef TRN_SETUP_SHARED_PRIMARY
#define TRN_SETUP_SHARED_PRIMARY 1
#endif
#ifndef TRN_SETUP_SHARED_DIRECT
#define TRN_SETUP_SHARED_DIRECT 0
#endif
#ifndef TRN_SETUP_SHARED_PIXEL
#define TRN_SETUP_SHARED_PIXEL 0
#endif

// Per-thread work counters behind the roofline's algorithmic-byte model:
// ray queries, shading vertices, light samples, gradient scatters, pixels.
enum { kCntClosest = 0, kCntShadow, kCntShade, kCntSmooth, kCntTex, kCntLight, kCntVScatter, kCntNScatter,
       kCntTScatter, kCntPixel, kCntNum };
struct Cnt {
  unsigned v[kCntNum];
  TRN_D Cnt() {
#pragma unroll
    for (int i = 0; i < kCntNum; i++) v[i] = 0u;
  }
};
TRN_D void flush_cnt(const Cnt& c, unsigned long long* stats) {
  if (!stats) return;
#pragma unroll
  for (int i = 0; i < kCntNum; i++) {
    const unsigned x = __reduce_add_sync(0xffffffffu, c.v[i]);
    if ((threadIdx.x & 31) == 0 && x) atomicAdd(stats + i, (unsigned long long)x);
  }
}
TRN_D void count_shade(Cnt& c, const DeviceScene& s, const SurfF& x) {
  c.v[kCntShade]++;
  if (s.smooth[x.tri]) c.v[kCntSmooth]++;
  if (s.bsdfs[x.bsdf].tex >= 0) c.v[kCntTex]++;
}

TRN_HD F3 F3z() { return F3(0.f, 0.f, 0.f); }
TRN_D F3 scrub(const F3& a) { return finite3(a) ? a : F3z(); }
TRN_D void atomic_add3(float* a, const F3& g) {
  if (g.x != 0.f) atomicAdd(a, g.x);
  if (g.y != 0.f) atomicAdd(a + 1, g.y);
  if (g.z != 0.f) atomicAdd(a + 2, g.z);
}

// Per-warp staging area for aggregated scatters (one per block, 8 warps max).
TRN_D float* warp_scratch() {
  __shared__ float buf[8 * 32 * 3];
  return buf + (threadIdx.x >> 5) * 96;
}

// Warp-aggregated scatter-add of a float3 into base[3*idx]: lanes of the
// converged warp that target the same index first sum in shared memory, then
// one lane per distinct index issues the global atomics. Replaces the plain
// per-element atomicAdd of IndexedWriteKernel (TensorKernels.cuh:177-209),
// which serialises when many paths hit the same few vertices (quads, lights).
TRN_D void agg_add3(float* base, long long idx, const F3& g) {
  const unsigned active = __activemask();
  const int lane = threadIdx.x & 31;
  // peers share the target address, not just the index: lanes of one warp can
  // scatter into different views' gradient buffers
  float* const target = base + 3 * idx;
  const unsigned peers = __match_any_sync(active, reinterpret_cast<unsigned long long>(target));
  const int leader = __ffs(peers) - 1;
  float* w = warp_scratch();
  if (lane == leader) { w[3 * lane] = g.x; w[3 * lane + 1] = g.y; w[3 * lane + 2] = g.z; }
  __syncwarp(active);
  if (lane != leader) {
    atomicAdd(w + 3 * leader, g.x); atomicAdd(w + 3 * leader + 1, g.y); atomicAdd(w + 3 * leader + 2, g.z);
  }
  __syncwarp(active);
  if (lane == leader) atomic_add3(target, F3(w[3 * lane], w[3 * lane + 1], w[3 * lane + 2]));
  __syncwarp(active);
}
TRN_D F3 g_at(const Params& P, const ViewDesc& V, int pix) {
  if (pix < 0) return F3z();
  const float* d = (V.dLdI ? V.dLdI : P.dLdI + 3 * V.pix_off) + 3 * pix;
  return F3(__ldg(d), __ldg(d + 1), __ldg(d + 2)) * V.inv_spp;
}

// the view owning global slot g (last view whose first slot is <= g)
// View of a launch-global slot. `hint` is the lane's previous view: a lane's
// consecutive slots nearly always fall in the same view, so the range check
// usually replaces the binary search over the view table.
TRN_D const ViewDesc& view_of(const Params& P, long long g, int& hint) {
  const int h = hint;
  if (__ldg(P.vbegin + h) <= g && (h + 1 >= P.nviews || g < __ldg(P.vbegin + h + 1))) return P.views[h];
  int lo = 0, hi = P.nviews - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(P.vbegin + mid) <= g) lo = mid; else hi = mid - 1;
  }
  hint = lo;
  return P.views[lo];
}

// Uniform sample `dim` of one slot: the table is indexed by the launch-global
// slot, the hash by (view seed, term, dim, view-local slot).
struct PathSmp {
  const Params* P;
  uint32_t seed;
  long long gslot, lslot;
  TRN_D float operator()(int dim) const {
    if (P->table) return __ldg(P->table + (long long)dim * P->stride + gslot);
    return hash_uniform(P->seed * 1000003u + seed, P->term, (uint32_t)dim, (uint32_t)lslot);
  }
};

// Persistent work loop: each warp fetches 32*chunk consecutive slots from a
// global counter, so uneven views and path lengths balance across SMs.
template <class F>
TRN_D void for_each_slot(const Params& P, F&& body) {
  const int lane = threadIdx.x & 31;
  const long long step = 32LL * P.chunk;
  for (;;) {
    unsigned long long start = 0;
    if (lane == 0) start = atomicAdd(P.work, (unsigned long long)step);
    start = __shfl_sync(0xffffffffu, start, 0);
    if ((long long)start >= P.total) break;
    for (int j = 0; j < P.chunk; j++) {
      const long long g = (long long)start + 32LL * j + lane;
      if (g < P.total) body(g);
    }
    __syncwarp();
  }
}
TRN_D F3 cam_pos(const CameraDesc& c) { return F3(c.pos[0], c.pos[1], c.pos[2]); }

// AreaLight::Eval (Light.cpp:134-138): radiance when the emitter faces wi
TRN_D F3 emitted(const DeviceScene& s, const SurfF& x, const F3& wi) {
  if (x.emitter < 0) return F3z();
  return dot(wi, x.ng) > 0.f ? light_radiance(s, x.emitter) : F3z();
}

// ---------------------------------------------------------------------------
// templated path factors (differentiated by the adjoint)
// ---------------------------------------------------------------------------
// Next-event estimation factor of EvalRadianceDirect (Integrator.cpp:186-228),
// excluding the incoming throughput and assuming the connection is valid.
template <class S>
TRN_HD V3<S> nee_factor(const BsdfDesc& b, const V3<S>& xprev, const V3<S>& x, const V3<S>& ns, const V3<S>& ng,
                        const V3<S>& kd, const V3<S>& y, const V3<S>& nl, const S& Jl, const F3& Le, float lpdf,
                        float mis) {
  const V3<S> wo = -normalize(x - xprev);
  const Frame<S> fr = make_frame(ns);
  V3<S> wi = y - x;
  const S d2 = dot(wi, wi);
  const S d = sqrt_(d2);
  wi = wi / d;
  const S dotSh = dot(ns, wi);
  const S G = abs_(dot(nl, -wi)) / d2;
  const V3<S> bv = bsdf_eval(b, fr, ng, kd, wo, wi, false) * abs_(dotSh);
  V3<S> out;
  for (int c = 0; c < 3; c++) out[c] = bv[c] * Jl * G * Le[c] / lpdf * mis;
  return out;
}

// BSDF-sampled continuation weight in area measure (Integrator.cpp:252-267).
template <class S>
TRN_HD V3<S> cont_factor(const BsdfDesc& b, const V3<S>& xprev, const V3<S>& x, const V3<S>& ns, const V3<S>& ng,
                         const V3<S>& kd, const V3<S>& xn, const V3<S>& ngn, const S& Jn, float prev_pdf) {
  const V3<S> wo = -normalize(x - xprev);
  const Frame<S> fr = make_frame(ns);
  V3<S> dir = xn - x;
  const S dist2 = dot(dir, dir);
  dir = dir / sqrt_(dist2);
  const S G = abs_(dot(ngn, -dir)) / dist2;
  const V3<S> bv = bsdf_eval(b, fr, ng, kd, wo, dir, false) * abs_(dot(ns, dir));
  V3<S> out;
  for (int c = 0; c < 3; c++) out[c] = bv[c] * G * Jn / prev_pdf;
  return out;
}

// xDotN of the boundary terms: RayIntersectAD (Utils.cpp:288-297) from `org`
// towards `target` against triangle (P0, P1, P2), then n . (w P0 + u P1 + v P2)
// with detached vertices (BoundaryPrimary.cpp:131-145, Edge.cpp:280-291).
template <class S>
TRN_HD S xdotn(const V3<S>& org, const V3<S>& target, const V3<S>& P0, const V3<S>& P1, const V3<S>& P2,
               const F3& n) {
  const V3<S> dir = normalize(target - org);
  const V3<S> e1 = P1 - P0, e2 = P2 - P0;
  const V3<S> h = cross(dir, e2);
  const S f = 1.f / dot(e1, h);
  const V3<S> sv = org - P0;
  const S u = f * dot(sv, h);
  const V3<S> q = cross(sv, e1);
  const S v = f * dot(dir, q);
  const S w = 1.f - u - v;
  const V3<S> u2 = vdetach(P0) * w + vdetach(P1) * u + vdetach(P2) * v;
  return dot(lift<S>(n), u2);
}


// ---------------------------------------------------------------------------
// vertex records -> triangle vertices (the reparameterised PostIntersect)
// ---------------------------------------------------------------------------
struct VAdj { F3 p, ns, ng; float J; };
TRN_D void vadj_zero(VAdj& a) { a.p = F3z(); a.ns = F3z(); a.ng = F3z(); a.J = 0.f; }

// position = w P0 + u P1 + v P2 (detached u, v), face normal c/|c| and
// J = A / Detach(A) with c = cross(P1 - P0, P2 - P0), shading normal
// w n0 + u n1 + v n2 (Scene.cpp:668-730, Primitive.cpp:299-340).
#ifndef TRN_SHARED_SCATTER
#define TRN_SHARED_SCATTER 0
#endif
#if TRN_SHARED_SCATTER
#define TRN_SCATTER_FN __device__ __noinline__
#else
#define TRN_SCATTER_FN TRN_D
#endif
TRN_SCATTER_FN void scatter_vertex(const Params& P, const ViewDesc& V, int tri, float u, float v, const VAdj& a,
                                   Cnt& cnt) {
  const DeviceScene& s = P.s;
  cnt.v[kCntVScatter] += 3;
  int i0, i1, i2; tri_vertices(s, tri, i0, i1, i2);
  const float w = 1.f - u - v;
  F3 g0 = a.p * w, g1 = a.p * u, g2 = a.p * v;
  F3 gng = a.ng;
  if (s.smooth[tri]) {
    cnt.v[kCntNScatter] += 3;
    agg_add3(V.gvn, i0, a.ns * w);
    agg_add3(V.gvn, i1, a.ns * u);
    agg_add3(V.gvn, i2, a.ns * v);
  } else {
    gng = gng + a.ns;
  }
  if (gng.x != 0.f || gng.y != 0.f || gng.z != 0.f || a.J != 0.f) {
    const F3 p0 = load3(s.pos, i0), p1 = load3(s.pos, i1), p2 = load3(s.pos, i2);
    const F3 e1 = p1 - p0, e2 = p2 - p0;
    const F3 c = cross(e1, e2);
    const float len = length(c);
    const F3 n = c / len;
    const float A = 0.5f * len;
    // d|c| from J: dJ/dA = 1/A, dA/d|c| = 1/2
    const float glen = a.J * (0.5f / A);
    const F3 gc = (gng - n * dot(n, gng)) / len + n * glen;
    const F3 ge1 = cross(e2, gc), ge2 = cross(gc, e1);
    g1 = g1 + ge1; g2 = g2 + ge2; g0 = g0 - (ge1 + ge2);
  }
  agg_add3(V.gpos, i0, g0);
  agg_add3(V.gpos, i1, g1);
  agg_add3(V.gpos, i2, g2);
}

TRN_D void scatter_point(const Params& P, const ViewDesc& V, int tri, float u, float v, const F3& gp, Cnt& cnt) {
  cnt.v[kCntVScatter] += 3;
  int i0, i1, i2; tri_vertices(P.s, tri, i0, i1, i2);
  const float w = 1.f - u - v;
  agg_add3(V.gpos, i0, gp * w);
  agg_add3(V.gpos, i1, gp * u);
  agg_add3(V.gpos, i2, gp * v);
}

// ---------------------------------------------------------------------------
// one EvalRadianceDirect step for one ray (Integrator.cpp:178-303)
// ---------------------------------------------------------------------------
struct BounceRec {
  // NEE
  int ltri; float lu, lv, lpdf, lmis; int nee_ok; F3 lLe;
  // continuation
  float prev_pdf; float emis; F3 eLe;  // MIS weight and radiance at the next vertex
  int next_ok;
  int scrubbed;                        // contribution was non-finite
};

// Returns the contribution of this bounce (already NaN-scrubbed). On return
// x/rdir/T hold the next vertex; the return flag says whether it exists.
template <bool NI = false>
TRN_D bool radiance_step(const DeviceScene& s, SurfF& x, F3& rdir, F3& T, float l0, float l1, float b0, float b1,
                         float b2, F3& contrib, BounceRec* rec, Cnt& cnt) {
  const BsdfDesc b = s.bsdfs[x.bsdf];
  count_shade(cnt, s, x);
  long long texel;
  const F3 kd = bsdf_albedo(s, b, x.tu, x.tv, texel);
  const Frame<float> fr = make_frame(x.ns);
  const F3 wo = -rdir;
  F3 val = F3z();
  if (rec) { rec->nee_ok = 0; rec->next_ok = 0; rec->scrubbed = 0; }
  LightSample ls;
  if (light_sample(s, l0, l1, ls)) {
    cnt.v[kCntLight]++;
    int j0, j1, j2; tri_vertices(s, ls.tri, j0, j1, j2);
    const F3 y = bary3(ls.bu, ls.bv, load3(s.pos, j0), load3(s.pos, j1), load3(s.pos, j2));
    const F3 nl = load3(s.fnormal, ls.tri);
    F3 wi = y - x.p;
    const float d2 = dot(wi, wi);
    const float d = sqrtf(d2);
    wi = wi / d;
    const float dotSh = dot(x.ns, wi), dotGeo = dot(x.ng, wi);
    const bool stable = d > kShadowEps && fabsf(dotSh) > kEdgeEps;
    const bool noleak = dotSh * dotGeo > 0.f;
    if (stable && noleak) cnt.v[kCntShadow]++;
    if (stable && noleak && !occluded_k<NI>(s, x.p, wi, kShadowEps, d - kShadowEps)) {
      const F3 Le = dot(-wi, nl) > 0.f ? light_radiance(s, ls.light) : F3z();
      const float G = fabsf(dot(nl, -wi)) / d2;
      const float bpdf = bsdf_pdf_local(b, fr.to_local(wo), fr.to_local(wi)) * G;
      const float mis = ls.pdf * ls.pdf / (ls.pdf * ls.pdf + bpdf * bpdf);
      const F3 bv = bsdf_eval(b, fr, x.ng, kd, wo, wi, false) * fabsf(dotSh);
      F3 v;
      for (int c = 0; c < 3; c++) v[c] = T[c] * (bv[c] * 1.f * G * Le[c] / ls.pdf * mis);
      val = val + v;
      if (rec) {
        rec->nee_ok = 1; rec->ltri = ls.tri; rec->lu = ls.bu; rec->lv = ls.bv; rec->lpdf = ls.pdf;
        rec->lmis = mis; rec->lLe = Le;
      }
    }
  }
  // continuation (BSDF sampling)
  F3 wi; float pdf;
  bsdf_sample_only(b, fr, wo, b0, b1, b2, wi, pdf);
  Hit h;
  bool ok = pdf > 0.f && out_dir_valid(b, x.ns, x.ng, wi);
  if (ok) { cnt.v[kCntClosest]++; ok = trace_k<NI, false>(s, x.p, wi, kShadowEps, kRayMax, h); }
  if (!ok) {
    contrib = scrub(val);
    if (rec) rec->scrubbed = !finite3(val);
    return false;
  }
  const SurfF xn = post_intersect(s, h.tri, h.u, h.v);
  F3 dir = xn.p - x.p;
  const float dist2 = dot(dir, dir);
  dir = dir / sqrtf(dist2);
  const float G = fabsf(dot(xn.ng, -dir)) / dist2;
  const F3 bv = bsdf_eval(b, fr, x.ng, kd, wo, dir, false) * fabsf(dot(x.ns, dir));
  const float prev_pdf = pdf * G;
  F3 Tn;
  for (int c = 0; c < 3; c++) Tn[c] = T[c] * bv[c] * G * 1.f / prev_pdf;
  if (!(G > 0.f)) Tn = F3z();
  float emis = 0.f;
  F3 eLe = F3z();
  if (xn.emitter >= 0) {
    eLe = emitted(s, xn, -dir);
    const float pn = light_pdf(s, xn.tri);
    emis = prev_pdf * prev_pdf / (prev_pdf * prev_pdf + pn * pn);
    val = val + Tn * eLe * emis;
  }
  contrib = scrub(val);
  if (rec) {
    rec->scrubbed = !finite3(val);
    rec->prev_pdf = prev_pdf; rec->emis = emis; rec->eLe = eLe; rec->next_ok = 1;
  }
  x = xn; rdir = dir; T = Tn;
  return true;
}

// One shared (non-inlined) copy of each per-bounce step, with the traversal
// inlined inside it. A shared copy keeps a kernel's code small (the fused
// kernels are instruction-fetch bound), but every object it takes by
// reference lives in local memory: about 0.6-1 KB of stack per thread, which
// at 512-768 threads per SM spills out of L1 and L2 into DRAM. Each kernel
// chooses (measured) between this and the inlined step; the split stage
// kernels are small enough to inline.
#ifndef TRN_SHARED_STEPS_PRIMARY
#define TRN_SHARED_STEPS_PRIMARY 0
#endif
#ifndef TRN_SHARED_STEPS_PIXEL
#define TRN_SHARED_STEPS_PIXEL 0
#endif
#ifndef TRN_SHARED_STEPS_FWD
#define TRN_SHARED_STEPS_FWD 0
#endif
#ifndef TRN_SHARED_STEPS_DIRECT
#define TRN_SHARED_STEPS_DIRECT 0
#endif
#ifndef TRN_SHARED_STEPS_PATHADJ
#define TRN_SHARED_STEPS_PATHADJ 0
#endif
// path_replay (k_path_replay, the fused k_path_adj and the loop-form recording
// forward); TRN_SHARED_STEPS_PATHADJ is the regenerating recording forward
#ifndef TRN_SHARED_STEPS_REPLAY
#define TRN_SHARED_STEPS_REPLAY 1
#endif
// the indirect term's regenerating sensor and emitter stages
#ifndef TRN_SHARED_STEPS_INDIRECT
#define TRN_SHARED_STEPS_INDIRECT 0
#endif
__device__ __noinline__ bool radiance_step_shared(const DeviceScene& s, SurfF& x, F3& rdir, F3& T, float l0, float l1,
                                                  float b0, float b1, float b2, F3& contrib, BounceRec* rec, Cnt& cnt) {
  return radiance_step<false>(s, x, rdir, T, l0, l1, b0, b1, b2, contrib, rec, cnt);
}
template <bool SHARED>
TRN_D bool radiance_step_k(const DeviceScene& s, SurfF& x, F3& rdir, F3& T, float l0, float l1, float b0, float b1,
                           float b2, F3& contrib, BounceRec* rec, Cnt& cnt) {
  if constexpr (SHARED) return radiance_step_shared(s, x, rdir, T, l0, l1, b0, b1, b2, contrib, rec, cnt);
  else return radiance_step<false>(s, x, rdir, T, l0, l1, b0, b1, b2, contrib, rec, cnt);
}


// Per-warp compaction of the work queue: lanes keep pulling sample slots (one
// warp-aggregated atomic per round) until each holds a slot that survives the
// cheap `setup` phase (primary hit, valid edge sample, visible, ...); then the
// warp runs the expensive `body` (path tracing + adjoint) together. Rejected
// samples therefore never hold a lane hostage while others trace long paths.
#ifndef TRN_COMPACT
#define TRN_COMPACT 1
#endif
// lanes that must hold a valid sample before the warp runs the body
#ifndef TRN_COMPACT_MIN
#define TRN_COMPACT_MIN 28
#endif

template <class State, class Setup, class Body>
TRN_D void for_each_valid(const Params& P, Setup&& setup, Body&& body) {
#if !TRN_COMPACT
  // lockstep variant: each warp takes 32 consecutive slots per round
  for_each_slot(P, [&](long long g) {
    State st;
    if (setup(g, st)) body(st);
  });
  return;
#endif
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  State st;
  bool have = false, done = false;
  for (;;) {
    for (;;) {
      const unsigned need = __ballot_sync(0xffffffffu, !have && !done);
      if (!need) break;
      // enough lanes are ready: run the body now rather than spend more
      // nearly-empty set-up rounds on the last rejections
      if (__popc(__ballot_sync(0xffffffffu, have)) >= TRN_COMPACT_MIN) break;
      const int leader = __ffs(need) - 1;
      unsigned long long base = 0;
      if (lane == leader) base = atomicAdd(P.work, (unsigned long long)__popc(need));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (!have && !done) {
        const long long g = (long long)base + __popc(need & lt);
        if (g >= P.total) done = true;
        else have = setup(g, st);
      }
    }
    if (!__any_sync(0xffffffffu, have)) break;
    if (have) { body(st); have = false; }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// interior term: forward
// ---------------------------------------------------------------------------
struct FwdState {
  const ViewDesc* V;
  long long gslot, p;
  int pix;
  SurfF x;
  F3 T, rdir, L;
};

__global__ void __launch_bounds__(256, TRN_MINB) k_path_fwd(TRN_KPARAMS) {
  Cnt cnt;
  stage_top(P.s);
  int vhint = 0;
  for_each_valid<FwdState>(P,
    [&](long long gslot, FwdState& st) -> bool {
      const ViewDesc& V = view_of(P, gslot, vhint);
      const long long p = gslot - V.begin;
      const CameraDesc& cam = V.cam;
      const PathSmp S{&P, V.seed, gslot, p + V.slot_off};
      const int W = cam.w, WH = cam.w * cam.h;
      const F3 org = cam_pos(cam);
      const int pix = (int)(p % WH);
      const F3 dir = camera_ray_dir(cam, pix % W, pix / W, S(0), S(1));
      Hit h;
      cnt.v[kCntClosest]++;
      if (!trace_k<TRN_SETUP_SHARED_FWD, false>(P.s, org, dir, kShadowEps, kRayMax, h, P.err)) return false;
      st.V = &V; st.gslot = gslot; st.p = p; st.pix = pix;
      st.x = post_intersect(P.s, h.tri, h.u, h.v);
      const float t1 = camera_factor<float>(cam, st.x.p, st.x.ng, 1.f);
      st.T = F3(t1, t1, t1);
      st.rdir = normalize(st.x.p - org);
      st.L = scrub(st.T * emitted(P.s, st.x, -st.rdir));
      return true;
    },
    [&](FwdState& st) {
      const ViewDesc& V = *st.V;
      const PathSmp S{&P, V.seed, st.gslot, st.p + V.slot_off};
      SurfF x = st.x;
      F3 T = st.T, rdir = st.rdir, L = st.L;
      for (int b = 0; b < V.D; b++) {
        const int o = 2 + 5 * b;
        F3 c;
        const bool more = radiance_step_k<TRN_SHARED_STEPS_FWD>(P.s, x, rdir, T, S(o), S(o + 1), S(o + 2), S(o + 3), S(o + 4), c, nullptr,
                                        cnt);
        L = L + c;
        if (!more || (T.x == 0.f && T.y == 0.f && T.z == 0.f)) break;
      }
      L = L * V.inv_spp;
      cnt.v[kCntPixel]++;
      atomic_add3((V.image ? V.image : P.image + 3 * V.pix_off) + 3 * st.pix, L);
    });
  flush_cnt(cnt, P.stats);
}

// ---------------------------------------------------------------------------
// interior term: replaying adjoint
// ---------------------------------------------------------------------------
// Gradient of NEE factor w.r.t. (xprev, x, ns, kd, y, nl, Jl).
// ---------------------------------------------------------------------------
// Hand-written reverse mode of the two path factors. Both have the form
//   F_c = B_c(kd, to_local(wo), to_local(wi)) |ns.wi| |nz.wi| / d^2 J K_c
// with wo = -normalize(x - xprev), wi = (z - x) / d, d^2 = |z - x|^2, the
// frame of the (unnormalised, as in the reference) shading normal ns built by
// coordinate_system, and K_c constant (NEE: Le_c mis / lpdf, z = light point,
// nz = light normal; continuation: 1 / prev_pdf, z = next vertex, nz = its
// geometric normal). The derivative conventions are the reference AD's
// (d|x|/dx = +1 for x > 0, else -1, AbsOp::Backward). One backward sweep
// replaces seven forward-mode evaluations per factor.
// ---------------------------------------------------------------------------

// eval_inner in the local frame: returns B and accumulates dB.gB into g_lo,
// g_li (local directions) and g_kd.
TRN_HD F3 eval_inner_vjp(const BsdfDesc& b, const F3& kd, const F3& lo, const F3& li, const F3& gB, F3& g_lo,
                        F3& g_li, F3& g_kd) {
  if (b.type == kDiffuse) {
    const bool reflect = lo.z > 0.f && lo.z * li.z > 0.f;
    if (!reflect) return F3z();
    const float inv_pi = kInvPi;
    g_kd = g_kd + gB * inv_pi;
    return kd * inv_pi;
  }
  const float cv = lo.z, cl = li.z;
  if (!(cv > 0.f && cl > 0.f)) return F3z();
  const F3 hs = lo + li;
  const float Lh = length(hs);
  const F3 wh = hs / Lh;
  const float nh = wh.z, vh = dot(lo, wh);
  const float r = b.roughness;
  const float alpha = r * r;
  const float k = (r + 1.f) * (r + 1.f) * 0.125f;
  const float am1 = alpha * alpha - 1.f;
  const float qd = nh * nh * am1 + 1.f;
  const float tmp = alpha / qd;
  const float ggx = tmp * tmp * kInvPi;
  const float coeff = vh * (vh * -5.55473f - 6.8316f);
  const float e = expf(logf(2.f) * coeff);
  const float q1 = cv * (1.f - k) + k, q2 = cl * (1.f - k) + k;
  const float G1 = cv / q1, G2 = cl / q2;
  const float G = G1 * G2;
  const float den = 4.f * fabsf(cv) * fabsf(cl) + 1e-6f;
  F3 B;
  float g_ggx = 0.f, g_G = 0.f, g_e = 0.f, g_den = 0.f;
  for (int c = 0; c < 3; c++) {
    const float F0 = b.spec[c];
    const float fres = F0 + (1.f - F0) * e;
    const float spec = ggx * G * fres / den;
    B[c] = kd[c] * kInvPi + spec;
    g_ggx += gB[c] * G * fres / den;
    g_G += gB[c] * ggx * fres / den;
    g_e += gB[c] * ggx * G * (1.f - F0) / den;
    g_den -= gB[c] * spec / den;
  }
  g_kd = g_kd + gB * (float)kInvPi;
  const float g_tmp = g_ggx * 2.f * tmp * kInvPi;
  const float g_qd = -g_tmp * tmp / qd;
  const float g_nh = g_qd * 2.f * nh * am1;
  const float g_coeff = g_e * e * logf(2.f);
  const float g_vh = g_coeff * (vh * (2.f * -5.55473f) - 6.8316f);
  float g_cv = g_G * G2 * k / (q1 * q1) + g_den * 4.f * fabsf(cl) * (cv > 0.f ? 1.f : -1.f);
  float g_cl = g_G * G1 * k / (q2 * q2) + g_den * 4.f * fabsf(cv) * (cl > 0.f ? 1.f : -1.f);
  const F3 g_wh = F3(0.f, 0.f, g_nh) + lo * g_vh;
  const F3 g_hs = (g_wh - wh * dot(g_wh, wh)) / Lh;
  g_lo = g_lo + g_hs + wh * g_vh;
  g_li = g_li + g_hs;
  g_lo.z += g_cv;
  g_li.z += g_cl;
  return B;
}

// coordinate_system (Utils.cpp:118-140): t = f(n) on the branch the value took;
// accumulates dt.g_t into g_n.
TRN_HD void tangent_vjp(const F3& n, const F3& g_t, F3& g_n) {
  if (fabsf(n.x) > fabsf(n.y)) {
    const float q = n.x * n.x + n.z * n.z;
    const float inv = 1.f / sqrtf(fmaxf(q, 1e-3f));
    // t = (-n.z inv, 0, n.x inv)
    g_n.z -= g_t.x * inv;
    g_n.x += g_t.z * inv;
    if (q > 1e-3f) {
      const float g_inv = -g_t.x * n.z + g_t.z * n.x;
      const float g_q = -0.5f * g_inv * inv * inv * inv;
      g_n.x += 2.f * g_q * n.x;
      g_n.z += 2.f * g_q * n.z;
    }
  } else {
    const float q = n.y * n.y + n.z * n.z;
    const float inv = 1.f / sqrtf(fmaxf(q, 1e-3f));
    // t = (0, n.z inv, -n.y inv)
    g_n.z += g_t.y * inv;
    g_n.y -= g_t.z * inv;
    if (q > 1e-3f) {
      const float g_inv = g_t.y * n.z - g_t.z * n.y;
      const float g_q = -0.5f * g_inv * inv * inv * inv;
      g_n.y += 2.f * g_q * n.y;
      g_n.z += 2.f * g_q * n.z;
    }
  }
}

// Reverse mode of F above for the output adjoint `adj`; accumulates into the
// gradient outputs (g_prev only if need_prev, g_kd only if need_kd).
#ifndef TRN_SHARED_FACTOR_VJP
#define TRN_SHARED_FACTOR_VJP 2
#endif
// 0: inlined at each call; 1: one shared copy with reference parameters (its
// callers keep every argument in local memory); 2: one shared copy that takes
// its inputs by value and returns its gradient increments
#if TRN_SHARED_FACTOR_VJP == 1
#define TRN_FACTOR_FN __host__ __device__ __noinline__
#else
#define TRN_FACTOR_FN TRN_HD
#endif
TRN_FACTOR_FN F3 factor_vjp_acc(const BsdfDesc& b, bool need_prev, bool need_kd, const F3& xprev, const F3& x,
                                const F3& ns, const F3& kd, const F3& z, const F3& nz, float J, const F3& K,
                                const F3& adj, F3& g_prev, F3& g_x, F3& g_ns, F3& g_kd, F3& g_z, F3& g_nz,
                                float& g_J) {
  const F3 v0 = x - xprev;
  const float L0 = length(v0);
  const F3 n0 = v0 / L0;
  const F3 wo = -n0;
  const F3 vi = z - x;
  const float d2 = dot(vi, vi);
  const float d = sqrtf(d2);
  const F3 wi = vi / d;
  const Frame<float> fr = make_frame(ns);
  const F3 lo = fr.to_local(wo), li = fr.to_local(wi);
  const float cs = dot(ns, wi);
  const float u = dot(nz, -wi);
  const float Q = fabsf(cs) * fabsf(u) / d2 * J;
  const F3 A = adj * K;
  // B(kd, lo, li) with its adjoint gB = A Q
  F3 g_lo = F3z(), g_li = F3z(), gkd = F3z();
  const F3 B = eval_inner_vjp(b, kd, lo, li, A * Q, g_lo, g_li, gkd);
  const F3 F(B.x * Q * K.x, B.y * Q * K.y, B.z * Q * K.z);
  if (need_kd) g_kd = g_kd + gkd;
  const float gQ = dot(A, B);
  if (gQ == 0.f && g_lo.x == 0.f && g_lo.y == 0.f && g_lo.z == 0.f && g_li.x == 0.f && g_li.y == 0.f &&
      g_li.z == 0.f)
    return F;
  // Q = |cs| |u| / d2 J
  const float g_cs = gQ * (cs > 0.f ? 1.f : -1.f) * fabsf(u) / d2 * J;
  const float g_u = gQ * fabsf(cs) * (u > 0.f ? 1.f : -1.f) / d2 * J;
  const float g_d2 = -gQ * Q / d2;
  g_J += gQ * fabsf(cs) * fabsf(u) / d2;
  F3 g_n = wi * g_cs;                    // cs = ns . wi
  F3 g_wi = ns * g_cs - nz * g_u;        // u = -nz . wi
  g_nz = g_nz - wi * g_u;
  // local coordinates (v.t, v.b, v.n)
  const F3 g_wo = fr.t * g_lo.x + fr.b * g_lo.y + fr.n * g_lo.z;
  g_wi = g_wi + fr.t * g_li.x + fr.b * g_li.y + fr.n * g_li.z;
  F3 g_t = wo * g_lo.x + wi * g_li.x;
  const F3 g_b = wo * g_lo.y + wi * g_li.y;
  g_n = g_n + wo * g_lo.z + wi * g_li.z;
  // b = n x t
  g_n = g_n + cross(fr.t, g_b);
  g_t = g_t + cross(g_b, fr.n);
  tangent_vjp(fr.n, g_t, g_n);
  g_ns = g_ns + g_n;
  // wi = vi / |vi|, d2 = vi . vi
  const F3 g_vi = (g_wi - wi * dot(g_wi, wi)) / d + vi * (2.f * g_d2);
  g_z = g_z + g_vi;
  g_x = g_x - g_vi;
  // wo = -v0 / |v0|
  const F3 g_n0 = -g_wo;
  const F3 g_v0 = (g_n0 - n0 * dot(g_n0, n0)) / L0;
  g_x = g_x + g_v0;
  if (need_prev) g_prev = g_prev - g_v0;
  return F;
}

#if TRN_SHARED_FACTOR_VJP == 2
struct FactorGrad {
  F3 F, g_prev, g_x, g_ns, g_kd, g_z, g_nz;
  float g_J;
};
__host__ __device__ __noinline__ FactorGrad factor_vjp_byval(BsdfDesc b, bool need_prev, bool need_kd, F3 xprev, F3 x,
                                                            F3 ns, F3 kd, F3 z, F3 nz, float J, F3 K, F3 adj) {
  FactorGrad r;
  r.g_prev = r.g_x = r.g_ns = r.g_kd = r.g_z = r.g_nz = F3z();
  r.g_J = 0.f;
  r.F = factor_vjp_acc(b, need_prev, need_kd, xprev, x, ns, kd, z, nz, J, K, adj, r.g_prev, r.g_x, r.g_ns, r.g_kd,
                       r.g_z, r.g_nz, r.g_J);
  return r;
}
#endif

TRN_HD F3 factor_vjp(const BsdfDesc& b, bool need_prev, bool need_kd, const F3& xprev, const F3& x, const F3& ns,
                     const F3& kd, const F3& z, const F3& nz, float J, const F3& K, const F3& adj, F3& g_prev,
                     F3& g_x, F3& g_ns, F3& g_kd, F3& g_z, F3& g_nz, float& g_J) {
#if TRN_SHARED_FACTOR_VJP == 2
  const FactorGrad r = factor_vjp_byval(b, need_prev, need_kd, xprev, x, ns, kd, z, nz, J, K, adj);
  g_prev = g_prev + r.g_prev; g_x = g_x + r.g_x; g_ns = g_ns + r.g_ns; g_kd = g_kd + r.g_kd;
  g_z = g_z + r.g_z; g_nz = g_nz + r.g_nz; g_J += r.g_J;
  return r.F;
#else
  return factor_vjp_acc(b, need_prev, need_kd, xprev, x, ns, kd, z, nz, J, K, adj, g_prev, g_x, g_ns, g_kd, g_z,
                        g_nz, g_J);
#endif
}

// Gradient of the NEE factor w.r.t. (xprev, x, ns, kd, y, nl, Jl).
// Reverse mode of camera_factor (Camera::EvalFilter, Camera.cpp:279-303) at
// J = 1: the value G / Detach(G) is 1, so the gradient is W grad(log G) with
// log G = log|cos_x| - 3 log cos_y - 2 log dist, plus W for J.
TRN_HD void camera_factor_grad(const CameraDesc& c, const F3& p, const F3& ng, float W, F3& g_p, F3& g_ng,
                               float& g_J) {
  const F3 v = p - F3(c.pos[0], c.pos[1], c.pos[2]);
  const float dist = length(v);
  const F3 dir = v / dist;
  const F3 cdir(c.dir[0], c.dir[1], c.dir[2]);
  const float cosy = dot(dir, cdir);
  const float cosx = dot(-dir, ng);
  const F3 g_dir = (-ng) * (W / cosx) - cdir * (3.f * W / cosy);
  g_p = (g_dir - dir * dot(g_dir, dir)) / dist - dir * (2.f * W / dist);
  g_ng = (-dir) * (W / cosx);
  g_J = W;
}

// Returns the factor's value.
TRN_HD F3 nee_vjp(const BsdfDesc& b, bool need_prev, bool need_kd, const F3& xprev, const F3& x, const F3& ns,
                  const F3& ng, const F3& kd, const F3& y, const F3& nl, const F3& Le, float lpdf, float mis,
                  const F3& adj, F3& g_prev, F3& g_x, F3& g_ns, F3& g_kd, F3& g_y, F3& g_nl, float& g_Jl) {
  (void)ng;  // the factor evaluates the BSDF without the shading-normal correction
  const F3 K(Le.x / lpdf * mis, Le.y / lpdf * mis, Le.z / lpdf * mis);
  return factor_vjp(b, need_prev, need_kd, xprev, x, ns, kd, y, nl, 1.f, K, adj, g_prev, g_x, g_ns, g_kd, g_y, g_nl,
                    g_Jl);
}

// Gradient of the continuation factor w.r.t. (xprev, x, ns, kd, xn, ngn, Jn).
// Returns the factor's value.
TRN_HD F3 cont_vjp(const BsdfDesc& b, bool need_prev, bool need_kd, const F3& xprev, const F3& x, const F3& ns,
                   const F3& ng, const F3& kd, const F3& xn, const F3& ngn, float prev_pdf, const F3& adj,
                   F3& g_prev, F3& g_x, F3& g_ns, F3& g_kd, F3& g_xn, F3& g_ngn, float& g_Jn) {
  (void)ng;
  const float ip = 1.f / prev_pdf;
  return factor_vjp(b, need_prev, need_kd, xprev, x, ns, kd, xn, ngn, 1.f, F3(ip, ip, ip), adj, g_prev, g_x, g_ns,
                    g_kd, g_xn, g_ngn, g_Jn);
}

struct VRec { int tri; float u, v; };

struct AdjState {
  const ViewDesc* V;
  long long gslot, p;
  int pix;
  F3 g;
  Hit h;
};

// Interior adjoint set-up: the camera ray of the slot (paths whose pixel has a
// zero dL/dI carry no gradient and are skipped; with need_g false, as in the
// recording forward render, no path is skipped and st.g is zero).
TRN_D bool path_adj_setup(const Params& P, long long gslot, AdjState& st, int& vhint, Cnt& cnt, bool need_g = true) {
  const DeviceScene& s = P.s;
  const ViewDesc& V = view_of(P, gslot, vhint);
  const long long p = gslot - V.begin;
  const CameraDesc& cam = V.cam;
  const PathSmp S{&P, V.seed, gslot, p + V.slot_off};
  const int W = cam.w, WH = cam.w * cam.h;
  const int pix = (int)(p % WH);
  if (need_g) cnt.v[kCntPixel]++;
  const F3 g = need_g ? g_at(P, V, pix) : F3z();
  if (need_g && g.x == 0.f && g.y == 0.f && g.z == 0.f) return false;
  const F3 dir = camera_ray_dir(cam, pix % W, pix / W, S(0), S(1));
  cnt.v[kCntClosest]++;
  if (!trace_k<TRN_SETUP_SHARED_PATHADJ, false>(s, cam_pos(cam), dir, kShadowEps, kRayMax, st.h, P.err)) return false;
  st.V = &V; st.gslot = gslot; st.p = p; st.pix = pix; st.g = g;
  return true;
}

struct LRec { int ltri; float lu, lv, lpdf, lmis, ppdf; };

// Everything the reverse sweep of one interior path needs from its forward
// replay: vertices (hit records), per-bounce NEE light samples and
// continuation pdfs, throughputs T_k and emission terms M_k.
template <int MAXD>
struct PathRec {
  long long gslot, p;
  int view, K, D;
  unsigned nee_mask;        // bit k: bounce k's NEE contributes
  F3 g;                     // dL/dI of the path's pixel (times 1/spp)
  VRec vr[MAXD + 2];
  LRec br[MAXD + 1];
  F3 Tk[MAXD + 2], Mk[MAXD + 2];
};

// Forward replay of one interior path from its primary hit, recording into r;
// returns the path's radiance (what k_path_fwd adds to its pixel before the
// 1/spp weight).
template <int MAXD, class Rec>
TRN_D F3 path_replay(const Params& P, const AdjState& st, Rec& r, Cnt& cnt) {
  const DeviceScene& s = P.s;
  const ViewDesc& V = *st.V;
  const CameraDesc& cam = V.cam;
  const PathSmp S{&P, V.seed, st.gslot, st.p + V.slot_off};
  const F3 org = cam_pos(cam);
  const Hit h = st.h;
  r.gslot = st.gslot; r.p = st.p; r.view = (int)(st.V - P.views); r.g = st.g;
  SurfF x = post_intersect(s, h.tri, h.u, h.v);
  r.vr[1] = {h.tri, h.u, h.v};
  const float t1 = camera_factor<float>(cam, x.p, x.ng, 1.f);
  F3 T(t1, t1, t1);
  F3 rdir = normalize(x.p - org);
  r.Tk[1] = T;
  F3 m1 = emitted(s, x, -rdir);
  if (!finite3(T * m1)) m1 = F3z();
  r.Mk[1] = m1;
  F3 L = T * m1;
  int K = 1;  // vertices reached
  const int D = min(V.D, MAXD);
  unsigned mask = 0u;
  for (int b = 0; b < D; b++) {
    const int k = b + 1;
    const int o = 2 + 5 * b;
    F3 c;
    BounceRec R;
    const bool more = radiance_step_k<TRN_SHARED_STEPS_REPLAY>(s, x, rdir, T, S(o), S(o + 1), S(o + 2),
                                    S(o + 3), S(o + 4), c, &R, cnt);
    // a scrubbed (non-finite) bounce contributes nothing and carries no gradient
    if (R.nee_ok && !R.scrubbed) mask |= 1u << k;
    L = L + c;
    r.br[k] = {R.ltri, R.lu, R.lv, R.lpdf, R.lmis, R.prev_pdf};
    if (!more) break;
    r.vr[k + 1] = {x.tri, x.u, x.v};
    r.Tk[k + 1] = T;
    r.Mk[k + 1] = (R.scrubbed || R.emis == 0.f) ? F3z() : R.eLe * R.emis;
    K = k + 1;
    if (T.x == 0.f && T.y == 0.f && T.z == 0.f) break;
  }
  r.K = K;
  r.D = D;
  r.nee_mask = mask;
  return L;
}

// Reverse sweep of one recorded interior path:
// a_k = g*(N_k + M_k) + phi_k * a_{k+1}, one vertex window at a time, then
// the camera factor at vertex 1.
template <int MAXD, class Rec>
TRN_D void path_reverse(const Params& P, const Rec& r, Cnt& cnt) {
  const DeviceScene& s = P.s;
  const ViewDesc& V = P.views[r.view];
  const CameraDesc& cam = V.cam;
  const F3 org = cam_pos(cam);
  const F3 g = r.g;
  const int K = r.K, D = r.D;
  struct VG { F3 p, ns, ng, kd; long long texel; int bsdf; };
  auto load_vg = [&](int k) {
    VG o;
    const SurfF xs = post_intersect(s, r.vr[k].tri, r.vr[k].u, r.vr[k].v);
    o.p = xs.p; o.ns = xs.ns; o.ng = xs.ng; o.bsdf = xs.bsdf;
    o.kd = bsdf_albedo(s, s.bsdfs[xs.bsdf], xs.tu, xs.tv, o.texel);
    return o;
  };
  VG Gk = load_vg(K), Gn = Gk;
  F3 a_next = F3z();
  VAdj acc_next, acc_k, acc_prev;
  vadj_zero(acc_next); vadj_zero(acc_k); vadj_zero(acc_prev);
  for (int k = K; k >= 1; k--) {
    VG Gp;
    if (k >= 2) Gp = load_vg(k - 1);
    else { Gp.p = org; Gp.ns = Gp.ng = Gp.kd = F3z(); Gp.texel = -1; Gp.bsdf = 0; }
    const BsdfDesc b = s.bsdfs[Gk.bsdf];
    const bool need_prev = b.type != kDiffuse;
    const bool need_kd = P.diff_tex && Gk.texel >= 0;
    F3 Nval = F3z(), Phi = F3z();
    F3 gkd = F3z(), gprev = F3z();
    if (k <= D && ((r.nee_mask >> k) & 1u)) {
      // NEE factor value and its reverse mode in one sweep
      const LRec& R = r.br[k];
      int j0, j1, j2; tri_vertices(s, R.ltri, j0, j1, j2);
      const F3 y = bary3(R.lu, R.lv, load3(s.pos, j0), load3(s.pos, j1), load3(s.pos, j2));
      const F3 nl = load3(s.fnormal, R.ltri);
      // the forward step's emitter radiance (one-sided, AreaLight::Eval), same arithmetic
      F3 wl = y - Gk.p;
      wl = wl / sqrtf(dot(wl, wl));
      const F3 Le = dot(-wl, nl) > 0.f ? light_radiance(s, s.emitter_id[R.ltri]) : F3z();
      F3 gy = F3z(), gnl = F3z();
      float gJl = 0.f;
      Nval = nee_vjp(b, need_prev, need_kd, Gp.p, Gk.p, Gk.ns, Gk.ng, Gk.kd, y, nl, Le, R.lpdf, R.lmis,
                     r.Tk[k] * g, gprev, acc_k.p, acc_k.ns, gkd, gy, gnl, gJl);
      VAdj la; la.p = gy; la.ns = F3z(); la.ng = gnl; la.J = gJl;
      scatter_vertex(P, V, R.ltri, R.lu, R.lv, la, cnt);
    }
    if (k < K) {
      // continuation factor value and its reverse mode; a non-finite weight
      // made the forward throughput non-finite: no value, no gradient
      F3 cprev = F3z(), cx = F3z(), cns = F3z(), ckd = F3z(), cxn = F3z(), cngn = F3z();
      float gJn = 0.f;
      Phi = cont_vjp(b, need_prev, need_kd, Gp.p, Gk.p, Gk.ns, Gk.ng, Gk.kd, Gn.p, Gn.ng, r.br[k].ppdf,
                     r.Tk[k] * a_next, cprev, cx, cns, ckd, cxn, cngn, gJn);
      if (finite3(Phi)) {
        gprev = gprev + cprev; acc_k.p = acc_k.p + cx; acc_k.ns = acc_k.ns + cns; gkd = gkd + ckd;
        acc_next.p = acc_next.p + cxn; acc_next.ng = acc_next.ng + cngn; acc_next.J += gJn;
      } else {
        Phi = F3z();
      }
    }
    const F3 a_k = g * (Nval + r.Mk[k]) + Phi * a_next;
    if (k >= 2) acc_prev.p = acc_prev.p + gprev;
    if (need_kd) { cnt.v[kCntTScatter]++; agg_add3(V.gtex, Gk.texel, gkd); }
    // vertex k+1 has received all of its contributions
    if (k < K) scatter_vertex(P, V, r.vr[k + 1].tri, r.vr[k + 1].u, r.vr[k + 1].v, acc_next, cnt);
    acc_next = acc_k; acc_k = acc_prev; vadj_zero(acc_prev);
    a_next = a_k; Gn = Gk; Gk = Gp;
  }
  // primary factor T1 = G / Detach(G) * J at vertex 1 (now in Gn / acc_next)
  {
    const float gam = a_next.x + a_next.y + a_next.z;
    if (gam != 0.f && isfinite(gam)) {
      F3 gp, gn;
      float gJ;
      camera_factor_grad(cam, Gn.p, Gn.ng, gam, gp, gn, gJ);
      acc_next.p = acc_next.p + gp;
      acc_next.ng = acc_next.ng + gn;
      acc_next.J += gJ;
    }
  }
  scatter_vertex(P, V, r.vr[1].tri, r.vr[1].u, r.vr[1].v, acc_next, cnt);
}

template <int MAXD>
__global__ void __launch_bounds__(256, TRN_MINB_PATHADJ) k_path_adj(TRN_KPARAMS) {
  Cnt cnt;
  stage_top(P.s);
  int vhint = 0;
  for_each_valid<AdjState>(P,
    [&](long long gslot, AdjState& st) -> bool { return path_adj_setup(P, gslot, st, vhint, cnt); },
    [&](AdjState& st) {
      PathRec<MAXD> r;
      path_replay<MAXD>(P, st, r, cnt);
      path_reverse<MAXD>(P, r, cnt);
    });
  flush_cnt(cnt, P.stats);
}

// Path records of the split interior adjoint in structure-of-arrays layout:
// field k of path i lives at k * cap + i, so the lanes of a warp (consecutive
// queue slots) read and write consecutive addresses. PathRecSoA gives the same
// member syntax as PathRec over that layout.
template <class T>
struct Strided {
  T* b;
  long long s;
  TRN_D T& operator[](int k) const { return b[(long long)k * s]; }
};

template <int MAXD>
struct PathRecSoA {
  long long& gslot;
  long long& p;
  int& view;
  int& K;
  int& D;
  unsigned& nee_mask;
  F3& g;
  Strided<VRec> vr;
  Strided<LRec> br;
  Strided<F3> Tk, Mk;
};

template <int MAXD>
TRN_HD size_t path_soa_bytes(long long cap) {
  return (size_t)cap * (2 * sizeof(long long) + 3 * sizeof(int) + sizeof(unsigned) + sizeof(F3) +
                        (MAXD + 2) * sizeof(VRec) + (MAXD + 1) * sizeof(LRec) + 2 * (MAXD + 2) * sizeof(F3)) +
         16 * 256;
}

template <int MAXD>
TRN_D PathRecSoA<MAXD> path_soa(void* base, long long cap, long long i) {
  char* c = static_cast<char*>(base);
  auto take = [&](size_t bytes) { char* r = c; c += (bytes + 255) / 256 * 256; return r; };
  long long* gslot = reinterpret_cast<long long*>(take(sizeof(long long) * cap));
  long long* pp = reinterpret_cast<long long*>(take(sizeof(long long) * cap));
  int* view = reinterpret_cast<int*>(take(sizeof(int) * cap));
  int* K = reinterpret_cast<int*>(take(sizeof(int) * cap));
  int* D = reinterpret_cast<int*>(take(sizeof(int) * cap));
  unsigned* nee = reinterpret_cast<unsigned*>(take(sizeof(unsigned) * cap));
  F3* g = reinterpret_cast<F3*>(take(sizeof(F3) * cap));
  VRec* vr = reinterpret_cast<VRec*>(take(sizeof(VRec) * (MAXD + 2) * cap));
  LRec* br = reinterpret_cast<LRec*>(take(sizeof(LRec) * (MAXD + 1) * cap));
  F3* Tk = reinterpret_cast<F3*>(take(sizeof(F3) * (MAXD + 2) * cap));
  F3* Mk = reinterpret_cast<F3*>(take(sizeof(F3) * (MAXD + 2) * cap));
  return PathRecSoA<MAXD>{gslot[i], pp[i], view[i], K[i], D[i], nee[i], g[i],
                          Strided<VRec>{vr + i, cap}, Strided<LRec>{br + i, cap},
                          Strided<F3>{Tk + i, cap}, Strided<F3>{Mk + i, cap}};
}

// Split form: k_path_replay traces and records every path into the queue;
// k_path_reverse runs the reverse sweep over the queue. Each kernel carries
// half of the fused kernel's code (the fused kernel is instruction-fetch
// bound).
template <int MAXD>
__global__ void __launch_bounds__(256, TRN_MINB_PATHADJ) k_path_replay(TRN_KPARAMS) {
  Cnt cnt;
  stage_top(P.s);
  int vhint = 0;
  for_each_valid<AdjState>(P,
    [&](long long gslot, AdjState& st) -> bool { return path_adj_setup(P, gslot, st, vhint, cnt); },
    [&](AdjState& st) {
      const unsigned act = __activemask();
      const int lane = threadIdx.x & 31;
      const int leader = __ffs(act) - 1;
      unsigned long long base = 0;
      if (lane == leader) base = atomicAdd(P.q_count, (unsigned long long)__popc(act));
      base = __shfl_sync(act, base, leader);
      const unsigned long long k = base + __popc(act & ((1u << lane) - 1u));
      if (k >= (unsigned long long)P.q_cap) { atomicExch(P.err, 2); return; }
      PathRecSoA<MAXD> r = path_soa<MAXD>(P.queue, P.q_cap, (long long)k);
      path_replay<MAXD>(P, st, r, cnt);
    });
  flush_cnt(cnt, P.stats);
}

// CACHED: the records come from the recording forward render (k_path_fwd_rec)
// and carry no dL/dI yet; each path reads its pixel's now and is skipped when
// that is zero, as path_adj_setup skips it in the replaying form.
template <int MAXD, bool CACHED = false>
__global__ void __launch_bounds__(256, TRN_MINB_REVERSE) k_path_reverse(TRN_KPARAMS) {
  Cnt cnt;
  stage_top(P.s);
  const unsigned long long n = min(*P.q_count, (unsigned long long)P.q_cap);
  for (unsigned long long k = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; k < n;
       k += (unsigned long long)gridDim.x * blockDim.x) {
    const PathRecSoA<MAXD> r = path_soa<MAXD>(P.queue, P.q_cap, (long long)k);
    if (CACHED) {
      const ViewDesc& V = P.views[r.view];
      const F3 g = g_at(P, V, (int)(r.p % ((long long)V.cam.w * V.cam.h)));
      if (g.x == 0.f && g.y == 0.f && g.z == 0.f) continue;
      r.g = g;
    }
    path_reverse<MAXD>(P, r, cnt);
  }
  flush_cnt(cnt, P.stats);
}

// Forward interior render that also keeps every path with a primary hit as a
// record (the records k_path_replay writes for the gradient call). A gradient
// call of the same paths then runs k_path_reverse<MAXD, true> over them
// instead of tracing them again. Same image as k_path_fwd.
template <int MAXD>
__global__ void __launch_bounds__(256, TRN_MINB_FWDREC) k_path_fwd_rec(TRN_KPARAMS) {
  Cnt cnt;
  stage_top(P.s);
  int vhint = 0;
  for_each_valid<AdjState>(P,
    [&](long long gslot, AdjState& st) -> bool { return path_adj_setup(P, gslot, st, vhint, cnt, false); },
    [&](AdjState& st) {
      const unsigned act = __activemask();
      const int lane = threadIdx.x & 31;
      const int leader = __ffs(act) - 1;
      unsigned long long base = 0;
      if (lane == leader) base = atomicAdd(P.q_count, (unsigned long long)__popc(act));
      base = __shfl_sync(act, base, leader);
      const unsigned long long k = base + __popc(act & ((1u << lane) - 1u));
      if (k >= (unsigned long long)P.q_cap) { atomicExch(P.err, 2); return; }
      PathRecSoA<MAXD> r = path_soa<MAXD>(P.queue, P.q_cap, (long long)k);
      const ViewDesc& V = *st.V;
      const F3 L = path_replay<MAXD>(P, st, r, cnt) * V.inv_spp;
      cnt.v[kCntPixel]++;
      atomic_add3((V.image ? V.image : P.image + 3 * V.pix_off) + 3 * st.pix, L);
    });
  flush_cnt(cnt, P.stats);
}

// k_path_fwd_rec with path regeneration: lanes fetch slots until at least
// TRN_COMPACT_MIN hold a path (as for_each_valid), then every lane with a
// path takes one bounce; a lane whose path has ended writes its record's
// totals and its pixel and takes the next slot at once. Each path runs
// exactly the steps of path_replay.
#ifndef TRN_FWD_REGEN
#define TRN_FWD_REGEN 1
#endif

template <int MAXD>
__global__ void __launch_bounds__(256, TRN_MINB_FWDREC) k_path_fwd_rec_regen(TRN_KPARAMS) {
  Cnt cnt;
  stage_top(P.s);
  const DeviceScene& s = P.s;
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  int vhint = 0;
  bool active = false, done = false;
  const ViewDesc* V = nullptr;
  long long gslot = 0, p = 0, kr = 0;
  int pix = 0, b = 0, K = 1, D = 0;
  unsigned mask = 0u;
  SurfF x;
  F3 T, rdir, L;
  for (;;) {
    // refill: fetch slots until enough lanes hold a path with a primary hit
    for (;;) {
      const unsigned need = __ballot_sync(0xffffffffu, !active && !done);
      if (!need || __popc(__ballot_sync(0xffffffffu, active)) >= TRN_COMPACT_MIN) break;
      const int leader = __ffs(need) - 1;
      unsigned long long base = 0;
      if (lane == leader) base = atomicAdd(P.work, (unsigned long long)__popc(need));
      base = __shfl_sync(0xffffffffu, base, leader);
      AdjState st;
      bool got = false;
      if (!active && !done) {
        const long long g = (long long)base + __popc(need & lt);
        if (g >= P.total) done = true;
        else got = path_adj_setup(P, g, st, vhint, cnt, false);
      }
      const unsigned gm = __ballot_sync(0xffffffffu, got);
      if (!gm) continue;
      const int gl = __ffs(gm) - 1;
      unsigned long long rb = 0;
      if (lane == gl) rb = atomicAdd(P.q_count, (unsigned long long)__popc(gm));
      rb = __shfl_sync(0xffffffffu, rb, gl);
      if (got) {
        kr = (long long)(rb + __popc(gm & lt));
        if (kr >= P.q_cap) {
          atomicExch(P.err, 2);
        } else {
          V = st.V; gslot = st.gslot; p = st.p; pix = st.pix;
          PathRecSoA<MAXD> r = path_soa<MAXD>(P.queue, P.q_cap, kr);
          r.gslot = gslot; r.p = p; r.view = (int)(V - P.views); r.g = F3z();
          x = post_intersect(s, st.h.tri, st.h.u, st.h.v);
          r.vr[1] = {st.h.tri, st.h.u, st.h.v};
          const F3 org = cam_pos(V->cam);
          const float t1 = camera_factor<float>(V->cam, x.p, x.ng, 1.f);
          T = F3(t1, t1, t1);
          rdir = normalize(x.p - org);
          r.Tk[1] = T;
          F3 m1 = emitted(s, x, -rdir);
          if (!finite3(T * m1)) m1 = F3z();
          r.Mk[1] = m1;
          L = T * m1;
          K = 1;
          D = min(V->D, MAXD);
          mask = 0u;
          b = 0;
          active = true;
        }
      }
    }
    if (!__any_sync(0xffffffffu, active)) break;
    if (active) {
      PathRecSoA<MAXD> r = path_soa<MAXD>(P.queue, P.q_cap, kr);
      bool fin = b >= D;
      if (!fin) {
        const PathSmp S{&P, V->seed, gslot, p + V->slot_off};
        const int k = b + 1;
        const int o = 2 + 5 * b;
        F3 c;
        BounceRec R;
        const bool more = radiance_step_k<TRN_SHARED_STEPS_PATHADJ>(s, x, rdir, T, S(o), S(o + 1), S(o + 2),
                                                                   S(o + 3), S(o + 4), c, &R, cnt);
        if (R.nee_ok && !R.scrubbed) mask |= 1u << k;
        L = L + c;
        r.br[k] = {R.ltri, R.lu, R.lv, R.lpdf, R.lmis, R.prev_pdf};
        if (!more) {
          fin = true;
        } else {
          r.vr[k + 1] = {x.tri, x.u, x.v};
          r.Tk[k + 1] = T;
          r.Mk[k + 1] = (R.scrubbed || R.emis == 0.f) ? F3z() : R.eLe * R.emis;
          K = k + 1;
          if (T.x == 0.f && T.y == 0.f && T.z == 0.f) fin = true;
        }
        b++;
        if (b >= D) fin = true;
      }
      if (fin) {
        r.K = K;
        r.D = D;
        r.nee_mask = mask;
        cnt.v[kCntPixel]++;
        atomic_add3((V->image ? V->image : P.image + 3 * V->pix_off) + 3 * pix, L * V->inv_spp);
        active = false;
      }
    }
  }
  flush_cnt(cnt, P.stats);
}


// ---------------------------------------------------------------------------
// EvalImportance for one ray (Integrator.cpp:75-176)
// ---------------------------------------------------------------------------
template <bool NI = false>
TRN_D bool importance_step(const DeviceScene& s, const CameraDesc& cam, SurfF& x, F3& rdir, F3& T, float b0,
                           float b1, float b2, F3& contrib, int& pix, Cnt& cnt) {
  contrib = F3z();
  pix = -1;
  const BsdfDesc b = s.bsdfs[x.bsdf];
  count_shade(cnt, s, x);
  long long texel;
  const F3 kd = bsdf_albedo(s, b, x.tu, x.tv, texel);
  const Frame<float> fr = make_frame(x.ns);
  const F3 wo = -rdir;
  const F3 cpos = cam_pos(cam);
  const SensorSample sds = sample_direct(cam, x.p);
  if (sds.valid) {
    const F3 dirc = sensor_ray_dir(cam, sds.qx, sds.qy);
    const float dist2cam = length(x.p - cpos);
    cnt.v[kCntShadow]++;
    if (!occluded_k<NI>(s, cpos, dirc, kShadowEps, dist2cam - kShadowEps)) {
      F3 val = F3z();
      if (out_dir_valid(b, x.ns, x.ng, wo)) {
        const F3 wi = normalize(cpos - x.p);
        if (out_dir_valid(b, x.ns, x.ng, wi))
          val = bsdf_eval(b, fr, x.ng, kd, wo, wi, true) * fabsf(dot(x.ns, wi));
      }
      contrib = scrub(T * sds.sensor_val * val);
      pix = image_pixel(cam, sds.qx, sds.qy);
    }
  }
  if (!out_dir_valid(b, x.ns, x.ng, wo)) return false;
  F3 wi; float pdf;
  bsdf_sample_only(b, fr, wo, b0, b1, b2, wi, pdf);
  const F3 bv = bsdf_eval(b, fr, x.ng, kd, wo, wi, true) * fabsf(dot(x.ns, wi));
  const F3 Tn = T * bv / pdf;
  if (!(pdf > 0.f) || !out_dir_valid(b, x.ns, x.ng, wi)) return false;
  Hit h;
  cnt.v[kCntClosest]++;
  if (!trace_k<NI, false>(s, x.p, wi, kShadowEps, kRayMax, h)) return false;
  x = post_intersect(s, h.tri, h.u, h.v);
  rdir = wi;
  T = Tn;
  return true;
}

__device__ __noinline__ bool importance_step_shared(const DeviceScene& s, const CameraDesc& cam, SurfF& x, F3& rdir,
                                                    F3& T, float b0, float b1, float b2, F3& contrib, int& pix,
                                                    Cnt& cnt) {
  return importance_step<false>(s, cam, x, rdir, T, b0, b1, b2, contrib, pix, cnt);
}
template <bool SHARED>
TRN_D bool importance_step_k(const DeviceScene& s, const CameraDesc& cam, SurfF& x, F3& rdir, F3& T, float b0,
                             float b1, float b2, F3& contrib, int& pix, Cnt& cnt) {
  if constexpr (SHARED) return importance_step_shared(s, cam, x, rdir, T, b0, b1, b2, contrib, pix, cnt);
  else return importance_step<false>(s, cam, x, rdir, T, b0, b1, b2, contrib, pix, cnt);
}

// scatter W * d xDotN / d(edge vertices, receiver point, far triangle)
// Reverse mode of xdotn (RayIntersectAD + n . (w P0 + u P1 + v P2) with
// detached vertices) for the upstream scalar W; returns the gradients w.r.t.
// org, target and the attached triangle vertices P0, P1, P2.
TRN_HD void xdotn_grad(const F3& org, const F3& target, const F3& P0, const F3& P1, const F3& P2, const F3& n,
                       float W, F3& g_org, F3& g_target, F3& g0, F3& g1, F3& g2) {
  const F3 vd = target - org;
  const float Ld = length(vd);
  const F3 dir = vd / Ld;
  const F3 e1 = P1 - P0, e2 = P2 - P0;
  const F3 h = cross(dir, e2);
  const float f = 1.f / dot(e1, h);
  const F3 sv = org - P0;
  const F3 q = cross(sv, e1);
  const float g_u = W * dot(n, P1 - P0);
  const float g_v = W * dot(n, P2 - P0);
  // v = f (dir . q), u = f (sv . h)
  const float g_f = g_v * dot(dir, q) + g_u * dot(sv, h);
  F3 g_dir = q * (g_v * f);
  const F3 g_q = dir * (g_v * f);
  F3 g_sv = h * (g_u * f);
  F3 g_h = sv * (g_u * f);
  // q = sv x e1
  g_sv = g_sv + cross(e1, g_q);
  F3 g_e1 = cross(g_q, sv);
  // f = 1 / (e1 . h)
  const float g_a = -g_f * f * f;
  g_e1 = g_e1 + h * g_a;
  g_h = g_h + e1 * g_a;
  // h = dir x e2
  g_dir = g_dir + cross(e2, g_h);
  const F3 g_e2 = cross(g_h, dir);
  // sv = org - P0, e1 = P1 - P0, e2 = P2 - P0
  g_org = g_sv;
  g0 = -(g_sv + g_e1 + g_e2);
  g1 = g_e1;
  g2 = g_e2;
  // dir = vd / |vd|
  const F3 g_vd = (g_dir - dir * dot(g_dir, dir)) / Ld;
  g_target = g_vd;
  g_org = g_org - g_vd;
}

// scatter W * d xDotN / d(edge vertices, receiver point, far triangle)
TRN_D void xdotn_vjp(const Params& P, const ViewDesc& V, float W, const F3& org, bool org_attached, int recv_tri, float ru, float rv,
                     int va_, int vb_, float sedge, const F3& target_const, int far_tri, const F3& n, Cnt& cnt) {
  const DeviceScene& s = P.s;
  cnt.v[kCntVScatter] += 3 + (va_ >= 0 ? 2 : 0);
  int i0, i1, i2; tri_vertices(s, far_tri, i0, i1, i2);
  const F3 P0 = load3(s.pos, i0), P1 = load3(s.pos, i1), P2 = load3(s.pos, i2);
  const bool edge_attached = va_ >= 0;
  F3 target = target_const, Pa = F3z(), Pb = F3z();
  if (edge_attached) {
    Pa = load3(s.pos, va_);
    Pb = load3(s.pos, vb_);
    target = Pa + (Pb - Pa) * sedge;
  }
  F3 gorg, gt, g0, g1, g2;
  xdotn_grad(org, target, P0, P1, P2, n, W, gorg, gt, g0, g1, g2);
  // a degenerate sample (the line org -> target parallel to the far
  // triangle, or org == target) has no finite derivative; it contributes
  // nothing instead of turning the whole gradient buffer into NaN
  if (!(finite3(g0) && finite3(g1) && finite3(g2) && (!edge_attached || finite3(gt)) &&
        (!org_attached || finite3(gorg))))
    return;
  agg_add3(V.gpos, i0, g0);
  agg_add3(V.gpos, i1, g1);
  agg_add3(V.gpos, i2, g2);
  if (edge_attached) {
    agg_add3(V.gpos, va_, gt * (1.f - sedge));
    agg_add3(V.gpos, vb_, gt * sedge);
  }
  if (org_attached) scatter_point(P, V, recv_tri, ru, rv, gorg, cnt);
}

// boundary geometry term baseVal (BoundaryPrimary.cpp:115-129, Edge.cpp:258-271)
TRN_D float base_val(float ratio, const F3& edge, const F3& d, const F3& nrm, const F3& edge2, F3& n_out) {
  const F3 e = cross(edge, d);
  const float sinphi = length(e);
  const F3 proj = normalize(cross(e, nrm));
  const float sinphi2 = length(cross(d, proj));
  n_out = normalize(cross(nrm, proj));
  const bool sign0 = dot(e, edge2) > 0.f;
  const bool sign1 = dot(e, n_out) > 0.f;
  float bv = ratio * (sinphi / sinphi2);
  bv = bv * (sinphi > kEps ? 1.f : 0.f) * (sinphi2 > kEps ? 1.f : 0.f);
  return bv * (sign0 == sign1 ? 1.f : -1.f);
}

// ---------------------------------------------------------------------------
// primary boundary (BoundaryPrimary.cpp:36-181, SampleFromPrimEdges Edge.cpp:350-367)
// ---------------------------------------------------------------------------
struct EdgeState {
  const ViewDesc* V;
  long long gslot, p;
  SurfF x;         // receiving surface (sensor side for direct/indirect)
  SurfF xe;        // emitter-side surface (indirect)
  F3 rdir;         // incoming direction at x
  F3 T0;           // start throughput / emitted radiance scale
  F3 p0;           // edge point
  F3 n;            // detached xDotN normal
  float w0;        // Detach(baseVal / pdf) factor
  float sedge;     // edge parameter of p0
  int v0, v1;      // edge vertices (-1: not a scene parameter)
  int far_tri;     // triangle intersected by RayIntersectAD
  int pix;         // primary / pixel: pixel of the sensor point
  F3 g;
};

// Primary boundary set-up (SampleFromPrimEdges, Edge.cpp:350-367;
// BoundaryPrimary.cpp:60-130): silhouette edge point, camera ray through it,
// visibility, boundary geometry. Returns false for a rejected sample.
TRN_D bool primary_setup(const Params& P, long long gslot, EdgeState& st, int& vhint, Cnt& cnt) {
  const DeviceScene& s = P.s;
  const ViewDesc& V = view_of(P, gslot, vhint);
  const long long p = gslot - V.begin;
  const CameraDesc& cam = V.cam;
  const PathSmp S{&P, V.seed, gslot, p + V.slot_off};
  const F3 cpos = cam_pos(cam);
  const float r0 = S(0), r1 = S(1);
  float reuse;
  const float integral = __ldg(V.pint);
  if (!(integral > 0.f)) return false;
  const int e = sample_discrete(V.pcdf, P.ne, r0, reuse);
  const int v0 = P.edges[5 * e], v1 = P.edges[5 * e + 1], v2 = P.edges[5 * e + 4];
  const float len_e = V.pfunc[e];
  if (!(len_e > 0.f)) return false;
  const float pmf = len_e / (integral * (float)P.ne);
  const float pdf = pmf / len_e;
  const F3 Pa = load3(s.pos, v0), Pb = load3(s.pos, v1), Pc = load3(s.pos, v2);
  const F3 e1 = Pb - Pa;
  const F3 p0 = Pa + e1 * r1;
  const F3 edge = normalize(e1), edge2 = normalize(Pc - Pa);
  const F3 dir = normalize(p0 - cpos);
  Hit h;
  cnt.v[kCntClosest]++;
  if (!trace_k<TRN_SETUP_SHARED_PRIMARY, false>(s, p0, dir, kShadowEps, kRayMax, h, P.err)) return false;
  const F3 hitP = p0 + dir * h.t;
  const SensorSample sds = sample_direct(cam, hitP);
  if (!sds.valid) return false;
  const F3 dirc = sensor_ray_dir(cam, sds.qx, sds.qy);
  const float dist2cam = length(p0 - cpos);
  cnt.v[kCntShadow]++;
  if (occluded_k<TRN_SETUP_SHARED_PRIMARY>(s, cpos, dirc, kShadowEps, dist2cam - kShadowEps)) return false;
  const SurfF x = post_intersect(s, h.tri, h.u, h.v);
  const float dist = length(x.p - cpos);
  const float dist1 = length(p0 - cpos);
  const float cos2 = fabsf(dot(x.ng, -dirc));
  F3 n;
  const float bval = base_val((dist / dist1), edge, dirc, x.ng, edge2, n) * cos2;
  const int pix = image_pixel(cam, sds.qx, sds.qy);
  const F3 g = g_at(P, V, pix);
  if (bval == 0.f || (g.x == 0.f && g.y == 0.f && g.z == 0.f)) return false;
  st.V = &V; st.gslot = gslot; st.p = p; st.x = x; st.rdir = dirc;
  st.T0 = F3(sds.sensor_val, sds.sensor_val, sds.sensor_val);
  st.p0 = p0; st.n = n; st.w0 = bval / pdf; st.sedge = r1; st.v0 = v0; st.v1 = v1; st.far_tri = h.tri;
  st.pix = pix; st.g = g;
  return true;
}

// Primary boundary body: detached radiance along the camera ray through the
// sensor point (BoundaryPrimary.cpp:150-175), then the xDotN scatter.
// (also the pixel boundary's body: its samples start at dimension 1 and its
// edge point is not a scene parameter, v0 = v1 = -1)
TRN_D void primary_body(const Params& P, const ViewDesc& V, long long gslot, long long p, SurfF x, F3 rdir, F3 T,
                        float w0, const F3& g, int v0, int v1, float sedge, const F3& p0, int far_tri, const F3& n,
                        Cnt& cnt, int dim0 = 2) {
  const DeviceScene& s = P.s;
  const PathSmp S{&P, V.seed, gslot, p + V.slot_off};
  F3 L = scrub(T * emitted(s, x, -rdir));
  for (int b = 0; b < V.D; b++) {
    const int o = dim0 + 5 * b;
    F3 c;
    const bool more = radiance_step_k<TRN_SHARED_STEPS_PRIMARY>(s, x, rdir, T, S(o), S(o + 1), S(o + 2), S(o + 3),
                                                                S(o + 4), c, nullptr, cnt);
    L = L + c;
    if (!more || (T.x == 0.f && T.y == 0.f && T.z == 0.f)) break;
  }
  const float W = dot(g, L * w0);
  if (W == 0.f || !isfinite(W)) return;
  xdotn_vjp(P, V, W, cam_pos(V.cam), false, -1, 0.f, 0.f, v0, v1, sedge, p0, far_tri, n, cnt);
}

__global__ void __launch_bounds__(256, TRN_MINB) k_primary_adj(TRN_KPARAMS) {
  Cnt cnt;
  stage_top(P.s);
  int vhint = 0;
  for_each_valid<EdgeState>(P,
    [&](long long gslot, EdgeState& st) -> bool { return primary_setup(P, gslot, st, vhint, cnt); },
    [&](EdgeState& st) {
      primary_body(P, *st.V, st.gslot, st.p, st.x, st.rdir, st.T0, st.w0, st.g, st.v0, st.v1, st.sedge, st.p0,
                   st.far_tri, st.n, cnt);
    });
  flush_cnt(cnt, P.stats);
}

// Split form: k_primary_setup tests every slot once (no lane waits for the
// others to find an accepted sample, which matters at the ~4 % acceptance of
// silhouette samples) and queues the accepted ones; k_primary_body runs the
// radiance path and the scatter for the queue.
struct PrimaryItem {
  long long gslot, p;
  int view, x_tri, dim0, pad_;
  float x_u, x_v, T0, w0, sedge;
  int v0, v1, far_tri;
  F3 rdir, p0, n, g;
};

__global__ void __launch_bounds__(256, TRN_MINB_SETUP) k_primary_setup(TRN_KPARAMS) {
  Cnt cnt;
  stage_top(P.s);
  int vhint = 0;
  PrimaryItem* q = reinterpret_cast<PrimaryItem*>(P.queue);
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  for (;;) {
    unsigned long long start = 0;
    if (lane == 0) start = atomicAdd(P.work, 32ull);
    start = __shfl_sync(0xffffffffu, start, 0);
    if ((long long)start >= P.total) break;
    const long long g = slot_at(P, (long long)start + lane);
    EdgeState st;
    const bool ok = g < P.total && primary_setup(P, g, st, vhint, cnt);
    const unsigned m = __ballot_sync(0xffffffffu, ok);
    if (!m) continue;
    const int leader = __ffs(m) - 1;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(P.q_count, (unsigned long long)__popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    const unsigned long long k = base + __popc(m & lt);
    if (ok && k >= (unsigned long long)P.q_cap) atomicExch(P.err, 2);
    if (ok && k < (unsigned long long)P.q_cap) {
      PrimaryItem& it = q[k];
      it.gslot = st.gslot; it.p = st.p; it.view = (int)(st.V - P.views); it.dim0 = 2;
      it.x_tri = st.x.tri; it.x_u = st.x.u; it.x_v = st.x.v; it.T0 = st.T0.x; it.w0 = st.w0; it.sedge = st.sedge;
      it.v0 = st.v0; it.v1 = st.v1; it.far_tri = st.far_tri;
      it.rdir = st.rdir; it.p0 = st.p0; it.n = st.n; it.g = st.g;
    }
  }
  flush_cnt(cnt, P.stats);
}

__global__ void __launch_bounds__(256, TRN_MINB_BODY) k_primary_body(TRN_KPARAMS) {
  Cnt cnt;
  stage_top(P.s);
  const PrimaryItem* q = reinterpret_cast<const PrimaryItem*>(P.queue);
  const unsigned long long n = min(*P.q_count, (unsigned long long)P.q_cap);
  for (unsigned long long k = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; k < n;
       k += (unsigned long long)gridDim.x * blockDim.x) {
    const PrimaryItem& it = q[k];
    const SurfF x = post_intersect(P.s, it.x_tri, it.x_u, it.x_v);
    primary_body(P, P.views[it.view], it.gslot, it.p, x, it.rdir, F3(it.T0, it.T0, it.T0), it.w0, it.g, it.v0, it.v1,
                 it.sedge, it.p0, it.far_tri, it.n, cnt, it.dim0);
  }
  flush_cnt(cnt, P.stats);
}

// Path regeneration for the queue's bodies: a lane whose radiance path has
// ended takes the next queue item at once instead of idling until the warp's
// longest path ends (the boundary paths end after one or two bounces on
// average, at most D). Each item runs exactly the steps of primary_body.
#ifndef TRN_BODY_REGEN
#define TRN_BODY_REGEN 1
#endif

__global__ void __launch_bounds__(256, TRN_MINB_BODY) k_primary_body_regen(TRN_KPARAMS) {
  Cnt cnt;
  stage_top(P.s);
  const DeviceScene& s = P.s;
  const PrimaryItem* q = reinterpret_cast<const PrimaryItem*>(P.queue);
  const unsigned long long n = min(*P.q_count, (unsigned long long)P.q_cap);
  unsigned long long* next = P.q_count + 1;  // items handed out (zeroed with the round)
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  bool active = false, done = false;
  unsigned long long k = 0;
  const ViewDesc* V = nullptr;
  SurfF x;
  F3 T, rdir, L;
  int b = 0, D = 0;
  for (;;) {
    const unsigned need = __ballot_sync(0xffffffffu, !active && !done);
    if (need) {
      const int leader = __ffs(need) - 1;
      unsigned long long base = 0;
      if (lane == leader) base = atomicAdd(next, (unsigned long long)__popc(need));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (!active && !done) {
        k = base + __popc(need & lt);
        if (k >= n) {
          done = true;
        } else {
          const PrimaryItem& it = q[k];
          V = P.views + it.view;
          D = V->D;
          x = post_intersect(s, it.x_tri, it.x_u, it.x_v);
          T = F3(it.T0, it.T0, it.T0);
          rdir = it.rdir;
          L = scrub(T * emitted(s, x, -rdir));
          b = 0;
          active = true;
        }
      }
    }
    if (!__any_sync(0xffffffffu, active)) break;
    if (active) {
      bool fin = b >= D;
      if (!fin) {
        const PrimaryItem& it = q[k];
        const PathSmp S{&P, V->seed, it.gslot, it.p + V->slot_off};
        const int o = it.dim0 + 5 * b;
        F3 c;
        const bool more = radiance_step_k<TRN_SHARED_STEPS_PRIMARY>(s, x, rdir, T, S(o), S(o + 1), S(o + 2),
                                                                    S(o + 3), S(o + 4), c, nullptr, cnt);
        L = L + c;
        b++;
        fin = !more || (T.x == 0.f && T.y == 0.f && T.z == 0.f) || b >= D;
      }
      if (fin) {
        const PrimaryItem& it = q[k];
        const float W = dot(it.g, L * it.w0);
        if (W != 0.f && isfinite(W))
          xdotn_vjp(P, *V, W, cam_pos(V->cam), false, -1, 0.f, 0.f, it.v0, it.v1, it.sedge, it.p0, it.far_tri, it.n,
                    cnt);
        active = false;
      }
    }
  }
  flush_cnt(cnt, P.stats);
}

// ---------------------------------------------------------------------------
// direct boundary (BoundaryDirect.cpp:38-143, Edge.cpp:90-144, 201-309)
// ---------------------------------------------------------------------------
// coordinate `axis` of a point placed by r in [0, 1) in guiding leaf `leaf`
TRN_D float aq_lerp(const float* box, long long cap, int leaf, int axis, float r) {
  const float lo = __ldg(box + axis * cap + leaf), hi = __ldg(box + (3 + axis) * cap + leaf);
  return __fadd_rn(lo, __fmul_rn(r, __fsub_rn(hi, lo)));
}

// Direct boundary set-up (SampleBoundarySegmentDirect, Edge.cpp:108-144, with
// AQ guiding when enabled; EvalBoundarySegmentDirect's geometry,
// Edge.cpp:201-291). Returns false for a rejected sample.
TRN_D bool direct_setup(const Params& P, long long gslot, EdgeState& st, int& vhint, Cnt& cnt) {
  const DeviceScene& s = P.s;
  const ViewDesc& V = view_of(P, gslot, vhint);
  const long long p = gslot - V.begin;
  const PathSmp S{&P, V.seed, gslot, p + V.slot_off};
  float r0 = S(0), r1 = S(1), r2 = S(2);
  float reuse;
  const float integral = __ldg(P.eint);
  if (!(integral > 0.f)) return false;
  float pdf_b = 1.f;
  if (P.aq_cdf) {
    // AdaptiveQuadratureDistribution::sample (AQ_distrb.h:176-195): pick a
    // leaf with the extra uniform, then place the (edge, light) sample point
    // uniformly in its box
    if (!(__ldg(P.aq_int) > 0.f)) return false;
    float unused;
    const int leaf = sample_discrete(P.aq_cdf, __ldg(P.aq_n), S(3 + 3 * V.D), unused);
    r0 = aq_lerp(P.aq_box, P.aq_cap, leaf, 0, r0);
    r1 = aq_lerp(P.aq_box, P.aq_cap, leaf, 1, r1);
    r2 = aq_lerp(P.aq_box, P.aq_cap, leaf, 2, r2);
    pdf_b = __fdiv_rn(__ldg(P.aq_poly + leaf), __ldg(P.aq_int + 1));
  }
  const int e = sample_discrete(P.ecdf, P.ne, r0, reuse);
  const int v0 = P.edges[5 * e], v1 = P.edges[5 * e + 1], f0 = P.edges[5 * e + 2], f1 = P.edges[5 * e + 3],
            v2 = P.edges[5 * e + 4];
  const float len_e = P.efunc[e];
  if (!(len_e > 0.f)) return false;
  const float pdf_e = (len_e / (integral * (float)P.ne)) / len_e;
  const F3 Pa = load3(s.pos, v0), Pb = load3(s.pos, v1), Pc = load3(s.pos, v2);
  const F3 e1 = Pb - Pa;
  const F3 p0 = Pa + e1 * reuse;
  const F3 edge = normalize(e1), edge2 = normalize(Pc - Pa);
  LightSample ls;
  if (!light_sample(s, r1, r2, ls)) return false;
  int j0, j1, j2; tri_vertices(s, ls.tri, j0, j1, j2);
  const F3 p2 = bary3(ls.bu, ls.bv, load3(s.pos, j0), load3(s.pos, j1), load3(s.pos, j2));
  const F3 nL = load3(s.fnormal, ls.tri);
  const F3 ev = p2 - p0;
  const float dist_sqr = dot(ev, ev);
  const float dist = sqrtf(dist_sqr);
  const F3 en = ev / dist;
  const float cos_t = dot(nL, -en);
  const F3 n0 = load3(s.fnormal, f0);
  const F3 n1 = f1 >= 0 ? load3(s.fnormal, f1) : F3z();
  const bool is_b = f1 < 0;
  const float c0 = dot(en, n0), c1 = dot(en, n1);
  const bool valid0 = fabsf(c0) > kEdgeEps;
  const bool valid1 = (c0 > kEdgeEps && c1 < -kEdgeEps) || (c0 < -kEdgeEps && c1 > kEdgeEps);
  const bool right = (is_b && valid0) || (!is_b && valid1);
  if (!(right && cos_t > kEps && dist > kShadowEps)) return false;
  const float pdf = pdf_e * ls.pdf * dist_sqr / cos_t * pdf_b;
  const F3 rdir = normalize(p0 - p2);
  Hit h0, h;
  cnt.v[kCntClosest] += 2;
  cnt.v[kCntLight]++;
  if (!trace_k<TRN_SETUP_SHARED_DIRECT, false>(s, p0, -rdir, kShadowEps, kRayMax, h0, P.err)) return false;
  if (!trace_k<TRN_SETUP_SHARED_DIRECT, false>(s, p0, rdir, kShadowEps, kRayMax, h, P.err)) return false;
  const F3 hp = p0 + (-rdir) * h0.t;
  if (!(length(hp - p2) < kShadowEps)) return false;
  const SurfF xl = post_intersect(s, h0.tri, h0.u, h0.v);
  const F3 E = emitted(s, xl, rdir);
  const SurfF x = post_intersect(s, h.tri, h.u, h.v);
  const float dl = length(p2 - x.p);
  const float cos2 = fabsf(dot(nL, rdir));
  const float its_t = length(x.p - p0);
  F3 n;
  const float bval = base_val(its_t / dl, edge, -rdir, nL, edge2, n) * cos2;
  if (bval == 0.f || (E.x == 0.f && E.y == 0.f && E.z == 0.f)) return false;
  st.V = &V; st.gslot = gslot; st.p = p; st.x = x; st.rdir = rdir; st.T0 = E; st.p0 = p0; st.n = n;
  st.w0 = bval / pdf; st.sedge = reuse; st.v0 = v0; st.v1 = v1; st.far_tri = h0.tri;
  return true;
}

// Direct boundary body: trace towards the sensor (EvalImportance per bounce,
// Integrator.cpp:75-176), then the xDotN scatter.
TRN_D void direct_body(const Params& P, const ViewDesc& V, long long gslot, long long p, const SurfF& x0, const F3& rdir,
                       const F3& ev0, int v0, int v1, float sedge, const F3& p0, int far_tri, const F3& n, Cnt& cnt) {
  const DeviceScene& s = P.s;
  const PathSmp S{&P, V.seed, gslot, p + V.slot_off};
  F3 T(1.f, 1.f, 1.f);
  F3 dirs = rdir;
  float W = 0.f;
  SurfF xs = x0;
  for (int b = 0; b < V.D; b++) {
    const int o = 3 + 3 * b;
    F3 c; int pix;
    const bool more = importance_step_k<TRN_SHARED_STEPS_DIRECT>(s, V.cam, xs, dirs, T, S(o), S(o + 1), S(o + 2), c,
                                                                 pix, cnt);
    if (pix >= 0) W += dot(g_at(P, V, pix), ev0 * c);
    if (!more) break;
  }
  if (W == 0.f || !isfinite(W)) return;
  xdotn_vjp(P, V, W, x0.p, true, x0.tri, x0.u, x0.v, v0, v1, sedge, p0, far_tri, n, cnt);
}

__global__ void __launch_bounds__(256, TRN_MINB) k_direct_adj(TRN_KPARAMS) {
  Cnt cnt;
  stage_top(P.s);
  int vhint = 0;
  for_each_valid<EdgeState>(P,
    [&](long long gslot, EdgeState& st) -> bool { return direct_setup(P, gslot, st, vhint, cnt); },
    [&](EdgeState& st) {
      direct_body(P, *st.V, st.gslot, st.p, st.x, st.rdir, st.T0 * st.w0, st.v0, st.v1, st.sedge, st.p0, st.far_tri,
                  st.n, cnt);
    });
  flush_cnt(cnt, P.stats);
}

// Split form: k_direct_setup tests every slot once and queues the accepted
// samples; k_direct_body runs their importance paths and scatters.
struct DirectItem {
  long long gslot, p;
  int view, x_tri, v0, v1, far_tri, pad_;
  float x_u, x_v, sedge, pad2_;
  F3 rdir, ev0, p0, n;
};

__global__ void __launch_bounds__(256, TRN_MINB_SETUP) k_direct_setup(TRN_KPARAMS) {
  Cnt cnt;
  stage_top(P.s);
  int vhint = 0;
  DirectItem* q = reinterpret_cast<DirectItem*>(P.queue);
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  for (;;) {
    unsigned long long start = 0;
    if (lane == 0) start = atomicAdd(P.work, 32ull);
    start = __shfl_sync(0xffffffffu, start, 0);
    if ((long long)start >= P.total) break;
    const long long g = slot_at(P, (long long)start + lane);
    EdgeState st;
    const bool ok = g < P.total && direct_setup(P, g, st, vhint, cnt);
    const unsigned m = __ballot_sync(0xffffffffu, ok);
    if (!m) continue;
    const int leader = __ffs(m) - 1;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(P.q_count, (unsigned long long)__popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    const unsigned long long k = base + __popc(m & lt);
    if (ok && k >= (unsigned long long)P.q_cap) atomicExch(P.err, 2);
    if (ok && k < (unsigned long long)P.q_cap) {
      DirectItem& it = q[k];
      it.gslot = st.gslot; it.p = st.p; it.view = (int)(st.V - P.views);
      it.x_tri = st.x.tri; it.x_u = st.x.u; it.x_v = st.x.v; it.v0 = st.v0; it.v1 = st.v1; it.far_tri = st.far_tri;
      it.sedge = st.sedge; it.rdir = st.rdir; it.ev0 = st.T0 * st.w0; it.p0 = st.p0; it.n = st.n;
    }
  }
  flush_cnt(cnt, P.stats);
}

__global__ void __launch_bounds__(256, TRN_MINB_BODY) k_direct_body(TRN_KPARAMS) {
  Cnt cnt;
  stage_top(P.s);
  const DirectItem* q = reinterpret_cast<const DirectItem*>(P.queue);
  const unsigned long long n = min(*P.q_count, (unsigned long long)P.q_cap);
  for (unsigned long long k = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; k < n;
       k += (unsigned long long)gridDim.x * blockDim.x) {
    const DirectItem& it = q[k];
    const SurfF x = post_intersect(P.s, it.x_tri, it.x_u, it.x_v);
    direct_body(P, P.views[it.view], it.gslot, it.p, x, it.rdir, it.ev0, it.v0, it.v1, it.sedge, it.p0, it.far_tri,
                it.n, cnt);
  }
  flush_cnt(cnt, P.stats);
}

// ---------------------------------------------------------------------------
// AQ guiding of the direct boundary term (AdaptiveQuadratureDistribution::setup,
// AQ_distrb.h:83-173; leaf boxes of NEE.cu:70-89 build_tree at depth 0)
// ---------------------------------------------------------------------------
constexpr uint32_t kGuideTerm = 5;  // hash-sampler term of the set-up samples

// |baseVal| of one (edge, light) sample in guiding mode (Edge.cpp:201-259 with
// guiding_mode=true): only the evaluation mask (same point, both rays hit)
// applies, and neither radiance nor pdf enters. Invalid samples give 0.
TRN_D float guide_base_val(const Params& P, float x, float y, float z) {
  const DeviceScene& s = P.s;
  float reuse;
  const int e = sample_discrete(P.ecdf, P.ne, x, reuse);
  const int v0 = P.edges[5 * e], v1 = P.edges[5 * e + 1], v2 = P.edges[5 * e + 4];
  const F3 Pa = load3(s.pos, v0), Pb = load3(s.pos, v1), Pc = load3(s.pos, v2);
  const F3 e1 = Pb - Pa;
  const F3 p0 = Pa + e1 * reuse;
  const F3 edge = normalize(e1), edge2 = normalize(Pc - Pa);
  LightSample ls;
  if (!light_sample(s, y, z, ls)) return 0.f;
  int j0, j1, j2; tri_vertices(s, ls.tri, j0, j1, j2);
  const F3 p2 = bary3(ls.bu, ls.bv, load3(s.pos, j0), load3(s.pos, j1), load3(s.pos, j2));
  const F3 nL = load3(s.fnormal, ls.tri);
  const F3 rdir = normalize(p0 - p2);
  Hit h0, h;
  if (!trace<false>(s, p0, -rdir, kShadowEps, kRayMax, h0, P.err)) return 0.f;
  if (!trace<false>(s, p0, rdir, kShadowEps, kRayMax, h, P.err)) return 0.f;
  const F3 hp = p0 + (-rdir) * h0.t;
  if (!(length(hp - p2) < kShadowEps)) return 0.f;
  const SurfF xs = post_intersect(s, h.tri, h.u, h.v);
  const float dl = length(p2 - xs.p);
  const float cos2 = fabsf(dot(nL, rdir));
  const float its_t = length(xs.p - p0);
  F3 n;
  const float bv = fabsf(base_val(its_t / dl, edge, -rdir, nL, edge2, n) * cos2);
  return isfinite(bv) ? bv : 0.f;
}

constexpr uint32_t kRefineTerm = 6;  // hash-sampler term of the refinement's random points
constexpr int kAqPoints = 36;        // evaluation points per leaf and refinement pass

// Depth-0 tree (build_tree, NEE.cu:70-89, with one y and one z cell): leaf i
// is edge i's interval of the secondary-edge CDF times [0, 1]^2.
__global__ void k_aq_init(int ne, const float* ecdf, float* box, int* edge, int* count, long long cap) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) { count[0] = ne; count[1] = ne; }
  if (i >= ne) return;
  box[i] = i > 0 ? ecdf[i - 1] : 0.f;
  box[cap + i] = 0.f;
  box[2 * cap + i] = 0.f;
  box[3 * cap + i] = ecdf[i];
  box[4 * cap + i] = 1.f;
  box[5 * cap + i] = 1.f;
  edge[i] = i;
}

// Evaluation point k of a leaf for a refinement pass (gen_eval_point,
// NEE.cu:91-240, with the box midpoint m = (p0 + p1) / 2): k < 16 are the
// corners and edge midpoints of the x = p0 and x = p1 faces, 16..19 the
// corners of the x = m section, and 20..35 two random points in each octant
// (octant bits x, y, z = bits 2, 1, 0 of k - 20; the second eight use 1 - r).
TRN_D void aq_point(const float* box, long long cap, int leaf, int k, uint32_t stream, float out[3]) {
  float lo[3], hi[3], mid[3];
  for (int a = 0; a < 3; a++) {
    lo[a] = box[a * cap + leaf];
    hi[a] = box[(3 + a) * cap + leaf];
    mid[a] = __fmul_rn(__fadd_rn(lo[a], hi[a]), 0.5f);
  }
  if (k < 20) {
    // (y, z) of the face points: low, high or middle per axis
    const unsigned char yz16[8][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 0}, {1, 1}, {1, 2}, {2, 0}, {2, 1}};
    const unsigned char yz4[4][2] = {{0, 0}, {0, 1}, {1, 0}, {1, 1}};
    const int sx = k < 8 ? 0 : (k < 16 ? 1 : 2);
    const unsigned char* yz = k < 16 ? yz16[k & 7] : yz4[k - 16];
    auto pick = [&](int a, int c) { return c == 0 ? lo[a] : (c == 1 ? hi[a] : mid[a]); };
    out[0] = pick(0, sx);
    out[1] = pick(1, yz[0]);
    out[2] = pick(2, yz[1]);
    return;
  }
  const int o = (k - 20) & 7;
  for (int a = 0; a < 3; a++) {
    float r = hash_uniform(stream, kRefineTerm, (uint32_t)(3 * (k - 20) + a), (uint32_t)leaf);
    if (k >= 28) r = __fsub_rn(1.f, r);
    const float base = ((o >> (2 - a)) & 1) ? mid[a] : lo[a];
    out[a] = __fadd_rn(base, __fmul_rn(__fsub_rn(mid[a], lo[a]), r));
  }
}

// One thread per (leaf, point): |baseVal| at the refinement's evaluation
// points (GuideDirectBoundary_Helper, AQ_distrb.h:65-79).
__global__ void k_aq_eval(TRN_KPARAMS, uint32_t stream, const float* box, const int* edge, const int* count,
                          long long cap, float* eval) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int leaf = (int)(t / kAqPoints), k = (int)(t % kAqPoints);
  if (leaf >= __ldg(count)) return;
  float v = 0.f;
  if (P.efunc[edge[leaf]] > 0.f && __ldg(P.eint) > 0.f) {
    float x[3];
    aq_point(box, cap, leaf, k, stream, x);
    v = guide_base_val(P, x[0], x[1], x[2]);
  }
  eval[t] = v;
}

// sum of the 8 listed evaluation values of a leaf, added in list order, over 8
TRN_D float aq_avg8(const float* e, int a, int b, int c, int d, int f, int g, int h, int i) {
  float s = __fadd_rn(e[a], e[b]);
  s = __fadd_rn(s, e[c]);
  s = __fadd_rn(s, e[d]);
  s = __fadd_rn(s, e[f]);
  s = __fadd_rn(s, e[g]);
  s = __fadd_rn(s, e[h]);
  s = __fadd_rn(s, e[i]);
  return __fdiv_rn(s, 8.f);
}

// Split decision per leaf (cut_tree, NEE.cu:243-396): the leaf's error is
// |corner average - Monte Carlo average| x volume; above `thold` it splits
// along the axis whose two halves disagree most between their corner and
// Monte Carlo averages (a random axis on ties). flag = 0 (keep) or 1 + axis.
__global__ void k_aq_flag(const float* box, const int* count, long long cap, const float* eval, float thold,
                          uint32_t stream, int* flag) {
  const int leaf = blockIdx.x * blockDim.x + threadIdx.x;
  if (leaf >= __ldg(count)) return;
  const float* e = eval + (long long)leaf * kAqPoints;
  const float vol = __fmul_rn(__fmul_rn(__fsub_rn(box[3 * cap + leaf], box[leaf]),
                                        __fsub_rn(box[4 * cap + leaf], box[cap + leaf])),
                              __fsub_rn(box[5 * cap + leaf], box[2 * cap + leaf]));
  const float lag = aq_avg8(e, 0, 1, 3, 4, 8, 9, 11, 12);
  float mc = 0.f;
  for (int k = 20; k < 36; k++) mc = __fadd_rn(mc, e[k]);
  mc = __fdiv_rn(mc, 16.f);
  const float err = __fmul_rn(fabsf(__fsub_rn(lag, mc)), vol);
  int f = 0;
  if (err > thold) {
    const float d1a = aq_avg8(e, 0, 1, 3, 4, 16, 17, 18, 19), d1b = aq_avg8(e, 8, 9, 11, 12, 16, 17, 18, 19);
    const float d2a = aq_avg8(e, 0, 1, 6, 7, 8, 9, 14, 15), d2b = aq_avg8(e, 3, 4, 6, 7, 11, 12, 14, 15);
    const float d3a = aq_avg8(e, 0, 2, 3, 5, 8, 10, 11, 13), d3b = aq_avg8(e, 1, 2, 4, 5, 9, 10, 12, 13);
    const float m1a = aq_avg8(e, 20, 21, 22, 23, 28, 29, 30, 31), m1b = aq_avg8(e, 24, 25, 26, 27, 32, 33, 34, 35);
    const float m2a = aq_avg8(e, 20, 21, 24, 25, 28, 29, 32, 33), m2b = aq_avg8(e, 22, 23, 26, 27, 30, 31, 34, 35);
    const float m3a = aq_avg8(e, 20, 22, 24, 26, 28, 30, 32, 34), m3b = aq_avg8(e, 21, 23, 25, 27, 29, 31, 33, 35);
    const float e0 = fabsf(__fsub_rn(fabsf(__fsub_rn(d1a, m1a)), fabsf(__fsub_rn(d1b, m1b))));
    const float e1 = fabsf(__fsub_rn(fabsf(__fsub_rn(d2a, m2a)), fabsf(__fsub_rn(d2b, m2b))));
    const float e2 = fabsf(__fsub_rn(fabsf(__fsub_rn(d3a, m3a)), fabsf(__fsub_rn(d3b, m3b))));
    int axis;
    if (e0 > e1 && e0 > e2) axis = 0;
    else if (e1 > e0 && e1 > e2) axis = 1;
    else if (e2 > e0 && e2 > e1) axis = 2;
    else {
      const float r = __fmul_rn(hash_uniform(stream, kRefineTerm, 48u, (uint32_t)leaf), 3.f);
      axis = r < 1.f ? 0 : (r < 2.f ? 1 : 2);
    }
    f = 1 + axis;
  }
  flag[leaf] = f;
}

// Exclusive prefix count of the split flags in leaf order (one block), so
// that new leaves are appended in a fixed order; count[1] = leaves after the
// pass, at most `limit`.
__global__ void k_aq_scan(const int* count, const int* flag, int* prefix, int* count_out, int limit) {
  __shared__ int part[1024];
  const int n = __ldg(count);
  const int T = blockDim.x, tid = threadIdx.x;
  const int chunk = (n + T - 1) / T;
  const int a = min(n, tid * chunk), b = min(n, a + chunk);
  int acc = 0;
  for (int i = a; i < b; i++) acc += flag[i] != 0;
  part[tid] = acc;
  __syncthreads();
  if (tid == 0) {
    int run = 0;
    for (int i = 0; i < T; i++) { const int x = part[i]; part[i] = run; run += x; }
    count_out[1] = min(n + run, limit);
  }
  __syncthreads();
  int run = part[tid];
  for (int i = a; i < b; i++) { prefix[i] = run; run += flag[i] != 0; }
}

// Split the flagged leaves: the leaf keeps the lower half along its axis and
// the new leaf n + prefix takes the upper half (cut_tree's split).
__global__ void k_aq_split(const int* count, const int* flag, const int* prefix, float* box, int* edge,
                           long long cap) {
  const int leaf = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = __ldg(count);
  if (leaf >= n || flag[leaf] == 0) return;
  const int idx = n + prefix[leaf];
  if (idx >= __ldg(count + 1)) return;
  const int axis = flag[leaf] - 1;
  const float lo = box[axis * cap + leaf], hi = box[(3 + axis) * cap + leaf];
  const float mid = __fmul_rn(__fadd_rn(lo, hi), 0.5f);
  for (int c = 0; c < 6; c++) box[c * cap + idx] = box[c * cap + leaf];
  box[axis * cap + idx] = mid;
  box[(3 + axis) * cap + leaf] = mid;
  edge[idx] = edge[leaf];
}

__global__ void k_aq_commit(int* count) { count[0] = count[1]; }

// Leaf weight = mean |baseVal| over gspp uniform samples in the leaf box
// (AQ_distrb.h:150-161). Leaves on non-secondary edges (zero length in the
// edge distribution) do not exist in the reference's compacted edge list and
// get weight 0 here.
__global__ void k_aq_poly(TRN_KPARAMS, uint32_t stream, int gspp, const float* box, const int* edge, const int* count,
                          long long cap, float* poly) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= __ldg(count)) return;
  float acc = 0.f;
  if (P.efunc[edge[i]] > 0.f && __ldg(P.eint) > 0.f) {
    const float fs = (float)gspp;
    for (int k = 0; k < gspp; k++) {
      const uint32_t slot = (uint32_t)i * (uint32_t)gspp + (uint32_t)k;
      const float x = aq_lerp(box, cap, i, 0, hash_uniform(stream, kGuideTerm, 0, slot));
      const float y = aq_lerp(box, cap, i, 1, hash_uniform(stream, kGuideTerm, 1, slot));
      const float z = aq_lerp(box, cap, i, 2, hash_uniform(stream, kGuideTerm, 2, slot));
      acc = __fadd_rn(acc, __fdiv_rn(guide_base_val(P, x, y, z), fs));
    }
  }
  poly[i] = acc;
}

// poly /= sum(poly); poly = eps + (1 - eps) poly; func = poly x leaf volume;
// out[1] = sum(func) (the pdf normaliser of AQ_distrb.h:194). One block of
// 1024 threads.
__global__ void k_aq_mix(const int* count, float* poly, const float* box, long long cap, float eps, float* func,
                         float* out) {
  __shared__ double part[1024];
  const int n = __ldg(count);
  const int tid = threadIdx.x, T = blockDim.x;
  double acc = 0.0;
  for (int i = tid; i < n; i += T) acc += (double)poly[i];
  part[tid] = acc;
  __syncthreads();
  for (int w = T / 2; w > 0; w >>= 1) {
    if (tid < w) part[tid] += part[tid + w];
    __syncthreads();
  }
  const double tot = part[0];
  __syncthreads();
  const float ftot = (float)tot;
  const float one_m = (float)(1.0 - (double)eps);
  acc = 0.0;
  for (int i = tid; i < n; i += T) {
    float p = poly[i];
    if (tot > 0.0) p = __fdiv_rn(p, ftot);
    p = __fadd_rn(eps, __fmul_rn(one_m, p));
    const float vol = __fmul_rn(__fmul_rn(__fsub_rn(box[3 * cap + i], box[i]), __fsub_rn(box[4 * cap + i], box[cap + i])),
                                __fsub_rn(box[5 * cap + i], box[2 * cap + i]));
    const float f = __fmul_rn(p, vol);
    poly[i] = p;
    func[i] = f;
    acc += (double)f;
  }
  part[tid] = acc;
  __syncthreads();
  for (int w = T / 2; w > 0; w >>= 1) {
    if (tid < w) part[tid] += part[tid + w];
    __syncthreads();
  }
  if (tid == 0) out[1] = (float)part[0];
}

// ---------------------------------------------------------------------------
// indirect boundary (BoundaryIndirect.cpp:38-192, Edge.cpp:146-199)
// ---------------------------------------------------------------------------
// Indirect boundary set-up (SampleBoundarySegmentIndirect, Edge.cpp:146-199,
// BoundaryIndirect.cpp:58-130): edge point, direction in the edge wedge, both
// rays, boundary geometry. Returns false for a rejected sample.
TRN_D bool indirect_setup(const Params& P, long long gslot, EdgeState& st, int& vhint, Cnt& cnt) {
  const DeviceScene& s = P.s;
  const ViewDesc& V = view_of(P, gslot, vhint);
  const long long p = gslot - V.begin;
  if (V.D < 2) return false;
  const PathSmp S{&P, V.seed, gslot, p + V.slot_off};
  const float r0 = S(0), r1 = S(1), r2 = S(2);
  float reuse;
  const float integral = __ldg(P.eint);
  if (!(integral > 0.f)) return false;
  const int e = sample_discrete(P.ecdf, P.ne, r0, reuse);
  const int v0 = P.edges[5 * e], v1 = P.edges[5 * e + 1], f0 = P.edges[5 * e + 2], f1 = P.edges[5 * e + 3],
            v2 = P.edges[5 * e + 4];
  const float len_e = P.efunc[e];
  if (!(len_e > 0.f)) return false;
  const float pdf_e = (len_e / (integral * (float)P.ne)) / len_e;
  const F3 Pa = load3(s.pos, v0), Pb = load3(s.pos, v1), Pc = load3(s.pos, v2);
  const F3 e1 = Pb - Pa;
  const F3 p0 = Pa + e1 * reuse;
  const F3 edge = normalize(e1), edge2 = normalize(Pc - Pa);
  const F3 n0 = load3(s.fnormal, f0);
  F3 dir;
  float pdf_d;
  if (f1 < 0) {
    const F3 nrm = cross(n0, edge);
    F3 tg, bt; coordinate_system(nrm, tg, bt);
    const float z = fminf(1.f - 2.f * r1, 1.f - kEdgeEps);
    const float r = sqrtf(fmaxf(0.f, 1.f - z * z));
    const float phi = 2.f * kPi * r2;
    float sp, cp;
    sincos_det(phi, sp, cp);
    dir = tg * (r * cp) + bt * (r * sp) + nrm * z;
    pdf_d = 0.25f / kPi;
  } else {
    const F3 n1 = load3(s.fnormal, f1);
    const float phi0 = acos_det(dot(n0, n1));
    pdf_d = 0.25f / phi0;
    const F3 zz = normalize(n0 + n1);
    const F3 yy = normalize(cross(n0, zz));
    const F3 xx = cross(yy, zz);
    float phi = (r1 - 0.5f) * phi0;
    phi = fminf(fmaxf(phi, -0.5f * phi0 + kEdgeEps), 0.5f * phi0 - kEdgeEps);
    float sp, cp;
    sincos_det(phi, sp, cp);
    const F3 x1 = xx * cp + zz * sp;
    const bool m0 = r2 > 0.5f;
    const float bq = 4.f * r2 - (m0 ? 3.f : 1.f);
    const float aq = sqrtf(1.f - bq * bq) * (1.f - (m0 ? 1.f : 0.f) * 2.f);
    dir = x1 * aq + yy * bq;
  }
  const float pdf = pdf_e * pdf_d;
  Hit he, hs;
  cnt.v[kCntClosest] += 2;
#if TRN_INDIRECT_SENSOR_FIRST
  if (!trace_k<TRN_INDIRECT_SETUP_SHARED, false>(s, p0, dir, kShadowEps, kRayMax, hs, P.err)) return false;
  if (!trace_k<TRN_INDIRECT_SETUP_SHARED, false>(s, p0, -dir, kShadowEps, kRayMax, he, P.err)) return false;
#else
  if (!trace_k<TRN_INDIRECT_SETUP_SHARED, false>(s, p0, -dir, kShadowEps, kRayMax, he, P.err)) return false;
  if (!trace_k<TRN_INDIRECT_SETUP_SHARED, false>(s, p0, dir, kShadowEps, kRayMax, hs, P.err)) return false;
#endif
  const SurfF xe = post_intersect(s, he.tri, he.u, he.v);
  const SurfF xs = post_intersect(s, hs.tri, hs.u, hs.v);
  const float dl = length(xe.p - xs.p);
  const float cos2 = fabsf(dot(xe.ng, dir));
  const float its_t = length(xs.p - p0);
  F3 n;
  const float bval = base_val(its_t / dl, edge, -dir, xe.ng, edge2, n) * cos2;
  if (bval == 0.f) return false;
  st.V = &V; st.gslot = gslot; st.p = p; st.x = xs; st.xe = xe; st.rdir = dir; st.p0 = p0; st.n = n;
  st.w0 = bval / pdf; st.sedge = reuse; st.v0 = v0; st.v1 = v1; st.far_tri = he.tri;
  return true;
}

// Indirect boundary sensor side (BoundaryIndirect.cpp:158-175 pairs sensor
// depth b with the emitter radiance accumulated over D-1-b bounces): the
// importance contributions of every depth, weighted by dL/dI of their pixels.
// Returns the shallowest depth that reached the image with a nonzero weight
// (D when none did).
template <int MAXD>
TRN_D int indirect_sensor(const Params& P, const EdgeState& st, int D, F3* sc, Cnt& cnt) {
  const DeviceScene& s = P.s;
  const ViewDesc& V = *st.V;
  const PathSmp S{&P, V.seed, st.gslot, st.p + V.slot_off};
  int bmin = D;
  F3 T(1.f, 1.f, 1.f);
  F3 rd = st.rdir;
  SurfF xx = st.x;
  for (int b = 0; b < D - 1; b++) sc[b] = F3z();
  for (int b = 0; b < D - 1; b++) {
    const int o = 3 + 5 * (D - 1) + 3 * b;
    F3 c; int pix;
    const bool more = importance_step_shared(s, V.cam, xx, rd, T, S(o), S(o + 1), S(o + 2), c, pix, cnt);
    if (pix >= 0) {
      sc[b] = g_at(P, V, pix) * c;
      if (sc[b].x != 0.f || sc[b].y != 0.f || sc[b].z != 0.f) bmin = min(bmin, b);
    }
    if (!more) break;
  }
  return bmin;
}

// Indirect boundary emitter side: the radiance accumulated over j+1 bounces
// from the emitter-side surface pairs with sensor depth D-2-j; returns the
// weight W of the xDotN scatter.
template <int MAXD>
TRN_D float indirect_emitter(const Params& P, const ViewDesc& V, long long gslot, long long p, const SurfF& xe,
                             const F3& rdir, float w0, int D, int jmax, const F3* sc, Cnt& cnt) {
  const DeviceScene& s = P.s;
  const PathSmp S{&P, V.seed, gslot, p + V.slot_off};
  float W = 0.f;
  F3 T(1.f, 1.f, 1.f);
  F3 rd = -rdir;
  SurfF xx = xe;
  F3 cur = F3z();
  bool alive = true;
  for (int j = 0; j <= jmax; j++) {
    if (alive) {
      const int o = 3 + 5 * j;
      F3 c;
      alive = radiance_step_shared(s, xx, rd, T, S(o), S(o + 1), S(o + 2), S(o + 3), S(o + 4), c, nullptr, cnt);
      cur = cur + c;
      if (T.x == 0.f && T.y == 0.f && T.z == 0.f) alive = false;
    }
    W += dot(sc[D - 2 - j], cur) * w0;
  }
  return W;
}

template <int MAXD>
__global__ void __launch_bounds__(256, TRN_MINB_INDIRECT) k_indirect_adj(TRN_KPARAMS) {
  Cnt cnt;
  stage_top(P.s);
  int vhint = 0;
  for_each_valid<EdgeState>(P,
    [&](long long gslot, EdgeState& st) -> bool { return indirect_setup(P, gslot, st, vhint, cnt); },
    [&](EdgeState& st) {
      const ViewDesc& V = *st.V;
      const int D = min(V.D, MAXD);
      // sensor side first; the emitter side then only runs as deep as the
      // shallowest sensor depth that reached the image needs, and not at all
      // when none did
      F3 sc[MAXD];
      const int bmin = indirect_sensor<MAXD>(P, st, D, sc, cnt);
      if (bmin >= D - 1) return;
      const float W = indirect_emitter<MAXD>(P, V, st.gslot, st.p, st.xe, st.rdir, st.w0, D, D - 2 - bmin, sc, cnt);
      if (W == 0.f || !isfinite(W)) return;
      xdotn_vjp(P, V, W, st.x.p, true, st.x.tri, st.x.u, st.x.v, st.v0, st.v1, st.sedge, st.p0, st.far_tri, st.n,
                cnt);
    });
  flush_cnt(cnt, P.stats);
}

// Split form of the same term: k_indirect_sensor runs the set-up and the
// sensor side and queues the samples whose sensor side reached the image;
// k_indirect_emitter runs the emitter side and the scatter for the queue.
// Each kernel carries half of the fused kernel's code (the fused kernel is
// instruction-fetch bound), and the emitter pass runs on survivors only.
template <int MAXD>
struct IndirectItem {
  long long gslot, p;
  int view, jmax, D;
  int xe_tri, xs_tri;
  float xe_u, xe_v, xs_u, xs_v;
  F3 rdir, p0, n;
  float w0, sedge;
  int v0, v1, far_tri;
  F3 sc[MAXD];
};

template <int MAXD>
__global__ void __launch_bounds__(256, TRN_MINB_INDIRECT) k_indirect_sensor(TRN_KPARAMS) {
  Cnt cnt;
  stage_top(P.s);
  int vhint = 0;
  IndirectItem<MAXD>* q = reinterpret_cast<IndirectItem<MAXD>*>(P.queue);
  for_each_valid<EdgeState>(P,
    [&](long long gslot, EdgeState& st) -> bool { return indirect_setup(P, gslot, st, vhint, cnt); },
    [&](EdgeState& st) {
      const int D = min(st.V->D, MAXD);
      F3 sc[MAXD];
      const int bmin = indirect_sensor<MAXD>(P, st, D, sc, cnt);
      if (bmin >= D - 1) return;
      const unsigned long long k = atomicAdd(P.q_count, 1ull);
      if (k >= (unsigned long long)P.q_cap) { atomicExch(P.err, 2); return; }
      IndirectItem<MAXD>& it = q[k];
      it.gslot = st.gslot; it.p = st.p;
      it.view = (int)(st.V - P.views); it.jmax = D - 2 - bmin; it.D = D;
      it.xe_tri = st.xe.tri; it.xe_u = st.xe.u; it.xe_v = st.xe.v;
      it.xs_tri = st.x.tri; it.xs_u = st.x.u; it.xs_v = st.x.v;
      it.rdir = st.rdir; it.p0 = st.p0; it.n = st.n; it.w0 = st.w0; it.sedge = st.sedge;
      it.v0 = st.v0; it.v1 = st.v1; it.far_tri = st.far_tri;
      for (int b = 0; b < D - 1; b++) it.sc[b] = sc[b];
    });
  flush_cnt(cnt, P.stats);
}

template <int MAXD>
__global__ void __launch_bounds__(256, TRN_MINB_INDIRECT) k_indirect_emitter(TRN_KPARAMS) {
  Cnt cnt;
  stage_top(P.s);
  // two-stage form: the queue and its count; three-stage form: the second queue
  const IndirectItem<MAXD>* q = reinterpret_cast<const IndirectItem<MAXD>*>(P.queue2 ? P.queue2 : P.queue);
  const unsigned long long n = min(P.q_count[P.queue2 ? 1 : 0], (unsigned long long)P.q_cap);
  for (unsigned long long k = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; k < n;
       k += (unsigned long long)gridDim.x * blockDim.x) {
    const IndirectItem<MAXD>& it = q[k];
    const ViewDesc& V = P.views[it.view];
    const SurfF xe = post_intersect(P.s, it.xe_tri, it.xe_u, it.xe_v);
    const float W = indirect_emitter<MAXD>(P, V, it.gslot, it.p, xe, it.rdir, it.w0, it.D, it.jmax, it.sc, cnt);
    if (W == 0.f || !isfinite(W)) continue;
    const SurfF xs = post_intersect(P.s, it.xs_tri, it.xs_u, it.xs_v);
    xdotn_vjp(P, V, W, xs.p, true, it.xs_tri, it.xs_u, it.xs_v, it.v0, it.v1, it.sedge, it.p0, it.far_tri, it.n,
              cnt);
  }
  flush_cnt(cnt, P.stats);
}

// Three-stage form of the indirect term: k_indirect_setup tests every slot
// once (the two set-up rays are most of the term's rays) and queues the
// accepted samples; k_indirect_sensor_q runs the sensor side over that queue
// and queues survivors for k_indirect_emitter.
struct IndirectSetupItem {
  long long gslot, p;
  int view, xe_tri, xs_tri, v0, v1, far_tri;
  float xe_u, xe_v, xs_u, xs_v, w0, sedge;
  F3 rdir, p0, n;
};

__global__ void __launch_bounds__(256, TRN_MINB_SETUP) k_indirect_setup(TRN_KPARAMS) {
  Cnt cnt;
  stage_top(P.s);
  int vhint = 0;
  IndirectSetupItem* q = reinterpret_cast<IndirectSetupItem*>(P.queue);
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  for (;;) {
    unsigned long long start = 0;
    if (lane == 0) start = atomicAdd(P.work, 32ull);
    start = __shfl_sync(0xffffffffu, start, 0);
    if ((long long)start >= P.total) break;
    const long long g = slot_at(P, (long long)start + lane);
    EdgeState st;
    const bool ok = g < P.total && indirect_setup(P, g, st, vhint, cnt);
    const unsigned m = __ballot_sync(0xffffffffu, ok);
    if (!m) continue;
    const int leader = __ffs(m) - 1;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(P.q_count, (unsigned long long)__popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    const unsigned long long k = base + __popc(m & lt);
    if (ok && k >= (unsigned long long)P.q_cap) atomicExch(P.err, 2);
    if (ok && k < (unsigned long long)P.q_cap) {
      IndirectSetupItem& it = q[k];
      it.gslot = st.gslot; it.p = st.p; it.view = (int)(st.V - P.views);
      it.xe_tri = st.xe.tri; it.xe_u = st.xe.u; it.xe_v = st.xe.v;
      it.xs_tri = st.x.tri; it.xs_u = st.x.u; it.xs_v = st.x.v;
      it.v0 = st.v0; it.v1 = st.v1; it.far_tri = st.far_tri; it.w0 = st.w0; it.sedge = st.sedge;
      it.rdir = st.rdir; it.p0 = st.p0; it.n = st.n;
    }
  }
  flush_cnt(cnt, P.stats);
}

template <int MAXD>
__global__ void __launch_bounds__(256, TRN_MINB_INDIRECT) k_indirect_sensor_q(TRN_KPARAMS) {
  Cnt cnt;
  stage_top(P.s);
  const IndirectSetupItem* qa = reinterpret_cast<const IndirectSetupItem*>(P.queue);
  IndirectItem<MAXD>* qb = reinterpret_cast<IndirectItem<MAXD>*>(P.queue2);
  const unsigned long long n = min(P.q_count[0], (unsigned long long)P.q_cap);
  const int lane = threadIdx.x & 31;
  for (unsigned long long k0 = (blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x) & ~31ull; k0 < n;
       k0 += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long k = k0 + lane;
    bool push = false;
    EdgeState st;
    F3 sc[MAXD];
    int D = 0, bmin = 0;
    if (k < n) {
      const IndirectSetupItem& a = qa[k];
      st.V = P.views + a.view; st.gslot = a.gslot; st.p = a.p;
      st.x = post_intersect(P.s, a.xs_tri, a.xs_u, a.xs_v);
      st.rdir = a.rdir;
      D = min(st.V->D, MAXD);
      bmin = indirect_sensor<MAXD>(P, st, D, sc, cnt);
      push = bmin < D - 1;
    }
    const unsigned m = __ballot_sync(0xffffffffu, push);
    if (!m) continue;
    const int leader = __ffs(m) - 1;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(P.q_count + 1, (unsigned long long)__popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    const unsigned long long j = base + __popc(m & ((1u << lane) - 1u));
    if (push && j >= (unsigned long long)P.q_cap) atomicExch(P.err, 2);
    if (push && j < (unsigned long long)P.q_cap) {
      const IndirectSetupItem& a = qa[k];
      IndirectItem<MAXD>& it = qb[j];
      it.gslot = a.gslot; it.p = a.p; it.view = a.view; it.jmax = D - 2 - bmin; it.D = D;
      it.xe_tri = a.xe_tri; it.xe_u = a.xe_u; it.xe_v = a.xe_v;
      it.xs_tri = a.xs_tri; it.xs_u = a.xs_u; it.xs_v = a.xs_v;
      it.rdir = a.rdir; it.p0 = a.p0; it.n = a.n; it.w0 = a.w0; it.sedge = a.sedge;
      it.v0 = a.v0; it.v1 = a.v1; it.far_tri = a.far_tri;
      for (int b = 0; b < D - 1; b++) it.sc[b] = sc[b];
    }
  }
  flush_cnt(cnt, P.stats);
}

// k_indirect_sensor_q with path regeneration: a lane whose importance path
// has ended queues its item (when a depth reached the image) and takes the
// next set-up item at once. Each item runs exactly the steps of
// indirect_sensor.
#ifndef TRN_SENSOR_REGEN
#define TRN_SENSOR_REGEN 1
#endif

template <int MAXD>
__global__ void __launch_bounds__(256, TRN_MINB_INDIRECT) k_indirect_sensor_regen(TRN_KPARAMS) {
  Cnt cnt;
  stage_top(P.s);
  const DeviceScene& s = P.s;
  const IndirectSetupItem* qa = reinterpret_cast<const IndirectSetupItem*>(P.queue);
  IndirectItem<MAXD>* qb = reinterpret_cast<IndirectItem<MAXD>*>(P.queue2);
  const unsigned long long n = min(P.q_count[0], (unsigned long long)P.q_cap);
  unsigned long long* next = P.q_count + 2;
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  bool active = false, done = false;
  unsigned long long k = 0;
  const ViewDesc* V = nullptr;
  SurfF xx;
  F3 T, rd;
  F3 sc[MAXD];
  int b = 0, D = 0, bmin = 0;
  for (;;) {
    const unsigned need = __ballot_sync(0xffffffffu, !active && !done);
    if (need) {
      const int leader = __ffs(need) - 1;
      unsigned long long base = 0;
      if (lane == leader) base = atomicAdd(next, (unsigned long long)__popc(need));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (!active && !done) {
        k = base + __popc(need & lt);
        if (k >= n) {
          done = true;
        } else {
          const IndirectSetupItem& a = qa[k];
          V = P.views + a.view;
          D = min(V->D, MAXD);
          xx = post_intersect(s, a.xs_tri, a.xs_u, a.xs_v);
          rd = a.rdir;
          T = F3(1.f, 1.f, 1.f);
          for (int j = 0; j < D - 1; j++) sc[j] = F3z();
          bmin = D;
          b = 0;
          active = true;
        }
      }
    }
    if (!__any_sync(0xffffffffu, active)) break;
    bool fin = false;
    if (active) {
      fin = b >= D - 1;
      if (!fin) {
        const IndirectSetupItem& a = qa[k];
        const PathSmp S{&P, V->seed, a.gslot, a.p + V->slot_off};
        const int o = 3 + 5 * (D - 1) + 3 * b;
        F3 c;
        int pix;
        const bool more = importance_step_k<TRN_SHARED_STEPS_INDIRECT>(s, V->cam, xx, rd, T, S(o), S(o + 1),
                                                                        S(o + 2), c, pix, cnt);
        if (pix >= 0) {
          sc[b] = g_at(P, *V, pix) * c;
          if (sc[b].x != 0.f || sc[b].y != 0.f || sc[b].z != 0.f) bmin = min(bmin, b);
        }
        b++;
        fin = !more || b >= D - 1;
      }
    }
    const bool push = fin && bmin < D - 1;
    const unsigned m = __ballot_sync(0xffffffffu, push);
    if (m) {
      const int leader = __ffs(m) - 1;
      unsigned long long base = 0;
      if (lane == leader) base = atomicAdd(P.q_count + 1, (unsigned long long)__popc(m));
      base = __shfl_sync(0xffffffffu, base, leader);
      const unsigned long long j = base + __popc(m & lt);
      if (push && j >= (unsigned long long)P.q_cap) atomicExch(P.err, 2);
      if (push && j < (unsigned long long)P.q_cap) {
        const IndirectSetupItem& a = qa[k];
        IndirectItem<MAXD>& it = qb[j];
        it.gslot = a.gslot; it.p = a.p; it.view = a.view; it.jmax = D - 2 - bmin; it.D = D;
        it.xe_tri = a.xe_tri; it.xe_u = a.xe_u; it.xe_v = a.xe_v;
        it.xs_tri = a.xs_tri; it.xs_u = a.xs_u; it.xs_v = a.xs_v;
        it.rdir = a.rdir; it.p0 = a.p0; it.n = a.n; it.w0 = a.w0; it.sedge = a.sedge;
        it.v0 = a.v0; it.v1 = a.v1; it.far_tri = a.far_tri;
        for (int q = 0; q < D - 1; q++) it.sc[q] = sc[q];
      }
    }
    if (fin) active = false;
  }
  flush_cnt(cnt, P.stats);
}

// k_indirect_emitter with path regeneration (three-stage form): a lane whose
// emitter-side path has ended adds the remaining depths' terms with its last
// radiance, as the loop form does after the path dies, scatters, and takes
// the next item at once. Each item runs exactly the steps and the
// additions of indirect_emitter.
#ifndef TRN_EMITTER_REGEN
#define TRN_EMITTER_REGEN 1
#endif

template <int MAXD>
__global__ void __launch_bounds__(256, TRN_MINB_INDIRECT) k_indirect_emitter_regen(TRN_KPARAMS) {
  Cnt cnt;
  stage_top(P.s);
  const DeviceScene& s = P.s;
  const IndirectItem<MAXD>* q = reinterpret_cast<const IndirectItem<MAXD>*>(P.queue2);
  const unsigned long long n = min(P.q_count[1], (unsigned long long)P.q_cap);
  unsigned long long* next = P.q_count + 3;
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  bool active = false, done = false;
  unsigned long long k = 0;
  const ViewDesc* V = nullptr;
  SurfF xx;
  F3 T, rd, cur;
  float W = 0.f;
  int j = 0;
  for (;;) {
    const unsigned need = __ballot_sync(0xffffffffu, !active && !done);
    if (need) {
      const int leader = __ffs(need) - 1;
      unsigned long long base = 0;
      if (lane == leader) base = atomicAdd(next, (unsigned long long)__popc(need));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (!active && !done) {
        k = base + __popc(need & lt);
        if (k >= n) {
          done = true;
        } else {
          const IndirectItem<MAXD>& it = q[k];
          V = P.views + it.view;
          xx = post_intersect(s, it.xe_tri, it.xe_u, it.xe_v);
          rd = -it.rdir;
          T = F3(1.f, 1.f, 1.f);
          cur = F3z();
          W = 0.f;
          j = 0;
          active = true;
        }
      }
    }
    if (!__any_sync(0xffffffffu, active)) break;
    if (active) {
      const IndirectItem<MAXD>& it = q[k];
      const int D = it.D, jmax = it.jmax;
      bool alive = false;
      if (j <= jmax) {
        const PathSmp S{&P, V->seed, it.gslot, it.p + V->slot_off};
        const int o = 3 + 5 * j;
        F3 c;
        alive = radiance_step_k<TRN_SHARED_STEPS_INDIRECT>(s, xx, rd, T, S(o), S(o + 1), S(o + 2), S(o + 3),
                                                           S(o + 4), c, nullptr, cnt);
        cur = cur + c;
        if (T.x == 0.f && T.y == 0.f && T.z == 0.f) alive = false;
        W += dot(it.sc[D - 2 - j], cur) * it.w0;
        j++;
      }
      if (!alive || j > jmax) {
        // the path has ended: the remaining depths pair with the last radiance
        for (; j <= jmax; j++) W += dot(it.sc[D - 2 - j], cur) * it.w0;
        if (W != 0.f && isfinite(W)) {
          const SurfF xs = post_intersect(s, it.xs_tri, it.xs_u, it.xs_v);
          xdotn_vjp(P, *V, W, xs.p, true, it.xs_tri, it.xs_u, it.xs_v, it.v0, it.v1, it.sedge, it.p0, it.far_tri,
                    it.n, cnt);
        }
        active = false;
      }
    }
  }
  flush_cnt(cnt, P.stats);
}

// Slot range of one split round: the work counter starts at `first`, the
// queue is empty.
__global__ void k_indirect_round(unsigned long long* work, unsigned long long first, unsigned long long* q_count) {
  if (threadIdx.x == 0) { *work = first; q_count[0] = 0ull; q_count[1] = 0ull; q_count[2] = 0ull; q_count[3] = 0ull; }
}

// Sort keys of one round of a split boundary set-up: view x (E + 1) + the
// edge that the slot's edge sample picks (E when it picks none), value = the
// slot's offset in the round. Run in key order, a warp's rays leave one edge
// (or a few neighbours) instead of 32 random ones; each slot's own result is
// unchanged, only the order of the gradient atomics moves.
// The edge pick restates the set-up functions' first step: primary_setup
// (view silhouette table), direct_setup (scene table, or the AQ leaf when
// guided), indirect_setup (scene table).
// bits_r1 + bits_r2 > 0 (indirect term) appends a direction bin below the
// edge: the set-up rays of one edge leave one point, and sorting them by the
// two samples that pick their direction (Edge.cpp:152-195) puts rays that
// head the same way into one warp. r2 is the major part: it picks the
// quadrant and the angle along the edge (or the azimuth of a boundary edge);
// r1 sweeps the wedge between the face normals, which is narrow on a smooth
// mesh (or the polar angle of a boundary edge).
__global__ void k_edge_keys(TRN_KPARAMS, int term, int bits_r1, int bits_r2, unsigned* keys, unsigned* vals) {
  const long long first = P.order_first, n = P.total - first;
  int vhint = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long g = first + i;
    const ViewDesc& V = view_of(P, g, vhint);
    const PathSmp S{&P, V.seed, g, g - V.begin + V.slot_off};
    int e = P.ne;
    float reuse;
    if (term == TRN_PRIMARY_EDGE) {
      if (__ldg(V.pint) > 0.f) e = sample_discrete(V.pcdf, P.ne, S(0), reuse);
    } else if (__ldg(P.eint) > 0.f && (term != TRN_INDIRECT_EDGE || V.D >= 2)) {
      if (term == TRN_DIRECT_EDGE && P.aq_cdf)
        e = __ldg(P.aq_edge + sample_discrete(P.aq_cdf, __ldg(P.aq_n), S(3 + 3 * V.D), reuse));
      else
        e = sample_discrete(P.ecdf, P.ne, S(0), reuse);
    }
    unsigned key = (unsigned)(&V - P.views) * (unsigned)(P.ne + 1) + (unsigned)e;
    if (bits_r1 + bits_r2 > 0) {
      const unsigned b1 = min((unsigned)(S(1) * (float)(1 << bits_r1)), (1u << bits_r1) - 1u);
      const unsigned b2 = min((unsigned)(S(2) * (float)(1 << bits_r2)), (1u << bits_r2) - 1u);
      key = (key << (bits_r1 + bits_r2)) | (b2 << bits_r1) | b1;
    }
    keys[i] = key;
    vals[i] = (unsigned)i;
  }
}


#ifndef TRN_PIXEL_INTERLEAVE
#define TRN_PIXEL_INTERLEAVE 1
#endif

// ---------------------------------------------------------------------------
// pixel boundary (BoundaryPixel.cpp:36-159, Edge.cpp:377-409, Camera.cpp:433-467)
// ---------------------------------------------------------------------------
// Pixel boundary set-up (SampleBoundarySegmentPixel, Edge.cpp:377-409;
// GeneratePixelBoundarySamples, Camera.cpp:433-467): a point on the pixel's
// boundary from the antithetic copy's sample, the camera ray through it, the
// boundary geometry. Returns false for a rejected sample.
TRN_D bool pixel_setup(const Params& P, long long gslot, EdgeState& st, int& vhint, Cnt& cnt) {
  const DeviceScene& s = P.s;
  const ViewDesc& V = view_of(P, gslot, vhint);
  const CameraDesc& cam = V.cam;
  const int W_ = cam.w, WH = cam.w * cam.h;
  const F3 cpos = cam_pos(cam);
  const long long nanti = V.n / 4;
#if TRN_PIXEL_INTERLEAVE
  // Run order: the 4 antithetic copies of a slot take adjacent lanes. Their
  // camera rays leave one pixel's border and share every later sample, so
  // their paths stay close together (coherent traversal). Sample index p
  // (copy * nanti + slot) and everything derived from it are unchanged.
  const long long i = gslot - V.begin;
  const long long p = (i & 3) * nanti + (i >> 2);
#else
  const long long p = gslot - V.begin;
#endif
  const long long slot = p % nanti;
  const int anti = (int)(p / nanti);
  // the 4 antithetic copies of a slot share its samples (BoundaryPixel.cpp:135-138)
  const PathSmp S{&P, V.seed, V.begin / 4 + slot, slot + V.slot_off};
  const float r = S(0);
  float rr;
  if (anti == 0) rr = r;
  else if (anti == 1) rr = r < 0.5f ? r + 0.5f : r - 0.5f;
  else if (anti == 2) rr = r < 0.75f ? 0.75f - r : 1.75f - r;
  else rr = r < 0.25f ? 0.25f - r : 1.25f - r;
  const float r4 = rr * 4.f;
  const int bi = (int)floorf(r4);
  float ox, oy;
  if (bi == 0) { ox = 0.f; oy = r4; }
  else if (bi == 1) { ox = r4 - 1.f; oy = 1.f; }
  else if (bi == 2) { ox = 1.f; oy = 3.f - r4; }
  else { ox = 4.f - r4; oy = 0.f; }
  const int bsel = bi < 0 ? 0 : (bi > 3 ? 3 : bi);
  const float pdf = (bsel & 1) ? 0.25f / (cam.plane_len_x * (float)cam.h) : 0.25f / (cam.plane_len_y * (float)cam.w);
  const F3 dedge = (bsel & 1) ? F3(1.f, 0.f, 0.f) : F3(0.f, 1.f, 0.f);
  const F3 dvis = bsel == 0 ? F3(1.f, 0.f, 0.f) : (bsel == 1 ? F3(0.f, -1.f, 0.f)
                                                : (bsel == 2 ? F3(-1.f, 0.f, 0.f) : F3(0.f, 1.f, 0.f)));
  const F3 edge = normalize(xform_vector(cam.raster_to_world, dedge));
  const F3 edge2 = normalize(xform_vector(cam.raster_to_world, dvis));
  const int pixel = (int)(p % WH);
  const F3 p0 = xform_point(cam.raster_to_world, F3((float)(pixel % W_) + ox, (float)(pixel / W_) + oy, 0.f));
  const F3 dir = normalize(p0 - cpos);
  Hit h;
  cnt.v[kCntClosest]++;
  if (!trace_k<TRN_SETUP_SHARED_PIXEL, false>(s, p0, dir, kShadowEps, kRayMax, h, P.err)) return false;
  const F3 hitP = p0 + dir * h.t;
  const SensorSample sds = sample_direct(cam, hitP);
  const F3 dirc = sensor_ray_dir(cam, sds.qx, sds.qy);
  const SurfF x = post_intersect(s, h.tri, h.u, h.v);
  const float dist = length(x.p - cpos);
  const float dist1 = length(p0 - cpos);
  const float cos2 = fabsf(dot(x.ng, -dirc));
  F3 n;
  // BoundaryPixel.cpp:92 reverses the sign convention
  const float bval = -base_val(dist / dist1, edge, dirc, x.ng, edge2, n) * cos2;
  const F3 g = g_at(P, V, pixel);
  if (bval == 0.f || (g.x == 0.f && g.y == 0.f && g.z == 0.f)) return false;
  st.V = &V; st.gslot = V.begin / 4 + slot; st.p = slot; st.x = x; st.rdir = dirc;
  st.T0 = F3(sds.sensor_val, sds.sensor_val, sds.sensor_val);
  st.p0 = p0; st.n = n; st.w0 = bval / pdf; st.far_tri = h.tri; st.g = g;
  return true;
}

__global__ void __launch_bounds__(256, TRN_MINB) k_pixel_adj(TRN_KPARAMS) {
  Cnt cnt;
  stage_top(P.s);
  int vhint = 0;
  for_each_valid<EdgeState>(P,
    [&](long long gslot, EdgeState& st) -> bool { return pixel_setup(P, gslot, st, vhint, cnt); },
    [&](EdgeState& st) {
      // the pixel-edge point is not a scene parameter: only the hit triangle moves
      primary_body(P, *st.V, st.gslot, st.p, st.x, st.rdir, st.T0, st.w0, st.g, -1, -1, 0.f, st.p0, st.far_tri,
                   st.n, cnt, 1);
    });
  flush_cnt(cnt, P.stats);
}

// Split form: k_pixel_setup queues the accepted samples as PrimaryItem
// (dimension 1 onwards, no edge vertices); k_primary_body runs them.
__global__ void __launch_bounds__(256, TRN_MINB_SETUP) k_pixel_setup(TRN_KPARAMS) {
  Cnt cnt;
  stage_top(P.s);
  int vhint = 0;
  PrimaryItem* q = reinterpret_cast<PrimaryItem*>(P.queue);
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  for (;;) {
    unsigned long long start = 0;
    if (lane == 0) start = atomicAdd(P.work, 32ull);
    start = __shfl_sync(0xffffffffu, start, 0);
    if ((long long)start >= P.total) break;
    const long long g = (long long)start + lane;
    EdgeState st;
    const bool ok = g < P.total && pixel_setup(P, g, st, vhint, cnt);
    const unsigned m = __ballot_sync(0xffffffffu, ok);
    if (!m) continue;
    const int leader = __ffs(m) - 1;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(P.q_count, (unsigned long long)__popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    const unsigned long long k = base + __popc(m & lt);
    if (ok && k >= (unsigned long long)P.q_cap) atomicExch(P.err, 2);
    if (ok && k < (unsigned long long)P.q_cap) {
      PrimaryItem& it = q[k];
      it.gslot = st.gslot; it.p = st.p; it.view = (int)(st.V - P.views); it.dim0 = 1;
      it.x_tri = st.x.tri; it.x_u = st.x.u; it.x_v = st.x.v; it.T0 = st.T0.x; it.w0 = st.w0; it.sedge = 0.f;
      it.v0 = -1; it.v1 = -1; it.far_tri = st.far_tri;
      it.rdir = st.rdir; it.p0 = st.p0; it.n = st.n; it.g = st.g;
    }
  }
  flush_cnt(cnt, P.stats);
}

// ---------------------------------------------------------------------------
// primary edge list for one camera (ConstructPrimEdgeList, Edge.cpp:313-348)
// ---------------------------------------------------------------------------
__global__ void k_prim_edges_views(int ne, const int* edges, const float* pos, const float* fn,
                                   const ViewDesc* views, float* func_all) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int v = blockIdx.y;
  if (e >= ne) return;
  const CameraDesc& c = views[v].cam;
  const F3 cpos(c.pos[0], c.pos[1], c.pos[2]);
  const int v0 = edges[5 * e], v1 = edges[5 * e + 1], f0 = edges[5 * e + 2], f1 = edges[5 * e + 3];
  const F3 p0 = make_f3(pos + 3 * v0);
  const F3 ev = cpos - p0;
  const F3 n0 = make_f3(fn + 3 * f0);
  const F3 n1 = f1 >= 0 ? make_f3(fn + 3 * f1) : F3(0.f, 0.f, 0.f);
  const bool ff0 = dot(ev, n0) > 0.f, ff1 = dot(ev, n1) > 0.f;
  const bool valid = f1 < 0 || (ff0 != ff1);
  func_all[(long long)v * ne + e] = valid ? length(make_f3(pos + 3 * v1) - p0) : 0.f;
}

// Distribution1D::SetFunction for one block per view (prefix sums in double)
// Distribution1D::SetFunction over n weights by one block (see k_cdf).
TRN_D void cdf_block(int n, const float* func, float* cdf, float* integral_out) {
  __shared__ double part[1024];
  __shared__ float integral;
  const int T = blockDim.x, tid = threadIdx.x;
  const int chunk = (n + T - 1) / T;
  const int a = min(n, tid * chunk), b = min(n, a + chunk);
  double sacc = 0.0;
  for (int i = a; i < b; i++) sacc += (double)func[i];
  part[tid] = sacc;
  __syncthreads();
  if (tid == 0) { double run = 0.0; for (int i = 0; i < T; i++) { double x = part[i]; part[i] = run; run += x; } }
  __syncthreads();
  const float inv_size = 1.0f / (float)n;
  double run = part[tid];
  for (int i = a; i < b; i++) { run += (double)func[i]; cdf[i] = (float)run * inv_size; }
  __syncthreads();
  if (tid == 0) { integral = n > 0 ? cdf[n - 1] : 0.f; *integral_out = integral; }
  __syncthreads();
  if (integral > 0.f) for (int i = a; i < b; i++) cdf[i] = cdf[i] / integral;
}

// one distribution per block: view v's n weights at func_all + v n
__global__ void k_cdf_views(int n, const float* func_all, float* cdf_all, float* integral_all) {
  const int v = blockIdx.x;
  cdf_block(n, func_all + (long long)v * n, cdf_all + (long long)v * n, integral_all + v);
}

// one distribution whose length is in device memory (the guiding tree's leaves)
__global__ void k_cdf_count(const int* count, const float* func, float* cdf, float* integral) {
  cdf_block(__ldg(count), func, cdf, integral);
}

// 0.5 |I - T|^2 per view and dL/dI = I - T (pyTensorRay/loss.py:34-38)
__global__ void k_view_loss(long long npix, const ViewDesc* views, const long long* pbegin, int nviews,
                            const float* img, const float* tgt, float* dLdI, float* loss) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  float l = 0.f;
  int v = -1;
  if (i < npix) {
    int lo = 0, hi = nviews - 1;
    while (lo < hi) { const int mid = (lo + hi + 1) >> 1; if (pbegin[mid] <= i) lo = mid; else hi = mid - 1; }
    v = lo;
    for (int c = 0; c < 3; c++) {
      const float d = img[3 * i + c] - tgt[3 * i + c];
      if (dLdI) dLdI[3 * i + c] = d;
      l += 0.5f * d * d;
    }
  }
  // warp-aggregate per view
  const unsigned m = __match_any_sync(0xffffffffu, v);
  float sum = 0.f;
  for (int k = 0; k < 32; k++) {
    const float y = __shfl_sync(0xffffffffu, l, k);
    if (m & (1u << k)) sum += y;
  }
  if (v >= 0 && (int)(threadIdx.x & 31) == __ffs(m) - 1 && loss) atomicAdd(loss + v, sum);
}

__global__ void k_intersect(DeviceScene s, int n, const float* org, const float* dir, const float* tmin,
                            const float* tmax, int* tri, float* u, float* v, float* t, int* err) {
  stage_top(s);
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Hit h;
  trace<false>(s, make_f3(org + 3 * i), make_f3(dir + 3 * i), tmin[i], tmax[i], h, err);
  tri[i] = h.tri; u[i] = h.u; v[i] = h.v; t[i] = h.t;
}
__global__ void k_occluded(DeviceScene s, int n, const float* org, const float* dir, const float* tmin,
                           const float* tmax, int* vis) {
  stage_top(s);
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  vis[i] = occluded(s, make_f3(org + 3 * i), make_f3(dir + 3 * i), tmin[i], tmax[i]) ? 0 : 1;
}

}  // namespace trn

using namespace trn;

// Pinned staging slots of a view set's table uploads. An upload waits only
// for the upload this many before it to have left its slot, so a loop that
// changes its views every call (a serving loop) runs that many uploads ahead
// of the device instead of waiting for the previous call's kernels.
constexpr int kStageRing = 4;

// A set of camera views rendered by one launch per integrator: the device view
// table plus per-view silhouette-edge workspace.
struct trn_viewset {
  trn_scene* scene = nullptr;
  int nviews = 0;
  int cap = 0;                    // allocated view capacity
  // pinned staging of the view table: kStageRing slots of `cap` views and
  // 2 * `cap` offsets (view begins, then pixel begins) each
  ViewDesc* h_stage = nullptr;
  long long* h_stage_begin = nullptr;
  cudaEvent_t stage_done[kStageRing] = {};
  int stage_next = 0;
  bool pbegin_dirty = true;
  long long npix = 0;
  std::vector<trn_view> h_views;
  std::vector<long long> h_pbegin;
  ViewDesc* views = nullptr;      // device [nviews]
  long long* vbegin = nullptr;    // device [nviews], rewritten per integrator (spp differs)
  long long* pbegin = nullptr;    // device [nviews] first pixel of each view
  float* pfunc = nullptr;         // device [nviews][E]
  float* pcdf = nullptr;          // device [nviews][E]
  float* pint = nullptr;          // device [nviews]
  unsigned long long* work = nullptr;
  // queue of the split indirect boundary term: one round of at most
  // kIndirectRound slots at a time
  void* iq = nullptr;
  size_t iq_bytes = 0;
  unsigned long long* iq_count = nullptr;
  // run order of the split set-up rounds: keys and values double-buffered for
  // one round, then the radix sort's temporary storage
  void* sq = nullptr;
  long long sq_cap = 0;  // slots per round the order buffers hold
  size_t sq_tmp = 0;     // bytes of the sort's temporary storage
  // path cache: interior path records of the last forward render, reused by
  // the gradient call of the same paths (same scene version, views, seed and
  // depth; hash samples only)
  void* pc = nullptr;
  size_t pc_bytes = 0;
  unsigned long long* pc_count = nullptr;
  long long pc_limit = 0;  // bytes the records may take (0 = off)
  bool pc_valid = false;
  std::vector<char> pc_key;
  int ne = 0;
  // slot layout currently uploaded: spp multiplier and per-view spp
  int uploaded_key = -2;
  long long total = 0;
  // image / dL/dI base buffers of the uploaded table (views without their own)
  int cur_depth = -1;
  int max_depth = kMaxDepth;
};

namespace {

int sms() {
  int dev = 0, n = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n;
}

int check_common(trn_scene* s, const trn_render_options* o, int integrator) {
  if (!s || !o) { set_error("null argument"); return -1; }
  if (!s->configured) { set_error("scene is not configured (call trn_scene_configure)"); return -1; }
  if (integrator < 0 || integrator > 4) { set_error("unknown integrator id"); return -1; }
  if (o->max_bounces < 0 || o->max_bounces > kMaxDepth) { set_error("max_bounces must be in [0, 16]"); return -1; }
  return 0;
}

int spp_of(const trn_render_options* o, int integrator) {
  switch (integrator) {
    case TRN_PATH_TRACER: return o->spp;
    case TRN_PRIMARY_EDGE: return o->sppe;
    case TRN_DIRECT_EDGE: return o->sppse0;
    case TRN_INDIRECT_EDGE: return o->sppse1;
    default: return o->sppe0;
  }
}

// Upload the view table for one integrator: per-view spp comes from the view
// (spp_override < 0) or from the options (single-view calls).
// The next staging slot, once the upload that last used it has left it.
int next_stage(trn_viewset* vs) {
  const int k = vs->stage_next;
  vs->stage_next = (k + 1) % kStageRing;
  if (vs->stage_done[k]) cudaEventSynchronize(vs->stage_done[k]);
  return k;
}

// Every staging slot free (before the staging is freed or reallocated).
void wait_stages(trn_viewset* vs) {
  for (cudaEvent_t e : vs->stage_done)
    if (e) cudaEventSynchronize(e);
}

int upload_views(trn_viewset* vs, const trn_render_options* o, int integrator, int spp_override, long long& total,
                 cudaStream_t st) {
  (void)o;
  float* s_gpos = vs->scene->g_pos;
  float* s_gvn = vs->scene->g_vnormal;
  float* s_gtex = vs->scene->g_texels;
  const int key = spp_override;  // the layout depends on the per-view spp, buffers and depth
  if (vs->uploaded_key == key && key != -2 && vs->cur_depth == o->max_bounces) {
    total = vs->total;
    if (integrator == TRN_PIXEL_EDGE)
      for (int v = 0; v < vs->nviews; v++) {
        const int spp = spp_override >= 0 ? spp_override : vs->h_views[v].spp;
        if (((long long)vs->h_views[v].camera.width * vs->h_views[v].camera.height * spp) % 4 != 0) {
          set_error("pixel boundary needs W*H*spp divisible by 4");
          return -1;
        }
      }
    return 0;
  }
  vs->cur_depth = o->max_bounces;
  vs->max_depth = 0;
  for (int v = 0; v < vs->nviews; v++)
    vs->max_depth = std::max(vs->max_depth, vs->h_views[v].max_bounces > 0 ? vs->h_views[v].max_bounces
                                                                            : o->max_bounces);
  const int slot = next_stage(vs);
  ViewDesc* d = vs->h_stage + (size_t)slot * vs->cap;
  long long* begin = vs->h_stage_begin + (size_t)slot * 2 * vs->cap;
  total = 0;
  for (int v = 0; v < vs->nviews; v++) {
    const trn_view& hv = vs->h_views[v];
    const int spp = spp_override >= 0 ? spp_override : hv.spp;
    if (spp < 0) { set_error("negative spp"); return -1; }
    std::memcpy(&d[v].cam, &hv.camera, sizeof(CameraDesc));
    d[v].begin = total;
    d[v].n = (long long)hv.camera.width * hv.camera.height * spp;
    if (integrator == TRN_PIXEL_EDGE && (d[v].n % 4) != 0) {
      set_error("pixel boundary needs W*H*spp divisible by 4");
      return -1;
    }
    d[v].pix_off = vs->h_pbegin[v];
    d[v].inv_spp = hv.weight > 0.f ? hv.weight : (spp > 0 ? 1.0f / (float)spp : 0.f);
    d[v].slot_off = hv.slot_offset;
    d[v].D = hv.max_bounces > 0 ? std::min(hv.max_bounces, (int)kMaxDepth) : o->max_bounces;
    d[v].image = hv.image;
    d[v].dLdI = hv.dLdI;
    d[v].gpos = hv.grad_positions ? hv.grad_positions : s_gpos;
    d[v].gvn = hv.grad_vertex_normals ? hv.grad_vertex_normals : s_gvn;
    d[v].gtex = hv.grad_texels ? hv.grad_texels : s_gtex;
    d[v].seed = (uint32_t)hv.seed;  // independent of the view's position in the set
    d[v].spp = spp;
    d[v].pad_ = 0;
    d[v].pfunc = vs->pfunc ? vs->pfunc + (long long)v * vs->ne : nullptr;
    d[v].pcdf = vs->pcdf ? vs->pcdf + (long long)v * vs->ne : nullptr;
    d[v].pint = vs->pint ? vs->pint + v : nullptr;
    begin[v] = total;
    total += d[v].n;
  }
  TRN_CUDA_TRY(cudaMemcpyAsync(vs->views, d, sizeof(ViewDesc) * vs->nviews, cudaMemcpyHostToDevice, st));
  TRN_CUDA_TRY(cudaMemcpyAsync(vs->vbegin, begin, sizeof(long long) * vs->nviews, cudaMemcpyHostToDevice, st));
  TRN_CUDA_TRY(cudaEventRecord(vs->stage_done[slot], st));
  vs->uploaded_key = key;
  vs->total = total;
  return 0;
}

Params base_params(trn_scene* s, trn_viewset* vs, const trn_render_options* o, int integrator,
                   const trn_samples* smp, const trn_launch* ln, long long total) {
  Params P;
  P.s = s->view();
  P.views = vs->views;
  P.vbegin = vs->vbegin;
  P.nviews = vs->nviews;
  P.total = total;
  P.work = vs->work;
  P.chunk = (ln && ln->chunk > 0) ? ln->chunk : 1;
  P.table = smp ? smp->samples : nullptr;
  P.stride = smp && smp->samples ? smp->stride : 0;
  P.term = (uint32_t)integrator;
  P.seed = (uint32_t)o->seed;
  P.D = o->max_bounces;
  P.g_pos = s->g_pos; P.g_vn = s->g_vnormal; P.g_tex = s->g_texels; P.diff_tex = s->ntexel > 0;
  P.edges = s->edges; P.ecdf = s->sec_cdf; P.efunc = s->sec_func; P.eint = s->sec_integral_dev; P.ne = s->ne;
  P.err = s->err;
  P.stats = s->stats_on ? s->stats : nullptr;
  P.aq_poly = P.aq_cdf = P.aq_int = nullptr;
  P.aq_box = nullptr;
  P.aq_edge = P.aq_n = nullptr;
  P.aq_cap = 0;
  P.queue = nullptr;
  P.queue2 = nullptr;
  P.q_count = nullptr;
  P.q_cap = 0;
  P.order = nullptr;
  P.order_first = 0;
  return P;
}

// Grow the guiding tree's arrays to `cap` leaves (the first refining call, or
// a larger g_direct_max_size); the depth-0 arrays are allocated with the scene.
int aq_reserve(trn_scene* s, long long cap) {
  if (cap <= s->aq_cap && s->aq_eval) return 0;
  cap = std::max(cap, s->aq_cap);
  float* f[4] = {nullptr, nullptr, nullptr, nullptr};
  int* i3[3] = {nullptr, nullptr, nullptr};
  float* eval = nullptr;
  const size_t n = (size_t)cap;
  bool ok = cudaMalloc(&f[0], n * sizeof(float)) == cudaSuccess && cudaMalloc(&f[1], n * sizeof(float)) == cudaSuccess &&
            cudaMalloc(&f[2], n * sizeof(float)) == cudaSuccess && cudaMalloc(&f[3], 6 * n * sizeof(float)) == cudaSuccess &&
            cudaMalloc(&i3[0], n * sizeof(int)) == cudaSuccess && cudaMalloc(&i3[1], n * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&i3[2], n * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&eval, (size_t)kAqPoints * n * sizeof(float)) == cudaSuccess;
  if (!ok) {
    for (float* p : f) if (p) cudaFree(p);
    for (int* p : i3) if (p) cudaFree(p);
    if (eval) cudaFree(eval);
    cudaGetLastError();
    set_error("guiding: cannot allocate the refined tree (g_direct_max_size leaves)");
    return -1;
  }
  void* old[] = {s->aq_poly, s->aq_func, s->aq_cdf, s->aq_box, s->aq_edge, s->aq_flag, s->aq_prefix, s->aq_eval};
  for (void* p : old) if (p) cudaFree(p);
  s->aq_poly = f[0]; s->aq_func = f[1]; s->aq_cdf = f[2]; s->aq_box = f[3];
  s->aq_edge = i3[0]; s->aq_flag = i3[1]; s->aq_prefix = i3[2]; s->aq_eval = eval;
  s->aq_cap = cap;
  return 0;
}

// AdaptiveQuadratureDistribution::setup (AQ_distrb.h:83-173) for one
// direct-boundary call: the depth-0 tree, g_direct_depth refinement passes
// (the loop the reference keeps commented out, AQ_distrb.h:121-136, with
// gen_eval_point and cut_tree of NEE.cu:91-396), leaf weights from
// g_direct_spp samples per leaf, eps mixing, leaf distribution. The tree
// holds at most max(E, g_direct_max_size) leaves. The set-up samples come
// from the counter hash (their own terms), also when the call's samples come
// from a table. may_alloc = false (the allocation-free entry point) refuses
// a refinement that would need larger arrays than the scene holds.
int guide_setup(trn_scene* s, const trn_render_options* o, Params& P, cudaStream_t st, bool may_alloc = true) {
  if (!o->g_direct || s->ne == 0) return 0;
  if (o->g_direct_spp <= 0) { set_error("g_direct_spp must be positive when g_direct is set"); return -1; }
  if (!(o->g_eps >= 0.f && o->g_eps <= 1.f)) { set_error("g_eps must be in [0, 1]"); return -1; }
  if (o->g_direct_depth < 0) { set_error("g_direct_depth must be >= 0"); return -1; }
  const int depth = o->g_direct_depth;
  const long long limit = depth > 0 ? std::max<long long>(s->ne, o->g_direct_max_size) : s->ne;
  if (limit > 0x7FFFFFFFLL / kAqPoints) { set_error("guiding: g_direct_max_size is too large"); return -1; }
  if (limit * o->g_direct_spp > 0xFFFFFFFFLL) {
    set_error("guiding: leaves x g_direct_spp exceeds 2^32 set-up samples");
    return -1;
  }
  if (depth > 0) {
    if (!(o->g_direct_thold >= 0.f)) { set_error("g_direct_thold must be >= 0"); return -1; }
    if ((limit > s->aq_cap || !s->aq_eval) && !may_alloc) {
      set_error("refining the guiding tree (g_direct_depth > 0) allocates its arrays on first use; call "
                "trn_render_grad once with the same options first");
      return -1;
    }
    if (aq_reserve(s, limit)) return -1;
  }
  Params G = P;
  G.table = nullptr;
  G.stats = nullptr;
  const long long cap = s->aq_cap;
  const uint32_t stream = (uint32_t)o->seed * 1000003u;
  k_aq_init<<<(s->ne + 255) / 256, 256, 0, st>>>(s->ne, s->sec_cdf, s->aq_box, s->aq_edge, s->aq_count, cap);
  int launches = 1;
  for (int pass = 0; pass < depth; pass++) {
    const uint32_t ps = stream + (uint32_t)pass;
    k_aq_eval<<<(unsigned)((limit * kAqPoints + 255) / 256), 256, 0, st>>>(G, ps, s->aq_box, s->aq_edge, s->aq_count,
                                                                           cap, s->aq_eval);
    k_aq_flag<<<(unsigned)((limit + 255) / 256), 256, 0, st>>>(s->aq_box, s->aq_count, cap, s->aq_eval,
                                                               o->g_direct_thold, ps, s->aq_flag);
    k_aq_scan<<<1, 1024, 0, st>>>(s->aq_count, s->aq_flag, s->aq_prefix, s->aq_count, (int)limit);
    k_aq_split<<<(unsigned)((limit + 255) / 256), 256, 0, st>>>(s->aq_count, s->aq_flag, s->aq_prefix, s->aq_box,
                                                                s->aq_edge, cap);
    k_aq_commit<<<1, 1, 0, st>>>(s->aq_count);
    launches += 5;
  }
  k_aq_poly<<<(unsigned)((limit + 255) / 256), 256, 0, st>>>(G, stream, o->g_direct_spp, s->aq_box, s->aq_edge,
                                                              s->aq_count, cap, s->aq_poly);
  k_aq_mix<<<1, 1024, 0, st>>>(s->aq_count, s->aq_poly, s->aq_box, cap, o->g_eps, s->aq_func, s->aq_int);
  k_cdf_count<<<1, 1024, 0, st>>>(s->aq_count, s->aq_func, s->aq_cdf, s->aq_int);
  count_launch(launches + 3);
  TRN_CUDA_TRY(cudaGetLastError());
  P.aq_poly = s->aq_poly;
  P.aq_cdf = s->aq_cdf;
  P.aq_int = s->aq_int;
  P.aq_box = s->aq_box;
  P.aq_edge = s->aq_edge;
  P.aq_n = s->aq_count;
  P.aq_cap = cap;
  return 0;
}

void launch_dims(const trn_launch* ln, long long total, int& grid, int& block) {
  block = (ln && ln->block > 0) ? ln->block : 128;
  const int per_sm = (ln && ln->blocks_per_sm > 0) ? ln->blocks_per_sm : 1024 / block;
  const long long chunk = (ln && ln->chunk > 0) ? ln->chunk : 1;
  long long want = (long long)sms() * per_sm;
  const long long need = (total + 32 * chunk - 1) / (32 * chunk) * 32 / block + 1;
  grid = (int)std::max<long long>(1, std::min(want, need));
}

int validate_launch(const trn_launch* ln) {
  if (!ln) return 0;
  if (ln->block != 0 && (ln->block < 32 || ln->block > 256 || ln->block % 32 != 0)) {
    set_error("launch block must be a multiple of 32 in [32, 256]");
    return -1;
  }
  if (ln->blocks_per_sm < 0 || ln->blocks_per_sm > 64 || ln->chunk < 0 || ln->chunk > 64) {
    set_error("launch blocks_per_sm must be in [0, 64] and chunk in [0, 64]");
    return -1;
  }
  if (ln->round_log2 != 0 && (ln->round_log2 < 16 || ln->round_log2 > 40)) {
    set_error("launch round_log2 must be 0 (default) or in [16, 40]");
    return -1;
  }
  return 0;
}

template <class K>
void launch(K kernel, const trn_launch* ln, long long total, const Params& P, cudaStream_t st) {
  int grid, block;
  launch_dims(ln, total, grid, block);
  kernel<<<grid, block, 0, st>>>(P);
  count_launch(1);
}

#ifndef TRN_INDIRECT_SPLIT
#define TRN_INDIRECT_SPLIT 1
#endif
// slots per round of the split boundary terms: 16M (one round for a 512² x
// 64 spp term). Larger rounds give each edge more samples per sort and the
// terms fewer kernel tails (measured: 4M 195.6, 8M 189.5, 16M 186.2 ms/step
// on that workload), at about 5.5 GB of queue per view set.
#ifndef TRN_ROUND_LOG2
#define TRN_ROUND_LOG2 24
#endif
constexpr long long kIndirectRound = 1LL << TRN_ROUND_LOG2;
constexpr long long kPathRound = 1LL << 21;  // paths per split round of the interior adjoint

// Slots (or paths) per round: the launch's round_log2 when set, never above
// the default that the queues are sized for.
long long round_cap(const trn_launch* ln, long long dflt) {
  if (ln && ln->round_log2 > 0) return std::min(dflt, 1LL << ln->round_log2);
  return dflt;
}

// Largest queue that any split term needs for one full round (depth <= 8
// when shallow, else up to kMaxDepth).
size_t full_queue_bytes(bool shallow) {
  const size_t c = (size_t)kIndirectRound;
  const size_t ind = (sizeof(IndirectSetupItem) * c + 255) / 256 * 256 +
                     (shallow ? sizeof(IndirectItem<8>) : sizeof(IndirectItem<kMaxDepth>)) * c;
  const size_t path = shallow ? path_soa_bytes<8>(kPathRound) : path_soa_bytes<kMaxDepth>(kPathRound);
  return std::max(std::max(ind, path), std::max(sizeof(PrimaryItem) * c, sizeof(DirectItem) * c));
}

#ifndef TRN_PRIMARY_SPLIT
#define TRN_PRIMARY_SPLIT 1
#endif

// The view set's queue of the split terms, grown on first use to at least
// `need` bytes (not inside stream capture: run the integrator once before
// capturing it, or reserve with trn_viewset_reserve). A growth at least
// doubles the queue, up to one full round, so that a set whose batches grow
// (a serving loop) reallocates a few times at most.
int ensure_queue(trn_viewset* vs, size_t need, cudaStream_t st) {
  if (vs->iq_bytes >= need && vs->iq_count) return 0;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  TRN_CUDA_TRY(cudaStreamIsCapturing(st, &cs));
  if (cs != cudaStreamCaptureStatusNone) {
    set_error("boundary term: its queue must be allocated before stream capture (run it once first)");
    return -1;
  }
  TRN_CUDA_TRY(cudaStreamSynchronize(st));
  if (vs->iq_bytes < need) {
    const size_t bytes = std::max(need, std::min(2 * vs->iq_bytes, full_queue_bytes(vs->max_depth <= 8)));
    if (vs->iq) cudaFree(vs->iq);
    vs->iq = nullptr;
    vs->iq_bytes = 0;
    if (cudaMalloc(&vs->iq, bytes) != cudaSuccess) { set_error("boundary term: out of memory for its queue"); return -1; }
    vs->iq_bytes = bytes;
  }
  if (!vs->iq_count && cudaMalloc(&vs->iq_count, 4 * sizeof(unsigned long long)) != cudaSuccess) {
    set_error("boundary term: out of memory");
    return -1;
  }
  return 0;
}

#ifndef TRN_PATHADJ_SPLIT
#define TRN_PATHADJ_SPLIT 1
#endif

// The split interior adjoint in rounds of at most kPathRound paths (a queue
// of about 1.3 GB at depth <= 8).
int path_adj_split(trn_viewset* vs, Params P, const trn_launch* ln, long long total, bool shallow, cudaStream_t st) {
  const long long cap = std::min(total, round_cap(ln, kPathRound));
  if (ensure_queue(vs, shallow ? path_soa_bytes<8>(cap) : path_soa_bytes<kMaxDepth>(cap), st)) return -1;
  P.queue = vs->iq;
  P.q_count = vs->iq_count;
  P.q_cap = cap;
  int grid, block;
  launch_dims(ln, cap, grid, block);
  for (long long first = 0; first < total; first += cap) {
    P.total = std::min(total, first + cap);
    k_indirect_round<<<1, 32, 0, st>>>(P.work, (unsigned long long)first, P.q_count);
    if (shallow) {
      k_path_replay<8><<<grid, block, 0, st>>>(P);
      k_path_reverse<8><<<grid, block, 0, st>>>(P);
    } else {
      k_path_replay<kMaxDepth><<<grid, block, 0, st>>>(P);
      k_path_reverse<kMaxDepth><<<grid, block, 0, st>>>(P);
    }
    count_launch(3);
  }
  TRN_CUDA_TRY(cudaGetLastError());
  return 0;
}

#ifndef TRN_PIXEL_SPLIT
#define TRN_PIXEL_SPLIT 1
#endif

// The split pixel boundary term in rounds of at most kIndirectRound samples.
int pixel_split(trn_viewset* vs, Params P, const trn_launch* ln, long long total, cudaStream_t st) {
  const long long cap = std::min(total, round_cap(ln, kIndirectRound));
  if (ensure_queue(vs, sizeof(PrimaryItem) * (size_t)cap, st)) return -1;
  P.queue = vs->iq;
  P.q_count = vs->iq_count;
  P.q_cap = cap;
  int grid, block;
  launch_dims(ln, cap, grid, block);
  for (long long first = 0; first < total; first += cap) {
    P.total = std::min(total, first + cap);
    k_indirect_round<<<1, 32, 0, st>>>(P.work, (unsigned long long)first, P.q_count);
    k_pixel_setup<<<grid, block, 0, st>>>(P);
    if (TRN_BODY_REGEN) k_primary_body_regen<<<grid, block, 0, st>>>(P);
    else k_primary_body<<<grid, block, 0, st>>>(P);
    count_launch(3);
  }
  TRN_CUDA_TRY(cudaGetLastError());
  return 0;
}

#ifndef TRN_DIRECT_SPLIT
#define TRN_DIRECT_SPLIT 1
#endif

#ifndef TRN_EDGE_ORDER
#define TRN_EDGE_ORDER 1
#endif

// Direction bins per edge in the indirect term's run order: bits of the sort
// key below the edge index taken from the samples r1 and r2 (0 and 0 sort by
// edge alone).
#ifndef TRN_INDIRECT_DIR_R1_BITS
#define TRN_INDIRECT_DIR_R1_BITS 2
#endif
#ifndef TRN_INDIRECT_DIR_R2_BITS
#define TRN_INDIRECT_DIR_R2_BITS 6
#endif

// Buffers of the edge-sorted run order for rounds of up to `cap` slots: keys
// and values double-buffered (16 bytes per slot) plus the radix sort's
// temporary storage for vs->sq_cap slots. Grown like the queue (at least
// doubling, up to one full round; not inside stream capture).
int alloc_order(trn_viewset* vs, long long cap, cudaStream_t st) {
  if (vs->sq && vs->sq_cap >= cap) return 0;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  TRN_CUDA_TRY(cudaStreamIsCapturing(st, &cs));
  if (cs != cudaStreamCaptureStatusNone) {
    set_error("boundary term: its sort buffers must be allocated before stream capture (run it once first)");
    return -1;
  }
  const long long n = std::max(cap, std::min(2 * vs->sq_cap, kIndirectRound));
  cub::DoubleBuffer<unsigned> k(nullptr, nullptr), v(nullptr, nullptr);
  size_t tmp = 0;
  TRN_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tmp, k, v, (int)n, 0, 32, st));
  TRN_CUDA_TRY(cudaStreamSynchronize(st));
  if (vs->sq) cudaFree(vs->sq);
  vs->sq = nullptr;
  vs->sq_cap = 0;
  if (cudaMalloc(&vs->sq, (16 * (size_t)n + 255) / 256 * 256 + tmp) != cudaSuccess) {
    set_error("boundary term: out of memory for its sort buffers");
    return -1;
  }
  vs->sq_cap = n;
  vs->sq_tmp = tmp;
  return 0;
}

// Order buffers for this launch's rounds; returns 1 (run in slot order) when
// the keys of this view set do not fit 32 bits.
int ensure_order(trn_viewset* vs, const Params& P, long long cap, cudaStream_t st) {
  if ((unsigned long long)P.nviews * (unsigned long long)(P.ne + 1) > 0xffffffffull) return 1;
  return alloc_order(vs, cap, st);
}

// Edge-sorted run order of the round [P.order_first, P.total): keys, then a
// stable radix sort over the bits the keys use; sets P.order.
int order_round(trn_viewset* vs, Params& P, int term, cudaStream_t st) {
  const long long n = P.total - P.order_first, cap = vs->sq_cap;
  unsigned* base = static_cast<unsigned*>(vs->sq);
  cub::DoubleBuffer<unsigned> k(base, base + cap), v(base + 2 * cap, base + 3 * cap);
  P.order = nullptr;
  const int grid = (int)std::min<long long>((n + 255) / 256, 16LL * sms());
  unsigned long long keys = (unsigned long long)P.nviews * (unsigned long long)(P.ne + 1);
  // direction bits of the indirect term, r2's given up last, as many as fit
  // the 32-bit key
  int bits_r1 = term == TRN_INDIRECT_EDGE ? TRN_INDIRECT_DIR_R1_BITS : 0;
  int bits_r2 = term == TRN_INDIRECT_EDGE ? TRN_INDIRECT_DIR_R2_BITS : 0;
  while (bits_r1 > 0 && (keys << (bits_r1 + bits_r2)) > 0x100000000ull) bits_r1--;
  while (bits_r2 > 0 && (keys << bits_r2) > 0x100000000ull) bits_r2--;
  keys <<= bits_r1 + bits_r2;
  k_edge_keys<<<grid, 256, 0, st>>>(P, term, bits_r1, bits_r2, k.Current(), v.Current());
  count_launch(1);
  int bits = 1;
  while (bits < 32 && (1ull << bits) < keys) bits++;
  void* tmp = reinterpret_cast<char*>(vs->sq) + (16 * (size_t)cap + 255) / 256 * 256;
  size_t tb = vs->sq_tmp;
  TRN_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, tb, k, v, (int)n, 0, bits, st));
  P.order = v.Current();
  return 0;
}

// The split direct term in rounds of at most kIndirectRound slots.
int direct_split(trn_viewset* vs, Params P, const trn_launch* ln, long long total, cudaStream_t st) {
  const long long cap = std::min(total, round_cap(ln, kIndirectRound));
  if (ensure_queue(vs, sizeof(DirectItem) * (size_t)cap, st)) return -1;
  P.queue = vs->iq;
  P.q_count = vs->iq_count;
  P.q_cap = cap;
  int grid, block;
  launch_dims(ln, cap, grid, block);
  const int ordered = TRN_EDGE_ORDER ? ensure_order(vs, P, cap, st) : 1;
  if (ordered < 0) return -1;
  for (long long first = 0; first < total; first += cap) {
    P.total = std::min(total, first + cap);
    P.order_first = first;
    if (!ordered && order_round(vs, P, TRN_DIRECT_EDGE, st)) return -1;
    k_indirect_round<<<1, 32, 0, st>>>(P.work, (unsigned long long)first, P.q_count);
    k_direct_setup<<<grid, block, 0, st>>>(P);
    k_direct_body<<<grid, block, 0, st>>>(P);
    count_launch(3);
  }
  TRN_CUDA_TRY(cudaGetLastError());
  return 0;
}

// The split primary term in rounds of at most kIndirectRound slots.
int primary_split(trn_viewset* vs, Params P, const trn_launch* ln, long long total, cudaStream_t st) {
  const long long cap = std::min(total, round_cap(ln, kIndirectRound));
  if (ensure_queue(vs, sizeof(PrimaryItem) * (size_t)cap, st)) return -1;
  P.queue = vs->iq;
  P.q_count = vs->iq_count;
  P.q_cap = cap;
  int grid, block;
  launch_dims(ln, cap, grid, block);
  const int ordered = TRN_EDGE_ORDER ? ensure_order(vs, P, cap, st) : 1;
  if (ordered < 0) return -1;
  for (long long first = 0; first < total; first += cap) {
    P.total = std::min(total, first + cap);
    P.order_first = first;
    if (!ordered && order_round(vs, P, TRN_PRIMARY_EDGE, st)) return -1;
    k_indirect_round<<<1, 32, 0, st>>>(P.work, (unsigned long long)first, P.q_count);
    k_primary_setup<<<grid, block, 0, st>>>(P);
    if (TRN_BODY_REGEN) k_primary_body_regen<<<grid, block, 0, st>>>(P);
    else k_primary_body<<<grid, block, 0, st>>>(P);
    count_launch(3);
  }
  TRN_CUDA_TRY(cudaGetLastError());
  return 0;
}

#ifndef TRN_INDIRECT_STAGES
#define TRN_INDIRECT_STAGES 3
#endif

// The split indirect term in rounds of at most kIndirectRound slots: two
// stages (set-up + sensor side, emitter side) or three (set-up, sensor side,
// emitter side; the default).
int indirect_split(trn_viewset* vs, Params P, const trn_launch* ln, long long total, bool shallow, cudaStream_t st) {
  const long long cap = std::min(total, round_cap(ln, kIndirectRound));
  const size_t item = shallow ? sizeof(IndirectItem<8>) : sizeof(IndirectItem<kMaxDepth>);
  const size_t item_a = TRN_INDIRECT_STAGES == 3 ? sizeof(IndirectSetupItem) : 0;
  const size_t bytes_a = (item_a * (size_t)cap + 255) / 256 * 256;
  if (ensure_queue(vs, bytes_a + item * (size_t)cap, st)) return -1;
  P.queue = vs->iq;
  P.queue2 = TRN_INDIRECT_STAGES == 3 ? static_cast<char*>(vs->iq) + bytes_a : nullptr;
  P.q_count = vs->iq_count;
  P.q_cap = cap;
  int grid, block;
  launch_dims(ln, cap, grid, block);
  const int ordered = TRN_EDGE_ORDER && TRN_INDIRECT_STAGES == 3 ? ensure_order(vs, P, cap, st) : 1;
  if (ordered < 0) return -1;
  for (long long first = 0; first < total; first += cap) {
    P.total = std::min(total, first + cap);
    P.order_first = first;
    if (!ordered && order_round(vs, P, TRN_INDIRECT_EDGE, st)) return -1;
    k_indirect_round<<<1, 32, 0, st>>>(P.work, (unsigned long long)first, P.q_count);
    if (TRN_INDIRECT_STAGES == 3) {
      k_indirect_setup<<<grid, block, 0, st>>>(P);
      if (shallow) {
        if (TRN_SENSOR_REGEN) k_indirect_sensor_regen<8><<<grid, block, 0, st>>>(P);
        else k_indirect_sensor_q<8><<<grid, block, 0, st>>>(P);
        if (TRN_EMITTER_REGEN) k_indirect_emitter_regen<8><<<grid, block, 0, st>>>(P);
        else k_indirect_emitter<8><<<grid, block, 0, st>>>(P);
      } else {
        if (TRN_SENSOR_REGEN) k_indirect_sensor_regen<kMaxDepth><<<grid, block, 0, st>>>(P);
        else k_indirect_sensor_q<kMaxDepth><<<grid, block, 0, st>>>(P);
        if (TRN_EMITTER_REGEN) k_indirect_emitter_regen<kMaxDepth><<<grid, block, 0, st>>>(P);
        else k_indirect_emitter<kMaxDepth><<<grid, block, 0, st>>>(P);
      }
      count_launch(4);
    } else {
      if (shallow) {
        k_indirect_sensor<8><<<grid, block, 0, st>>>(P);
        k_indirect_emitter<8><<<grid, block, 0, st>>>(P);
      } else {
        k_indirect_sensor<kMaxDepth><<<grid, block, 0, st>>>(P);
        k_indirect_emitter<kMaxDepth><<<grid, block, 0, st>>>(P);
      }
      count_launch(3);
    }
  }
  TRN_CUDA_TRY(cudaGetLastError());
  return 0;
}

#ifndef TRN_PATH_CACHE
#define TRN_PATH_CACHE 1
#endif

// What the interior paths of a launch depend on: the scene version, seed,
// depth, slot count and, per view, camera, spp, seed, slot offset and depth.
// (Weights, pixel offsets and buffers only enter the image write and dL/dI.)
std::vector<char> path_key(const trn_viewset* vs, const trn_render_options* o, int spp_override, long long total) {
  std::vector<char> k;
  auto put = [&](const void* p, size_t n) {
    const char* c = static_cast<const char*>(p);
    k.insert(k.end(), c, c + n);
  };
  put(&vs->scene->version, sizeof(vs->scene->version));
  put(&o->seed, sizeof(o->seed));
  put(&o->max_bounces, sizeof(o->max_bounces));
  put(&spp_override, sizeof(spp_override));
  put(&total, sizeof(total));
  for (const trn_view& v : vs->h_views) {
    put(&v.camera, sizeof(v.camera));
    put(&v.spp, sizeof(v.spp));
    put(&v.seed, sizeof(v.seed));
    put(&v.slot_offset, sizeof(v.slot_offset));
    put(&v.max_bounces, sizeof(v.max_bounces));
  }
  return k;
}

bool capturing(cudaStream_t st) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  return cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone;
}

// Recording forward render of the interior term into the view set's path
// cache. Returns 1 when the cache is not used (off, a sample table, stream
// capture, above the limit, or no memory for it): the caller then renders
// with k_path_fwd.
int path_cache_fwd(trn_viewset* vs, Params P, const trn_launch* ln, const trn_render_options* o, int spp_override,
                   long long total, cudaStream_t st) {
  vs->pc_valid = false;
  if (!TRN_PATH_CACHE || vs->pc_limit <= 0 || P.table || capturing(st)) return 1;
  const bool shallow = vs->max_depth <= 8;
  const size_t bytes = shallow ? path_soa_bytes<8>(total) : path_soa_bytes<kMaxDepth>(total);
  if (bytes > (size_t)vs->pc_limit) return 1;
  if (vs->pc_bytes < bytes || !vs->pc_count) {
    TRN_CUDA_TRY(cudaStreamSynchronize(st));
    if (vs->pc) cudaFree(vs->pc);
    vs->pc = nullptr;
    vs->pc_bytes = 0;
    if (cudaMalloc(&vs->pc, bytes) != cudaSuccess ||
        (!vs->pc_count && cudaMalloc(&vs->pc_count, sizeof(unsigned long long)) != cudaSuccess)) {
      cudaGetLastError();  // out of memory: render without records
      if (vs->pc) cudaFree(vs->pc);
      vs->pc = nullptr;
      return 1;
    }
    vs->pc_bytes = bytes;
  }
  TRN_CUDA_TRY(cudaMemsetAsync(vs->pc_count, 0, sizeof(unsigned long long), st));
  P.queue = vs->pc;
  P.q_count = vs->pc_count;
  P.q_cap = total;
  if (TRN_FWD_REGEN) {
    if (shallow) launch(k_path_fwd_rec_regen<8>, ln, total, P, st);
    else launch(k_path_fwd_rec_regen<kMaxDepth>, ln, total, P, st);
  } else {
    if (shallow) launch(k_path_fwd_rec<8>, ln, total, P, st); else launch(k_path_fwd_rec<kMaxDepth>, ln, total, P, st);
  }
  TRN_CUDA_TRY(cudaGetLastError());
  vs->pc_key = path_key(vs, o, spp_override, total);
  vs->pc_valid = true;
  return 0;
}

// Reverse sweep over the cached records when they are the paths of this
// gradient call. Returns 1 when they are not (the caller replays).
int path_cache_grad(trn_viewset* vs, Params P, const trn_launch* ln, const trn_render_options* o, int spp_override,
                    long long total, cudaStream_t st) {
  if (!vs->pc_valid || P.table || capturing(st)) return 1;
  if (vs->pc_key != path_key(vs, o, spp_override, total)) return 1;
  P.queue = vs->pc;
  P.q_count = vs->pc_count;
  P.q_cap = total;
  int grid, block;
  launch_dims(ln, total, grid, block);
  if (vs->max_depth <= 8) k_path_reverse<8, true><<<grid, block, 0, st>>>(P);
  else k_path_reverse<kMaxDepth, true><<<grid, block, 0, st>>>(P);
  count_launch(1);
  TRN_CUDA_TRY(cudaGetLastError());
  return 0;
}

int render_views(trn_scene* s, trn_viewset* vs, const trn_render_options* o, int integrator,
                 const trn_samples* smp, const trn_launch* ln, int spp_override, bool forward, float* image,
                 const float* dLdI, cudaStream_t st) {
  if (check_common(s, o, integrator)) return -1;
  if (!vs || vs->nviews <= 0) { set_error("empty view set"); return -1; }
  if (validate_launch(ln)) return -1;
  long long total = 0;
  if (upload_views(vs, o, integrator, spp_override, total, st)) return -1;
  Params P = base_params(s, vs, o, integrator, smp, ln, total);
  P.image = forward ? image : nullptr;
  P.dLdI = forward ? nullptr : dLdI;
  const long long slots = integrator == TRN_PIXEL_EDGE ? total / 4 : total;
  if (P.table && P.stride < slots) { set_error("sample table too small"); return -1; }
  if (forward) {
    // a call buffer is cleared; views with their own image accumulate into it
    if (image) TRN_CUDA_TRY(cudaMemsetAsync(image, 0, sizeof(float) * 3 * vs->npix, st));
    if (integrator != TRN_PATH_TRACER || total == 0) return 0;  // edge terms have no primal image
    TRN_CUDA_TRY(cudaMemsetAsync(vs->work, 0, sizeof(unsigned long long), st));
    const int cached = path_cache_fwd(vs, P, ln, o, spp_override, total, st);
    if (cached <= 0) return cached;
    launch(k_path_fwd, ln, total, P, st);
    TRN_CUDA_TRY(cudaGetLastError());
    return 0;
  }
  if (total == 0) return 0;
  s->grads_finalized = false;
  if (integrator == TRN_PRIMARY_EDGE) {
    if (s->ne == 0) return 0;
    dim3 g((s->ne + 255) / 256, vs->nviews);
    k_prim_edges_views<<<g, 256, 0, st>>>(s->ne, s->edges, s->pos, s->fnormal, vs->views, vs->pfunc);
    k_cdf_views<<<vs->nviews, 1024, 0, st>>>(s->ne, vs->pfunc, vs->pcdf, vs->pint);
    count_launch(2);
  } else if ((integrator == TRN_DIRECT_EDGE || integrator == TRN_INDIRECT_EDGE) && s->ne == 0) {
    return 0;
  }
  if (integrator == TRN_DIRECT_EDGE && guide_setup(s, o, P, st)) return -1;
  TRN_CUDA_TRY(cudaMemsetAsync(vs->work, 0, sizeof(unsigned long long), st));
  const bool shallow = vs->max_depth <= 8;  // smaller per-thread path records
  switch (integrator) {
    case TRN_PATH_TRACER: {
      const int cached = path_cache_grad(vs, P, ln, o, spp_override, total, st);
      if (cached <= 0) return cached;
      if (TRN_PATHADJ_SPLIT) return path_adj_split(vs, P, ln, total, shallow, st);
      if (shallow) launch(k_path_adj<8>, ln, total, P, st); else launch(k_path_adj<kMaxDepth>, ln, total, P, st);
      break;
    }
    case TRN_PRIMARY_EDGE:
      if (TRN_PRIMARY_SPLIT) return primary_split(vs, P, ln, total, st);
      launch(k_primary_adj, ln, total, P, st);
      break;
    case TRN_DIRECT_EDGE:
      if (TRN_DIRECT_SPLIT) return direct_split(vs, P, ln, total, st);
      launch(k_direct_adj, ln, total, P, st);
      break;
    case TRN_INDIRECT_EDGE:
      if (TRN_INDIRECT_SPLIT) return indirect_split(vs, P, ln, total, shallow, st);
      if (shallow) launch(k_indirect_adj<8>, ln, total, P, st); else launch(k_indirect_adj<kMaxDepth>, ln, total, P, st);
      break;
    default:
      if (TRN_PIXEL_SPLIT) return pixel_split(vs, P, ln, total, st);
      launch(k_pixel_adj, ln, total, P, st);
      break;
  }
  TRN_CUDA_TRY(cudaGetLastError());
  return 0;
}

// (Re)define the views of a set. Device arrays grow to the largest view count
// seen; the per-view silhouette workspace is E floats x 2 per view.
int set_views(trn_viewset* vs, int nviews, const trn_view* views) {
  std::vector<long long> pb;
  long long pix = 0;
  for (int v = 0; v < nviews; v++) {
    const trn_view& hv = views[v];
    if (hv.camera.width <= 0 || hv.camera.height <= 0 || hv.spp < 0 || hv.max_bounces < 0 ||
        hv.max_bounces > kMaxDepth) {
      set_error("viewset: invalid view (resolution, spp or max_bounces)");
      return -1;
    }
    const long long off = hv.pixel_offset >= 0 ? hv.pixel_offset : pix;
    if (!pb.empty() && off < pb.back()) { set_error("viewset: pixel offsets must be non-decreasing"); return -1; }
    pb.push_back(off);
    pix = std::max(pix, off + (long long)hv.camera.width * hv.camera.height);
  }
  if (nviews > vs->cap) {
    wait_stages(vs);
    void* old[] = {vs->views, vs->vbegin, vs->pbegin, vs->pfunc, vs->pcdf, vs->pint};
    for (void* q : old) if (q) cudaFree(q);
    if (vs->h_stage) cudaFreeHost(vs->h_stage);
    if (vs->h_stage_begin) cudaFreeHost(vs->h_stage_begin);
    vs->views = nullptr; vs->vbegin = vs->pbegin = nullptr; vs->pfunc = vs->pcdf = vs->pint = nullptr;
    vs->h_stage = nullptr; vs->h_stage_begin = nullptr;
    const int cap = std::max(nviews, 2 * vs->cap);
    bool ok = cudaMalloc(&vs->views, sizeof(ViewDesc) * cap) == cudaSuccess &&
              cudaMalloc(&vs->vbegin, sizeof(long long) * cap) == cudaSuccess &&
              cudaMalloc(&vs->pbegin, sizeof(long long) * cap) == cudaSuccess &&
              cudaMalloc(&vs->pint, sizeof(float) * cap) == cudaSuccess &&
              cudaMallocHost(&vs->h_stage, sizeof(ViewDesc) * cap * kStageRing) == cudaSuccess &&
              cudaMallocHost(&vs->h_stage_begin, sizeof(long long) * 2 * cap * kStageRing) == cudaSuccess;
    if (ok && vs->ne > 0)
      ok = cudaMalloc(&vs->pfunc, sizeof(float) * (size_t)cap * vs->ne) == cudaSuccess &&
           cudaMalloc(&vs->pcdf, sizeof(float) * (size_t)cap * vs->ne) == cudaSuccess;
    if (!ok) { set_error("viewset: out of memory"); vs->cap = 0; return -1; }
    cudaMemset(vs->pint, 0, sizeof(float) * cap);
    vs->cap = cap;
  }
  vs->nviews = nviews;
  vs->h_views.assign(views, views + nviews);
  vs->h_pbegin = pb;
  vs->npix = pix;
  vs->uploaded_key = -2;
  vs->pbegin_dirty = true;
  return 0;
}

// upload the per-view pixel offsets (used by the loss kernel) when they changed
int upload_pbegin(trn_viewset* vs, cudaStream_t st) {
  if (!vs->pbegin_dirty) return 0;
  const int slot = next_stage(vs);
  long long* stage = vs->h_stage_begin + (size_t)slot * 2 * vs->cap + vs->cap;
  std::memcpy(stage, vs->h_pbegin.data(), sizeof(long long) * vs->nviews);
  TRN_CUDA_TRY(cudaMemcpyAsync(vs->pbegin, stage, sizeof(long long) * vs->nviews, cudaMemcpyHostToDevice, st));
  TRN_CUDA_TRY(cudaEventRecord(vs->stage_done[slot], st));
  vs->pbegin_dirty = false;
  return 0;
}

// The scene's cached one-view set, re-pointed at `cam`: the first call
// allocates it, later calls only restage the view table (a pinned slot of
// the set's staging ring), so single-view calls neither allocate nor
// synchronise the stream.
int single_view(trn_scene* s, const trn_camera* cam, trn_viewset** out) {
  if (!cam) { set_error("null camera"); return -1; }
  trn_view v;
  std::memset(&v, 0, sizeof(v));
  std::memcpy(&v.camera, cam, sizeof(trn_camera));
  if (s->single) {
    // an unchanged camera keeps the uploaded table: no restaging, so the host
    // does not wait for the previous call's upload and can run ahead
    const bool same = s->single->nviews == 1 && s->single->h_views.size() == 1 &&
                      std::memcmp(&s->single->h_views[0], &v, sizeof(v)) == 0;
    if (!same && set_views(s->single, 1, &v)) return -1;
  } else if (trn_viewset_create(s, 1, &v, &s->single)) {
    return -1;
  }
  s->single->pc_limit = s->single_path_cache;
  *out = s->single;
  return 0;
}

}  // namespace

extern "C" {

int trn_viewset_create(trn_scene* s, int nviews, const trn_view* views, trn_viewset** out) {
  if (!s || !views || !out || nviews <= 0) { set_error("trn_viewset_create: invalid arguments"); return -1; }
  *out = nullptr;
  trn_viewset* vs = new trn_viewset();
  vs->scene = s;
  vs->ne = s->ne;
  bool ok = cudaMalloc(&vs->work, sizeof(unsigned long long)) == cudaSuccess;
  for (cudaEvent_t& e : vs->stage_done) ok = ok && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    set_error("trn_viewset_create: out of memory");
    trn_viewset_destroy(vs);
    return -1;
  }
  if (set_views(vs, nviews, views)) { trn_viewset_destroy(vs); return -1; }
  *out = vs;
  return 0;
}

int trn_viewset_update(trn_viewset* vs, int nviews, const trn_view* views) {
  if (!vs || !views || nviews <= 0) { set_error("trn_viewset_update: invalid arguments"); return -1; }
  return set_views(vs, nviews, views);
}

int trn_viewset_destroy(trn_viewset* vs) {
  if (!vs) return 0;
  wait_stages(vs);
  void* ptrs[] = {vs->views, vs->vbegin, vs->pbegin, vs->pfunc, vs->pcdf, vs->pint, vs->work, vs->iq, vs->iq_count, vs->sq, vs->pc, vs->pc_count};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (vs->h_stage) cudaFreeHost(vs->h_stage);
  if (vs->h_stage_begin) cudaFreeHost(vs->h_stage_begin);
  for (cudaEvent_t e : vs->stage_done)
    if (e) cudaEventDestroy(e);
  delete vs;
  return 0;
}

int trn_viewset_num_pixels(const trn_viewset* vs, long long* npix) {
  if (!vs || !npix) { set_error("trn_viewset_num_pixels: null argument"); return -1; }
  *npix = vs->npix;
  return 0;
}

int trn_viewset_reserve(trn_viewset* vs, int max_bounces, cudaStream_t st) {
  if (!vs) { set_error("trn_viewset_reserve: null view set"); return -1; }
  if (max_bounces < 0 || max_bounces > kMaxDepth) { set_error("trn_viewset_reserve: max_bounces must be in [0, 16]"); return -1; }
  if (ensure_queue(vs, full_queue_bytes(max_bounces <= 8), st)) return -1;
  if (TRN_EDGE_ORDER && alloc_order(vs, kIndirectRound, st)) return -1;
  return 0;
}

int trn_viewset_path_cache(trn_viewset* vs, long long max_bytes) {
  if (!vs || max_bytes < 0) { set_error("trn_viewset_path_cache: invalid arguments"); return -1; }
  vs->pc_limit = max_bytes;
  vs->pc_valid = false;
  if (max_bytes == 0 && vs->pc) {
    wait_stages(vs);
    TRN_CUDA_TRY(cudaDeviceSynchronize());
    cudaFree(vs->pc);
    vs->pc = nullptr;
    vs->pc_bytes = 0;
  }
  return 0;
}

int trn_scene_path_cache(trn_scene* s, long long max_bytes) {
  if (!s || max_bytes < 0) { set_error("trn_scene_path_cache: invalid arguments"); return -1; }
  s->single_path_cache = max_bytes;
  if (s->single) return trn_viewset_path_cache(s->single, max_bytes);
  return 0;
}

int trn_render_views_fwd(trn_scene* s, trn_viewset* vs, const trn_render_options* o, int integrator,
                         const trn_samples* smp, const trn_launch* ln, float* images, cudaStream_t st) {
  if (!images)
    for (const trn_view& v : vs->h_views)
      if (!v.image) { set_error("trn_render_views_fwd: no image buffer for a view"); return -1; }
  return render_views(s, vs, o, integrator, smp, ln, -1, true, images, nullptr, st);
}

int trn_render_views_grad(trn_scene* s, trn_viewset* vs, const trn_render_options* o, int integrator,
                          const trn_samples* smp, const trn_launch* ln, const float* dLdI, cudaStream_t st) {
  if (!dLdI)
    for (const trn_view& v : vs->h_views)
      if (!v.dLdI) { set_error("trn_render_views_grad: no dL/dI buffer for a view"); return -1; }
  return render_views(s, vs, o, integrator, smp, ln, -1, false, nullptr, dLdI, st);
}

int trn_views_loss(trn_viewset* vs, const float* images, const float* targets, float* dLdI, float* loss,
                   cudaStream_t st) {
  if (!vs || !images || !targets) { set_error("trn_views_loss: null argument"); return -1; }
  if (upload_pbegin(vs, st)) return -1;
  if (loss) TRN_CUDA_TRY(cudaMemsetAsync(loss, 0, sizeof(float) * vs->nviews, st));
  const long long n = vs->npix;
  k_view_loss<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, vs->views, vs->pbegin, vs->nviews, images, targets,
                                                          dLdI, loss);
  count_launch(1);
  TRN_CUDA_TRY(cudaGetLastError());
  return 0;
}

int trn_render_fwd(trn_scene* s, const trn_camera* cam, const trn_render_options* o, int integrator,
                   const trn_samples* smp, float* image, cudaStream_t st) {
  if (check_common(s, o, integrator)) return -1;
  if (!image) { set_error("trn_render_fwd: null image"); return -1; }
  trn_viewset* vs = nullptr;
  if (single_view(s, cam, &vs)) return -1;
  return render_views(s, vs, o, integrator, smp, nullptr, spp_of(o, integrator), true, image, nullptr, st);
}

int trn_render_grad(trn_scene* s, const trn_camera* cam, const trn_render_options* o, int integrator,
                    const trn_samples* smp, const float* dLdI, cudaStream_t st) {
  if (check_common(s, o, integrator)) return -1;
  if (!dLdI) { set_error("trn_render_grad: null dLdI"); return -1; }
  trn_viewset* vs = nullptr;
  if (single_view(s, cam, &vs)) return -1;
  return render_views(s, vs, o, integrator, smp, nullptr, spp_of(o, integrator), false, nullptr, dLdI, st);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free single-view gradient.
//
// trn_render_grad allocates device memory (the scene's one-view table, work
// counter and silhouette-edge distribution) on a scene's first single-view
// call. Callers that may not allocate (a host that forbids cudaMalloc
// between set-up and teardown, a caching allocator that must not be bypassed,
// a real-time loop that cannot afford the implicit synchronisation of
// cudaFree) use trn_render_grad_noalloc instead: all of its scratch lives in
// the fixed-size array below, which is part of the loaded module.
//
// Scratch layout (each part 256-byte aligned): the view table (one ViewDesc),
// the first-sample index of that view, the work counter, the silhouette
// integral, then the silhouette function and its CDF (kNoAllocMaxEdges floats
// each). Every call rewrites all of it that it reads, so it keeps the last
// call's contents but never needs clearing from the outside. Two calls that
// overlap in time on one device share this one array and race; such callers
// must serialise them.
constexpr int kNoAllocMaxEdges = 1 << 20;
constexpr size_t kNoAllocHeader = 4096;  // ViewDesc, vbegin, work counter, integral
constexpr size_t kNoAllocScratchBytes = kNoAllocHeader + 2 * sizeof(float) * (size_t)kNoAllocMaxEdges;
static_assert(sizeof(ViewDesc) + 3 * 256 <= kNoAllocHeader, "view table does not fit the scratch header");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

constexpr int kNoAllocMaxDevices = 64;
std::atomic<unsigned char*> g_noalloc_base[kNoAllocMaxDevices];

// Device address of the scratch array for the current device. In host code
// the array's name only stands in for it, so the address comes from
// cudaGetSymbolAddress, once per device (this may load the module on that
// device, which is why the first call must not run inside stream capture).
// The scene's buffers must live on the current device: the address looked up
// is that device's copy of the array, and kernels launched there would
// otherwise read another GPU's scene.
unsigned char* noalloc_scratch(const trn_scene* s) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) {
    set_error("trn_render_grad_noalloc: no usable current device");
    return nullptr;
  }
  cudaPointerAttributes pa;
  if (cudaPointerGetAttributes(&pa, s->pos) != cudaSuccess || pa.type != cudaMemoryTypeDevice) {
    cudaGetLastError();
    set_error("trn_render_grad_noalloc: cannot tell which device holds the scene");
    return nullptr;
  }
  if (pa.device != dev) {
    set_error("trn_render_grad_noalloc: the scene lives on device " + std::to_string(pa.device) +
              " but device " + std::to_string(dev) + " is current; make the scene's device current");
    return nullptr;
  }
  unsigned char* p = g_noalloc_base[dev].load(std::memory_order_acquire);
  if (p) return p;
  void* addr = nullptr;
  const cudaError_t rc = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
  if (rc != cudaSuccess || !addr) {
    set_error(std::string("trn_render_grad_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(rc));
    return nullptr;
  }
  g_noalloc_base[dev].store((unsigned char*)addr, std::memory_order_release);
  return (unsigned char*)addr;
}

// Write the one-view table, its first-sample index (0) and a zero work
// counter into the scratch header; the view is passed by value, so no host
// staging buffer is involved.
__global__ void k_noalloc_setup(ViewDesc v, ViewDesc* table, long long* vbegin, unsigned long long* work) {
  if (threadIdx.x == 0) {
    *table = v;
    *vbegin = 0;
    *work = 0ull;
  }
}

}  // namespace

extern "C" {

int trn_render_grad_noalloc(trn_scene* s, const trn_camera* cam, const trn_render_options* o, int integrator,
                            const trn_samples* smp, const float* dLdI, cudaStream_t st) {
  if (check_common(s, o, integrator)) return -1;
  if (!cam || !dLdI) { set_error("trn_render_grad_noalloc: null camera or dLdI"); return -1; }
  if (cam->width <= 0 || cam->height <= 0) { set_error("trn_render_grad_noalloc: invalid resolution"); return -1; }
  if (integrator == TRN_PRIMARY_EDGE && s->ne > kNoAllocMaxEdges) {
    set_error("trn_render_grad_noalloc: the scene has " + std::to_string(s->ne) +
              " edges; the static scratch holds the silhouette distribution of at most " +
              std::to_string(kNoAllocMaxEdges));
    return -1;
  }
  const int spp = spp_of(o, integrator);
  if (spp < 0) { set_error("trn_render_grad_noalloc: negative spp"); return -1; }
  const long long total = (long long)cam->width * cam->height * spp;
  if (integrator == TRN_PIXEL_EDGE && total % 4 != 0) {
    set_error("pixel boundary needs W*H*spp divisible by 4");
    return -1;
  }
  unsigned char* base = noalloc_scratch(s);
  if (!base) return -1;
  ViewDesc* table = (ViewDesc*)base;
  long long* vbegin = (long long*)(base + kNoAllocHeader - 3 * 256);
  unsigned long long* work = (unsigned long long*)(base + kNoAllocHeader - 2 * 256);
  float* pint = (float*)(base + kNoAllocHeader - 256);
  float* pfunc = (float*)(base + kNoAllocHeader);
  float* pcdf = pfunc + kNoAllocMaxEdges;

  ViewDesc v;
  std::memset(&v, 0, sizeof(v));
  std::memcpy(&v.cam, cam, sizeof(CameraDesc));
  v.begin = 0;
  v.n = total;
  v.pix_off = 0;
  v.slot_off = 0;
  v.inv_spp = spp > 0 ? 1.0f / (float)spp : 0.f;
  v.seed = 0;
  v.spp = spp;
  v.D = o->max_bounces;
  v.gpos = s->g_pos;
  v.gvn = s->g_vnormal;
  v.gtex = s->g_texels;
  v.pfunc = pfunc;
  v.pcdf = pcdf;
  v.pint = pint;

  // host-side view of the scratch (no device memory of its own)
  trn_viewset vs;
  vs.scene = s;
  vs.nviews = 1;
  vs.ne = s->ne;
  vs.views = table;
  vs.vbegin = vbegin;
  vs.work = work;
  Params P = base_params(s, &vs, o, integrator, smp, nullptr, total);
  P.image = nullptr;
  P.dLdI = dLdI;
  const long long slots = integrator == TRN_PIXEL_EDGE ? total / 4 : total;
  if (P.table && P.stride < slots) { set_error("sample table too small"); return -1; }
  if (total == 0) return 0;
  if ((integrator == TRN_PRIMARY_EDGE || integrator == TRN_DIRECT_EDGE || integrator == TRN_INDIRECT_EDGE) &&
      s->ne == 0)
    return 0;

  k_noalloc_setup<<<1, 32, 0, st>>>(v, table, vbegin, work);
  count_launch(1);
  s->grads_finalized = false;
  if (integrator == TRN_PRIMARY_EDGE) {
    dim3 g((s->ne + 255) / 256, 1);
    k_prim_edges_views<<<g, 256, 0, st>>>(s->ne, s->edges, s->pos, s->fnormal, table, pfunc);
    k_cdf_views<<<1, 1024, 0, st>>>(s->ne, pfunc, pcdf, pint);
    count_launch(2);
  }
  // the guiding distribution lives in buffers the scene allocated at creation
  // (a refined tree in those of an earlier allocating call)
  if (integrator == TRN_DIRECT_EDGE && guide_setup(s, o, P, st, false)) return -1;
  const bool shallow = o->max_bounces <= 8;
  switch (integrator) {
    case TRN_PATH_TRACER:
      if (shallow) launch(k_path_adj<8>, nullptr, total, P, st); else launch(k_path_adj<kMaxDepth>, nullptr, total, P, st);
      break;
    case TRN_PRIMARY_EDGE: launch(k_primary_adj, nullptr, total, P, st); break;
    case TRN_DIRECT_EDGE: launch(k_direct_adj, nullptr, total, P, st); break;
    case TRN_INDIRECT_EDGE:
      if (shallow) launch(k_indirect_adj<8>, nullptr, total, P, st);
      else launch(k_indirect_adj<kMaxDepth>, nullptr, total, P, st);
      break;
    default: launch(k_pixel_adj, nullptr, total, P, st); break;
  }
  TRN_CUDA_TRY(cudaGetLastError());
  return 0;
}

int trn_intersect(trn_scene* s, int n, const float* org, const float* dir, const float* tmin, const float* tmax,
                  int* tri, float* u, float* v, float* t, cudaStream_t st) {
  if (!s || !s->configured) { set_error("trn_intersect: scene not configured"); return -1; }
  if (n <= 0) return 0;
  if (!org || !dir || !tmin || !tmax || !tri || !u || !v || !t) { set_error("trn_intersect: null argument"); return -1; }
  k_intersect<<<(n + 127) / 128, 128, 0, st>>>(s->view(), n, org, dir, tmin, tmax, tri, u, v, t, s->err);
  count_launch(1);
  TRN_CUDA_TRY(cudaGetLastError());
  return 0;
}

int trn_occluded(trn_scene* s, int n, const float* org, const float* dir, const float* tmin, const float* tmax,
                 int* vis, cudaStream_t st) {
  if (!s || !s->configured) { set_error("trn_occluded: scene not configured"); return -1; }
  if (n <= 0) return 0;
  if (!org || !dir || !tmin || !tmax || !vis) { set_error("trn_occluded: null argument"); return -1; }
  k_occluded<<<(n + 127) / 128, 128, 0, st>>>(s->view(), n, org, dir, tmin, tmax, vis);
  count_launch(1);
  TRN_CUDA_TRY(cudaGetLastError());
  return 0;
}

}  // extern "C"
