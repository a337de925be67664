// Shared device/host math for the trn path-space differentiable renderer.
//
// Everything here is templated on the scalar type S so that the same source
// evaluates a path factor in plain float (forward kernels) and in forward-mode
// dual numbers (local Jacobians inside the adjoint kernels, see dual.cuh).
//
// Constants follow LibTensorRay/Renderer/Config.h:33-35 (EPSILON, EDGE_EPSILON,
// SHADOW_EPSILON) and EDXUtil/Math/Constants.h (pi).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>
#include <type_traits>

#define TRN_HD __host__ __device__ __forceinline__
#define TRN_D __device__ __forceinline__

namespace trn {

constexpr float kEps = 1e-6f;         // Config.h:33 EPSILON
constexpr float kEdgeEps = 1e-8f;     // Config.h:34 EDGE_EPSILON
constexpr float kShadowEps = 1e-2f;   // Config.h:35 SHADOW_EPSILON
constexpr float kRayMax = 1e32f;      // Camera.cpp:246 ray.mMax
constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 0.31830988618379067154f;
constexpr float kPiOver2 = 1.57079632679489661923f;
constexpr float kPiOver4 = 0.78539816339744830962f;

// ---- scalar helpers that dispatch on float / dual --------------------------
TRN_HD float val(float x) { return x; }
TRN_HD float sqrt_(float x) { return sqrtf(x); }
TRN_HD float abs_(float x) { return fabsf(x); }
TRN_HD float exp_(float x) { return expf(x); }
TRN_HD float log_(float x) { return logf(x); }
TRN_HD float cos_(float x) { return cosf(x); }
TRN_HD float sin_(float x) { return sinf(x); }
TRN_HD float acos_(float x) { return acosf(x); }
TRN_HD float detach(float x) { return x; }
TRN_HD float fmax_(float a, float b) { return fmaxf(a, b); }
TRN_HD float fmin_(float a, float b) { return fminf(a, b); }
TRN_HD float select(bool c, float a, float b) { return c ? a : b; }

template <class S>
struct V3 {
  S x, y, z;
  TRN_HD V3() {}
  TRN_HD V3(S a, S b, S c) : x(a), y(b), z(c) {}
  template <class T>
  TRN_HD explicit V3(const V3<T>& o) : x(S(o.x)), y(S(o.y)), z(S(o.z)) {}
  TRN_HD S& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  TRN_HD const S& operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
using F3 = V3<float>;

template <class S> TRN_HD V3<S> operator+(const V3<S>& a, const V3<S>& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class S> TRN_HD V3<S> operator-(const V3<S>& a, const V3<S>& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class S> TRN_HD V3<S> operator-(const V3<S>& a) { return {-a.x, -a.y, -a.z}; }
template <class S> TRN_HD V3<S> operator*(const V3<S>& a, const V3<S>& b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class S> TRN_HD V3<S> operator*(const V3<S>& a, const S& s) { return {a.x * s, a.y * s, a.z * s}; }
template <class S> TRN_HD V3<S> operator*(const S& s, const V3<S>& a) { return {a.x * s, a.y * s, a.z * s}; }
template <class S> TRN_HD V3<S> operator/(const V3<S>& a, const S& s) { return {a.x / s, a.y / s, a.z / s}; }
// mixed float scalar (only instantiated when S is not float)
template <class S, class = typename std::enable_if<!std::is_same<S, float>::value>::type>
TRN_HD V3<S> operator*(const V3<S>& a, float s) { return {a.x * s, a.y * s, a.z * s}; }
template <class S, class = typename std::enable_if<!std::is_same<S, float>::value>::type>
TRN_HD V3<S> operator*(float s, const V3<S>& a) { return {a.x * s, a.y * s, a.z * s}; }

template <class S> TRN_HD S dot(const V3<S>& a, const V3<S>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class S> TRN_HD V3<S> cross(const V3<S>& a, const V3<S>& b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class S> TRN_HD S length2(const V3<S>& a) { return dot(a, a); }
template <class S> TRN_HD S length(const V3<S>& a) { return sqrt_(dot(a, a)); }
template <class S> TRN_HD V3<S> normalize(const V3<S>& a) { return a / length(a); }
template <class S> TRN_HD V3<float> vval(const V3<S>& a) { return {val(a.x), val(a.y), val(a.z)}; }
template <class S> TRN_HD V3<S> vdetach(const V3<S>& a) { return {detach(a.x), detach(a.y), detach(a.z)}; }
template <class S> TRN_HD V3<S> vselect(bool c, const V3<S>& a, const V3<S>& b) {
  return {select(c, a.x, b.x), select(c, a.y, b.y), select(c, a.z, b.z)};
}
template <class S> TRN_HD V3<S> lift(const F3& a) { return {S(a.x), S(a.y), S(a.z)}; }

TRN_HD F3 make_f3(const float* p) { return {p[0], p[1], p[2]}; }
TRN_HD bool finite3(const F3& a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }

// ---- counter-based uniform sampler --------------------------------------
// One uniform float per (seed, term, dimension, slot). The hash is the
// "lowbias32" integer mixer (Wellons, hash-prospector, 2018), applied to a key
// that folds the stream (seed, term, dim) and then the slot. Output is
// (k + 0.5) * 2^-23 with k the top 23 bits: exactly representable, and always
// inside [2^-24, 1 - 2^-24] like the clamped sample tensor.
TRN_HD uint32_t mix32(uint32_t x) {
  x ^= x >> 16; x *= 0x7feb352dU;
  x ^= x >> 15; x *= 0x846ca68bU;
  x ^= x >> 16;
  return x;
}
TRN_HD float hash_uniform(uint32_t seed, uint32_t term, uint32_t dim, uint32_t slot) {
  uint32_t s = mix32(seed * 0x9E3779B9U + 0x632BE5ABU);
  s = mix32(s ^ (term * 0x85EBCA6BU + 0x1B873593U));
  s = mix32(s ^ (dim * 0xC2B2AE35U + 0x27D4EB2FU));
  uint32_t h = mix32(s ^ mix32(slot + 0x165667B1U));
  return ((float)(h >> 9) + 0.5f) * (1.0f / 8388608.0f);
}

// Sample source: either a caller-provided uniform tensor laid out as
// [dim][slot] (SoA blocks per call site, like Tensorf::RandomFloat of
// Shape({N}, VecN) in Tensor.h:2793-2799) or the counter hash above.
struct SampleSource {
  const float* table;   // nullptr => hash
  int64_t stride;       // number of slots per dimension in the table
  uint32_t seed;
  uint32_t term;
  TRN_HD float get(int dim, int64_t slot) const {
    if (table) return table[(int64_t)dim * stride + slot];
    return hash_uniform(seed, term, (uint32_t)dim, (uint32_t)slot);
  }
};

}  // namespace trn
