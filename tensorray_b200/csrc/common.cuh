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

// ---- deterministic trigonometry for the sampling code ----------------------
// The directions a path takes depend on sin/cos (cosine-weighted hemisphere,
// concentric disk, edge-wedge sampling) and acos (wedge angle). CUDA's cosf
// and the CPU's libm round differently in the last ulp, and one ulp in a
// sampled direction can send a grazing ray to another triangle. These
// versions are evaluated in binary64 with individually rounded operations
// only (explicit _rn intrinsics on the device; no contraction on the host),
// then rounded once to float, so the CPU restatement reproduces every bit
// with numpy float64. Methods (no library code involved):
//   * sin/cos: reduction by the nearest multiple k of pi/2 (Cody & Waite,
//     "Software Manual for the Elementary Functions", 1980; one binary64 pi/2
//     is exact enough for |x| < 64), then the Taylor polynomials of sin and
//     cos, coefficients (-1)^j/(2j+1)! and (-1)^j/(2j)!, to degree 15 and 16
//     on |y| <= pi/4 (truncation below 2e-14);
//   * acos: the Maclaurin series of asin, coefficients
//     (2n)! / (4^n (n!)^2 (2n+1)), n <= 20, on [0, 1/2] (truncation below
//     1e-15), and acos(a) = 2 asin(sqrt((1 - a)/2)) for a > 1/2.
// Inputs outside [-1, 1] give NaN from acos_det, as acosf does.
#ifdef __CUDA_ARCH__
#define TRN_DMUL(a, b) __dmul_rn((a), (b))
#define TRN_DADD(a, b) __dadd_rn((a), (b))
#define TRN_DSUB(a, b) __dsub_rn((a), (b))
#define TRN_DSQRT(a) __dsqrt_rn((a))
#else
#define TRN_DMUL(a, b) ((a) * (b))
#define TRN_DADD(a, b) ((a) + (b))
#define TRN_DSUB(a, b) ((a) - (b))
#define TRN_DSQRT(a) sqrt((a))
#endif
constexpr double kPiD = 3.141592653589793;
constexpr double kPiOver2D = 1.5707963267948966;
constexpr double kTwoOverPiD = 0.6366197723675814;

TRN_HD double sin_poly_d(double y) {  // |y| <= pi/4
  const double y2 = TRN_DMUL(y, y);
  double p = -1.0 / 1307674368000.0;
  p = TRN_DADD(1.0 / 6227020800.0, TRN_DMUL(y2, p));
  p = TRN_DADD(-1.0 / 39916800.0, TRN_DMUL(y2, p));
  p = TRN_DADD(1.0 / 362880.0, TRN_DMUL(y2, p));
  p = TRN_DADD(-1.0 / 5040.0, TRN_DMUL(y2, p));
  p = TRN_DADD(1.0 / 120.0, TRN_DMUL(y2, p));
  p = TRN_DADD(-1.0 / 6.0, TRN_DMUL(y2, p));
  return TRN_DADD(y, TRN_DMUL(TRN_DMUL(y, y2), p));
}
TRN_HD double cos_poly_d(double y) {  // |y| <= pi/4
  const double y2 = TRN_DMUL(y, y);
  double p = 1.0 / 20922789888000.0;
  p = TRN_DADD(-1.0 / 87178291200.0, TRN_DMUL(y2, p));
  p = TRN_DADD(1.0 / 479001600.0, TRN_DMUL(y2, p));
  p = TRN_DADD(-1.0 / 3628800.0, TRN_DMUL(y2, p));
  p = TRN_DADD(1.0 / 40320.0, TRN_DMUL(y2, p));
  p = TRN_DADD(-1.0 / 720.0, TRN_DMUL(y2, p));
  p = TRN_DADD(1.0 / 24.0, TRN_DMUL(y2, p));
  p = TRN_DADD(-0.5, TRN_DMUL(y2, p));
  return TRN_DADD(1.0, TRN_DMUL(y2, p));
}
TRN_HD void sincos_det(float x, float& s, float& c) {
  const double xd = (double)x;
  const double k = floor(TRN_DADD(TRN_DMUL(xd, kTwoOverPiD), 0.5));
  const double y = TRN_DSUB(xd, TRN_DMUL(k, kPiOver2D));
  const double sy = sin_poly_d(y), cy = cos_poly_d(y);
  const int q = ((int)k) & 3;
  double sd, cd;
  if (q == 0) { sd = sy; cd = cy; }
  else if (q == 1) { sd = cy; cd = -sy; }
  else if (q == 2) { sd = -sy; cd = -cy; }
  else { sd = -cy; cd = sy; }
  s = (float)sd;
  c = (float)cd;
}
TRN_HD double asin_series_d(double z) {  // 0 <= z <= 1/2
  const double z2 = TRN_DMUL(z, z);
  double p = 0.0030578216492580306;
  p = TRN_DADD(0.003297059503473485, TRN_DMUL(z2, p));
  p = TRN_DADD(0.0035692053938259347, TRN_DMUL(z2, p));
  p = TRN_DADD(0.003880964558837669, TRN_DMUL(z2, p));
  p = TRN_DADD(0.004240907093679363, TRN_DMUL(z2, p));
  p = TRN_DADD(0.004660143486915096, TRN_DMUL(z2, p));
  p = TRN_DADD(0.005153309682319905, TRN_DMUL(z2, p));
  p = TRN_DADD(0.005740037670841924, TRN_DMUL(z2, p));
  p = TRN_DADD(0.006447210311889649, TRN_DMUL(z2, p));
  p = TRN_DADD(0.0073125258735988454, TRN_DMUL(z2, p));
  p = TRN_DADD(0.008390335809616815, TRN_DMUL(z2, p));
  p = TRN_DADD(0.009761609529194078, TRN_DMUL(z2, p));
  p = TRN_DADD(0.011551800896139705, TRN_DMUL(z2, p));
  p = TRN_DADD(0.01396484375, TRN_DMUL(z2, p));
  p = TRN_DADD(0.017352764423076924, TRN_DMUL(z2, p));
  p = TRN_DADD(0.022372159090909092, TRN_DMUL(z2, p));
  p = TRN_DADD(0.030381944444444444, TRN_DMUL(z2, p));
  p = TRN_DADD(0.044642857142857144, TRN_DMUL(z2, p));
  p = TRN_DADD(0.075, TRN_DMUL(z2, p));
  p = TRN_DADD(0.16666666666666666, TRN_DMUL(z2, p));
  return TRN_DADD(z, TRN_DMUL(TRN_DMUL(z, z2), p));
}
TRN_HD float acos_det(float x) {
  const double xd = (double)x;
  const double a = xd < 0.0 ? -xd : xd;
  if (!(a <= 1.0)) return nanf("");
  double r;
  if (a <= 0.5) {
    const double t = asin_series_d(a);
    r = xd < 0.0 ? TRN_DADD(kPiOver2D, t) : TRN_DSUB(kPiOver2D, t);
  } else {
    const double z = TRN_DSQRT(TRN_DMUL(TRN_DSUB(1.0, a), 0.5));
    const double t = TRN_DMUL(2.0, asin_series_d(z));
    r = xd < 0.0 ? TRN_DSUB(kPiD, t) : t;
  }
  return (float)r;
}
TRN_HD float cos_det(float x) { float s, c; sincos_det(x, s, c); return c; }
TRN_HD float sin_det(float x) { float s, c; sincos_det(x, s, c); return s; }

// ---- scalar helpers that dispatch on float / dual --------------------------
TRN_HD float val(float x) { return x; }
TRN_HD float sqrt_(float x) { return sqrtf(x); }
TRN_HD float abs_(float x) { return fabsf(x); }
TRN_HD float exp_(float x) { return expf(x); }
TRN_HD float log_(float x) { return logf(x); }
TRN_HD float cos_(float x) { return cos_det(x); }
TRN_HD float sin_(float x) { return sin_det(x); }
TRN_HD float acos_(float x) { return acos_det(x); }
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
