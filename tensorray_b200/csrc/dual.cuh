// Forward-mode dual numbers with N tangent lanes.
//
// The adjoint kernels use these to take the local Jacobian of one path factor
// (a handful of float3 inputs -> an RGB or scalar output) and contract it with
// the reverse-accumulated path adjoint. Values are computed with exactly the
// same float operations as the plain float instantiation, so the value part of
// a dual evaluation equals the forward kernel's result.
#pragma once
#include "common.cuh"

namespace trn {

template <int N>
struct Dual {
  float v;
  float d[N];
  TRN_HD Dual() {}
  TRN_HD Dual(float x) : v(x) {
#pragma unroll
    for (int i = 0; i < N; i++) d[i] = 0.f;
  }
};

template <int N> TRN_HD float val(const Dual<N>& a) { return a.v; }
template <int N> TRN_HD Dual<N> detach(const Dual<N>& a) { return Dual<N>(a.v); }

#define TRN_DUAL_BIN(OP, VEXPR, DEXPR)                                          \
  template <int N> TRN_HD Dual<N> operator OP(const Dual<N>& a, const Dual<N>& b) { \
    Dual<N> r; r.v = VEXPR;                                                     \
    _Pragma("unroll") for (int i = 0; i < N; i++) r.d[i] = DEXPR;               \
    return r;                                                                   \
  }
TRN_DUAL_BIN(+, a.v + b.v, a.d[i] + b.d[i])
TRN_DUAL_BIN(-, a.v - b.v, a.d[i] - b.d[i])
TRN_DUAL_BIN(*, a.v * b.v, a.d[i] * b.v + a.v * b.d[i])
#undef TRN_DUAL_BIN

template <int N> TRN_HD Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v / b.v;
  float inv = 1.f / b.v;
#pragma unroll
  for (int i = 0; i < N; i++) r.d[i] = (a.d[i] - r.v * b.d[i]) * inv;
  return r;
}
template <int N> TRN_HD Dual<N> operator-(const Dual<N>& a) {
  Dual<N> r; r.v = -a.v;
#pragma unroll
  for (int i = 0; i < N; i++) r.d[i] = -a.d[i];
  return r;
}
// scalar-float mixes
template <int N> TRN_HD Dual<N> operator+(const Dual<N>& a, float b) { Dual<N> r = a; r.v = a.v + b; return r; }
template <int N> TRN_HD Dual<N> operator+(float b, const Dual<N>& a) { Dual<N> r = a; r.v = b + a.v; return r; }
template <int N> TRN_HD Dual<N> operator-(const Dual<N>& a, float b) { Dual<N> r = a; r.v = a.v - b; return r; }
template <int N> TRN_HD Dual<N> operator-(float b, const Dual<N>& a) {
  Dual<N> r; r.v = b - a.v;
#pragma unroll
  for (int i = 0; i < N; i++) r.d[i] = -a.d[i];
  return r;
}
template <int N> TRN_HD Dual<N> operator*(const Dual<N>& a, float b) {
  Dual<N> r; r.v = a.v * b;
#pragma unroll
  for (int i = 0; i < N; i++) r.d[i] = a.d[i] * b;
  return r;
}
template <int N> TRN_HD Dual<N> operator*(float b, const Dual<N>& a) {
  Dual<N> r; r.v = b * a.v;
#pragma unroll
  for (int i = 0; i < N; i++) r.d[i] = b * a.d[i];
  return r;
}
template <int N> TRN_HD Dual<N> operator/(const Dual<N>& a, float b) {
  Dual<N> r; r.v = a.v / b;
#pragma unroll
  for (int i = 0; i < N; i++) r.d[i] = a.d[i] / b;
  return r;
}
template <int N> TRN_HD Dual<N> operator/(float a, const Dual<N>& b) {
  Dual<N> r; r.v = a / b.v;
  float k = -r.v / b.v;
#pragma unroll
  for (int i = 0; i < N; i++) r.d[i] = k * b.d[i];
  return r;
}

template <int N> TRN_HD bool operator<(const Dual<N>& a, const Dual<N>& b) { return a.v < b.v; }
template <int N> TRN_HD bool operator>(const Dual<N>& a, const Dual<N>& b) { return a.v > b.v; }
template <int N> TRN_HD bool operator<=(const Dual<N>& a, const Dual<N>& b) { return a.v <= b.v; }
template <int N> TRN_HD bool operator>=(const Dual<N>& a, const Dual<N>& b) { return a.v >= b.v; }
template <int N> TRN_HD bool operator<(const Dual<N>& a, float b) { return a.v < b; }
template <int N> TRN_HD bool operator>(const Dual<N>& a, float b) { return a.v > b; }
template <int N> TRN_HD bool operator<=(const Dual<N>& a, float b) { return a.v <= b; }
template <int N> TRN_HD bool operator>=(const Dual<N>& a, float b) { return a.v >= b; }
template <int N> TRN_HD bool operator==(const Dual<N>& a, float b) { return a.v == b; }
template <int N> TRN_HD bool operator!=(const Dual<N>& a, float b) { return a.v != b; }

template <int N> TRN_HD Dual<N> sqrt_(const Dual<N>& a) {
  Dual<N> r; r.v = sqrtf(a.v);
  float k = 0.5f / r.v;
#pragma unroll
  for (int i = 0; i < N; i++) r.d[i] = k * a.d[i];
  return r;
}
template <int N> TRN_HD Dual<N> abs_(const Dual<N>& a) {
  // d|x|/dx follows AbsOp::Backward (TemplateExpression.h:1546-1548): +1 for
  // x > 0, -1 otherwise (including x == 0).
  float s = a.v > 0.f ? 1.f : -1.f;
  Dual<N> r; r.v = fabsf(a.v);
#pragma unroll
  for (int i = 0; i < N; i++) r.d[i] = s * a.d[i];
  return r;
}
template <int N> TRN_HD Dual<N> exp_(const Dual<N>& a) {
  Dual<N> r; r.v = expf(a.v);
#pragma unroll
  for (int i = 0; i < N; i++) r.d[i] = r.v * a.d[i];
  return r;
}
template <int N> TRN_HD Dual<N> log_(const Dual<N>& a) {
  Dual<N> r; r.v = logf(a.v);
  float k = 1.f / a.v;
#pragma unroll
  for (int i = 0; i < N; i++) r.d[i] = k * a.d[i];
  return r;
}
template <int N> TRN_HD Dual<N> cos_(const Dual<N>& a) {
  Dual<N> r; float s, c; sincos_det(a.v, s, c); r.v = c;
#pragma unroll
  for (int i = 0; i < N; i++) r.d[i] = -s * a.d[i];
  return r;
}
template <int N> TRN_HD Dual<N> sin_(const Dual<N>& a) {
  Dual<N> r; float s, c; sincos_det(a.v, s, c); r.v = s;
#pragma unroll
  for (int i = 0; i < N; i++) r.d[i] = c * a.d[i];
  return r;
}
template <int N> TRN_HD Dual<N> acos_(const Dual<N>& a) {
  Dual<N> r; r.v = acos_det(a.v);
  float k = -1.f / sqrtf(1.f - a.v * a.v);
#pragma unroll
  for (int i = 0; i < N; i++) r.d[i] = k * a.d[i];
  return r;
}
// Maximum/Minimum: the gradient follows the selected operand.
template <int N> TRN_HD Dual<N> fmax_(const Dual<N>& a, const Dual<N>& b) { return a.v >= b.v ? a : b; }
template <int N> TRN_HD Dual<N> fmin_(const Dual<N>& a, const Dual<N>& b) { return a.v <= b.v ? a : b; }
template <int N> TRN_HD Dual<N> fmax_(const Dual<N>& a, float b) { return a.v >= b ? a : Dual<N>(b); }
template <int N> TRN_HD Dual<N> fmin_(const Dual<N>& a, float b) { return a.v <= b ? a : Dual<N>(b); }
template <int N> TRN_HD Dual<N> select(bool c, const Dual<N>& a, const Dual<N>& b) { return c ? a : b; }

// Seed lane `lane0 .. lane0+2` of a float3 input.
template <int N>
TRN_HD V3<Dual<N>> seed3(const F3& a, int lane0) {
  V3<Dual<N>> r{Dual<N>(a.x), Dual<N>(a.y), Dual<N>(a.z)};
  if (lane0 >= 0) { r.x.d[lane0] = 1.f; r.y.d[lane0 + 1] = 1.f; r.z.d[lane0 + 2] = 1.f; }
  return r;
}
template <int N>
TRN_HD Dual<N> seed1(float a, int lane) {
  Dual<N> r(a);
  if (lane >= 0) r.d[lane] = 1.f;
  return r;
}

}  // namespace trn
