// Surface records, BSDFs, the merged area light and the pinhole sensor.
//
// Each function restates one reference routine (file:line given per function)
// for a single path vertex instead of a tensor of them. Functions that take a
// template scalar S are differentiated by the adjoint kernels with dual.cuh;
// the rest only ever run on detached values.
#pragma once
#include "dual.cuh"
#include "scene_types.cuh"
#include "trace.cuh"

namespace trn {

// ---- frames ---------------------------------------------------------------
// CoordinateSystem, Utils.cpp:118-140.
template <class S>
TRN_HD void coordinate_system(const V3<S>& n, V3<S>& t, V3<S>& b) {
  const bool cond = fabsf(val(n.x)) > fabsf(val(n.y));
  if (cond) {
    S inv = 1.f / sqrt_(fmax_(n.x * n.x + n.z * n.z, 1e-3f));
    t = V3<S>(-n.z * inv, S(0.f), n.x * inv);
  } else {
    S inv = 1.f / sqrt_(fmax_(n.y * n.y + n.z * n.z, 1e-3f));
    t = V3<S>(S(0.f), n.z * inv, -n.y * inv);
  }
  b = cross(n, t);
}

// Intersection::WorldToLocal / LocalToWorld, Records.cpp:165-181.
template <class S>
struct Frame {
  V3<S> t, b, n;
  TRN_HD V3<S> to_local(const V3<S>& v) const { return V3<S>(dot(v, t), dot(v, b), dot(v, n)); }
  TRN_HD V3<S> to_world(const V3<S>& v) const { return t * v.x + b * v.y + n * v.z; }
};
template <class S>
TRN_HD Frame<S> make_frame(const V3<S>& n) {
  Frame<S> f; f.n = n; coordinate_system(n, f.t, f.b); return f;
}

// ---- surface record (Scene::PostIntersect, Scene.cpp:668-730) -------------
struct SurfF {
  F3 p, ng, ns;
  float u, v;           // detached barycentrics of the hit (Scene.cpp:677)
  float tu, tv;         // texture coordinate
  int tri, bsdf, emitter;
};

TRN_D F3 load3(const float* a, int i) { return F3(__ldg(a + 3 * i), __ldg(a + 3 * i + 1), __ldg(a + 3 * i + 2)); }

TRN_D void tri_vertices(const DeviceScene& s, int tri, int& i0, int& i1, int& i2) {
  i0 = __ldg(s.idx + 3 * tri); i1 = __ldg(s.idx + 3 * tri + 1); i2 = __ldg(s.idx + 3 * tri + 2);
}

// barycentric interpolation w*a + u*b + v*c with w = (1 - u) - v
template <class S>
TRN_HD V3<S> bary3(float u, float v, const V3<S>& a, const V3<S>& b, const V3<S>& c) {
  const float w = 1.f - u - v;
  return a * w + b * u + c * v;
}

TRN_D SurfF post_intersect(const DeviceScene& s, int tri, float u, float v) {
  SurfF r;
  int i0, i1, i2; tri_vertices(s, tri, i0, i1, i2);
  r.p = bary3(u, v, load3(s.pos, i0), load3(s.pos, i1), load3(s.pos, i2));
  r.ng = load3(s.fnormal, tri);
  if (s.smooth[tri]) r.ns = bary3(u, v, load3(s.vnormal, i0), load3(s.vnormal, i1), load3(s.vnormal, i2));
  else r.ns = r.ng;
  if (s.uvidx) {
    const int j0 = __ldg(s.uvidx + 3 * tri), j1 = __ldg(s.uvidx + 3 * tri + 1), j2 = __ldg(s.uvidx + 3 * tri + 2);
    const float w = 1.f - u - v;
    r.tu = w * __ldg(s.uv + 2 * j0) + u * __ldg(s.uv + 2 * j1) + v * __ldg(s.uv + 2 * j2);
    r.tv = w * __ldg(s.uv + 2 * j0 + 1) + u * __ldg(s.uv + 2 * j1 + 1) + v * __ldg(s.uv + 2 * j2 + 1);
  } else {
    r.tu = 0.f; r.tv = 0.f;
  }
  r.u = u; r.v = v; r.tri = tri;
  r.bsdf = __ldg(s.bsdf_id + tri);
  r.emitter = __ldg(s.emitter_id + tri);
  return r;
}

// ---- textures (ImageTexture::Eval, BSDF.cpp:72-98; nearest texel) ---------
TRN_D int texel_index(const TexDesc& t, float u, float v) {
  const float tu = u - floorf(u), tv = v - floorf(v);
  const int ox = (int)(tu * (float)(t.w - 1));
  const int oy = (int)(tv * (float)(t.h - 1));
  return oy * t.w + ox;
}
// albedo of material b at (u,v); texel_out = global texel index or -1
TRN_D F3 bsdf_albedo(const DeviceScene& s, const BsdfDesc& b, float u, float v, long long& texel_out) {
  if (b.tex >= 0) {
    const TexDesc t = s.texs[b.tex];
    const long long k = t.offset + texel_index(t, u, v);
    texel_out = k;
    return load3(s.texels, (int)k);
  }
  texel_out = -1;
  return F3(b.albedo[0], b.albedo[1], b.albedo[2]);
}

// ---- BSDFs ----------------------------------------------------------------
// Diffuse::EvalInner (Diffuse.cpp:37-41) times the albedo texture
// (BSDF::Eval, BSDF.cpp:172-195) and Microfacet::EvalInner
// (Microfacet.cpp:37-79). `kd` is the albedo / diffuse reflectance.
template <class S>
TRN_HD V3<S> eval_inner(const BsdfDesc& b, const V3<S>& kd, const V3<S>& wo, const V3<S>& wi) {
  if (b.type == kDiffuse) {
    const bool reflect = (wo.z > 0.f) && (val(wo.z) * val(wi.z) > 0.f);
    return reflect ? kd * S(kInvPi) : V3<S>(S(0.f), S(0.f), S(0.f));
  }
  // microfacet
  const S nDotV = wo.z, nDotL = wi.z;
  const bool active = nDotV > 0.f && nDotL > 0.f;
  if (!active) return V3<S>(S(0.f), S(0.f), S(0.f));
  const V3<S> diffuse = kd * S(kInvPi);
  const V3<S> wh = normalize(wo + wi);
  const S nDotH = wh.z;
  const S vDotH = dot(wo, wh);
  const float r = b.roughness;
  const float alpha = r * r;
  const float k = (r + 1.f) * (r + 1.f) * 0.125f;
  const S tmp = alpha / (nDotH * nDotH * (alpha * alpha - 1.f) + 1.f);
  const S ggx = tmp * tmp * kInvPi;
  const S coeff = vDotH * (vDotH * -5.55473f - 6.8316f);
  const S e = exp_(log_(2.f) * coeff);
  const S G1 = nDotV / (nDotV * (1.f - k) + k);
  const S G2 = nDotL / (nDotL * (1.f - k) + k);
  const S G = G1 * G2;
  const S denom = 4.f * abs_(nDotV) * abs_(nDotL) + 1e-6f;
  V3<S> out;
  for (int c = 0; c < 3; c++) {
    const float F0 = b.spec[c];
    const S fres = F0 + (1.f - F0) * e;
    const S spec = ggx * G * fres / denom;
    out[c] = diffuse[c] + spec;
  }
  return out;
}

// BSDF::Eval with the optional shading-normal correction (BSDF.cpp:172-195).
template <class S>
TRN_HD V3<S> bsdf_eval(const BsdfDesc& b, const Frame<S>& f, const V3<S>& ng, const V3<S>& kd,
                       const V3<S>& wo, const V3<S>& wi, bool correction) {
  const V3<S> lwo = f.to_local(wo), lwi = f.to_local(wi);
  V3<S> v = eval_inner(b, kd, lwo, lwi);
  if (correction) {
    const S corr = abs_(lwo.z * dot(ng, wi) / (lwi.z * dot(ng, wo)));
    v = v * corr;
  }
  return v;
}

// GGX helpers (BSDF.cpp:232-302); only ever evaluated on detached values.
TRN_HD float tan_theta2(const F3& w) {
  const float c2 = w.z * w.z;
  return fmaxf(1.f - c2, 0.f) / c2;
}
TRN_HD float ggx_D(const F3& wh, float alpha) {
  const float tan2 = tan_theta2(wh);
  const bool valid = tan2 < 3.402823466e+38f;
  const float cos2 = wh.z * wh.z;
  const float e = 1.f / (alpha * alpha) * tan2;
  const float root = alpha * cos2 * (1.f + e);
  const float D = kInvPi / (root * root);
  return valid ? D : 0.f;
}
TRN_HD float smith_G(const F3& v, const F3& wh, float alpha) {
  const float tan2 = tan_theta2(wh);
  const bool valid = tan2 < 3.402823466e+38f;
  const float root = alpha * alpha * tan2;
  float G = 2.f / (1.f + sqrtf(1.f + root * root));
  G = valid ? G : 0.f;
  G = tan2 == 0.f ? 1.f : G;
  G = (dot(v, wh) * v.z) <= 0.f ? 0.f : G;
  return G;
}
TRN_HD float ggx_vndf_pdf(const F3& v, const F3& wh, float alpha) {
  return ggx_D(wh, alpha) * smith_G(v, wh, alpha) * fabsf(dot(v, wh)) / fabsf(v.z);
}
// Sampling::SquareToUniformDiskConcentric, Utils.cpp:97-115
TRN_HD void disk_concentric(float sx, float sy, float& ox, float& oy) {
  const float x = 2.f * sx - 1.f, y = 2.f * sy - 1.f;
  const bool is_zero = x == 0.f && y == 0.f;
  const bool q13 = fabsf(x) < fabsf(y);
  const float r = q13 ? y : x;
  const float rp = q13 ? x : y;
  const float phi_ = 0.25f * kPi * rp / r;
  const float phi = is_zero ? 0.f : (q13 ? 0.5f * kPi - phi_ : phi_);
  float sp, cp;
  sincos_det(phi, sp, cp);
  ox = r * cp;
  oy = r * sp;
}
// BSDF::GGX_VNDF_Sample / SampleVisible11, BSDF.cpp:272-302
TRN_HD F3 ggx_vndf_sample(const F3& v, float alpha, float s0, float s1) {
  const F3 V = normalize(F3(v.x * alpha, v.y * alpha, v.z));
  const float sinT = sqrtf(fmaxf(1.f - V.z * V.z, 0.f));
  const float sin_phi = sinT == 0.f ? 0.f : fminf(fmaxf(V.y / sinT, -1.f), 1.f);
  const float cos_phi = sinT == 0.f ? 1.f : fminf(fmaxf(V.x / sinT, -1.f), 1.f);
  const float cos_theta = V.z;
  float px, py; disk_concentric(s0, s1, px, py);
  const float s = 0.5f * (1.f + cos_theta);
  const float x = px;
  const float a = sqrtf(fmaxf(1.f - x * x, 0.f));
  const float y = (1.f - s) * a + s * py;
  const float z = sqrtf(fmaxf(1.f - (px * px + py * py), 0.f));
  const float sin_theta = sqrtf(fmaxf(1.f - cos_theta * cos_theta, 0.f));
  const float norm = 1.f / (sin_theta * y + cos_theta * z);
  const float slx = (cos_theta * y - sin_theta * z) * norm;
  const float sly = x * norm;
  const float slope_x = (cos_phi * slx - sin_phi * sly) * alpha;
  const float slope_y = (sin_phi * slx + cos_phi * sly) * alpha;
  return normalize(F3(-slope_x, -slope_y, 1.f));
}

// BSDF::Pdf -> Diffuse::PdfInner (Diffuse.cpp:78-84) /
// Microfacet::PdfInner (Microfacet.cpp:150-164). Detached values only.
TRN_HD float bsdf_pdf_local(const BsdfDesc& b, const F3& wo, const F3& wi) {
  if (b.type == kDiffuse) {
    const bool reflect = wo.z > 0.f && wo.z * wi.z > 0.f;
    return reflect ? fabsf(wi.z) / kPi : 0.f;
  }
  const float r = b.roughness;
  const F3 wh = normalize(wo + wi);
  const float mp = ggx_vndf_pdf(wo, wh, r);
  const float dwh_dwi = 1.f / (4.f * dot(wi, wh));
  const float pdf = fabsf(mp * dwh_dwi);
  const bool reflect = wo.z > 0.f && mp != 0.f && wi.z > 0.f;
  return reflect ? pdf : 0.f;
}

// Sampling::CosineSampleHemisphere, Utils.cpp:70-95
TRN_HD F3 cosine_hemisphere(float s0, float s1) {
  const float r1 = 2.f * s0 - 1.f, r2 = 2.f * s1 - 1.f;
  const bool cond = (r1 * r1) > (r2 * r2);
  const float r = cond ? r1 : r2;
  const float phi = cond ? kPiOver4 * (r2 / r1) : kPiOver2 - (r1 / r2) * kPiOver4;
  const bool zero = r1 == 0.f && r2 == 0.f;
  const float rr = zero ? 0.f : r, pp = zero ? 0.f : phi;
  float sp, cp;
  sincos_det(pp, sp, cp);
  const float x = rr * cp, y = rr * sp;
  const float z = sqrtf(fmaxf(1e-4f, 1.f - x * x - y * y));
  return F3(x, y, z);
}

// SampleOnly: Diffuse.cpp:61-76, Microfacet.cpp:127-148. Returns world wi and
// the (detached) solid-angle pdf.
TRN_HD void bsdf_sample_only(const BsdfDesc& b, const Frame<float>& f, const F3& wo, float s0, float s1,
                             float s2, F3& wi, float& pdf) {
  (void)s2;
  const F3 lwo = f.to_local(wo);
  if (b.type == kDiffuse) {
    const F3 lwi = cosine_hemisphere(s0, s1);
    wi = f.to_world(lwi);
    pdf = bsdf_pdf_local(b, lwo, lwi);
    return;
  }
  const float r = b.roughness;
  bool reflect = lwo.z > 0.f;
  const F3 wh = ggx_vndf_sample(lwo, r, s0, s1);
  const float mp = ggx_vndf_pdf(lwo, wh, r);
  // VectorReflect(-wo, wh) = -wo + 2 dot(wo, wh) wh (Tensor.cpp:848-851)
  const F3 nwo = -lwo;
  const float d = dot(-nwo, wh);
  const F3 lwi = nwo + wh * (2.f * d);
  reflect = reflect && mp != 0.f && lwi.z > 0.f;
  const float dwh_dwi = 1.f / (4.f * dot(lwi, wh));
  const float p = fabsf(mp * dwh_dwi);
  pdf = reflect ? p : 0.f;
  wi = f.to_world(lwi);
}

// OutDirValid: Diffuse.cpp:43-48 (strict, EDGE_EPSILON) and the BSDF default
// (BSDF.h: sign agreement of shading and geometric cosines).
TRN_HD bool out_dir_valid(const BsdfDesc& b, const F3& ns, const F3& ng, const F3& w) {
  const float ds = dot(ns, w), dg = dot(ng, w);
  if (b.type == kDiffuse) return ds > kEdgeEps && dg > kEdgeEps;
  return ds * dg > 0.f;
}

// ---- merged area light (AreaLight, Light.cpp:134-184) ---------------------
struct LightSample {
  int tri;       // global triangle id of the sampled emitter triangle
  float bu, bv;  // barycentrics of the point (u weights P1, v weights P2)
  float pdf;     // pdf / Detach(area) (detached value)
  int light;     // light id (radiance index)
};

// Distribution1D::SampleDiscrete (Distribution.cu:37-48, upper bound with
// LessEQ = first index with cdf >= u) and ReuseSample (Distribution.cpp:37-43).
TRN_HD int sample_discrete(const float* cdf, int n, float u, float& reuse) {
  int lo = 0, count = n;
  while (count > 0) {
    int step = count / 2;
    int mid = lo + step;
    if (!(u <= cdf[mid])) { lo = mid + 1; count -= step + 1; } else { count = step; }
  }
  int idx = lo < 0 ? 0 : (lo > n - 1 ? n - 1 : lo);
  const float pmin = idx > 0 ? cdf[idx - 1] : 0.f;
  const float pmax = cdf[idx];
  reuse = (u - pmin) / (pmax - pmin);
  return idx;
}

TRN_D bool light_sample(const DeviceScene& s, float s0, float s1, LightSample& ls) {
  if (s.n_emit <= 0) return false;
  float reuse;
  const int e = sample_discrete(s.light_cdf, s.n_emit, s0, reuse);
  const float pmf = s.light_func[e] / (__ldg(s.light_integral) * (float)s.n_emit);
  const float t = sqrtf(reuse);
  ls.bu = 1.f - t;
  ls.bv = t * s1;
  ls.tri = s.emit_tris[e];
  ls.pdf = pmf / s.area[ls.tri];
  ls.light = s.emitter_id[ls.tri];
  return true;
}

// AreaLight::Pdf (Light.cpp:176-183), detached
TRN_D float light_pdf(const DeviceScene& s, int tri) {
  const int e = s.tri_to_emit[tri];
  if (e < 0) return 0.f;
  const float pmf = s.light_func[e] / (__ldg(s.light_integral) * (float)s.n_emit);
  return pmf / s.area[tri];
}

TRN_D F3 light_radiance(const DeviceScene& s, int light) { return load3(s.light_radiance, light); }

// ---- pinhole sensor ---------------------------------------------------------
TRN_HD F3 xform_point(const float* m, const F3& p) {
  const float x = m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3];
  const float y = m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7];
  const float z = m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11];
  const float w = m[12] * p.x + m[13] * p.y + m[14] * p.z + m[15];
  return F3(x / w, y / w, z / w);
}
TRN_HD F3 xform_vector(const float* m, const F3& v) {
  return F3(m[0] * v.x + m[1] * v.y + m[2] * v.z, m[4] * v.x + m[5] * v.y + m[6] * v.z,
            m[8] * v.x + m[9] * v.y + m[10] * v.z);
}

// Camera::GenerateAntitheticRays with the box filter (Camera.cpp:224-277):
// raster point (px + sx, py + sy), camera-space point by the homogeneous
// raster->camera transform, normalised, rotated by the inverse view matrix.
// Explicitly rounded so it is bit-identical to the CPU restatement.
TRN_D F3 camera_ray_dir(const CameraDesc& c, int ix, int iy, float sx, float sy) {
  const float* m = c.raster_to_camera;
  const float rx = __fadd_rn((float)ix, sx), ry = __fadd_rn((float)iy, sy);
  // Dot(mat, (rx, ry, 0, 1))
  auto row = [&](int r) {
    return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[4 * r], rx), __fmul_rn(m[4 * r + 1], ry)),
                               __fmul_rn(m[4 * r + 2], 0.f)), m[4 * r + 3]);
  };
  const float hx = row(0), hy = row(1), hz = row(2), hw = row(3);
  const float cx = __fdiv_rn(hx, hw), cy = __fdiv_rn(hy, hw), cz = __fdiv_rn(hz, hw);
  const float len = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(cx, cx), __fmul_rn(cy, cy)), __fmul_rn(cz, cz)));
  const float dx = __fdiv_rn(cx, len), dy = __fdiv_rn(cy, len), dz = __fdiv_rn(cz, len);
  const float* v = c.view_inv;
  auto vrow = [&](int r) {
    return __fadd_rn(__fadd_rn(__fmul_rn(v[4 * r], dx), __fmul_rn(v[4 * r + 1], dy)), __fmul_rn(v[4 * r + 2], dz));
  };
  return F3(vrow(0), vrow(1), vrow(2));
}

// Camera::EvalFilter with USE_BOX_FILTER (Camera.cpp:279-303) times the
// intersection's J = A / Detach(A) (PathTracer.cpp:49).
template <class S>
TRN_HD S camera_factor(const CameraDesc& c, const V3<S>& p, const V3<S>& ng, const S& J) {
  V3<S> dir = p - lift<S>(F3(c.pos[0], c.pos[1], c.pos[2]));
  const S dist = length(dir);
  dir = dir / dist;
  const S cosy = dot(dir, lift<S>(F3(c.dir[0], c.dir[1], c.dir[2])));
  const S cosx = dot(-dir, ng);
  const S G = abs_(cosx) / (cosy * cosy * cosy * (dist * dist));
  return G / detach(G) * J;
}

// Camera::sampleDirect (Camera.cpp:399-416)
struct SensorSample {
  float qx, qy;
  bool valid;
  int pixel;
  float sensor_val;
};
TRN_HD SensorSample sample_direct(const CameraDesc& c, const F3& p) {
  SensorSample r;
  const F3 q = xform_point(c.world_to_sample, p);
  r.qx = q.x; r.qy = q.y;
  r.valid = q.x >= 0.f && q.x < 1.f && q.y >= 0.f && q.y < 1.f;
  r.pixel = (int)floorf(q.y * (float)c.h) * c.w + (int)floorf(q.x * (float)c.w);
  F3 dir = p - F3(c.pos[0], c.pos[1], c.pos[2]);
  const float dist2 = dot(dir, dir);
  dir = dir / sqrtf(dist2);
  const float cosT = dot(F3(c.dir[0], c.dir[1], c.dir[2]), dir);
  const float ic = 1.f / cosT;
  r.sensor_val = 1.f / dist2 * ic * ic * ic * c.inv_area;
  return r;
}
// Camera::GenerateBoundaryRays(sds, ray) direction (Camera.cpp:379-397)
TRN_HD F3 sensor_ray_dir(const CameraDesc& c, float qx, float qy) {
  const F3 cc = xform_point(c.sample_to_camera, F3(qx, qy, 0.f));
  return xform_vector(c.view_inv, normalize(cc));
}
// Camera::WriteToImage with the box filter (Camera.cpp:418-431): the pixel a
// sensor coordinate lands on, or -1.
TRN_HD int image_pixel(const CameraDesc& c, float qx, float qy) {
  const float px = qx * (float)c.w, py = qy * (float)c.h;
  const float fx = floorf(px), fy = floorf(py);
  if (!(fx >= 0.f && fx < (float)c.w && fy >= 0.f && fy < (float)c.h)) return -1;
  return (int)fy * c.w + (int)fx;
}

}  // namespace trn
