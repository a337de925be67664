// Host-side check of the hand-written reverse-mode adjoints against
// forward-mode dual numbers of the same factor code (test infrastructure).
// Prints one line per check: "<name> <cases> <worst relative L2 error>".
#include "../../tensorray_b200/csrc/render.cu"
#include <cmath>
#include <cstdio>
#include <random>
#include <string>
#include <vector>
using namespace trn;

namespace {

using D3 = Dual<3>;

F3 contract3(const V3<D3>& r, const F3& adj) {
  F3 g;
  for (int i = 0; i < 3; i++) g[i] = adj.x * r.x.d[i] + adj.y * r.y.d[i] + adj.z * r.z.d[i];
  return g;
}

// forward-mode gradients of the NEE / continuation factors w.r.t. the six
// vector inputs and J, in groups of three lanes
void dual_factor(bool nee, const BsdfDesc& b, const F3& xprev, const F3& x, const F3& ns, const F3& ng, const F3& kd,
                 const F3& z, const F3& nz, const F3& Le, float lpdf, float mis, float pp, const F3& adj, F3 g[6],
                 float& gJ) {
  for (int grp = 0; grp < 7; grp++) {
    const V3<D3> a_prev = seed3<3>(xprev, grp == 0 ? 0 : -1);
    const V3<D3> a_x = seed3<3>(x, grp == 1 ? 0 : -1);
    const V3<D3> a_ns = seed3<3>(ns, grp == 2 ? 0 : -1);
    const V3<D3> a_kd = seed3<3>(kd, grp == 3 ? 0 : -1);
    const V3<D3> a_z = seed3<3>(z, grp == 4 ? 0 : -1);
    const V3<D3> a_nz = seed3<3>(nz, grp == 5 ? 0 : -1);
    const D3 a_J = seed1<3>(1.f, grp == 6 ? 0 : -1);
    const V3<D3> r = nee ? nee_factor<D3>(b, a_prev, a_x, a_ns, lift<D3>(ng), a_kd, a_z, a_nz, a_J, Le, lpdf, mis)
                         : cont_factor<D3>(b, a_prev, a_x, a_ns, lift<D3>(ng), a_kd, a_z, a_nz, a_J, pp);
    const F3 gg = contract3(r, adj);
    if (grp < 6) g[grp] = gg; else gJ = gg.x;
  }
}

double rel(const double* a, const double* b, int n) {
  double num = 0, den = 0;
  for (int i = 0; i < n; i++) { num += (a[i] - b[i]) * (a[i] - b[i]); den += b[i] * b[i]; }
  return den > 0 ? std::sqrt(num / den) : (num > 0 ? 1.0 : 0.0);
}

}  // namespace

// File-driven modes: int32 n, `header_bytes` of header (copied to `header`),
// then n records of in_w float32; writes n records of out_w float32 that
// `body(in, out)` fills.
template <class Body>
int run_records(const char* in_path, const char* out_path, int in_w, int out_w, void* header, size_t header_bytes,
                Body&& body) {
  FILE* fi = std::fopen(in_path, "rb");
  if (!fi) return 1;
  int n = 0;
  if (std::fread(&n, sizeof n, 1, fi) != 1 || n < 0) return 1;
  if (header_bytes && std::fread(header, header_bytes, 1, fi) != 1) return 1;
  std::vector<float> in((size_t)n * in_w), out((size_t)n * out_w, 0.f);
  if (std::fread(in.data(), sizeof(float), in.size(), fi) != in.size()) return 1;
  std::fclose(fi);
  for (int i = 0; i < n; i++) body(&in[(size_t)i * in_w], &out[(size_t)i * out_w]);
  FILE* fo = std::fopen(out_path, "wb");
  if (!fo) return 1;
  std::fwrite(out.data(), sizeof(float), out.size(), fo);
  std::fclose(fo);
  return 0;
}

BsdfDesc bsdf_of(const float* c) {
  BsdfDesc b{};
  b.type = (int)c[0];
  b.tex = -1;
  b.roughness = c[1];
  for (int k = 0; k < 3; k++) b.spec[k] = c[2 + k];
  return b;
}

// Mode "eval_inner_vjp IN OUT": records of 17 float32 (type, roughness,
// spec[3], kd[3], lo[3], li[3], gB[3]) in; 12 float32 (B[3], g_lo[3], g_li[3],
// g_kd[3]) out.
int run_eval_inner_vjp(const char* in_path, const char* out_path) {
  return run_records(in_path, out_path, 17, 12, nullptr, 0, [](const float* c, float* o) {
    const BsdfDesc b = bsdf_of(c);
    const F3 kd(c[5], c[6], c[7]), lo(c[8], c[9], c[10]), li(c[11], c[12], c[13]), gB(c[14], c[15], c[16]);
    F3 g_lo = F3z(), g_li = F3z(), g_kd = F3z();
    const F3 r[4] = {eval_inner_vjp(b, kd, lo, li, gB, g_lo, g_li, g_kd), g_lo, g_li, g_kd};
    for (int j = 0; j < 4; j++)
      for (int k = 0; k < 3; k++) o[3 * j + k] = r[j][k];
  });
}

// Mode "xdotn_grad IN OUT": records of 19 float32 (org[3], target[3], P0[3],
// P1[3], P2[3], n[3], W) in; 16 float32 (xdotn, g_org[3], g_target[3], g0[3],
// g1[3], g2[3]) out.
int run_xdotn_grad(const char* in_path, const char* out_path) {
  return run_records(in_path, out_path, 19, 16, nullptr, 0, [](const float* c, float* o) {
    const F3 org(c[0], c[1], c[2]), target(c[3], c[4], c[5]), P0(c[6], c[7], c[8]), P1(c[9], c[10], c[11]),
        P2(c[12], c[13], c[14]), nn(c[15], c[16], c[17]);
    F3 g[5];
    xdotn_grad(org, target, P0, P1, P2, nn, c[18], g[0], g[1], g[2], g[3], g[4]);
    o[0] = xdotn<float>(org, target, P0, P1, P2, nn);
    for (int j = 0; j < 5; j++)
      for (int k = 0; k < 3; k++) o[1 + 3 * j + k] = g[j][k];
  });
}

// Mode "camera_factor_grad IN OUT": the CameraDesc bytes after n, then
// records of 7 float32 (p[3], ng[3], W) in; 7 float32 (g_p[3], g_ng[3], g_J)
// out.
int run_camera_factor_grad(const char* in_path, const char* out_path) {
  CameraDesc cam;
  return run_records(in_path, out_path, 7, 7, &cam, sizeof cam, [&cam](const float* c, float* o) {
    F3 g_p, g_ng;
    float g_J = 0.f;
    camera_factor_grad(cam, F3(c[0], c[1], c[2]), F3(c[3], c[4], c[5]), c[6], g_p, g_ng, g_J);
    o[0] = g_p.x; o[1] = g_p.y; o[2] = g_p.z; o[3] = g_ng.x; o[4] = g_ng.y; o[5] = g_ng.z; o[6] = g_J;
  });
}

// Mode "factor_vjp IN OUT": records of 30 float32 (type, roughness, spec[3],
// xprev[3], x[3], ns[3], kd[3], z[3], nz[3], J, K[3], adj[3]) in; 22 float32
// (F[3], g_prev[3], g_x[3], g_ns[3], g_kd[3], g_z[3], g_nz[3], g_J) out.
int run_factor_vjp(const char* in_path, const char* out_path) {
  return run_records(in_path, out_path, 30, 22, nullptr, 0, [](const float* c, float* o) {
    const BsdfDesc b = bsdf_of(c);
    auto v3 = [&](int k) { return F3(c[k], c[k + 1], c[k + 2]); };
    F3 g[6] = {F3z(), F3z(), F3z(), F3z(), F3z(), F3z()};
    float gJ = 0.f;
    const F3 F = factor_vjp(b, true, true, v3(5), v3(8), v3(11), v3(14), v3(17), v3(20), c[23], v3(24), v3(27),
                            g[0], g[1], g[2], g[3], g[4], g[5], gJ);
    o[0] = F.x; o[1] = F.y; o[2] = F.z;
    for (int j = 0; j < 6; j++)
      for (int k = 0; k < 3; k++) o[3 + 3 * j + k] = g[j][k];
    o[21] = gJ;
  });
}

int main(int argc, char** argv) {
  if (argc == 4 && std::string(argv[1]) == "eval_inner_vjp") return run_eval_inner_vjp(argv[2], argv[3]);
  if (argc == 4 && std::string(argv[1]) == "factor_vjp") return run_factor_vjp(argv[2], argv[3]);
  if (argc == 4 && std::string(argv[1]) == "camera_factor_grad") return run_camera_factor_grad(argv[2], argv[3]);
  if (argc == 4 && std::string(argv[1]) == "xdotn_grad") return run_xdotn_grad(argv[2], argv[3]);
  std::mt19937 rng(1);
  std::uniform_real_distribution<float> U(-1.f, 1.f);
  auto rv = [&]() { return F3(U(rng), U(rng), U(rng)); };
  // NEE and continuation factors: diffuse and GGX, both coordinate_system
  // branches, unnormalised shading normals; values and gradients
  double worst = 0, worst_val = 0;
  int n = 0;
  for (int it = 0; it < 20000; it++) {
    BsdfDesc b{};
    b.type = (it % 3 == 0) ? kDiffuse : 1;
    b.roughness = 0.1f + 0.8f * std::fabs(U(rng));
    b.spec[0] = 0.04f; b.spec[1] = 0.05f; b.spec[2] = 0.5f;
    F3 ns = normalize(F3(0.f, 1.f, 0.f) + rv() * 0.6f) * (0.9f + 0.1f * std::fabs(U(rng)));
    if (it % 5 == 1) ns = normalize(F3(1.f, 0.2f, 0.1f) + rv() * 0.3f) * 0.97f;
    const F3 ng = normalize(ns + rv() * 0.05f);
    const F3 x = rv();
    const F3 xprev = x + normalize(ns + rv() * 0.8f) * (1.f + std::fabs(U(rng)));
    const F3 z = x + normalize(ns + rv() * 0.8f) * (0.5f + 2.f * std::fabs(U(rng)));
    const F3 nz = normalize(rv());
    const F3 kd(0.3f, 0.5f, 0.7f), Le(10.f, 9.f, 8.f), adj = rv();
    const bool nee = it & 1;
    F3 gd[6]; float gJd = 0;
    dual_factor(nee, b, xprev, x, ns, ng, kd, z, nz, Le, 0.7f, 0.6f, 0.8f, adj, gd, gJd);
    F3 gh[6] = {F3z(), F3z(), F3z(), F3z(), F3z(), F3z()};
    float gJh = 0;
    F3 Fh, Fd;
    if (nee) {
      Fh = nee_vjp(b, true, true, xprev, x, ns, ng, kd, z, nz, Le, 0.7f, 0.6f, adj, gh[0], gh[1], gh[2], gh[3], gh[4],
                   gh[5], gJh);
      Fd = nee_factor<float>(b, xprev, x, ns, ng, kd, z, nz, 1.f, Le, 0.7f, 0.6f);
    } else {
      Fh = cont_vjp(b, true, true, xprev, x, ns, ng, kd, z, nz, 0.8f, adj, gh[0], gh[1], gh[2], gh[3], gh[4], gh[5],
                    gJh);
      Fd = cont_factor<float>(b, xprev, x, ns, ng, kd, z, nz, 1.f, 0.8f);
    }
    double a[19], r[19], fa[3], fr[3];
    for (int i = 0; i < 6; i++) for (int c = 0; c < 3; c++) { a[3 * i + c] = gh[i][c]; r[3 * i + c] = gd[i][c]; }
    a[18] = gJh; r[18] = gJd;
    for (int c = 0; c < 3; c++) { fa[c] = Fh[c]; fr[c] = Fd[c]; }
    double den = 0;
    for (int i = 0; i < 19; i++) den += r[i] * r[i];
    if (den == 0) continue;
    n++;
    worst = std::fmax(worst, rel(a, r, 19));
    worst_val = std::fmax(worst_val, rel(fa, fr, 3));
  }
  std::printf("factor_vjp %d %.3e\n", n, worst);
  std::printf("factor_value %d %.3e\n", n, worst_val);
  // xDotN (RayIntersectAD): gradients w.r.t. origin, target and the vertices
  worst = 0; n = 0;
  for (int it = 0; it < 20000; it++) {
    const F3 P0 = rv(), P1 = P0 + rv(), P2 = P0 + rv();
    const F3 c = (P0 + P1 + P2) * (1.f / 3.f);
    const F3 org = c + rv() * 3.f + F3(0.f, 3.f, 0.f);
    const F3 target = c + (P1 - P0) * (0.3f * U(rng)) + rv() * 0.1f;
    const F3 nn = normalize(rv());
    const float W = U(rng);
    double a[15], r[15];
    for (int grp = 0; grp < 5; grp++) {
      const V3<D3> o = seed3<3>(org, grp == 0 ? 0 : -1), t = seed3<3>(target, grp == 1 ? 0 : -1);
      const V3<D3> q0 = seed3<3>(P0, grp == 2 ? 0 : -1), q1 = seed3<3>(P1, grp == 3 ? 0 : -1),
                   q2 = seed3<3>(P2, grp == 4 ? 0 : -1);
      const D3 d = xdotn<D3>(o, t, q0, q1, q2, nn);
      for (int k = 0; k < 3; k++) r[3 * grp + k] = d.d[k] * W;
    }
    F3 g[5];
    xdotn_grad(org, target, P0, P1, P2, nn, W, g[0], g[1], g[2], g[3], g[4]);
    for (int i = 0; i < 5; i++) for (int k = 0; k < 3; k++) a[3 * i + k] = g[i][k];
    double den = 0;
    for (int i = 0; i < 15; i++) den += r[i] * r[i];
    if (den == 0) continue;
    n++;
    worst = std::fmax(worst, rel(a, r, 15));
  }
  std::printf("xdotn_grad %d %.3e\n", n, worst);
  // camera factor G / Detach(G) * J
  worst = 0; n = 0;
  for (int it = 0; it < 20000; it++) {
    CameraDesc cam{};
    cam.pos[0] = 0; cam.pos[1] = 0.5f * U(rng); cam.pos[2] = 4.f;
    cam.dir[0] = 0; cam.dir[1] = 0; cam.dir[2] = -1.f;
    const F3 p = rv() * 0.9f;
    const F3 ng = normalize(F3(0.f, 0.f, 1.f) + rv() * 0.7f);
    const float W = U(rng);
    double a[7], r[7];
    for (int grp = 0; grp < 3; grp++) {
      const V3<D3> dx = seed3<3>(p, grp == 0 ? 0 : -1);
      const V3<D3> dn = seed3<3>(ng, grp == 1 ? 0 : -1);
      const D3 dJ = seed1<3>(1.f, grp == 2 ? 0 : -1);
      const D3 d = camera_factor<D3>(cam, dx, dn, dJ);
      if (grp < 2) for (int k = 0; k < 3; k++) r[3 * grp + k] = d.d[k] * W;
      else r[6] = d.d[0] * W;
    }
    F3 gp, gn;
    float gJ;
    camera_factor_grad(cam, p, ng, W, gp, gn, gJ);
    for (int k = 0; k < 3; k++) { a[k] = gp[k]; a[3 + k] = gn[k]; }
    a[6] = gJ;
    n++;
    worst = std::fmax(worst, rel(a, r, 7));
  }
  std::printf("camera_factor_grad %d %.3e\n", n, worst);
  return 0;
}
