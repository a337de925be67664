// Host build of the library's shading and camera functions (test
// infrastructure). Reads cases from a file and writes the library's values
// to another, for the comparison with the oracle's restatements in
// tests/test_shading_host.py.
//
// Input: int32 n, then n records of kIn float32:
//   type, roughness, spec[3], kd[3], wo[3], wi[3], s0, s1, n[3], ng[3]
// Output: n records of kOut float32:
//   eval_inner[3], bsdf_pdf_local, cosine_hemisphere[3], disk_concentric[2],
//   ggx_vndf_sample[3] (zeros when wo.z <= 0), coordinate_system t[3], b[3],
//   out_dir_valid (0 or 1)
#include "../../tensorray_b200/csrc/shading.cuh"

#include <cstdio>
#include <string>
#include <vector>

using namespace trn;

namespace {
constexpr int kIn = 22;
constexpr int kOut = 19;
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

// Mode "camera IN OUT": the CameraDesc bytes (the library's trn_camera, same
// layout) after n, then records of 9 float32 (p[3], ng[3], J, qx, qy) in; 10
// float32 out: sample_direct (qx, qy, valid, pixel, sensor_val),
// sensor_ray_dir[3], image_pixel, camera_factor.
int run_camera(const char* in_path, const char* out_path) {
  CameraDesc cam;
  return run_records(in_path, out_path, 9, 10, &cam, sizeof cam, [&cam](const float* c, float* o) {
    const F3 p(c[0], c[1], c[2]), ng(c[3], c[4], c[5]);
    const SensorSample sd = sample_direct(cam, p);
    o[0] = sd.qx; o[1] = sd.qy; o[2] = sd.valid ? 1.f : 0.f; o[3] = (float)sd.pixel; o[4] = sd.sensor_val;
    const F3 d = sensor_ray_dir(cam, c[7], c[8]);
    o[5] = d.x; o[6] = d.y; o[7] = d.z;
    o[8] = (float)image_pixel(cam, c[7], c[8]);
    o[9] = camera_factor<float>(cam, p, ng, c[6]);
  });
}

// Mode "IN OUT" (no name): the shading records described at the top.
int run_shading(const char* in_path, const char* out_path) {
  return run_records(in_path, out_path, kIn, kOut, nullptr, 0, [](const float* c, float* o) {
    BsdfDesc b{};
    b.type = (int)c[0];
    b.tex = -1;
    b.roughness = c[1];
    for (int k = 0; k < 3; k++) b.spec[k] = c[2 + k];
    const F3 kd(c[5], c[6], c[7]), wo(c[8], c[9], c[10]), wi(c[11], c[12], c[13]);
    const float s0 = c[14], s1 = c[15];
    const F3 nn(c[16], c[17], c[18]), ng(c[19], c[20], c[21]);
    const F3 e = eval_inner<float>(b, kd, wo, wi);
    o[0] = e.x; o[1] = e.y; o[2] = e.z;
    o[3] = bsdf_pdf_local(b, wo, wi);
    const F3 ch = cosine_hemisphere(s0, s1);
    o[4] = ch.x; o[5] = ch.y; o[6] = ch.z;
    disk_concentric(s0, s1, o[7], o[8]);
    if (wo.z > 0.f) {
      const F3 v = ggx_vndf_sample(wo, b.roughness, s0, s1);
      o[9] = v.x; o[10] = v.y; o[11] = v.z;
    }
    F3 t, bb;
    coordinate_system<float>(nn, t, bb);
    o[12] = t.x; o[13] = t.y; o[14] = t.z;
    o[15] = bb.x; o[16] = bb.y; o[17] = bb.z;
    o[18] = out_dir_valid(b, nn, ng, wi) ? 1.f : 0.f;
  });
}

// Mode "hash IN OUT": int32 n, then n records of 4 uint32 (seed, term, dim,
// slot) in; n float32 hash_uniform values out.
int run_hash(const char* in_path, const char* out_path) {
  FILE* fi = std::fopen(in_path, "rb");
  if (!fi) return 1;
  int n = 0;
  if (std::fread(&n, sizeof n, 1, fi) != 1 || n < 0) return 1;
  std::vector<uint32_t> in((size_t)n * 4);
  std::vector<float> out(n);
  if (std::fread(in.data(), sizeof(uint32_t), in.size(), fi) != in.size()) return 1;
  std::fclose(fi);
  for (int i = 0; i < n; i++) out[i] = hash_uniform(in[4 * i], in[4 * i + 1], in[4 * i + 2], in[4 * i + 3]);
  FILE* fo = std::fopen(out_path, "wb");
  if (!fo) return 1;
  std::fwrite(out.data(), sizeof(float), out.size(), fo);
  std::fclose(fo);
  return 0;
}

// Mode "discrete IN OUT": int32 c, c float32 CDF values, int32 m, m float32
// samples in; m records (int32 index, float32 reused sample) out.
int run_discrete(const char* in_path, const char* out_path) {
  FILE* fi = std::fopen(in_path, "rb");
  if (!fi) return 1;
  int c = 0, m = 0;
  if (std::fread(&c, sizeof c, 1, fi) != 1 || c <= 0) return 1;
  std::vector<float> cdf(c);
  if (std::fread(cdf.data(), sizeof(float), c, fi) != (size_t)c) return 1;
  if (std::fread(&m, sizeof m, 1, fi) != 1 || m < 0) return 1;
  std::vector<float> u(m);
  if (std::fread(u.data(), sizeof(float), m, fi) != (size_t)m) return 1;
  std::fclose(fi);
  FILE* fo = std::fopen(out_path, "wb");
  if (!fo) return 1;
  for (int i = 0; i < m; i++) {
    float reuse = 0.f;
    const int idx = sample_discrete(cdf.data(), c, u[i], reuse);
    std::fwrite(&idx, sizeof idx, 1, fo);
    std::fwrite(&reuse, sizeof reuse, 1, fo);
  }
  std::fclose(fo);
  return 0;
}

int main(int argc, char** argv) {
  if (argc == 4 && std::string(argv[1]) == "camera") return run_camera(argv[2], argv[3]);
  if (argc == 4 && std::string(argv[1]) == "hash") return run_hash(argv[2], argv[3]);
  if (argc == 4 && std::string(argv[1]) == "discrete") return run_discrete(argv[2], argv[3]);
  if (argc == 3) return run_shading(argv[1], argv[2]);
  std::fprintf(stderr, "usage: shading_harness IN OUT | shading_harness camera|hash|discrete IN OUT\n");
  return 2;
}
