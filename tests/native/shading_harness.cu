// Host build of the library's shading functions (test infrastructure). Reads
// cases from argv[1] and writes the library's values to argv[2], for the
// comparison with the oracle's restatements in tests/test_shading_host.py.
//
// Input: int32 n, then n records of kIn float32:
//   type, roughness, spec[3], kd[3], wo[3], wi[3], s0, s1, n[3], ng[3]
// Output: n records of kOut float32:
//   eval_inner[3], bsdf_pdf_local, cosine_hemisphere[3], disk_concentric[2],
//   ggx_vndf_sample[3] (zeros when wo.z <= 0), coordinate_system t[3], b[3],
//   out_dir_valid (0 or 1)
#include "../../tensorray_b200/csrc/shading.cuh"

#include <cstdio>
#include <vector>

using namespace trn;

namespace {
constexpr int kIn = 22;
constexpr int kOut = 19;
}  // namespace

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: shading_harness IN OUT\n");
    return 2;
  }
  FILE* fi = std::fopen(argv[1], "rb");
  if (!fi) return 1;
  int n = 0;
  if (std::fread(&n, sizeof n, 1, fi) != 1 || n < 0) return 1;
  std::vector<float> in((size_t)n * kIn), out((size_t)n * kOut, 0.f);
  if (std::fread(in.data(), sizeof(float), in.size(), fi) != in.size()) return 1;
  std::fclose(fi);
  for (int i = 0; i < n; i++) {
    const float* c = &in[(size_t)i * kIn];
    float* o = &out[(size_t)i * kOut];
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
  }
  FILE* fo = std::fopen(argv[2], "wb");
  if (!fo) return 1;
  std::fwrite(out.data(), sizeof(float), out.size(), fo);
  std::fclose(fo);
  return 0;
}
