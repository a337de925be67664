// Deterministic sampling trigonometry (sincos_det / acos_det, csrc/common.cuh)
// evaluated on the host and, when a GPU is present, on the device, over the
// float32 inputs of a binary file (test infrastructure).
// usage: trig_harness <in.f32> <out_prefix> [device]
// writes <out_prefix>.host.f32 and, with "device", <out_prefix>.dev.f32:
// per input x the triple (sin_det(x), cos_det(x), acos_det(x)), followed in
// the device file by CUDA's (sinf(x), cosf(x), acosf(x)) for an accuracy
// comparison.
#include "../../tensorray_b200/csrc/common.cuh"
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>
using namespace trn;

__global__ void k_trig(int n, const float* x, float* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float s, c;
  sincos_det(x[i], s, c);
  out[3 * i] = s;
  out[3 * i + 1] = c;
  out[3 * i + 2] = acos_det(x[i]);
  out[3 * (n + i)] = sinf(x[i]);
  out[3 * (n + i) + 1] = cosf(x[i]);
  out[3 * (n + i) + 2] = acosf(x[i]);
}

static bool write_all(const char* path, const std::vector<float>& v) {
  FILE* f = fopen(path, "wb");
  if (!f) return false;
  const size_t w = fwrite(v.data(), sizeof(float), v.size(), f);
  fclose(f);
  return w == v.size();
}

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  FILE* f = fopen(argv[1], "rb");
  if (!f) return 2;
  std::vector<float> x;
  float buf[4096];
  size_t r;
  while ((r = fread(buf, sizeof(float), 4096, f)) > 0) x.insert(x.end(), buf, buf + r);
  fclose(f);
  const int n = (int)x.size();
  std::vector<float> host(3 * (size_t)n);
  for (int i = 0; i < n; i++) {
    float s, c;
    sincos_det(x[i], s, c);
    host[3 * i] = s;
    host[3 * i + 1] = c;
    host[3 * i + 2] = acos_det(x[i]);
  }
  std::string p = std::string(argv[2]) + ".host.f32";
  if (!write_all(p.c_str(), host)) return 3;
  if (argc > 3 && std::string(argv[3]) == "device") {
    float *dx = nullptr, *dout = nullptr;
    if (cudaMalloc(&dx, sizeof(float) * n) != cudaSuccess) return 4;
    if (cudaMalloc(&dout, sizeof(float) * 6 * (size_t)n) != cudaSuccess) return 4;
    cudaMemcpy(dx, x.data(), sizeof(float) * n, cudaMemcpyHostToDevice);
    k_trig<<<(n + 255) / 256, 256>>>(n, dx, dout);
    std::vector<float> dev(6 * (size_t)n);
    if (cudaMemcpy(dev.data(), dout, sizeof(float) * 6 * n, cudaMemcpyDeviceToHost) != cudaSuccess) return 5;
    cudaFree(dx);
    cudaFree(dout);
    p = std::string(argv[2]) + ".dev.f32";
    if (!write_all(p.c_str(), dev)) return 3;
  }
  return 0;
}
