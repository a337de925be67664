// Reference probe (test infrastructure, never part of the product). It runs
// the reference's own EDXUtil code, compiled from the reference's sources by
// oracle/edx/Makefile, on the inputs given on the command line and prints the
// results as one JSON object. Every float is printed as its IEEE-754 bit
// pattern (an unsigned 32-bit integer), so the comparison is exact.
//
//   edx_probe obj FILE
//     ObjMesh::LoadFromObj(FILE, makeLeftHanded = false), the call every
//     reference Primitive makes (Renderer/Primitive.cpp:213-245), then what
//     TriangleMesh::LoadRawBuffer reads from it (Primitive.cpp:39-110): the
//     position and texture-coordinate buffers, the faces' position and
//     texture indices, and the edge lists processEdges built
//     (EDXUtil/Graphics/ObjMesh.cpp:584-632).
//
//   edx_probe bitmap FILE
//     Bitmap::ReadFromFile<float>(FILE, ..., 3), the call the renderer's
//     ImageTexture makes (Renderer/BSDF.cpp:57-70). That function is one call
//     of stbi_loadf with 3 required channels (EDXUtil/Windows/Bitmap.cpp:
//     187-190) into the stb_image the reference compiles inside Bitmap.cpp
//     (stb_image.h v2.02 with STB_IMAGE_IMPLEMENTATION, in C++), which is what
//     this file compiles too.
//
//   edx_probe camera PX PY PZ TX TY TZ UX UY UZ W H FOV
//     EDX::Camera::Init (EDXUtil/Graphics/BaseCamera.cpp:45-88) with the
//     clip planes of the renderer's Camera::Init (Renderer/Camera.cpp:89-103),
//     then the quantities the renderer's Camera::Resize derives from it
//     (Renderer/Camera.cpp:105-137). The derivation calls the same EDX::Matrix
//     and EDX::Math functions, in the same order and precision, as that
//     method: it is restated here because Renderer/Camera.cpp itself needs the
//     reference's tensor library.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "Graphics/BaseCamera.h"
#include "Graphics/ObjMesh.h"

#define STB_IMAGE_IMPLEMENTATION
#include "Windows/stb_image.h"

namespace {

unsigned bits(float f) {
  unsigned u;
  std::memcpy(&u, &f, sizeof u);
  return u;
}

void put_floats(const char* key, const float* v, size_t n, bool last = false) {
  std::printf("\"%s\": [", key);
  for (size_t i = 0; i < n; i++) std::printf(i ? ",%u" : "%u", bits(v[i]));
  std::printf("]%s\n", last ? "" : ",");
}

void put_ints(const char* key, const std::vector<int>& v, bool last = false) {
  std::printf("\"%s\": [", key);
  for (size_t i = 0; i < v.size(); i++) std::printf(i ? ",%d" : "%d", v[i]);
  std::printf("]%s\n", last ? "" : ",");
}

void put_matrix(const char* key, const EDX::Matrix& m, bool last = false) {
  put_floats(key, &m.m[0][0], 16, last);
}

int probe_obj(const char* path) {
  EDX::ObjMesh mesh;
  if (!mesh.LoadFromObj(path, false)) {
    std::fprintf(stderr, "edx_probe: LoadFromObj failed on %s\n", path);
    return 1;
  }
  const int nt = (int)mesh.GetTriangleCount();
  std::vector<float> pos, tex;
  for (const auto& p : mesh.GetVertexPositionBuf()) { pos.push_back(p.x); pos.push_back(p.y); pos.push_back(p.z); }
  for (const auto& t : mesh.GetVertexTextureBuf()) { tex.push_back(t.x); tex.push_back(t.y); }
  std::vector<int> fpos, ftex;
  for (int i = 0; i < nt; i++) {
    const EDX::MeshFace& f = mesh.GetFaceAt(i);
    for (int j = 0; j < 3; j++) {
      fpos.push_back(f.posIndices[j]);
      ftex.push_back(mesh.IsTextured() ? f.texIndices[j] : 0);
    }
  }
  const EDX::EdgeList& e = mesh.getEdgeList();
  std::printf("{\n\"vertex_count\": %u,\n\"triangle_count\": %d,\n\"textured\": %s,\n", mesh.GetVertexCount(), nt,
              mesh.IsTextured() ? "true" : "false");
  put_floats("positions", pos.data(), pos.size());
  put_floats("texcoords", tex.data(), tex.size());
  put_ints("face_positions", fpos);
  put_ints("face_texcoords", ftex);
  std::printf("\"num_edges\": %d,\n", e.numEdges);
  put_ints("edge_vertex0", e.indexVertex0);
  put_ints("edge_vertex1", e.indexVertex1);
  put_ints("edge_face0", e.indexFace0);
  put_ints("edge_face1", e.indexFace1);
  put_ints("edge_vertex2", e.indexVertex2, true);
  std::printf("}\n");
  return 0;
}

int probe_bitmap(const char* path) {
  int w = 0, h = 0, c = 0;
  float* px = stbi_loadf(path, &w, &h, &c, 3);
  if (!px) {
    std::printf("{\n\"error\": \"%s\"\n}\n", stbi_failure_reason());
    return 0;
  }
  std::printf("{\n\"width\": %d,\n\"height\": %d,\n\"channels_in_file\": %d,\n", w, h, c);
  put_floats("texels", px, (size_t)w * h * 3, true);
  std::printf("}\n");
  stbi_image_free(px);
  return 0;
}

// EDX::Camera keeps its matrices protected; the renderer's camera reads them
// as a subclass, and so does this probe.
struct CameraProbe : EDX::Camera {
  int print() const {
    using EDX::Matrix;
    using EDX::Vector3;
    using EDX::Vector4;
    // Renderer/Camera.cpp:118-136
    const Matrix camera_to_sample = Matrix::Scale(1.0 / float(mFilmResX), 1.0 / float(mFilmResY), 1.0f) * mCameraToRaster;
    const Matrix sample_to_camera_img = mRasterToCamera * Matrix::Scale(float(mFilmResX), float(mFilmResY), 1.0f);
    const Vector4 v00 = Matrix::TransformPoint(Vector4(0.0f, 0.0f, 0.0f, 1.0f), sample_to_camera_img);
    const Vector4 v10 = Matrix::TransformPoint(Vector4(1.0f, 0.0f, 0.0f, 1.0f), sample_to_camera_img);
    const Vector4 v11 = Matrix::TransformPoint(Vector4(1.0f, 1.0f, 0.0f, 1.0f), sample_to_camera_img);
    const Vector4 vc = Matrix::TransformPoint(Vector4(0.5f, 0.5f, 0.0f, 1.0f), sample_to_camera_img);
    const Vector3 horizontal = Vector3(v00.x / v00.w, v00.y / v00.w, v00.z / v00.w) -
                               Vector3(v10.x / v10.w, v10.y / v10.w, v10.z / v10.w);
    const Vector3 vertical = Vector3(v11.x / v11.w, v11.y / v11.w, v11.z / v11.w) -
                             Vector3(v10.x / v10.w, v10.y / v10.w, v10.z / v10.w);
    const float len_x = EDX::Math::Length(horizontal);
    const float len_y = EDX::Math::Length(vertical);
    const float inv_area =
        1.0 / (len_x * len_y) * EDX::Math::LengthSquared(Vector3(vc.x / vc.w, vc.y / vc.w, vc.z / vc.w));
    const Matrix world_to_sample = Matrix::Mul(camera_to_sample, mView);
    const Matrix sample_to_camera = Matrix::Inverse(camera_to_sample);
    const float pos[3] = {mPos.x, mPos.y, mPos.z}, dir[3] = {mDir.x, mDir.y, mDir.z};
    std::printf("{\n\"width\": %d,\n\"height\": %d,\n", mFilmResX, mFilmResY);
    put_floats("pos", pos, 3);
    put_floats("dir", dir, 3);
    put_matrix("view", mView);
    put_matrix("view_inv", mViewInv);
    put_matrix("proj", mProj);
    put_matrix("raster_to_camera", mRasterToCamera);
    put_matrix("camera_to_raster", mCameraToRaster);
    put_matrix("raster_to_world", mRasterToWorld);
    put_matrix("world_to_sample", world_to_sample);
    put_matrix("sample_to_camera", sample_to_camera);
    put_floats("plane_len_x", &len_x, 1);
    put_floats("plane_len_y", &len_y, 1);
    put_floats("inv_area", &inv_area, 1, true);
    std::printf("}\n");
    return 0;
  }
};

int probe_camera(char** a) {
  float v[9];
  for (int i = 0; i < 9; i++) v[i] = std::strtof(a[i], nullptr);
  const int w = std::atoi(a[9]), h = std::atoi(a[10]);
  const float fov = std::strtof(a[11], nullptr);
  if (w <= 0 || h <= 0) {
    std::fprintf(stderr, "edx_probe: bad resolution\n");
    return 1;
  }
  CameraProbe cam;
  // Renderer Camera::Init's clip planes: nearClip 1, farClip 1000
  cam.Init(EDX::Vector3(v[0], v[1], v[2]), EDX::Vector3(v[3], v[4], v[5]), EDX::Vector3(v[6], v[7], v[8]), w, h, fov,
           1.0f, 1000.0f);
  return cam.print();
}

}  // namespace

int main(int argc, char** argv) {
  if (argc == 3 && !std::strcmp(argv[1], "obj")) return probe_obj(argv[2]);
  if (argc == 3 && !std::strcmp(argv[1], "bitmap")) return probe_bitmap(argv[2]);
  if (argc == 14 && !std::strcmp(argv[1], "camera")) return probe_camera(argv + 2);
  std::fprintf(stderr,
               "usage: edx_probe obj FILE\n"
               "       edx_probe bitmap FILE\n"
               "       edx_probe camera PX PY PZ TX TY TZ UX UY UZ W H FOV\n");
  return 2;
}
