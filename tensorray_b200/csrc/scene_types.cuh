// Device-side views of the scene, camera and render options.
//
// HBM layout (all arrays are device pointers owned by the trn_scene handle):
//   pos        [V][3] f32  world-space vertex positions (Primitive::Configure
//                          output, Primitive.cpp:193 TransformPoints)
//   idx        [T][3] i32  position indices (TriangleMesh::mIndexPosBuffer)
//   fnormal    [T][3] f32  unit face normals   (Primitive.cpp:299-321)
//   area       [T]    f32  triangle areas      (Primitive.cpp:316)
//   vnormal    [V][3] f32  averaged vertex normals (Primitive.cpp:323-340)
//   smooth     [T]    u8   shading-normal flag (mUseSmoothShadingBuffer)
//   uv/uvidx   [NUV][2], [T][3]  texture coordinates (Scene.cpp:687-697)
//   bsdf_id    [T]    i32  material per triangle (mSbtIndexBuffer)
//   emitter_id [T]    i32  area-light id or -1 (mEmitterIDBuffer)
//   tri_verts  [T][12] f32 leaf-ordered triangle vertices for traversal:
//                          (P0.xyz, tri_id) (P1.xyz, 0) (P2.xyz, 0)
//   nodes      [T-1]  BvhNode  binary LBVH, child boxes stored in the parent
#pragma once
#include "common.cuh"

namespace trn {

enum BsdfType : int { kDiffuse = 0, kMicrofacet = 1 };

struct BsdfDesc {
  int type;          // BsdfType
  int tex;           // texture index for the (diffuse) albedo, -1 = constant
  float albedo[3];   // Diffuse albedo / Microfacet diffuse reflectance
  float spec[3];     // Microfacet specular reflectance (F0)
  float roughness;   // Microfacet roughness (Microfacet.cpp:51 alpha = r^2)
};

struct TexDesc {
  int w, h;
  long long offset;  // texel offset into the texel array (RGB triples)
};

struct alignas(16) BvhNode {
  // child 0 box (lo, hi), child 1 box (lo, hi), children (>=0 node, <0 ~leaf)
  float4 a;  // l0x l0y l0z h0x
  float4 b;  // h0y h0z l1x l1y
  float4 c;  // l1z h1x h1y h1z
  int4 d;    // c0 c1 - -
};

// 8-wide BVH node with quantised child boxes (80 bytes). Child boxes are
// stored as 8-bit offsets from `origin` in units of a per-axis power of two,
// rounded outwards, so decoding is conservative. Internal children of a node
// are stored contiguously from child_base, leaf triangles from tri_base;
// meta[i]: bit 7 = slot used, bit 6 = leaf, bits 0-5 = offset from the base.
struct alignas(16) WNode {
  float ox, oy, oz;
  unsigned char ex, ey, ez, nchild;  // biased exponents (IEEE bias 127)
  int child_base;
  int tri_base;
  unsigned char meta[8];
  unsigned char qlo[3][8];
  unsigned char qhi[3][8];
};
static_assert(sizeof(WNode) == 80, "WNode must be 80 bytes");

constexpr int kTopNodes = 73;  // root + 8 + 64 wide nodes staged in shared memory

// Traversal structure: the binary LBVH with child boxes in the parent (default;
// measured faster on B200 for the scenes here) or the 8-wide quantised BVH.
// most triangles in one leaf of the traversed LBVH (1 = the binary tree's
// one-triangle leaves, the default: leaves of up to 2 measured the same, up
// to 4 slower, because a leaf's box admits more rays than its triangles'
// boxes did and each costs exact watertight tests)
#ifndef TRN_LEAF_MAX
#define TRN_LEAF_MAX 1
#endif
#ifndef TRN_WIDE_BVH
#define TRN_WIDE_BVH 0
#endif

struct DeviceScene {
  int nv, nt;
  const float* pos;
  const int* idx;
  const float* fnormal;
  const float* area;
  const float* vnormal;
  const unsigned char* smooth;
  const float* uv;
  const int* uvidx;
  const int* bsdf_id;
  const int* emitter_id;
  // merged area light (Scene::ConfigureLight, Scene.cpp:471-520)
  int n_emit;                 // emitter triangles
  const int* emit_tris;       // [n_emit] global triangle ids
  const int* tri_to_emit;     // [T] index into emit_tris or -1
  const float* light_func;    // [n_emit] luminance * area (detached)
  const float* light_cdf;     // [n_emit] normalised inclusive CDF
  const float* light_integral;  // Distribution1D::mIntegralVal (device scalar)
  const float* light_radiance;// [n_lights][3]
  // materials
  int n_bsdf;
  const BsdfDesc* bsdfs;
  const TexDesc* texs;
  const float* texels;        // [sum w*h][3]
  // acceleration structure
  const BvhNode* nodes;
  const float4* tri_verts;    // [T][3] float4 (binary-leaf order)
  const WNode* wnodes;        // 8-wide quantised BVH
  const float4* wtri;         // [T][3] float4 in wide-leaf order
  int n_wnodes;
  int root_is_leaf;
};

// Pinhole camera (Camera.cpp:89-137, BaseCamera.cpp:45-88). Matrices are
// row-major 4x4 acting on column vectors (M * v).
struct CameraDesc {
  int w, h;
  float pos[3];
  float dir[3];
  float raster_to_camera[16];
  float view_inv[16];
  float world_to_sample[16];
  float sample_to_camera[16];
  float raster_to_world[16];
  float inv_area;            // Camera::mInvArea
  float plane_len_x, plane_len_y;
};

// One camera view of a batched launch. Path slots of all views are
// concatenated: view v owns slots [begin, begin + n) with n = W*H*spp, and
// its pixels start at pix_off in the image / dL/dI buffers.
struct ViewDesc {
  CameraDesc cam;
  long long begin;
  long long n;
  long long pix_off;
  long long slot_off;  // added to the view-local slot of the hash sampler
  float inv_spp;       // contribution weight (1/spp of the whole render)
  uint32_t seed;
  int spp;
  int pad_;
  float* image;        // forward radiance of this view [W*H*3] (accumulated)
  const float* dLdI;   // dL/dI of this view [W*H*3]
  int D;               // max bounces of this view
  int pad2_;
  float* gpos;         // gradient destinations of this view
  float* gvn;
  float* gtex;
  // silhouette-edge distribution of this view (ConstructPrimEdgeList)
  const float* pfunc;
  const float* pcdf;
  const float* pint;
};

}  // namespace trn
