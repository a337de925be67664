// Host-side scene object shared by scene.cu (build, configure, gradients) and
// render.cu (integrators). Not part of the public C-ABI.
#pragma once
#include <string>
#include <vector>
#include "scene_types.cuh"

struct trn_viewset;

struct trn_scene {
  // one-view set reused by trn_render_fwd / trn_render_grad (no per-call
  // allocation); created on the first single-view call
  trn_viewset* single = nullptr;
  // bytes of interior path records the single-view calls may keep between a
  // forward render and the gradient call of the same paths (0 = off)
  long long single_path_cache = 16LL << 30;
  // ---- sizes -----------------------------------------------------------------
  int nv = 0, nt = 0, nuv = 0, nmesh = 0, nlight = 0, nbsdf = 0, ntex = 0, ne = 0;
  long long ntexel = 0;
  // ---- parameters (device) ---------------------------------------------------
  float* raw_pos = nullptr;       // [V][3] positions before the mesh translation
  float* translation = nullptr;   // [M][3] per-mesh translation parameter
  float* texels = nullptr;        // [ntexel][3]
  // ---- derived geometry (device) --------------------------------------------
  float* pos = nullptr;           // [V][3]
  int* idx = nullptr;             // [T][3]
  float* fnormal = nullptr;       // [T][3]
  float* area = nullptr;          // [T]
  float* vnormal = nullptr;       // [V][3]
  unsigned char* smooth = nullptr;// [T]
  float* uv = nullptr;            // [NUV][2]
  int* uvidx = nullptr;           // [T][3]
  int* bsdf_id = nullptr;         // [T]
  int* emitter_id = nullptr;      // [T]
  int* vert_mesh = nullptr;       // [V]
  int* vf_off = nullptr;          // [V+1] vertex -> incident faces (CSR)
  int* vf_list = nullptr;         // [3T]
  // merged light
  int n_emit = 0;
  int* emit_tris = nullptr;
  int* tri_to_emit = nullptr;
  float* light_func = nullptr;
  float* light_cdf = nullptr;
  float* light_radiance = nullptr;
  float* light_integral_dev = nullptr;
  float light_lum[64];
  std::vector<float> h_light_radiance;
  // materials
  trn::BsdfDesc* bsdfs = nullptr;
  trn::TexDesc* texs = nullptr;
  std::vector<trn::BsdfDesc> h_bsdfs;
  std::vector<trn::TexDesc> h_texs;
  // edges (ObjMesh::processEdges, ObjMesh.cpp:584-632): v0 v1 f0 f1 v2
  int* edges = nullptr;           // [E][5]
  float* sec_func = nullptr;      // [E] length if the edge is a secondary edge else 0
  float* sec_cdf = nullptr;       // [E]
  float* sec_integral_dev = nullptr;
  // AQ guiding of the direct boundary term, one leaf per edge
  // (AdaptiveQuadratureDistribution, AQ_distrb.h:62-197)
  float* aq_poly = nullptr;       // [E] leaf weight after eps mixing
  float* aq_func = nullptr;       // [E] weight x leaf volume
  float* aq_cdf = nullptr;        // [E]
  float* aq_int = nullptr;        // [2] integral of aq_func/E, sum of aq_func
  // leaf boxes of the guiding tree: [6][aq_cap] (x0, y0, z0, x1, y1, z1) in
  // the (edge, light u, light v) sample cube, each leaf's edge, and the leaf
  // count (aq_count[0]; [1] is the count after the pass being built)
  float* aq_box = nullptr;
  int* aq_edge = nullptr;
  int* aq_count = nullptr;
  long long aq_cap = 0;           // leaves the aq_* arrays hold
  // refinement passes (g_direct_depth > 0): 36 evaluations per leaf, split
  // flags and their prefix sums; allocated by the first refining call
  float* aq_eval = nullptr;
  int* aq_flag = nullptr;
  int* aq_prefix = nullptr;
  // acceleration structure
  trn::BvhNode* nodes = nullptr;  // [T-1]
  float4* tri_verts = nullptr;    // [T][3]
  // multi-triangle leaves (TRN_LEAF_MAX > 1): the traversal uses these when
  // `collapsed`; leaf_cnt holds subtree counts, slots and slot bases [3][T-1]
  trn::BvhNode* cnodes = nullptr; // [T-1]
  float4* ctri = nullptr;         // [T][3]
  int* leaf_cnt = nullptr;
  void* leaf_scan_tmp = nullptr;
  size_t leaf_scan_bytes = 0;
  bool collapsed = false;
  int* parent = nullptr;          // [2T-1]
  int* flags = nullptr;           // [T-1]
  unsigned long long* keys = nullptr;     // [T]
  unsigned long long* keys_alt = nullptr; // [T]
  void* sort_tmp = nullptr;
  size_t sort_tmp_bytes = 0;
  // PLOC build scratch (cluster node ids and boxes, current + merged copies)
  int* ploc_node = nullptr;       // [2][T]
  float* ploc_box = nullptr;      // [2][T][6]
  int* ploc_nn = nullptr;         // [T]
  int* ploc_flag = nullptr;       // [T]
  int* ploc_pos = nullptr;        // [T]
  int* ploc_count = nullptr;      // [3] merge counter, cluster count, rounds that merged
  int ploc_rounds = 0;            // rounds the last build needed (0 = none yet)
  void* scan_tmp = nullptr;
  size_t scan_tmp_bytes = 0;
  float* bounds = nullptr;        // [6]
  trn::WNode* wnodes = nullptr;   // [<= T] 8-wide nodes
  float4* wtri = nullptr;         // [T][3]
  int* wqueue = nullptr;          // [2][T] (binary node, wide node) work pairs
  int* wcount = nullptr;          // [4] counters
  int n_wnodes = 0;
  // ---- gradients (device) ------------------------------------------------------
  float* g_pos = nullptr;         // [V][3] dL/d(world position)
  float* g_vnormal = nullptr;     // [V][3] dL/d(vertex normal)
  float* g_texels = nullptr;      // [ntexel][3]
  float* g_translation = nullptr; // [M][3]
  int* err = nullptr;             // device error word
  unsigned long long* stats = nullptr;  // [16] work counters of the integrator kernels
  bool stats_on = false;
  float h_light_integral = 0.f;
  bool configured = false;
  bool built = false;             // an LBVH topology exists (refit possible)
  bool grads_finalized = true;
  // bumped by every change of parameters or geometry: path records of an
  // older version are not reused
  unsigned long long version = 0;

  trn::DeviceScene view() const {
    trn::DeviceScene s;
    s.nv = nv; s.nt = nt;
    s.pos = pos; s.idx = idx; s.fnormal = fnormal; s.area = area; s.vnormal = vnormal;
    s.smooth = smooth; s.uv = uv; s.uvidx = uvidx; s.bsdf_id = bsdf_id; s.emitter_id = emitter_id;
    s.n_emit = n_emit; s.emit_tris = emit_tris; s.tri_to_emit = tri_to_emit;
    s.light_func = light_func; s.light_cdf = light_cdf; s.light_integral = light_integral_dev;
    s.light_radiance = light_radiance;
    s.n_bsdf = nbsdf; s.bsdfs = bsdfs; s.texs = texs; s.texels = texels;
    s.nodes = collapsed ? cnodes : nodes;
    s.tri_verts = collapsed ? ctri : tri_verts;
    s.root_is_leaf = nt == 1;
    s.wnodes = wnodes; s.wtri = wtri; s.n_wnodes = n_wnodes;
    return s;
  }
};

namespace trn {
void set_error(const std::string& msg);
void count_launch(int n = 1);  // host-side count of this library's kernel launches
}

#define TRN_CUDA_TRY(expr)                                                        \
  do {                                                                            \
    cudaError_t _e = (expr);                                                      \
    if (_e != cudaSuccess) {                                                      \
      trn::set_error(std::string(#expr) + ": " + cudaGetErrorString(_e));        \
      return -1;                                                                  \
    }                                                                             \
  } while (0)
