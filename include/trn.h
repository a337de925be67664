/*
 * trn: B200-native path-space differentiable rendering, C-ABI.
 *
 * Drop-in replacement for the execution layer behind TensorRay's integrator
 * and scene API (LibTensorRay/Renderer). Every function returns 0 on success
 * and -1 on failure; trn_last_error() then describes the failure (the
 * reference throws std::runtime_error from CUDA_CHECK/OPTIX_CHECK,
 * LibTensorRay/Renderer/Optix.h:38-80, and pybind turns it into RuntimeError).
 * Bulk arrays passed to trn_render_* and trn_scene_get_* are DEVICE pointers;
 * the scene description passed to trn_scene_create is HOST memory. All work
 * is enqueued on the caller's stream (the reference runs on stream 0 and
 * synchronises after every kernel).
 */
#ifndef TRN_H_
#define TRN_H_

#include <cuda_runtime.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct trn_scene trn_scene;

/* Integrator ids (TensorRay.cpp:190-222 Python classes). */
enum {
  TRN_PATH_TRACER = 0,     /* PathTracer (PathTracer.cpp:37-123) */
  TRN_PRIMARY_EDGE = 1,    /* PrimaryEdgeIntegrator (BoundaryPrimary.cpp:36-181) */
  TRN_DIRECT_EDGE = 2,     /* DirectEdgeIntegrator (BoundaryDirect.cpp:38-143) */
  TRN_INDIRECT_EDGE = 3,   /* IndirectEdgeIntegrator (BoundaryIndirect.cpp:38-192) */
  TRN_PIXEL_EDGE = 4       /* PixelBoundaryIntegrator (BoundaryPixel.cpp:36-159) */
};

/* BSDF description (Diffuse.h, Microfacet.h; SceneLoader.cpp:265-305). */
typedef struct {
  int type;            /* 0 = diffuse, 1 = microfacet */
  int texture;         /* albedo / diffuse-reflectance texture index, -1 = constant */
  float albedo[3];     /* constant albedo / diffuse reflectance */
  float specular[3];   /* microfacet specular reflectance F0 */
  float roughness;     /* microfacet roughness */
} trn_bsdf;

/* RGB float texture, texel (x, y) at data[3 * (y * width + x)]
 * (ImageTexture, BSDF.cpp:56-98, stores the same texels channel-major). */
typedef struct {
  int width, height;
  const float* data;   /* host */
} trn_texture;

/* Whole-scene description: meshes are concatenated, indices are global.
 * Replaces Scene::ExtractGeometry / ConfigureLight inputs
 * (Scene.cpp:46-124, 471-520). All pointers are HOST memory. */
typedef struct {
  int num_vertices;
  int num_triangles;
  int num_uvs;
  int num_meshes;
  int num_lights;
  int num_bsdfs;
  int num_textures;
  const float* positions;        /* [V*3] raw positions (before the translation parameter) */
  const int* indices;            /* [T*3] */
  const float* uvs;              /* [NUV*2] or NULL */
  const int* uv_indices;         /* [T*3] or NULL */
  const int* vertex_mesh;        /* [V] mesh id of each vertex */
  const int* triangle_mesh;      /* [T] mesh id of each triangle */
  const unsigned char* mesh_smooth; /* [M] 1 = averaged vertex normals (Primitive.cpp:323-340) */
  const int* mesh_bsdf;          /* [M] bsdf id */
  const int* mesh_light;         /* [M] area-light id or -1 */
  const float* mesh_translation; /* [M*3] translation parameter (Primitive::mTrans) or NULL */
  const float* light_radiance;   /* [L*3] */
  const trn_bsdf* bsdfs;         /* [num_bsdfs] */
  const trn_texture* textures;   /* [num_textures] */
} trn_scene_desc;

/* Pinhole camera (Camera::Init, Camera.cpp:89-137 + BaseCamera.cpp:45-88).
 * Matrices are row-major and act on column vectors. */
typedef struct {
  int width, height;
  float pos[3];
  float dir[3];
  float raster_to_camera[16];
  float view_inv[16];
  float world_to_sample[16];
  float sample_to_camera[16];
  float raster_to_world[16];
  float inv_area;
  float plane_len_x, plane_len_y;
} trn_camera;

/* RenderOptions (Integrator.h:47-78). spp counts are per integrator;
 * batches only bound memory in the reference and are ignored here. */
typedef struct {
  int seed;
  int max_bounces;
  int spp;        /* interior (PathTracer) */
  int sppe;       /* primary edge */
  int sppse0;     /* direct edge */
  int sppse1;     /* indirect edge */
  int sppe0;      /* pixel boundary */
  /* AQ guiding of the direct boundary term (RenderOptions::g_*,
   * Integrator.h:72-77; AdaptiveQuadratureDistribution, AQ_distrb.h:62-197).
   * g_direct != 0 builds a guiding distribution per direct-boundary call:
   * one leaf per secondary edge (depth 0), then g_direct_depth refinement
   * passes that evaluate 36 points per leaf and split the leaves whose error
   * exceeds g_direct_thold (the reference's gen_eval_point / cut_tree,
   * NEE.cu:91-396, whose loop it keeps commented out, AQ_distrb.h:121-136),
   * up to max(edges, g_direct_max_size) leaves; leaf weights come from
   * g_direct_spp samples per leaf, mixed with g_eps. Guided samples use one
   * extra sample dimension (3 + 3*max_bounces). A refining call allocates
   * the tree's arrays on first use. */
  int g_direct;
  int g_direct_depth;
  int g_direct_max_size;
  int g_direct_spp;
  float g_direct_thold;
  float g_eps;
} trn_render_options;

/* Sample source for one integrator call. If `samples` is non-NULL it is a
 * device tensor of uniform floats laid out [dim][slot] with `stride` slots per
 * dimension (Tensorf::RandomFloat SoA blocks, Tensor.h:2793-2799); otherwise
 * samples come from the counter hash keyed by (options.seed, integrator). */
typedef struct {
  const float* samples;
  long long stride;
} trn_samples;

/* Launch shape of the persistent integrator kernels (0 = library default):
 * threads per block, resident blocks per SM, sample slots each lane takes
 * per fetch from the work queue, and the sample slots (boundary terms) or
 * paths (interior adjoint) per round of the split kernels, log2, at most the
 * default (boundary 24, interior 21), at least 16. Chosen by the autotuner
 * (tensorray_b200/autotune.py). */
typedef struct {
  int block;
  int blocks_per_sm;
  int chunk;
  int round_log2;
} trn_launch;

/* One camera view of a batched render (the reference renders one view per
 * call and loops over views in Python, pyTensorRay/renderer_multi_view.py:53-61).
 * pixel_offset: first pixel of this view in the concatenated image / dL/dI
 * buffers (-1 = right after the previous view). slot_offset shifts the
 * view's hash-sampler slots (a render split into spp chunks uses disjoint
 * slots per chunk); weight scales contributions (0 = 1/spp). grad_*: device
 * gradient destinations of this view ([V*3], [V*3], [texels*3]); NULL = the
 * scene's own buffers. image / dLdI: per-view buffers (a request of a serving
 * loop); a NULL call buffer in trn_render_views_fwd/grad then means "use the
 * per-view buffers". */
typedef struct {
  trn_camera camera;
  int spp;
  int seed;
  long long pixel_offset;
  long long slot_offset;
  float weight;
  int max_bounces;          /* 0 = options.max_bounces */
  float* grad_positions;
  float* grad_vertex_normals;
  float* grad_texels;
  float* image;             /* own image [W*H*3] (accumulated, not cleared); NULL = the call's buffer */
  const float* dLdI;        /* own dL/dI [W*H*3]; NULL = the call's buffer */
} trn_view;

typedef struct trn_viewset trn_viewset;

/* Last error message of this thread ("" if none). */
const char* trn_last_error(void);
/* Library version string. */
const char* trn_version(void);

/* Build a camera. Replaces Camera::Init (Camera.cpp:89-103). */
int trn_camera_init(trn_camera* out, const float pos[3], const float target[3], const float up[3],
                    int width, int height, float fov_deg);

/* The edge list of a triangle mesh, host-only (no device work). Replaces
 * ObjMesh::processEdges (EDXUtil/Graphics/ObjMesh.cpp:584-632), which the
 * secondary and primary edge lists start from: one row (v0, v1, f0, f1, v2)
 * per unique undirected edge, v0 < v1, rows in (v0, v1) order. f0 is the first
 * face (in face order) that has the edge and v2 that face's third vertex; f1
 * is the second face when exactly two faces share the edge, else -1.
 * indices: [num_triangles*3]. Writes min(rows, cap) rows of 5 ints to out and
 * returns the number of rows (call with cap = 0 to size out), or -1 on
 * invalid arguments. */
long long trn_mesh_edges(int num_triangles, const int* indices, int* out, long long cap);

/* Scene lifetime. Replaces Scene::Configure (Scene.cpp:522-533): create
 * uploads the description; configure runs Primitive::Configure, face/vertex
 * normals, light distribution, secondary edge list and the LBVH build. */
int trn_scene_create(const trn_scene_desc* desc, trn_scene** out);
int trn_scene_configure(trn_scene* scene, cudaStream_t stream);
int trn_scene_destroy(trn_scene* scene);
/* Re-run the geometry chain for new parameters and refit the LBVH boxes
 * without rebuilding its topology (Scene::Update / UpdateAccelerationStructure,
 * Scene.cpp:368-469, 535-546). Falls back to trn_scene_configure the first time. */
int trn_scene_refit(trn_scene* scene, cudaStream_t stream);

/* Parameter access (TensorRay.cpp: get_var/set_var; Primitive::mTrans,
 * mPositionBufferRaw, BSDF texture). Device pointers. set_* marks the scene
 * for re-configuration. */
int trn_scene_set_translation(trn_scene* scene, const float* translation_dev, cudaStream_t stream);
int trn_scene_set_positions(trn_scene* scene, const float* raw_positions_dev, cudaStream_t stream);
int trn_scene_set_texels(trn_scene* scene, const float* texels_dev, cudaStream_t stream);

/* Read back derived geometry for checks (device destinations). */
int trn_scene_get_geometry(trn_scene* scene, float* pos, float* fnormal, float* area, float* vnormal,
                           cudaStream_t stream);
int trn_scene_counts(const trn_scene* scene, int* num_vertices, int* num_triangles, int* num_edges,
                     long long* num_texels, int* num_meshes);

/* Closest-hit ray query over the LBVH. Replaces RayIntersectOptix
 * (Optix.h:149, Optix.cpp:252-305): out_tri = -1 on a miss. Device arrays of
 * n rays: org/dir [n*3], tmin/tmax [n]; outputs tri [n], u/v/t [n]. */
int trn_intersect(trn_scene* scene, int n, const float* org, const float* dir, const float* tmin,
                  const float* tmax, int* out_tri, float* out_u, float* out_v, float* out_t,
                  cudaStream_t stream);
/* Occlusion query (Scene::Occluded, Scene.cpp:548-562): out_visible[i] = 1
 * when nothing is hit inside (tmin, tmax). */
int trn_occluded(trn_scene* scene, int n, const float* org, const float* dir, const float* tmin,
                 const float* tmax, int* out_visible, cudaStream_t stream);

/* Single-view calls (trn_render_fwd / trn_render_grad) reuse one view table
 * held by the scene: the first such call allocates it, later calls neither
 * allocate nor synchronise the stream. Calls on one scene must therefore be
 * ordered on one stream (as the reference's single default stream orders
 * them); use view sets for concurrent rendering.
 *
 * Forward render of one integrator (Integrator::RenderC, Integrator.h:96-104,
 * PathTracer.h:60-68). image_out [W*H*3] is overwritten. Only
 * TRN_PATH_TRACER produces radiance; edge integrators produce their
 * (zero-valued in the reference) primal and return 0. */
int trn_render_fwd(trn_scene* scene, const trn_camera* camera, const trn_render_options* options,
                   int integrator, const trn_samples* samples, float* image_out, cudaStream_t stream);

/* Reverse-mode pass of one integrator (Integrator::RenderD, Integrator.h:106-121):
 * replays the paths of the same seed/samples and accumulates dL/dparameters
 * into the scene's gradient buffers given dL/dI [W*H*3]. */
int trn_render_grad(trn_scene* scene, const trn_camera* camera, const trn_render_options* options,
                    int integrator, const trn_samples* samples, const float* dLdI, cudaStream_t stream);

/* trn_render_grad without any device allocation. No counterpart in the
 * reference: it is for callers that may not call cudaMalloc or cudaFree while
 * rendering (a host application that owns all device memory through its own
 * allocator, or a loop that cannot take the device-wide synchronisation of
 * cudaFree). Same arguments and results as trn_render_grad, but all scratch
 * (view table, work counter, silhouette-edge distribution) lives in one fixed
 * array compiled into the library (about 8 MiB, held on every GPU that loads
 * the library until the process exits), and the call does not synchronise
 * the stream.
 * - Speed: it runs each term as one fused kernel (no split stages, no queues,
 *   no edge-sorted set-up order, since those need scratch that grows with
 *   the launch), which is about 20-50 % slower per term than
 *   trn_render_grad.
 * - Limit: for TRN_PRIMARY_EDGE the scene may have at most 1048576 edges;
 *   larger scenes are rejected with an error.
 * - A guided direct term with g_direct_depth > 0 needs the refined tree's
 *   arrays, which the first refining trn_render_grad call allocates; before
 *   that call it is rejected with an error.
 * - The scene's device must be the current device; otherwise the call
 *   returns an error.
 * - The first call on each device looks up the array's device address
 *   (cudaGetSymbolAddress); make that first call before any stream capture.
 *   The fused kernels keep large per-thread stack frames, so the first call
 *   in a process may also make the CUDA driver enlarge its local-memory
 *   reservation for the context (the driver's own allocation, not one by
 *   this library); making the first call during set-up keeps that out of the
 *   loop that must not allocate.
 * - Calls that overlap on the GPU (other streams or host threads, same
 *   device) share the array and race; the array keeps the last call's
 *   contents, and each call rewrites what it reads. */
int trn_render_grad_noalloc(trn_scene* scene, const trn_camera* camera, const trn_render_options* options,
                            int integrator, const trn_samples* samples, const float* dLdI, cudaStream_t stream);

/* Batched multi-view rendering: all views of a view set in one persistent
 * launch per integrator, images concatenated [npix*3]. The per-view spp of
 * trn_view applies to the integrator being rendered; options supplies
 * max_bounces and the seed. */
int trn_viewset_create(trn_scene* scene, int nviews, const trn_view* views, trn_viewset** out);
int trn_viewset_destroy(trn_viewset* views);
/* Replace the views of a set (storage grows as needed; a serving loop
 * re-uses one set per scene and phase). The next render call uploads the new
 * table on its stream from one of four pinned staging slots, so a caller that
 * changes the views on every call runs up to four calls ahead of the device;
 * only a growth of the set waits for the uploads in flight. Successive calls
 * on one set must use one stream (the table is rewritten in stream order). */
int trn_viewset_update(trn_viewset* views, int nviews, const trn_view* view_array);
int trn_viewset_num_pixels(const trn_viewset* views, long long* npix);
/* Allocate the set's round buffers now: the queue of the split integrator
 * kernels (one full round of any term at up to max_bounces) and the buffers
 * of the edge-sorted run order of the boundary set-up. Without it the first
 * gradient call of each term allocates them, and a larger batch later grows
 * them (each growth synchronises the stream and frees the old buffer). For a
 * serving loop, or before capturing render calls into a CUDA graph. No
 * counterpart in the reference (its tensor library allocates per call).
 * About 5.5 GB for max_bounces <= 8 (rounds of 16M boundary samples). */
int trn_viewset_reserve(trn_viewset* views, int max_bounces, cudaStream_t stream);
/* Path cache. A forward render of TRN_PATH_TRACER can keep the record of
 * every path it traced (hit points, light samples, throughputs: about 620
 * bytes per path at max_bounces <= 8). The next trn_render_views_grad of
 * TRN_PATH_TRACER over the same paths then runs only the reverse sweep
 * instead of tracing them again. The reference re-traces them: its RenderD
 * rebuilds the forward tensor program (Integrator.h:106-121). The gradients
 * are the same either way. Records are reused only when nothing the paths
 * depend on has changed since the forward call: the scene (any set_* call,
 * configure or refit), the views' cameras, spp, seeds, slot offsets and
 * depths, and the options' seed and max_bounces. Calls with a sample table
 * and calls under stream capture neither write nor read records.
 * max_bytes bounds the records' memory (0 = off, the default for view sets);
 * a forward render whose records would exceed it renders without them. */
int trn_viewset_path_cache(trn_viewset* views, long long max_bytes);
/* The same bound for the single-view calls trn_render_fwd / trn_render_grad
 * (default 16 GiB). */
int trn_scene_path_cache(trn_scene* scene, long long max_bytes);
int trn_render_views_fwd(trn_scene* scene, trn_viewset* views, const trn_render_options* options, int integrator,
                         const trn_samples* samples, const trn_launch* launch, float* images, cudaStream_t stream);
int trn_render_views_grad(trn_scene* scene, trn_viewset* views, const trn_render_options* options, int integrator,
                          const trn_samples* samples, const trn_launch* launch, const float* dLdI,
                          cudaStream_t stream);
/* Per-view image loss 0.5*|I - T|^2 (pyTensorRay/loss.py:34-38) into loss[nviews]
 * and dL/dI = I - T into dLdI (either may be NULL). */
int trn_views_loss(trn_viewset* views, const float* images, const float* targets, float* dLdI, float* loss,
                   cudaStream_t stream);

/* Finish the geometry-chain adjoint and copy gradients out (get_grad with
 * clear_grad, pybind_utils.h:133-142). Any destination may be NULL.
 * d_translation [M*3], d_positions [V*3] (raw positions), d_texels [ntexel*3]. */
int trn_scene_get_grads(trn_scene* scene, float* d_translation, float* d_positions, float* d_texels,
                        int clear, cudaStream_t stream);
int trn_scene_clear_grads(trn_scene* scene, cudaStream_t stream);
/* Geometry-chain adjoint for caller-owned gradient buffers (per-request
 * gradients of the serving loop): folds grad_vertex_normals [V*3] into
 * grad_positions [V*3] (and zeroes it), and writes d_translation [M*3]. */
int trn_scene_finalize_grads(trn_scene* scene, float* grad_positions, float* grad_vertex_normals,
                             float* d_translation, cudaStream_t stream);

/* Instrumentation (the reference counts JIT launches per pass with
 * KernelLaunchCounter, Tensor.h:1526-1547, printed at PathTracer.cpp:114).
 * trn_kernel_launches: kernels this library has launched since load.
 * trn_stats_enable / trn_stats_read: per-scene device work counters of the
 * integrator kernels, 16 x u64: closest-hit queries, shadow queries, shading
 * vertices, smooth-shaded vertices, textured vertices, light samples,
 * position-gradient vertex updates, normal-gradient vertex updates, texel
 * gradient updates, pixel accesses (rest reserved). */
unsigned long long trn_kernel_launches(void);
int trn_stats_enable(trn_scene* scene, int on);
int trn_stats_read(trn_scene* scene, unsigned long long* out16, int reset, cudaStream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* TRN_H_ */
