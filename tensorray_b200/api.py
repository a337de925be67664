"""Python mirror of the reference's ``TensorRay`` module (TensorRay.cpp:48-222).

Names, arguments and error behaviour follow the reference: ``Scene``,
``RenderOptions``, ``PathTracer`` / ``PrimaryEdgeIntegrator`` /
``DirectEdgeIntegrator`` / ``IndirectEdgeIntegrator`` /
``PixelBoundaryIntegrator`` with ``renderC`` and ``renderD``, shapes with
``diff_translation`` / ``diff_all_vertex_pos``, BSDFs with ``diff_texture``.
Failures raise ``RuntimeError`` with the library's message, as pybind does for
the reference's std::runtime_error. Device memory and streams come from
PyTorch; all rendering runs in the native library.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _abi
from ._abi import (TRN_DIRECT_EDGE, TRN_INDIRECT_EDGE, TRN_PATH_TRACER, TRN_PIXEL_EDGE, TRN_PRIMARY_EDGE,
                   TrnBsdf, TrnCamera, TrnLaunch, TrnRenderOptions, TrnSamples, TrnSceneDesc, TrnTexture, TrnView,
                   check)
from .scenes import SceneSpec


def _require_cuda() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("tensorray_b200 renders on a CUDA device; none is available")
    return torch.device("cuda", torch.cuda.current_device())


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def _fptr(a: np.ndarray | None):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _iptr(a: np.ndarray | None):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_int))


def env_create() -> None:
    """Load the native library (EnvCreate, pybind_utils.h:38-53)."""
    _abi.load()


def env_release() -> None:
    torch.cuda.empty_cache()


class RenderOptions:
    """RenderOptions (Integrator.h:47-78, bound at TensorRay.cpp:165-188)."""

    def __init__(self, seed: int, max_bounces: int, spp: int, sppe: int, sppse0: int, sppse1: int, sppe0: int = 0):
        self.seed = seed
        self.max_bounces = max_bounces
        self.spp = spp
        self.sppe = sppe
        self.sppse0 = sppse0
        self.sppse1 = sppse1
        self.sppe0 = sppe0
        self.spp_batch, self.sppe_batch, self.sppse0_batch = spp, sppe, sppse0
        self.sppse1_batch, self.sppe0_batch = sppse1, sppe0
        self.export_deriv = False
        self.quiet = True
        # guiding options (Integrator.h:72-77)
        self.g_direct = False
        self.g_direct_depth = 0
        self.g_direct_max_size = 100000
        self.g_direct_spp = 16
        self.g_direct_thold = 0.01
        self.g_eps = 0.01

    def _c(self) -> TrnRenderOptions:
        return TrnRenderOptions(int(self.seed), int(self.max_bounces), int(self.spp), int(self.sppe),
                                int(self.sppse0), int(self.sppse1), int(self.sppe0), int(bool(self.g_direct)),
                                int(self.g_direct_depth), int(self.g_direct_max_size), int(self.g_direct_spp),
                                float(self.g_direct_thold), float(self.g_eps))


class Camera:
    """Pinhole sensor (Camera::Init, Camera.cpp:89-103; the binding,
    TensorRay.cpp:143-151): Camera() is empty until init(); update(other)
    copies another camera's pose; resize(width, height) keeps the pose."""

    def __init__(self, pos=None, target=None, up=None, width: int = 0, height: int = 0, fov: float = 35.0):
        self.c = TrnCamera()
        self.width = self.height = 0
        self.pos = self.target = self.up = None
        self.fov = float(fov)
        if pos is not None:
            self.init(pos, target, up, width, height, fov)

    def init(self, pos, target, up, width: int, height: int, fov: float = 35.0) -> None:
        """Camera::Init with the reference's defaults (fov 35 degrees; clip
        planes 1 and 1000, Camera.h:115-123)."""
        c = TrnCamera()
        f3 = lambda v: (C.c_float * 3)(*[float(x) for x in v])
        check(_abi.load().trn_camera_init(C.byref(c), f3(pos), f3(target), f3(up), int(width), int(height),
                                          C.c_float(float(fov))), "trn_camera_init")
        self.c = c
        self.width, self.height = int(width), int(height)
        self.pos, self.target, self.up, self.fov = tuple(pos), tuple(target), tuple(up), float(fov)

    def update(self, other: "Camera") -> None:
        """Camera::Update (Camera.h:110-113): this camera takes the other's
        pose, resolution and field of view."""
        self.init(other.pos, other.target, other.up, other.width, other.height, other.fov)

    def resize(self, width: int, height: int) -> None:
        """Camera::Resize (Camera.cpp:105-137): a new resolution, same pose."""
        if self.pos is None:
            raise RuntimeError("camera not initialised")
        self.init(self.pos, self.target, self.up, width, height, self.fov)

    def matrices(self) -> dict:
        c = self.c
        m = lambda a: np.array(list(a), np.float32).reshape(4, 4)
        return {"pos": np.array(list(c.pos), np.float32), "dir": np.array(list(c.dir), np.float32),
                "raster_to_camera": m(c.raster_to_camera), "view_inv": m(c.view_inv),
                "world_to_sample": m(c.world_to_sample), "sample_to_camera": m(c.sample_to_camera),
                "raster_to_world": m(c.raster_to_world), "inv_area": np.float32(c.inv_area),
                "plane_len_x": np.float32(c.plane_len_x), "plane_len_y": np.float32(c.plane_len_y),
                "width": c.width, "height": c.height}


def _host_f32(x) -> torch.Tensor:
    """A float32 CPU tensor of a tensor (any device), array or sequence."""
    if isinstance(x, torch.Tensor):
        return x.detach().to("cpu", torch.float32)
    return torch.as_tensor(np.asarray(x, np.float32))


def rotation_axis_angle(angle, axis, derivative: bool = False) -> torch.Tensor:
    """CalcRotateAxisAngle (Renderer/Utils.cpp:200-232): the right-handed
    rotation by `angle` radians about the normalised `axis`, a 3x3 matrix on
    column vectors, c I + s [k]x + (1 - c) k k^T. With derivative=True its
    derivative with respect to the angle, -s I + c [k]x + s k k^T."""
    k = _host_f32(axis).reshape(3)
    k = k / torch.linalg.vector_norm(k)
    a = _host_f32(angle).reshape(())
    s, c = torch.sin(a), torch.cos(a)
    K = torch.zeros(3, 3)
    K[0, 1], K[0, 2], K[1, 0], K[1, 2], K[2, 0], K[2, 1] = -k[2], k[1], k[2], -k[0], -k[1], k[0]
    kk = torch.outer(k, k)
    eye = torch.eye(3)
    if derivative:
        return -s * eye + c * K + s * kk
    return c * eye + s * K + (1.0 - c) * kk


class Shape:
    """Primitive parameters (Primitive.cpp:374-388), and its rotations
    (Primitive::Configure, Primitive.cpp:158-189):

    - rotate_matrix (3x3 or 4x4, p' = M p on column vectors) with obj_center c:
      the fixed pose rotation of multi-pose optimisation, p' = M (p - c) + c.
      The reference's own pose tensors (pyTensorRay/multi_pose.py:53-64) pack
      a row-major matrix into its column layout, so a pose built there from
      `mat` is `mat.reshape(3, 3).T` here.
    - diff_rotation(axis) with rotate_angle: a differentiable rotation about
      the world origin, applied after the pose; dL/d(angle) comes back from
      Scene.get_grads() as "rotation_angle".
    - vertex_id with vertex_translation: one vertex moved in world space after
      the rotations (Primitive.cpp:194-199); dL/d(vertex_translation) comes
      back as "vertex_translation".

    Translation is applied last. The reference applies the pose in object
    space, before the shape's XML to_world; here meshes are held in world
    space, so the two agree for shapes without a to_world transform."""

    def __init__(self, scene: "Scene", index: int, vstart: int, vcount: int, fcount: int):
        self._scene, self.index = scene, index
        self._vstart, self._vcount, self._fcount = vstart, vcount, fcount
        self.requires_translation_grad = False
        self.requires_vertex_grad = False
        self.requires_rotation_grad = False
        self._rotate_matrix = None
        self._obj_center = None
        self._rotate_axis = None
        self._rotate_angle = 0.0
        self._vertex_id = -1
        self._vertex_translation = None

    def _changed(self) -> None:
        if self._scene is not None:
            self._scene._dirty = True

    @property
    def translation(self) -> torch.Tensor:
        return self._scene._translation[self.index].clone()

    @translation.setter
    def translation(self, t) -> None:
        self._scene._translation[self.index] = torch.as_tensor(t, dtype=torch.float32,
                                                               device=self._scene.device).reshape(3)
        self._scene._dirty = True

    @property
    def rotate_matrix(self):
        return self._rotate_matrix

    @rotate_matrix.setter
    def rotate_matrix(self, m) -> None:
        if m is not None:
            m = _host_f32(m)
            if m.shape not in ((3, 3), (4, 4)):
                raise RuntimeError("rotate_matrix must be 3x3 or 4x4")
            m = m[:3, :3].clone()
        self._rotate_matrix = m
        self._changed()

    @property
    def obj_center(self):
        return self._obj_center

    @obj_center.setter
    def obj_center(self, c) -> None:
        self._obj_center = None if c is None else _host_f32(c).reshape(3).clone()
        self._changed()

    @property
    def rotate_axis(self):
        return self._rotate_axis

    @rotate_axis.setter
    def rotate_axis(self, axis) -> None:
        self._rotate_axis = None if axis is None else tuple(float(x) for x in _host_f32(axis).reshape(3))
        self._changed()

    @property
    def rotate_angle(self) -> float:
        return self._rotate_angle

    @rotate_angle.setter
    def rotate_angle(self, a) -> None:
        self._rotate_angle = float(a)
        self._changed()

    @property
    def vertex_id(self) -> int:
        return self._vertex_id

    @vertex_id.setter
    def vertex_id(self, i) -> None:
        i = int(i)
        if i >= self._vcount:
            raise RuntimeError(f"vertex_id {i} is out of range for a shape of {self._vcount} vertices")
        self._vertex_id = i
        self._changed()

    @property
    def vertex_translation(self):
        return self._vertex_translation

    @vertex_translation.setter
    def vertex_translation(self, t) -> None:
        self._vertex_translation = None if t is None else _host_f32(t).reshape(3).clone()
        self._changed()

    def _moves_vertex(self) -> bool:
        return self._vertex_id >= 0 and self._vertex_translation is not None

    def _posed(self) -> bool:
        return self._rotate_matrix is not None or self._rotate_axis is not None or self._moves_vertex()

    def diff_translation(self) -> None:
        self.requires_translation_grad = True

    def diff_all_vertex_pos(self) -> None:
        self.requires_vertex_grad = True

    def diff_rotation(self, rotate_axis) -> None:
        """Primitive::DiffRotation (Primitive.cpp:379-383): rotate about
        `rotate_axis` by an angle that starts at 0 and is differentiated."""
        self.rotate_axis = rotate_axis
        self.rotate_angle = 0.0
        self.requires_rotation_grad = True

    def get_obj_center(self) -> torch.Tensor:
        """Primitive::GetObjCenter (Primitive.cpp:444-450): the centre of the
        shape's bounding box over its unrotated positions."""
        p = self._scene._raw_positions[self.vertex_slice()]
        return (0.5 * (p.min(0).values + p.max(0).values)).cpu()

    def _rotations(self):
        """(pose matrix or None, centre, rotation matrix or None, its
        derivative or None), on the CPU."""
        c = self._obj_center if self._obj_center is not None else torch.zeros(3)
        if self._rotate_axis is None:
            return self._rotate_matrix, c, None, None
        return (self._rotate_matrix, c, rotation_axis_angle(self._rotate_angle, self._rotate_axis),
                rotation_axis_angle(self._rotate_angle, self._rotate_axis, derivative=True))

    def get_vertex_count(self) -> int:
        return self._vcount

    def get_face_count(self) -> int:
        return self._fcount

    def _faces(self) -> np.ndarray:
        return np.ascontiguousarray(self._scene.spec.meshes[self.index].faces, np.int32).reshape(-1, 3)

    def get_face_indices(self, out=None) -> np.ndarray:
        """Primitive::GetFaceIndices (Primitive.cpp:419-433): the shape's
        triangles as vertex indices local to the shape, 3 per face. The
        reference writes them through a pointer; here they are returned, and
        copied into `out` (an array or tensor of 3 * faces ints) when given."""
        f = self._faces().reshape(-1)
        return _fill(out, f)

    def get_edge_count(self) -> int:
        """Primitive::GetEdgeCount (Primitive.cpp:400-403): the edges
        ObjMesh::processEdges finds in the shape's mesh."""
        return int(len(mesh_edges(self._faces())))

    def get_edge_data(self, out=None) -> np.ndarray:
        """Primitive::GetEdgeData (Primitive.cpp:435-442): the first vertex of
        every edge, then the second (2 * edges ints, local to the shape),
        copied into `out` when given."""
        e = mesh_edges(self._faces())
        return _fill(out, np.concatenate([e[:, 0], e[:, 1]]).astype(np.int32))

    def export_mesh(self, filename: str) -> None:
        """Primitive::ExportMesh (Primitive.cpp:452-469): an OBJ of the shape's
        unrotated, untranslated positions ("v x y z", 6 significant digits as
        the reference's stream writes them) and its faces (1-based)."""
        P = self._scene._raw_positions[self.vertex_slice()].detach().cpu().numpy()
        F = self._faces()
        with open(filename, "w") as f:
            for p in P:
                f.write("v %g %g %g\n" % (float(p[0]), float(p[1]), float(p[2])))
            for t in F:
                f.write("f %d %d %d\n" % (int(t[0]) + 1, int(t[1]) + 1, int(t[2]) + 1))

    def vertex_slice(self) -> slice:
        return slice(self._vstart, self._vstart + self._vcount)


def _fill(out, values: np.ndarray) -> np.ndarray:
    """`values`, also copied into `out` (a numpy array or a tensor) when given."""
    if out is not None:
        n = out.numel() if isinstance(out, torch.Tensor) else out.size
        if n != values.size:
            raise RuntimeError(f"output holds {n} elements, {values.size} needed")
        if isinstance(out, torch.Tensor):
            out.view(-1).copy_(torch.from_numpy(values).to(out.dtype))
        else:
            out.reshape(-1)[:] = values
    return values


def posed_positions(raw: torch.Tensor, shapes: list):
    """The positions the library transforms (world = these + translation):
    each shape's raw positions through its pose, p' = M (p - c) + c, then its
    differentiable rotation, R p', then its one moved vertex. None when no
    shape is posed."""
    posed = [s for s in shapes if s._posed()]
    if not posed:
        return None
    out = raw.clone()
    for s in posed:
        M, c, R, _ = s._rotations()
        sl = s.vertex_slice()
        q = raw[sl]
        if M is not None:
            cd = c.to(q.device)
            q = (q - cd) @ M.to(q.device).T + cd
        if R is not None:
            q = q @ R.to(q.device).T
        if s._moves_vertex():
            q = q.clone()
            q[s._vertex_id] += s._vertex_translation.to(q.device)
        out[sl] = q
    return out


def pose_grads(raw: torch.Tensor, grad: torch.Tensor, shapes: list):
    """Chain rule through posed_positions. `grad` is dL/d(posed positions);
    returns dL/d(raw positions) (rows of rotated shapes through R and M),
    dL/d(rotate_angle) per shape (0 for shapes without diff_rotation) and
    dL/d(vertex_translation) per shape [shapes, 3] (0 where no vertex moves)."""
    out = grad.clone()
    d_angle = torch.zeros(len(shapes), device=grad.device)
    d_vertex = torch.zeros(len(shapes), 3, device=grad.device)
    for i, s in enumerate(shapes):
        M, c, R, dR = s._rotations()
        sl = s.vertex_slice()
        if s._moves_vertex():
            d_vertex[i] = grad[sl][s._vertex_id]
        if M is None and R is None:
            continue
        g = grad[sl]
        q = raw[sl]
        if M is not None:
            cd = c.to(q.device)
            q = (q - cd) @ M.to(q.device).T + cd
        if R is not None:
            d_angle[i] = (g * (q @ dR.to(q.device).T)).sum()
            g = g @ R.to(g.device)
        if M is not None:
            g = g @ M.to(g.device)
        out[sl] = g
    return out, d_angle, d_vertex


class BSDF:
    def __init__(self, scene: "Scene", index: int, texture: int):
        self._scene, self.index, self.texture = scene, index, texture
        self.requires_texture_grad = False

    def diff_texture(self, name: str = "") -> None:
        if self.texture < 0:
            raise RuntimeError("BSDF has no texture to differentiate")
        self.requires_texture_grad = True


class Scene:
    """Scene (Scene.h:98-130) over a native trn_scene handle."""

    def __init__(self, spec: SceneSpec | None = None):
        self.device = _require_cuda()
        self._lib = _abi.load()
        self._h = C.c_void_p()
        self._dirty = True
        self.shapes: list[Shape] = []
        self.bsdfs: list[BSDF] = []
        self.cameras: list[Camera] = []
        if spec is not None:
            self.load_spec(spec)

    # -- construction -------------------------------------------------------
    def load_file(self, filename: str) -> None:
        """Scene::LoadFromFile (Scene.cpp:41-44): the reference's XML scene
        format (scene_xml.load_xml) into this scene; configure() follows."""
        from . import scene_xml
        self.load_spec(scene_xml.load_xml(filename))

    def load_spec(self, spec: SceneSpec) -> None:
        a = spec.arrays()
        self.spec = spec
        self._keep = a
        nb = len(spec.bsdfs)
        bs = (TrnBsdf * nb)()
        for i, b in enumerate(spec.bsdfs):
            bs[i] = TrnBsdf(b.type, b.texture, (C.c_float * 3)(*b.albedo), (C.c_float * 3)(*b.specular),
                            b.roughness)
        texs = (TrnTexture * max(1, len(spec.textures)))()
        self._tex_keep = []
        for i, t in enumerate(spec.textures):
            arr = np.ascontiguousarray(t, np.float32)
            self._tex_keep.append(arr)
            texs[i] = TrnTexture(arr.shape[1], arr.shape[0], _fptr(arr))
        d = TrnSceneDesc()
        d.num_vertices = len(a["positions"])
        d.num_triangles = len(a["indices"])
        d.num_uvs = 0 if a["uvs"] is None else len(a["uvs"])
        d.num_meshes = len(spec.meshes)
        d.num_lights = len(spec.lights)
        d.num_bsdfs = nb
        d.num_textures = len(spec.textures)
        d.positions = _fptr(a["positions"])
        d.indices = _iptr(a["indices"])
        d.uvs = _fptr(a["uvs"])
        d.uv_indices = _iptr(a["uv_indices"])
        d.vertex_mesh = _iptr(a["vertex_mesh"])
        d.triangle_mesh = _iptr(a["triangle_mesh"])
        d.mesh_smooth = a["mesh_smooth"].ctypes.data_as(C.POINTER(C.c_ubyte))
        d.mesh_bsdf = _iptr(a["mesh_bsdf"])
        d.mesh_light = _iptr(a["mesh_light"])
        d.mesh_translation = _fptr(a["mesh_translation"])
        d.light_radiance = _fptr(a["light_radiance"])
        d.bsdfs = bs
        d.textures = texs
        check(self._lib.trn_scene_create(C.byref(d), C.byref(self._h)), "trn_scene_create")
        nv, nt, ne, nm = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        ntex = C.c_longlong()
        check(self._lib.trn_scene_counts(self._h, C.byref(nv), C.byref(nt), C.byref(ne), C.byref(ntex),
                                         C.byref(nm)), "trn_scene_counts")
        self.num_vertices, self.num_triangles, self.num_edges = nv.value, nt.value, ne.value
        self.num_texels, self.num_meshes = ntex.value, nm.value
        self._translation = torch.as_tensor(a["mesh_translation"], device=self.device).clone()
        self._raw_positions = torch.as_tensor(a["positions"], device=self.device).clone()
        vstart = 0
        for i, m in enumerate(spec.meshes):
            self.shapes.append(Shape(self, i, vstart, len(m.positions), len(m.faces)))
            vstart += len(m.positions)
        self.bsdfs = [BSDF(self, i, b.texture) for i, b in enumerate(spec.bsdfs)]
        self.cameras = [Camera(c.pos, c.target, c.up, c.width, c.height, c.fov) for c in spec.cameras]
        self._dirty = True

    def __del__(self):
        try:
            if self._h:
                self._lib.trn_scene_destroy(self._h)
                self._h = C.c_void_p()
        except Exception:
            pass

    # -- parameters -----------------------------------------------------------
    def set_vertex_positions(self, raw: torch.Tensor) -> None:
        raw = raw.detach().to(self.device, torch.float32).contiguous().reshape(-1, 3)
        if raw.shape[0] != self.num_vertices:
            raise RuntimeError("vertex count mismatch")
        self._raw_positions.copy_(raw)
        self._dirty = True

    def set_texels(self, texels: torch.Tensor) -> None:
        t = texels.detach().to(self.device, torch.float32).contiguous()
        if t.numel() != 3 * self.num_texels:
            raise RuntimeError("texel count mismatch")
        check(self._lib.trn_scene_set_texels(self._h, C.c_void_p(t.data_ptr()), C.c_void_p(_stream())),
              "trn_scene_set_texels")

    def configure(self, refit: bool = False) -> None:
        """Scene::Configure (Scene.cpp:522-533): geometry chain + LBVH build, or
        with refit=True Scene::Update: geometry chain + LBVH refit."""
        st = C.c_void_p(_stream())
        check(self._lib.trn_scene_set_translation(self._h, C.c_void_p(self._translation.data_ptr()), st),
              "trn_scene_set_translation")
        # rotated shapes upload their posed positions (kept alive for the copy)
        posed = posed_positions(self._raw_positions, self.shapes)
        self._posed = posed if posed is not None else self._raw_positions
        check(self._lib.trn_scene_set_positions(self._h, C.c_void_p(self._posed.data_ptr()), st),
              "trn_scene_set_positions")
        if refit:
            check(self._lib.trn_scene_refit(self._h, st), "trn_scene_refit")
        else:
            check(self._lib.trn_scene_configure(self._h, st), "trn_scene_configure")
        self._dirty = False

    def _ensure(self) -> None:
        if self._dirty:
            self.configure()

    def get_width(self, i: int = 0) -> int:
        """Scene::GetImageWidth (Scene.h:127): sensor i's image width."""
        return self.cameras[i].width

    def get_height(self, i: int = 0) -> int:
        """Scene::GetImageHeight (Scene.h:128): sensor i's image height."""
        return self.cameras[i].height

    @property
    def num_bsdf(self) -> int:
        """The scene's BSDF count (Scene::mBSDFCount)."""
        return len(self.bsdfs)

    @property
    def emitters(self) -> list:
        """The area lights, one per emitting shape, in shape order
        (Scene::mLights; the reference binds no methods on them)."""
        return [s for s, m in zip(self.shapes, self.spec.meshes) if m.light >= 0]

    @property
    def handle(self):
        return self._h

    def geometry(self) -> dict:
        self._ensure()
        d = self.device
        pos = torch.empty(self.num_vertices, 3, device=d)
        fn = torch.empty(self.num_triangles, 3, device=d)
        ar = torch.empty(self.num_triangles, device=d)
        vn = torch.empty(self.num_vertices, 3, device=d)
        check(self._lib.trn_scene_get_geometry(self._h, C.c_void_p(pos.data_ptr()), C.c_void_p(fn.data_ptr()),
                                               C.c_void_p(ar.data_ptr()), C.c_void_p(vn.data_ptr()),
                                               C.c_void_p(_stream())), "trn_scene_get_geometry")
        return {"positions": pos, "face_normals": fn, "areas": ar, "vertex_normals": vn}

    # -- gradients ---------------------------------------------------------------
    def get_grads(self, clear: bool = True) -> dict:
        """Finish the geometry adjoint and return dL/d(translation per mesh),
        dL/d(raw vertex positions), dL/d(texels) (get_grad, pybind_utils.h:133-142),
        and, when a shape asked for them, dL/d(rotate_angle) per mesh as
        "rotation_angle" (diff_rotation) and dL/d(vertex_translation) per mesh
        as "vertex_translation" (vertex_id)."""
        d = self.device
        gt = torch.zeros(self.num_meshes, 3, device=d)
        gp = torch.zeros(self.num_vertices, 3, device=d)
        gx = torch.zeros(max(1, self.num_texels), 3, device=d)
        check(self._lib.trn_scene_get_grads(self._h, C.c_void_p(gt.data_ptr()), C.c_void_p(gp.data_ptr()),
                                            C.c_void_p(gx.data_ptr()), int(clear), C.c_void_p(_stream())),
              "trn_scene_get_grads")
        out = {"translation": gt, "positions": gp, "texels": gx[: self.num_texels]}
        if any(s._posed() for s in self.shapes):
            out["positions"], d_angle, d_vertex = pose_grads(self._raw_positions, gp, self.shapes)
            if any(s.requires_rotation_grad for s in self.shapes):
                out["rotation_angle"] = d_angle
            if any(s._moves_vertex() for s in self.shapes):
                out["vertex_translation"] = d_vertex
        return out

    def set_path_cache(self, max_bytes: int) -> None:
        """Bound (bytes; 0 = off; default 16 GiB) on the path records that the
        single-view renderC of the interior term keeps for its renderD."""
        self._ensure()
        check(self._lib.trn_scene_path_cache(self.handle, int(max_bytes)), "trn_scene_path_cache")

    def clear_grads(self) -> None:
        check(self._lib.trn_scene_clear_grads(self._h, C.c_void_p(_stream())), "trn_scene_clear_grads")

    def finalize_grads(self, grad_positions: torch.Tensor, grad_vertex_normals: torch.Tensor,
                       d_translation: torch.Tensor | None = None) -> None:
        """Geometry adjoint for caller-owned gradient buffers (one request)."""
        check(self._lib.trn_scene_finalize_grads(self._h, C.c_void_p(grad_positions.data_ptr()),
                                                 C.c_void_p(grad_vertex_normals.data_ptr()),
                                                 C.c_void_p(d_translation.data_ptr()) if d_translation is not None
                                                 else None, C.c_void_p(_stream())), "trn_scene_finalize_grads")

    # -- ray queries (RayIntersectOptix replacement) -------------------------------
    def intersect(self, org: torch.Tensor, dir: torch.Tensor, tmin: torch.Tensor, tmax: torch.Tensor):
        self._ensure()
        n = org.shape[0]
        d = self.device
        org, dir = org.contiguous().float(), dir.contiguous().float()
        tmin, tmax = tmin.contiguous().float(), tmax.contiguous().float()
        tri = torch.empty(n, dtype=torch.int32, device=d)
        u, v, t = (torch.empty(n, device=d) for _ in range(3))
        check(self._lib.trn_intersect(self._h, n, *(C.c_void_p(x.data_ptr()) for x in (org, dir, tmin, tmax, tri,
                                                                                        u, v, t)),
                                      C.c_void_p(_stream())), "trn_intersect")
        return tri, u, v, t

    def occluded(self, org, dir, tmin, tmax) -> torch.Tensor:
        self._ensure()
        n = org.shape[0]
        vis = torch.empty(n, dtype=torch.int32, device=self.device)
        org, dir = org.contiguous().float(), dir.contiguous().float()
        tmin, tmax = tmin.contiguous().float(), tmax.contiguous().float()
        check(self._lib.trn_occluded(self._h, n, *(C.c_void_p(x.data_ptr()) for x in (org, dir, tmin, tmax, vis)),
                                     C.c_void_p(_stream())), "trn_occluded")
        return vis


def _samples_struct(samples: torch.Tensor | None) -> TrnSamples:
    if samples is None:
        return TrnSamples(None, 0)
    if not (samples.is_cuda and samples.dtype == torch.float32 and samples.is_contiguous() and samples.dim() == 2):
        raise RuntimeError("samples must be a contiguous float32 CUDA tensor [dims, slots]")
    return TrnSamples(C.c_void_p(samples.data_ptr()), samples.shape[1])


class Integrator:
    integrator_id = TRN_PATH_TRACER

    def __init__(self):
        self.options: RenderOptions | None = None

    def set_param(self, options: RenderOptions) -> None:
        self.options = options

    def _camera(self, scene: Scene, camera: Camera | None) -> Camera:
        return camera if camera is not None else scene.cameras[0]

    def renderC(self, scene: Scene, options: RenderOptions, samples: torch.Tensor | None = None,
                camera: Camera | None = None, out: torch.Tensor | None = None) -> torch.Tensor:
        """Forward render; returns an (H, W, 3) float32 CUDA image."""
        scene._ensure()
        cam = self._camera(scene, camera)
        img = out if out is not None else torch.empty(cam.height, cam.width, 3, device=scene.device)
        smp = _samples_struct(samples)
        o = options._c()
        check(scene._lib.trn_render_fwd(scene.handle, C.byref(cam.c), C.byref(o), self.integrator_id, C.byref(smp),
                                        C.c_void_p(img.data_ptr()), C.c_void_p(_stream())), "trn_render_fwd")
        return img

    def renderD(self, scene: Scene, options: RenderOptions, dLdI: torch.Tensor,
                samples: torch.Tensor | None = None, camera: Camera | None = None) -> torch.Tensor:
        """Replay the integrator's paths and accumulate parameter gradients for
        dL/dI (H, W, 3); returns the (zero) derivative image like RenderD
        without export_deriv."""
        scene._ensure()
        cam = self._camera(scene, camera)
        g = dLdI.detach().to(scene.device, torch.float32).contiguous()
        if g.numel() != cam.width * cam.height * 3:
            raise RuntimeError("dLdI must have H*W*3 elements")
        smp = _samples_struct(samples)
        o = options._c()
        check(scene._lib.trn_render_grad(scene.handle, C.byref(cam.c), C.byref(o), self.integrator_id, C.byref(smp),
                                         C.c_void_p(g.data_ptr()), C.c_void_p(_stream())), "trn_render_grad")
        return torch.zeros(cam.height, cam.width, 3, device=scene.device)


class PathTracer(Integrator):
    integrator_id = TRN_PATH_TRACER


class PrimaryEdgeIntegrator(Integrator):
    integrator_id = TRN_PRIMARY_EDGE


class DirectEdgeIntegrator(Integrator):
    integrator_id = TRN_DIRECT_EDGE


class IndirectEdgeIntegrator(Integrator):
    integrator_id = TRN_INDIRECT_EDGE


class PixelBoundaryIntegrator(Integrator):
    integrator_id = TRN_PIXEL_EDGE


def sample_dims(integrator_id: int, max_bounces: int, guided: bool = False) -> int:
    """Uniform dimensions one sample slot consumes (see the sample layout in
    the library: camera/edge draws first, then per-bounce light and BSDF draws).
    A guided direct-boundary sample takes one more (the guiding leaf)."""
    D = max_bounces
    return {TRN_PATH_TRACER: 2 + 5 * D, TRN_PRIMARY_EDGE: 2 + 5 * D,
            TRN_DIRECT_EDGE: 3 + 3 * D + (1 if guided else 0),
            TRN_INDIRECT_EDGE: 3 + 8 * max(D - 1, 0), TRN_PIXEL_EDGE: 1 + 5 * D}[integrator_id]


def mesh_edges(faces: np.ndarray) -> np.ndarray:
    """The edge list the library builds for a triangle mesh (trn_mesh_edges,
    ObjMesh::processEdges): int32 rows (v0, v1, f0, f1, v2), v0 < v1, in
    (v0, v1) order. Host-only."""
    lib = _abi.load()
    F = np.ascontiguousarray(np.asarray(faces, np.int32).reshape(-1, 3))
    ip = F.ctypes.data_as(C.POINTER(C.c_int))
    n = lib.trn_mesh_edges(len(F), ip, None, 0)
    _abi.check(-1 if n < 0 else 0, "trn_mesh_edges")
    out = np.empty((n, 5), np.int32)
    if n:
        _abi.check(0 if lib.trn_mesh_edges(len(F), ip, out.ctypes.data_as(C.POINTER(C.c_int)), n) == n else -1,
                   "trn_mesh_edges")
    return out


def sample_slots(integrator_id: int, width: int, height: int, spp: int) -> int:
    n = width * height * spp
    return n // 4 if integrator_id == TRN_PIXEL_EDGE else n


class ViewSet:
    """Many camera views rendered by one persistent launch per integrator.

    Replaces the reference's Python loop over cameras
    (pyTensorRay/renderer_multi_view.py:53-61): images of all views are
    concatenated [npix, 3]; per-view spp and seeds are part of the set."""

    def __init__(self, scene: Scene, cameras: list, spps: list, seeds: list | None = None, views=None):
        n = len(cameras)
        if n == 0 or len(spps) != n:
            raise RuntimeError("ViewSet needs one spp per camera")
        seeds = seeds if seeds is not None else list(range(n))
        if views is None:
            arr = (TrnView * n)()
            for i, (c, sp, sd) in enumerate(zip(cameras, spps, seeds)):
                arr[i] = TrnView(c.c, int(sp), int(sd), -1, 0, 0.0, 0, None, None, None, None, None)
        else:
            arr = views
        self._arr = arr
        self.scene = scene
        self.cameras = list(cameras)
        self.spps = [int(x) for x in spps]
        self._h = C.c_void_p()
        check(scene._lib.trn_viewset_create(scene.handle, n, arr, C.byref(self._h)), "trn_viewset_create")
        npix = C.c_longlong()
        check(scene._lib.trn_viewset_num_pixels(self._h, C.byref(npix)), "trn_viewset_num_pixels")
        self.npix = npix.value
        self.offsets = self._offsets(arr, n)

    @staticmethod
    def _offsets(arr, n: int) -> list:
        """First pixel of each view in the concatenated image, as the library
        places them (set_views): a view's own pixel_offset when it gives one,
        else right after the views before it."""
        offs, pix = [], 0
        for i in range(n):
            v = arr[i]
            off = int(v.pixel_offset) if v.pixel_offset >= 0 else pix
            offs.append(off)
            pix = max(pix, off + int(v.camera.width) * int(v.camera.height))
        return offs

    def __del__(self):
        try:
            if self._h:
                self.scene._lib.trn_viewset_destroy(self._h)
                self._h = C.c_void_p()
        except Exception:
            pass

    def update(self, cameras: list, spps: list, views) -> None:
        """Replace the views (serving loop); `views` is a ctypes TrnView array."""
        self._arr = views
        check(self.scene._lib.trn_viewset_update(self._h, len(cameras), views), "trn_viewset_update")
        npix = C.c_longlong()
        check(self.scene._lib.trn_viewset_num_pixels(self._h, C.byref(npix)), "trn_viewset_num_pixels")
        self.npix = npix.value
        self.offsets = self._offsets(views, len(cameras))
        self.cameras = list(cameras)
        self.spps = [int(x) for x in spps]

    def reserve(self, max_bounces: int = 8) -> None:
        """Allocate the split kernels' round buffers now (about 5.5 GB at
        max_bounces <= 8), so that no later render call of this set allocates
        device memory or synchronises to grow them."""
        check(self.scene._lib.trn_viewset_reserve(self._h, int(max_bounces), C.c_void_p(_stream())),
              "trn_viewset_reserve")

    def set_path_cache(self, max_bytes: int) -> None:
        """Let forward renders of the interior term keep their path records
        (up to max_bytes; 0 = off) for the gradient call of the same paths."""
        check(self.scene._lib.trn_viewset_path_cache(self._h, int(max_bytes)), "trn_viewset_path_cache")

    def slots(self, integrator_id: int) -> int:
        n = sum(c.width * c.height * s for c, s in zip(self.cameras, self.spps))
        return n // 4 if integrator_id == TRN_PIXEL_EDGE else n

    def render(self, integrator_id: int, options: RenderOptions, samples=None, launch: TrnLaunch | None = None,
               out: torch.Tensor | None = None) -> torch.Tensor:
        self.scene._ensure()
        per_view = out is False  # views carry their own image buffers (accumulate)
        img = None if per_view else (out if out is not None else torch.empty(self.npix, 3, device=self.scene.device))
        smp = _samples_struct(samples)
        o = options._c()
        check(self.scene._lib.trn_render_views_fwd(self.scene.handle, self._h, C.byref(o), integrator_id,
                                                   C.byref(smp), C.byref(launch) if launch else None,
                                                   C.c_void_p(img.data_ptr()) if img is not None else None,
                                                   C.c_void_p(_stream())), "trn_render_views_fwd")
        return img

    def render_grad(self, integrator_id: int, options: RenderOptions, dLdI: torch.Tensor, samples=None,
                    launch: TrnLaunch | None = None) -> None:
        self.scene._ensure()
        g = None if dLdI is None else dLdI.contiguous()
        if g is not None and g.numel() != 3 * self.npix:
            raise RuntimeError("dLdI must have npix*3 elements")
        smp = _samples_struct(samples)
        o = options._c()
        check(self.scene._lib.trn_render_views_grad(self.scene.handle, self._h, C.byref(o), integrator_id,
                                                    C.byref(smp), C.byref(launch) if launch else None,
                                                    C.c_void_p(g.data_ptr()) if g is not None else None,
                                                    C.c_void_p(_stream())), "trn_render_views_grad")

    def loss(self, images: torch.Tensor, targets: torch.Tensor, dLdI: torch.Tensor | None = None):
        """Per-view 0.5*|I - T|^2 and dL/dI (one launch for all views)."""
        loss = torch.empty(len(self.cameras), device=self.scene.device)
        check(self.scene._lib.trn_views_loss(self._h, C.c_void_p(images.data_ptr()), C.c_void_p(targets.data_ptr()),
                                             C.c_void_p(dLdI.data_ptr()) if dLdI is not None else None,
                                             C.c_void_p(loss.data_ptr()), C.c_void_p(_stream())), "trn_views_loss")
        return loss

    def view_image(self, images: torch.Tensor, v: int) -> torch.Tensor:
        c = self.cameras[v]
        o = self.offsets[v]
        return images[o:o + c.width * c.height].reshape(c.height, c.width, 3)


def launch_config(block: int = 0, blocks_per_sm: int = 0, chunk: int = 0, round_log2: int = 0) -> TrnLaunch:
    return TrnLaunch(int(block), int(blocks_per_sm), int(chunk), int(round_log2))
