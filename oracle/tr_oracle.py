"""CPU oracle for the trn path-space differentiable renderer (TEST INFRASTRUCTURE).

This module is test infrastructure only: tests, ``__graft_entry__.smoke`` and
``bench.py``'s CPU-baseline leg may import it, as the checker. The product
(tensorray_b200) never imports it.

What it is: a restatement of the reference's tensor-expression integrators in
PyTorch CPU float32 with autograd. The reference (LibTensorRay) builds every
per-ray quantity as a lazy tensor expression with Detach nodes and gets
gradients from its reverse-mode AD over that graph (Tensor.cpp:601-635);
here the same expressions are torch tensors with ``.detach()`` in the same
places and torch autograd plays the part of Tensor::Backward. Functions cite
the reference file:line they restate. Gradients of the GPU's hand-written
adjoint are therefore checked against an independent, automatic derivation.

Differences that are deliberate and shared with the GPU path:
  * ray queries are a brute-force watertight ray/triangle test (Woop et al.
    2013) instead of OptiX (closed; LibTensorRay/Renderer/Optix.cpp:252-305),
    with the closest hit the lexicographic minimum of (t, triangle id);
  * random numbers are read from a [dims, slots] uniform table in which each
    sample slot owns fixed dimensions (camera/edge first, then per-bounce
    light and BSDF draws), instead of per-call cuRAND tensors whose element
    order depends on stream compaction;
  * the edge CDFs keep zero-weight entries instead of compacting the edge
    list first (the same distribution).

  * a boundary sample whose xDotN derivative is not finite contributes
    nothing (_SampleGuard); the reference would turn the whole gradient NaN;
  * square roots are correctly rounded (sqrt_rn), like the GPU's.

Parity status: partly pinned to the reference's own outputs.
  * Pinned by the reference's code: the edge lists (build_edges equals
    ObjMesh::processEdges row for row) and the camera (camera_matrices within
    1e-6 relative of EDX::Camera and the renderer's derived matrices on the
    fixtures, 2e-6 on seeded random cameras). The
    reference's EDXUtil mesh and camera sources are plain C++ and are built
    into oracle/_ref/edx_probe (oracle/edx/Makefile); its outputs on seeded
    inputs are the fixtures in tests/golden/edx_pins.json.
  * Unpinned by the reference's code: the integrators. Their sources cannot
    be built or run here: they need OptiX 7.4 for every ray query and the
    reference's tensor library, whose JIT compiles kernels at run time from
    the reference's source tree and which includes MSVC-only headers (ppl.h
    for concurrency::parallel_for). No reference test pins render outputs.
    The integrators are pinned by closed-form answers (Lambert's polygon
    irradiance for direct light from a quad emitter, a clamped-cosine
    furnace) and by the reference's finite-difference-vs-AD validation
    pattern (Tensor.h:2968-3021) applied to this render path.
"""
from __future__ import annotations

import math

import numpy as np
import torch

SHADOW_EPS = 1e-2   # Config.h:35
CULL_MIN_TRIANGLES = 4096  # scenes this large cull ray queries by triangle clusters
EDGE_EPS = 1e-8     # Config.h:34
EPS = 1e-6          # Config.h:33
RAY_MAX = 1e32
INV_PI = 0.31830988618379067154
PI = 3.14159265358979323846
F32 = torch.float32


# ---------------------------------------------------------------------------
# counter-hash uniform sampler (numpy restatement of the library's sampler)
# ---------------------------------------------------------------------------
def _mix32(x: np.ndarray) -> np.ndarray:
    x = x.astype(np.uint64) & 0xFFFFFFFF
    x ^= x >> 16
    x = (x * 0x7FEB352D) & 0xFFFFFFFF
    x ^= x >> 15
    x = (x * 0x846CA68B) & 0xFFFFFFFF
    x ^= x >> 16
    return x


def hash_uniform(seed: int, term: int, dim: int, slots: np.ndarray) -> np.ndarray:
    s = _mix32(np.array([(seed * 0x9E3779B9 + 0x632BE5AB) & 0xFFFFFFFF], np.uint64))
    s = _mix32(s ^ np.uint64((term * 0x85EBCA6B + 0x1B873593) & 0xFFFFFFFF))
    s = _mix32(s ^ np.uint64((dim * 0xC2B2AE35 + 0x27D4EB2F) & 0xFFFFFFFF))
    h = _mix32(s ^ _mix32((slots.astype(np.uint64) + 0x165667B1) & 0xFFFFFFFF))
    k = (h >> 9).astype(np.float32)
    return ((k + np.float32(0.5)) * np.float32(1.0 / 8388608.0)).astype(np.float32)


def hash_table(seed: int, term: int, dims: int, slots: int, view_seed: int = 0) -> torch.Tensor:
    """The library's hash sampler for one view: the stream seed folds the
    render seed with the view's own seed."""
    stream = (seed * 1000003 + view_seed) & 0xFFFFFFFF
    idx = np.arange(slots, dtype=np.uint64)
    return torch.from_numpy(np.stack([hash_uniform(stream, term, d, idx) for d in range(dims)]))


def uniform_table(seed: int, dims: int, slots: int) -> torch.Tensor:
    """Seeded uniform table clamped to [2^-24, 1 - 2^-24] (the reference draws
    on (0, 1], Tensor.h:2793-2799)."""
    g = torch.Generator().manual_seed(seed)
    t = torch.rand(dims, slots, generator=g, dtype=F32)
    return t.clamp_(2.0 ** -24, 1.0 - 2.0 ** -24)


# ---------------------------------------------------------------------------
# deterministic trigonometry (the library's sincos_det / acos_det, csrc/common.cuh)
# ---------------------------------------------------------------------------
# binary64 evaluation with individually rounded operations, rounded once to
# float32: Cody & Waite reduction by pi/2 plus Taylor polynomials for sin and
# cos, the Maclaurin series of asin for acos. The GPU runs the identical
# sequence of IEEE operations, so sampled directions agree bit for bit.
_PI_D = 3.141592653589793
_PIO2_D = 1.5707963267948966
_TWO_OVER_PI_D = 0.6366197723675814
_SIN_C = (-1.0 / 1307674368000.0, 1.0 / 6227020800.0, -1.0 / 39916800.0, 1.0 / 362880.0, -1.0 / 5040.0,
          1.0 / 120.0, -1.0 / 6.0)
_COS_C = (1.0 / 20922789888000.0, -1.0 / 87178291200.0, 1.0 / 479001600.0, -1.0 / 3628800.0, 1.0 / 40320.0,
          -1.0 / 720.0, 1.0 / 24.0, -0.5)
_ASIN_C = (0.0030578216492580306, 0.003297059503473485, 0.0035692053938259347, 0.003880964558837669,
           0.004240907093679363, 0.004660143486915096, 0.005153309682319905, 0.005740037670841924,
           0.006447210311889649, 0.0073125258735988454, 0.008390335809616815, 0.009761609529194078,
           0.011551800896139705, 0.01396484375, 0.017352764423076924, 0.022372159090909092,
           0.030381944444444444, 0.044642857142857144, 0.075, 0.16666666666666666)


def _horner(c, z2):
    p = np.full_like(z2, c[0])
    for k in c[1:]:
        p = k + z2 * p
    return p


def _np64(x):
    if torch.is_tensor(x):
        x = x.detach().cpu().numpy()
    return np.asarray(x, np.float32).astype(np.float64)


def sincos_det(x):
    """sin and cos of a float32 tensor, bit-identical to the GPU's sincos_det."""
    xd = _np64(x)
    k = np.floor(xd * _TWO_OVER_PI_D + 0.5)
    y = xd - k * _PIO2_D
    y2 = y * y
    sy = y + (y * y2) * _horner(_SIN_C, y2)
    cy = 1.0 + y2 * _horner(_COS_C, y2)
    q = k.astype(np.int64) & 3
    sd = np.select([q == 0, q == 1, q == 2], [sy, cy, -sy], -cy)
    cd = np.select([q == 0, q == 1, q == 2], [cy, -sy, -cy], sy)
    return torch.from_numpy(sd.astype(np.float32)), torch.from_numpy(cd.astype(np.float32))


def acos_det(x):
    """acos of a float32 tensor, bit-identical to the GPU's acos_det."""
    xd = _np64(x)
    a = np.abs(xd)
    with np.errstate(invalid="ignore"):
        lo = np.minimum(a, 0.5)
        t_lo = lo + (lo * (lo * lo)) * _horner(_ASIN_C, lo * lo)
        r_lo = np.where(xd < 0, _PIO2_D + t_lo, _PIO2_D - t_lo)
        z = np.sqrt(np.clip((1.0 - a) * 0.5, 0.0, None))
        z = np.minimum(z, 0.5)
        t_hi = 2.0 * (z + (z * (z * z)) * _horner(_ASIN_C, z * z))
        r_hi = np.where(xd < 0, _PI_D - t_hi, t_hi)
        r = np.where(a <= 0.5, r_lo, r_hi)
        r = np.where(a <= 1.0, r, np.nan)
    return torch.from_numpy(r.astype(np.float32))


# ---------------------------------------------------------------------------
# small vector helpers on [N, 3] tensors
# ---------------------------------------------------------------------------
def sqrt_rn(x):
    """Correctly rounded float32 square root (IEEE 754, as the GPU's sqrtf and
    numpy compute it): torch's vectorised CPU sqrt is off by one ulp on some
    small arguments (e.g. 5.9935515e-11), which flips threshold tests on the
    tiny triangles of a 100K-triangle mesh. The float64 root of a float32
    argument rounds to the correctly rounded float32 root."""
    return torch.sqrt(x.to(torch.float64)).to(x.dtype)


def dot(a, b):
    return a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1] + a[..., 2] * b[..., 2]


def cross(a, b):
    return torch.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1],
                        a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                        a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], -1)


def length(a):
    # VectorLength (Tensor.cpp:695-702): Sqrt(X^2 + Y^2 + Z^2)
    return sqrt_rn(dot(a, a))


def normalize(a):
    # VectorNormalize (Tensor.cpp:684-693)
    return a / length(a)[..., None]


def nan_to_zero(v):
    # NaNToZero (Utils.cpp:273-277)
    ok = torch.isfinite(v).all(-1, keepdim=True)
    return torch.where(ok, v, torch.zeros_like(v))


# ---------------------------------------------------------------------------
# camera (BaseCamera.cpp:45-88, Camera.cpp:89-137, Matrix.cpp:181-220)
# ---------------------------------------------------------------------------
def camera_matrices(pos, target, up, w, h, fov):
    P, T, U = (np.asarray(v, np.float64) for v in (pos, target, up))
    nrm = lambda v: v / np.linalg.norm(v)
    d = nrm(T - P)
    right = nrm(np.cross(nrm(U), d))
    nup = np.cross(d, right)
    cam2world = np.eye(4)
    cam2world[:3, 0], cam2world[:3, 1], cam2world[:3, 2], cam2world[:3, 3] = right, nup, d, P
    view = np.linalg.inv(cam2world)
    near, far = 1.0, 1000.0
    persp = np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, far / (far - near), -far * near / (far - near)],
                      [0, 0, 1, 0]], np.float64)
    it = 1.0 / math.tan(math.radians(fov) / 2.0)
    S = lambda x, y, z: np.diag([x, y, z, 1.0])
    Tr = lambda x, y, z: np.array([[1, 0, 0, x], [0, 1, 0, y], [0, 0, 1, z], [0, 0, 0, 1]], np.float64)
    proj = S(it / (w / h), it, 1.0) @ persp
    s2r = S(w, h, 1.0) @ S(-0.5, -0.5, 1.0) @ Tr(-1.0, -1.0, 0.0)
    r2c = np.linalg.inv(proj) @ np.linalg.inv(s2r)
    c2r = np.linalg.inv(r2c)
    r2w = cam2world @ r2c
    c2s = S(1.0 / w, 1.0 / h, 1.0) @ c2r
    s2c_img = r2c @ S(w, h, 1.0)

    def xf(m, p):
        q = m @ np.array(p, np.float64)
        return q[:3] / q[3]

    v00, v10, v11, vc = (xf(s2c_img, q) for q in ([0, 0, 0, 1], [1, 0, 0, 1], [1, 1, 0, 1], [0.5, 0.5, 0, 1]))
    lx = np.linalg.norm(v00 - v10)
    ly = np.linalg.norm(v11 - v10)
    inv_area = 1.0 / (lx * ly) * float(vc @ vc)
    f = lambda m: np.asarray(m, np.float32)
    return {"pos": f(P), "dir": f(d), "raster_to_camera": f(r2c), "view_inv": f(cam2world),
            "world_to_sample": f(c2s @ view), "sample_to_camera": f(np.linalg.inv(c2s)),
            "raster_to_world": f(r2w), "inv_area": np.float32(inv_area), "plane_len_x": np.float32(lx),
            "plane_len_y": np.float32(ly), "width": w, "height": h}


def camera_ray_dir(cam, ix, iy, sx, sy):
    """GenerateAntitheticRays with the box filter (Camera.cpp:224-277), op
    order fixed so it is bit-identical to the GPU."""
    m = torch.from_numpy(cam["raster_to_camera"]).reshape(-1)
    v = torch.from_numpy(cam["view_inv"]).reshape(-1)
    rx = ix.to(F32) + sx
    ry = iy.to(F32) + sy
    zero = torch.zeros_like(rx)
    row = lambda r: ((m[4 * r] * rx + m[4 * r + 1] * ry) + m[4 * r + 2] * zero) + m[4 * r + 3]
    hx, hy, hz, hw = row(0), row(1), row(2), row(3)
    cx, cy, cz = hx / hw, hy / hw, hz / hw
    ln = sqrt_rn((cx * cx + cy * cy) + cz * cz)
    dx, dy, dz = cx / ln, cy / ln, cz / ln
    vr = lambda r: (v[4 * r] * dx + v[4 * r + 1] * dy) + v[4 * r + 2] * dz
    return torch.stack([vr(0), vr(1), vr(2)], -1)


def xform_point(m, p):
    m = torch.from_numpy(np.asarray(m, np.float32)).reshape(-1)
    x = m[0] * p[..., 0] + m[1] * p[..., 1] + m[2] * p[..., 2] + m[3]
    y = m[4] * p[..., 0] + m[5] * p[..., 1] + m[6] * p[..., 2] + m[7]
    z = m[8] * p[..., 0] + m[9] * p[..., 1] + m[10] * p[..., 2] + m[11]
    w = m[12] * p[..., 0] + m[13] * p[..., 1] + m[14] * p[..., 2] + m[15]
    return torch.stack([x / w, y / w, z / w], -1)


def xform_vector(m, v):
    m = torch.from_numpy(np.asarray(m, np.float32)).reshape(-1)
    return torch.stack([m[0] * v[..., 0] + m[1] * v[..., 1] + m[2] * v[..., 2],
                        m[4] * v[..., 0] + m[5] * v[..., 1] + m[6] * v[..., 2],
                        m[8] * v[..., 0] + m[9] * v[..., 1] + m[10] * v[..., 2]], -1)


def sample_direct(cam, p):
    """Camera::sampleDirect (Camera.cpp:399-416)."""
    q = xform_point(cam["world_to_sample"], p)
    qx, qy = q[:, 0], q[:, 1]
    valid = (qx >= 0) & (qx < 1) & (qy >= 0) & (qy < 1)
    W, H = cam["width"], cam["height"]
    pixel = torch.floor(qy * H).long() * W + torch.floor(qx * W).long()
    cpos = torch.from_numpy(cam["pos"])
    d = p.detach() - cpos
    dist2 = dot(d, d)
    d = d / sqrt_rn(dist2)[:, None]
    cos_t = dot(torch.from_numpy(cam["dir"]).expand_as(d), d)
    ic = 1.0 / cos_t
    sval = 1.0 / dist2 * ic * ic * ic * float(cam["inv_area"])
    return qx, qy, valid, pixel, sval


def sensor_ray_dir(cam, qx, qy):
    cc = xform_point(cam["sample_to_camera"], torch.stack([qx, qy, torch.zeros_like(qx)], -1))
    return xform_vector(cam["view_inv"], normalize(cc))


def image_pixel(cam, qx, qy):
    """WriteToImage with the box filter (Camera.cpp:418-431)."""
    W, H = cam["width"], cam["height"]
    fx, fy = torch.floor(qx * W), torch.floor(qy * H)
    ok = (fx >= 0) & (fx < W) & (fy >= 0) & (fy < H)
    return torch.where(ok, fy.long() * W + fx.long(), torch.full_like(fx, -1).long())


# ---------------------------------------------------------------------------
# edges (ObjMesh::processEdges, ObjMesh.cpp:584-632)
# ---------------------------------------------------------------------------
def build_edges(faces: np.ndarray) -> np.ndarray:
    rows = {}
    order = []
    for i, f in enumerate(faces.tolist()):
        for j in range(3):
            a, b, c = f[j], f[(j + 1) % 3], f[(j + 2) % 3]
            key = (min(a, b), max(a, b))
            if key not in rows:
                rows[key] = [c]
                order.append(key)
            rows[key].append(i)
    out = []
    for key in sorted(rows):
        r = rows[key]
        if len(r) == 3:
            out.append((key[0], key[1], r[1], r[2], r[0]))
        else:
            out.append((key[0], key[1], r[1], -1, r[0]))
    return np.array(out, np.int64).reshape(-1, 5)


def cdf_of(func: torch.Tensor):
    """Distribution1D::SetFunction (Distribution.cpp:45-58): the inclusive
    scan is accumulated in double, scaled by 1/size and normalised."""
    f = func.detach().to(torch.float64)
    n = f.shape[0]
    s = torch.cumsum(f, 0).to(F32) * np.float32(1.0 / n)
    integral = s[-1].clone()
    if integral > 0:
        s = s / integral
    return s, integral


def sample_discrete(cdf, integral, func, u):
    """SampleDiscrete1D (Distribution.cu:37-48) + ReuseSample
    (Distribution.cpp:37-43); returns index, pmf, reused sample."""
    n = cdf.shape[0]
    idx = torch.searchsorted(cdf, u, right=False).clamp(0, n - 1)
    pmf = func.detach()[idx] / (integral * n)
    pmin = torch.where(idx > 0, cdf[(idx - 1).clamp(min=0)], torch.zeros_like(u))
    pmax = cdf[idx]
    reuse = (u - pmin) / (pmax - pmin)
    return idx, pmf, reuse


# ---------------------------------------------------------------------------
# scene (Scene.cpp:46-124, 471-520; Primitive.cpp:134-210, 299-340)
# ---------------------------------------------------------------------------
class OracleScene:
    def __init__(self, spec, requires_grad=("translation",)):
        a = spec.arrays()
        self.spec = spec
        self.raw = torch.from_numpy(a["positions"].copy())
        self.translation = torch.from_numpy(a["mesh_translation"].copy())
        self.texels = (torch.cat([torch.from_numpy(np.ascontiguousarray(t, np.float32)).reshape(-1, 3)
                                  for t in spec.textures]) if spec.textures else torch.zeros(1, 3))
        self.tex_desc = []
        off = 0
        for t in spec.textures:
            self.tex_desc.append((t.shape[1], t.shape[0], off))
            off += t.shape[0] * t.shape[1]
        if "translation" in requires_grad:
            self.translation.requires_grad_(True)
        if "positions" in requires_grad:
            self.raw.requires_grad_(True)
        if "texels" in requires_grad:
            self.texels.requires_grad_(True)
        self.idx = torch.from_numpy(a["indices"].astype(np.int64))
        self.vmesh = torch.from_numpy(a["vertex_mesh"].astype(np.int64))
        tmesh = a["triangle_mesh"].astype(np.int64)
        self.smooth = torch.from_numpy(a["mesh_smooth"][tmesh].astype(bool))
        self.bsdf_id = torch.from_numpy(a["mesh_bsdf"][tmesh].astype(np.int64))
        self.emitter = torch.from_numpy(a["mesh_light"][tmesh].astype(np.int64))
        self.uv = torch.from_numpy(a["uvs"]) if a["uvs"] is not None else None
        self.uvidx = torch.from_numpy(a["uv_indices"].astype(np.int64)) if a["uv_indices"] is not None else None
        self.radiance = torch.from_numpy(a["light_radiance"])
        self.bsdfs = spec.bsdfs
        self.emit_tris = torch.nonzero(self.emitter >= 0).reshape(-1)
        self.tri_to_emit = torch.full((len(self.emitter),), -1, dtype=torch.long)
        self.tri_to_emit[self.emit_tris] = torch.arange(len(self.emit_tris))
        self.edges = torch.from_numpy(build_edges(a["indices"]))
        self.configure()

    def configure(self):
        # Primitive::Configure with a translation parameter: P = raw + t
        self.pos = self.raw + self.translation[self.vmesh]
        p0, p1, p2 = (self.pos[self.idx[:, k]] for k in range(3))
        c = cross(p1 - p0, p2 - p0)
        ln = length(c)
        self.fn = c / ln[:, None]
        self.area = ln * 0.5
        # ComputeVertexNormal: averaged face normals, normalised
        nv = self.pos.shape[0]
        acc = torch.zeros(nv, 3)
        cnt = torch.zeros(nv)
        for k in range(3):
            acc = acc.index_add(0, self.idx[:, k], self.fn)
            cnt = cnt.index_add(0, self.idx[:, k], torch.ones(len(self.idx)))
        self.vn = normalize(acc / cnt[:, None])
        # ConfigureLight: luminance * area over emitter triangles
        lum = (0.212671 * self.radiance[:, 0] + 0.715160 * self.radiance[:, 1] + 0.072169 * self.radiance[:, 2])
        if len(self.emit_tris):
            self.light_func = (lum[self.emitter[self.emit_tris]] * self.area[self.emit_tris]).detach()
            self.light_cdf, self.light_integral = cdf_of(self.light_func)
        # ConstructSecEdgeList (Edge.cpp:42-88), zero weight for non-edges
        e = self.edges
        pa, pb, pc = self.pos[e[:, 0]], self.pos[e[:, 1]], self.pos[e[:, 4]]
        n0 = self.fn[e[:, 2]]
        isb = e[:, 3] < 0
        n1 = torch.where(isb[:, None], torch.zeros(1, 3), self.fn[e[:, 3].clamp(min=0)])
        valid0 = dot(n0, n1) < np.float32(1.0 - 1e-6)
        valid1 = dot(n1, normalize(pc - pa)) < -EDGE_EPS
        valid = isb | (valid0 & valid1)
        self.sec_func = torch.where(valid, length(pb - pa), torch.zeros(len(e))).detach()
        self.sec_cdf, self.sec_integral = cdf_of(self.sec_func)

    def prim_edges(self, cam):
        """ConstructPrimEdgeList (Edge.cpp:313-348), zero weight for non-edges."""
        e = self.edges
        cpos = torch.from_numpy(cam["pos"])
        p0 = self.pos[e[:, 0]]
        ev = cpos - p0
        n0 = self.fn[e[:, 2]]
        isb = e[:, 3] < 0
        n1 = torch.where(isb[:, None], torch.zeros(1, 3), self.fn[e[:, 3].clamp(min=0)])
        ff0, ff1 = dot(ev, n0) > 0, dot(ev, n1) > 0
        valid = isb | (ff0 != ff1)
        func = torch.where(valid, length(self.pos[e[:, 1]] - p0), torch.zeros(len(e))).detach()
        cdf, integral = cdf_of(func)
        return func, cdf, integral

    # --- PostIntersect (Scene.cpp:668-730) ----------------------------------
    def post_intersect(self, tri, u, v):
        w = 1.0 - u - v
        i0, i1, i2 = (self.idx[tri, k] for k in range(3))
        p = w[:, None] * self.pos[i0] + u[:, None] * self.pos[i1] + v[:, None] * self.pos[i2]
        ng = self.fn[tri]
        ns_s = w[:, None] * self.vn[i0] + u[:, None] * self.vn[i1] + v[:, None] * self.vn[i2]
        sm = self.smooth[tri][:, None]
        ns = torch.where(sm, ns_s, ng)
        A = self.area[tri]
        J = A / A.detach()
        if self.uvidx is not None:
            j0, j1, j2 = (self.uvidx[tri, k] for k in range(3))
            uvs = w[:, None] * self.uv[j0] + u[:, None] * self.uv[j1] + v[:, None] * self.uv[j2]
        else:
            uvs = torch.zeros(len(tri), 2)
        return {"p": p, "ng": ng, "ns": ns, "J": J, "uv": uvs.detach(), "tri": tri, "u": u, "v": v,
                "bsdf": self.bsdf_id[tri], "emitter": self.emitter[tri]}

    # --- textures (ImageTexture::Eval, BSDF.cpp:72-98) ----------------------
    def albedo(self, bsdf_index, uv):
        b = self.bsdfs[bsdf_index]
        if b.texture < 0:
            return torch.tensor(b.albedo, dtype=F32).expand(uv.shape[0], 3)
        w, h, off = self.tex_desc[b.texture]
        tu = uv[:, 0] - torch.floor(uv[:, 0])
        tv = uv[:, 1] - torch.floor(uv[:, 1])
        ox = (tu * np.float32(w - 1)).to(torch.int64)
        oy = (tv * np.float32(h - 1)).to(torch.int64)
        return self.texels[off + oy * w + ox]

    # --- merged area light (Light.cpp:134-184) ----------------------------------
    def light_sample(self, s0, s1):
        e, pmf, reuse = sample_discrete(self.light_cdf, self.light_integral, self.light_func, s0)
        t = sqrt_rn(reuse)
        bu = 1.0 - t
        bv = t * s1
        tri = self.emit_tris[e]
        w = 1.0 - bu - bv
        i0, i1, i2 = (self.idx[tri, k] for k in range(3))
        p = w[:, None] * self.pos[i0] + bu[:, None] * self.pos[i1] + bv[:, None] * self.pos[i2]
        A = self.area[tri]
        return {"p": p, "n": self.fn[tri], "J": A / A.detach(), "pdf": (pmf / A.detach()).detach(),
                "light": self.emitter[tri], "tri": tri}

    def light_pdf(self, tri):
        e = self.tri_to_emit[tri]
        pmf = self.light_func[e.clamp(min=0)] / (self.light_integral * len(self.light_func))
        return torch.where(e >= 0, pmf / self.area[tri].detach(), torch.zeros_like(pmf)).detach()

    # --- ray queries --------------------------------------------------------------
    def intersect(self, org, dir, tmin, tmax, any_hit=False):
        p = self.pos.detach()
        P0, P1, P2 = p[self.idx[:, 0]], p[self.idx[:, 1]], p[self.idx[:, 2]]
        if P0.shape[0] < CULL_MIN_TRIANGLES:
            return intersect_brute(P0, P1, P2, org.detach(), dir.detach(), tmin, tmax)
        key = p.data_ptr(), p._version
        if getattr(self, "_clusters_key", None) != key:
            self._clusters = TriangleClusters(P0, P1, P2)
            self._clusters_key = key
        return intersect_culled(self._clusters, P0, P1, P2, org.detach(), dir.detach(), tmin, tmax)

    def occluded(self, org, dir, tmin, tmax):
        tri, _, _, _ = self.intersect(org, dir, tmin, tmax)
        return tri >= 0


def _ray_frame(dir):
    """Per-ray permutation and shear of the watertight test (Woop et al. 2013,
    section 3): kz = the largest |d| axis, kx/ky the others (swapped when
    d[kz] < 0), and the shear constants."""
    n = dir.shape[0]
    ad = dir.abs()
    kz = torch.zeros(n, dtype=torch.long)
    kz = torch.where(ad[:, 1] > ad[:, 0], torch.ones_like(kz), kz)
    m = torch.gather(ad, 1, kz[:, None])[:, 0]
    kz = torch.where(ad[:, 2] > m, torch.full_like(kz, 2), kz)
    kx = (kz + 1) % 3
    ky = (kx + 1) % 3
    dkz = torch.gather(dir, 1, kz[:, None])[:, 0]
    swap = dkz < 0
    kx, ky = torch.where(swap, ky, kx), torch.where(swap, kx, ky)
    g = lambda a, k: torch.gather(a, 1, k[:, None])[:, 0]
    sx = g(dir, kx) / dkz
    sy = g(dir, ky) / dkz
    sz = torch.ones_like(dkz) / dkz
    return kx, ky, kz, sx, sy, sz


def _watertight(A, B, Cc, KX, KY, KZ, SX, SY, SZ, tmin, tmax):
    """The watertight test on triangles given relative to the ray origins
    (A, B, Cc: [..., 3]), with the ray frame broadcast to the same leading
    shape; returns (hit, t, u, v)."""
    gk = lambda X, K: torch.gather(X, -1, K[..., None])[..., 0]
    Akz, Bkz, Ckz = gk(A, KZ), gk(B, KZ), gk(Cc, KZ)
    Ax = gk(A, KX) - SX * Akz
    Ay = gk(A, KY) - SY * Akz
    Bx = gk(B, KX) - SX * Bkz
    By = gk(B, KY) - SY * Bkz
    Cx = gk(Cc, KX) - SX * Ckz
    Cy = gk(Cc, KY) - SY * Ckz
    U = Cx * By - Cy * Bx
    V = Ax * Cy - Ay * Cx
    W = Bx * Ay - By * Ax
    z = (U == 0) | (V == 0) | (W == 0)
    if bool(z.any()):
        d = lambda a: a.double()
        U = torch.where(z, (d(Cx) * d(By) - d(Cy) * d(Bx)).float(), U)
        V = torch.where(z, (d(Ax) * d(Cy) - d(Ay) * d(Cx)).float(), V)
        W = torch.where(z, (d(Bx) * d(Ay) - d(By) * d(Ax)).float(), W)
    neg = (U < 0) | (V < 0) | (W < 0)
    pos = (U > 0) | (V > 0) | (W > 0)
    det = (U + V) + W
    Az, Bz, Cz = SZ * Akz, SZ * Bkz, SZ * Ckz
    Tt = (U * Az + V * Bz) + W * Cz
    rcp = torch.ones_like(det) / det
    t = Tt * rcp
    ok = ~(neg & pos) & (det != 0) & (t > tmin) & (t < tmax)
    return ok, t, V * rcp, W * rcp


def intersect_brute(P0, P1, P2, org, dir, tmin, tmax, chunk=None):
    """Watertight ray/triangle test (Woop, Benthin, Wald, JCGT 2013) against
    every triangle; closest hit = lexicographic min of (t, triangle id)."""
    n = org.shape[0]
    T = P0.shape[0]
    if chunk is None:
        chunk = max(1, min(512, (1 << 22) // max(T, 1)))
    out_tri = torch.full((n,), -1, dtype=torch.long)
    out_u, out_v, out_t = torch.zeros(n), torch.zeros(n), torch.full((n,), -1.0)
    if n == 0:
        return out_tri, out_u, out_v, out_t
    tmin = torch.as_tensor(tmin, dtype=F32).expand(n).contiguous()
    tmax = torch.as_tensor(tmax, dtype=F32).expand(n).contiguous()
    kx, ky, kz, sx, sy, sz = _ray_frame(dir)
    tri_ids = torch.arange(T)
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        o = org[s:e, None, :]
        A, B, Cc = P0[None] - o, P1[None] - o, P2[None] - o
        ex = lambda k: k[s:e, None].expand(-1, T)
        ok, t, uu_all, vv_all = _watertight(A, B, Cc, ex(kx), ex(ky), ex(kz), sx[s:e, None], sy[s:e, None],
                                            sz[s:e, None], tmin[s:e, None], tmax[s:e, None])
        tt = torch.where(ok, t, torch.full_like(t, float("inf")))
        best_t = tt.min(1).values
        cand = ok & (tt == best_t[:, None])
        idx = torch.where(cand, tri_ids[None].expand_as(cand), torch.full_like(cand, T, dtype=torch.long)).min(1).values
        hit = idx < T
        idc = idx.clamp(max=T - 1)
        uu = torch.gather(uu_all, 1, idc[:, None])[:, 0]
        vv = torch.gather(vv_all, 1, idc[:, None])[:, 0]
        out_tri[s:e] = torch.where(hit, idx, torch.full_like(idx, -1))
        out_u[s:e] = torch.where(hit, uu, torch.zeros_like(uu))
        out_v[s:e] = torch.where(hit, vv, torch.zeros_like(vv))
        out_t[s:e] = torch.where(hit, best_t, torch.full_like(best_t, -1.0))
    return out_tri, out_u, out_v, out_t


def _morton3(q):
    """Interleave the low 10 bits of three integer coordinates [n, 3]."""
    key = torch.zeros(q.shape[0], dtype=torch.long)
    for b in range(10):
        for a in range(3):
            key |= ((q[:, a] >> b) & 1) << (3 * b + a)
    return key


class TriangleClusters:
    """Culling structure of the oracle's ray queries: the triangles in
    Morton order of their centroids, cut into clusters of `size`, each with
    a padded float64 box. A ray's candidate triangles are those of the
    clusters whose box it crosses within [tmin, tmax]. The padding (1e-4 of
    the scene extent) and the float64 slab test keep the culling
    conservative, so the exact test over the candidates returns what the
    brute-force test over every triangle returns."""

    def __init__(self, P0, P1, P2, size=64):
        T = P0.shape[0]
        cent = (P0.double() + P1.double() + P2.double()) / 3.0
        lo, hi = cent.min(0).values, cent.max(0).values
        q = ((cent - lo) / (hi - lo).clamp_min(1e-30) * 1023.0).long().clamp(0, 1023)
        order = torch.argsort(_morton3(q), stable=True)
        nc = (T + size - 1) // size
        members = torch.full((nc * size,), -1, dtype=torch.long)
        members[:T] = order
        self.members = members.view(nc, size)
        V = torch.stack([P0, P1, P2], 1).double()[order]            # [T, 3, 3]
        pad_rows = nc * size - T
        if pad_rows:
            V = torch.cat([V, V[-1:].expand(pad_rows, 3, 3)], 0)
        V = V.view(nc, size * 3, 3)
        ext = float((V.amax((0, 1)) - V.amin((0, 1))).max())
        eps = 1e-4 * max(ext, 1e-30) + 1e-12
        self.lo = V.amin(1) - eps
        self.hi = V.amax(1) + eps

    def candidates(self, org, dir, tmin, tmax, chunk=2048):
        """(ray index, triangle index) pairs whose cluster box the ray crosses."""
        rays, tris = [], []
        for s in range(0, org.shape[0], chunk):
            o = org[s:s + chunk].double()[:, None, :]
            d = dir[s:s + chunk].double()[:, None, :]
            with np.errstate(all="ignore"):
                inv = 1.0 / d
                t0 = (self.lo[None] - o) * inv
                t1 = (self.hi[None] - o) * inv
            tn = torch.minimum(t0, t1).nan_to_num(nan=-float("inf"))
            tf = torch.maximum(t0, t1).nan_to_num(nan=float("inf"))
            near = torch.maximum(tn.amax(-1), tmin[s:s + chunk].double()[:, None])
            far = torch.minimum(tf.amin(-1), tmax[s:s + chunk].double()[:, None])
            r, c = torch.nonzero(near <= far * (1 + 1e-9) + 1e-9, as_tuple=True)
            m = self.members[c]                                      # [pairs, size]
            rr = (r + s)[:, None].expand_as(m)
            keep = m >= 0
            rays.append(rr[keep])
            tris.append(m[keep])
        return torch.cat(rays), torch.cat(tris)


def intersect_culled(clusters, P0, P1, P2, org, dir, tmin, tmax):
    """intersect_brute's result (same arithmetic, same (t, id) order) over the
    candidate triangles of TriangleClusters."""
    n = org.shape[0]
    out_tri = torch.full((n,), -1, dtype=torch.long)
    out_u, out_v, out_t = torch.zeros(n), torch.zeros(n), torch.full((n,), -1.0)
    if n == 0:
        return out_tri, out_u, out_v, out_t
    tmin = torch.as_tensor(tmin, dtype=F32).expand(n).contiguous()
    tmax = torch.as_tensor(tmax, dtype=F32).expand(n).contiguous()
    r, tri = clusters.candidates(org, dir, tmin, tmax)
    if r.numel() == 0:
        return out_tri, out_u, out_v, out_t
    kx, ky, kz, sx, sy, sz = _ray_frame(dir)
    o = org[r]
    ok, t, uu, vv = _watertight(P0[tri] - o, P1[tri] - o, P2[tri] - o, kx[r], ky[r], kz[r], sx[r], sy[r], sz[r],
                                tmin[r], tmax[r])
    tt = torch.where(ok, t, torch.full_like(t, float("inf")))
    best_t = torch.full((n,), float("inf")).scatter_reduce(0, r, tt, "amin")
    cand = ok & (tt == best_t[r])
    big = torch.iinfo(torch.long).max
    best_id = torch.full((n,), big, dtype=torch.long).scatter_reduce(
        0, r, torch.where(cand, tri, torch.full_like(tri, big)), "amin")
    hit = best_id < big
    pick = cand & (tri == best_id[r])
    pr = r[pick]
    out_tri[hit] = best_id[hit]
    out_t[hit] = best_t[hit]
    out_u[pr] = uu[pick]
    out_v[pr] = vv[pick]
    return out_tri, out_u, out_v, out_t


# ---------------------------------------------------------------------------
# BSDFs (Diffuse.cpp, Microfacet.cpp, BSDF.cpp)
# ---------------------------------------------------------------------------
def coordinate_system(n):
    """CoordinateSystem (Utils.cpp:118-140)."""
    nx, ny, nz = n[:, 0], n[:, 1], n[:, 2]
    cond = nx.abs() > ny.abs()
    inv_a = 1.0 / sqrt_rn(torch.clamp(nx * nx + nz * nz, min=1e-3))
    inv_b = 1.0 / sqrt_rn(torch.clamp(ny * ny + nz * nz, min=1e-3))
    zero = torch.zeros_like(nx)
    ta = torch.stack([-nz * inv_a, zero, nx * inv_a], -1)
    tb = torch.stack([zero, nz * inv_b, -ny * inv_b], -1)
    t = torch.where(cond[:, None], ta, tb)
    return t, cross(n, t)


def to_local(v, t, b, n):
    return torch.stack([dot(v, t), dot(v, b), dot(v, n)], -1)


def eval_inner(bsdf, kd, wo, wi):
    """Diffuse::EvalInner (Diffuse.cpp:37-41, times the albedo texture as in
    BSDF::Eval) / Microfacet::EvalInner (Microfacet.cpp:37-79)."""
    if bsdf.type == 0:
        reflect = (wo[:, 2] > 0) & (wo[:, 2] * wi[:, 2] > 0)
        return kd * INV_PI * reflect[:, None].to(F32)
    nDotV, nDotL = wo[:, 2], wi[:, 2]
    active = (nDotV > 0) & (nDotL > 0)
    diffuse = kd * INV_PI
    wh = normalize(wo + wi)
    nDotH = wh[:, 2]
    vDotH = dot(wo, wh)
    r = bsdf.roughness
    alpha = np.float32(r * r)
    k = np.float32((r + 1.0) * (r + 1.0) * 0.125)
    tmp = alpha / (nDotH * nDotH * (alpha * alpha - 1.0) + 1.0)
    ggx = tmp * tmp * INV_PI
    coeff = vDotH * (vDotH * -5.55473 - 6.8316)
    e = torch.exp(math.log(2.0) * coeff)
    G = nDotV / (nDotV * (1.0 - k) + k) * (nDotL / (nDotL * (1.0 - k) + k))
    denom = 4.0 * nDotV.abs() * nDotL.abs() + 1e-6
    F0 = torch.tensor(bsdf.specular, dtype=F32)
    spec = (ggx * G / denom)[:, None] * (F0 + (1.0 - F0) * e[:, None])
    val = diffuse + spec
    return torch.where(active[:, None], val, torch.zeros_like(val))


def bsdf_eval(bsdf, frame, ng, kd, wo, wi, correction):
    """BSDF::Eval (BSDF.cpp:172-195)."""
    t, b, n = frame
    lwo, lwi = to_local(wo, t, b, n), to_local(wi, t, b, n)
    v = eval_inner(bsdf, kd, lwo, lwi)
    if correction:
        v = v * (lwo[:, 2] * dot(ng, wi) / (lwi[:, 2] * dot(ng, wo))).abs()[:, None]
    return v


def _tan2(w):
    c2 = w[:, 2] * w[:, 2]
    return torch.clamp(1.0 - c2, min=0.0) / c2


def ggx_D(wh, alpha):
    tan2 = _tan2(wh)
    cos2 = wh[:, 2] * wh[:, 2]
    e = 1.0 / (alpha * alpha) * tan2
    root = alpha * cos2 * (1.0 + e)
    D = INV_PI / (root * root)
    return torch.where(tan2 < 3.402823466e38, D, torch.zeros_like(D))


def smith_G(v, wh, alpha):
    tan2 = _tan2(wh)
    root = alpha * alpha * tan2
    G = 2.0 / (1.0 + sqrt_rn(1.0 + root * root))
    G = torch.where(tan2 < 3.402823466e38, G, torch.zeros_like(G))
    G = torch.where(tan2 == 0, torch.ones_like(G), G)
    return torch.where(dot(v, wh) * v[:, 2] <= 0, torch.zeros_like(G), G)


def vndf_pdf(v, wh, alpha):
    return ggx_D(wh, alpha) * smith_G(v, wh, alpha) * dot(v, wh).abs() / v[:, 2].abs()


def bsdf_pdf_local(bsdf, wo, wi):
    if bsdf.type == 0:
        reflect = (wo[:, 2] > 0) & (wo[:, 2] * wi[:, 2] > 0)
        return torch.where(reflect, wi[:, 2].abs() / PI, torch.zeros_like(wi[:, 2]))
    r = np.float32(bsdf.roughness)
    wh = normalize(wo + wi)
    mp = vndf_pdf(wo, wh, r)
    pdf = (mp * (1.0 / (4.0 * dot(wi, wh)))).abs()
    reflect = (wo[:, 2] > 0) & (mp != 0) & (wi[:, 2] > 0)
    return torch.where(reflect, pdf, torch.zeros_like(pdf))


def cosine_hemisphere(s0, s1):
    """Sampling::CosineSampleHemisphere (Utils.cpp:70-95)."""
    r1, r2 = 2.0 * s0 - 1.0, 2.0 * s1 - 1.0
    cond = (r1 * r1) > (r2 * r2)
    r = torch.where(cond, r1, r2)
    phi = torch.where(cond, 0.78539816339744830962 * (r2 / r1), 1.57079632679489661923 - (r1 / r2) * 0.78539816339744830962)
    zero = (r1 == 0) & (r2 == 0)
    r = torch.where(zero, torch.zeros_like(r), r)
    phi = torch.where(zero, torch.zeros_like(phi), phi)
    sp, cp = sincos_det(phi)
    x, y = r * cp, r * sp
    z = sqrt_rn(torch.clamp(1.0 - x * x - y * y, min=1e-4))
    return torch.stack([x, y, z], -1)


def disk_concentric(s0, s1):
    x, y = 2.0 * s0 - 1.0, 2.0 * s1 - 1.0
    is_zero = (x == 0) & (y == 0)
    q13 = x.abs() < y.abs()
    r = torch.where(q13, y, x)
    rp = torch.where(q13, x, y)
    phi_ = 0.25 * PI * rp / r
    phi = torch.where(is_zero, torch.zeros_like(phi_), torch.where(q13, 0.5 * PI - phi_, phi_))
    sp, cp = sincos_det(phi)
    return r * cp, r * sp


def vndf_sample(v, alpha, s0, s1):
    """GGX_VNDF_Sample / SampleVisible11 (BSDF.cpp:272-302)."""
    V = normalize(torch.stack([v[:, 0] * alpha, v[:, 1] * alpha, v[:, 2]], -1))
    sinT = sqrt_rn(torch.clamp(1.0 - V[:, 2] * V[:, 2], min=0.0))
    sin_phi = torch.where(sinT == 0, torch.zeros_like(sinT), torch.clamp(V[:, 1] / sinT, -1.0, 1.0))
    cos_phi = torch.where(sinT == 0, torch.ones_like(sinT), torch.clamp(V[:, 0] / sinT, -1.0, 1.0))
    ct = V[:, 2]
    px, py = disk_concentric(s0, s1)
    s = 0.5 * (1.0 + ct)
    a = sqrt_rn(torch.clamp(1.0 - px * px, min=0.0))
    y = (1.0 - s) * a + s * py
    z = sqrt_rn(torch.clamp(1.0 - (px * px + py * py), min=0.0))
    st = sqrt_rn(torch.clamp(1.0 - ct * ct, min=0.0))
    norm = 1.0 / (st * y + ct * z)
    slx, sly = (ct * y - st * z) * norm, px * norm
    sx = (cos_phi * slx - sin_phi * sly) * alpha
    sy = (sin_phi * slx + cos_phi * sly) * alpha
    return normalize(torch.stack([-sx, -sy, torch.ones_like(sx)], -1))


def bsdf_sample(bsdf, frame, wo, s0, s1, s2):
    """SampleOnly (Diffuse.cpp:61-76, Microfacet.cpp:127-148), detached."""
    t, b, n = (f.detach() for f in frame)
    lwo = to_local(wo.detach(), t, b, n)
    if bsdf.type == 0:
        lwi = cosine_hemisphere(s0, s1)
        pdf = bsdf_pdf_local(bsdf, lwo, lwi)
    else:
        r = np.float32(bsdf.roughness)
        wh = vndf_sample(lwo, r, s0, s1)
        mp = vndf_pdf(lwo, wh, r)
        nwo = -lwo
        lwi = nwo + wh * (2.0 * dot(-nwo, wh))[:, None]
        reflect = (lwo[:, 2] > 0) & (mp != 0) & (lwi[:, 2] > 0)
        pdf = (mp * (1.0 / (4.0 * dot(lwi, wh)))).abs()
        pdf = torch.where(reflect, pdf, torch.zeros_like(pdf))
    wi = t * lwi[:, 0:1] + b * lwi[:, 1:2] + n * lwi[:, 2:3]
    return wi, pdf


def out_dir_valid(bsdf, ns, ng, w):
    ds, dg = dot(ns, w), dot(ng, w)
    if bsdf.type == 0:
        return (ds > EDGE_EPS) & (dg > EDGE_EPS)
    return ds * dg > 0


# ---------------------------------------------------------------------------
# path state helpers
# ---------------------------------------------------------------------------
def _take(d, m):
    return {k: (v[m] if torch.is_tensor(v) and v.dim() > 0 else v) for k, v in d.items()}


def emitted(scene, surf, wi):
    """AreaLight::Eval (Light.cpp:134-138)."""
    em = surf["emitter"]
    rad = scene.radiance[em.clamp(min=0)]
    on = (em >= 0) & (dot(wi, surf["ng"]) > 0)
    return torch.where(on[:, None], rad, torch.zeros_like(rad))


def radiance_direct(scene, surf, rdir, T, l0, l1, b0, b1, b2):
    """EvalRadianceDirect (Integrator.cpp:178-303) over the active paths.
    Returns (NaN-scrubbed contribution [n,3], keep mask, next surf, next
    rdir, next T) where the next state covers only kept paths."""
    n = rdir.shape[0]
    ret = torch.zeros(n, 3)
    ls = scene.light_sample(l0, l1)
    next_surf, next_dir, next_T, keep_all = [], [], [], torch.zeros(n, dtype=torch.bool)
    order = []
    for bi, bsdf in enumerate(scene.bsdfs):
        m = surf["bsdf"] == bi
        if not bool(m.any()):
            continue
        ids = torch.nonzero(m).reshape(-1)
        sx = _take(surf, m)
        L = _take(ls, m)
        Tm, rd = T[m], rdir[m]
        frame = (*coordinate_system(sx["ns"]), sx["ns"])
        kd = scene.albedo(bi, sx["uv"])
        wo = -rd
        wi = L["p"] - sx["p"]
        d2 = dot(wi, wi)
        d = sqrt_rn(d2)
        wi = wi / d[:, None]
        dotSh, dotGeo = dot(sx["ns"], wi), dot(sx["ng"], wi)
        stable = (d > SHADOW_EPS) & (dotSh.abs() > EDGE_EPS)
        noleak = (dotSh * dotGeo) > 0
        vis = ~scene.occluded(sx["p"].detach(), wi.detach(), SHADOW_EPS, (d - SHADOW_EPS).detach())
        valid = stable & noleak & vis
        G = dot(L["n"], -wi).abs() / d2
        bv = bsdf_eval(bsdf, frame, sx["ng"], kd, wo, wi, False) * dotSh.abs()[:, None]
        Le = torch.where((dot(-wi, L["n"]) > 0)[:, None], scene.radiance[L["light"]], torch.zeros(1, 3))
        val = valid[:, None].to(F32) * Tm * bv * L["J"][:, None] * G[:, None] * Le / L["pdf"][:, None]
        mis_b = (bsdf_pdf_local(bsdf, to_local(wo.detach(), *[f.detach() for f in frame]),
                                to_local(wi.detach(), *[f.detach() for f in frame])) * G.detach())
        pl = L["pdf"]
        mis = (pl * pl / (pl * pl + mis_b * mis_b)).detach()
        val = torch.where(valid[:, None], val * mis[:, None], torch.zeros_like(val))
        # continuation
        wib, pdfb = bsdf_sample(bsdf, frame, wo, b0[m], b1[m], b2[m])
        tri, u, v, _ = scene.intersect(sx["p"], wib, SHADOW_EPS, RAY_MAX)
        hit = (tri >= 0) & (pdfb > 0) & out_dir_valid(bsdf, sx["ns"].detach(), sx["ng"].detach(), wib)
        if bool(hit.any()):
            sh = _take(sx, hit)
            nx = scene.post_intersect(tri[hit], u[hit], v[hit])
            dr = nx["p"] - sh["p"]
            dist2 = dot(dr, dr)
            dr = dr / sqrt_rn(dist2)[:, None]
            Gn = dot(nx["ng"], -dr).abs() / dist2
            fr_h = tuple(f[hit] for f in frame)
            bvn = bsdf_eval(bsdf, fr_h, sh["ng"], kd[hit], wo[hit], dr, False) * dot(sh["ns"], dr).abs()[:, None]
            prev = pdfb[hit].detach() * Gn.detach()
            Tn = Tm[hit] * bvn * Gn[:, None] * nx["J"][:, None] / prev[:, None]
            Tn = torch.where((Gn > 0)[:, None], Tn, torch.zeros_like(Tn))
            # MIS on emitter hits (Integrator.cpp:269-290)
            pe = scene.light_pdf(nx["tri"])
            emis = (prev * prev / (prev * prev + pe * pe)).detach()
            ve = Tn * emitted(scene, nx, -dr) * emis[:, None]
            ve = torch.where((nx["emitter"] >= 0)[:, None], ve, torch.zeros_like(ve))
            add = torch.zeros_like(val).index_put((torch.nonzero(hit).reshape(-1),), ve)
            val = val + add
            gids = ids[hit]
            keep_all[gids] = True
            next_surf.append(nx)
            next_dir.append(dr)
            next_T.append(Tn)
            order.append(gids)
        ret = ret.index_put((ids,), val)
    ret = nan_to_zero(ret)
    if order:
        gids = torch.cat(order)
        perm = torch.argsort(gids)
        cat = lambda key: torch.cat([s[key] for s in next_surf])[perm]
        ns_ = {k: cat(k) for k in next_surf[0]}
        return ret, keep_all, ns_, torch.cat(next_dir)[perm], torch.cat(next_T)[perm]
    return ret, keep_all, None, None, None


def camera_factor(cam, p, ng, J):
    """Camera::EvalFilter with the box filter (Camera.cpp:279-303) times J."""
    cpos = torch.from_numpy(cam["pos"])
    cdir = torch.from_numpy(cam["dir"])
    d = p - cpos
    dist = length(d)
    d = d / dist[:, None]
    cosy = dot(d, cdir.expand_as(d))
    cosx = dot(-d, ng)
    G = cosx.abs() / (cosy * cosy * cosy * (dist * dist))
    return G / G.detach() * J


# ---------------------------------------------------------------------------
# integrators
# ---------------------------------------------------------------------------
def _trace_radiance(scene, surf, rdir, T, smp, slots, base, D):
    """Per-bounce EvalRadianceDirect loop; returns per-path radiance [n,3]."""
    n = rdir.shape[0]
    L = torch.zeros(n, 3)
    alive = torch.arange(n)
    for b in range(D):
        o = base + 5 * b
        s = slots[alive]
        c, keep, ns_, nd, nT = radiance_direct(scene, surf, rdir, T, smp[o][s], smp[o + 1][s], smp[o + 2][s],
                                               smp[o + 3][s], smp[o + 4][s])
        L = L.index_add(0, alive, c)
        if ns_ is None:
            break
        alive = alive[keep]
        nz = (nT != 0).any(-1)
        surf, rdir, T = _take(ns_, nz), nd[nz], nT[nz]
        alive = alive[nz]
        if len(alive) == 0:
            break
    return L


def path_tracer(scene, cam, spp, D, smp):
    """PathTracer::Integrate / Radiance (PathTracer.cpp:37-123) with
    spp_batch = spp. Returns the (H*W, 3) image; differentiable."""
    W, H = cam["width"], cam["height"]
    N = W * H * spp
    slots = torch.arange(N)
    pix = slots % (W * H)
    d = camera_ray_dir(cam, pix % W, pix // W, smp[0][slots], smp[1][slots])
    org = torch.from_numpy(cam["pos"]).expand(N, 3).contiguous()
    tri, u, v, _ = scene.intersect(org, d, SHADOW_EPS, RAY_MAX)
    hit = tri >= 0
    slots, pix = slots[hit], pix[hit]
    surf = scene.post_intersect(tri[hit], u[hit], v[hit])
    T1 = camera_factor(cam, surf["p"], surf["ng"], surf["J"])
    T = T1[:, None].expand(-1, 3)
    rdir = normalize(surf["p"] - torch.from_numpy(cam["pos"]))
    img = torch.zeros(W * H, 3)
    img = img.index_add(0, pix, nan_to_zero(T * emitted(scene, surf, -rdir)))
    L = _trace_radiance(scene, surf, rdir, T, smp, slots, 2, D)
    img = img.index_add(0, pix, L)
    return img * (1.0 / spp)


def _edge_point(scene, func, cdf, integral, r0, r1=None):
    e, pmf, reuse = sample_discrete(cdf, integral, func, r0)
    E = scene.edges[e]
    pa, pb, pc = scene.pos[E[:, 0]], scene.pos[E[:, 1]], scene.pos[E[:, 4]]
    s = reuse if r1 is None else r1
    p0 = pa + s[:, None] * (pb - pa)
    pdf = pmf / func[e]
    return {"e": e, "E": E, "p0": p0, "pdf": pdf.detach(), "edge": normalize(pb - pa).detach(),
            "edge2": normalize(pc.detach() - pa.detach())}


def _base_val(ratio, edge, d, nrm, edge2):
    e = cross(edge, d)
    sinphi = length(e)
    proj = normalize(cross(e, nrm))
    sinphi2 = length(cross(d, proj))
    n = normalize(cross(nrm, proj)).detach()
    sign0 = dot(e, edge2) > 0
    sign1 = dot(e, n) > 0
    bv = ratio * (sinphi / sinphi2)
    bv = bv * (sinphi > EPS).to(F32) * (sinphi2 > EPS).to(F32)
    return bv * torch.where(sign0 == sign1, torch.ones_like(bv), -torch.ones_like(bv)), n


def ray_intersect_ad(d, org, p0, e1, e2):
    """RayIntersectAD (Utils.cpp:288-297)."""
    h = cross(d, e2)
    f = 1.0 / dot(e1, h)
    s = org - p0
    u = f * dot(s, h)
    q = cross(s, e1)
    v = f * dot(d, q)
    return u, v


class _SampleGuard(torch.autograd.Function):
    """Identity on per-sample rows; in the backward pass a sample (row) whose
    gradient is not finite in any of the inputs contributes zero to all of
    them. The CUDA path skips such a sample's xDotN scatter (a line parallel
    to the far triangle, or a receiver on the edge point); the reference has
    no guard there and would turn the whole gradient into NaN."""

    @staticmethod
    def forward(ctx, *xs):
        return tuple(x.clone() for x in xs)

    @staticmethod
    def backward(ctx, *gs):
        bad = None
        for g in gs:
            if g is not None:
                b = ~torch.isfinite(g).all(-1)
                bad = b if bad is None else bad | b
        if bad is None or not bool(bad.any()):
            return gs
        return tuple(None if g is None else torch.where(bad[:, None], torch.zeros_like(g), g) for g in gs)


def _xdotn(scene, org, target, tri, n):
    i0, i1, i2 = (scene.idx[tri, k] for k in range(3))
    P0, P1, P2 = scene.pos[i0], scene.pos[i1], scene.pos[i2]
    org, target, P0, P1, P2 = _SampleGuard.apply(org, target, P0, P1, P2)
    u, v = ray_intersect_ad(normalize(target - org), org, P0, P1 - P0, P2 - P0)
    w = 1.0 - u - v
    u2 = w[:, None] * P0.detach() + u[:, None] * P1.detach() + v[:, None] * P2.detach()
    return dot(n, u2)


def primary_edge(scene, cam, spp, D, smp):
    """PrimaryBoundaryIntegrator::Integrate (BoundaryPrimary.cpp:36-181).
    Returns the boundary image Detach(radiance*baseVal/pdf)*xDotN/spp."""
    W, H = cam["width"], cam["height"]
    N = W * H * spp
    img = torch.zeros(W * H, 3)
    func, cdf, integral = scene.prim_edges(cam)
    if not integral > 0:
        return img
    slots = torch.arange(N)
    es = _edge_point(scene, func, cdf, integral, smp[0][slots], smp[1][slots])
    cpos = torch.from_numpy(cam["pos"])
    p0 = es["p0"]
    d = normalize(p0.detach() - cpos)
    tri, u, v, t = scene.intersect(p0.detach(), d, SHADOW_EPS, RAY_MAX)
    ok = tri >= 0
    hitP = p0.detach() + t[:, None] * d
    qx, qy, valid, _, sval = sample_direct(cam, hitP)
    ok = ok & valid
    dirc = sensor_ray_dir(cam, qx, qy)
    d2c = length(p0.detach() - cpos)
    occ = scene.occluded(cpos.expand(N, 3).contiguous(), dirc, SHADOW_EPS, d2c - SHADOW_EPS)
    ok = ok & ~occ
    m = torch.nonzero(ok).reshape(-1)
    if len(m) == 0:
        return img
    surf = scene.post_intersect(tri[m], u[m], v[m])
    dist = length(surf["p"] - cpos)
    dist1 = length(p0[m] - cpos)
    cos2 = dot(surf["ng"], -dirc[m]).abs()
    bval, n = _base_val(dist / dist1, es["edge"][m], dirc[m], surf["ng"], es["edge2"][m])
    bval = bval * cos2
    T = sval[m][:, None].expand(-1, 3)
    L = nan_to_zero(T * emitted(scene, surf, -dirc[m]))
    L = L + _trace_radiance(scene, surf, dirc[m], T, smp, slots[m], 2, D)
    xdn = _xdotn(scene, cpos.expand(len(m), 3), p0[m], tri[m], n)
    term = (L * (bval / es["pdf"][m])[:, None]).detach() * xdn[:, None]
    pix = image_pixel(cam, qx[m], qy[m])
    okp = pix >= 0
    return img.index_add(0, pix[okp], term[okp] * (1.0 / spp))


def importance_step(scene, cam, surf, rdir, T, b0, b1, b2):
    """EvalImportance (Integrator.cpp:75-176), detached; returns contribution,
    pixel (or -1), keep mask and next state."""
    n = rdir.shape[0]
    cpos = torch.from_numpy(cam["pos"])
    qx, qy, valid, _, sval = sample_direct(cam, surf["p"].detach())
    dirc = sensor_ray_dir(cam, qx, qy)
    d2c = length(surf["p"].detach() - cpos)
    vis = valid & ~scene.occluded(cpos.expand(n, 3).contiguous(), dirc, SHADOW_EPS, d2c - SHADOW_EPS)
    contrib = torch.zeros(n, 3)
    keep = torch.zeros(n, dtype=torch.bool)
    nxt_T = torch.zeros(n, 3)
    nxt_dir = torch.zeros(n, 3)
    nxt = {"tri": torch.full((n,), -1, dtype=torch.long), "u": torch.zeros(n), "v": torch.zeros(n)}
    for bi, bsdf in enumerate(scene.bsdfs):
        m = surf["bsdf"] == bi
        if not bool(m.any()):
            continue
        sx = {k: (v.detach() if torch.is_tensor(v) and v.dtype == F32 else v) for k, v in _take(surf, m).items()}
        frame = (*coordinate_system(sx["ns"]), sx["ns"])
        kd = scene.albedo(bi, sx["uv"]).detach()
        wo = -rdir[m]
        wi = normalize(cpos - sx["p"])
        wo_ok = out_dir_valid(bsdf, sx["ns"], sx["ng"], wo)
        wi_ok = out_dir_valid(bsdf, sx["ns"], sx["ng"], wi)
        val = bsdf_eval(bsdf, frame, sx["ng"], kd, wo, wi, True) * dot(sx["ns"], wi).abs()[:, None]
        val = torch.where((wo_ok & wi_ok)[:, None], val, torch.zeros_like(val))
        c = T[m] * sval[m][:, None] * val
        contrib[m] = torch.where(vis[m][:, None], c, torch.zeros_like(c))
        wib, pdf = bsdf_sample(bsdf, frame, wo, b0[m], b1[m], b2[m])
        bv = bsdf_eval(bsdf, frame, sx["ng"], kd, wo, wib, True) * dot(sx["ns"], wib).abs()[:, None]
        Tn = T[m] * bv / pdf[:, None]
        tri, u, v, _ = scene.intersect(sx["p"], wib, SHADOW_EPS, RAY_MAX)
        ok = wo_ok & (pdf > 0) & out_dir_valid(bsdf, sx["ns"], sx["ng"], wib) & (tri >= 0)
        ids = torch.nonzero(m).reshape(-1)
        keep[ids] = ok
        nxt_T[ids] = Tn
        nxt_dir[ids] = wib
        nxt["tri"][ids] = tri
        nxt["u"][ids] = u
        nxt["v"][ids] = v
    contrib = nan_to_zero(contrib)
    pix = torch.where(vis, image_pixel(cam, qx, qy), torch.full((n,), -1, dtype=torch.long))
    if bool(keep.any()):
        ns_ = scene.post_intersect(nxt["tri"][keep], nxt["u"][keep], nxt["v"][keep])
        ns_ = {k: (v.detach() if torch.is_tensor(v) and v.dtype == F32 else v) for k, v in ns_.items()}
        return contrib, pix, keep, ns_, nxt_dir[keep], nxt_T[keep]
    return contrib, pix, keep, None, None, None


GUIDE_TERM = 5  # hash-sampler term of the guiding set-up samples


def _guide_base_val(scene, x, y, z):
    """|baseVal| of EvalBoundarySegmentDirect in guiding mode (Edge.cpp:201-259
    with guiding_mode=true): the sample-stage mask of SampleBoundarySegmentDirect
    is replaced by the evaluation mask (same point, both rays hit), and the
    value is |baseVal| without radiance or pdf. Invalid samples give 0."""
    es = _edge_point(scene, scene.sec_func, scene.sec_cdf, scene.sec_integral, x)
    ls = scene.light_sample(y, z)
    p0, p2, nL = es["p0"].detach(), ls["p"].detach(), ls["n"].detach()
    rdir = normalize(p0 - p2)
    tri0, _, _, t0 = scene.intersect(p0, -rdir, SHADOW_EPS, RAY_MAX)
    tri, u, v, _ = scene.intersect(p0, rdir, SHADOW_EPS, RAY_MAX)
    hp = p0 + t0[:, None] * (-rdir)
    ok = (length(hp - p2) < SHADOW_EPS) & (tri0 >= 0) & (tri >= 0)
    out = torch.zeros(x.shape[0])
    m = torch.nonzero(ok).reshape(-1)
    if len(m) == 0:
        return out
    surf = scene.post_intersect(tri[m], u[m], v[m])
    xp = surf["p"].detach()
    dl = length(p2[m] - xp)
    cos2 = dot(nL[m], rdir[m]).abs()
    its_t = length(xp - p0[m])
    bval, _ = _base_val(its_t / dl, es["edge"][m], -rdir[m], nL[m], es["edge2"][m])
    bval = (bval * cos2).abs()
    out[m] = torch.where(torch.isfinite(bval), bval, torch.zeros_like(bval))
    return out


REFINE_TERM = 6   # hash-sampler term of the refinement's random points
AQ_POINTS = 36


def _f32(x):
    return np.asarray(x, np.float32)


def _aq_points(box, stream):
    """The 36 evaluation points of every leaf for one refinement pass
    (gen_eval_point, NEE.cu:91-240, with the box midpoint m = (p0 + p1) / 2):
    corners and edge midpoints of the x = p0 and x = p1 faces (0-15), corners
    of the x = m section (16-19), two random points per octant (20-35; octant
    bits x, y, z = bits 2, 1, 0 of k - 20; the second eight use 1 - r).
    box is [6, n] float32; returns [n, 36, 3] float32."""
    lo, hi = box[0:3], box[3:6]
    mid = _f32((lo + hi) * np.float32(0.5))
    n = lo.shape[1]
    pts = np.zeros((n, AQ_POINTS, 3), np.float32)
    sel = [lo, hi, mid]
    yz16 = [(0, 0), (0, 1), (0, 2), (1, 0), (1, 1), (1, 2), (2, 0), (2, 1)]
    yz4 = [(0, 0), (0, 1), (1, 0), (1, 1)]
    for k in range(20):
        sx = 0 if k < 8 else (1 if k < 16 else 2)
        yz = yz16[k & 7] if k < 16 else yz4[k - 16]
        pts[:, k, 0] = sel[sx][0]
        pts[:, k, 1] = sel[yz[0]][1]
        pts[:, k, 2] = sel[yz[1]][2]
    half = _f32(mid - lo)
    leaves = np.arange(n, dtype=np.uint64)
    for k in range(20, 36):
        o = (k - 20) & 7
        for a in range(3):
            r = hash_uniform(stream, REFINE_TERM, 3 * (k - 20) + a, leaves)
            if k >= 28:
                r = _f32(np.float32(1.0) - r)
            base = mid[a] if (o >> (2 - a)) & 1 else lo[a]
            pts[:, k, a] = _f32(base + _f32(half[a] * r))
    return pts


def _avg8(e, idx):
    s = _f32(e[:, idx[0]] + e[:, idx[1]])
    for j in idx[2:]:
        s = _f32(s + e[:, j])
    return _f32(s / np.float32(8.0))


def _aq_refine(box, edge, ev, thold, stream, limit):
    """One cut_tree pass (NEE.cu:243-396): split the leaves whose corner and
    Monte Carlo averages disagree by more than thold (times the box volume)
    along the axis whose halves disagree most (a random axis on ties). New
    leaves take the upper half and are appended in leaf order, up to `limit`."""
    n = box.shape[1]
    vol = _f32(_f32(_f32(box[3] - box[0]) * _f32(box[4] - box[1])) * _f32(box[5] - box[2]))
    lag = _avg8(ev, [0, 1, 3, 4, 8, 9, 11, 12])
    mc = np.zeros(n, np.float32)
    for k in range(20, 36):
        mc = _f32(mc + ev[:, k])
    mc = _f32(mc / np.float32(16.0))
    err = _f32(np.abs(_f32(lag - mc)) * vol)
    split = err > np.float32(thold)
    ad = lambda a, b: np.abs(_f32(a - b))
    e0 = np.abs(_f32(ad(_avg8(ev, [0, 1, 3, 4, 16, 17, 18, 19]), _avg8(ev, [20, 21, 22, 23, 28, 29, 30, 31])) -
                     ad(_avg8(ev, [8, 9, 11, 12, 16, 17, 18, 19]), _avg8(ev, [24, 25, 26, 27, 32, 33, 34, 35]))))
    e1 = np.abs(_f32(ad(_avg8(ev, [0, 1, 6, 7, 8, 9, 14, 15]), _avg8(ev, [20, 21, 24, 25, 28, 29, 32, 33])) -
                     ad(_avg8(ev, [3, 4, 6, 7, 11, 12, 14, 15]), _avg8(ev, [22, 23, 26, 27, 30, 31, 34, 35]))))
    e2 = np.abs(_f32(ad(_avg8(ev, [0, 2, 3, 5, 8, 10, 11, 13]), _avg8(ev, [20, 22, 24, 26, 28, 30, 32, 34])) -
                     ad(_avg8(ev, [1, 2, 4, 5, 9, 10, 12, 13]), _avg8(ev, [21, 23, 25, 27, 29, 31, 33, 35]))))
    r = _f32(hash_uniform(stream, REFINE_TERM, 48, np.arange(n, dtype=np.uint64)) * np.float32(3.0))
    axis = np.where(r < 1.0, 0, np.where(r < 2.0, 1, 2))
    axis = np.where((e2 > e0) & (e2 > e1), 2, axis)
    axis = np.where((e1 > e0) & (e1 > e2), 1, axis)
    axis = np.where((e0 > e1) & (e0 > e2), 0, axis)
    new_box, new_edge = [], []
    box = box.copy()
    for leaf in np.nonzero(split)[0]:
        if n + len(new_box) >= limit:
            break
        a = axis[leaf]
        mid = _f32((box[a, leaf] + box[3 + a, leaf]) * np.float32(0.5))
        nb = box[:, leaf].copy()
        nb[a] = mid
        box[3 + a, leaf] = mid
        new_box.append(nb)
        new_edge.append(edge[leaf])
    if new_box:
        box = np.concatenate([box, np.stack(new_box, 1)], 1)
        edge = np.concatenate([edge, np.array(new_edge, edge.dtype)])
    return box, edge


def aq_guide(scene, seed, g_spp, eps, depth=0, max_size=100000, thold=0.01):
    """AdaptiveQuadratureDistribution::setup (AQ_distrb.h:83-173). The depth-0
    tree (build_tree, NEE.cu:70-89) has one leaf per secondary edge, box
    [cdf[i-1], cdf[i]] x [0,1] x [0,1] of the (edge, light) sample cube.
    `depth` refinement passes then evaluate 36 points per leaf and split
    leaves (the loop the reference keeps commented out, AQ_distrb.h:121-136;
    see _aq_points, _aq_refine); the tree holds at most max(E, max_size)
    leaves. The leaf weight is the mean |baseVal| of g_spp uniform samples in
    the box, normalised to sum 1, mixed with eps, and the leaf distribution is
    weight x box volume. Leaves on non-secondary edges (zero length in the
    edge distribution) get weight 0 and zero volume, as if absent.
    Returns a dict: box [6, n], poly, cdf, integral, fsum (sum of weight x
    volume)."""
    E = scene.edges.shape[0]
    cdf = scene.sec_cdf.numpy().astype(np.float32)
    box = np.zeros((6, E), np.float32)
    box[0, 1:] = cdf[:-1]
    box[3] = cdf
    box[4] = 1.0
    box[5] = 1.0
    edge = np.arange(E)
    efunc = scene.sec_func.detach().numpy()
    live_scene = float(scene.sec_integral) > 0
    stream = (seed * 1000003) & 0xFFFFFFFF
    limit = max(E, max_size) if depth > 0 else E
    for p in range(depth):
        ps = (stream + p) & 0xFFFFFFFF
        pts = _aq_points(box, ps)
        n = box.shape[1]
        flat = torch.from_numpy(pts.reshape(-1, 3))
        live = np.repeat((efunc[edge] > 0) & live_scene, AQ_POINTS)
        ev = np.zeros(n * AQ_POINTS, np.float32)
        if live.any():
            m = np.nonzero(live)[0]
            ev[m] = _guide_base_val(scene, flat[m, 0], flat[m, 1], flat[m, 2]).numpy()
        box, edge = _aq_refine(box, edge, ev.reshape(n, AQ_POINTS), thold, ps, limit)
    n = box.shape[1]
    live = torch.from_numpy((efunc[edge] > 0) & live_scene)
    tb = torch.from_numpy(box)
    poly = torch.zeros(n)
    leaf = torch.arange(n)
    for k in range(g_spp):
        slot = (leaf * g_spp + k).numpy().astype(np.uint64)
        r = [torch.from_numpy(hash_uniform(stream, GUIDE_TERM, d, slot)) for d in range(3)]
        x = tb[0] + r[0] * (tb[3] - tb[0])
        y = tb[1] + r[1] * (tb[4] - tb[1])
        z = tb[2] + r[2] * (tb[5] - tb[2])
        bv = _guide_base_val(scene, x, y, z)
        poly = poly + torch.where(live, bv, torch.zeros_like(bv)) / np.float32(g_spp)
    tot = float(poly.double().sum())
    if tot > 0:
        poly = poly / np.float32(tot)
    poly = np.float32(eps) + np.float32(1.0 - eps) * poly
    vol = ((tb[3] - tb[0]) * (tb[4] - tb[1])) * (tb[5] - tb[2])
    func = poly * vol
    gcdf, gint = cdf_of(func)
    fsum = torch.tensor(float(func.double().sum()), dtype=F32)
    return {"box": tb, "edge": torch.from_numpy(edge), "poly": poly, "cdf": gcdf, "integral": gint, "fsum": fsum}


def direct_edge(scene, cam, spp, D, smp, guide=None):
    """DirectBoundaryIntegrator::Integrate (BoundaryDirect.cpp:38-143,
    Edge.cpp:90-144, 201-309). With guide = aq_guide(...) the (edge, light)
    sample comes from the leaf distribution (AdaptiveQuadratureDistribution::sample,
    AQ_distrb.h:176-195): a leaf by the extra uniform of dimension 3+3D, then a
    point uniform in its box; the sample pdf is multiplied by weight/sum."""
    W, H = cam["width"], cam["height"]
    N = W * H * spp
    img = torch.zeros(W * H, 3)
    if not scene.sec_integral > 0:
        return img
    slots = torch.arange(N)
    r0 = smp[0][slots]
    pdf_b = torch.ones(N)
    r1, r2 = smp[1][slots], smp[2][slots]
    if guide is not None:
        gcdf = guide["cdf"]
        if not guide["integral"] > 0:
            return img
        leaf = torch.searchsorted(gcdf, smp[3 + 3 * D][slots], right=False).clamp(0, gcdf.shape[0] - 1)
        b = guide["box"][:, leaf]
        r0 = b[0] + r0 * (b[3] - b[0])
        r1 = b[1] + r1 * (b[4] - b[1])
        r2 = b[2] + r2 * (b[5] - b[2])
        pdf_b = guide["poly"][leaf] / guide["fsum"]
    es = _edge_point(scene, scene.sec_func, scene.sec_cdf, scene.sec_integral, r0)
    ls = scene.light_sample(r1, r2)
    p0, p2, nL = es["p0"], ls["p"], ls["n"]
    ev = p2.detach() - p0.detach()
    dsq = dot(ev, ev)
    dist = sqrt_rn(dsq)
    en = ev / dist[:, None]
    cos_t = dot(nL.detach(), -en)
    E = es["E"]
    n0 = scene.fn[E[:, 2]].detach()
    isb = E[:, 3] < 0
    n1 = torch.where(isb[:, None], torch.zeros(1, 3), scene.fn[E[:, 3].clamp(min=0)].detach())
    c0, c1 = dot(en, n0), dot(en, n1)
    v0 = c0.abs() > EDGE_EPS
    v1 = ((c0 > EDGE_EPS) & (c1 < -EDGE_EPS)) | ((c0 < -EDGE_EPS) & (c1 > EDGE_EPS))
    right = (isb & v0) | (~isb & v1)
    ok = right & (cos_t > EPS) & (dist > SHADOW_EPS)
    pdf = es["pdf"] * ls["pdf"] * dsq / cos_t * pdf_b
    rdir = normalize(p0.detach() - p2.detach())
    tri0, u0, v0_, t0 = scene.intersect(p0.detach(), -rdir, SHADOW_EPS, RAY_MAX)
    tri, u, v, _ = scene.intersect(p0.detach(), rdir, SHADOW_EPS, RAY_MAX)
    hp = p0.detach() + t0[:, None] * (-rdir)
    same = length(hp - p2.detach()) < SHADOW_EPS
    ok = ok & same & (tri0 >= 0) & (tri >= 0)
    m = torch.nonzero(ok).reshape(-1)
    if len(m) == 0:
        return img
    sl = scene.post_intersect(tri0[m], u0[m], v0_[m])
    Em = emitted(scene, {k: (v.detach() if torch.is_tensor(v) and v.dtype == F32 else v) for k, v in sl.items()},
                 rdir[m])
    surf = scene.post_intersect(tri[m], u[m], v[m])
    dl = length(p2[m].detach() - surf["p"].detach())
    cos2 = dot(nL[m].detach(), rdir[m]).abs()
    its_t = length(surf["p"].detach() - p0[m].detach())
    bval, n = _base_val(its_t / dl, es["edge"][m], -rdir[m], nL[m].detach(), es["edge2"][m])
    bval = bval * cos2
    xdn = _xdotn(scene, surf["p"], p0[m], tri0[m], n)
    value0 = (Em * (bval / pdf[m])[:, None]).detach() * xdn[:, None]
    # trace towards the sensor
    sdet = {k: (v.detach() if torch.is_tensor(v) and v.dtype == F32 else v) for k, v in surf.items()}
    T = torch.ones(len(m), 3)
    rd = rdir[m]
    alive = torch.arange(len(m))
    s_all = slots[m]
    for b in range(D):
        o = 3 + 3 * b
        s = s_all[alive]
        c, pix, keep, ns_, nd, nT = importance_step(scene, cam, sdet, rd, T, smp[o][s], smp[o + 1][s], smp[o + 2][s])
        okp = pix >= 0
        if bool(okp.any()):
            img = img.index_add(0, pix[okp], (value0[alive][okp] * c[okp]) * (1.0 / spp))
        if ns_ is None:
            break
        alive = alive[keep]
        sdet, rd, T = ns_, nd, nT
    return img - img.detach()


def indirect_edge(scene, cam, spp, D, smp):
    """IndirectBoundaryIntegrator::Integrate (BoundaryIndirect.cpp:38-192,
    Edge.cpp:146-199)."""
    W, H = cam["width"], cam["height"]
    N = W * H * spp
    img = torch.zeros(W * H, 3)
    if D < 2 or not scene.sec_integral > 0:
        return img
    slots = torch.arange(N)
    es = _edge_point(scene, scene.sec_func, scene.sec_cdf, scene.sec_integral, smp[0][slots])
    E = es["E"]
    r1, r2 = smp[1][slots], smp[2][slots]
    n0 = scene.fn[E[:, 2]].detach()
    isb = E[:, 3] < 0
    n1 = scene.fn[E[:, 3].clamp(min=0)].detach()
    edge = es["edge"]
    # boundary edges: uniform sphere around cross(n0, edge)
    nrm = cross(n0, edge)
    tg, bt = coordinate_system(nrm)
    z = torch.clamp(1.0 - 2.0 * r1, max=np.float32(1.0 - EDGE_EPS))
    r = sqrt_rn(torch.clamp(1.0 - z * z, min=0.0))
    phi = 2.0 * PI * r2
    sp, cp = sincos_det(phi)
    dir_b = tg * (r * cp)[:, None] + bt * (r * sp)[:, None] + nrm * z[:, None]
    # interior edges: two-sided wedge
    phi0 = acos_det(dot(n0, n1))
    zz = normalize(n0 + n1)
    yy = normalize(cross(n0, zz))
    xx = cross(yy, zz)
    ph = (r1 - 0.5) * phi0
    ph = torch.minimum(torch.maximum(ph, -0.5 * phi0 + EDGE_EPS), 0.5 * phi0 - EDGE_EPS)
    sp, cp = sincos_det(ph)
    x1 = xx * cp[:, None] + zz * sp[:, None]
    m0 = r2 > 0.5
    bq = 4.0 * r2 - torch.where(m0, torch.full_like(r2, 3.0), torch.ones_like(r2))
    aq = sqrt_rn(1.0 - bq * bq) * (1.0 - m0.to(F32) * 2.0)
    dir_i = x1 * aq[:, None] + yy * bq[:, None]
    dirv = torch.where(isb[:, None], dir_b, dir_i).detach()
    pdf_d = torch.where(isb, torch.full_like(r1, 0.25 / PI), 0.25 / phi0)
    pdf = es["pdf"] * pdf_d.detach()
    p0 = es["p0"]
    te, ue, ve, _ = scene.intersect(p0.detach(), -dirv, SHADOW_EPS, RAY_MAX)
    ts, us, vs, _ = scene.intersect(p0.detach(), dirv, SHADOW_EPS, RAY_MAX)
    m = torch.nonzero((te >= 0) & (ts >= 0)).reshape(-1)
    if len(m) == 0:
        return img
    xe = scene.post_intersect(te[m], ue[m], ve[m])
    xs = scene.post_intersect(ts[m], us[m], vs[m])
    dl = length(xe["p"].detach() - xs["p"].detach())
    cos2 = dot(xe["ng"].detach(), dirv[m]).abs()
    its_t = length(xs["p"].detach() - p0[m].detach())
    bval, n = _base_val(its_t / dl, edge[m], -dirv[m], xe["ng"].detach(), es["edge2"][m])
    bval = bval * cos2
    xdn = _xdotn(scene, xs["p"], p0[m], te[m], n)
    value0 = (bval / pdf[m]).detach() * xdn
    det = lambda d: {k: (v.detach() if torch.is_tensor(v) and v.dtype == F32 else v) for k, v in d.items()}
    nm = len(m)
    # emitter side: cumulative radiance per depth
    rad = []
    cur = torch.zeros(nm, 3)
    surf, rd, T = det(xe), -dirv[m], torch.ones(nm, 3)
    alive = torch.arange(nm)
    s_all = slots[m]
    dead = False
    for b in range(D - 1):
        if not dead:
            o = 3 + 5 * b
            s = s_all[alive]
            with torch.no_grad():
                c, keep, ns_, nd, nT = radiance_direct(scene, surf, rd, T, smp[o][s], smp[o + 1][s], smp[o + 2][s],
                                                       smp[o + 3][s], smp[o + 4][s])
            cur = cur.index_add(0, alive, c.detach())
            if ns_ is None:
                dead = True
            else:
                alive = alive[keep]
                nz = (nT != 0).any(-1)
                surf, rd, T = det(_take(ns_, nz)), nd[nz].detach(), nT[nz].detach()
                alive = alive[nz]
                dead = len(alive) == 0
        rad.append(cur.clone())
    # sensor side
    surf, rd, T = det(xs), dirv[m], torch.ones(nm, 3)
    alive = torch.arange(nm)
    for b in range(D - 1):
        o = 3 + 5 * (D - 1) + 3 * b
        s = s_all[alive]
        c, pix, keep, ns_, nd, nT = importance_step(scene, cam, surf, rd, T, smp[o][s], smp[o + 1][s], smp[o + 2][s])
        okp = pix >= 0
        if bool(okp.any()):
            ra = rad[D - b - 2][alive][okp]
            img = img.index_add(0, pix[okp], value0[alive][okp][:, None] * ra * c[okp] * (1.0 / spp))
        if ns_ is None:
            break
        alive = alive[keep]
        surf, rd, T = ns_, nd, nT
    return img - img.detach()


def pixel_edge(scene, cam, spp, D, smp):
    """PixelBoundaryIntegrator::Integrate (BoundaryPixel.cpp:36-159) with 4
    antithetic copies (Edge.cpp:377-409, Camera.cpp:433-467)."""
    W, H = cam["width"], cam["height"]
    N = W * H * spp
    img = torch.zeros(W * H, 3)
    na = N // 4
    p = torch.arange(N)
    slot = p % na
    anti = p // na
    r = smp[0][slot]
    rr = torch.where(anti == 0, r,
                     torch.where(anti == 1, torch.where(r < 0.5, r + 0.5, r - 0.5),
                                 torch.where(anti == 2, torch.where(r < 0.75, 0.75 - r, 1.75 - r),
                                             torch.where(r < 0.25, 0.25 - r, 1.25 - r))))
    r4 = rr * 4.0
    bi = torch.floor(r4).long().clamp(0, 3)
    ox = torch.stack([torch.zeros_like(r4), r4 - 1.0, torch.ones_like(r4), 4.0 - r4], -1).gather(1, bi[:, None])[:, 0]
    oy = torch.stack([r4, torch.ones_like(r4), 3.0 - r4, torch.zeros_like(r4)], -1).gather(1, bi[:, None])[:, 0]
    lx, ly = float(cam["plane_len_x"]), float(cam["plane_len_y"])
    pdfs = torch.tensor([0.25 / (ly * W), 0.25 / (lx * H), 0.25 / (ly * W), 0.25 / (lx * H)], dtype=F32)
    pdf = pdfs[bi]
    dedge = torch.tensor([[0, 1, 0], [1, 0, 0], [0, 1, 0], [1, 0, 0]], dtype=F32)
    dvis = torch.tensor([[1, 0, 0], [0, -1, 0], [-1, 0, 0], [0, 1, 0]], dtype=F32)
    edge = normalize(xform_vector(cam["raster_to_world"], dedge))[bi]
    edge2 = normalize(xform_vector(cam["raster_to_world"], dvis))[bi]
    pixel = p % (W * H)
    rp = torch.stack([(pixel % W).to(F32) + ox, (pixel // W).to(F32) + oy, torch.zeros_like(ox)], -1)
    p0 = xform_point(cam["raster_to_world"], rp)
    cpos = torch.from_numpy(cam["pos"])
    d = normalize(p0 - cpos)
    tri, u, v, t = scene.intersect(p0, d, SHADOW_EPS, RAY_MAX)
    m = torch.nonzero(tri >= 0).reshape(-1)
    if len(m) == 0:
        return img
    hitP = p0[m] + t[m][:, None] * d[m]
    qx, qy, _, _, sval = sample_direct(cam, hitP)
    dirc = sensor_ray_dir(cam, qx, qy)
    surf = scene.post_intersect(tri[m], u[m], v[m])
    dist = length(surf["p"] - cpos)
    dist1 = length(p0[m] - cpos)
    cos2 = dot(surf["ng"], -dirc).abs()
    bval, n = _base_val(dist / dist1, edge[m], dirc, surf["ng"], edge2[m])
    bval = -bval * cos2
    T = sval[:, None].expand(-1, 3)
    sdet = {k: (v.detach() if torch.is_tensor(v) and v.dtype == F32 else v) for k, v in surf.items()}
    with torch.no_grad():
        L = nan_to_zero(T * emitted(scene, sdet, -dirc))
        L = L + _trace_radiance(scene, sdet, dirc, T, smp, slot[m], 1, D)
    xdn = _xdotn(scene, cpos.expand(len(m), 3), p0[m], tri[m], n)
    term = (L * (bval / pdf[m])[:, None]).detach() * xdn[:, None]
    img = img.index_add(0, pixel[m], term * (1.0 / spp))
    return img - img.detach()


INTEGRATORS = {0: path_tracer, 1: primary_edge, 2: direct_edge, 3: indirect_edge, 4: pixel_edge}


def render(scene, cam, integrator, spp, D, smp, guiding=None):
    """guiding = (seed, g_direct_spp, g_eps[, depth, max_size, thold]) turns on AQ guiding of the direct
    boundary term."""
    if integrator == 2 and guiding is not None:
        return direct_edge(scene, cam, spp, D, smp, guide=aq_guide(scene, *guiding))
    return INTEGRATORS[integrator](scene, cam, spp, D, smp)


def grads(scene, cam, integrator, spp, D, smp, dLdI, guiding=None):
    """dL/d(parameters) for loss sum(dLdI * image), via autograd."""
    for t in (scene.translation, scene.raw, scene.texels):
        if t.grad is not None:
            t.grad = None
    scene.configure()  # rebuild the differentiable geometry chain
    img = render(scene, cam, integrator, spp, D, smp, guiding)
    loss = (img * dLdI.reshape(-1, 3)).sum()
    params = [t for t in (scene.translation, scene.raw, scene.texels) if t.requires_grad]
    if loss.requires_grad:
        gs = torch.autograd.grad(loss, params, allow_unused=True)
    else:
        gs = [None] * len(params)
    out = {}
    for t, g in zip(params, gs):
        name = "translation" if t is scene.translation else ("positions" if t is scene.raw else "texels")
        out[name] = torch.zeros_like(t) if g is None else g
    return out, img.detach()
