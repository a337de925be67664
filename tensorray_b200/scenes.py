"""Procedural scene descriptions for the benchmark configurations.

Every scene is built here from seeds (no external assets): an icosphere, a
displaced UV sphere, quads for the ground and the area light, and a random
albedo texture. A :class:`SceneSpec` holds the concatenated, host-side arrays
that ``trn_scene_create`` consumes (the reference assembles the same buffers
in Scene::ExtractGeometry, LibTensorRay/Renderer/Scene.cpp:46-124).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

DIFFUSE = 0
MICROFACET = 1


@dataclass
class MeshSpec:
    positions: np.ndarray            # [V, 3] float32
    faces: np.ndarray                # [T, 3] int32
    bsdf: int = 0
    light: int = -1                  # area-light id or -1
    smooth: bool = False
    uvs: np.ndarray | None = None    # [NUV, 2] float32
    uv_faces: np.ndarray | None = None  # [T, 3] int32
    translation: tuple = (0.0, 0.0, 0.0)


@dataclass
class BsdfSpec:
    type: int = DIFFUSE
    albedo: tuple = (0.5, 0.5, 0.5)
    specular: tuple = (0.04, 0.04, 0.04)
    roughness: float = 0.3
    texture: int = -1


@dataclass
class CameraSpec:
    pos: tuple
    target: tuple
    up: tuple
    width: int
    height: int
    fov: float


@dataclass
class SceneSpec:
    meshes: list = field(default_factory=list)
    bsdfs: list = field(default_factory=list)
    lights: list = field(default_factory=list)      # radiance triples
    textures: list = field(default_factory=list)    # [H, W, 3] float32 arrays
    cameras: list = field(default_factory=list)

    # ---- concatenated arrays ------------------------------------------------
    def arrays(self) -> dict:
        pos, idx, vmesh, tmesh, uvs, uvidx = [], [], [], [], [], []
        voff = 0
        uvoff = 0
        any_uv = any(m.uvs is not None for m in self.meshes)
        for mi, m in enumerate(self.meshes):
            pos.append(np.asarray(m.positions, np.float32))
            idx.append(np.asarray(m.faces, np.int32) + voff)
            vmesh.append(np.full(len(m.positions), mi, np.int32))
            tmesh.append(np.full(len(m.faces), mi, np.int32))
            if any_uv:
                if m.uvs is not None:
                    uvs.append(np.asarray(m.uvs, np.float32))
                    uvidx.append(np.asarray(m.uv_faces, np.int32) + uvoff)
                    uvoff += len(m.uvs)
                else:
                    uvs.append(np.zeros((1, 2), np.float32))
                    uvidx.append(np.full((len(m.faces), 3), uvoff, np.int32))
                    uvoff += 1
            voff += len(m.positions)
        out = {
            "positions": np.ascontiguousarray(np.concatenate(pos)),
            "indices": np.ascontiguousarray(np.concatenate(idx)),
            "vertex_mesh": np.concatenate(vmesh),
            "triangle_mesh": np.concatenate(tmesh),
            "mesh_smooth": np.array([1 if m.smooth else 0 for m in self.meshes], np.uint8),
            "mesh_bsdf": np.array([m.bsdf for m in self.meshes], np.int32),
            "mesh_light": np.array([m.light for m in self.meshes], np.int32),
            "mesh_translation": np.array([m.translation for m in self.meshes], np.float32).reshape(-1, 3),
            "light_radiance": np.array(self.lights, np.float32).reshape(-1, 3),
            "uvs": np.ascontiguousarray(np.concatenate(uvs)) if any_uv else None,
            "uv_indices": np.ascontiguousarray(np.concatenate(uvidx)) if any_uv else None,
        }
        return out

    @property
    def num_triangles(self) -> int:
        return sum(len(m.faces) for m in self.meshes)


# ---------------------------------------------------------------------------
# meshes
# ---------------------------------------------------------------------------
def icosphere(subdiv: int, radius: float = 1.0) -> tuple[np.ndarray, np.ndarray]:
    """Icosahedron subdivided `subdiv` times (20*4^s faces), outward winding."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
         (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = [np.array(p, np.float64) / np.linalg.norm(p) for p in v]
    faces = list(f)
    for _ in range(subdiv):
        cache: dict = {}

        def mid(a: int, b: int) -> int:
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    P = (np.array(verts) * radius).astype(np.float32)
    F = np.array(faces, np.int32)
    # make the winding outward: cross(p1-p0, p2-p0) . centroid > 0
    p0, p1, p2 = P[F[:, 0]].astype(np.float64), P[F[:, 1]].astype(np.float64), P[F[:, 2]].astype(np.float64)
    n = np.cross(p1 - p0, p2 - p0)
    flip = (n * (p0 + p1 + p2)).sum(1) < 0
    F[flip] = F[flip][:, [0, 2, 1]]
    return P, F


def _hash3(ix, iy, iz, seed):
    h = (ix.astype(np.int64) * 73856093) ^ (iy.astype(np.int64) * 19349663) ^ (iz.astype(np.int64) * 83492791)
    h = (h ^ (seed * 2654435761)) & 0xFFFFFFFF
    h = (h ^ (h >> 16)) * 0x7FEB352D & 0xFFFFFFFF
    h = (h ^ (h >> 15)) * 0x846CA68B & 0xFFFFFFFF
    h = h ^ (h >> 16)
    return (h.astype(np.float64) / 4294967295.0) * 2.0 - 1.0


def value_noise3(p: np.ndarray, seed: int) -> np.ndarray:
    """Trilinear value noise on the integer lattice with smoothstep weights."""
    i = np.floor(p).astype(np.int64)
    f = p - i
    w = f * f * (3.0 - 2.0 * f)
    out = np.zeros(len(p))
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                c = _hash3(i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz, seed)
                wx = w[:, 0] if dx else 1 - w[:, 0]
                wy = w[:, 1] if dy else 1 - w[:, 1]
                wz = w[:, 2] if dz else 1 - w[:, 2]
                out += c * wx * wy * wz
    return out


def displaced_uv_sphere(target_tris: int, radius: float = 1.0, amplitude: float = 0.1, seed: int = 0,
                        octaves: int = 3, base_freq: float = 2.0):
    """Welded UV sphere with 2*slices*(stacks-1) triangles, displaced radially
    by `octaves` octaves of value noise of the given amplitude. Returns
    positions, faces, uvs, uv_faces."""
    stacks = max(3, int(round((target_tris / 4.0) ** 0.5)) + 1)
    slices = max(3, int(round(target_tris / (2.0 * (stacks - 1)))))
    th = np.pi * np.arange(1, stacks) / stacks            # interior rings
    ph = 2.0 * np.pi * np.arange(slices) / slices
    st, ct = np.sin(th)[:, None], np.cos(th)[:, None]
    ring = np.stack([st * np.cos(ph)[None], ct * np.ones_like(ph)[None], st * np.sin(ph)[None]], -1).reshape(-1, 3)
    dirs = np.concatenate([[[0.0, 1.0, 0.0]], ring, [[0.0, -1.0, 0.0]]])
    n = np.zeros(len(dirs))
    amp = 1.0
    for o in range(octaves):
        n += amp * value_noise3(dirs * base_freq * (2 ** o), seed + 7919 * o)
        amp *= 0.5
    n /= (1.0 + 0.5 + 0.25)
    P = (dirs * (radius * (1.0 + amplitude * n))[:, None]).astype(np.float32)
    top, bot = 0, len(dirs) - 1
    R = lambda i, j: 1 + i * slices + (j % slices)
    faces = []
    for j in range(slices):
        faces.append((top, R(0, j + 1), R(0, j)))
    for i in range(stacks - 2):
        for j in range(slices):
            a, b, c, d = R(i, j), R(i, j + 1), R(i + 1, j), R(i + 1, j + 1)
            faces.append((a, b, c))
            faces.append((b, d, c))
    for j in range(slices):
        faces.append((bot, R(stacks - 2, j), R(stacks - 2, j + 1)))
    F = np.array(faces, np.int32)
    # uv with a seam column: u = j / slices, v = theta / pi
    uv_ring = np.stack(np.meshgrid(np.arange(slices + 1) / slices, np.arange(1, stacks) / stacks), -1).reshape(-1, 2)
    uvs = np.concatenate([[[0.5, 0.0]], uv_ring, [[0.5, 1.0]]]).astype(np.float32)
    U = lambda i, j: 1 + i * (slices + 1) + j
    ubot = len(uvs) - 1
    uvf = []
    for j in range(slices):
        uvf.append((0, U(0, j + 1), U(0, j)))
    for i in range(stacks - 2):
        for j in range(slices):
            a, b, c, d = U(i, j), U(i, j + 1), U(i + 1, j), U(i + 1, j + 1)
            uvf.append((a, b, c))
            uvf.append((b, d, c))
    for j in range(slices):
        uvf.append((ubot, U(stacks - 2, j), U(stacks - 2, j + 1)))
    UVF = np.array(uvf, np.int32)
    # outward winding
    p0, p1, p2 = (P[F[:, k]].astype(np.float64) for k in range(3))
    nrm = np.cross(p1 - p0, p2 - p0)
    flip = (nrm * (p0 + p1 + p2)).sum(1) < 0
    F[flip] = F[flip][:, [0, 2, 1]]
    UVF[flip] = UVF[flip][:, [0, 2, 1]]
    return P, F, uvs, UVF


def quad(center, half: float, axis: str = "y", up: bool = True):
    """Axis-aligned square of half-size `half` facing +axis (up) or -axis."""
    c = np.asarray(center, np.float32)
    if axis != "y":
        raise ValueError("only horizontal quads are used")
    P = np.array([[-half, 0, -half], [half, 0, -half], [half, 0, half], [-half, 0, half]], np.float32) + c
    F = np.array([[0, 2, 1], [0, 3, 2]], np.int32) if up else np.array([[0, 1, 2], [0, 2, 3]], np.int32)
    return P, F


def random_texture(size: int, seed: int, lo: float = 0.2, hi: float = 0.8) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.uniform(lo, hi, size=(size, size, 3)).astype(np.float32)


# ---------------------------------------------------------------------------
# benchmark configurations
# ---------------------------------------------------------------------------
def _ground_and_light(spec: SceneSpec, ground_bsdf: int, radiance: float = 10.0):
    gp, gf = quad((0.0, -1.0, 0.0), 5.0, up=True)
    spec.meshes.append(MeshSpec(gp, gf, bsdf=ground_bsdf))
    lp, lf = quad((0.0, 4.0, 0.0), 0.5, up=False)
    spec.lights.append((radiance, radiance, radiance))
    spec.meshes.append(MeshSpec(lp, lf, bsdf=ground_bsdf, light=len(spec.lights) - 1))


def config1_scene(width: int = 256, height: int = 256, sphere_offset=(0.0, 0.0, 0.0)) -> SceneSpec:
    """Icosphere (subdivision 3, 1280 triangles, radius 1, albedo 0.7) over a
    two-triangle ground quad (albedo 0.5) under a 1x1 quad light of radiance
    10 at height 4; pinhole camera at distance 4, fov 45 degrees."""
    spec = SceneSpec()
    spec.bsdfs = [BsdfSpec(DIFFUSE, (0.7, 0.7, 0.7)), BsdfSpec(DIFFUSE, (0.5, 0.5, 0.5))]
    P, F = icosphere(3, 1.0)
    spec.meshes.append(MeshSpec(P, F, bsdf=0, smooth=True, translation=tuple(sphere_offset)))
    _ground_and_light(spec, 1)
    spec.cameras = [CameraSpec((0.0, 0.0, 4.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), width, height, 45.0)]
    return spec


def config2_scene(width: int = 512, height: int = 512, tris: int = 100_000, seed: int = 0,
                  tex_size: int = 512) -> SceneSpec:
    """100K-triangle sphere displaced by 3-octave value noise (amplitude 0.1),
    GGX microfacet (roughness 0.3, F0 0.04) with a 512x512 RGB albedo texture
    in U[0.2, 0.8]; ground and light as in config 1."""
    spec = SceneSpec()
    spec.textures = [random_texture(tex_size, seed + 1)]
    spec.bsdfs = [BsdfSpec(MICROFACET, (0.5, 0.5, 0.5), (0.04, 0.04, 0.04), 0.3, texture=0),
                  BsdfSpec(DIFFUSE, (0.5, 0.5, 0.5))]
    P, F, uv, uvf = displaced_uv_sphere(tris, 1.0, 0.1, seed)
    spec.meshes.append(MeshSpec(P, F, bsdf=0, smooth=True, uvs=uv, uv_faces=uvf))
    _ground_and_light(spec, 1)
    spec.cameras = [CameraSpec((0.0, 0.0, 4.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), width, height, 45.0)]
    return spec


def served_scene(tris: int, seed: int = 0) -> SceneSpec:
    """A diffuse displaced sphere of about `tris` triangles over the ground
    quad, lit by the quad light (the resident scenes of the serving workload)."""
    spec = SceneSpec()
    spec.bsdfs = [BsdfSpec(DIFFUSE, (0.7, 0.7, 0.7)), BsdfSpec(DIFFUSE, (0.5, 0.5, 0.5))]
    if tris <= 2000:
        P, F = icosphere(3, 1.0)
        spec.meshes.append(MeshSpec(P, F, bsdf=0, smooth=True))
    else:
        P, F, uv, uvf = displaced_uv_sphere(tris, 1.0, 0.1, seed)
        spec.meshes.append(MeshSpec(P, F, bsdf=0, smooth=True))
    _ground_and_light(spec, 1)
    spec.cameras = [CameraSpec((0.0, 0.0, 4.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 256, 256, 45.0)]
    return spec


def fibonacci_cameras(n: int, radius: float, resolutions, seed: int = 0):
    """`n` poses on a Fibonacci sphere looking at the origin; resolutions are
    drawn from `resolutions` with a seeded generator."""
    rng = np.random.default_rng(seed)
    cams = []
    ga = np.pi * (3.0 - 5.0 ** 0.5)
    for i in range(n):
        y = 1.0 - 2.0 * (i + 0.5) / n
        r = (1.0 - y * y) ** 0.5
        th = ga * i
        p = (radius * r * np.cos(th), radius * y, radius * r * np.sin(th))
        up = (0.0, 1.0, 0.0) if abs(y) < 0.99 else (1.0, 0.0, 0.0)
        res = int(rng.choice(resolutions))
        cams.append(CameraSpec(tuple(float(x) for x in p), (0.0, 0.0, 0.0), up, res, res, 45.0))
    return cams


_LIBC = None


def _strtof(token: str) -> np.float32:
    global _LIBC
    if _LIBC is None:
        import ctypes
        _LIBC = ctypes.CDLL(None)
        _LIBC.strtof.restype = ctypes.c_float
        _LIBC.strtof.argtypes = [ctypes.c_char_p, ctypes.c_void_p]
    return np.float32(_LIBC.strtof(token.encode(), None))


def parse_f32(tokens) -> np.ndarray:
    """Decimal strings -> float32, rounded once, as C's strtof (behind the
    reference's fscanf("%f")) rounds them. Python parses to the nearest
    double, and rounding that to float32 can differ from a single rounding
    only when the double lies exactly halfway between two float32 values;
    those few are parsed again by the C library."""
    d = np.asarray([float(t) for t in tokens], np.float64)
    f = d.astype(np.float32)
    tie = (d.view(np.uint64) & np.uint64((1 << 29) - 1)) == np.uint64(1 << 28)
    for i in np.flatnonzero(tie):
        f[i] = _strtof(tokens[i])
    return f


def load_obj(path: str, bsdf: int = 0, smooth: bool = True, light: int = -1,
             translation=(0.0, 0.0, 0.0)) -> MeshSpec:
    """Wavefront OBJ -> MeshSpec, following ObjMesh::LoadFromObj
    (EDXUtil/Graphics/ObjMesh.cpp:39-345) with makeLeftHanded = false, as every
    reference Primitive loads meshes (Renderer/Primitive.cpp:213-245):
    `v` positions as given, `vt` texture coordinates with v flipped to
    1.0f - v in float32 arithmetic (ObjMesh.cpp:73-78), numbers rounded to
    float32 as strtof rounds them, faces of 3 or 4 corners in the forms i,
    i/t, i/t/n, i//n with 1-based or negative (relative) indices, quads split
    into (0, 1, 2) and (3, 0, 2). Smoothing groups and materials are not
    used by the renderer and are skipped. Normals (`vn`) are skipped too, and
    that is a difference: for a smooth mesh whose file has normals, the
    reference shades with those (per face corner, constant with respect to
    the vertex positions; Primitive.cpp:113-131, 205-208), while this renderer
    always uses the area-weighted vertex normals of the positions, which the
    reference computes when the file has none (Primitive.cpp:323-340). The
    reference leaves the texture indices of a quad's second triangle unset;
    here they follow its position corners. A comment line is skipped whole; the
    reference reads the tokens after a lone '#' as commands, so a comment
    such as "# v 1 2 3" would add a vertex there. A face line that ends in a
    blank before a CRLF line end is read as its corners here; the reference
    takes the carriage return for one more corner that it cannot parse
    (ObjMesh.cpp:101-135), with an uninitialised index."""
    pos, us, vs, faces, uvf = [], [], [], [], []
    textured = False
    with open(path, "r") as f:
        for raw in f:
            parts = raw.split()
            if not parts or parts[0].startswith("#"):
                continue
            tag = parts[0]
            if tag == "v":
                if len(parts) < 4:
                    raise ValueError(f"{path}: a vertex needs 3 coordinates: {raw.strip()!r}")
                pos.extend(parts[1:4])
            elif tag == "vt":
                if len(parts) < 3:
                    raise ValueError(f"{path}: a texture coordinate needs 2 values: {raw.strip()!r}")
                us.append(parts[1])
                vs.append(parts[2])
                textured = True
            elif tag == "f":
                corners = parts[1:]
                if len(corners) not in (3, 4):
                    raise ValueError(f"{path}: faces must have 3 or 4 corners, got {len(corners)}")
                pi, ti = [], []
                for c in corners:
                    fields = c.split("/")
                    p = int(fields[0])
                    pi.append(p - 1 if p > 0 else len(pos) // 3 + p)
                    if len(fields) > 1 and fields[1]:
                        t = int(fields[1])
                        ti.append(t - 1 if t > 0 else len(us) + t)
                    else:
                        ti.append(0)
                faces.append([pi[0], pi[1], pi[2]])
                uvf.append([ti[0], ti[1], ti[2]])
                if len(corners) == 4:
                    faces.append([pi[3], pi[0], pi[2]])
                    uvf.append([ti[3], ti[0], ti[2]])
    P = parse_f32(pos).reshape(-1, 3)
    F = np.asarray(faces, np.int32).reshape(-1, 3)
    if F.size and (F.min() < 0 or F.max() >= len(P)):
        raise ValueError(f"{path}: face index out of range")
    m = MeshSpec(P, F, bsdf=bsdf, light=light, smooth=smooth, translation=tuple(translation))
    if textured:
        m.uvs = np.stack([parse_f32(us), np.float32(1.0) - parse_f32(vs)], 1).astype(np.float32)
        m.uv_faces = np.asarray(uvf, np.int32).reshape(-1, 3)
    return m
