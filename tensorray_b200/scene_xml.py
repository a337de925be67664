"""XML scene files -> SceneSpec (the reference's SceneLoader,
LibTensorRay/Renderer/SceneLoader.cpp:36-408), for trn_scene_create.

The same Mitsuba-style subset as the reference:

* `<bsdf type="diffuse">` with `reflectance` as `<rgb>`, `<spectrum>` or
  `<float>`, or a `<texture type="bitmap">` with a filename
  (SceneLoader.cpp:204-221). Bitmaps are read like stb_image's stbi_loadf
  (EDXUtil/Windows/Bitmap.cpp:187-190): 8-bit images become (v/255)^2.2,
  float images are taken as they are, and `.npy` arrays as [H, W, 3] floats.
* `<bsdf type="microfacet">` with `roughness` (float) and
  `diffuseReflectance` / `specularReflectance` (spectrum)
  (SceneLoader.cpp:258-301).
* `<shape type="obj">` with a `<ref id=...>` to its BSDF, a `filename`, an
  optional `face_normals`/`faceNormals` boolean (default true: flat shading)
  and an optional `<transform name="to_world">` of translate / rotate (degrees
  about an axis) / scale steps, each applied after the previous ones
  (SceneLoader.cpp:127-175, 310-372). The transform is applied to the
  vertices at load time.
* `<emitter type="area">` inside a shape with `radiance`
  (SceneLoader.cpp:373-391).
* `<sensor type="perspective">` with a `<film>` width/height, a `<lookat>`
  origin/target/up and `fov` (vertical, degrees) (SceneLoader.cpp:394-416).

The reference also reads `roughconductor`, a BSDF that no configuration of
this path uses and that it does not implement. It is rejected here with a
clear error, as is anything else outside this subset. Relative file names are
looked up first as given (the reference's behaviour, relative to the working
directory) and then relative to the XML file's directory.
"""
from __future__ import annotations

import math
import os
import xml.etree.ElementTree as ET

import numpy as np

from . import scenes


class SceneXmlError(ValueError):
    pass


def _require(cond, msg):
    if not cond:
        raise SceneXmlError(msg)


def parse_vector(text: str, length: int = 3, allow_empty: bool = False) -> np.ndarray:
    """Comma/space separated floats; with allow_empty a short list repeats its
    last value (parse_vector, SceneLoader.cpp:45-74)."""
    vals = [float(t) for t in text.replace(",", " ").split()]
    _require(len(vals) <= length, f"too many components in {text!r}")
    if len(vals) < length:
        _require(allow_empty, f"too few components in {text!r}")
        fill = vals[-1] if vals else 0.0
        vals += [fill] * (length - len(vals))
    return np.array(vals, np.float32)


def _named(parent, names, allow_empty=False):
    for child in parent:
        if child.get("name") in names:
            return child
    _require(allow_empty, f"missing child {sorted(names)[0]!r} in <{parent.tag}>")
    return None


def _rgb(node) -> tuple:
    if node.tag == "float":
        v = float(node.get("value"))
        return (v, v, v)
    _require(node.tag in ("rgb", "spectrum"), f"unsupported RGB type <{node.tag}>")
    return tuple(float(x) for x in parse_vector(node.get("value"), 3, allow_empty=True))


def _resolve(path: str, base: str) -> str:
    if os.path.isabs(path) or os.path.exists(path):
        return path
    cand = os.path.join(base, path)
    _require(os.path.exists(cand), f"file not found: {path}")
    return cand


_GAMMA_LUT = None

# the image formats stb_image 2.02 reads that PIL decodes to the same 8-bit
# values (JPEG: see load_bitmap)
_STB_8BIT_FORMATS = ("PNG", "BMP", "TGA", "PPM", "GIF", "JPEG")


def _gamma_lut() -> np.ndarray:
    """stb_image's 8-bit to float conversion (stbi__ldr_to_hdr, stb_image.h
    v2.02 as the reference builds it inside Bitmap.cpp, a C++ unit):
    powf(v / 255.0f, 2.2f) * 1.0f for each 8-bit value v, with the C
    library's powf (a vectorised float32 power can differ in the last bit)."""
    global _GAMMA_LUT
    if _GAMMA_LUT is None:
        import ctypes
        import ctypes.util
        libm = ctypes.CDLL(ctypes.util.find_library("m"))
        libm.powf.restype = ctypes.c_float
        libm.powf.argtypes = [ctypes.c_float, ctypes.c_float]
        x = np.arange(256, dtype=np.float32) / np.float32(255.0)
        g = float(np.float32(2.2))
        _GAMMA_LUT = np.array([libm.powf(float(v), g) for v in x], np.float32)
    return _GAMMA_LUT


def _read_radiance(path: str) -> np.ndarray:
    """Radiance RGBE (.hdr) -> [H, W, 3] float32, as stbi__hdr_load
    (stb_image.h v2.02) decodes it with 3 channels: a "#?RADIANCE" first line,
    a header that must hold "FORMAT=32-bit_rle_rgbe" and ends at an empty
    line, a "-Y H +X W" resolution line, then the pixels: flat RGBE when
    W < 8 or W >= 32768, else run-length-encoded scanlines (2, 2, W >> 8,
    W & 255, then each channel as runs (count > 128: count - 128 copies of one
    byte) and dumps (count literal bytes)). A scanline without that marker
    makes stb decode the whole image again as flat RGBE from that point.
    Channel value c with exponent e becomes c * ldexp(1.0f, e - 136) in
    float32; e = 0 is black. Corrupt data that stb would loop on or overrun
    is an error here."""
    with open(path, "rb") as f:
        data = f.read()
    pos = 0

    def line() -> bytes:
        nonlocal pos
        end = data.find(b"\n", pos)
        end = len(data) if end < 0 else end
        out = data[pos:end]
        pos = end + 1
        return out

    _require(line() == b"#?RADIANCE", f"{path}: not a Radiance HDR image")
    valid = False
    while pos < len(data):
        tok = line()
        if not tok:
            break
        valid |= tok == b"FORMAT=32-bit_rle_rgbe"
    _require(valid, f"{path}: unsupported HDR format")
    res = line().decode("latin-1").split()
    _require(len(res) == 4 and res[0] == "-Y" and res[2] == "+X", f"{path}: unsupported HDR data layout")
    H, W = int(res[1]), int(res[3])
    _require(H > 0 and W > 0, f"{path}: bad HDR resolution")

    def flat(at: int) -> np.ndarray:
        _require(at + H * W * 4 <= len(data), f"{path}: truncated HDR data")
        return np.frombuffer(data, np.uint8, H * W * 4, at).reshape(H, W, 4)

    if W < 8 or W >= 32768:
        rgbe = flat(pos)
    else:
        rgbe = np.empty((H, W, 4), np.uint8)
        for j in range(H):
            _require(pos + 4 <= len(data), f"{path}: truncated HDR data")
            c1, c2, hi = data[pos], data[pos + 1], data[pos + 2]
            if c1 != 2 or c2 != 2 or hi & 0x80:
                rgbe = flat(pos)
                break
            _require(((hi << 8) | data[pos + 3]) == W, f"{path}: invalid decoded scanline length")
            pos += 4
            for k in range(4):
                i = 0
                while i < W:
                    _require(pos < len(data), f"{path}: truncated HDR data")
                    count = data[pos]
                    pos += 1
                    if count > 128:
                        n = count - 128
                        _require(i + n <= W and pos < len(data), f"{path}: corrupt HDR run")
                        rgbe[j, i:i + n, k] = data[pos]
                        pos += 1
                    else:
                        n = count
                        _require(0 < n and i + n <= W and pos + n <= len(data), f"{path}: corrupt HDR dump")
                        rgbe[j, i:i + n, k] = np.frombuffer(data, np.uint8, n, pos)
                        pos += n
                    i += n
    e = rgbe[..., 3].astype(np.int64)
    scale = np.ldexp(np.float64(1.0), e - 136).astype(np.float32)
    out = rgbe[..., :3].astype(np.float32) * scale[..., None]
    out[e == 0] = 0.0
    return np.ascontiguousarray(out, np.float32)


def load_bitmap(path: str) -> np.ndarray:
    """[H, W, 3] float32 texels, top row first, as the reference's texture
    load gives them: Bitmap::ReadFromFile<float>(path, ..., 3)
    (EDXUtil/Windows/Bitmap.cpp:187-190, called by ImageTexture,
    Renderer/BSDF.cpp:57-70), one stbi_loadf call of stb_image 2.02.

    - 8-bit images (PNG, BMP, TGA, binary PPM/PGM, GIF, JPEG): gray is
      replicated, alpha dropped, and each value v becomes powf(v/255, 2.2).
    - Radiance .hdr: linear RGBE (_read_radiance).
    - 16-bit PNGs and other formats are refused, as stb_image 2.02 refuses
      them, and so are colour-mapped TGA images, which it decodes into
      uninitialised channels.
    - .npy [H, W, 3] arrays are taken as they are (this package's own format
      for generated textures).

    JPEG is decoded by PIL (libjpeg), whose IDCT and chroma upsampling are not
    stb_image's: its values can differ from the reference's by a few 8-bit
    levels. Every other format gives the reference's bits."""
    if path.endswith(".npy"):
        a = np.load(path).astype(np.float32)
        _require(a.ndim == 3 and a.shape[2] == 3, f"{path}: expected an [H, W, 3] array")
        return np.ascontiguousarray(a)
    with open(path, "rb") as f:
        head = f.read(32)
    if head.startswith(b"#?RADIANCE"):
        return _read_radiance(path)
    _require(not (head.startswith(b"\x89PNG\r\n\x1a\n") and len(head) > 24 and head[24] == 16),
             f"{path}: 16-bit PNGs are not loaded (the reference's stb_image 2.02 reads 8-bit PNGs only)")
    from PIL import Image
    img = Image.open(path)
    _require(img.format in _STB_8BIT_FORMATS and img.mode in ("1", "L", "LA", "P", "PA", "RGB", "RGBA"),
             f"{path}: {img.format} {img.mode} images are not loaded (the reference's stb_image 2.02 reads "
             "8-bit JPEG, PNG, BMP, TGA, PNM, GIF and Radiance HDR)")
    # stb_image 2.02 reads a colour-mapped TGA's palette entries one byte wide
    # and leaves the other channels uninitialised (stbi__tga_load)
    _require(not (img.format == "TGA" and img.mode in ("P", "PA")),
             f"{path}: colour-mapped TGA images are not loaded (the reference's stb_image 2.02 does not "
             "decode them)")
    a = np.asarray(img.convert("RGB"), np.uint8)
    return np.ascontiguousarray(_gamma_lut()[a])


def _transform(node) -> np.ndarray:
    m = np.eye(4)
    if node is None:
        return m
    _require(node.get("name") in ("to_world", "toWorld"), f"invalid transformation name {node.get('name')!r}")
    for step in node:
        if step.tag == "translate":
            t = np.eye(4)
            t[:3, 3] = [float(step.get(k, 0.0)) for k in "xyz"]
        elif step.tag == "scale":
            t = np.diag([float(step.get(k, 1.0)) for k in "xyz"] + [1.0])
        elif step.tag == "rotate":
            a = np.array([float(step.get(k, 0.0)) for k in "xyz"])
            a = a / np.linalg.norm(a)
            th = math.radians(float(step.get("angle", 0.0)))
            s, c = math.sin(th), math.cos(th)
            x, y, z = a
            t = np.eye(4)
            t[:3, :3] = [[x * x + (1 - x * x) * c, x * y * (1 - c) - z * s, x * z * (1 - c) + y * s],
                         [x * y * (1 - c) + z * s, y * y + (1 - y * y) * c, y * z * (1 - c) - x * s],
                         [x * z * (1 - c) - y * s, y * z * (1 - c) + x * s, z * z + (1 - z * z) * c]]
        else:
            raise SceneXmlError(f"unsupported transformation <{step.tag}>")
        m = t @ m
    return m


def load_xml(path: str) -> "scenes.SceneSpec":
    """Parse a scene file into a SceneSpec (BSDFs, shapes, lights, cameras)."""
    base = os.path.dirname(os.path.abspath(path))
    root = ET.parse(path).getroot()
    _require(root.tag == "scene", "the root element must be <scene>")
    spec = scenes.SceneSpec()
    bsdf_ids = {}
    for node in root.findall("bsdf"):
        bid = node.get("id")
        _require(bid, "a BSDF must have an id")
        kind = node.get("type")
        if kind == "diffuse":
            refl = _named(node, {"reflectance"})
            if refl.tag == "texture":
                _require(refl.get("type") == "bitmap", f"unsupported texture type {refl.get('type')!r}")
                fn = _named(refl, {"filename"})
                _require(fn is not None and fn.tag == "string", "failed to read the bitmap filename")
                spec.textures.append(load_bitmap(_resolve(fn.get("value"), base)))
                b = scenes.BsdfSpec(scenes.DIFFUSE, (0.5, 0.5, 0.5), texture=len(spec.textures) - 1)
            else:
                b = scenes.BsdfSpec(scenes.DIFFUSE, _rgb(refl))
        elif kind == "microfacet":
            rough = _named(node, {"roughness"})
            _require(rough.tag == "float", f"unsupported roughness <{rough.tag}>")
            dif = _named(node, {"diffuseReflectance"})
            spc = _named(node, {"specularReflectance"})
            _require(dif.tag == "spectrum", f"unsupported diffuseReflectance <{dif.tag}>")
            _require(spc.tag == "spectrum", f"unsupported specularReflectance <{spc.tag}>")
            b = scenes.BsdfSpec(scenes.MICROFACET, _rgb(dif), _rgb(spc), float(rough.get("value")))
        else:
            raise SceneXmlError(f"unsupported BSDF {kind!r}")
        bsdf_ids[bid] = len(spec.bsdfs)
        spec.bsdfs.append(b)
    for node in root.findall("shape"):
        _require(node.get("type") == "obj", f"unsupported shape {node.get('type')!r}")
        ref = node.find("ref")
        _require(ref is not None, "missing BSDF reference")
        _require(ref.get("id") in bsdf_ids, f"unknown BSDF id {ref.get('id')!r}")
        name = node.find("string")
        _require(name is not None and name.get("name") == "filename", "a shape needs a filename")
        fnode = _named(node, {"face_normals", "faceNormals"}, allow_empty=True)
        face_normals = True if fnode is None else fnode.get("value") == "true"
        light = -1
        em = node.find("emitter")
        if em is not None:
            _require(em.get("type") == "area", f"unsupported emitter {em.get('type')!r}")
            spec.lights.append(_rgb(_named(em, {"radiance"})))
            light = len(spec.lights) - 1
        mesh = scenes.load_obj(_resolve(name.get("value"), base), bsdf=bsdf_ids[ref.get("id")],
                               smooth=not face_normals, light=light)
        m = _transform(node.find("transform"))
        p = np.concatenate([mesh.positions.astype(np.float64), np.ones((len(mesh.positions), 1))], 1) @ m.T
        mesh.positions = np.ascontiguousarray(p[:, :3].astype(np.float32))
        spec.meshes.append(mesh)
    for node in root.findall("sensor"):
        _require(node.get("type") == "perspective", f"unsupported sensor {node.get('type')!r}")
        film = node.find("film")
        _require(film is not None, "a sensor needs a <film>")
        w = int(_named(film, {"width"}).get("value"))
        h = int(_named(film, {"height"}).get("value"))
        tr = node.find("transform")
        _require(tr is not None and tr.find("lookat") is not None, "the sensor's lookat transformation is missing")
        la = tr.find("lookat")
        spec.cameras.append(scenes.CameraSpec(tuple(float(x) for x in parse_vector(la.get("origin"))),
                                              tuple(float(x) for x in parse_vector(la.get("target"))),
                                              tuple(float(x) for x in parse_vector(la.get("up"))), w, h,
                                              float(_named(node, {"fov"}).get("value"))))
    return spec
