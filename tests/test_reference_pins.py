"""Pins against the reference's own code, on the CPU.

tests/golden/edx_pins.json holds what the reference's EDXUtil computes on
seeded inputs, written by tests/golden/make_edx_goldens.py from
oracle/_ref/edx_probe (a g++ build of EDXUtil/Graphics/ObjMesh.cpp,
BaseCamera.cpp and EDXUtil/Math/Matrix.cpp from the reference's sources):

- OBJ ingest, ObjMesh::LoadFromObj (ObjMesh.cpp:39-345) as every Primitive
  calls it: scenes.load_obj must give the same float32 bits for positions and
  texture coordinates and the same face indices;
- edge lists, ObjMesh::processEdges (ObjMesh.cpp:584-632): the oracle's
  build_edges and the library's trn_mesh_edges must give the same rows;
- texture images, Bitmap::ReadFromFile<float>(path, ..., 3) (Bitmap.cpp:
  187-190, one stbi_loadf call of stb_image 2.02): scene_xml.load_bitmap must
  give the same float32 bits for 8-bit PNG, BMP, TGA, PNM and GIF images and
  for flat, run-length-encoded and unmarked Radiance HDR files, and refuse the
  16-bit PNG the reference cannot load; JPEG goes through another decoder
  (libjpeg) and is held to a bound instead;
- the camera, EDX::Camera::Init (BaseCamera.cpp:45-88) and the quantities the
  renderer's Camera::Resize derives (Camera.cpp:105-137): the library's
  trn_camera_init and the oracle's camera_matrices must agree with it within
  CAMERA_TOL relative per quantity (scaled by its largest entry).

The camera cannot agree bit for bit. The reference normalises vectors with the
SSE reciprocal-square-root estimate and one Newton step (EDXMath.h:223-229,
Vec3.h:256-259), whose bits differ between CPU vendors, and inverts its
matrices in float32; the library and the oracle compute in double and round
once. The largest difference seen is 3.3e-7 (inv_area).
"""
import base64
import json
import os
import subprocess

import numpy as np
import pytest

from oracle import tr_oracle as O
from tensorray_b200 import api, scene_xml, scenes

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "edx_pins.json")
PROBE = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "edx_probe")
CAMERA_TOL = 1e-6
CAMERA_KEYS = ("pos", "dir", "raster_to_camera", "view_inv", "world_to_sample", "sample_to_camera", "raster_to_world",
               "inv_area", "plane_len_x", "plane_len_y")


@pytest.fixture(scope="module")
def pins():
    with open(GOLDEN) as f:
        return json.load(f)


def _f32(bits) -> np.ndarray:
    return np.asarray(bits, np.uint32).view(np.float32)


def _load(text, tmp_path, name):
    path = tmp_path / f"{name}.obj"
    path.write_text(text)
    return scenes.load_obj(str(path)), str(path)


def _quad_second_rows(text):
    """Rows of the faces list that are the second triangle of a quad."""
    rows, k = [], 0
    for line in text.splitlines():
        parts = line.split()
        if parts and parts[0] == "f":
            k += 1
            if len(parts) == 5:
                rows.append(k)
                k += 1
    return rows


def _reference_edges(r):
    return np.stack([r["edge_vertex0"], r["edge_vertex1"], r["edge_face0"], r["edge_face1"], r["edge_vertex2"]], 1)


def test_fixture_covers_the_edge_cases(pins):
    objs = pins["obj"]
    edges = np.concatenate([_reference_edges(c["reference"]) for c in objs.values()])
    assert (edges[:, 3] == -1).any() and (edges[:, 3] >= 0).any()
    # non-manifold edges: three or more faces on one (v0, v1)
    soup = objs["soup"]["reference"]
    F = np.asarray(soup["face_positions"]).reshape(-1, 3)
    und = np.sort(np.stack([F, np.roll(F, -1, 1)], 2).reshape(-1, 2), 1)
    _, cnt = np.unique(und, axis=0, return_counts=True)
    assert cnt.max() >= 3
    assert any("-" in c["text"] for c in objs.values())          # relative indices
    assert any(c["reference"]["textured"] for c in objs.values())
    assert len(pins["camera"]) >= 8


@pytest.mark.parametrize("name", ["tetra_vt_vn", "quads_untextured_forms", "quads_textured", "icosphere_level2",
                                  "soup"])
def test_obj_ingest_matches_reference_bits(pins, tmp_path, name):
    case = pins["obj"][name]
    r = case["reference"]
    m, _ = _load(case["text"], tmp_path, name)
    P = _f32(r["positions"]).reshape(-1, 3)
    assert m.positions.dtype == np.float32
    assert np.array_equal(m.positions.view(np.uint32), P.view(np.uint32))
    assert np.array_equal(m.faces, np.asarray(r["face_positions"]).reshape(-1, 3))
    assert r["triangle_count"] == len(m.faces) and r["vertex_count"] == len(m.positions)
    if r["textured"]:
        T = _f32(r["texcoords"]).reshape(-1, 2)
        assert np.array_equal(m.uvs.view(np.uint32), T.view(np.uint32))
        FT = np.asarray(r["face_texcoords"]).reshape(-1, 3)
        # the reference leaves a textured quad's second triangle's texture
        # indices unset (ObjMesh.cpp:221-262); every other row must agree
        keep = np.ones(len(FT), bool)
        keep[_quad_second_rows(case["text"])] = False
        assert np.array_equal(m.uv_faces[keep], FT[keep])
    else:
        assert m.uvs is None


@pytest.mark.parametrize("name", ["tetra_vt_vn", "quads_untextured_forms", "quads_textured", "icosphere_level2",
                                  "soup"])
def test_edge_lists_match_processEdges(pins, tmp_path, name):
    r = pins["obj"][name]["reference"]
    F = np.asarray(r["face_positions"]).reshape(-1, 3)
    ref = _reference_edges(r)
    assert r["num_edges"] == len(ref)
    assert np.array_equal(O.build_edges(F), ref)
    assert np.array_equal(api.mesh_edges(F), ref)


def test_mesh_edges_rejects_bad_arguments():
    lib = api._abi.load()
    assert lib.trn_mesh_edges(-1, None, None, 0) == -1
    assert "trn_mesh_edges" in lib.trn_last_error().decode()
    assert lib.trn_mesh_edges(1, None, None, 0) == -1
    assert api.mesh_edges(np.zeros((0, 3), np.int32)).shape == (0, 5)


def test_parse_f32_rounds_once_like_strtof():
    # 1 + 2^-24 is halfway between the float32 values 1 and 1 + 2^-23; the
    # decimal just above it is nearest to that double, so a parse through
    # double and then float32 rounds to even (1.0) where strtof gives 1 + 2^-23
    above = "1.0000000596046447753906250000001"
    below = "1.0000000596046447753906249999999"
    f = scenes.parse_f32([above, below, "0.1", "-2.5e-3"])
    assert f[0] == np.float32(1.0) + np.float32(2.0 ** -23)
    assert f[1] == np.float32(1.0)
    assert f[2] == np.float32(0.1) and f[3] == np.float32(-2.5e-3)


BITMAPS = ["rgb.png", "gray.png", "gray_alpha.png", "rgba.png", "palette.png", "gray16.png", "rgb.bmp", "rgb.tga",
           "rgb.ppm", "gray.pgm", "palette.gif", "rgb.jpg", "flat_w4.hdr", "rle_w16.hdr", "unmarked_w12.hdr"]


@pytest.mark.parametrize("name", BITMAPS)
def test_texture_images_match_reference_bits(pins, tmp_path, name):
    case = pins["bitmap"][name]
    r = case["reference"]
    path = tmp_path / name
    path.write_bytes(base64.b64decode(case["bytes"]))
    if "error" in r:
        with pytest.raises(scene_xml.SceneXmlError):
            scene_xml.load_bitmap(str(path))
        return
    ref = _f32(r["texels"]).reshape(r["height"], r["width"], 3)
    got = scene_xml.load_bitmap(str(path))
    assert got.dtype == np.float32 and got.shape == ref.shape
    if name.endswith(".jpg"):
        # libjpeg's IDCT and chroma upsampling are not stb_image's
        d = np.abs(got.astype(np.float64) - ref)
        assert d.max() <= 0.03 and d.mean() <= 2e-3, (d.max(), d.mean())
    else:
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_hdr_fixtures_cover_the_decoder_paths(pins):
    raw = {n: base64.b64decode(pins["bitmap"][n]["bytes"]) for n in ("flat_w4.hdr", "rle_w16.hdr",
                                                                      "unmarked_w12.hdr")}
    body = {n: b[b.index(b"+X"):].split(b"\n", 1)[1] for n, b in raw.items()}
    assert body["rle_w16.hdr"][:4] == bytes([2, 2, 0, 16])
    assert body["unmarked_w12.hdr"][:2] != bytes([2, 2])
    ref = _f32(pins["bitmap"]["rle_w16.hdr"]["reference"]["texels"])
    tiny = ref[(ref > 0) & (ref < np.finfo(np.float32).tiny)]
    assert tiny.size > 0          # subnormal results from the low exponents
    assert (ref == 0).any()       # exponent 0 is black


def _rel(a, r):
    a = np.asarray(a, np.float64).reshape(-1)
    r = np.asarray(r, np.float64).reshape(-1)
    return float(np.abs(a - r).max() / max(np.abs(r).max(), 1e-30))


def test_camera_matches_reference(pins):
    worst = 0.0
    for case in pins["camera"]:
        a, r = case["args"], case["reference"]
        v = [float(x) for x in a[:9]]
        w, h, fov = int(a[9]), int(a[10]), float(a[11])
        lib_cam = api.Camera(v[0:3], v[3:6], v[6:9], w, h, fov).matrices()
        ora_cam = O.camera_matrices(v[0:3], v[3:6], v[6:9], w, h, fov)
        assert (lib_cam["width"], lib_cam["height"]) == (r["width"], r["height"])
        for k in CAMERA_KEYS:
            ref = _f32(r[k])
            for got in (lib_cam[k], ora_cam[k]):
                e = _rel(got, ref)
                worst = max(worst, e)
                assert e <= CAMERA_TOL, (a, k, e)
    assert worst > 0.0        # the float32/rsqrt path is not the double one


@pytest.mark.skipif(not os.path.exists(PROBE), reason="the reference probe is built only where the reference is")
def test_fixture_is_what_the_reference_computes(pins, tmp_path):
    """Replays the mesh inputs through the probe itself. Mesh ingest and edge
    lists are integer and parse work, the same on every CPU; the camera is
    replayed against the same tolerance as above (the SSE estimate's bits are
    the CPU's)."""
    for name, case in pins["obj"].items():
        _, path = _load(case["text"], tmp_path, name)
        live = json.loads(subprocess.run([PROBE, "obj", path], capture_output=True, text=True, check=True).stdout)
        r = case["reference"]
        keep = np.ones(len(r["face_texcoords"]), bool)
        for row in _quad_second_rows(case["text"]) if r["textured"] else []:
            keep[3 * row:3 * row + 3] = False
        for k, v in r.items():
            if k == "face_texcoords":
                assert np.array_equal(np.asarray(live[k])[keep], np.asarray(v)[keep]), name
            else:
                assert live[k] == v, (name, k)
    for name, case in pins["bitmap"].items():
        path = tmp_path / name
        path.write_bytes(base64.b64decode(case["bytes"]))
        live = json.loads(subprocess.run([PROBE, "bitmap", str(path)], capture_output=True, text=True,
                                         check=True).stdout)
        assert live == case["reference"], name
    for case in pins["camera"]:
        live = json.loads(subprocess.run([PROBE, "camera", *case["args"]], capture_output=True, text=True,
                                         check=True).stdout)
        for k in CAMERA_KEYS:
            assert _rel(_f32(live[k]), _f32(case["reference"][k])) <= CAMERA_TOL


def _random_obj(seed: int) -> str:
    """A seeded OBJ: 4-40 vertices written with 0-9 decimals, exponents,
    integers or 17 digits, space or tab separators, optional texture
    coordinates and normals, comments, blank, 'o', 'g', 's' and 'usemtl'
    lines, triangles and quads in every corner form, negative indices, and
    LF or CRLF line ends. With CRLF no line ends in a blank: the reference's
    face parser would then read the carriage return as one more corner
    (ObjMesh.cpp:101-135 splits only at ' ', '\\t', '\\n'), an index sscanf
    cannot parse, which leaves its corner uninitialised."""
    rng = np.random.default_rng(seed)

    def num():
        x = rng.normal(0, 2)
        k = rng.integers(0, 5)
        if k == 0:
            return f"{x:.{rng.integers(0, 10)}f}"
        if k == 1:
            return f"{x:.{rng.integers(1, 8)}e}"
        if k == 2:
            return repr(float(np.float32(x)))
        if k == 3:
            return f"{int(x * 10)}"
        return f"{x:.17g}"

    def sep():
        return " " if rng.random() < 0.8 else "\t"

    nv = int(rng.integers(4, 40))
    textured, normals = rng.random() < 0.6, rng.random() < 0.5
    lines = []
    for _ in range(nv):
        lines.append("v" + sep() + sep().join(num() for _ in range(3)))
        if rng.random() < 0.1:
            lines.append("# comment words here")
        if rng.random() < 0.05:
            lines.append("")
    for _ in range(nv if textured else 0):
        lines.append(f"vt {rng.random():.{rng.integers(1, 9)}f} {rng.random():.{rng.integers(1, 9)}f}")
    for _ in range(nv if normals else 0):
        lines.append("vn 0 0 1")
    lines += ["o object", "g group", "s 1", "usemtl material"]
    for _ in range(int(rng.integers(1, 30))):
        idx = rng.choice(nv, 3 if rng.random() < 0.6 else 4, replace=False)
        neg = rng.random() < 0.2
        corners = []
        for i in idx:
            p = str(int(i) - nv) if neg else str(int(i) + 1)
            t = int(i) + 1
            corners.append(f"{p}/{t}/{t}" if textured and normals else f"{p}/{t}" if textured
                           else f"{p}//{t}" if normals else p)
        lines.append("f " + sep().join(corners) + (" " if rng.random() < 0.2 else ""))
        if rng.random() < 0.1:
            lines.append("s off")
    end = "\n" if rng.random() < 0.9 else "\r\n"
    if end == "\r\n":
        lines = [line.rstrip(" \t") for line in lines]
    return end.join(lines) + end


@pytest.mark.skipif(not os.path.exists(PROBE), reason="the reference probe is built only where the reference is")
def test_random_obj_files_load_as_the_reference_loads_them(tmp_path):
    """150 seeded OBJ files through the reference's own loader and this one:
    the same float32 positions and texture coordinates, the same faces
    (texture indices of a quad's second triangle aside) and edge lists."""
    for seed in range(150):
        text = _random_obj(seed)
        path = tmp_path / f"r{seed}.obj"
        path.write_bytes(text.encode())
        r = json.loads(subprocess.run([PROBE, "obj", str(path)], capture_output=True, text=True,
                                      check=True).stdout)
        m = scenes.load_obj(str(path))
        P = _f32(r["positions"]).reshape(-1, 3)
        assert np.array_equal(m.positions.view(np.uint32), P.view(np.uint32)), seed
        F = np.asarray(r["face_positions"]).reshape(-1, 3)
        assert np.array_equal(m.faces, F), seed
        assert np.array_equal(api.mesh_edges(F), _reference_edges(r)), seed
        if r["textured"]:
            assert np.array_equal(m.uvs.view(np.uint32), _f32(r["texcoords"]).reshape(-1, 2).view(np.uint32)), seed
            keep = np.ones(len(F), bool)
            keep[_quad_second_rows(text)] = False
            FT = np.asarray(r["face_texcoords"]).reshape(-1, 3)
            assert np.array_equal(m.uv_faces[keep], FT[keep]), seed


@pytest.mark.skipif(not os.path.exists(PROBE), reason="the reference probe is built only where the reference is")
def test_random_cameras_match_the_reference(tmp_path):
    """100 seeded poses, resolutions (16-2047 per side) and fields of view
    (10-120 degrees) through the reference's EDX::Camera and through
    trn_camera_init and the oracle. Over 300 such cameras the largest
    relative difference seen was 7.3e-7 (inv_area); the bound leaves a few
    float32 ulps of room for the reference's reciprocal-square-root estimate,
    whose bits are the CPU's."""
    rng = np.random.default_rng(11)
    for _ in range(100):
        pos, tgt, up = rng.normal(0, 5, 3), rng.normal(0, 1, 3), rng.normal(0, 1, 3)
        w, h, fov = int(rng.integers(16, 2048)), int(rng.integers(16, 2048)), float(np.float32(rng.uniform(10, 120)))
        args = [repr(float(np.float32(x))) for x in (*pos, *tgt, *up)] + [str(w), str(h), repr(fov)]
        r = json.loads(subprocess.run([PROBE, "camera", *args], capture_output=True, text=True, check=True).stdout)
        v = [float(x) for x in args[:9]]
        lib_cam = api.Camera(v[0:3], v[3:6], v[6:9], w, h, fov).matrices()
        ora_cam = O.camera_matrices(v[0:3], v[3:6], v[6:9], w, h, fov)
        for k in CAMERA_KEYS:
            for got in (lib_cam[k], ora_cam[k]):
                assert _rel(got, _f32(r[k])) <= 2e-6, (args, k)


def _random_image(rng, i):
    """A seeded image file the reference's stb_image decodes: 8-bit PNG, BMP,
    TGA (not colour-mapped), PPM/PGM or GIF in gray, gray+alpha, RGB, RGBA
    or palette form, or a Radiance file (flat, or run-length encoded where
    the format allows it, 8 <= width < 32768) with runs, dumps and black
    pixels. Returns (name, bytes)."""
    import io

    from PIL import Image
    if i % 3 < 2:
        H, W = int(rng.integers(1, 40)), int(rng.integers(1, 40))
        mode = ["L", "LA", "RGB", "RGBA", "P"][int(rng.integers(0, 5))]
        fmt = ["PNG", "BMP", "TGA", "PPM", "GIF"][int(rng.integers(0, 5))]
        ch = {"L": 1, "LA": 2, "RGB": 3, "RGBA": 4, "P": 3}[mode]
        a = rng.integers(0, 256, (H, W, ch), dtype=np.uint8)
        img = Image.fromarray(a[:, :, 0] if ch == 1 else a, "RGB" if mode == "P" else mode)
        if mode == "P" and fmt != "TGA":
            img = img.convert("P")
        if (fmt in ("BMP", "PPM") and mode in ("LA", "RGBA")) or (fmt == "PPM" and img.mode == "P"):
            img = img.convert("RGB")
        if fmt == "GIF" and img.mode not in ("L", "P"):
            img = img.convert("P")
        b = io.BytesIO()
        img.save(b, fmt)
        return f"r{i}.{fmt.lower()}", b.getvalue()
    from tests.golden.make_edx_goldens import _hdr_bytes
    H, W = int(rng.integers(1, 12)), int(rng.choice([3, 7, 8, 9, 40, 200, 300]))
    rgbe = rng.integers(0, 256, (H, W, 4), dtype=np.uint8)
    for j in range(H):
        for k in range(4):
            s = int(rng.integers(0, W))
            rgbe[j, s:min(W, s + int(rng.integers(1, 160))), k] = rng.integers(0, 256)
    rgbe[..., 3] = np.where(rng.random((H, W)) < 0.1, 0, rgbe[..., 3])
    return f"r{i}.hdr", _hdr_bytes(rgbe, W >= 8 and rng.random() < 0.8)


@pytest.mark.skipif(not os.path.exists(PROBE), reason="the reference probe is built only where the reference is")
def test_random_images_load_as_the_reference_loads_them(tmp_path):
    """150 seeded image files through the reference's stb_image and
    scene_xml.load_bitmap: the same float32 texels (JPEG is not among them:
    another decoder), or an error from both."""
    rng = np.random.default_rng(21)
    for i in range(150):
        name, raw = _random_image(rng, i)
        path = tmp_path / name
        path.write_bytes(raw)
        r = json.loads(subprocess.run([PROBE, "bitmap", str(path)], capture_output=True, text=True,
                                      check=True).stdout)
        if "error" in r:
            with pytest.raises(scene_xml.SceneXmlError):
                scene_xml.load_bitmap(str(path))
            continue
        ref = _f32(r["texels"]).reshape(r["height"], r["width"], 3)
        got = scene_xml.load_bitmap(str(path))
        assert got.shape == ref.shape and np.array_equal(got.view(np.uint32), ref.view(np.uint32)), name


def test_colour_mapped_tga_is_refused(tmp_path):
    from PIL import Image
    p = tmp_path / "pal.tga"
    Image.fromarray(np.zeros((4, 4, 3), np.uint8)).convert("P").save(str(p), "TGA")
    with pytest.raises(scene_xml.SceneXmlError, match="colour-mapped TGA"):
        scene_xml.load_bitmap(str(p))
