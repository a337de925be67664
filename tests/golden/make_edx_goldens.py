"""Writes tests/golden/edx_pins.json: what the reference's own EDXUtil code
computes for the mesh ingest, the edge lists, the texture images and the
camera, on seeded inputs.

The outputs come from oracle/_ref/edx_probe, which oracle/edx/Makefile builds
from the reference's sources (EDXUtil/Graphics/ObjMesh.cpp, BaseCamera.cpp,
EDXUtil/Math/Matrix.cpp, EDXUtil/Windows/stb_image.h). The inputs (OBJ text,
image file bytes, camera arguments) are stored
beside the outputs, so tests/test_reference_pins.py replays them without the
reference. Run it where the reference checkout is present:

    python tests/golden/make_edx_goldens.py [REFERENCE_ROOT]
"""
import base64
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from tensorray_b200 import scenes  # noqa: E402

PROBE = os.path.join(ROOT, "oracle", "_ref", "edx_probe")
OUT = os.path.join(ROOT, "tests", "golden", "edx_pins.json")


def _grid(n, textured, forms, seed):
    """An n x n grid of quads in the z = 0 plane. `forms` cycles the corner
    syntax over the faces: 'i', 'i//n', 'i/t', 'i/t/n' or 'neg' (negative,
    relative position indices)."""
    rng = np.random.default_rng(seed)
    lines = ["# grid of quads, seeded"]
    k = n + 1
    for y in range(k):
        for x in range(k):
            lines.append(f"v {x / n - 0.5:.6f} {y / n - 0.5:.6f} {rng.uniform(-0.01, 0.01):.7f}")
    if textured:
        for y in range(k):
            for x in range(k):
                lines.append(f"vt {x / n:.6f} {y / n:.6f}")
    lines.append("vn 0 0 1")
    nv = k * k
    for y in range(n):
        for x in range(n):
            q = [y * k + x, y * k + x + 1, (y + 1) * k + x + 1, (y + 1) * k + x]
            form = forms[(y * n + x) % len(forms)]
            if form == "neg":
                corners = [str(i - nv) for i in q]
            elif form == "i":
                corners = [str(i + 1) for i in q]
            elif form == "i//n":
                corners = [f"{i + 1}//1" for i in q]
            elif form == "i/t":
                corners = [f"{i + 1}/{i + 1}" for i in q]
            else:
                corners = [f"{i + 1}/{i + 1}/1" for i in q]
            lines.append("f " + " ".join(corners))
    return "\n".join(lines) + "\n"


def _triangles_with_vt_vn():
    return "\n".join([
        "# a tetrahedron with texture coordinates and normals",
        "v 0.0 0.0 0.0", "v 1.0 0.0 0.0", "v 0.0 1.0 0.0", "v 0.0 0.0 1.0",
        "vt 0.125 0.875", "vt 0.3 0.7", "vt 0.6180339887 0.1", "vt 0.999999 0.000001",
        "vn 0 0 -1", "vn 0 -1 0", "vn -1 0 0", "vn 0.57735 0.57735 0.57735",
        "f 1/1/1 3/3/1 2/2/1", "f 1/1/2 2/2/2 4/4/2", "f 1/1/3 4/4/3 3/3/3", "f 2/2/4 3/3/4 4/4/4",
    ]) + "\n"


def _icosphere(level, seed):
    """The icosphere of the small configuration, written with 6 decimals and
    spherical texture coordinates with 9 significant digits."""
    P, F = scenes.icosphere(level, 1.0)
    rng = np.random.default_rng(seed)
    lines = ["# icosphere"]
    for p in P:
        lines.append("v " + " ".join(f"{float(c):.6f}" for c in p))
    for _ in range(len(P)):
        u, v = rng.uniform(0.0, 1.0, 2)
        lines.append(f"vt {u:.9g} {v:.9g}")
    for f in F:
        lines.append("f " + " ".join(f"{int(i) + 1}/{int(i) + 1}" for i in f))
    return "\n".join(lines) + "\n"


def _soup(nv, nf, seed):
    """Random vertices printed with 1-9 decimals or in exponent form, and
    random triangles over them: boundary, interior and non-manifold edges
    (three or more faces on one edge) all occur."""
    rng = np.random.default_rng(seed)
    lines = ["# random triangle soup"]
    for _ in range(nv):
        cs = []
        for c in rng.normal(0.0, 3.0, 3):
            kind = rng.integers(0, 3)
            if kind == 0:
                cs.append(f"{c:.{int(rng.integers(1, 10))}f}")
            elif kind == 1:
                cs.append(f"{c:.6e}")
            else:
                cs.append(repr(float(np.float32(c))))
        lines.append("v " + " ".join(cs))
    for _ in range(nv):
        u, v = rng.uniform(0.0, 1.0, 2)
        lines.append(f"vt {u:.{int(rng.integers(2, 10))}f} {v:.{int(rng.integers(2, 10))}f}")
    hub = [0, 1]
    for i in range(nf):
        if i % 10 == 0:
            # faces on the shared edge (0, 1): a non-manifold fan
            c = int(rng.integers(2, nv))
            tri = [hub[0], hub[1], c] if i % 20 == 0 else [hub[1], hub[0], c]
        else:
            tri = [int(x) for x in rng.choice(nv, 3, replace=False)]
        lines.append("f " + " ".join(f"{t + 1}/{t + 1}" for t in tri))
    return "\n".join(lines) + "\n"


def obj_cases():
    return {
        "tetra_vt_vn": _triangles_with_vt_vn(),
        "quads_untextured_forms": _grid(4, False, ["i", "i//n", "neg"], 1),
        "quads_textured": _grid(3, True, ["i/t", "i/t/n"], 2),
        "icosphere_level2": _icosphere(2, 3),
        "soup": _soup(150, 240, 4),
    }


def _hdr_bytes(rgbe: np.ndarray, rle: bool) -> bytes:
    """A Radiance file of the given [H, W, 4] RGBE bytes: flat, or with
    run-length-encoded scanlines (runs of 3 or more equal bytes, dumps of at
    most 128 between them)."""
    H, W, _ = rgbe.shape
    out = bytearray(b"#?RADIANCE\n# seeded test image\nFORMAT=32-bit_rle_rgbe\n\n" + f"-Y {H} +X {W}\n".encode())
    if not rle:
        return bytes(out + rgbe.tobytes())
    for j in range(H):
        out += bytes([2, 2, W >> 8, W & 255])
        for k in range(4):
            row = rgbe[j, :, k]
            i = 0
            while i < W:
                n = 1
                while i + n < W and n < 127 and row[i + n] == row[i]:
                    n += 1
                if n >= 3:
                    out += bytes([128 + n, int(row[i])])
                    i += n
                    continue
                s0 = i
                while i < W and i - s0 < 128 and not (i + 2 < W and row[i] == row[i + 1] == row[i + 2]):
                    i += 1
                out += bytes([i - s0]) + row[s0:i].tobytes()
    return bytes(out)


def bitmap_cases():
    """Seeded images in every format the reference's stb_image reads and PIL
    writes, as file bytes."""
    import io

    from PIL import Image
    rng = np.random.default_rng(5)
    rgb = (np.arange(16 * 16 * 3) % 256).astype(np.uint8).reshape(16, 16, 3)   # every 8-bit value
    rgb[8:] = rng.integers(0, 256, (8, 16, 3), dtype=np.uint8)

    def enc(img, fmt):
        b = io.BytesIO()
        img.save(b, fmt)
        return b.getvalue()

    cases = {
        "rgb.png": enc(Image.fromarray(rgb, "RGB"), "PNG"),
        "gray.png": enc(Image.fromarray(rgb[:, :, 0], "L"), "PNG"),
        "gray_alpha.png": enc(Image.fromarray(rgb[:, :, :2].copy(), "LA"), "PNG"),
        "rgba.png": enc(Image.fromarray(np.concatenate([rgb, rgb[:, :, :1]], 2), "RGBA"), "PNG"),
        "palette.png": enc(Image.fromarray(rgb, "RGB").convert("P"), "PNG"),
        "gray16.png": enc(Image.fromarray(rng.integers(0, 65536, (8, 8), dtype=np.uint16)), "PNG"),
        "rgb.bmp": enc(Image.fromarray(rgb, "RGB"), "BMP"),
        "rgb.tga": enc(Image.fromarray(rgb, "RGB"), "TGA"),
        "rgb.ppm": enc(Image.fromarray(rgb, "RGB"), "PPM"),
        "gray.pgm": enc(Image.fromarray(rgb[:, :, 0], "L"), "PPM"),
        "palette.gif": enc(Image.fromarray(rgb, "RGB").convert("P"), "GIF"),
        "rgb.jpg": enc(Image.fromarray(rgb, "RGB"), "JPEG"),
    }
    e = rng.integers(100, 160, (5, 4, 1), dtype=np.uint8)
    e[0, 0] = 0
    flat = np.concatenate([rng.integers(0, 256, (5, 4, 3), dtype=np.uint8), e], 2)
    cases["flat_w4.hdr"] = _hdr_bytes(flat, False)
    blocks = np.repeat(np.repeat(rng.integers(0, 256, (3, 4, 4), dtype=np.uint8), 2, 0), 4, 1)   # 6 x 16, runs
    blocks[..., 3] = np.where(blocks[..., 3] < 8, 0, blocks[..., 3] // 2 + 1)   # low exponents: subnormal scales
    blocks[1, 3:9] = rng.integers(0, 256, (6, 4), dtype=np.uint8)                # a stretch to dump
    blocks[4, 0:4] = [[1, 17, 255, 1], [3, 5, 7, 2], [200, 1, 9, 3], [255, 255, 255, 1]]   # subnormal results
    blocks[5, 4:8, 3] = 0                                                          # exponent 0: black
    cases["rle_w16.hdr"] = _hdr_bytes(blocks, True)
    unmarked = np.concatenate([rng.integers(3, 256, (3, 12, 3), dtype=np.uint8),
                               rng.integers(120, 140, (3, 12, 1), dtype=np.uint8)], 2)
    cases["unmarked_w12.hdr"] = _hdr_bytes(unmarked, False)
    return cases


def camera_cases():
    cams = [
        ((0.0, 0.0, 4.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 256, 256, 45.0),
        ((0.0, 0.0, 4.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 512, 512, 45.0),
        ((3.0, 2.0, -5.0), (0.0, 0.5, 0.0), (0.0, 1.0, 0.0), 320, 240, 30.0),
        ((0.1, 5.0, 0.2), (0.0, 0.0, 0.0), (1.0, 0.0, 0.0), 64, 128, 90.0),
    ]
    for c in scenes.fibonacci_cameras(6, 4.0, [128, 384], seed=1):
        cams.append((tuple(float(x) for x in c.pos), tuple(float(x) for x in c.target), tuple(float(x) for x in c.up),
                     c.width, c.height, float(c.fov)))
    return cams


def _probe(*args):
    out = subprocess.run([PROBE, *args], capture_output=True, text=True, check=True)
    return json.loads(out.stdout)


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle", "edx"), f"REF={ref}"], check=True)
    out = {"obj": {}, "camera": []}
    with tempfile.TemporaryDirectory() as d:
        for name, text in obj_cases().items():
            path = os.path.join(d, name + ".obj")
            with open(path, "w") as f:
                f.write(text)
            out["obj"][name] = {"text": text, "reference": _probe("obj", path)}
    out["bitmap"] = {}
    with tempfile.TemporaryDirectory() as d:
        for name, raw in bitmap_cases().items():
            path = os.path.join(d, name)
            with open(path, "wb") as f:
                f.write(raw)
            out["bitmap"][name] = {"bytes": base64.b64encode(raw).decode(), "reference": _probe("bitmap", path)}
    for pos, tgt, up, w, h, fov in camera_cases():
        args = [repr(float(np.float32(x))) for x in (*pos, *tgt, *up)] + [str(w), str(h), repr(float(fov))]
        out["camera"].append({"args": args, "reference": _probe("camera", *args)})
    with open(OUT, "w") as f:
        json.dump(out, f, separators=(",", ":"))
    print(f"wrote {OUT}: {len(out['obj'])} meshes, {len(out['bitmap'])} images, {len(out['camera'])} cameras")


if __name__ == "__main__":
    main()
