"""XML scene ingest (SceneLoader.cpp:36-408) on the CPU: the supported
elements, transforms, bitmap textures and error reporting, and an XML copy
of the icosphere configuration that loads to the same scene arrays as the
programmatic one."""
import os

import numpy as np
import pytest
import torch

from tensorray_b200 import scene_xml, scenes


def write_obj(path, P, F, uv=None):
    with open(path, "w") as f:
        for p in P:
            f.write("v %.9g %.9g %.9g\n" % tuple(float(x) for x in p))
        if uv is not None:
            for t in uv:
                f.write("vt %.9g %.9g\n" % (float(t[0]), 1.0 - float(t[1])))
        for tri in F:
            if uv is None:
                f.write("f %d %d %d\n" % tuple(int(i) + 1 for i in tri))
            else:
                f.write("f %s\n" % " ".join(f"{int(i) + 1}/{int(i) + 1}" for i in tri))


def config1_xml(d, width=64, height=48):
    """The icosphere configuration as an XML scene with three OBJ files."""
    spec = scenes.config1_scene(width, height)
    names = ["sphere.obj", "ground.obj", "light.obj"]
    for m, n in zip(spec.meshes, names):
        write_obj(os.path.join(d, n), m.positions, m.faces)
    xml = f"""<?xml version="1.0"?>
<scene version="0.5.0">
  <bsdf type="diffuse" id="sphere_mat"><rgb name="reflectance" value="0.7"/></bsdf>
  <bsdf type="diffuse" id="gray"><spectrum name="reflectance" value="0.5, 0.5, 0.5"/></bsdf>
  <shape type="obj" id="sphere">
    <string name="filename" value="{names[0]}"/>
    <boolean name="face_normals" value="false"/>
    <ref id="sphere_mat"/>
  </shape>
  <shape type="obj" id="ground"><string name="filename" value="{names[1]}"/><ref id="gray"/></shape>
  <shape type="obj" id="light">
    <string name="filename" value="{names[2]}"/>
    <ref id="gray"/>
    <emitter type="area"><rgb name="radiance" value="10"/></emitter>
  </shape>
  <sensor type="perspective">
    <float name="fov" value="45"/>
    <transform name="to_world"><lookat origin="0, 0, 4" target="0, 0, 0" up="0, 1, 0"/></transform>
    <film type="hdrfilm"><integer name="width" value="{width}"/><integer name="height" value="{height}"/></film>
  </sensor>
</scene>
"""
    path = os.path.join(d, "scene.xml")
    with open(path, "w") as f:
        f.write(xml)
    return path, spec


def test_xml_copy_of_the_icosphere_configuration_loads_the_same_arrays(tmp_path):
    path, ref = config1_xml(str(tmp_path))
    spec = scene_xml.load_xml(path)
    a, b = spec.arrays(), ref.arrays()
    for k in ("positions", "indices", "mesh_bsdf", "mesh_light", "mesh_smooth", "light_radiance"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    # albedos as the renderer reads them: float32
    assert [(x.type, tuple(np.float32(x.albedo))) for x in spec.bsdfs] == \
        [(x.type, tuple(np.float32(x.albedo))) for x in ref.bsdfs]
    assert spec.cameras == ref.cameras


def test_transforms_textures_microfacet_and_errors(tmp_path):
    d = str(tmp_path)
    P = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], np.float32)
    F = np.array([[0, 1, 2], [0, 2, 3]])
    write_obj(os.path.join(d, "quad.obj"), P, F, uv=P[:, :2])
    from PIL import Image
    tex = (np.arange(4 * 5 * 3).reshape(4, 5, 3) * 4).astype(np.uint8)
    Image.fromarray(tex).save(os.path.join(d, "tex.png"))
    xml = """<scene>
  <bsdf type="diffuse" id="t"><texture type="bitmap" name="reflectance"><string name="filename" value="tex.png"/></texture></bsdf>
  <bsdf type="microfacet" id="g"><float name="roughness" value="0.3"/>
    <spectrum name="diffuseReflectance" value="0.2 0.3 0.4"/><spectrum name="specularReflectance" value="0.04"/></bsdf>
  <shape type="obj"><string name="filename" value="quad.obj"/><ref id="t"/>
    <transform name="toWorld"><scale x="2"/><rotate z="1" angle="90"/><translate x="1" y="2" z="3"/></transform>
  </shape>
  <shape type="obj"><string name="filename" value="quad.obj"/><ref id="g"/></shape>
</scene>"""
    with open(os.path.join(d, "s.xml"), "w") as f:
        f.write(xml)
    spec = scene_xml.load_xml(os.path.join(d, "s.xml"))
    np.testing.assert_allclose(spec.textures[0], (tex / 255.0) ** 2.2, rtol=1e-6)
    assert spec.bsdfs[0].texture == 0
    g = spec.bsdfs[1]
    assert g.type == scenes.MICROFACET and g.roughness == pytest.approx(0.3)
    assert g.albedo == pytest.approx((0.2, 0.3, 0.4)) and g.specular == pytest.approx((0.04, 0.04, 0.04))
    # scale x2, then 90 degrees about z, then translate (1, 2, 3)
    q = P.astype(np.float64) * [2, 1, 1]
    q = np.stack([-q[:, 1], q[:, 0], q[:, 2]], 1) + [1, 2, 3]
    np.testing.assert_allclose(spec.meshes[0].positions, q, atol=1e-6)
    np.testing.assert_array_equal(spec.meshes[1].positions, P)
    assert spec.meshes[0].smooth is False and spec.meshes[0].uvs is not None
    for bad, msg in [('<bsdf type="roughconductor" id="r"/>', "unsupported BSDF"),
                     ('<shape type="obj"><string name="filename" value="quad.obj"/><ref id="nope"/></shape>',
                      "unknown BSDF id"),
                     ('<shape type="sphere"/>', "unsupported shape")]:
        with open(os.path.join(d, "bad.xml"), "w") as f:
            f.write("<scene>" + bad + "</scene>")
        with pytest.raises(scene_xml.SceneXmlError, match=msg):
            scene_xml.load_xml(os.path.join(d, "bad.xml"))


def test_parse_vector_repeats_the_last_component():
    np.testing.assert_array_equal(scene_xml.parse_vector("0.5", 3, allow_empty=True), [0.5, 0.5, 0.5])
    np.testing.assert_array_equal(scene_xml.parse_vector("1, 2 3"), [1, 2, 3])
    with pytest.raises(scene_xml.SceneXmlError):
        scene_xml.parse_vector("1 2")


def _hdr(rows, header=b"FORMAT=32-bit_rle_rgbe\n", res=None, body=None):
    """A flat Radiance file of the given RGBE rows."""
    a = np.asarray(rows, np.uint8)
    H, W = a.shape[:2]
    res = res if res is not None else f"-Y {H} +X {W}\n".encode()
    return b"#?RADIANCE\n" + header + b"\n" + res + (a.tobytes() if body is None else body)


def test_radiance_textures_load_linear_and_through_xml(tmp_path):
    d = str(tmp_path)
    # (r, g, b, e): value = c * 2^(e - 136); e = 0 is black
    rows = [[[128, 64, 32, 129], [255, 0, 1, 136], [9, 9, 9, 0]]]
    with open(os.path.join(d, "sky.hdr"), "wb") as f:
        f.write(_hdr(rows))
    t = scene_xml.load_bitmap(os.path.join(d, "sky.hdr"))
    assert t.dtype == np.float32 and t.shape == (1, 3, 3)
    np.testing.assert_array_equal(t[0, 0], np.float32([128, 64, 32]) * np.float32(2.0 ** -7))
    np.testing.assert_array_equal(t[0, 1], np.float32([255, 0, 1]))
    np.testing.assert_array_equal(t[0, 2], np.zeros(3, np.float32))
    P = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0]], np.float32)
    write_obj(os.path.join(d, "tri.obj"), P, np.array([[0, 1, 2]]), uv=P[:, :2])
    with open(os.path.join(d, "s.xml"), "w") as f:
        f.write('<scene><bsdf type="diffuse" id="t"><texture type="bitmap" name="reflectance">'
                '<string name="filename" value="sky.hdr"/></texture></bsdf>'
                '<shape type="obj"><string name="filename" value="tri.obj"/><ref id="t"/></shape></scene>')
    spec = scene_xml.load_xml(os.path.join(d, "s.xml"))
    np.testing.assert_array_equal(spec.textures[0], t)


@pytest.mark.parametrize("raw, msg", [
    (_hdr([[[1, 2, 3, 130]]], header=b"FORMAT=32-bit_rle_xyze\n"), "unsupported HDR format"),
    (_hdr([[[1, 2, 3, 130]]], res=b"+Y 1 +X 1\n"), "unsupported HDR data layout"),
    (_hdr([[[1, 2, 3, 130]] * 2], body=b"\x01\x02\x03"), "truncated HDR data"),
    # an RLE scanline whose length field disagrees with the width
    (_hdr([[[0, 0, 0, 0]] * 8], body=bytes([2, 2, 0, 9]) + bytes(64)), "invalid decoded scanline length"),
    # a dump of zero bytes (stb would loop on it) and a run past the scanline's end
    (_hdr([[[0, 0, 0, 0]] * 8], body=bytes([2, 2, 0, 8, 0])), "corrupt HDR dump"),
    (_hdr([[[0, 0, 0, 0]] * 8], body=bytes([2, 2, 0, 8, 128 + 9, 5])), "corrupt HDR run"),
])
def test_radiance_errors(tmp_path, raw, msg):
    path = os.path.join(str(tmp_path), "bad.hdr")
    with open(path, "wb") as f:
        f.write(raw)
    with pytest.raises(scene_xml.SceneXmlError, match=msg):
        scene_xml.load_bitmap(path)


def test_images_the_reference_cannot_load_are_refused(tmp_path):
    from PIL import Image
    d = str(tmp_path)
    Image.fromarray(np.arange(16, dtype=np.uint16).reshape(4, 4) * 4000).save(os.path.join(d, "g16.png"))
    Image.fromarray(np.zeros((4, 4, 3), np.uint8)).save(os.path.join(d, "t.tiff"))
    for name, msg in [("g16.png", "16-bit PNGs"), ("t.tiff", "TIFF")]:
        with pytest.raises(scene_xml.SceneXmlError, match=msg):
            scene_xml.load_bitmap(os.path.join(d, name))


class _FakeSceneLib:
    """The library's scene creation and counts, without a device: records
    the descriptor's sizes."""

    def trn_scene_create(self, d, out):
        self.desc = (d._obj.num_vertices, d._obj.num_triangles, d._obj.num_meshes, d._obj.num_bsdfs)
        return 0

    def trn_scene_counts(self, h, nv, nt, ne, ntex, nm):
        nv._obj.value, nt._obj.value = self.desc[0], self.desc[1]
        ne._obj.value, ntex._obj.value, nm._obj.value = 0, 0, self.desc[2]
        return 0


def test_scene_load_file_reads_the_xml(tmp_path):
    """Scene().load_file(path), as the reference's scripts load a scene
    (Scene::LoadFromFile, Scene.cpp:41-44), gives the shapes, BSDFs and
    cameras of scene_xml.load_xml (library calls faked: no GPU here)."""
    import ctypes

    from tensorray_b200 import api
    path, ref = config1_xml(str(tmp_path))
    sc = api.Scene.__new__(api.Scene)
    sc.device, sc._lib, sc._h, sc._dirty = torch.device("cpu"), _FakeSceneLib(), ctypes.c_void_p(), True
    sc.shapes, sc.bsdfs, sc.cameras = [], [], []
    sc.load_file(path)
    assert sc._lib.desc == (sum(len(m.positions) for m in ref.meshes), sum(len(m.faces) for m in ref.meshes),
                            len(ref.meshes), len(ref.bsdfs))
    assert [s.get_vertex_count() for s in sc.shapes] == [len(m.positions) for m in ref.meshes]
    assert [(c.width, c.height) for c in sc.cameras] == [(c.width, c.height) for c in ref.cameras]
    assert sc.num_bsdf == len(ref.bsdfs) and sc.get_width(0) == ref.cameras[0].width
