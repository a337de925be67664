"""The C-ABI library loads without a GPU, exports every symbol include/trn.h
declares, and its host-only entry points behave (camera construction and
argument validation)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from oracle import tr_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    txt = open(os.path.join(ROOT, "include", "trn.h")).read()
    return sorted(set(re.findall(r"\b(trn_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol(built_lib):
    lib = C.CDLL(built_lib)
    names = _declared()
    assert "trn_render_grad" in names and "trn_scene_create" in names
    for n in names:
        assert hasattr(lib, n), n


def test_python_binding_covers_header(built_lib):
    from tensorray_b200 import _abi
    assert sorted(_abi.exported_symbols()) == _declared()


def test_camera_init_matches_oracle_restatement(built_lib):
    from tensorray_b200.api import Camera
    for pos, tgt, w, h, fov in [((0, 0, 4), (0, 0, 0), 256, 256, 45.0), ((1, 2, 3), (0, -1, 0), 320, 200, 30.0)]:
        cam = Camera(pos, tgt, (0, 1, 0), w, h, fov).matrices()
        ref = O.camera_matrices(pos, tgt, (0, 1, 0), w, h, fov)
        for k in ("raster_to_camera", "view_inv", "world_to_sample", "sample_to_camera", "raster_to_world"):
            np.testing.assert_allclose(cam[k], ref[k], rtol=2e-6, atol=1e-7)
        np.testing.assert_allclose(cam["inv_area"], ref["inv_area"], rtol=1e-6)
        np.testing.assert_allclose(cam["plane_len_x"], ref["plane_len_x"], rtol=1e-6)


def test_invalid_arguments_are_reported(built_lib):
    from tensorray_b200 import _abi
    lib = _abi.load()
    cam = _abi.TrnCamera()
    z = (C.c_float * 3)(0, 0, 0)
    assert lib.trn_camera_init(C.byref(cam), z, z, z, 0, 10, C.c_float(45.0)) == -1
    assert b"invalid" in lib.trn_last_error()
    h = C.c_void_p()
    d = _abi.TrnSceneDesc()
    assert lib.trn_scene_create(C.byref(d), C.byref(h)) == -1
    assert b"incomplete" in lib.trn_last_error()
    # an out-of-range index is rejected on the host before any device work
    pos = np.zeros((3, 3), np.float32)
    idx = np.array([[0, 1, 5]], np.int32)
    one = np.zeros(3, np.int32)
    d = _abi.TrnSceneDesc()
    d.num_vertices, d.num_triangles, d.num_meshes, d.num_bsdfs = 3, 1, 1, 1
    d.positions = pos.ctypes.data_as(C.POINTER(C.c_float))
    d.indices = idx.ctypes.data_as(C.POINTER(C.c_int))
    d.vertex_mesh = one.ctypes.data_as(C.POINTER(C.c_int))
    d.triangle_mesh = one.ctypes.data_as(C.POINTER(C.c_int))
    sm = np.zeros(1, np.uint8)
    d.mesh_smooth = sm.ctypes.data_as(C.POINTER(C.c_ubyte))
    mb = np.zeros(1, np.int32)
    ml = np.full(1, -1, np.int32)
    d.mesh_bsdf = mb.ctypes.data_as(C.POINTER(C.c_int))
    d.mesh_light = ml.ctypes.data_as(C.POINTER(C.c_int))
    bs = (_abi.TrnBsdf * 1)()
    d.bsdfs = bs
    assert lib.trn_scene_create(C.byref(d), C.byref(h)) == -1
    assert b"index out of range" in lib.trn_last_error()


def test_sample_layout_dims():
    from tensorray_b200 import api
    assert api.sample_dims(0, 3) == 17
    assert api.sample_dims(2, 3) == 12
    assert api.sample_dims(3, 3) == 19
    assert api.sample_slots(4, 8, 8, 4) == 64


def test_camera_init_update_resize():
    """The binding's Camera() / init / update / resize (TensorRay.cpp:143-151)
    over trn_camera_init: an empty camera takes a pose with init, copies one
    with update, and keeps its pose through resize."""
    from tensorray_b200 import api
    a = api.Camera((0.0, 0.0, 4.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 256, 128, 45.0)
    b = api.Camera()
    assert b.width == 0 and b.pos is None
    b.update(a)
    ma, mb = a.matrices(), b.matrices()
    assert all(np.array_equal(ma[k], mb[k]) for k in ma)
    b.resize(512, 256)
    ref = api.Camera((0.0, 0.0, 4.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 512, 256, 45.0).matrices()
    assert (b.width, b.height) == (512, 256) and all(np.array_equal(b.matrices()[k], ref[k]) for k in ref)
    c = api.Camera()
    c.init((1.0, 2.0, 3.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 64, 64)
    assert c.fov == 35.0
    with pytest.raises(RuntimeError, match="not initialised"):
        api.Camera().resize(8, 8)
