"""ctypes binding of the trn C-ABI (include/trn.h).

This is the same binding a maintainer would add on the reference side: plain
pointers and sizes, status codes, a thread-local error string. Loading fails
loudly when the shared library is missing; there is no fallback path.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("TRN_LIB") or os.path.join(_HERE, "_lib", "libtrn.so")

TRN_PATH_TRACER = 0
TRN_PRIMARY_EDGE = 1
TRN_DIRECT_EDGE = 2
TRN_INDIRECT_EDGE = 3
TRN_PIXEL_EDGE = 4


class TrnBsdf(C.Structure):
    _fields_ = [("type", C.c_int), ("texture", C.c_int), ("albedo", C.c_float * 3),
                ("specular", C.c_float * 3), ("roughness", C.c_float)]


class TrnTexture(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("data", C.POINTER(C.c_float))]


class TrnSceneDesc(C.Structure):
    _fields_ = [
        ("num_vertices", C.c_int), ("num_triangles", C.c_int), ("num_uvs", C.c_int),
        ("num_meshes", C.c_int), ("num_lights", C.c_int), ("num_bsdfs", C.c_int),
        ("num_textures", C.c_int),
        ("positions", C.POINTER(C.c_float)), ("indices", C.POINTER(C.c_int)),
        ("uvs", C.POINTER(C.c_float)), ("uv_indices", C.POINTER(C.c_int)),
        ("vertex_mesh", C.POINTER(C.c_int)), ("triangle_mesh", C.POINTER(C.c_int)),
        ("mesh_smooth", C.POINTER(C.c_ubyte)), ("mesh_bsdf", C.POINTER(C.c_int)),
        ("mesh_light", C.POINTER(C.c_int)), ("mesh_translation", C.POINTER(C.c_float)),
        ("light_radiance", C.POINTER(C.c_float)), ("bsdfs", C.POINTER(TrnBsdf)),
        ("textures", C.POINTER(TrnTexture)),
    ]


class TrnCamera(C.Structure):
    _fields_ = [
        ("width", C.c_int), ("height", C.c_int), ("pos", C.c_float * 3), ("dir", C.c_float * 3),
        ("raster_to_camera", C.c_float * 16), ("view_inv", C.c_float * 16),
        ("world_to_sample", C.c_float * 16), ("sample_to_camera", C.c_float * 16),
        ("raster_to_world", C.c_float * 16), ("inv_area", C.c_float),
        ("plane_len_x", C.c_float), ("plane_len_y", C.c_float),
    ]


class TrnRenderOptions(C.Structure):
    _fields_ = [("seed", C.c_int), ("max_bounces", C.c_int), ("spp", C.c_int), ("sppe", C.c_int),
                ("sppse0", C.c_int), ("sppse1", C.c_int), ("sppe0", C.c_int),
                ("g_direct", C.c_int), ("g_direct_depth", C.c_int), ("g_direct_max_size", C.c_int),
                ("g_direct_spp", C.c_int), ("g_direct_thold", C.c_float), ("g_eps", C.c_float)]


class TrnSamples(C.Structure):
    _fields_ = [("samples", C.c_void_p), ("stride", C.c_longlong)]


class TrnLaunch(C.Structure):
    _fields_ = [("block", C.c_int), ("blocks_per_sm", C.c_int), ("chunk", C.c_int), ("round_log2", C.c_int)]


class TrnView(C.Structure):
    _fields_ = [("camera", TrnCamera), ("spp", C.c_int), ("seed", C.c_int), ("pixel_offset", C.c_longlong),
                ("slot_offset", C.c_longlong), ("weight", C.c_float), ("max_bounces", C.c_int),
                ("grad_positions", C.c_void_p), ("grad_vertex_normals", C.c_void_p), ("grad_texels", C.c_void_p),
                ("image", C.c_void_p), ("dLdI", C.c_void_p)]


_SIGNATURES = {
    "trn_last_error": (C.c_char_p, []),
    "trn_version": (C.c_char_p, []),
    "trn_camera_init": (C.c_int, [C.POINTER(TrnCamera), C.POINTER(C.c_float), C.POINTER(C.c_float),
                                  C.POINTER(C.c_float), C.c_int, C.c_int, C.c_float]),
    "trn_mesh_edges": (C.c_longlong, [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_longlong]),
    "trn_scene_create": (C.c_int, [C.POINTER(TrnSceneDesc), C.POINTER(C.c_void_p)]),
    "trn_scene_configure": (C.c_int, [C.c_void_p, C.c_void_p]),
    "trn_scene_destroy": (C.c_int, [C.c_void_p]),
    "trn_scene_refit": (C.c_int, [C.c_void_p, C.c_void_p]),
    "trn_scene_set_translation": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "trn_scene_set_positions": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "trn_scene_set_texels": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "trn_scene_get_geometry": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "trn_scene_counts": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                   C.POINTER(C.c_longlong), C.POINTER(C.c_int)]),
    "trn_intersect": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "trn_occluded": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                               C.c_void_p, C.c_void_p]),
    "trn_render_fwd": (C.c_int, [C.c_void_p, C.POINTER(TrnCamera), C.POINTER(TrnRenderOptions), C.c_int,
                                 C.POINTER(TrnSamples), C.c_void_p, C.c_void_p]),
    "trn_render_grad": (C.c_int, [C.c_void_p, C.POINTER(TrnCamera), C.POINTER(TrnRenderOptions), C.c_int,
                                  C.POINTER(TrnSamples), C.c_void_p, C.c_void_p]),
    "trn_render_grad_noalloc": (C.c_int, [C.c_void_p, C.POINTER(TrnCamera), C.POINTER(TrnRenderOptions), C.c_int,
                                          C.POINTER(TrnSamples), C.c_void_p, C.c_void_p]),
    "trn_scene_get_grads": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "trn_scene_clear_grads": (C.c_int, [C.c_void_p, C.c_void_p]),
    "trn_viewset_create": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(TrnView), C.POINTER(C.c_void_p)]),
    "trn_viewset_destroy": (C.c_int, [C.c_void_p]),
    "trn_viewset_update": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(TrnView)]),
    "trn_viewset_num_pixels": (C.c_int, [C.c_void_p, C.POINTER(C.c_longlong)]),
    "trn_viewset_reserve": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "trn_viewset_path_cache": (C.c_int, [C.c_void_p, C.c_longlong]),
    "trn_scene_path_cache": (C.c_int, [C.c_void_p, C.c_longlong]),
    "trn_render_views_fwd": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(TrnRenderOptions), C.c_int,
                                       C.POINTER(TrnSamples), C.POINTER(TrnLaunch), C.c_void_p, C.c_void_p]),
    "trn_render_views_grad": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(TrnRenderOptions), C.c_int,
                                        C.POINTER(TrnSamples), C.POINTER(TrnLaunch), C.c_void_p, C.c_void_p]),
    "trn_views_loss": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "trn_scene_finalize_grads": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "trn_kernel_launches": (C.c_ulonglong, []),
    "trn_stats_enable": (C.c_int, [C.c_void_p, C.c_int]),
    "trn_stats_read": (C.c_int, [C.c_void_p, C.POINTER(C.c_ulonglong), C.c_int, C.c_void_p]),
}

_lib = None


def load() -> C.CDLL:
    """Load libtrn.so and declare every exported prototype."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"trn native library not built: {LIB_PATH} (run tensorray_b200/build.py)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def exported_symbols() -> list[str]:
    return list(_SIGNATURES)


def check(rc: int, what: str) -> None:
    if rc != 0:
        msg = load().trn_last_error().decode()
        raise RuntimeError(f"{what} failed: {msg}")
