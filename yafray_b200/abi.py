"""ctypes mirror of include/yr.h (the C ABI) and the loader of the native library.

The native library is ``yafray_b200/libyafray_b200.so`` (CUDA + host C++,
built in-tree by ``yafray_b200.build``).  There is no Python or CPU fallback
for any compute entry: if the library or a CUDA device is missing, calls fail
with an error.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# YAFRAY_B200_LIB selects another build of the library (variant builds for A/B timing)
LIB_PATH = os.environ.get("YAFRAY_B200_LIB", os.path.join(HERE, "libyafray_b200.so"))

YR_OK = 0
STATUS_NAMES = {
    0: "YR_OK", 1: "YR_ERR_INVALID_ARG", 2: "YR_ERR_CUDA", 3: "YR_ERR_OUT_OF_MEMORY",
    4: "YR_ERR_ITERATION_CAP", 5: "YR_ERR_STACK_OVERFLOW", 6: "YR_ERR_BAD_TREE",
    7: "YR_ERR_CANCELLED", 8: "YR_ERR_UNSUPPORTED", 9: "YR_ERR_EMPTY_SCENE",
    10: "YR_ERR_NO_DEVICE", 11: "YR_ERR_TOO_LARGE",
}

YR_TEX_NONE, YR_TEX_MUSGRAVE_FBM, YR_TEX_CLOUDS, YR_TEX_MARBLE, YR_TEX_WOOD, YR_TEX_VORONOI = 0, 1, 2, 3, 4, 5
(YR_TEX_MUSGRAVE_MULTIFRACTAL, YR_TEX_MUSGRAVE_HETEROTERRAIN, YR_TEX_MUSGRAVE_HYBRIDMF,
 YR_TEX_MUSGRAVE_RIDGEDMF) = 6, 7, 8, 9
YR_TEX_DISTORTED_NOISE, YR_TEX_GRADIENT = 10, 11
# noise_type names in newNoise order (basictex.cc:34-60) -> YR_NOISE_*
NOISE_TYPES = {"newperlin": 0, "stdperlin": 1, "blender": 2, "voronoi_f1": 3, "voronoi_f2": 4, "voronoi_f3": 5,
               "voronoi_f4": 6, "voronoi_f2f1": 7, "voronoi_crackle": 8, "cellnoise": 9}
WAVE_SHAPES = {"sin": 0, "saw": 1, "tri": 2}
DIST_METRICS = {"real": 0, "squared": 1, "manhattan": 2, "chebychev": 3, "minkovsky_half": 4,
                "minkovsky_four": 5, "minkovsky": 6}
GRADIENT_TYPES = {"linear": 0, "quadratic": 1, "cubic": 2, "diagonal": 3, "sphere": 4, "halo": 5}
MOD_MODES = {"mix": 0, "mul": 1, "add": 2, "sub": 3}
YR_LIGHT_POINT, YR_LIGHT_AREA, YR_LIGHT_HEMI, YR_LIGHT_PATH = 0, 1, 2, 3
YR_BATCH_AUTO, YR_BATCH_TILES, YR_BATCH_WAVES = 0, 1, 2
YR_TEXCO_GLOBAL, YR_TEXCO_ORCO, YR_TEXCO_NORMAL, YR_TEXCO_WINDOW, YR_TEXCO_REFLECT, YR_TEXCO_UV = 0, 1, 2, 3, 4, 5
YR_PROJ_DEFAULT, YR_PROJ_X, YR_PROJ_Y, YR_PROJ_Z, YR_PROJ_NONE = 0, 1, 2, 3, 4
YR_RENDER_SHADOW_TREE, YR_RENDER_EXACT_ORDER, YR_RENDER_TONEMAP = 1, 2, 4
YR_RENDER_CLAMP_RGB, YR_RENDER_ALPHA_PREMULTIPLY = 8, 16
YR_RENDER_GPU_KD_BUILD = 32
YR_IMAGE_TGA, YR_IMAGE_HDR, YR_IMAGE_ALPHA = 0, 1, 1
YR_PER_TRIANGLE = 0xFFFFFFFF
MISS = 0xFFFFFFFF

f3 = C.c_float * 3


class YrKdNode(C.Structure):
    _fields_ = [("word", C.c_uint32), ("flags", C.c_uint32)]


class YrKdTree(C.Structure):
    _fields_ = [
        ("nodes", C.POINTER(YrKdNode)), ("nnodes", C.c_uint32),
        ("prims", C.POINTER(C.c_uint32)), ("nprims", C.c_uint32),
        ("bound", C.c_float * 6), ("max_depth", C.c_int32), ("max_leaf_size", C.c_int32),
        ("cost_ratio", C.c_float), ("empty_bonus", C.c_float),
    ]


class YrObjectNode(C.Structure):
    _fields_ = [("bmin", f3), ("left", C.c_int32), ("bmax", f3), ("right", C.c_int32)]


class YrKdTreeParams(C.Structure):
    _fields_ = [("max_depth", C.c_int32), ("max_leaf_size", C.c_int32), ("cost_ratio", C.c_float),
                ("empty_bonus", C.c_float), ("large_scene_penalty", C.c_int32), ("reserved", C.c_int32)]


class YrKdTreeMesh(C.Structure):
    _fields_ = [("verts", C.POINTER(C.c_float)), ("nverts", C.c_uint32),
                ("tris", C.POINTER(C.c_uint32)), ("ntris", C.c_uint32)]


class YrCameraDesc(C.Structure):
    _fields_ = [("pos", f3), ("look", f3), ("up", f3), ("resx", C.c_int32), ("resy", C.c_int32),
                ("aspect", C.c_float), ("focal", C.c_float)]


class YrShaderDesc(C.Structure):
    _fields_ = [
        ("color", f3), ("specular", f3), ("hard", C.c_float), ("tex_type", C.c_uint32),
        ("tex_color1", f3), ("tex_color2", f3), ("tex_H", C.c_float), ("tex_lacunarity", C.c_float),
        ("tex_octaves", C.c_float), ("tex_size", C.c_float), ("tex_intensity", C.c_float),
        ("mod_color", C.c_float), ("mod_size", f3), ("mod_ofs", f3), ("tex_noise", C.c_uint32),
        ("tex_depth", C.c_int32), ("tex_hard", C.c_uint32), ("tex_map", C.c_uint32),
        # record version 2
        ("mod_mode", C.c_uint32), ("tex_shape", C.c_uint32), ("tex_variant", C.c_uint32),
        ("tex_turbulence", C.c_float), ("tex_sharpness", C.c_float), ("tex_offset", C.c_float),
        ("tex_gain", C.c_float), ("tex_distort", C.c_float), ("tex_noise2", C.c_uint32),
        ("tex_weights", C.c_float * 4), ("tex_mk_exponent", C.c_float), ("tex_metric", C.c_uint32),
        # record version 3
        ("mod_specular", C.c_float), ("mod_hard", C.c_float),
    ]


class YrLightDesc(C.Structure):
    _fields_ = [
        ("type", C.c_uint32), ("color", f3), ("power", C.c_float), ("p", (C.c_float * 3) * 4),
        ("samples", C.c_int32), ("depth", C.c_int32), ("maxdist", C.c_float),
        ("cast_shadows", C.c_uint32), ("psamples", C.c_int32), ("threshold", C.c_float),
        ("reserved", C.c_uint32),
    ]


class YrRenderParams(C.Structure):
    _fields_ = [("self_bias", C.c_float), ("raydepth", C.c_int32), ("spp", C.c_uint32),
                ("aa_pixelwidth", C.c_float), ("seed", C.c_uint32), ("background", f3),
                ("flags", C.c_uint32), ("region", C.c_int32 * 4),
                # record version 3
                ("exposure", C.c_float), ("gamma", C.c_float)]


class YrObjectDesc(C.Structure):
    _fields_ = [("verts", C.POINTER(C.c_float)), ("nverts", C.c_uint32),
                ("tris", C.POINTER(C.c_uint32)), ("ntris", C.c_uint32),
                ("shader", C.c_uint32), ("cast_shadows", C.c_uint32),
                ("tri_shaders", C.POINTER(C.c_uint32)), ("tree", C.POINTER(YrKdTree)),
                ("smooth_angle", C.c_float), ("reserved", C.c_uint32),
                ("instance_matrix", C.POINTER(C.c_float)), ("instance_inverse", C.POINTER(C.c_float)),
                ("instance_of", C.c_uint32), ("reserved2", C.c_uint32),
                ("uvs", C.POINTER(C.c_float)), ("orco_matrix", C.POINTER(C.c_float))]


class YrSceneDesc(C.Structure):
    _fields_ = [("objects", C.POINTER(YrObjectDesc)), ("nobjects", C.c_uint32),
                ("shaders", C.POINTER(YrShaderDesc)), ("nshaders", C.c_uint32),
                ("lights", C.POINTER(YrLightDesc)), ("nlights", C.c_uint32),
                ("camera", YrCameraDesc), ("render", YrRenderParams)]


class YrSceneInfo(C.Structure):
    _fields_ = [("nobjects", C.c_uint32), ("ntriangles", C.c_uint32), ("nnodes", C.c_uint32),
                ("nprims", C.c_uint32), ("nlights", C.c_uint32), ("device_bytes", C.c_uint64),
                ("build_seconds", C.c_double)]


class YrRay(C.Structure):
    _fields_ = [("org", f3), ("tmax", C.c_float), ("dir", f3), ("flags", C.c_uint32)]


class YrHit(C.Structure):
    _fields_ = [("t", C.c_float), ("object", C.c_uint32), ("triangle", C.c_uint32),
                ("nodes_visited", C.c_uint32)]


class YrShadowRay(C.Structure):
    _fields_ = [("p", f3), ("object", C.c_uint32), ("l", f3), ("flags", C.c_uint32)]


YR_K_COUNT = 8
KERNEL_CLASSES = ["primary", "shade_camera", "shadow", "gather", "bounce", "shade_path", "other", "unused"]


class YrRenderStats(C.Structure):
    _fields_ = [("rays_primary", C.c_uint64), ("rays_shadow", C.c_uint64),
                ("rays_bounce", C.c_uint64), ("ms", C.c_double),
                ("want_kernel_stats", C.c_uint32), ("reserved", C.c_uint32),
                ("kernel_ms", C.c_double * YR_K_COUNT), ("kernel_launches", C.c_uint32 * YR_K_COUNT),
                ("kernel_rays", C.c_uint64 * YR_K_COUNT), ("kernel_nodes", C.c_uint64 * YR_K_COUNT),
                ("kernel_tests", C.c_uint64 * YR_K_COUNT)]


class YrBatchParams(C.Structure):
    _fields_ = [("block_size", C.c_int32), ("queue_tile", C.c_int32), ("use_graph", C.c_int32),
                ("stack_entries", C.c_int32), ("mode", C.c_int32), ("streams", C.c_int32)]


class YrBackwardDesc(C.Structure):
    _fields_ = [("target", C.c_void_p), ("image", C.c_void_p), ("loss_scale", C.c_float),
                ("reserved", C.c_uint32)]


# Every symbol include/yr.h declares, with its ctypes signature.
_P = C.c_void_p
# yr_pixels_fn: int (*)(void *user, uint32_t first, uint32_t count)
PIXELS_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_uint32, C.c_uint32)

SIGNATURES = {
    "yr_status_string": (C.c_char_p, [C.c_int]),
    "yr_version": (C.c_char_p, []),
    "yr_kdtree_build": (C.c_int, [C.POINTER(C.c_float), C.c_uint32, C.POINTER(C.c_uint32), C.c_uint32,
                                  C.POINTER(C.POINTER(YrKdTree))]),
    "yr_kdtree_free": (None, [C.POINTER(YrKdTree)]),
    "yr_kdtree_build_ex": (C.c_int, [C.POINTER(C.c_float), C.c_uint32, C.POINTER(C.c_uint32), C.c_uint32,
                                     C.POINTER(YrKdTreeParams), C.c_int, C.POINTER(C.POINTER(YrKdTree))]),
    "yr_kdtree_build_gpu": (C.c_int, [C.POINTER(YrKdTreeMesh), C.c_uint32, C.POINTER(YrKdTreeParams), C.c_int32,
                                      C.POINTER(C.POINTER(YrKdTree))]),
    "yr_object_tree_build": (C.c_int, [C.POINTER(C.c_float), C.c_uint32, C.POINTER(YrObjectNode),
                                       C.POINTER(C.c_uint32)]),
    "yr_instance_bound": (C.c_int, [C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "yr_scene_create": (C.c_int, [C.POINTER(YrSceneDesc), C.c_int, C.POINTER(_P)]),
    "yr_scene_destroy": (C.c_int, [_P]),
    "yr_scene_info_get": (C.c_int, [_P, C.POINTER(YrSceneInfo)]),
    "yr_scene_set_params": (C.c_int, [_P, C.POINTER(YrShaderDesc), C.POINTER(YrLightDesc)]),
    "yr_scene_set_camera_vectors": (C.c_int, [_P, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float),
                                              C.POINTER(C.c_float)]),
    "yr_trace_closest": (C.c_int, [_P, _P, C.c_uint32, _P, C.c_int, _P]),
    "yr_trace_shadow": (C.c_int, [_P, _P, C.c_uint32, _P, _P]),
    "yr_render": (C.c_int, [_P, _P, C.c_int, C.POINTER(YrRenderStats), _P]),
    "yr_render_progressive": (C.c_int, [_P, _P, C.c_uint32, _P, _P, C.POINTER(YrRenderStats), _P]),
    "yr_render_noalloc": (C.c_int, [_P, _P, C.POINTER(YrRenderStats), _P]),
    "yr_render_batch": (C.c_int, [C.POINTER(_P), C.c_uint32, C.POINTER(_P), C.POINTER(YrBatchParams),
                                  C.POINTER(YrRenderStats), _P]),
    "yr_param_count": (C.c_uint32, [_P]),
    "yr_params_get": (C.c_int, [_P, C.POINTER(C.c_float)]),
    "yr_params_set": (C.c_int, [_P, C.POINTER(C.c_float)]),
    "yr_backward": (C.c_int, [_P, C.POINTER(YrBackwardDesc), _P, C.POINTER(C.c_float), _P]),
    "yr_backward_batch": (C.c_int, [C.POINTER(_P), C.c_uint32, C.POINTER(YrBackwardDesc), C.POINTER(_P),
                                    C.POINTER(C.c_float), C.c_int32, _P]),
    "yr_image_encode": (C.c_int, [C.c_int32, C.POINTER(C.c_float), C.c_int32, C.c_int32, C.c_int32, _P, C.c_size_t,
                                  C.POINTER(C.c_size_t)]),
    "yr_image_write": (C.c_int, [C.c_char_p, C.c_int32, C.POINTER(C.c_float), C.c_int32, C.c_int32, C.c_int32]),
}

_lib = None


class YrError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}")


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load the native library (raises OSError when it has not been built,
    AttributeError when it lacks a symbol that include/yr.h declares)."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise OSError(f"{path} is missing: build it with `python -m yafray_b200.build`")
        lib = C.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def load_host_only(path: str = LIB_PATH) -> C.CDLL:
    """Load the library binding only the host entry points that are present
    (used while bringing up new entry points)."""
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        if hasattr(lib, name):
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
    return lib


def check(status: int, where: str) -> None:
    if status != YR_OK:
        raise YrError(status, where)
