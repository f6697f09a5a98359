"""The C ABI library: loads on a CPU-only machine, exports every symbol
include/yr.h declares, and rejects bad arguments without a device."""
import ctypes as C
import os
import re

import numpy as np

import yrtest as T
from yafray_b200 import abi, scenes


def declared_symbols():
    hdr = open(os.path.join(T.ROOT, "include", "yr.h")).read()
    return sorted(set(re.findall(r"YR_API\s+[\w\s\*]+?\b(yr_\w+)\s*\(", hdr)))


def test_every_declared_symbol_is_exported():
    lib = C.CDLL(abi.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 17
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(abi.SIGNATURES), set(names) ^ set(abi.SIGNATURES)


def test_status_strings():
    lib = abi.load()
    for code in abi.STATUS_NAMES:
        assert lib.yr_status_string(code)
    assert b"sm_100a" in lib.yr_version()


def test_kdtree_build_rejects_bad_input():
    lib = abi.load()
    p = C.POINTER(abi.YrKdTree)()
    v = np.zeros((3, 3), np.float32)
    t = np.array([[0, 1, 5]], np.uint32)  # vertex index out of range
    st = lib.yr_kdtree_build(v.ctypes.data_as(C.POINTER(C.c_float)), 3, t.ctypes.data_as(C.POINTER(C.c_uint32)), 1,
                             C.byref(p))
    assert st == 1  # YR_ERR_INVALID_ARG
    assert lib.yr_kdtree_build(None, 0, None, 0, C.byref(p)) == 9  # YR_ERR_EMPTY_SCENE


def test_scene_create_without_device_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        return
    lib = abi.load()
    desc = abi.YrSceneDesc()
    h = C.c_void_p()
    assert lib.yr_scene_create(C.byref(desc), 0, C.byref(h)) in (9, 10)  # empty scene / no device
    assert not h.value


def test_scene_file_roundtrip(tmp_path):
    sc = scenes.config_diff(res=32, spp=2, groups=4, nlights=2)
    p = str(tmp_path / "s.yrs")
    scenes.write_yrs(sc, p)
    back = scenes.read_yrs(p)
    assert len(back.meshes) == len(sc.meshes)
    assert bytes(back.camera) == bytes(sc.camera) and bytes(back.render) == bytes(sc.render)
    for a, b in zip(sc.shaders, back.shaders):
        assert bytes(a) == bytes(b)
    for a, b in zip(sc.meshes, back.meshes):
        assert np.array_equal(a.verts, b.verts) and np.array_equal(a.tris, b.tris)
    assert np.array_equal(back.meshes[0].tri_shaders, sc.meshes[0].tri_shaders)


def test_uv_sphere_counts():
    v, t = scenes.uv_sphere()
    assert v.shape == (8066, 3) and t.shape == (16128, 3)
    sc = scenes.config_large()
    assert sc.ntris == 256 * 16128 + 2 and len(sc.meshes) == 257
