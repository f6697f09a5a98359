"""The GPU kd build (yr_kdtree_build_gpu) against the reference's trees and
the host build: node for node, leaf lists in the same order."""
import ctypes as C
import os

import numpy as np
import pytest

import yrtest as T
from yafray_b200 import abi, api, scenes

pytestmark = pytest.mark.gpu

G = T.GOLDEN


def _mg():
    import importlib.util
    spec = importlib.util.spec_from_file_location("mg", os.path.join(G, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    return mg


def _same(a, b, what):
    assert np.array_equal(a["nodes"], b["nodes"]), what
    assert np.array_equal(a["prims"], b["prims"]), what
    assert np.array_equal(a["tb"].view(np.uint32), b["tb"].view(np.uint32)), what
    assert (a["max_depth"], a["max_leaf"], a["cost_ratio"]) == (b["max_depth"], b["max_leaf"], b["cost_ratio"]), what


def test_gpu_kdtree_matches_reference():
    """kdTree_t's trees (kdtree.cc:57-582) from the reference harness."""
    mg = _mg()
    g = np.load(os.path.join(G, "trees.npz"))
    for name, sc in (("sphere16", mg.small_sphere_scene()), ("random3000", mg.random_mesh_scene(3000, 11))):
        for i, t in enumerate(T.gpu_trees(sc.meshes)):
            assert np.array_equal(t["nodes"], g[f"{name}_{i}_nodes"]), (name, i)
            assert np.array_equal(t["prims"], g[f"{name}_{i}_prims"]), (name, i)
            assert np.array_equal(t["tb"].view(np.uint32), g[f"{name}_{i}_tb"].view(np.uint32)), (name, i)
    g = np.load(os.path.join(G, "trees_ties.npz"))
    for i, t in enumerate(T.gpu_trees(mg.tie_scene().meshes)):
        assert np.array_equal(t["nodes"], g[f"ties_{i}_nodes"]), i
        assert np.array_equal(t["prims"], g[f"ties_{i}_prims"]), i


def _soup(rng, n, spread=5.0, size=0.3):
    c = rng.uniform(-spread, spread, (n, 1, 3))
    v = (c + size * rng.uniform(-1, 1, (n, 3, 3))).reshape(-1, 3).astype(np.float32)
    return scenes.Mesh(v, np.arange(3 * n, dtype=np.uint32).reshape(n, 3), 0)


def _varied_meshes():
    rng = np.random.default_rng(5)
    mg = _mg()
    ms = [_soup(rng, n) for n in (1, 2, 16, 31, 32, 33, 100, 128, 129, 130, 257, 1000, 5000)]
    bv, bt = mg.box_soup(rng, 900)  # flats and shared planes above 128 triangles per node
    ms.append(scenes.Mesh(bv, bt, 0))
    tv, tt = mg.terrace(70, 60, 9)
    ms.append(scenes.Mesh(tv, tt, 0))
    # quantised coordinates: many equal bin values and edges
    q = _soup(rng, 4000)
    q.verts = np.round(q.verts * 2.0).astype(np.float32) / 2.0
    ms.append(q)
    # thin slabs: flat bounds on one axis
    s = _soup(rng, 3000)
    s.verts[:, 1] = np.round(s.verts[:, 1])
    ms.append(s)
    sv, st = scenes.uv_sphere((0.0, 0.0, 0.0), 2.0, rings=64, segments=128)
    ms.append(scenes.Mesh(sv, st, 0))
    pv, pt = scenes.ground_plane(10.0, 0.0)
    ms.append(scenes.Mesh(pv, pt, 0))
    return ms


def test_gpu_kdtree_matches_host_build():
    """Many meshes in one GPU build, each equal to its own host build."""
    ms = _varied_meshes()
    for i, (a, m) in enumerate(zip(T.gpu_trees(ms), ms)):
        _same(a, T.product_tree(m), i)


@pytest.mark.parametrize("params", [(4, -1, 1.2, 0.4, 1), (-1, 6, 1.2, 0.4, 1), (-1, -1, 0.3, 0.9, 0),
                                    (12, 2, 3.0, 0.0, 1)])
def test_gpu_kdtree_parameters(params):
    """Depth / leaf limits (leaves above 128 triangles), cost ratio, empty
    bonus and the large-scene penalty as kdTree_t's constructor takes them."""
    p = abi.YrKdTreeParams(*params, 0)
    ms = _varied_meshes()[10:17]
    for i, (a, m) in enumerate(zip(T.gpu_trees(ms, p), ms)):
        _same(a, T.product_tree(m, p), i)


def test_gpu_kdtree_large_mesh():
    """A 262k-triangle sphere plus a 40k-triangle soup: many binned levels."""
    rng = np.random.default_rng(8)
    sv, st = scenes.uv_sphere((0.0, 0.0, 0.0), 1.0, rings=256, segments=512)
    ms = [scenes.Mesh(sv, st, 0), _soup(rng, 40000, 20.0, 0.5)]
    for i, (a, m) in enumerate(zip(T.gpu_trees(ms), ms)):
        _same(a, T.product_tree(m, nthreads=8), i)


def test_gpu_kdtree_degenerate_and_errors():
    """All-degenerate meshes (zero diagonal) and the argument checks."""
    v = np.zeros((3, 3), np.float32)
    m = scenes.Mesh(v, np.array([[0, 1, 2]] * 200, np.uint32), 0)
    w = np.full((3, 3), -0.0, np.float32)
    m2 = scenes.Mesh(w, np.array([[0, 1, 2]] * 5, np.uint32), 0)
    for i, (a, mm) in enumerate(zip(T.gpu_trees([m, m2]), [m, m2])):
        _same(a, T.product_tree(mm), i)
    lib = abi.load()
    outs = (C.POINTER(abi.YrKdTree) * 1)()
    arr = (abi.YrKdTreeMesh * 1)()
    arr[0].verts = v.ctypes.data_as(C.POINTER(C.c_float))
    arr[0].nverts = 3
    bad = np.array([[0, 1, 3]], np.uint32)
    arr[0].tris = bad.ctypes.data_as(C.POINTER(C.c_uint32))
    arr[0].ntris = 1
    assert lib.yr_kdtree_build_gpu(arr, 1, None, 0, outs) == 1  # index out of range
    arr[0].ntris = 0
    assert lib.yr_kdtree_build_gpu(arr, 1, None, 0, outs) == 9  # empty mesh
    assert lib.yr_kdtree_build_gpu(arr, 0, None, 0, outs) == 1


def test_scene_gpu_kd_build_renders_identically():
    """YR_RENDER_GPU_KD_BUILD: same trees, so the same image bit for bit."""
    mg = _mg()
    sc = mg.small_sphere_scene()
    img0 = api.DeviceScene(sc).render()
    sc.render.flags |= abi.YR_RENDER_GPU_KD_BUILD
    ds = api.DeviceScene(sc)
    img1 = ds.render()
    assert np.array_equal(img0.view(np.uint32), img1.view(np.uint32))
    inf = ds.info()
    assert inf.nnodes > 0


def test_gpu_kdtree_rejects_non_finite():
    lib = abi.load()
    v = np.array([[0, 0, 0], [1, 0, 0], [0, np.nan, 0]], np.float32)
    t = np.array([[0, 1, 2]], np.uint32)
    arr = (abi.YrKdTreeMesh * 1)()
    arr[0].verts = v.ctypes.data_as(C.POINTER(C.c_float))
    arr[0].nverts = 3
    arr[0].tris = t.ctypes.data_as(C.POINTER(C.c_uint32))
    arr[0].ntris = 1
    outs = (C.POINTER(abi.YrKdTree) * 1)()
    assert lib.yr_kdtree_build_gpu(arr, 1, None, 0, outs) == 1


def test_scene_gpu_kd_build_with_instances_and_many_objects():
    """Instances share their original's GPU-built tree; a scene of many
    meshes of every size class renders as with host-built trees."""
    rng = np.random.default_rng(12)
    sc = scenes.config_small(96, 72)
    sv, st = scenes.uv_sphere((0.0, 0.0, 0.0), 0.6, rings=24, segments=48)
    pv, pt = scenes.ground_plane(20.0, -1.0)
    sc.meshes = [scenes.Mesh(sv, st, 0), scenes.Mesh(pv, pt, 0),
                 scenes.instance(0, scenes.transform(translate=(1.2, 0.1, 0.3), rotate_deg=(0, 30, 0)))]
    for n in (1, 7, 40, 129, 600):
        m = _soup(rng, n, 1.5, 0.2)
        m.verts = (m.verts + np.array([0.0, 0.5, -2.0], np.float32)).astype(np.float32)
        sc.meshes.append(m)
    img0 = api.DeviceScene(sc).render()
    sc.render.flags |= abi.YR_RENDER_GPU_KD_BUILD
    img1 = api.DeviceScene(sc).render()
    assert np.array_equal(img0.view(np.uint32), img1.view(np.uint32))
