"""Failure paths end in a status code, never in a device fault: a corrupt
prebuilt tree (a link out of range or back up the tree, a bad leaf) is
rejected on the host when the scene is created, rays with NaN
components miss (infinite ones are answered without an error), an empty
scene is refused, and the library keeps working after each error."""
import ctypes as C

import numpy as np
import pytest

from yafray_b200 import abi, api, scenes

pytestmark = pytest.mark.gpu


def _tree(mesh):
    lib = abi.load()
    v = np.ascontiguousarray(mesh.verts, np.float32)
    t = np.ascontiguousarray(mesh.tris, np.uint32)
    p = C.POINTER(abi.YrKdTree)()
    abi.check(lib.yr_kdtree_build(v.ctypes.data_as(C.POINTER(C.c_float)), v.shape[0],
                                  t.ctypes.data_as(C.POINTER(C.c_uint32)), t.shape[0], C.byref(p)), "build")
    return p


@pytest.mark.parametrize("what", ["child", "cycle", "leaf_triangle", "prim_range"])
def test_corrupt_prebuilt_tree_is_rejected(cuda, what):
    sc = scenes.config_small(32, 24)
    lib = abi.load()
    tree = _tree(sc.meshes[0])
    nodes = tree.contents.nodes
    n = tree.contents.nnodes
    interior = next(i for i in range(n) if nodes[i].flags & 3 != 3)
    single = next(i for i in range(n) if nodes[i].flags & 3 == 3 and nodes[i].flags >> 2 == 1)
    multi = next((i for i in range(n) if nodes[i].flags & 3 == 3 and nodes[i].flags >> 2 > 1), None)
    if what == "child":
        nodes[interior].flags = (nodes[interior].flags & 3) | ((n + 7) << 2)
    elif what == "cycle":  # right child pointing back at the node: a walk that would never end
        nodes[interior].flags = (nodes[interior].flags & 3) | (interior << 2)
    elif what == "leaf_triangle":
        nodes[single].word = sc.meshes[0].tris.shape[0] + 3
    else:
        if multi is None:
            pytest.skip("tree has no multi-triangle leaf")
        nodes[multi].word = tree.contents.nprims
    with pytest.raises(abi.YrError) as e:
        api.DeviceScene(sc, trees=[tree, None])
    assert e.value.status == 6  # YR_ERR_BAD_TREE
    lib.yr_kdtree_free(tree)
    # the device is fine: the same scene without the bad tree renders
    img = api.DeviceScene(sc).render()
    assert np.isfinite(img).all() and img[..., 3].sum() > 0


def test_prebuilt_tree_gives_the_same_image(cuda):
    sc = scenes.config_small(40, 30)
    tree = _tree(sc.meshes[0])
    a = api.DeviceScene(sc, trees=[tree, None]).render()
    b = api.DeviceScene(sc).render()
    abi.load().yr_kdtree_free(tree)
    assert np.array_equal(a, b)


def test_nan_and_infinite_rays_miss(cuda):
    import torch
    sc = scenes.config_small(32, 24)
    ds = api.DeviceScene(sc)
    inf, nan = np.inf, np.nan
    rays = np.array([[0, 1, 5, 0, nan, nan, nan, 0],
                     [0, 1, 5, 0, 0, 0, -1, 0],        # a normal ray for reference
                     [nan, 1, 5, 0, 0, 0, -1, 0],
                     [0, 1, 5, 0, inf, 0, -1, 0],
                     [inf, inf, inf, 0, 0, 0, -1, 0]], np.float32)
    d_rays = torch.from_numpy(rays).cuda()
    hits = torch.zeros((len(rays), 4), dtype=torch.int32, device="cuda")
    api.trace_closest(ds, d_rays.data_ptr(), len(rays), hits.data_ptr())
    torch.cuda.synchronize()
    h = hits.cpu().numpy().view(np.uint32)
    assert h[1, 1] != 0xFFFFFFFF  # the normal ray hits the sphere
    assert (h[[0, 2], 1] == 0xFFFFFFFF).all()  # NaN: every comparison fails, nothing is hit
    # infinite components: answered without an error (what they hit is not specified)


def test_empty_scene_is_refused(cuda):
    lib = abi.load()
    desc = abi.YrSceneDesc()
    desc.camera = scenes.camera((0, 1, 5), (0, 0, 0), (0, 2, 5), 8, 8)
    desc.render = scenes.render_params()
    h = C.c_void_p()
    assert lib.yr_scene_create(C.byref(desc), 0, C.byref(h)) == 9  # YR_ERR_EMPTY_SCENE
    assert not h.value
    assert api.DeviceScene(scenes.config_small(8, 8)).render().shape == (8, 8, 4)
