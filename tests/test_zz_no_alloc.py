"""yr_render_noalloc, the render entry point for hosts that cannot allocate
GPU memory while they render (the library's own allocation-free path; its
scratch is a fixed block inside the library).  Through the C ABI, two calls
in a row must give the image of the allocating yr_render.

Collected last on purpose (file name): if it fails, a run that stops at the
first failure has already run every other test."""
import ctypes as C

import numpy as np
import pytest

from yafray_b200 import abi, api, scenes

pytestmark = pytest.mark.gpu

RTOL = 1e-4  # the tolerance of the render parity tests


def _render(torch, ds, fn):
    out = torch.zeros((ds.sc.resy, ds.sc.resx, 4), dtype=torch.float32, device="cuda")
    st = abi.YrRenderStats()
    if fn == "noalloc":
        rc = ds.lib.yr_render_noalloc(ds.handle, C.c_void_p(out.data_ptr()), C.byref(st), C.c_void_p(0))
    else:
        rc = ds.lib.yr_render(ds.handle, C.c_void_p(out.data_ptr()), 0, C.byref(st), C.c_void_p(0))
    abi.check(rc, fn)
    torch.cuda.synchronize()
    return out.cpu().numpy(), st


def _close(a, b):
    rel = np.abs(a - b) / np.maximum(np.abs(b), 1e-3)
    return float(rel.max())


@pytest.mark.parametrize("which", ["point", "gi"])
def test_noalloc_matches_render(cuda, which):
    if which == "point":
        sc = scenes.config_small(160, 120)
        sc.render.spp = 3
    else:  # area lights + path GI: scratch larger than one block -> several passes
        sc = scenes.config_large(seed=5, resx=256, resy=160, spp=8, grid=3)
    ds = api.DeviceScene(sc)
    ref, st_ref = _render(cuda, ds, "render")
    for _ in range(2):  # two calls in a row share the block
        img, st = _render(cuda, ds, "noalloc")
        assert _close(img, ref) <= RTOL
        assert st.rays_primary == st_ref.rays_primary
        assert st.rays_shadow == st_ref.rays_shadow and st.rays_bounce == st_ref.rays_bounce


def test_noalloc_rejects_oversized_pixels(cuda):
    """One pixel's samples must fit in the block: otherwise a clear error."""
    sc = scenes.config_large(seed=5, resx=32, resy=16, spp=65536, grid=2)
    ds = api.DeviceScene(sc)
    out = cuda.zeros((sc.resy, sc.resx, 4), dtype=cuda.float32, device="cuda")
    st = abi.YrRenderStats()
    rc = ds.lib.yr_render_noalloc(ds.handle, C.c_void_p(out.data_ptr()), C.byref(st), C.c_void_p(0))
    assert rc == 11  # YR_ERR_TOO_LARGE
