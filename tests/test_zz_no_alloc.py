"""yr_render_noalloc, the render entry point for hosts that cannot allocate
GPU memory while they render - a renderer plugin inside an application that
owns all device memory through its own allocator and forbids cudaMalloc to
its plugins.  Its scratch is a fixed block inside the library.  Through the
C ABI, two calls in a row must give the allocating yr_render's image bit for
bit (both run the same kernels in the same summation order), and a call must
leave the device's free memory unchanged.

Collected last on purpose (file name): if it fails, a run that stops at the
first failure has already run every other test."""
import ctypes as C

import numpy as np
import pytest

from yafray_b200 import abi, api, scenes

pytestmark = pytest.mark.gpu


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
        assert np.array_equal(img.view(np.uint32), ref.view(np.uint32))
        assert st.rays_primary == st_ref.rays_primary
        assert st.rays_shadow == st_ref.rays_shadow and st.rays_bounce == st_ref.rays_bounce
        assert st.ms == 0.0  # no CUDA events either


def test_noalloc_allocates_nothing(cuda):
    """After a first call (which looks the block's address up), further
    calls change neither the device's free memory nor the image."""
    sc = scenes.config_large(seed=5, resx=128, resy=96, spp=4, grid=2)
    ds = api.DeviceScene(sc)
    out = cuda.zeros((sc.resy, sc.resx, 4), dtype=cuda.float32, device="cuda")
    st = abi.YrRenderStats()
    abi.check(ds.lib.yr_render_noalloc(ds.handle, C.c_void_p(out.data_ptr()), C.byref(st), C.c_void_p(0)), "noalloc")
    cuda.cuda.synchronize()
    first = out.cpu().numpy().copy()
    free0, _ = cuda.cuda.mem_get_info()
    for _ in range(3):
        abi.check(ds.lib.yr_render_noalloc(ds.handle, C.c_void_p(out.data_ptr()), C.byref(st), C.c_void_p(0)),
                  "noalloc")
    cuda.cuda.synchronize()
    free1, _ = cuda.cuda.mem_get_info()
    assert free1 == free0
    assert np.array_equal(out.cpu().numpy().view(np.uint32), first.view(np.uint32))


def test_noalloc_rejects_oversized_pixels(cuda):
    """One pixel's samples must fit in the block: otherwise a clear error."""
    sc = scenes.config_large(seed=5, resx=32, resy=16, spp=65536, grid=2)
    ds = api.DeviceScene(sc)
    out = cuda.zeros((sc.resy, sc.resx, 4), dtype=cuda.float32, device="cuda")
    st = abi.YrRenderStats()
    rc = ds.lib.yr_render_noalloc(ds.handle, C.c_void_p(out.data_ptr()), C.byref(st), C.c_void_p(0))
    assert rc == 11  # YR_ERR_TOO_LARGE
