"""yr_render_progressive: the frame delivered wave by wave to a callback,
the library's form of YafRay's colorOutput_t::putPixel per finished block,
and the render stopped when the callback says so (putPixel returning false
stops scene_t::render, renderblock.cc:8-20, threadedscene.cc:186-197)."""
import numpy as np
import pytest

from yafray_b200 import api, scenes

pytestmark = pytest.mark.gpu


def test_progressive_equals_render(cuda):
    sc = scenes.config_large(seed=2, resx=96, resy=64, spp=3, grid=2)
    ds = api.DeviceScene(sc)
    ref = ds.render()
    ranges = []
    img, rc = ds.render_progressive(lambda first, count: ranges.append((first, count)), wave_pixels=1000)
    assert rc == 0
    assert np.array_equal(img.view(np.uint32), ref.view(np.uint32))
    # consecutive ranges covering every pixel once, in order
    assert len(ranges) == (96 * 64 + 999) // 1000
    assert ranges[0][0] == 0 and all(a[0] + a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
    assert sum(c for _, c in ranges) == 96 * 64
    assert ds.last_stats.rays_primary == 96 * 64 * 3


def test_progressive_cancel(cuda):
    """A callback that stops after the second wave: YR_ERR_CANCELLED, the
    delivered pixels are the full render's, the rest keep the buffer's
    content, and only the delivered waves' camera rays were traced."""
    sc = scenes.config_small(160, 120)
    sc.render.spp = 2
    ds = api.DeviceScene(sc)
    ref = ds.render()
    buf = np.full((120, 160, 4), -7.0, np.float32)
    got = []

    def stop_after_two(first, count):
        got.append((first, count))
        return len(got) < 2

    img, rc = ds.render_progressive(stop_after_two, wave_pixels=2500, img=buf)
    assert rc == 7  # YR_ERR_CANCELLED
    n = sum(c for _, c in got)
    assert n == 5000 and len(got) == 2
    flat, rflat = img.reshape(-1, 4), ref.reshape(-1, 4)
    assert np.array_equal(flat[:n], rflat[:n])
    assert (flat[n:] == -7.0).all()
    assert ds.last_stats.rays_primary == n * 2


def test_progressive_region(cuda):
    """With a render region, the delivered pixels are the region's in its
    row-major order and everything outside it is 0."""
    sc = scenes.config_small(128, 96)
    sc.render.region[:] = [20, 100, 10, 70]
    ds = api.DeviceScene(sc)
    ref = ds.render()
    seen = np.zeros(80 * 60, bool)

    def mark(first, count):
        seen[first:first + count] = True

    img, rc = ds.render_progressive(mark, wave_pixels=700, img=np.full((96, 128, 4), 5.0, np.float32))
    assert rc == 0 and seen.all()
    assert np.array_equal(img.view(np.uint32), ref.view(np.uint32))
    out = np.ones((96, 128), bool)
    out[10:70, 20:100] = False
    assert not img[out].any()
