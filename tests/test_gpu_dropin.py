"""The drop-in, end to end: a scene built from the reference's own objects
(meshObject_t, genericShader_t, pointLight_t, camera_t - the harness's
scene construction) and rendered by cudascene_t::render, the scene class a
YafRay maintainer adds (oracle/cudascene.{h,cc}, compiled against the
reference's headers and linked with libyafray_b200.so), against the stock
scene_t::render of the same objects.  Config 1 (the point-light sphere) is
deterministic in the reference, so the two images must agree pixel for
pixel within 1e-4 (alpha identical); with AA every pixel is resampled in
one pass (AA_threshold 0) and the positions are the reference's."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import yrtest as T
from yafray_b200 import scenes

pytestmark = pytest.mark.gpu

CUDASCENE = os.path.join(T.ROOT, "oracle", "_ref", "yr_ref_cudascene")
RTOL = 1e-4


def _run(cmd, sc, *extra):
    with tempfile.TemporaryDirectory() as d:
        sp, op = os.path.join(d, "s.yrs"), os.path.join(d, "o.bin")
        scenes.write_yrs(sc, sp)
        r = subprocess.run([cmd[0], cmd[1], sp, op] + [str(a) for a in extra], capture_output=True, text=True,
                           timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        img = np.fromfile(op, np.float32).reshape(sc.resy, sc.resx, 4)
    import json
    return img, json.loads(r.stdout.strip().splitlines()[-1])


def _need():
    if not (os.path.exists(CUDASCENE) and T.has_harness()):
        pytest.skip("reference harness / cudascene build not present (make -C oracle all)")


@pytest.mark.parametrize("spp", [1, 5])
def test_cudascene_matches_stock_render(cuda, spp):
    _need()
    sc = scenes.config_small()
    sc.render.spp = spp
    dev, st = _run([CUDASCENE, "cudarender"], sc)
    assert st["status"] == 0
    ref, _ = _run([T.HARNESS, "render"], sc, 1)   # scene_t::render, one thread
    assert np.array_equal(dev[..., 3], ref[..., 3]), "pixel coverage differs"
    rel = np.abs(dev[..., :3] - ref[..., :3]) / np.maximum(np.abs(ref[..., :3]), 1e-3)
    assert rel.max() <= RTOL, f"max rel {rel.max()}"
    assert (ref[..., 3] > 0).mean() > 0.5 and ref[..., :3].max() > 0.01


def test_cudascene_region(cuda):
    """scene_t::setRegion: only the region's pixels are rendered, the rest
    are written as 0, as scene_t::render does."""
    _need()
    sc = scenes.config_small(160, 120)
    crop = (30, 110, 20, 90)
    dev, st = _run([CUDASCENE, "cudarender"], sc, *crop)
    assert st["status"] == 0
    ref, _ = _run([T.HARNESS, "render"], sc, 1, *crop)
    assert np.array_equal(dev[..., 3], ref[..., 3])
    rel = np.abs(dev[..., :3] - ref[..., :3]) / np.maximum(np.abs(ref[..., :3]), 1e-3)
    assert rel.max() <= RTOL
    out = np.ones(dev.shape[:2], bool)
    out[crop[2]:crop[3], crop[0]:crop[1]] = False
    assert not dev[out].any()


def test_cudascene_refuses_what_it_cannot_take(cuda):
    """A scene with an area light and path GI is refused with
    YR_ERR_UNSUPPORTED before any device work; the output stays untouched
    (no CPU fallback)."""
    _need()
    sc = scenes.config_large(seed=2, resx=32, resy=24, spp=1, grid=2)
    dev, st = _run([CUDASCENE, "cudarender"], sc)
    assert st["status"] == 8  # YR_ERR_UNSUPPORTED
    assert not dev.any()


def test_cudascene_output_can_stop_the_render(cuda):
    """An output whose putPixel returns false after 5000 pixels stops the
    render, as it stops scene_t::render: YR_ERR_CANCELLED, the pixels it
    took are the full render's, no more are written."""
    _need()
    sc = scenes.config_small(160, 120)
    full, _ = _run([CUDASCENE, "cudarender"], sc)
    part, st = _run([CUDASCENE, "cudarender"], sc, 0, 160, 0, 120, 5000)
    assert st["status"] == 7 and st["pixels"] == 5000  # YR_ERR_CANCELLED
    flat, ref = part.reshape(-1, 4), full.reshape(-1, 4)
    assert np.array_equal(flat[:5000], ref[:5000])
    assert not flat[5000:].any()
