"""yr_render_batch: every image of a batch equals yr_render's for that scene.

The batched launch runs the same stage code over tiles of whole pixels with
block-local queues; sample indices, QMC dimensions and the order of every
sum are those of the per-scene render, so the images are compared bit for
bit."""
import numpy as np
import pytest

from yafray_b200 import abi, api, scenes

pytestmark = pytest.mark.gpu


def _small_batch(count, seed=11):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        sc = scenes.config_batch_scene(rng, i, tri_lo=200, tri_hi=6000)
        res = int(rng.choice([16, 24, 40]))
        sc.camera.resx = sc.camera.resy = res
        sc.render.spp = int(rng.integers(1, 6))
        out.append(sc)
    return out


def _per_scene(torch, dss):
    imgs = []
    for d in dss:
        t = torch.zeros((d.sc.resy, d.sc.resx, 4), dtype=torch.float32, device="cuda")
        d.render_into(t.data_ptr())
        imgs.append(t)
    torch.cuda.synchronize()
    return [t.cpu().numpy() for t in imgs]


def _batched(torch, dss, **kw):
    outs = [torch.full((d.sc.resy, d.sc.resx, 4), -1.0, dtype=torch.float32, device="cuda") for d in dss]
    st, p = api.render_batch(dss, [t.data_ptr() for t in outs], **kw)
    torch.cuda.synchronize()
    return [t.cpu().numpy() for t in outs], st, p


@pytest.mark.parametrize("kw", [dict(), dict(use_graph=False), dict(block_size=128, queue_tile=64),
                                dict(block_size=256, queue_tile=1000, use_graph=True),
                                dict(mode=abi.YR_BATCH_TILES), dict(mode=abi.YR_BATCH_WAVES),
                                dict(mode=abi.YR_BATCH_WAVES, streams=3)])
def test_batch_matches_per_scene(cuda, kw):
    import torch
    dss = [api.DeviceScene(sc) for sc in _small_batch(10)]
    ref = _per_scene(torch, dss)
    for rep in range(2):  # second call replays the cached launch / graph
        got, st, p = _batched(torch, dss, **kw)
        for a, b in zip(got, ref):
            assert np.array_equal(a, b)
        assert p.mode in (abi.YR_BATCH_TILES, abi.YR_BATCH_WAVES)
        if "mode" in kw:
            assert p.mode == kw["mode"]
        if p.mode == abi.YR_BATCH_TILES:
            assert p.block_size in (32 * k for k in range(1, 33)) and p.queue_tile > 0
        else:
            assert p.streams == kw.get("streams", p.streams) and p.streams >= 1
        assert p.stack_entries >= 32
    tot = sum(d.sc.resx * d.sc.resy * d.sc.render.spp for d in dss)
    assert st.rays_primary == tot
    assert st.rays_shadow > 0 and st.rays_bounce > 0 and st.ms > 0


def test_batch_sees_param_changes(cuda):
    """A scene's render parameters changed between batched calls are used."""
    import torch
    scs = _small_batch(3, seed=5)
    dss = [api.DeviceScene(sc) for sc in scs]
    _batched(torch, dss)
    scs[1].lights[0].power *= 2.0
    scs[2].shaders[0].color[0] = 0.1
    dss[1].set_params(lights=scs[1].lights)
    dss[2].set_params(shaders=scs[2].shaders)
    got, _, _ = _batched(torch, dss)
    ref = _per_scene(torch, dss)
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)


def test_batch_rejects_bad_args(cuda):
    import torch
    dss = [api.DeviceScene(sc) for sc in _small_batch(2)]
    outs = [torch.zeros((d.sc.resy, d.sc.resx, 4), device="cuda") for d in dss]
    with pytest.raises(abi.YrError):
        api.render_batch(dss, [t.data_ptr() for t in outs], block_size=100, queue_tile=64)
    with pytest.raises(abi.YrError):
        api.render_batch(dss, [outs[0].data_ptr(), 0])
