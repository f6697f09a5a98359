"""The host API as a drop-in: the scene handed to a yafrayInterface_t call
by call, as the Blender exporter and the XML loader's front ends do
(addShader / addTexture with their parameter maps, addObject_trimesh,
transformPush + addObject_reference, addLight, addCamera, addBackground,
render(params, output)), once to the reference's own interfaceImpl_t (the
CPU renderer) and once to cudaInterface_t (oracle/cudainterface.{h,cc}: the
same class with its renders through cudascene_t and the library; the
harness's iface command).

Point-light scenes are deterministic in the reference, so the two images
must agree within 1e-4 per pixel (alpha identical): flat and smoothed
meshes, per-triangle shaders, procedural textures under every texture
coordinate kind ("orco" here means backOrco * P, since the interface makes
every mesh through meshObject_t::transform), the specular / hardness
channels, references placed by transformPush, AA.  With area, hemi and
path lights the reference draws its own sample sequences, so there the
captured scene must render exactly as the same scene given to the library
directly."""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

import yrtest as T
from yafray_b200 import abi, api, scenes

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden  # noqa: E402

pytestmark = pytest.mark.gpu

CUDASCENE = os.path.join(T.ROOT, "oracle", "_ref", "yr_ref_cudascene")
RTOL = 1e-4


def _iface(sc, arm, *extra):
    with tempfile.TemporaryDirectory() as d:
        sp, op = os.path.join(d, "s.yrs"), os.path.join(d, "o.bin")
        scenes.write_yrs(sc, sp)
        r = subprocess.run([CUDASCENE, "iface", sp, op, arm] + list(extra), capture_output=True, text=True,
                           timeout=900)
        assert r.returncode == 0, r.stderr[-2000:]
        img = np.fromfile(op, np.float32).reshape(sc.resy, sc.resx, 4)
    return img, json.loads(r.stdout.strip().splitlines()[-1])


def _need():
    if not os.path.exists(CUDASCENE):
        pytest.skip("cudascene build not present (make -C oracle all)")


def _fbm_only(sc):
    # through addTexture a musgrave texture is always fBm (its "type"
    # parameter is the texture type), so the scene asks for that
    for s in sc.shaders:
        if s.tex_type in (abi.YR_TEX_MUSGRAVE_MULTIFRACTAL, abi.YR_TEX_MUSGRAVE_HETEROTERRAIN,
                          abi.YR_TEX_MUSGRAVE_HYBRIDMF, abi.YR_TEX_MUSGRAVE_RIDGEDMF):
            s.tex_type = abi.YR_TEX_MUSGRAVE_FBM
    return sc


def _small_aa():
    sc = scenes.config_small()
    sc.render.spp = 5
    return sc


SCENES = {
    "config1": scenes.config_small,
    "config1_aa": _small_aa,
    "smooth": make_golden.smooth_scene,
    "textures": lambda: _fbm_only(make_golden.texture_scene()),
    "texco_orco_normal": make_golden.texco_scene,
    "texco_window_reflect": make_golden.texco_view_scene,
    "texco_uv": make_golden.texco_uv_scene,
    "specular_hardness": make_golden.specmod_scene,
    "references": make_golden.instance_scene,
}


@pytest.mark.parametrize("name", sorted(SCENES))
def test_interface_render_matches_reference(cuda, name):
    _need()
    sc = SCENES[name]()
    dev, st = _iface(sc, "cuda")
    assert st["status"] == 0
    ref, _ = _iface(sc, "ref")
    assert np.array_equal(dev[..., 3], ref[..., 3]), "pixel coverage differs"
    rel = np.abs(dev[..., :3] - ref[..., :3]) / np.maximum(np.abs(ref[..., :3]), 1e-3)
    assert rel.max() <= RTOL, f"max rel {rel.max()}"
    assert (ref[..., 3] > 0).mean() > 0.3 and ref[..., :3].max() > 0.01


def test_interface_gi_scene_is_captured_exactly(cuda):
    """Area lights, a path light with adaptive rounds, a hemi light, a
    constant background, textures and a smoothed mesh: the scene captured
    from the calls renders bit for bit as the scene given to the library
    directly."""
    _need()
    sc = scenes.config_large(seed=4, resx=64, resy=48, spp=2, grid=2)
    sc.shaders[0] = scenes.texture_shader((0.6, 0.5, 0.4), "clouds", (0.1, 0.2, 0.3), (0.9, 0.8, 0.6),
                                          mod_color=0.8, depth=3, size=1.5)
    sc.meshes[1].smooth_angle = 180.0
    sc.lights.append(scenes.hemi_light(samples=4, power=0.3, maxdist=3.0))
    for l in sc.lights:
        if l.type == abi.YR_LIGHT_PATH:
            l.threshold = 0.05
    sc.render.background[:] = [0.05, 0.1, 0.2]
    sc.render.seed = 0  # the QMC rotation seed is the library's; a captured scene takes 0
    dev, st = _iface(sc, "cuda")
    assert st["status"] == 0
    # an external render always tone-maps (interface_impl.cc:812-814)
    sc.render.flags |= abi.YR_RENDER_TONEMAP
    direct = api.DeviceScene(sc).render()
    assert np.array_equal(dev, direct)
    assert dev[..., :3].max() > 0.01


def test_interface_refuses_the_irradiance_cache(cuda):
    """A path light with its irradiance cache on is refused with
    YR_ERR_UNSUPPORTED; nothing is rendered (no CPU fallback)."""
    _need()
    sc = scenes.config_large(seed=2, resx=32, resy=24, spp=1, grid=2)
    dev, st = _iface(sc, "cuda", "pathcache")
    assert st["status"] == 8  # YR_ERR_UNSUPPORTED
    assert not dev.any()
