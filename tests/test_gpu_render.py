"""yr_render against the oracle on the same scenes and QMC indices.

Tolerances (from the specification of this path): radiance within 1e-4
relative for every pixel; pixel coverage (alpha) identical.  A pixel beyond
1e-4 is accepted only when an energy cut-off of the estimators explains it
(a path stopping below 0.05, pathlight.cc:315 / 398; a hemi point skipped,
hemilight.cc:67): the oracle re-renders that pixel taking the other branch
of every cut-off within 1e-5 (relative) of its threshold, and that render
must agree with the device's."""
import numpy as np
import pytest

import yrtest as T
from yafray_b200 import abi, api, scenes

pytestmark = pytest.mark.gpu

RTOL = 1e-4


FLIP_BAND = 1e-5


def _cmp(img, ref, O=None):
    """Every pixel within RTOL, or explained by an energy cut-off flip
    (needs the oracle scene `O` that rendered `ref`)."""
    assert img.shape == ref.shape
    assert np.isfinite(img).all()
    rel = np.abs(img[..., :3] - ref[..., :3]) / np.maximum(np.abs(ref[..., :3]), 1e-3)
    bad = np.argwhere((rel > RTOL).any(-1))
    unexplained = []
    for y, x in bad:
        if O is not None:
            fl, _, margin = O.render_ex(int(x), int(x) + 1, int(y), int(y) + 1, flip_band=FLIP_BAND)
            r2 = np.abs(img[y, x, :3] - fl[y, x, :3]) / np.maximum(np.abs(fl[y, x, :3]), 1e-3)
            if margin[y, x] <= FLIP_BAND and (r2 <= RTOL).all():
                continue
        unexplained.append((int(x), int(y), float(rel[y, x].max())))
    assert not unexplained, (f"{len(unexplained)} of {len(bad)} pixels beyond {RTOL} without a cut-off flip: "
                             f"{unexplained[:6]}")
    return rel


@pytest.mark.parametrize("idx", [0, 5, 11, 17, 23, 29])
def test_render_uneven_batch_scenes(cuda, idx):
    """Scenes of the uneven batch (spheres and tori, 1-4 point and area
    lights, GI of 1-3 bounces) at a reduced frame, some with a hemi light
    or a penumbra guess added, against the oracle: the shading warps' queue
    reservations, the path vertices' lane-major places and the hits-first
    path-shading order on many scene shapes."""
    sc = scenes.config_batch(count=30)[idx]
    sc.camera.resx, sc.camera.resy = 40, 30
    sc.render.spp = 2
    if idx % 2:
        sc.lights.append(scenes.hemi_light(samples=4, power=0.4, maxdist=2.5))
    if idx % 4 == 1:
        for l in sc.lights:
            if l.type == abi.YR_LIGHT_AREA and l.samples > 1:
                l.psamples = 3
    img = api.DeviceScene(sc).render()
    O = T.OracleScene(sc)
    ref, _ = O.render()
    assert np.array_equal(img[..., 3], ref[..., 3])
    _cmp(img, ref, O)


def test_render_small_point_light(cuda):
    """320x240 point light, 1 spp: the benchmark's CPU-runnable case."""
    sc = scenes.config_small()
    ds = api.DeviceScene(sc)
    img = ds.render()
    O = T.OracleScene(sc)
    ref, stats = O.render()
    assert np.array_equal(img[..., 3], ref[..., 3])
    _cmp(img, ref, O)
    st = ds.last_stats
    assert st.rays_primary == stats[0] and st.rays_shadow == stats[1]


def test_render_small_aa(cuda):
    sc = scenes.config_small(96, 72)
    sc.render.spp = 5
    ds = api.DeviceScene(sc)
    img = ds.render()
    O = T.OracleScene(sc)
    ref, _ = O.render()
    _cmp(img, ref, O)


def test_render_gi_area_lights(cuda):
    """Area lights + path GI with 2 bounces on a small sphere grid."""
    sc = scenes.config_large(seed=2, resx=64, resy=40, spp=4, grid=2)
    ds = api.DeviceScene(sc)
    img = ds.render()
    O = T.OracleScene(sc)
    ref, stats = O.render()
    _cmp(img, ref, O)
    st = ds.last_stats
    assert st.rays_primary == stats[0]
    assert abs(int(st.rays_shadow) - int(stats[1])) <= 0.001 * stats[1] + 4
    assert abs(int(st.rays_bounce) - int(stats[2])) <= 0.001 * stats[2] + 4


def test_render_hemi_and_texture(cuda):
    sc = scenes.config_small(64, 48)
    sc.shaders[0] = scenes.fbm_shader((0.8, 0.8, 0.8), (0.2, 0.5, 0.7), (1.0, 1.0, 1.0), 0.7, 3.0)
    sc.lights.append(scenes.hemi_light(samples=8, power=0.5))
    sc.render.spp = 2
    ds = api.DeviceScene(sc)
    img = ds.render()
    O = T.OracleScene(sc)
    ref, _ = O.render()
    _cmp(img, ref, O)


def test_render_per_triangle_materials(cuda):
    sc = scenes.config_diff(res=48, spp=2, groups=8, nlights=2)
    ds = api.DeviceScene(sc)
    img = ds.render()
    O = T.OracleScene(sc)
    ref, _ = O.render()
    _cmp(img, ref, O)


@pytest.mark.parametrize("flags", [1, 2, 3])
def test_render_gi_traversal_variants(cuda, flags):
    """The same image with the shadow-ray tree and/or the exact object order."""
    sc = scenes.config_large(seed=2, resx=48, resy=32, spp=2, grid=2)
    a = api.DeviceScene(sc).render()
    sc.render.flags = flags
    b = api.DeviceScene(sc).render()
    assert np.array_equal(a, b)


def _layered_spheres_scene(res=40, layers=4, n=7):
    """Layers of small spheres between a ground plane and a point light
    overhead: shadow rays cross the bounds of several objects on their way,
    so the casters' BVH walk shoots many objects per ray."""
    pv, pt = scenes.ground_plane(half=20.0, y=-1.0)
    sc = scenes.Scene(name="layered")
    sc.shaders = [scenes.shader((0.8, 0.8, 0.8)), scenes.shader((0.6, 0.3, 0.2), (0.2, 0.2, 0.2), hard=10.0)]
    sc.meshes = [scenes.Mesh(pv, pt, 0)]
    for L in range(layers):
        for i in range(n):
            for j in range(n):
                c = (-1.5 + 0.5 * i + 0.13 * L, -0.4 + 0.9 * L, -1.5 + 0.5 * j - 0.07 * L)
                v, t = scenes.uv_sphere(c, 0.24, rings=6, segments=10)
                sc.meshes.append(scenes.Mesh(v, t, 1))
    sc.lights = [scenes.point_light((0.3, 9.0, 0.2), 60.0)]
    sc.camera = scenes.camera((0, 2.5, 6), (0, 0, 0), (0, 3.5, 6), res, res)
    sc.render = scenes.render_params(spp=2, seed=3)
    return sc


def test_render_many_shadow_candidates(cuda):
    sc = _layered_spheres_scene()
    ds = api.DeviceScene(sc)
    img = ds.render()
    O = T.OracleScene(sc)
    ref, stats = O.render()
    assert np.array_equal(img[..., 3], ref[..., 3])
    _cmp(img, ref, O)
    assert ds.last_stats.rays_shadow == stats[1]
    sc.render.flags = 2  # exact order: the nested walk, same image
    assert np.array_equal(api.DeviceScene(sc).render(), img)


@pytest.mark.parametrize("gi", [False, True])
def test_render_smoothed_meshes(cuda, gi):
    """Interpolated shading normals of smoothed meshes (autoSmooth at 180 and
    40 degrees), with a point light, and with area light + path GI."""
    import sys, os
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_golden
    sc = make_golden.smooth_scene()
    if gi:
        sc.lights = [scenes.quad_light_down(0.5, 5.0, 0.5, 2.0, 2.0, 30.0, 4),
                     scenes.path_light(samples=1, depth=2, power=1.0)]
        sc.render.spp = 3
    ds = api.DeviceScene(sc)
    img = ds.render()
    O = T.OracleScene(sc)
    ref, _ = O.render()
    assert np.array_equal(img[..., 3], ref[..., 3])
    _cmp(img, ref, O)


def test_render_texture_coordinates(cuda):
    """fBm modulators addressed by the shading normal, by orco, and through
    swapped / switched-off projection axes."""
    import sys, os
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_golden
    sc = make_golden.texco_scene()
    img = api.DeviceScene(sc).render()
    O = T.OracleScene(sc)
    ref, _ = O.render()
    assert np.array_equal(img[..., 3], ref[..., 3])
    _cmp(img, ref, O)


@pytest.mark.parametrize("gi", [False, True])
def test_render_procedural_textures(cuda, gi):
    """Marble, wood, voronoi, the musgrave types, distorted noise, clouds and
    gradients over every noise basis, with the mix / mul / add / sub
    modulator modes; with point lights, and with area light + path GI (the
    modulated colour at every bounce)."""
    import sys, os
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_golden
    sc = make_golden.texture_scene()
    if gi:
        sc.lights = [scenes.quad_light_down(0.0, 5.0, 0.0, 3.0, 2.0, 40.0, 4),
                     scenes.path_light(samples=1, depth=2, power=1.0)]
        sc.render.spp = 2
    img = api.DeviceScene(sc).render()
    O = T.OracleScene(sc)
    ref, _ = O.render()
    assert np.array_equal(img[..., 3], ref[..., 3])
    _cmp(img, ref, O)


def test_render_window_reflect_texco(cuda):
    """Textures addressed by the screen position ("window") and the
    reflected eye ("reflect"), with AA samples; and with a 2-bounce path
    light, where the path vertices have no screen position and reflect the
    bounce ray."""
    import sys, os
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_golden
    for gi in (False, True):
        sc = make_golden.texco_view_scene()
        if gi:
            sc.lights = [scenes.quad_light_down(0.0, 4.0, 1.0, 2.0, 2.0, 30.0, 4),
                         scenes.path_light(samples=1, depth=2, power=1.0)]
        img = api.DeviceScene(sc).render()
        O = T.OracleScene(sc)
        ref, _ = O.render()
        assert np.array_equal(img[..., 3], ref[..., 3])
        _cmp(img, ref, O)


def test_render_uv_texco(cuda):
    """Textures addressed by per-triangle texture coordinates ("uv"), the
    smoothed and flat meshes without them at (0, 0) and (-1, -1); with a
    2-bounce path light too."""
    import sys, os
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_golden
    for gi in (False, True):
        sc = make_golden.texco_uv_scene()
        if gi:
            sc.lights = [scenes.quad_light_down(0.0, 4.0, 1.0, 2.0, 2.0, 30.0, 4),
                         scenes.path_light(samples=1, depth=2, power=1.0)]
        img = api.DeviceScene(sc).render()
        O = T.OracleScene(sc)
        ref, _ = O.render()
        assert np.array_equal(img[..., 3], ref[..., 3])
        _cmp(img, ref, O)


def test_render_orco_of_transformed_meshes(cuda):
    """"orco" coordinates through each mesh's orco matrix (the reference's
    backOrco), on a smoothed mesh too; with a 2-bounce path light as well."""
    import sys, os
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_golden
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "render_texco_orco_80x60.npz"))
    for gi in (False, True):
        sc = make_golden.texco_orco_scene(dict(zip(g["orco_idx"], g["orco"])))
        if gi:
            sc.lights = [scenes.quad_light_down(0.0, 4.0, 1.0, 2.0, 2.0, 30.0, 4),
                         scenes.path_light(samples=1, depth=2, power=1.0)]
        img = api.DeviceScene(sc).render()
        O = T.OracleScene(sc)
        ref, _ = O.render()
        assert np.array_equal(img[..., 3], ref[..., 3])
        _cmp(img, ref, O)


def test_render_specular_hardness_modulation(cuda):
    """The modulator's "specular" and "hard" weights: the texture also
    drives the specular colour and the Phong exponent, every mode."""
    import sys, os
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_golden
    sc = make_golden.specmod_scene()
    img = api.DeviceScene(sc).render()
    O = T.OracleScene(sc)
    ref, _ = O.render()
    assert np.array_equal(img[..., 3], ref[..., 3])
    _cmp(img, ref, O)


@pytest.mark.parametrize("gi", [False, True])
def test_render_penumbra_guess(cuda, gi):
    """Area lights that guess the penumbra first (psamples 4, 6 and 3):
    the probes, the decision (lit: every grid point without a shadow ray;
    shadow: nothing; penumbra: the jittered samples) at the camera hit and,
    with a 2-bounce path light, at every path vertex."""
    import sys, os
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_golden
    sc = make_golden.guess_scene()
    sc.render.spp = 2
    if gi:
        sc.lights.append(scenes.path_light(samples=1, depth=2, power=1.0))
    ds = api.DeviceScene(sc)
    img = ds.render()
    O = T.OracleScene(sc)
    ref, _ = O.render()
    assert np.array_equal(img[..., 3], ref[..., 3])
    _cmp(img, ref, O)
    # the guess changes the image
    for l in sc.lights:
        l.psamples = 0
    assert np.abs(api.DeviceScene(sc).render() - img).max() > 1e-3


def test_render_penumbra_guess_batch(cuda):
    """The batched renderer on scenes with the penumbra guess and with the
    path light's adaptive rounds (waves schedule): each image equals
    yr_render's."""
    import torch
    import sys, os
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_golden
    scs = [make_golden.guess_scene(), scenes.config_small(64, 48), make_golden.rounds_scene(0.005)]
    scs[0].render.spp = 2
    scs[2].camera.resx, scs[2].camera.resy = 40, 30
    dss = [api.DeviceScene(sc) for sc in scs]
    outs = [torch.zeros((sc.resy, sc.resx, 4), dtype=torch.float32, device="cuda") for sc in scs]
    api.render_batch(dss, [o.data_ptr() for o in outs])
    torch.cuda.synchronize()
    for d, o in zip(dss, outs):
        assert np.array_equal(o.cpu().numpy().view(np.uint32), d.render().view(np.uint32))


@pytest.mark.parametrize("threshold", [0.1, 0.005])
def test_render_path_adaptive_rounds(cuda, threshold):
    """The path light's adaptive extra rounds (threshold 0.1, the factory's
    default, and 0.005): round 0's partial sums decide up to three more
    rounds of paths per camera sample, with their own QMC indices."""
    import sys, os
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_golden
    sc = make_golden.rounds_scene(threshold)
    sc.camera.resx, sc.camera.resy = 48, 36
    sc.render.spp = 2
    ds = api.DeviceScene(sc)
    img = ds.render()
    O = T.OracleScene(sc)
    ref, stats = O.render()
    assert np.array_equal(img[..., 3], ref[..., 3])
    _cmp(img, ref, O)
    st = ds.last_stats
    assert abs(int(st.rays_bounce) - int(stats[2])) <= 0.001 * stats[2] + 4
    # extra rounds were taken, and they change the image
    sc.lights[1].threshold = 0.0
    d1 = api.DeviceScene(sc)
    one = d1.render()
    assert d1.last_stats.rays_bounce < st.rays_bounce
    assert np.abs(one - img).max() > 1e-4


def test_render_path_rounds_large_config(cuda):
    """The benchmark's GI scene (2x2 grid) with the path light at its
    factory default threshold 0.1."""
    sc = scenes.config_large(seed=2, resx=48, resy=32, spp=2, grid=2)
    sc.lights[-1].threshold = 0.1
    ds = api.DeviceScene(sc)
    img = ds.render()
    O = T.OracleScene(sc)
    ref, _ = O.render()
    assert np.array_equal(img[..., 3], ref[..., 3])
    _cmp(img, ref, O)


def test_render_texture_board(cuda):
    """All 95 texture configurations of the golden texture set, one quad
    each (per-triangle materials)."""
    import sys, os
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_golden
    sc = make_golden.texture_board()
    img = api.DeviceScene(sc).render()
    O = T.OracleScene(sc)
    ref, _ = O.render()
    assert np.array_equal(img[..., 3], ref[..., 3])
    _cmp(img, ref, O)


def test_invalid_texture_records_rejected(cuda):
    """Out-of-range texture enums are refused at scene creation."""
    for field, val in (("tex_type", 12), ("tex_noise", 10), ("mod_mode", 4), ("tex_metric", 7)):
        sc = scenes.config_small(16, 12)
        s = scenes.texture_shader((0.5, 0.5, 0.5), "voronoi")
        setattr(s, field, val)
        sc.shaders = [s]
        with pytest.raises(RuntimeError):
            api.DeviceScene(sc)


@pytest.mark.parametrize("k", range(5))
def test_render_tone_mapping(cuda, k):
    """Per-sample exposure / gamma / clamp (the loader's TGA path) and alpha
    premultiply on a constant background, against the oracle."""
    import sys, os
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_golden
    sc = make_golden.tonemap_scene(make_golden.tonemap_configs()[k])
    img = api.DeviceScene(sc).render()
    O = T.OracleScene(sc)
    ref, _ = O.render()
    assert np.array_equal(img[..., 3], ref[..., 3])
    _cmp(img, ref, O)


def test_tone_mapping_gamma_zero_refused(cuda):
    sc = scenes.config_small(16, 12)
    sc.render = scenes.render_params(tonemap=True, gamma=0.0)
    with pytest.raises(RuntimeError):
        api.DeviceScene(sc)


@pytest.mark.parametrize("gi", [False, True])
@pytest.mark.parametrize("reference_inverses", [False, True])
def test_render_instances(cuda, gi, reference_inverses):
    """References (instanced meshes) shaded through MRot / M, orco at M^-1 P,
    smoothed originals; point light, and area light + path GI."""
    import sys, os
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_golden
    sc = make_golden.instance_scene()
    if reference_inverses:
        g = np.load(os.path.join(T.GOLDEN, "instances.npz"))
        for i, inv in zip(g["inv_idx"], g["inv"]):
            sc.meshes[int(i)].inverse = inv
    if gi:
        sc.lights = [scenes.quad_light_down(0.0, 4.0, 0.5, 2.0, 2.0, 30.0, 4),
                     scenes.path_light(samples=1, depth=2, power=1.0)]
        sc.render.spp = 2
    img = api.DeviceScene(sc).render()
    O = T.OracleScene(sc)
    ref, _ = O.render()
    assert np.array_equal(img[..., 3], ref[..., 3])
    _cmp(img, ref, O)
