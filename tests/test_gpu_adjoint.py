"""yr_backward against central finite differences of the loss.

L(theta) = sum over pixels and RGB of (render(theta) - target)^2, accumulated
in FP64 from the FP32 images; FD step 1e-3 (the step actually taken in
float32 is the denominator).  Tolerance: 1e-3 relative, plus an absolute
floor of 1e-3 of the largest gradient for parameters whose gradient is
near zero.  Scenes with a path light or a hemi light have energy cut-offs
(paths stop below 0.05) that the adjoint treats as fixed; their test
scenes are checked, through the oracle, to keep every cut-off value far
from its threshold, so that the finite-difference steps flip none."""
import numpy as np
import pytest

from yafray_b200 import api, scenes

pytestmark = pytest.mark.gpu


def _loss(img, target):
    d = img[..., :3].astype(np.float64) - target[..., :3].astype(np.float64)
    return float((d * d).sum())


def _render(torch, ds):
    t = torch.zeros((ds.sc.resy, ds.sc.resx, 4), dtype=torch.float32, device="cuda")
    ds.render_into(t.data_ptr())
    torch.cuda.synchronize()
    return t


def _check(torch, sc, hidden_params_fn, nsample=16, rtol=1e-3, seed=0):
    ds = api.DeviceScene(sc)
    theta = ds.params_get().astype(np.float32)
    n = theta.size
    ds.params_set(hidden_params_fn(theta))
    target = _render(torch, ds)
    ds.params_set(theta)
    img = _render(torch, ds)
    grad = torch.zeros(n, dtype=torch.float32, device="cuda")
    loss = ds.backward(img.data_ptr(), target.data_ptr(), grad.data_ptr(), 1.0)
    g = grad.cpu().numpy().astype(np.float64)
    tgt = target.cpu().numpy()
    assert loss == pytest.approx(_loss(img.cpu().numpy(), tgt), rel=1e-5)
    rng = np.random.default_rng(seed)
    idx = rng.choice(n, size=min(nsample, n), replace=False)
    fd = np.zeros(idx.size)
    for q, k in enumerate(idx):
        tp, tm = theta.copy(), theta.copy()
        tp[k] = np.float32(theta[k] + 1e-3)
        tm[k] = np.float32(theta[k] - 1e-3)
        ds.params_set(tp)
        lp = _loss(_render(torch, ds).cpu().numpy(), tgt)
        ds.params_set(tm)
        lm = _loss(_render(torch, ds).cpu().numpy(), tgt)
        fd[q] = (lp - lm) / (float(tp[k]) - float(tm[k]))
    ds.params_set(theta)
    floor = 1e-3 * np.abs(fd).max()
    err = np.abs(g[idx] - fd)
    bad = err > rtol * np.abs(fd) + floor
    assert not bad.any(), (f"params {idx[bad]}: adjoint {g[idx][bad]} vs FD {fd[bad]} "
                           f"(rel {(err / np.maximum(np.abs(fd), 1e-30))[bad]})")
    return ds, g, fd


def _margin_ok(sc, least=0.2):
    """Every energy cut-off value of the scene's render lies at least
    `least` (relative) away from its 0.05 threshold (oracle)."""
    import yrtest as T
    _, _, m = T.OracleScene(sc).render_ex(0, sc.resx, 0, sc.resy)
    assert m.min() > least, f"a cut-off value within {m.min():.3g} of its threshold"


def _hidden(seed):
    def f(theta):
        rng = np.random.default_rng(seed)
        return (theta * rng.uniform(0.7, 1.3, theta.size)).astype(np.float32)
    return f


def test_param_layout_and_roundtrip(cuda):
    sc = scenes.config_diff(res=32, spp=1, groups=64, nlights=8)
    ds = api.DeviceScene(sc)
    assert ds.param_count() == 64 * 4 + 8
    p = ds.params_get()
    assert np.allclose(p[0:3], sc.shaders[0].color[:])
    assert p[3] == pytest.approx(max(sc.shaders[0].specular[:]))
    assert p[-1] == pytest.approx(sc.lights[-1].power)
    q = (p * 1.1).astype(np.float32)
    ds.params_set(q)
    assert np.allclose(ds.params_get(), q, rtol=1e-6)


def test_grad_materials_and_area_lights(cuda):
    """Config-4 shape at reduced size: 16 material groups (diffuse RGB +
    specular weight) and 4 area lights."""
    import torch
    sc = scenes.config_diff(res=64, spp=4, groups=16, nlights=4)
    _check(torch, sc, _hidden(1))


def test_grad_point_light_and_specular(cuda):
    import torch
    sc = scenes.config_small(48, 36)
    sc.shaders[0].specular[:] = [0.3, 0.3, 0.3]
    sc.shaders[0].hard = 10.0
    sc.lights.append(scenes.point_light((-3.0, 4.0, 3.0), 0.7, color=(1.0, 0.8, 0.6)))
    sc.render.spp = 2
    _check(torch, sc, _hidden(2), nsample=7)


def test_grad_path_light_and_fbm_texture(cuda):
    """Path GI (2 bounces) with an fBm-modulated albedo: amplitude and base
    colour of the texture, the path light's power."""
    import torch
    sc = scenes.config_small(48, 36)
    sc.shaders = [scenes.fbm_shader((0.6, 0.5, 0.4), (0.7, 0.3, 0.2), (1.0, 1.0, 1.0), 0.6, 3.0, mod_color=0.7),
                  scenes.shader((0.8, 0.8, 0.8), (0.2, 0.2, 0.2), hard=8.0)]
    sc.meshes[1].shader = 1
    sc.lights = [scenes.quad_light_down(1.0, 5.0, 1.0, 2.0, 2.0, 30.0, 4),
                 scenes.path_light(samples=2, depth=2, power=1.0)]
    sc.render.spp = 4
    _margin_ok(sc)
    ds, g, fd = _check(torch, sc, _hidden(3), nsample=14, rtol=1e-3)
    assert ds.param_count() == 8 + 4 + 2


def test_grad_hemi_light(cuda):
    import torch
    sc = scenes.config_small(40, 30)
    sc.lights = [scenes.hemi_light(samples=8, power=0.8)]
    sc.render.spp = 2
    _margin_ok(sc)
    _check(torch, sc, _hidden(4), nsample=5, rtol=1e-3)


def _scene_with_params(sc, theta):
    """A copy of the scene description with the parameter vector written
    into its shader and light records the way yr_params_set maps it (per
    shader: colour, the specular weight along the specular colour's
    direction, and for textured shaders the texture amplitude and base
    colour; per light: power), in float32 as the library does."""
    import copy
    from yafray_b200 import abi
    s2 = copy.copy(sc)
    s2.shaders, s2.lights = [], []
    f32 = np.float32
    n = 0
    for d in sc.shaders:
        e = abi.YrShaderDesc.from_buffer_copy(d)
        ks = [f32(x) for x in d.specular]
        w = max(ks)
        sdir = [k / w if w > 0 else f32(1.0) for k in ks]
        e.color[:] = [float(theta[n + c]) for c in range(3)]
        e.specular[:] = [float(f32(theta[n + 3]) * sdir[c]) for c in range(3)]
        n += 4
        if d.tex_type != abi.YR_TEX_NONE:
            e.tex_intensity = float(theta[n])
            e.tex_color1[:] = [float(theta[n + 1 + c]) for c in range(3)]
            n += 4
        s2.shaders.append(e)
    for l in sc.lights:
        e = abi.YrLightDesc.from_buffer_copy(l)
        e.power = float(theta[n])
        n += 1
        s2.lights.append(e)
    assert n == len(theta)
    return s2


@pytest.mark.parametrize("gi", [False, True])
def test_grad_against_oracle_finite_differences(cuda, gi):
    """The adjoint against central differences of the ORACLE's forward
    render (the CPU restatement of the reference's estimators, FP64 loss
    accumulation, step 1e-3) on a config-4-shaped scene at small size: 8
    material groups (diffuse RGB + specular weight) and 2 area lights, 48x48,
    4 spp; with `gi` also a 2-bounce path light.  The oracle's renders
    are checked to keep every energy cut-off decision at least 20% away from
    its threshold, so a step of 1e-3 cannot flip one."""
    import torch
    import yrtest as T
    sc = scenes.config_diff(res=48, spp=4, groups=8, nlights=2)
    if gi:
        sc.lights.append(scenes.path_light(samples=1, depth=2, power=1.0))
    ds = api.DeviceScene(sc)
    theta = ds.params_get().astype(np.float32)
    n = theta.size
    assert n == 8 * 4 + len(sc.lights)
    ds.params_set(_hidden(7)(theta))
    target = _render(torch, ds)
    ds.params_set(theta)
    img = _render(torch, ds)
    grad = torch.zeros(n, dtype=torch.float32, device="cuda")
    ds.backward(img.data_ptr(), target.data_ptr(), grad.data_ptr(), 1.0)
    g = grad.cpu().numpy().astype(np.float64)
    tgt = target.cpu().numpy()
    trees = [T.product_tree(m) for m in sc.meshes]

    def oracle_loss(th):
        O = T.OracleScene(_scene_with_params(sc, th), trees=trees)
        im, _, margin = O.render_ex(0, sc.resx, 0, sc.resy)
        O.close()
        return _loss(im, tgt), float(margin.min())

    l0, m0 = oracle_loss(theta)
    assert m0 > 0.2, f"an energy cut-off value lies within {m0:.3g} (relative) of its threshold"
    assert l0 == pytest.approx(_loss(img.cpu().numpy(), tgt), rel=1e-4)  # oracle and device forwards agree
    rng = np.random.default_rng(11)
    idx = rng.choice(n, size=16, replace=False)
    fd = np.zeros(idx.size)
    for q, k in enumerate(idx):
        tp, tm = theta.copy(), theta.copy()
        tp[k] = np.float32(theta[k] + 1e-3)
        tm[k] = np.float32(theta[k] - 1e-3)
        (lp, mp), (lm, mm) = oracle_loss(tp), oracle_loss(tm)
        assert min(mp, mm) > 0.2
        fd[q] = (lp - lm) / (float(tp[k]) - float(tm[k]))
    big = np.abs(fd) > 1e-3 * np.abs(fd).max()
    rel = np.abs(g[idx] - fd) / np.maximum(np.abs(fd), 1e-30)
    assert big.sum() >= 12
    assert (rel[big] <= 1e-3).all(), f"params {idx[big][rel[big] > 1e-3]}: rel {rel[big][rel[big] > 1e-3]}"
    assert (np.abs(g[idx] - fd)[~big] <= 1e-4 * np.abs(fd).max()).all()


def test_backward_rejects_bad_args(cuda):
    import torch
    from yafray_b200 import abi
    ds = api.DeviceScene(scenes.config_small(16, 12))
    img = _render(torch, ds)
    with pytest.raises(abi.YrError):
        ds.backward(img.data_ptr(), 0, 0)


def _noise_scenes(n, seed=9):
    rng = np.random.default_rng(seed)
    return [scenes.config_diffnoise_scene(rng, i, res=32, spp=4, tri_lo=2000, tri_hi=6000) for i in range(n)]


def test_backward_batch_matches_per_scene(cuda):
    """yr_backward_batch: images equal yr_render's; gradients and losses equal
    yr_backward's up to the order of FP32 atomic sums."""
    import torch
    scs = _noise_scenes(3)
    dss = [api.DeviceScene(sc) for sc in scs]
    targets = []
    for d in dss:
        th = d.params_get()
        d.params_set(_hidden(5)(th))
        targets.append(_render(torch, d))
        d.params_set(th)
    imgs = [torch.empty_like(t) for t in targets]
    grads = [torch.zeros(d.param_count(), dtype=torch.float32, device="cuda") for d in dss]
    for rep in range(2):  # capture, then replay
        losses = api.backward_batch(dss, [t.data_ptr() for t in imgs], [t.data_ptr() for t in targets],
                                    [g.data_ptr() for g in grads], 1.0, streams=2)
        torch.cuda.synchronize()
        for i, d in enumerate(dss):
            ref_img = _render(torch, d)
            assert torch.equal(imgs[i], ref_img)
            g1 = torch.zeros_like(grads[i])
            l1 = d.backward(ref_img.data_ptr(), targets[i].data_ptr(), g1.data_ptr(), 1.0)
            assert losses[i] == pytest.approx(l1, rel=1e-6)
            a, b = grads[i].cpu().numpy(), g1.cpu().numpy()
            assert np.allclose(a, b, rtol=1e-4, atol=1e-5 * np.abs(b).max())
        # a parameter change between steps is seen by the replayed graph
        th = dss[0].params_get()
        dss[0].params_set((th * 1.05).astype(np.float32))


def test_inverse_fit_recovers_parameters(cuda):
    """Adam through the batched step: the loss falls and the parameters move
    toward the hidden ones on every problem."""
    import torch
    from yafray_b200 import optim
    scs = _noise_scenes(2, seed=12)
    dss = [api.DeviceScene(sc) for sc in scs]
    targets, hidden, start = [], [], []
    for d in dss:
        th = d.params_get()
        hd = _hidden(6)(th)
        d.params_set(hd)
        targets.append(_render(torch, d))
        d.params_set(th)
        hidden.append(hd)
        start.append(th)
    params, hist, secs = optim.fit(dss, targets, steps=60, lr=2e-2, batched=True, streams=2)
    for i in range(len(dss)):
        assert hist[-1, i] < 0.2 * hist[0, i]


def test_grad_procedural_textures_and_modes(cuda):
    """Texture amplitude and base colour through ridged musgrave (mix),
    voronoi cell colours (add), marble (mul) and clouds (sub), point and area
    light."""
    import torch
    ts = scenes.texture_shader
    sc = scenes.config_small(48, 36)
    sc.shaders = [ts((0.6, 0.5, 0.4), "musgrave", (0.2, 0.4, 0.1), (0.9, 0.9, 0.7), mod_color=0.7, type="ridgedmf",
                     noise_type="blender", octaves=3.0, offset=1.0, gain=2.0, size=2.0, intensity=0.6),
                  ts((0.3, 0.3, 0.3), "voronoi", (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), mode="add", mod_color=0.5,
                     color_type="col2", weight1=1.0, weight2=-0.6, size=3.0, intensity=0.8)]
    sv, st = scenes.uv_sphere((1.3, 0.0, 0.0), 0.6, rings=16, segments=32)
    tv, tt = scenes.uv_sphere((-1.3, 0.0, 0.0), 0.6, rings=16, segments=32)
    sc.shaders += [ts((0.7, 0.6, 0.5), "marble", (0.9, 0.9, 0.8), (0.3, 0.2, 0.2), mode="mul", mod_color=0.8,
                      turbulence=2.0, depth=2, size=1.5),
                   ts((0.8, 0.8, 0.8), "clouds", (0.1, 0.2, 0.3), (0.5, 0.4, 0.3), mode="sub", mod_color=0.4,
                      noise_type="stdperlin", depth=3, size=1.2)]
    sc.meshes[0].shader = 0
    sc.meshes[1].shader = 1
    sc.meshes += [scenes.Mesh(sv, st, 2), scenes.Mesh(tv, tt, 3)]
    sc.lights = [scenes.point_light((3.0, 5.0, 2.0), 20.0), scenes.quad_light_down(0.0, 4.0, 1.0, 2.0, 2.0, 20.0, 4)]
    sc.render.spp = 2
    ds, g, fd = _check(torch, sc, _hidden(5), nsample=20, rtol=1e-3, seed=1)
    assert ds.param_count() == 4 * 8 + 2


def test_grad_alpha_premultiply(cuda):
    """With alpha premultiply the image is the sample average times its
    alpha coverage; gradients follow through the coverage."""
    import torch
    sc = scenes.config_small(40, 30)
    sc.render = scenes.render_params(spp=2, alpha_premultiply=True, background=(0.1, 0.2, 0.4))
    _check(torch, sc, _hidden(6), nsample=5)


def test_backward_refuses_tone_mapping(cuda):
    """Per-sample exposure / gamma is not differentiated: refused."""
    import torch
    from yafray_b200 import abi
    sc = scenes.config_small(16, 12)
    sc.render = scenes.render_params(tonemap=True, gamma=2.2)
    ds = api.DeviceScene(sc)
    img = _render(torch, ds)
    grad = torch.zeros(ds.param_count(), dtype=torch.float32, device="cuda")
    with pytest.raises(abi.YrError):
        ds.backward(img.data_ptr(), img.data_ptr(), grad.data_ptr())
