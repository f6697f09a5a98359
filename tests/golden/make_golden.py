"""Regenerate the golden vectors in this folder from the UNMODIFIED reference.

Run in the build container (needs oracle/_ref/yr_ref_harness, built from the
reference sources by `make -C oracle`):

    python tests/golden/make_golden.py

Every fixture is produced by the reference harness on seeded inputs; the
inputs themselves are either stored alongside or regenerated from the seeds
by yafray_b200.scenes.
"""
import os
import struct
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import yrtest as T  # noqa: E402
from yafray_b200 import abi, scenes  # noqa: E402


def small_sphere_scene():
    sv, st = scenes.uv_sphere((0.0, 0.0, 0.0), 1.0, rings=16, segments=32)
    pv, pt = scenes.ground_plane(20.0, -1.0)
    sc = scenes.config_small(80, 60)
    sc.meshes = [scenes.Mesh(sv, st, 0), scenes.Mesh(pv, pt, 0)]
    return sc


def random_mesh_scene(n, seed):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-5, 5, (n, 1, 3))
    v = (c + 0.3 * rng.uniform(-1, 1, (n, 3, 3))).reshape(-1, 3).astype(np.float32)
    t = np.arange(3 * n, dtype=np.uint32).reshape(n, 3)
    sc = scenes.config_small(80, 60)
    sc.meshes = [scenes.Mesh(v, t, 0)]
    return sc


def box_soup(rng, n):
    """n axis-aligned boxes (12 triangles each) on an integer grid, some
    stacked: many coplanar, flat and coincident triangle bounds."""
    faces = [(0, 1, 3, 2), (4, 6, 7, 5), (0, 4, 5, 1), (2, 3, 7, 6), (0, 2, 6, 4), (1, 5, 7, 3)]
    vs, ts = [], []
    for k in range(n):
        x, z = rng.integers(0, 24, 2)
        y = rng.integers(0, 3)
        w = rng.integers(1, 3)
        c = np.array([[x + (i & 1) * w, y + ((i >> 1) & 1), z + ((i >> 2) & 1) * w] for i in range(8)], np.float32)
        b = 8 * k
        for a0, a1, a2, a3 in faces:
            ts += [(b + a0, b + a1, b + a2), (b + a0, b + a2, b + a3)]
        vs.append(c)
    return np.concatenate(vs), np.array(ts, np.uint32)


def terrace(nx, nz, seed):
    """A height field on an nx x nz grid with heights quantised to 4 levels."""
    rng = np.random.default_rng(seed)
    h = rng.integers(0, 4, (nz + 1, nx + 1)).astype(np.float32) * 0.5
    xs, zs = np.meshgrid(np.arange(nx + 1, dtype=np.float32), np.arange(nz + 1, dtype=np.float32))
    v = np.stack([xs, h, zs], -1).reshape(-1, 3)
    t = []
    for j in range(nz):
        for i in range(nx):
            a = j * (nx + 1) + i
            t += [(a, a + 1, a + nx + 2), (a, a + nx + 2, a + nx + 1)]
    return v, np.array(t, np.uint32)


def tie_scene():
    """Meshes whose kd builds are decided by ties: equal split candidates
    (shared vertices, coplanar faces) and flat bounds, above and below the
    128-triangle switch between the binned and the sorted sweeps."""
    rng = np.random.default_rng(21)
    sc = scenes.config_small(80, 60)
    bv, bt = box_soup(rng, 400)
    tv, tt = terrace(40, 30, 22)
    sv, st = scenes.uv_sphere((0.0, 0.0, 0.0), 1.0, rings=48, segments=96)
    gv, gt = terrace(6, 5, 23)
    sc.meshes = [scenes.Mesh(bv, bt, 0), scenes.Mesh(tv, tt, 0), scenes.Mesh(sv, st, 0), scenes.Mesh(gv, gt, 0)]
    return sc


def tie_trees():
    out = {}
    tr, _ = T.harness_trees(tie_scene())
    for i, t in enumerate(tr):
        for k in ("nodes", "prims", "tb"):
            out[f"ties_{i}_{k}"] = t[k]
    np.savez_compressed(os.path.join(HERE, "trees_ties.npz"), **out)


def trees():
    out = {}
    for name, sc in (("sphere16", small_sphere_scene()), ("random3000", random_mesh_scene(3000, 11))):
        tr, ot = T.harness_trees(sc)
        for i, t in enumerate(tr):
            for k in ("nodes", "prims", "tb", "ob"):
                out[f"{name}_{i}_{k}"] = t[k]
            out[f"{name}_{i}_params"] = np.array([t["max_depth"], t["max_leaf"]], np.int32)
            out[f"{name}_{i}_cost"] = np.array([t["cost_ratio"]], np.float32)
        out[f"{name}_otree"] = ot
    np.savez_compressed(os.path.join(HERE, "trees.npz"), **out)


def rays():
    sc = scenes.config_small()
    n = 8192
    rng = np.random.default_rng(2)
    base = T.random_rays(sc, n, 1)
    recs = np.zeros(n, T.RAY_REC)
    recs["mode"] = rng.integers(0, 5, n)
    recs["object"] = rng.integers(0, 2, n)
    recs["frm"] = base[:, :3]
    recs["dir"] = base[:, 4:7]
    recs["dist"] = np.where(rng.random(n) < 0.5, -1.0, rng.uniform(0.5, 10, n))
    recs["l"] = base[:, :3] + base[:, 4:7] * rng.uniform(0.5, 8, (n, 1))
    res = T.harness_rays(sc, recs)
    np.savez_compressed(os.path.join(HERE, "rays_small.npz"), recs=recs, res=res)


def camera_and_render():
    sc = scenes.config_small(160, 120)
    cam = T.harness_camera(sc)
    img, _ = T.harness_render(sc)
    np.savez_compressed(os.path.join(HERE, "render_small_160x120.npz"), camera=cam, image=img)


def smooth_scene():
    """A coarse sphere smoothed at 180 degrees (one normal per vertex), a
    torus smoothed at 40 degrees (per-corner normals) and a flat plane;
    point light, a specular shader so that the normal shows."""
    sc = scenes.config_small(96, 72)
    sv, st = scenes.uv_sphere((-0.6, 0.0, 0.0), 0.8, rings=10, segments=20)
    tv, tt = scenes.torus((1.2, -0.3, 0.5), 0.6, 0.25, nu=24, nv=12)
    pv, pt = scenes.ground_plane(20.0, -1.0)
    sc.shaders = [scenes.shader((0.8, 0.7, 0.6), (0.4, 0.4, 0.4), hard=25.0), scenes.shader((0.8, 0.8, 0.8))]
    sc.meshes = [scenes.Mesh(sv, st, 0, smooth_angle=180.0), scenes.Mesh(tv, tt, 0, smooth_angle=40.0),
                 scenes.Mesh(pv, pt, 1)]
    return sc


def texco_scene():
    """fBm textures addressed by the shading normal and by swapped / switched
    off projection axes, on smoothed and flat meshes."""
    sc = smooth_scene()
    sc.shaders = [scenes.fbm_shader((0.6, 0.5, 0.4), (0.7, 0.3, 0.2), (1.0, 1.0, 1.0), 0.8, 2.5, mod_color=0.8,
                                    texco="normal", proj=("y", "x", "z")),
                  scenes.fbm_shader((0.8, 0.8, 0.8), (0.2, 0.5, 0.7), (1.0, 1.0, 1.0), 0.6, 1.5, mod_color=0.9,
                                    texco="orco", proj=("z", "n", "x"))]
    sc.shaders[1].mod_size[:] = [1.0, 2.0, 0.5]
    sc.shaders[1].mod_ofs[:] = [0.3, -0.2, 0.1]
    return sc


def smooth_render():
    sc = smooth_scene()
    img, _ = T.harness_render(sc)
    np.savez_compressed(os.path.join(HERE, "render_smooth_96x72.npz"), image=img)
    img, _ = T.harness_render(texco_scene())
    np.savez_compressed(os.path.join(HERE, "render_texco_96x72.npz"), image=img)


def illum_scene():
    """Smoothed sphere, torus and plane (textured and specular shaders) lit
    by a 16-sample and a 1-sample area light, two hemi lights (unbounded and
    at maxdist 2.5) and a point light."""
    sc = texco_scene()
    sc.shaders.append(scenes.shader((0.7, 0.6, 0.5), (0.5, 0.5, 0.5), hard=12.0))
    sc.meshes[2].shader = 2
    sc.lights = [scenes.quad_light_down(0.5, 3.0, 0.5, 2.0, 1.5, 3.0, samples=16, color=(1.0, 0.9, 0.8)),
                 scenes.area_light((-2.0, 2.5, -1.0), (-1.0, 2.5, -1.0), (-1.0, 2.5, 0.0), (-2.0, 2.5, 0.0), 2.0,
                                   samples=1),
                 scenes.hemi_light(samples=9, power=0.8, color=(0.9, 0.95, 1.0)),
                 scenes.hemi_light(samples=4, power=1.2, maxdist=2.5),
                 scenes.point_light((2.0, 3.0, 2.0), 4.0)]
    return sc


def box_mesh(lo, hi, shader):
    """Closed axis-aligned box, 12 triangles."""
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    v = np.array([[x0, y0, z0], [x1, y0, z0], [x1, y1, z0], [x0, y1, z0],
                  [x0, y0, z1], [x1, y0, z1], [x1, y1, z1], [x0, y1, z1]], np.float32)
    t = np.array([[0, 2, 1], [0, 3, 2], [4, 5, 6], [4, 6, 7], [0, 1, 5], [0, 5, 4],
                  [3, 6, 2], [3, 7, 6], [0, 4, 7], [0, 7, 3], [1, 2, 6], [1, 6, 5]], np.uint32)
    return scenes.Mesh(v, t, shader)


def path_scene():
    """A closed room (no path reaches the background) with a smoothed sphere
    and a torus, bright albedos (no path ends early), a point light for the
    direct light at the bounce vertices and a 4-sample, 3-bounce path light."""
    sc = smooth_scene()
    sc.shaders = [scenes.shader((0.9, 0.8, 0.7), (0.3, 0.3, 0.3), hard=20.0),
                  scenes.fbm_shader((0.85, 0.85, 0.8), (0.7, 0.8, 0.9), (0.95, 0.85, 0.7), 0.7, 1.5, mod_color=0.8),
                  scenes.shader((0.8, 0.85, 0.9))]
    sc.meshes = [sc.meshes[0], sc.meshes[1], box_mesh((-4.0, -1.0, -4.0), (4.0, 4.0, 6.0), 2)]
    sc.meshes[1].shader = 1
    sc.lights = [scenes.point_light((0.5, 3.0, 1.0), 6.0), scenes.path_light(samples=4, depth=3, power=1.0)]
    return sc


def illum_queries(sc, n, seed):
    """Rays from the camera towards random points of the image, each for one
    light (in turn), with a random QMC sample index and LCG seed."""
    rng = np.random.default_rng(seed)
    q = np.zeros(n, T.ILLUM_REC)
    cam = sc.camera
    pos = np.array(cam.pos[:], np.float32)
    look = np.array(cam.look[:], np.float32)
    tgt = look + rng.uniform(-2.5, 2.5, (n, 3)).astype(np.float32) * np.float32([1.0, 0.6, 1.0])
    d = tgt - pos
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    q["light"] = np.arange(n) % len(sc.lights)
    q["m0"] = rng.integers(0, 4096, n)
    q["lcg"] = rng.integers(1, 2 ** 31 - 2, n)
    q["eye"] = pos
    q["frm"] = pos
    q["dir"] = d.astype(np.float32)
    return q


def illum():
    out = {}
    for name, sc, n, seed in (("gi", illum_scene(), 600, 11), ("path", path_scene(), 200, 12)):
        q = illum_queries(sc, n, seed)
        out[name + "_q"] = q
        out[name + "_o"] = T.harness_illum(sc, q)
    np.savez_compressed(os.path.join(HERE, "illum.npz"), **out)


def guess_scene():
    """The illumination scene lit by area lights with the penumbra guess
    (psamples 4 over a 12-point grid, 6 over 9, 3 over 2): the objects put
    points in full light, in full shadow and in penumbra."""
    sc = illum_scene()
    sc.lights = [scenes.quad_light_down(0.5, 3.0, 0.5, 2.0, 1.5, 3.0, samples=16, color=(1.0, 0.9, 0.8),
                                        psamples=4),
                 scenes.quad_light_down(-1.0, 2.5, -0.5, 1.2, 1.2, 2.0, samples=9, psamples=6),
                 scenes.quad_light_down(1.5, 2.0, -1.0, 0.8, 0.6, 1.5, samples=4, psamples=3)]
    return sc


def rounds_scene(threshold):
    """The path scene with the path light's adaptive rounds on."""
    sc = path_scene()
    sc.lights[1] = scenes.path_light(samples=4, depth=3, power=1.0, threshold=threshold)
    return sc


def illum_rounds():
    out = {}
    for name, thr, seed in (("t10", 0.1, 31), ("t005", 0.005, 32), ("t001", 0.001, 33)):
        sc = rounds_scene(thr)
        q = illum_queries(sc, 200, seed)
        q["light"] = 1
        out[name + "_q"] = q
        out[name + "_o"] = T.harness_illum(sc, q)
    np.savez_compressed(os.path.join(HERE, "illum_rounds.npz"), **out)


def illum_guess():
    sc = guess_scene()
    q = illum_queries(sc, 900, 21)
    np.savez_compressed(os.path.join(HERE, "illum_guess.npz"), q=q, o=T.harness_illum(sc, q))


def texture_shaders():
    """One shader per texture configuration: every noise basis under clouds,
    the marble / wood shapes and variants, voronoi under every metric and
    colour type, the musgrave types over three bases and fractional
    octaves, distorted noise and the gradient types."""
    ts, c1, c2 = scenes.texture_shader, (0.1, 0.3, 0.8), (0.9, 0.6, 0.2)
    out = []
    for nt in abi.NOISE_TYPES:
        out.append(ts((0.5,) * 3, "clouds", c1, c2, noise_type=nt, depth=3, size=1.3))
    out += [ts((0.5,) * 3, "clouds", c1, c2, hard=True, bias="positive", depth=2),
            ts((0.5,) * 3, "clouds", c1, c2, bias="negative", noise_type="blender")]
    for sh in ("sin", "saw", "tri"):
        out.append(ts((0.5,) * 3, "marble", c1, c2, shape=sh, turbulence=2.5, sharpness=3.0, depth=3, size=0.7))
        out.append(ts((0.5,) * 3, "wood", c1, c2, shape=sh, wood_type="rings", turbulence=1.5,
                      noise_type="stdperlin"))
        out.append(ts((0.5,) * 3, "wood", c1, c2, shape=sh, hard=True, turbulence=0.5))
    out.append(ts((0.5,) * 3, "marble", c1, c2, turbulence=0.0))
    for m in abi.DIST_METRICS:
        for ct in ("int", "col1", "col2", "col3"):
            out.append(ts((0.5,) * 3, "voronoi", c1, c2, color_type=ct, distance_metric=m, weight1=1.0, weight2=-0.5,
                          weight3=0.3, weight4=0.2, intensity=1.7, size=2.0, mk_exponent=1.7))
    for mt in ("fBm", "multifractal", "heteroterrain", "hybridmf", "ridgedmf"):
        for nt in ("newperlin", "blender", "voronoi_f2f1"):
            for oc in (3.0, 4.5):
                out.append(ts((0.5,) * 3, "musgrave", c1, c2, type=mt, noise_type=nt, octaves=oc, H=0.8,
                              lacunarity=2.2, offset=0.9, gain=1.7, size=1.4, intensity=0.6))
    for n1, n2 in (("newperlin", "stdperlin"), ("voronoi_crackle", "blender"), ("cellnoise", "newperlin")):
        out.append(ts((0.5,) * 3, "distorted_noise", c1, c2, noise_type1=n1, noise_type2=n2, distort=2.2, size=1.1))
    for gt in abi.GRADIENT_TYPES:
        for fl in (False, True):
            out.append(ts((0.5,) * 3, "gradient", c1, c2, gradient_type=gt, flip_xy=fl))
    return out


def texture_points():
    rng = np.random.default_rng(3)
    return np.concatenate([rng.uniform(-1.5, 1.5, (96, 3)), rng.uniform(-40, 40, (32, 3))]).astype(np.float32)


def textures():
    """noise bases (newNoise, turbulence, voronoi metrics) and every texture
    configuration's getColor / getFloat, from the reference."""
    pts = texture_points()
    sc = scenes.config_small(8, 8)
    sc.shaders = texture_shaders()
    with tempfile.TemporaryDirectory() as d:
        sp, pp, op, np_ = (os.path.join(d, n) for n in ("s.yrs", "p.bin", "t.bin", "n.bin"))
        scenes.write_yrs(sc, sp)
        with open(pp, "wb") as f:
            f.write(struct.pack("<I", len(pts)))
            f.write(pts.tobytes())
        T.run_harness("texeval", sp, pp, op)
        tex = np.fromfile(op, np.float32).reshape(len(sc.shaders), len(pts), 4)
        T.run_harness("noisegen", pp, np_)
        gen = np.fromfile(np_, np.float32).reshape(len(pts), 58)
    np.savez_compressed(os.path.join(HERE, "textures.npz"), pts=pts, tex=tex, noisegen=gen)


def texture_scene():
    """A 4 x 3 grid of small spheres, each with another texture, noise basis
    and modulator mode, on a plane with a voronoi colour texture; two point
    lights."""
    sc = scenes.config_small(128, 96)
    ts = scenes.texture_shader
    sc.shaders = [
        ts((0.6, 0.6, 0.6), "marble", (0.9, 0.9, 0.85), (0.2, 0.2, 0.3), mod_color=0.9, shape="sin", turbulence=3.0,
           sharpness=2.0, depth=3, size=2.0),
        ts((0.7, 0.5, 0.3), "wood", (0.5, 0.3, 0.1), (0.8, 0.6, 0.3), mode="mul", mod_color=0.8, wood_type="rings",
           shape="tri", noise_type="stdperlin", turbulence=0.8),
        ts((0.3, 0.3, 0.3), "voronoi", (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), mode="add", mod_color=0.5, color_type="col2",
           distance_metric="manhattan", weight1=1.0, weight2=-0.6, size=4.0),
        ts((0.5, 0.5, 0.6), "musgrave", (0.2, 0.4, 0.1), (0.9, 0.9, 0.7), type="ridgedmf", noise_type="blender",
           octaves=4.0, H=1.0, offset=1.0, gain=2.0, size=2.5, intensity=0.5),
        ts((0.5, 0.5, 0.5), "musgrave", (0.3, 0.2, 0.1), (0.8, 0.7, 0.9), type="hybridmf", noise_type="voronoi_f1",
           octaves=3.5, H=0.25, offset=0.7, gain=1.0, size=1.5, intensity=0.8, mod_color=0.7),
        ts((0.8, 0.8, 0.8), "musgrave", (0.1, 0.1, 0.1), (0.6, 0.5, 0.4), mode="sub", mod_color=0.4,
           type="heteroterrain", noise_type="cellnoise", octaves=3.0, offset=0.5, size=3.0, intensity=0.4),
        ts((0.4, 0.6, 0.5), "musgrave", (0.9, 0.2, 0.2), (0.2, 0.2, 0.9), type="multifractal", noise_type="stdperlin",
           octaves=5.0, H=0.7, size=2.0, intensity=0.5, texco="normal"),
        ts((0.5, 0.5, 0.5), "distorted_noise", (0.1, 0.5, 0.2), (0.9, 0.8, 0.1), noise_type1="voronoi_crackle",
           noise_type2="newperlin", distort=1.5, size=2.0, mod_color=0.9),
        ts((0.5, 0.4, 0.3), "gradient", (0.0, 0.0, 0.2), (1.0, 0.9, 0.6), gradient_type="halo", texco="normal",
           mode="mul", mod_color=1.0),
        ts((0.6, 0.6, 0.6), "clouds", (0.2, 0.3, 0.6), (0.9, 0.9, 0.9), noise_type="blender", bias="negative",
           depth=4, size=0.8, hard=True, mod_color=0.8),
        ts((0.5, 0.5, 0.5), "gradient", (0.2, 0.2, 0.2), (0.9, 0.8, 0.3), gradient_type="cubic", flip_xy=True,
           proj=("y", "n", "x"), mod_color=0.95),
        ts((0.5, 0.6, 0.4), "voronoi", (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), mode="mix", mod_color=0.6,
           color_type="int", distance_metric="minkovsky", mk_exponent=3.5, weight1=0.5, weight2=0.5, size=3.0,
           intensity=1.2),
        ts((0.7, 0.7, 0.7), "voronoi", (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), mod_color=0.7, color_type="col3",
           distance_metric="minkovsky_half", weight1=1.0, weight2=-1.0, size=1.0, intensity=2.0),
    ]
    meshes = []
    for k in range(12):
        v, t = scenes.uv_sphere((-1.8 + 1.2 * (k % 4), -0.5, -1.0 + 1.1 * (k // 4)), 0.5, rings=12, segments=24)
        meshes.append(scenes.Mesh(v, t, k))
    pv, pt = scenes.ground_plane(20.0, -1.0)
    meshes.append(scenes.Mesh(pv, pt, 12))
    sc.meshes = meshes
    sc.lights = [scenes.point_light((2.0, 4.0, 3.0), 14.0), scenes.point_light((-3.0, 3.0, -1.0), 6.0,
                                                                               color=(0.8, 0.9, 1.0))]
    sc.camera = scenes.camera((0.0, 3.0, 4.5), (0.0, -0.5, 0.0), (0.0, 4.0, 4.5), 128, 96)
    return sc


def texture_board():
    """Every texture configuration of texture_shaders() on its own quad of a
    10 x 10 board (per-triangle materials), seen from above, point light."""
    shs = texture_shaders()
    n = len(shs)
    verts, tris, tsh = [], [], []
    for k in range(n):
        x0, z0 = -5.0 + (k % 10), -5.0 + (k // 10)
        b = len(verts)
        verts += [(x0, 0.0, z0), (x0 + 1.0, 0.0, z0), (x0 + 1.0, 0.0, z0 + 1.0), (x0, 0.0, z0 + 1.0)]
        tris += [(b, b + 2, b + 1), (b, b + 3, b + 2)]
        tsh += [k, k]
    sc = scenes.config_small(160, 160)
    sc.shaders = shs
    sc.meshes = [scenes.Mesh(np.array(verts, np.float32), np.array(tris, np.uint32), abi.YR_PER_TRIANGLE,
                             np.array(tsh, np.uint32))]
    sc.lights = [scenes.point_light((0.5, 6.0, 1.0), 40.0)]
    sc.camera = scenes.camera((0.0, 9.0, 0.01), (0.0, 0.0, 0.0), (0.0, 10.0, 0.01), 160, 160, fov_deg=65.0)
    return sc


def texture_render():
    img, _ = T.harness_render(texture_scene())
    np.savez_compressed(os.path.join(HERE, "render_textures_128x96.npz"), image=img)


def specmod_scene():
    """Six spheres and the plane whose modulators also drive the specular
    colour and the Phong exponent (the modulator's "specular" and "hard"
    weights) in every mode - some with the colour channel off - over a
    specular base colour; two point lights."""
    sc = scenes.config_small(96, 72)
    ts = scenes.texture_shader
    base = dict(mod_specular=0.7, mod_hard=0.5)
    sc.shaders = [
        ts((0.6, 0.6, 0.6), "marble", (0.9, 0.9, 0.85), (0.2, 0.2, 0.3), mod_color=0.6, turbulence=2.0, size=2.0,
           **base),
        ts((0.7, 0.5, 0.3), "musgrave", (0.5, 0.3, 0.1), (0.8, 0.6, 0.3), mode="mul", mod_color=0.8, size=2.5,
           intensity=0.6, mod_specular=0.9, mod_hard=0.3),
        ts((0.3, 0.3, 0.3), "voronoi", (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), mode="add", mod_color=0.5,
           color_type="col2", weight1=1.0, weight2=-0.6, size=4.0, mod_specular=0.4, mod_hard=0.25),
        ts((0.8, 0.8, 0.8), "clouds", (0.1, 0.1, 0.1), (0.6, 0.5, 0.4), mode="sub", mod_color=0.4, depth=3,
           size=1.5, mod_specular=0.2, mod_hard=0.2),
        ts((0.5, 0.5, 0.6), "wood", (0.5, 0.3, 0.1), (0.8, 0.6, 0.3), mod_color=0.0, turbulence=0.8,
           mod_specular=1.0, mod_hard=0.0),
        ts((0.4, 0.6, 0.5), "gradient", (0.0, 0.0, 0.2), (1.0, 0.9, 0.6), gradient_type="sphere", texco="normal",
           mode="mul", mod_color=0.0, mod_specular=0.0, mod_hard=0.8),
        ts((0.7, 0.7, 0.7), "voronoi", (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), mod_color=0.3, color_type="int",
           size=1.0, intensity=1.0, **base),
    ]
    for s in sc.shaders:
        s.specular[:] = [0.35, 0.3, 0.25]
        s.hard = 18.0
    meshes = []
    for k in range(6):
        v, t = scenes.uv_sphere((-1.5 + 1.5 * (k % 3), -0.45, -0.6 + 1.3 * (k // 3)), 0.55, rings=16, segments=32)
        meshes.append(scenes.Mesh(v, t, k))
    pv, pt = scenes.ground_plane(20.0, -1.0)
    meshes.append(scenes.Mesh(pv, pt, 6))
    sc.meshes = meshes
    sc.lights = [scenes.point_light((2.0, 4.0, 3.0), 14.0), scenes.point_light((-3.0, 3.0, 1.0), 6.0,
                                                                               color=(0.8, 0.9, 1.0))]
    sc.camera = scenes.camera((0.0, 3.0, 4.5), (0.0, -0.5, 0.0), (0.0, 4.0, 4.5), 96, 72)
    return sc


def texco_view_scene():
    """Textures addressed by the screen position ("window") and by the
    reflected eye direction ("reflect"), on spheres and the plane, with
    AA samples (so the screen positions move inside the pixel)."""
    sc = scenes.config_small(80, 60)
    ts = scenes.texture_shader
    sc.shaders = [
        ts((0.6, 0.6, 0.6), "marble", (0.9, 0.9, 0.85), (0.2, 0.2, 0.3), mod_color=0.8, turbulence=2.0, size=2.0,
           texco="window"),
        ts((0.5, 0.5, 0.6), "musgrave", (0.2, 0.4, 0.1), (0.9, 0.9, 0.7), size=2.5, intensity=0.6, texco="reflect"),
        ts((0.7, 0.7, 0.7), "clouds", (0.1, 0.2, 0.3), (0.9, 0.8, 0.6), mode="mul", mod_color=0.9, depth=3,
           size=1.5, texco="reflect", proj=("z", "x", "y")),
        ts((0.5, 0.6, 0.4), "voronoi", (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), mod_color=0.6, color_type="col1",
           weight1=1.0, size=4.0, texco="window", proj=("y", "x", "n")),
    ]
    meshes = []
    for k in range(3):
        v, t = scenes.uv_sphere((-1.4 + 1.4 * k, -0.4, 0.0), 0.6, rings=16, segments=32)
        meshes.append(scenes.Mesh(v, t, k))
    pv, pt = scenes.ground_plane(20.0, -1.0)
    meshes.append(scenes.Mesh(pv, pt, 3))
    sc.meshes = meshes
    sc.lights = [scenes.point_light((2.0, 4.0, 3.0), 14.0)]
    sc.camera = scenes.camera((0.0, 2.5, 4.5), (0.0, -0.4, 0.0), (0.0, 3.5, 4.5), 80, 60)
    sc.render.spp = 3
    return sc


def sphere_uvs(verts, tris, center):
    """Per-corner (u, v) of a sphere's triangles from each corner's
    longitude and latitude about `center` (seams are not fixed up)."""
    d = verts[tris.reshape(-1)].astype(np.float64) - np.asarray(center, np.float64)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    u = (np.arctan2(d[:, 2], d[:, 0]) / (2 * np.pi)) % 1.0
    v = np.arccos(np.clip(d[:, 1], -1, 1)) / np.pi
    return np.stack([u, v], -1).reshape(-1, 6).astype(np.float32)


def texco_uv_scene():
    """Textures addressed by the triangles' texture coordinates ("uv"): a
    sphere and the plane with coordinates, a smoothed sphere and a flat
    sphere without them (u, v = 0 and -1), each with its own texture."""
    sc = scenes.config_small(80, 60)
    ts = scenes.texture_shader
    sc.shaders = [
        ts((0.6, 0.6, 0.6), "marble", (0.9, 0.9, 0.85), (0.2, 0.2, 0.3), mod_color=0.8, turbulence=1.0, size=3.0,
           texco="uv"),
        ts((0.5, 0.5, 0.6), "voronoi", (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), mod_color=0.7, color_type="col1",
           weight1=1.0, size=3.0, texco="uv"),
        ts((0.7, 0.6, 0.5), "clouds", (0.1, 0.2, 0.3), (0.9, 0.8, 0.6), mode="mul", mod_color=0.9, depth=3,
           size=1.5, texco="uv", proj=("y", "x", "n")),
        ts((0.5, 0.6, 0.4), "musgrave", (0.2, 0.4, 0.1), (0.9, 0.9, 0.7), size=2.0, intensity=0.6, texco="uv"),
    ]
    meshes = []
    for k in range(3):
        c = (-1.4 + 1.4 * k, -0.4, 0.0)
        v, t = scenes.uv_sphere(c, 0.6, rings=16, segments=32)
        m = scenes.Mesh(v, t, k)
        if k == 0:
            m.uvs = sphere_uvs(v, t, c)
        if k == 1:
            m.smooth_angle = 180.0
        meshes.append(m)
    pv, pt = scenes.ground_plane(20.0, -1.0)
    plane = scenes.Mesh(pv, pt, 3)
    plane.uvs = ((pv[pt.reshape(-1)][:, [0, 2]] + 20.0) / 40.0).astype(np.float32).reshape(-1, 6)
    meshes.append(plane)
    sc.meshes = meshes
    sc.lights = [scenes.point_light((2.0, 4.0, 3.0), 14.0)]
    sc.camera = scenes.camera((0.0, 2.5, 4.5), (0.0, -0.4, 0.0), (0.0, 3.5, 4.5), 80, 60)
    sc.render.spp = 2
    return sc


def texco_orco_scene(mats=None):
    """Textures addressed by "orco" on meshes made as the loader makes them
    (through meshObject_t::transform, so orco = backOrco * P: the mesh's
    bound mapped onto [-1, 1]^3), one of them smoothed, beside a mesh made
    without a transform (orco = P).  `mats`: {mesh index: backOrco} from
    the reference; None = placeholders (the reference computes its own)."""
    sc = scenes.config_small(80, 60)
    ts = scenes.texture_shader
    sc.shaders = [
        ts((0.6, 0.6, 0.6), "marble", (0.9, 0.9, 0.85), (0.2, 0.2, 0.3), mod_color=0.8, turbulence=1.0, size=2.0,
           texco="orco"),
        ts((0.5, 0.5, 0.6), "voronoi", (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), mod_color=0.7, color_type="col1",
           weight1=1.0, size=1.5, texco="orco"),
        ts((0.7, 0.6, 0.5), "clouds", (0.1, 0.2, 0.3), (0.9, 0.8, 0.6), mode="mul", mod_color=0.9, depth=3,
           size=1.0, texco="orco", proj=("y", "x", "n")),
        ts((0.5, 0.6, 0.4), "musgrave", (0.2, 0.4, 0.1), (0.9, 0.9, 0.7), size=1.0, intensity=0.6, texco="orco"),
    ]
    meshes = []
    for k in range(3):
        c = (-1.4 + 1.4 * k, -0.4 + 0.1 * k, 0.2 * k)
        v, t = scenes.uv_sphere(c, 0.6 - 0.1 * k, rings=16, segments=32)
        m = scenes.Mesh(v, t, k)
        if k == 1:
            m.smooth_angle = 180.0
        if k != 2:  # the third sphere is made without a transform
            m.orco = np.eye(4, dtype=np.float32)
        meshes.append(m)
    pv, pt = scenes.ground_plane(20.0, -1.0)
    plane = scenes.Mesh(pv, pt, 3)
    plane.orco = np.eye(4, dtype=np.float32)
    meshes.append(plane)
    sc.meshes = meshes
    sc.lights = [scenes.point_light((2.0, 4.0, 3.0), 14.0)]
    sc.camera = scenes.camera((0.0, 2.5, 4.5), (0.0, -0.4, 0.0), (0.0, 3.5, 4.5), 80, 60)
    sc.render.spp = 2
    if mats is not None:
        for i, m in mats.items():
            sc.meshes[int(i)].orco = np.asarray(m, np.float32)
    return sc


def texco_orco_render():
    sc = texco_orco_scene()
    mats = T.harness_orco_matrices(sc)
    img, _ = T.harness_render(sc)
    idx = np.array(sorted(mats))
    np.savez_compressed(os.path.join(HERE, "render_texco_orco_80x60.npz"), image=img, orco_idx=idx,
                        orco=np.stack([mats[i] for i in idx]))


def texco_uv_render():
    img, _ = T.harness_render(texco_uv_scene())
    np.savez_compressed(os.path.join(HERE, "render_texco_uv_80x60.npz"), image=img)


def texco_view_render():
    img, _ = T.harness_render(texco_view_scene())
    np.savez_compressed(os.path.join(HERE, "render_texco_view_80x60.npz"), image=img)


def specmod_render():
    img, _ = T.harness_render(specmod_scene())
    np.savez_compressed(os.path.join(HERE, "render_specmod_96x72.npz"), image=img)


def tonemap_configs():
    """The render block's tone mapping variants: clamp_rgb, exposure, gamma,
    both, and gamma with alpha premultiply, on a constant background."""
    return [dict(tonemap=True, clamp_rgb=True), dict(tonemap=True, exposure=1.5), dict(tonemap=True, gamma=2.2),
            dict(tonemap=True, exposure=0.7, gamma=1.8), dict(tonemap=True, gamma=2.0, alpha_premultiply=True)]


def tonemap_scene(cfg):
    sc = smooth_scene()
    sc.render = scenes.render_params(spp=3, background=(0.2, 0.3, 0.9), **cfg)
    sc.camera = scenes.camera((0, 1.5, 4.5), (0, -0.3, 0), (0, 2.5, 4.5), 48, 36, fov_deg=70)
    return sc


def tonemap_renders():
    imgs = [T.harness_render(tonemap_scene(c))[0] for c in tonemap_configs()]
    np.savez_compressed(os.path.join(HERE, "render_tonemap_48x36.npz"), images=np.stack(imgs))


def sample_images():
    rng = np.random.default_rng(2)
    a = rng.uniform(-0.2, 1.3, (17, 23, 4)).astype(np.float32)
    b = np.zeros((6, 300, 4), np.float32)
    b[:, 40:200] = (0.5, 0.25, 2.0, 1.0)
    b[2:4] = rng.uniform(0, 100, (2, 300, 4))
    c = rng.uniform(0, 5, (9, 5, 4)).astype(np.float32)
    d = np.exp(rng.normal(0, 4, (8, 64, 4))).astype(np.float32)
    return [a, b, c, d]


def image_outputs():
    """The reference's outTga_t (with and without alpha) and outHDR_t bytes
    for a few float images (out-of-range values, runs, a row too narrow to
    run-length encode, a wide dynamic range)."""
    out = {}
    with tempfile.TemporaryDirectory() as dd:
        for i, im in enumerate(sample_images()):
            ip = os.path.join(dd, "i.bin")
            with open(ip, "wb") as f:
                f.write(struct.pack("<2I", im.shape[1], im.shape[0]))
                f.write(np.ascontiguousarray(im).tobytes())
            out[f"img{i}"] = im
            for kind in ("tga", "tga_alpha", "hdr"):
                op = os.path.join(dd, "o.bin")
                T.run_harness("imgout", kind, ip, op)
                out[f"img{i}_{kind}"] = np.frombuffer(open(op, "rb").read(), np.uint8)
    np.savez_compressed(os.path.join(HERE, "image_outputs.npz"), **out)


def instance_scene():
    """References (referenceObject_t): a smoothed torus and a smoothed,
    orco-textured sphere, each placed twice by rotation, non-uniform scale and
    translation (the originals moved off to the side), over a plane."""
    sc = scenes.config_small(96, 72)
    tv, tt = scenes.torus((0.0, 0.0, 0.0), 0.6, 0.25, nu=24, nv=12)
    sv, st = scenes.uv_sphere((0.0, 0.0, 0.0), 0.5, rings=10, segments=20)
    pv, pt = scenes.ground_plane(20.0, -1.0)
    sc.shaders = [scenes.shader((0.8, 0.6, 0.5), (0.4, 0.4, 0.4), hard=20.0),
                  scenes.texture_shader((0.5, 0.5, 0.5), "marble", (0.9, 0.9, 0.8), (0.2, 0.3, 0.5), texco="orco",
                                        turbulence=2.0, size=2.0, mod_color=0.9),
                  scenes.shader((0.8, 0.8, 0.8))]
    sc.meshes = [scenes.Mesh(tv + np.float32([5.0, 0.0, 0.0]), tt, 0, smooth_angle=40.0),
                 scenes.Mesh(sv, st, 1, smooth_angle=180.0), scenes.Mesh(pv, pt, 2),
                 scenes.instance(0, scenes.transform((-6.4, -0.4, 0.3), (30, 0, 10), (1.0, 1.0, 1.0))),
                 scenes.instance(0, scenes.transform((-3.7, 0.1, -0.5), (70, 20, 0), (1.2, 0.7, 1.0))),
                 scenes.instance(1, scenes.transform((0.2, 0.8, -1.2), (0, 45, 0), (1.5, 0.6, 1.5))),
                 scenes.instance(1, scenes.transform((-0.3, -0.6, 1.2), (10, 0, 0), (0.5, 0.5, 0.5)))]
    sc.lights = [scenes.point_light((2.0, 4.0, 3.0), 14.0)]
    sc.camera = scenes.camera((0.0, 1.5, 4.5), (0.0, -0.2, 0.0), (0.0, 2.5, 4.5), 96, 72, fov_deg=60)
    return sc


def instance_rays(n=2000, seed=4):
    rng = np.random.default_rng(seed)
    frm = rng.uniform(-2.5, 2.5, (n, 3)).astype(np.float32)
    frm[:, 1] = rng.uniform(-0.9, 2.0, n)
    tgt = rng.uniform(-2, 2, (n, 3)).astype(np.float32)
    tgt[:, 1] = rng.uniform(-1.2, 1.2, n)
    d = tgt - frm
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    own = rng.integers(0, 7, n)
    return frm, d.astype(np.float32), tgt, own


def instances():
    """The reference's M^-1 of each reference, its object tree (the placed
    boxes), closest and shadow answers through the references, and a render."""
    sc = instance_scene()
    inv = T.harness_instance_inverses(sc)
    _, ot = T.harness_trees(sc)
    frm, d, tgt, own = instance_rays()
    recs = np.zeros(len(frm), T.RAY_REC)
    recs["mode"], recs["frm"], recs["dir"], recs["dist"] = 2, frm, d, -1
    closest = T.harness_rays(sc, recs)
    recs3 = np.zeros(len(frm), T.RAY_REC)
    recs3["mode"], recs3["frm"], recs3["object"], recs3["l"] = 3, frm, own, tgt
    shadow = T.harness_rays(sc, recs3)[:, 0]
    img, _ = T.harness_render(sc)
    np.savez_compressed(os.path.join(HERE, "instances.npz"), inv_idx=np.array(sorted(inv)),
                        inv=np.stack([inv[i] for i in sorted(inv)]), otree=ot, closest=closest, shadow=shadow,
                        image=img)


def halton_noise():
    with tempfile.TemporaryDirectory() as d:
        hp = os.path.join(d, "h.bin")
        T.run_harness("halton", hp)
        raw = np.fromfile(hp, np.float32)
        hal = raw[: 12 * 4096].reshape(12, 4096)
        ri = raw[12 * 4096:].reshape(4096, 3)
        rng = np.random.default_rng(5)
        pts = np.concatenate([rng.uniform(-300, 300, (2048, 3)), rng.uniform(-4, 4, (2048, 3))]).astype(np.float32)
        pp, op = os.path.join(d, "p.bin"), os.path.join(d, "n.bin")
        with open(pp, "wb") as f:
            f.write(struct.pack("<I", pts.shape[0]))
            f.write(pts.tobytes())
        T.run_harness("noise", pp, op)
        noise = np.fromfile(op, np.float32).reshape(-1, 5)
    np.savez_compressed(os.path.join(HERE, "qmc_noise.npz"), halton=hal, ri=ri, pts=pts, noise=noise)


if __name__ == "__main__":
    assert T.has_harness(), "build the reference first: make -C oracle"
    trees()
    tie_trees()
    rays()
    camera_and_render()
    smooth_render()
    textures()
    texture_render()
    specmod_render()
    texco_view_render()
    texco_uv_render()
    texco_orco_render()
    tonemap_renders()
    image_outputs()
    instances()
    illum()
    illum_guess()
    illum_rounds()
    halton_noise()
    for f in sorted(os.listdir(HERE)):
        print(f, os.path.getsize(os.path.join(HERE, f)))
