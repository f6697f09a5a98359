"""Seeded synthetic scenes with the shapes of the benchmark configurations.

A scene is what a YafRay host would hand to the C ABI: meshes (object list),
genericShader_t parameters, light plugin parameters, the camera and render
settings.  ``write_yrs`` stores it in the "YRS1" layout of include/yr.h.

Configurations (sizes as in the benchmark definitions):
  * ``config_small``   UV sphere (64 rings x 128 segments) on a 2-triangle
                       ground plane, point light, 320x240, 1 spp, no GI.
  * ``config_large``   16x16 jittered grid of those spheres on a 40x40 plane,
                       4 area lights (16 samples), 1920x1080, 16 spp, path GI
                       with 2 bounces.
  * ``config_batch``   256 independent scenes (spheres + tori), uneven sizes.
  * ``config_diff``    the small scene at 512x512 / 64 spp with 64 material
                       groups and 8 area lights (264 parameters).
  * ``config_diffnoise`` 32 inverse problems with fBm-modulated albedo.

UV sphere construction (pinned, the benchmark text leaves it open): 64
latitude bands and 128 segments; the two polar bands are triangle fans, the
62 inner bands are quads split in two, which gives 128 + 128 + 62*256 =
16,128 non-degenerate triangles and 63*128 + 2 = 8,066 vertices.
"""
from __future__ import annotations

import math
import struct
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import abi


# --------------------------------------------------------------------- meshes
def uv_sphere(center=(0.0, 0.0, 0.0), radius=1.0, rings=64, segments=128):
    """Vertices (float32 [V,3]) and triangles (uint32 [T,3]) of a UV sphere."""
    cx, cy, cz = center
    k = np.arange(1, rings, dtype=np.float64)
    th = np.pi * k / rings
    ph = 2.0 * np.pi * np.arange(segments, dtype=np.float64) / segments
    y = np.cos(th)[:, None] * np.ones_like(ph)[None, :]
    rr = np.sin(th)[:, None]
    ring_v = np.stack([cx + radius * rr * np.cos(ph)[None, :], cy + radius * y,
                       cz + radius * rr * np.sin(ph)[None, :]], -1).reshape(-1, 3)
    verts = np.concatenate([[[cx, cy + radius, cz]], ring_v, [[cx, cy - radius, cz]]])
    south = verts.shape[0] - 1
    s = np.arange(segments)
    s1 = (s + 1) % segments

    def ring(kk, ss):  # kk in 1..rings-1
        return 1 + (kk - 1) * segments + ss

    north = np.stack([np.zeros(segments, np.int64), ring(1, s1), ring(1, s)], -1)
    kk = np.arange(1, rings - 1)[:, None]
    a, b = ring(kk, s[None, :]), ring(kk, s1[None, :])
    c, d = ring(kk + 1, s[None, :]), ring(kk + 1, s1[None, :])
    band = np.stack([np.stack([a, b, d], -1), np.stack([a, d, c], -1)], 2).reshape(-1, 3)
    southf = np.stack([np.full(segments, south), ring(rings - 1, s), ring(rings - 1, s1)], -1)
    tris = np.concatenate([north, band, southf])
    return verts.astype(np.float32), tris.astype(np.uint32)


def torus(center, R, r, nu=64, nv=32):
    cx, cy, cz = center
    verts = []
    for i in range(nu):
        u = 2 * math.pi * i / nu
        for j in range(nv):
            v = 2 * math.pi * j / nv
            x = (R + r * math.cos(v)) * math.cos(u)
            z = (R + r * math.cos(v)) * math.sin(u)
            y = r * math.sin(v)
            verts.append((cx + x, cy + y, cz + z))
    tris = []
    for i in range(nu):
        for j in range(nv):
            a = i * nv + j
            b = ((i + 1) % nu) * nv + j
            c = i * nv + (j + 1) % nv
            d = ((i + 1) % nu) * nv + (j + 1) % nv
            tris.append((a, c, d))
            tris.append((a, d, b))
    return np.asarray(verts, dtype=np.float32), np.asarray(tris, dtype=np.uint32)


def ground_plane(half=20.0, y=-1.0):
    v = np.array([(-half, y, -half), (half, y, -half), (half, y, half), (-half, y, half)], dtype=np.float32)
    t = np.array([(0, 2, 1), (0, 3, 2)], dtype=np.uint32)
    return v, t


# ---------------------------------------------------------------------- scene
@dataclass
class Mesh:
    verts: np.ndarray
    tris: np.ndarray
    shader: int = 0
    tri_shaders: Optional[np.ndarray] = None
    cast_shadows: bool = True
    smooth_angle: float = 0.0   # meshObject_t::autoSmooth angle (degrees); < 1 = flat
    instance_of: int = -1       # >= 0: a referenceObject_t of that mesh, placed by `matrix`
    matrix: Optional[np.ndarray] = None   # 4x4 row-major (instances only)
    inverse: Optional[np.ndarray] = None  # optional M^-1 (else computed by the library)
    uvs: Optional[np.ndarray] = None      # optional (ntris, 6) texture coordinates (u, v at a, b, c)
    orco: Optional[np.ndarray] = None     # optional 4x4 "orco" matrix (meshObject_t::backOrco)

    @property
    def is_instance(self) -> bool:
        return self.instance_of >= 0


def instance(original: int, matrix, inverse=None) -> "Mesh":
    """A reference to mesh `original` placed by the 4x4 row-major `matrix`
    (the loader's object with an "original" attribute, render.cc:650-680);
    `inverse`: optional M^-1 as the caller computed it."""
    m = np.ascontiguousarray(np.asarray(matrix, np.float32).reshape(4, 4))
    inv = None if inverse is None else np.ascontiguousarray(np.asarray(inverse, np.float32).reshape(4, 4))
    return Mesh(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.uint32), 0, instance_of=int(original), matrix=m,
                inverse=inv)


def transform(translate=(0.0, 0.0, 0.0), rotate_deg=(0.0, 0.0, 0.0), scale=(1.0, 1.0, 1.0)) -> np.ndarray:
    """A 4x4 row-major matrix: scale, then rotations about x, y and z, then
    the translation."""
    s = np.diag([*scale, 1.0])
    rx, ry, rz = (np.radians(a) for a in rotate_deg)
    Rx = np.array([[1, 0, 0, 0], [0, np.cos(rx), -np.sin(rx), 0], [0, np.sin(rx), np.cos(rx), 0], [0, 0, 0, 1]])
    Ry = np.array([[np.cos(ry), 0, np.sin(ry), 0], [0, 1, 0, 0], [-np.sin(ry), 0, np.cos(ry), 0], [0, 0, 0, 1]])
    Rz = np.array([[np.cos(rz), -np.sin(rz), 0, 0], [np.sin(rz), np.cos(rz), 0, 0], [0, 0, 1, 0], [0, 0, 0, 1]])
    t = np.eye(4)
    t[:3, 3] = translate
    return (t @ Rz @ Ry @ Rx @ s).astype(np.float32)


@dataclass
class Scene:
    meshes: List[Mesh] = field(default_factory=list)
    shaders: List[abi.YrShaderDesc] = field(default_factory=list)
    lights: List[abi.YrLightDesc] = field(default_factory=list)
    camera: abi.YrCameraDesc = field(default_factory=abi.YrCameraDesc)
    render: abi.YrRenderParams = field(default_factory=abi.YrRenderParams)
    name: str = ""

    @property
    def ntris(self) -> int:
        return int(sum(m.tris.shape[0] for m in self.meshes))

    @property
    def resx(self) -> int:
        return int(self.camera.resx)

    @property
    def resy(self) -> int:
        return int(self.camera.resy)


def shader(color, specular=(0.0, 0.0, 0.0), hard=1.0) -> abi.YrShaderDesc:
    s = abi.YrShaderDesc()
    s.color[:] = [float(c) for c in color]
    s.specular[:] = [float(c) for c in specular]
    s.hard = float(hard)
    s.tex_type = abi.YR_TEX_NONE
    s.mod_size[:] = [1.0, 1.0, 1.0]
    return s


def tex_map(texco="global", proj=("x", "y", "z")) -> int:
    """yr_shader_desc.tex_map from the modulator's "texco" and "proj_x/y/z"
    parameters ("global" / "orco" / "normal" / "window" / "reflect" / "uv"; axes
    "x" "y" "z" or "n")."""
    tc = {"global": abi.YR_TEXCO_GLOBAL, "orco": abi.YR_TEXCO_ORCO, "normal": abi.YR_TEXCO_NORMAL,
          "window": abi.YR_TEXCO_WINDOW, "reflect": abi.YR_TEXCO_REFLECT, "uv": abi.YR_TEXCO_UV}[texco]
    pc = {"x": abi.YR_PROJ_X, "y": abi.YR_PROJ_Y, "z": abi.YR_PROJ_Z, "n": abi.YR_PROJ_NONE}
    return tc | (pc[proj[0]] << 8) | (pc[proj[1]] << 16) | (pc[proj[2]] << 24)


def fbm_shader(color, color1, color2, intensity, size, octaves=6.0, lacunarity=2.0, H=1.0,
               mod_color=1.0, texco="global", proj=("x", "y", "z")) -> abi.YrShaderDesc:
    """genericShader_t whose albedo is mixed with a musgrave fBm texture."""
    s = shader(color)
    s.tex_type = abi.YR_TEX_MUSGRAVE_FBM
    s.tex_color1[:] = [float(c) for c in color1]
    s.tex_color2[:] = [float(c) for c in color2]
    s.tex_H = float(H)
    s.tex_lacunarity = float(lacunarity)
    s.tex_octaves = float(octaves)
    s.tex_size = float(size)
    s.tex_intensity = float(intensity)
    s.mod_color = float(mod_color)
    s.tex_noise = 0
    s.tex_map = tex_map(texco, proj)
    return s


# Procedural textures: the parameters of each factory with its defaults
# (basictex.cc: clouds :94-104, marble :155-175, wood :222-249, voronoi
# :619-650, musgrave :683-709, distorted_noise :731-746, gradient :805-815).
_TEX_DEFAULTS = {
    "clouds": dict(depth=2, size=1.0, hard=False, bias="", noise_type="newperlin"),
    "marble": dict(depth=2, turbulence=1.0, sharpness=1.0, size=1.0, hard=False, shape="sin",
                   noise_type="newperlin"),
    "wood": dict(depth=2, turbulence=1.0, size=1.0, hard=False, wood_type="bands", shape="sin",
                 noise_type="newperlin"),
    "voronoi": dict(color_type="int", weight1=1.0, weight2=0.0, weight3=0.0, weight4=0.0, mk_exponent=2.5,
                    intensity=1.0, size=1.0, distance_metric="real"),
    "musgrave": dict(type="fBm", noise_type="newperlin", H=1.0, lacunarity=2.0, octaves=2.0, offset=1.0,
                     gain=1.0, size=1.0, intensity=1.0),
    "distorted_noise": dict(noise_type1="newperlin", noise_type2="newperlin", distort=1.0, size=1.0),
    "gradient": dict(gradient_type="linear", flip_xy=False),
}
_MUSGRAVE_TYPES = {"fBm": abi.YR_TEX_MUSGRAVE_FBM, "multifractal": abi.YR_TEX_MUSGRAVE_MULTIFRACTAL,
                   "heteroterrain": abi.YR_TEX_MUSGRAVE_HETEROTERRAIN, "hybridmf": abi.YR_TEX_MUSGRAVE_HYBRIDMF,
                   "ridgedmf": abi.YR_TEX_MUSGRAVE_RIDGEDMF}


def texture_shader(color, kind, color1=(0.0, 0.0, 0.0), color2=(1.0, 1.0, 1.0), mod_color=1.0, mode="mix",
                   texco="global", proj=("x", "y", "z"), mod_specular=0.0, mod_hard=0.0,
                   **params) -> abi.YrShaderDesc:
    """genericShader_t whose diffuse colour is modulated by one procedural
    texture `kind` ("clouds", "marble", "wood", "voronoi", "musgrave",
    "distorted_noise", "gradient") with the factory's parameter names and
    defaults; unknown parameter names raise.  mod_specular / mod_hard: the
    modulator's "specular" and "hard" weights (the texture also modulates
    the specular colour and the Phong exponent)."""
    p = dict(_TEX_DEFAULTS[kind])
    for k in params:
        if k not in p:
            raise KeyError(f"{kind} has no parameter {k!r}")
    p.update(params)
    s = shader(color)
    s.tex_color1[:] = [float(c) for c in color1]
    s.tex_color2[:] = [float(c) for c in color2]
    s.mod_color = float(mod_color)
    s.mod_specular = float(mod_specular)
    s.mod_hard = float(mod_hard)
    s.mod_mode = abi.MOD_MODES[mode]
    s.tex_map = tex_map(texco, proj)
    nt = lambda name: abi.NOISE_TYPES.get(name, 0)  # newNoise: unknown names give newperlin
    if kind == "clouds":
        s.tex_type = abi.YR_TEX_CLOUDS
        s.tex_depth, s.tex_size, s.tex_hard = int(p["depth"]), float(p["size"]), int(bool(p["hard"]))
        s.tex_variant = {"positive": 1, "negative": 2}.get(p["bias"], 0)
        s.tex_noise = nt(p["noise_type"])
    elif kind in ("marble", "wood"):
        s.tex_type = abi.YR_TEX_MARBLE if kind == "marble" else abi.YR_TEX_WOOD
        s.tex_depth, s.tex_size, s.tex_hard = int(p["depth"]), float(p["size"]), int(bool(p["hard"]))
        s.tex_turbulence = float(p["turbulence"])
        s.tex_shape = abi.WAVE_SHAPES.get(p["shape"], 0)
        s.tex_noise = nt(p["noise_type"])
        if kind == "marble":
            s.tex_sharpness = float(p["sharpness"])
        else:
            s.tex_variant = 1 if p["wood_type"] == "rings" else 0
    elif kind == "voronoi":
        s.tex_type = abi.YR_TEX_VORONOI
        s.tex_shape = {"col1": 1, "col2": 2, "col3": 3}.get(p["color_type"], 0)
        s.tex_weights[:] = [float(p[f"weight{i}"]) for i in range(1, 5)]
        s.tex_mk_exponent = float(p["mk_exponent"])
        s.tex_intensity = float(p["intensity"])
        s.tex_size = float(p["size"])
        s.tex_metric = abi.DIST_METRICS.get(p["distance_metric"], 0)
    elif kind == "musgrave":
        s.tex_type = _MUSGRAVE_TYPES.get(p["type"], abi.YR_TEX_MUSGRAVE_FBM)
        s.tex_noise = nt(p["noise_type"])
        s.tex_H, s.tex_lacunarity, s.tex_octaves = float(p["H"]), float(p["lacunarity"]), float(p["octaves"])
        s.tex_offset, s.tex_gain = float(p["offset"]), float(p["gain"])
        s.tex_size, s.tex_intensity = float(p["size"]), float(p["intensity"])
    elif kind == "distorted_noise":
        s.tex_type = abi.YR_TEX_DISTORTED_NOISE
        s.tex_noise, s.tex_noise2 = nt(p["noise_type1"]), nt(p["noise_type2"])
        s.tex_distort, s.tex_size = float(p["distort"]), float(p["size"])
    elif kind == "gradient":
        s.tex_type = abi.YR_TEX_GRADIENT
        s.tex_shape = abi.GRADIENT_TYPES.get(p["gradient_type"], 0)
        s.tex_variant = int(bool(p["flip_xy"]))
    else:
        raise KeyError(kind)
    return s


def point_light(pos, power=1.0, color=(1.0, 1.0, 1.0), cast_shadows=True) -> abi.YrLightDesc:
    l = abi.YrLightDesc()
    l.type = abi.YR_LIGHT_POINT
    l.color[:] = [float(c) for c in color]
    l.power = float(power)
    l.p[0][:] = [float(c) for c in pos]
    l.cast_shadows = 1 if cast_shadows else 0
    return l


def area_light(a, b, c, d, power=1.0, samples=16, color=(1.0, 1.0, 1.0), psamples=0) -> abi.YrLightDesc:
    """areaLight_t: corners a, b, c, d; `psamples` probes of the penumbra
    guess (0 = off, the factory's default)."""
    l = abi.YrLightDesc()
    l.type = abi.YR_LIGHT_AREA
    l.color[:] = [float(x) for x in color]
    l.power = float(power)
    for i, p in enumerate((a, b, c, d)):
        l.p[i][:] = [float(x) for x in p]
    l.samples = int(samples)
    l.cast_shadows = 1
    l.psamples = int(psamples)
    return l


def quad_light_down(cx, y, cz, w, h, power, samples=16, color=(1.0, 1.0, 1.0), psamples=0) -> abi.YrLightDesc:
    """Horizontal quad at height y facing down ((b-a)x(d-a) points to -y)."""
    a = (cx - w / 2, y, cz - h / 2)
    b = (cx + w / 2, y, cz - h / 2)
    c = (cx + w / 2, y, cz + h / 2)
    d = (cx - w / 2, y, cz + h / 2)
    return area_light(a, b, c, d, power, samples, color, psamples)


def hemi_light(samples=16, power=1.0, color=(1.0, 1.0, 1.0), maxdist=-1.0) -> abi.YrLightDesc:
    l = abi.YrLightDesc()
    l.type = abi.YR_LIGHT_HEMI
    l.color[:] = [float(x) for x in color]
    l.power = float(power)
    l.samples = int(samples)
    l.maxdist = float(maxdist)
    return l


def path_light(samples=1, depth=2, power=1.0, threshold=0.0) -> abi.YrLightDesc:
    """pathLight_t with use_QMC; `threshold` > 0 turns the adaptive extra
    rounds of paths on (the factory's default is 0.1), 0 = one round."""
    l = abi.YrLightDesc()
    l.type = abi.YR_LIGHT_PATH
    l.color[:] = [1.0, 1.0, 1.0]
    l.power = float(power)
    l.samples = int(samples)
    l.depth = int(depth)
    l.threshold = float(threshold)
    return l


def camera(pos, look, up, resx, resy, fov_deg=45.0, aspect=1.0) -> abi.YrCameraDesc:
    """Pinhole camera; focal = 0.5 / tan(fov/2) because camera_t puts a
    width-1 image plane at distance `focal` (camera.cc:53-60)."""
    c = abi.YrCameraDesc()
    c.pos[:] = [float(x) for x in pos]
    c.look[:] = [float(x) for x in look]
    c.up[:] = [float(x) for x in up]
    c.resx, c.resy = int(resx), int(resy)
    c.aspect = float(aspect)
    c.focal = float(0.5 / math.tan(math.radians(fov_deg) / 2.0))
    return c


def render_params(spp=1, seed=0, bias=0.1, raydepth=3, pixelwidth=1.0, background=(0.0, 0.0, 0.0),
                  exposure=0.0, gamma=1.0, tonemap=False, clamp_rgb=False, alpha_premultiply=False):
    """The render block's parameters (loader/render.cc:1025-1225); `tonemap`
    is what the loader sets for TGA output (exposure / gamma / clamp_rgb per
    camera sample), off for HDR / EXR."""
    r = abi.YrRenderParams()
    r.self_bias = float(bias)
    r.raydepth = int(raydepth)
    r.spp = int(spp)
    r.aa_pixelwidth = float(pixelwidth)
    r.seed = int(seed) & 0xFFFFFFFF
    r.background[:] = [float(x) for x in background]
    r.flags = ((abi.YR_RENDER_TONEMAP if tonemap else 0) | (abi.YR_RENDER_CLAMP_RGB if clamp_rgb else 0) |
               (abi.YR_RENDER_ALPHA_PREMULTIPLY if alpha_premultiply else 0))
    r.exposure = float(exposure)
    r.gamma = float(gamma)
    return r


# -------------------------------------------------------------- configurations
def config_small(resx=320, resy=240) -> Scene:
    """UV sphere r=1 at the origin on a 2-triangle plane at y=-1; point light
    (3,5,2) power 1; albedo 0.8; camera at (0,1,5) looking at the origin."""
    sv, st = uv_sphere()
    pv, pt = ground_plane(half=20.0, y=-1.0)
    sc = Scene(name=f"small_{resx}x{resy}")
    sc.shaders = [shader((0.8, 0.8, 0.8))]
    sc.meshes = [Mesh(sv, st, 0), Mesh(pv, pt, 0)]
    sc.lights = [point_light((3.0, 5.0, 2.0), 1.0)]
    sc.camera = camera((0, 1, 5), (0, 0, 0), (0, 2, 5), resx, resy)
    sc.render = render_params(spp=1)
    return sc


def config_large(seed=1, resx=1920, resy=1080, spp=16, grid=16) -> Scene:
    """grid x grid jittered spheres (radius U(0.3,0.5), centre jitter
    U(-0.2,0.2)) on a 40x40 plane, four area lights (power U(1,5), 16
    samples), path GI with 2 bounces, albedos U(0.2,0.9)."""
    rng = np.random.default_rng(seed)
    sc = Scene(name=f"large_g{grid}_{resx}x{resy}_spp{spp}")
    spacing = 2.0
    off = (grid - 1) / 2.0
    sc.shaders.append(shader(tuple(rng.uniform(0.2, 0.9, 3))))
    pv, pt = ground_plane(half=20.0, y=-1.0)
    sc.meshes.append(Mesh(pv, pt, 0))
    for i in range(grid):
        for k in range(grid):
            r = float(rng.uniform(0.3, 0.5))
            jx, jz = rng.uniform(-0.2, 0.2, 2)
            c = ((i - off) * spacing + jx, -1.0 + r, (k - off) * spacing + jz)
            v, t = uv_sphere(c, r)
            sc.shaders.append(shader(tuple(rng.uniform(0.2, 0.9, 3))))
            sc.meshes.append(Mesh(v, t, len(sc.shaders) - 1))
    for lx, lz in ((-8.0, -8.0), (8.0, -8.0), (-8.0, 8.0), (8.0, 8.0)):
        sc.lights.append(quad_light_down(lx, 12.0, lz, 4.0, 4.0, float(rng.uniform(1.0, 5.0)) * 30.0, 16))
    sc.lights.append(path_light(samples=1, depth=2, power=1.0))
    sc.camera = camera((0.0, 14.0, 26.0), (0.0, -1.0, 0.0), (0.0, 15.0, 26.0), resx, resy)
    sc.render = render_params(spp=spp, seed=seed)
    return sc


def _random_object(rng, tri_budget):
    """A sphere or a torus with roughly tri_budget triangles."""
    if rng.random() < 0.6:
        seg = max(8, int(math.sqrt(tri_budget)))
        rings = max(4, seg // 2)
        seg = max(8, tri_budget // (2 * rings))
        return "sphere", rings, seg
    nu = max(8, int(math.sqrt(tri_budget)))
    nv = max(4, tri_budget // (2 * nu))
    return "torus", nu, nv


def config_batch_scene(rng, idx, tri_lo=1_000, tri_hi=200_000) -> Scene:
    ntri = int(math.exp(rng.uniform(math.log(tri_lo), math.log(tri_hi))))
    nobj = int(rng.integers(1, 33))
    size = int(rng.choice([64, 128, 256, 512]))
    spp = int(rng.integers(4, 65))
    bounces = int(rng.integers(1, 4))
    sc = Scene(name=f"batch{idx}_t{ntri}_o{nobj}_{size}_spp{spp}_b{bounces}")
    pv, pt = ground_plane(half=20.0, y=-1.0)
    sc.shaders.append(shader(tuple(rng.uniform(0.2, 0.9, 3))))
    sc.meshes.append(Mesh(pv, pt, 0))
    per = max(64, ntri // nobj)
    for o in range(nobj):
        kind, a, b = _random_object(rng, per)
        c = (float(rng.uniform(-4, 4)), float(rng.uniform(-0.5, 1.5)), float(rng.uniform(-4, 4)))
        if kind == "sphere":
            v, t = uv_sphere(c, float(rng.uniform(0.3, 1.0)), rings=a, segments=b)
        else:
            v, t = torus(c, float(rng.uniform(0.5, 1.0)), float(rng.uniform(0.1, 0.3)), nu=a, nv=b)
        sc.shaders.append(shader(tuple(rng.uniform(0.2, 0.9, 3))))
        sc.meshes.append(Mesh(v, t, len(sc.shaders) - 1))
    for _ in range(int(rng.integers(1, 5))):
        if rng.random() < 0.5:
            sc.lights.append(point_light((rng.uniform(-6, 6), rng.uniform(6, 10), rng.uniform(-6, 6)),
                                         float(rng.uniform(20, 60))))
        else:
            sc.lights.append(quad_light_down(float(rng.uniform(-5, 5)), float(rng.uniform(7, 10)),
                                             float(rng.uniform(-5, 5)), 2.0, 2.0, float(rng.uniform(20, 60)),
                                             int(rng.choice([4, 9, 16]))))
    sc.lights.append(path_light(samples=1, depth=bounces, power=1.0))
    sc.camera = camera((0.0, 5.0, 12.0), (0.0, 0.0, 0.0), (0.0, 6.0, 12.0), size, size)
    sc.render = render_params(spp=spp, seed=idx + 1)
    return sc


def config_batch(seed=3, count=256, **kw) -> List[Scene]:
    rng = np.random.default_rng(seed)
    return [config_batch_scene(rng, i, **kw) for i in range(count)]


def config_diff(seed=4, res=512, spp=64, groups=64, nlights=8, hidden=False) -> Scene:
    """The small scene at res^2 with `groups` material groups on the sphere
    (triangles assigned round-robin by latitude band), diffuse U(0.2,0.9),
    specular weight U(0,0.5), and `nlights` area lights power U(1,5)."""
    rng = np.random.default_rng(seed + (1000 if hidden else 0))
    sv, st = uv_sphere()
    pv, pt = ground_plane(half=20.0, y=-1.0)
    sc = Scene(name=f"diff_{res}_spp{spp}")
    for g in range(groups):
        spec = float(rng.uniform(0.0, 0.5))
        sc.shaders.append(shader(tuple(rng.uniform(0.2, 0.9, 3)), (spec, spec, spec), hard=20.0))
    band = np.arange(st.shape[0]) // 256
    tri_sh = (band % groups).astype(np.uint32)
    sc.meshes = [Mesh(sv, st, abi.YR_PER_TRIANGLE, tri_sh), Mesh(pv, pt, 0)]
    for i in range(nlights):
        ang = 2 * math.pi * i / nlights
        sc.lights.append(quad_light_down(4.0 * math.cos(ang), 6.0, 4.0 * math.sin(ang), 1.5, 1.5,
                                         float(rng.uniform(1.0, 5.0)) * 10.0, 4))
    sc.camera = camera((0, 1, 5), (0, 0, 0), (0, 2, 5), res, res)
    sc.render = render_params(spp=spp, seed=seed)
    return sc


def config_diffnoise_scene(rng, idx, res=256, spp=32, tri_lo=20_000, tri_hi=500_000) -> Scene:
    ntri = int(math.exp(rng.uniform(math.log(tri_lo), math.log(tri_hi))))
    seg = max(16, int(math.sqrt(ntri)))
    rings = max(8, ntri // (2 * seg))
    sv, st = uv_sphere((0.0, 0.0, 0.0), 1.0, rings=rings, segments=seg)
    pv, pt = ground_plane(half=20.0, y=-1.0)
    sc = Scene(name=f"diffnoise{idx}_t{st.shape[0]}")
    sc.shaders.append(fbm_shader(tuple(rng.uniform(0.2, 0.9, 3)), tuple(rng.uniform(0.2, 0.9, 3)),
                                 (1.0, 1.0, 1.0), float(rng.uniform(0.3, 1.0)), float(rng.uniform(1, 8))))
    sc.shaders.append(shader((0.8, 0.8, 0.8)))
    sc.meshes = [Mesh(sv, st, 0), Mesh(pv, pt, 1)]
    sc.lights = [quad_light_down(2.0, 6.0, 2.0, 2.0, 2.0, 40.0, 4)]
    sc.camera = camera((0, 1, 5), (0, 0, 0), (0, 2, 5), res, res)
    sc.render = render_params(spp=spp, seed=idx + 7)
    return sc


def config_diffnoise(seed=5, count=32, **kw) -> List[Scene]:
    rng = np.random.default_rng(seed)
    return [config_diffnoise_scene(rng, i, **kw) for i in range(count)]


# ------------------------------------------------------------------ YRS1 file
def write_yrs(sc: Scene, path: str) -> None:
    with open(path, "wb") as f:
        f.write(b"YRS1")
        # last header word: record version; 1 = object records carry the
        # smoothing angle; 2 = shader records carry the version-2 texture
        # fields; 3 = render parameters carry exposure and gamma; 4 = object
        # records carry the instance index (-1: a mesh) and, for instances,
        # the 4x4 matrix; 5 = shader records carry the specular / hardness
        # modulation weights; 6 = object records end with a flag and, when
        # set, 6 texture coordinates per triangle; 7 = then a flag and, when
        # set, the 4x4 orco matrix (meshes only)
        f.write(struct.pack("<4I", len(sc.meshes), len(sc.shaders), len(sc.lights), 7))
        f.write(bytes(sc.camera))
        f.write(bytes(sc.render))
        for s in sc.shaders:
            f.write(bytes(s))
        for l in sc.lights:
            f.write(bytes(l))
        for m in sc.meshes:
            v = np.ascontiguousarray(m.verts, dtype=np.float32)
            t = np.ascontiguousarray(m.tris, dtype=np.uint32)
            f.write(struct.pack("<4Ifi", v.shape[0], t.shape[0], m.shader & 0xFFFFFFFF, 1 if m.cast_shadows else 0,
                                float(m.smooth_angle), int(m.instance_of)))
            if m.is_instance:  # M, then a flag and M^-1 when given
                f.write(np.ascontiguousarray(m.matrix, np.float32).reshape(16).tobytes())
                f.write(struct.pack("<i", 0 if m.inverse is None else 1))
                if m.inverse is not None:
                    f.write(np.ascontiguousarray(m.inverse, np.float32).reshape(16).tobytes())
            f.write(v.tobytes())
            f.write(t.tobytes())
            if m.shader == abi.YR_PER_TRIANGLE:
                f.write(np.ascontiguousarray(m.tri_shaders, dtype=np.uint32).tobytes())
            f.write(struct.pack("<i", 0 if m.uvs is None else 1))
            if m.uvs is not None:
                f.write(np.ascontiguousarray(m.uvs, np.float32).reshape(-1, 6).tobytes())
            f.write(struct.pack("<i", 0 if m.orco is None else 1))
            if m.orco is not None:
                f.write(np.ascontiguousarray(m.orco, np.float32).reshape(16).tobytes())


def read_yrs(path: str) -> Scene:
    data = open(path, "rb").read()
    assert data[:4] == b"YRS1", "bad magic"
    nobj, nsh, nl, version = struct.unpack_from("<4I", data, 4)
    off = 20
    sc = Scene()
    sc.camera = abi.YrCameraDesc.from_buffer_copy(data, off)
    off += C_sizeof(abi.YrCameraDesc)
    # render parameters before version 3 end at exposure (gamma then 1)
    rpsize = C_sizeof(abi.YrRenderParams) if version >= 3 else abi.YrRenderParams.exposure.offset
    sc.render = abi.YrRenderParams()
    C_memmove(sc.render, data[off:off + rpsize])
    if version < 3:
        sc.render.gamma = 1.0
    off += rpsize
    # shader records before version 2 end at mod_mode, before version 5 at
    # mod_specular
    shsize = (C_sizeof(abi.YrShaderDesc) if version >= 5 else
              abi.YrShaderDesc.mod_specular.offset if version >= 2 else abi.YrShaderDesc.mod_mode.offset)
    for _ in range(nsh):
        s = abi.YrShaderDesc()
        C_memmove(s, data[off:off + shsize])
        sc.shaders.append(s)
        off += shsize
    for _ in range(nl):
        sc.lights.append(abi.YrLightDesc.from_buffer_copy(data, off))
        off += C_sizeof(abi.YrLightDesc)
    for _ in range(nobj):
        nv, nt, shid, cast = struct.unpack_from("<4I", data, off)
        off += 16
        smooth = 0.0
        if version >= 1:
            (smooth,) = struct.unpack_from("<f", data, off)
            off += 4
        inst, mat, inv = -1, None, None
        if version >= 4:
            (inst,) = struct.unpack_from("<i", data, off)
            off += 4
            if inst >= 0:
                mat = np.frombuffer(data, np.float32, 16, off).reshape(4, 4).copy()
                off += 64
                (has_inv,) = struct.unpack_from("<i", data, off)
                off += 4
                if has_inv:
                    inv = np.frombuffer(data, np.float32, 16, off).reshape(4, 4).copy()
                    off += 64
        v = np.frombuffer(data, np.float32, 3 * nv, off).reshape(nv, 3).copy()
        off += 12 * nv
        t = np.frombuffer(data, np.uint32, 3 * nt, off).reshape(nt, 3).copy()
        off += 12 * nt
        ts = None
        if shid == abi.YR_PER_TRIANGLE:
            ts = np.frombuffer(data, np.uint32, nt, off).copy()
            off += 4 * nt
        uvs = None
        if version >= 6:
            (has_uv,) = struct.unpack_from("<i", data, off)
            off += 4
            if has_uv:
                uvs = np.frombuffer(data, np.float32, 6 * nt, off).reshape(nt, 6).copy()
                off += 24 * nt
        orco = None
        if version >= 7:
            (has_orco,) = struct.unpack_from("<i", data, off)
            off += 4
            if has_orco:
                orco = np.frombuffer(data, np.float32, 16, off).reshape(4, 4).copy()
                off += 64
        sc.meshes.append(Mesh(v, t, shid, ts, bool(cast), float(smooth), inst, mat, inv, uvs, orco))
    return sc


def C_sizeof(t) -> int:
    import ctypes
    return ctypes.sizeof(t)


def C_memmove(dst, raw: bytes) -> None:
    import ctypes
    ctypes.memmove(ctypes.addressof(dst), raw, len(raw))
