"""CUDA ray queries against the oracle, through the C ABI (yr_trace_closest,
yr_trace_shadow).  Integer results (object, triangle, node counts) must be
identical; hit distances bit for bit."""
import numpy as np
import pytest

import yrtest as T
from yafray_b200 import api, scenes

pytestmark = pytest.mark.gpu


def _run_closest(torch, ds, rays, shadow_only=False):
    n = rays.shape[0]
    d_rays = torch.from_numpy(np.ascontiguousarray(rays, np.float32)).cuda()
    d_hits = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    api.trace_closest(ds, d_rays.data_ptr(), n, d_hits.data_ptr(), shadow_only)
    torch.cuda.synchronize()
    return d_hits.cpu().numpy().view(np.uint32)


def _run_shadow(torch, ds, srays):
    n = srays.shape[0]
    d_rays = torch.from_numpy(np.ascontiguousarray(srays, np.float32)).cuda()
    d_occ = torch.zeros(n, dtype=torch.uint8, device="cuda")
    api.trace_shadow(ds, d_rays.data_ptr(), n, d_occ.data_ptr())
    torch.cuda.synchronize()
    return d_occ.cpu().numpy()


def _shadow_rays(sc, n, seed):
    rng = np.random.default_rng(seed)
    base = T.random_rays(sc, n, seed)
    s = np.zeros((n, 8), np.float32)
    s[:, :3] = base[:, :3]
    s[:, 3] = rng.integers(0, len(sc.meshes), n).astype(np.uint32).view(np.float32)
    s[:, 4:7] = base[:, :3] + base[:, 4:7] * rng.uniform(0.5, 8, (n, 1)).astype(np.float32)
    dirmode = rng.random(n) < 0.25
    s[dirmode, 4:7] = base[dirmode, 4:7]
    s[:, 7] = dirmode.astype(np.uint32).view(np.float32)
    return s


EXACT = 2        # YR_RENDER_EXACT_ORDER
SHADOW_TREE = 1  # YR_RENDER_SHADOW_TREE


@pytest.mark.parametrize("shadow_only", [False, True])
@pytest.mark.parametrize("exact", [False, True])
def test_closest_small_scene(cuda, shadow_only, exact):
    """Object, triangle and distance bit for bit; with the exact object-tree
    order also the number of kd and object-tree nodes visited."""
    sc = scenes.config_small()
    sc.render.flags = EXACT if exact else 0
    ds = api.DeviceScene(sc)
    O = T.OracleScene(sc)
    rays = T.random_rays(sc, 60000, 7)
    got = _run_closest(cuda, ds, rays, shadow_only)
    ref = O.trace_closest(rays, shadow_only)
    assert np.array_equal(got[:, 1], ref[:, 1]), "object ids differ"
    assert np.array_equal(got[:, 2], ref[:, 2]), "triangle ids differ"
    assert np.array_equal(got[:, 0], ref[:, 0]), "hit distances differ"
    if exact:
        assert np.array_equal(got[:, 3], ref[:, 3]), "node visit counts differ"
    assert (ref[:, 1] != 0xFFFFFFFF).sum() > 5000


@pytest.mark.parametrize("exact", [False, True])
def test_closest_many_objects(cuda, exact):
    sc = scenes.config_large(seed=3, resx=64, resy=48, spp=1, grid=4)
    sc.render.flags = EXACT if exact else 0
    ds = api.DeviceScene(sc)
    O = T.OracleScene(sc)
    rays = T.random_rays(sc, 40000, 9)
    got = _run_closest(cuda, ds, rays)
    ref = O.trace_closest(rays)
    assert np.array_equal(got[:, :3], ref[:, :3])
    if exact:
        assert np.array_equal(got[:, 3], ref[:, 3])


@pytest.mark.parametrize("flags", [0, SHADOW_TREE, EXACT])
def test_shadow_small_scene(cuda, flags):
    """Object-tree walk (default, exact order) and the shadow-ray tree give
    the oracle's answers bit for bit."""
    sc = scenes.config_small()
    sc.render.flags = flags
    ds = api.DeviceScene(sc)
    O = T.OracleScene(sc)
    s = _shadow_rays(sc, 60000, 5)
    assert np.array_equal(_run_shadow(cuda, ds, s), O.trace_shadow(s))


@pytest.mark.parametrize("flags", [0, SHADOW_TREE, EXACT])
def test_shadow_many_objects(cuda, flags):
    sc = scenes.config_large(seed=3, resx=64, resy=48, spp=1, grid=4)
    sc.render.flags = flags
    ds = api.DeviceScene(sc)
    O = T.OracleScene(sc)
    s = _shadow_rays(sc, 40000, 6)
    occ = _run_shadow(cuda, ds, s)
    ref = O.trace_shadow(s)
    assert np.array_equal(occ, ref)
    assert 0 < ref.sum() < len(ref)


def _flat_dirs(d, seed):
    """Directions with one or two components zero (rays parallel to a
    coordinate plane or along an axis) or subnormal (1/d overflows)."""
    rng = np.random.default_rng(seed)
    d = d.astype(np.float64).copy()
    n = len(d)
    kind = rng.integers(0, 4, n)   # 0: as given, 1: one zero, 2: two zeros, 3: one subnormal
    ax = rng.integers(0, 3, n)
    rows = np.arange(n)
    one = (kind == 1) | (kind == 3)
    d[rows[one], ax[one]] = 0.0
    two = kind == 2
    keep = ax[two]
    sign = np.sign(d[rows[two], keep])
    sign[sign == 0] = 1.0
    d[two] = 0.0
    d[rows[two], keep] = sign
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    d = d.astype(np.float32)
    sub = kind == 3
    d[rows[sub], ax[sub]] = np.float32(1e-40) * np.sign(rng.standard_normal(sub.sum())).astype(np.float32)
    return d, kind


@pytest.mark.parametrize("flags", [0, SHADOW_TREE, EXACT])
def test_axis_parallel_rays(cuda, flags):
    """Rays with zero or subnormal direction components, whose reciprocals
    are infinite (bound_t::cross skips a zero axis): closest hits and shadow
    answers bit for bit, on the many-object scene."""
    sc = scenes.config_large(seed=3, resx=64, resy=48, spp=1, grid=4)
    sc.render.flags = flags
    ds = api.DeviceScene(sc)
    O = T.OracleScene(sc)
    rays = T.random_rays(sc, 30000, 21)
    rays[:, 4:7], kind = _flat_dirs(rays[:, 4:7], 22)
    got, ref = _run_closest(cuda, ds, rays), O.trace_closest(rays)
    assert np.array_equal(got[:, :3], ref[:, :3])
    for k in range(4):
        assert (ref[kind == k, 1] != 0xFFFFFFFF).sum() > 200
    s = np.zeros((len(rays), 8), np.float32)
    s[:, :3] = rays[:, :3]
    s[:, 3] = np.random.default_rng(23).integers(0, len(sc.meshes), len(rays)).astype(np.uint32).view(np.float32)
    # half directional (l = the direction), half towards a point along it
    dirmode = np.arange(len(rays)) % 2 == 0
    dist = np.random.default_rng(24).uniform(0.5, 8, (len(rays), 1)).astype(np.float32)
    s[:, 4:7] = np.where(dirmode[:, None], rays[:, 4:7], rays[:, :3] + rays[:, 4:7] * dist)
    s[:, 7] = dirmode.astype(np.uint32).view(np.float32)
    occ, oref = _run_shadow(cuda, ds, s), O.trace_shadow(s)
    assert np.array_equal(occ, oref)
    assert 0 < oref.sum() < len(oref)


def test_empty_query(cuda):
    sc = scenes.config_small(32, 24)
    ds = api.DeviceScene(sc)
    assert _run_closest(cuda, ds, np.zeros((0, 8), np.float32)).shape == (0, 4)


def _instance_scene(reference_inverses):
    import sys, os
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_golden
    sc = make_golden.instance_scene()
    if reference_inverses:
        g = np.load(os.path.join(T.GOLDEN, "instances.npz"))
        for i, inv in zip(g["inv_idx"], g["inv"]):
            sc.meshes[int(i)].inverse = inv
    return make_golden, sc


@pytest.mark.parametrize("reference_inverses", [False, True])
@pytest.mark.parametrize("exact", [False, True])
def test_instances_closest_and_shadow(cuda, reference_inverses, exact):
    """Rays through references (referenceObject_t): the original's tree with
    the ray taken there by M^-1; hits and shadow answers bit for bit."""
    mg, sc = _instance_scene(reference_inverses)
    if exact:
        sc.render.flags = EXACT
    ds = api.DeviceScene(sc)
    O = T.OracleScene(sc)
    frm, d, tgt, own = mg.instance_rays(20000, 9)
    rays = np.zeros((len(frm), 8), np.float32)
    rays[:, :3], rays[:, 3], rays[:, 4:7] = frm, np.inf, d
    got, ref = _run_closest(cuda, ds, rays), O.trace_closest(rays)
    assert np.array_equal(got[:, :3], ref[:, :3])
    assert np.isin(ref[:, 1], [3, 4, 5, 6]).sum() > 1000
    s = np.zeros((len(frm), 8), np.float32)
    s[:, :3], s[:, 3], s[:, 4:7] = frm, own.astype(np.uint32).view(np.float32), tgt
    assert np.array_equal(_run_shadow(cuda, ds, s), O.trace_shadow(s))


def test_instance_records_checked(cuda):
    """A reference to a reference, a singular matrix and references with
    the shadow-ray tree are refused."""
    from yafray_b200 import abi
    _, sc = _instance_scene(False)
    sc.meshes.append(scenes.instance(3, np.eye(4)))
    with pytest.raises(abi.YrError):
        api.DeviceScene(sc)
    _, sc = _instance_scene(False)
    sc.meshes.append(scenes.instance(0, np.diag([1.0, 0.0, 1.0, 1.0])))
    with pytest.raises(abi.YrError):
        api.DeviceScene(sc)
    _, sc = _instance_scene(False)
    sc.render.flags = SHADOW_TREE
    with pytest.raises(abi.YrError):
        api.DeviceScene(sc)
