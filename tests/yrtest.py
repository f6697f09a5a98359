"""Shared helpers for the tests: the CPU oracle (ctypes), the reference
harness (oracle/_ref, present only where the reference was built), and
host-side tree extraction through the product's C ABI."""
from __future__ import annotations

import ctypes as C
import os
import struct
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from yafray_b200 import abi, scenes  # noqa: E402

ORACLE_LIB = os.path.join(ROOT, "oracle", "_build", "liboracle.so")
HARNESS = os.path.join(ROOT, "oracle", "_ref", "yr_ref_harness")
GOLDEN = os.path.join(ROOT, "tests", "golden")

_orc = None


def oracle() -> C.CDLL:
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_LIB):
            subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True,
                           capture_output=True)
        lib = C.CDLL(ORACLE_LIB)
        P, F, U = C.c_void_p, C.c_float, C.c_uint32
        sig = {
            "orc_load": (P, [C.c_char_p]),
            "orc_free": (None, [P]),
            "orc_set_tree": (C.c_int, [P, U, P, U, P, U, P, P]),
            "orc_set_object_tree": (C.c_int, [P, P, U]),
            "orc_trace_closest": (None, [P, P, U, P, C.c_int]),
            "orc_trace_shadow": (None, [P, P, U, P]),
            "orc_kd": (None, [P, U, P, P, F, C.c_int, P]),
            "orc_render": (None, [P, P, C.c_int, C.c_int, C.c_int, C.c_int, P]),
            "orc_render_ex": (None, [P, P, C.c_int, C.c_int, C.c_int, C.c_int, P, F, P]),
            "orc_camera_rays": (None, [P, P]),
            "orc_illum": (C.c_int, [P, U, P, P, P, U, P, P]),
            "orc_noise_gen": (F, [U, F, F, F]),
            "orc_turbulence_gen": (F, [U, F, F, F, C.c_int, F, C.c_int]),
            "orc_vor_features": (None, [C.c_int, F, F, F, F, P]),
            "orc_texture": (None, [P, F, F, F, P]),
            "orc_halton": (F, [U, U]),
            "orc_ri_lp": (F, [U]),
            "orc_cp_rot": (F, [U, U, U]),
            "orc_perlin": (F, [F, F, F]),
            "orc_fbm": (F, [F, F, F, F, F, F]),
            "orc_turbulence": (F, [F, F, F, C.c_int, F, C.c_int]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _orc = lib
    return _orc


def has_harness() -> bool:
    return os.path.exists(HARNESS)


def ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


# ----------------------------------------------------------- product trees
def product_tree(mesh: scenes.Mesh, params=None, nthreads=1) -> dict:
    lib = abi.load()
    v = np.ascontiguousarray(mesh.verts, np.float32)
    t = np.ascontiguousarray(mesh.tris, np.uint32)
    p = C.POINTER(abi.YrKdTree)()
    st = lib.yr_kdtree_build_ex(v.ctypes.data_as(C.POINTER(C.c_float)), v.shape[0],
                                t.ctypes.data_as(C.POINTER(C.c_uint32)), t.shape[0],
                                C.byref(params) if params is not None else None, nthreads, C.byref(p))
    abi.check(st, "yr_kdtree_build")
    tr = p.contents
    nodes = np.ctypeslib.as_array(C.cast(tr.nodes, C.POINTER(C.c_uint32)), (2 * tr.nnodes,)).reshape(-1, 2).copy()
    prims = np.ctypeslib.as_array(tr.prims, (max(tr.nprims, 1),))[:tr.nprims].copy()
    out = dict(nodes=nodes, prims=prims, tb=np.array(tr.bound[:], np.float32), max_depth=tr.max_depth,
               max_leaf=tr.max_leaf_size, cost_ratio=np.float32(tr.cost_ratio))
    lib.yr_kdtree_free(p)
    return out


def gpu_trees(meshes, params=None, device=0) -> list:
    """yr_kdtree_build_gpu over several meshes: one dict per mesh, as
    product_tree returns."""
    from yafray_b200 import api
    return api.kdtrees_gpu(meshes, params, device)


def mesh_bound(mesh: scenes.Mesh) -> np.ndarray:
    """meshObject_t::recalcBound: vertex bound grown by BOX_MIN = 1e-5 in double."""
    v = mesh.verts[mesh.tris.reshape(-1)].astype(np.float32)
    lo = (v.min(0).astype(np.float64) - 0.00001).astype(np.float32)
    hi = (v.max(0).astype(np.float64) + 0.00001).astype(np.float32)
    return np.concatenate([lo, hi]).astype(np.float32)


def object_bound(sc: scenes.Scene, i: int) -> np.ndarray:
    """object3d_t::getBound of object i: the mesh bound, or for a reference
    the placed box of its original's (yr_instance_bound)."""
    m = sc.meshes[i]
    if not m.is_instance:
        return mesh_bound(m)
    b = np.ascontiguousarray(mesh_bound(sc.meshes[m.instance_of]), np.float32)
    mat = np.ascontiguousarray(m.matrix, np.float32).reshape(16)
    out = np.zeros(6, np.float32)
    fp = C.POINTER(C.c_float)
    abi.check(abi.load().yr_instance_bound(b.ctypes.data_as(fp), mat.ctypes.data_as(fp), out.ctypes.data_as(fp)),
              "yr_instance_bound")
    return out


def product_object_tree(sc: scenes.Scene) -> np.ndarray:
    """(n, 8) float32 records bmin[3], left(int bits), bmax[3], right(int bits)."""
    lib = abi.load()
    b = np.ascontiguousarray(np.stack([object_bound(sc, i) for i in range(len(sc.meshes))]), np.float32)
    n = len(sc.meshes)
    out = (abi.YrObjectNode * (2 * n - 1))()
    nout = C.c_uint32()
    st = lib.yr_object_tree_build(b.ctypes.data_as(C.POINTER(C.c_float)), n, out, C.byref(nout))
    abi.check(st, "yr_object_tree_build")
    return np.frombuffer(bytes(out), np.float32).reshape(-1, 8)[: nout.value].copy()


# ------------------------------------------------------------------ oracle
class OracleScene:
    """The oracle loaded with a scene and the given (or product-built) trees."""

    def __init__(self, sc: scenes.Scene, trees=None, otree=None):
        self.sc = sc
        fd, self.path = tempfile.mkstemp(suffix=".yrs")
        os.close(fd)
        scenes.write_yrs(sc, self.path)
        self.lib = oracle()
        self.h = self.lib.orc_load(self.path.encode())
        assert self.h, "oracle could not load the scene"
        trees = trees if trees is not None else [None if m.is_instance else product_tree(m) for m in sc.meshes]
        self._keep = []
        for i, (m, t) in enumerate(zip(sc.meshes, trees)):
            if m.is_instance:  # shares its original's tree
                continue
            nodes = np.ascontiguousarray(t["nodes"], np.uint32)
            prims = np.ascontiguousarray(t["prims"], np.uint32) if len(t["prims"]) else np.zeros(1, np.uint32)
            tb = np.ascontiguousarray(t["tb"], np.float32)
            ob = mesh_bound(m)
            self._keep += [nodes, prims, tb, ob]
            self.lib.orc_set_tree(self.h, i, ptr(nodes), nodes.shape[0], ptr(prims), len(t["prims"]), ptr(tb), ptr(ob))
        ot = otree if otree is not None else product_object_tree(sc)
        ot = np.ascontiguousarray(ot, np.float32)
        self._keep.append(ot)
        self.lib.orc_set_object_tree(self.h, ptr(ot), ot.shape[0])

    def close(self):
        if self.h:
            self.lib.orc_free(self.h)
            self.h = None
        if os.path.exists(self.path):
            os.unlink(self.path)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def trace_closest(self, rays: np.ndarray, shadow_only=False) -> np.ndarray:
        rays = np.ascontiguousarray(rays, np.float32)
        hits = np.zeros((rays.shape[0], 4), np.uint32)
        self.lib.orc_trace_closest(self.h, ptr(rays), rays.shape[0], ptr(hits), int(shadow_only))
        return hits

    def trace_shadow(self, rays: np.ndarray) -> np.ndarray:
        rays = np.ascontiguousarray(rays, np.float32)
        occ = np.zeros(rays.shape[0], np.uint8)
        self.lib.orc_trace_shadow(self.h, ptr(rays), rays.shape[0], ptr(occ))
        return occ

    def kd(self, obj, frm, d, dist, any_hit):
        out = np.zeros(4, np.uint32)
        f = np.ascontiguousarray(frm, np.float32)
        dd = np.ascontiguousarray(d, np.float32)
        self.lib.orc_kd(self.h, obj, ptr(f), ptr(dd), float(dist), int(any_hit), ptr(out))
        return out

    def render(self, x0=0, x1=None, y0=0, y1=None):
        sc = self.sc
        x1 = sc.resx if x1 is None else x1
        y1 = sc.resy if y1 is None else y1
        img = np.zeros((sc.resy, sc.resx, 4), np.float32)
        stats = np.zeros(7, np.uint64)
        self.lib.orc_render(self.h, ptr(img), x0, x1, y0, y1, ptr(stats))
        return img, stats

    def render_ex(self, x0, x1, y0, y1, img=None, flip_band=0.0):
        """Render pixels [x0,x1) x [y0,y1) into `img` (full image layout;
        a new one when None), taking the other branch of every energy
        cut-off within `flip_band` (relative) of its threshold.  Returns
        (img, stats, margin): margin[y, x] = the smallest relative distance
        of any cut-off value of the pixel from its threshold."""
        sc = self.sc
        if img is None:
            img = np.zeros((sc.resy, sc.resx, 4), np.float32)
        margin = np.full((sc.resy, sc.resx), np.inf, np.float32)
        stats = np.zeros(7, np.uint64)
        self.lib.orc_render_ex(self.h, ptr(img), x0, x1, y0, y1, ptr(stats), float(flip_band), ptr(margin))
        return img, stats, margin

    def render_regions(self, regions, threads=None):
        """Render several disjoint pixel regions (x0, x1, y0, y1) on host
        threads; returns (img, stats summed, margin)."""
        import concurrent.futures as cf
        sc = self.sc
        img = np.zeros((sc.resy, sc.resx, 4), np.float32)
        margin = np.full((sc.resy, sc.resx), np.inf, np.float32)
        stats = np.zeros(7, np.uint64)

        def one(r):
            m = np.full((sc.resy, sc.resx), np.inf, np.float32)
            st = np.zeros(7, np.uint64)
            self.lib.orc_render_ex(self.h, ptr(img), r[0], r[1], r[2], r[3], ptr(st), 0.0, ptr(m))
            return r, st, m

        with cf.ThreadPoolExecutor(threads or min(len(regions), os.cpu_count() or 1)) as ex:
            for r, st, m in ex.map(one, regions):
                stats += st
                margin[r[2]:r[3], r[0]:r[1]] = m[r[2]:r[3], r[0]:r[1]]
        return img, stats, margin

    def camera_rays(self):
        d = np.zeros((self.sc.resy, self.sc.resx, 3), np.float32)
        self.lib.orc_camera_rays(self.h, ptr(d))
        return d

    def illum(self, q: np.ndarray, vals: np.ndarray):
        """One light's contribution at the first hit of each ILLUM_REC query,
        rotation off, area lights fed `vals` (n, 64).  Returns (hit, rgb)."""
        n = q.shape[0]
        hit = np.zeros(n, np.int32)
        rgb = np.zeros((n, 3), np.float32)
        for i in range(n):
            e = np.ascontiguousarray(q["eye"][i], np.float32)
            f = np.ascontiguousarray(q["frm"][i], np.float32)
            d = np.ascontiguousarray(q["dir"][i], np.float32)
            v = np.ascontiguousarray(vals[i], np.float32)
            out = np.zeros(3, np.float32)
            hit[i] = self.lib.orc_illum(self.h, int(q["light"][i]), ptr(e), ptr(f), ptr(d), int(q["m0"][i]), ptr(v),
                                        ptr(out))
            rgb[i] = out
        return hit, rgb


# ----------------------------------------------------------------- harness
def run_harness(*args, timeout=600):
    r = subprocess.run([HARNESS] + [str(a) for a in args], capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"harness {args[0]} failed: {r.stderr[-2000:]}")
    return r.stdout


def harness_trees(sc: scenes.Scene):
    with tempfile.TemporaryDirectory() as d:
        sp, op = os.path.join(d, "s.yrs"), os.path.join(d, "t.bin")
        scenes.write_yrs(sc, sp)
        run_harness("tree", sp, op)
        data = open(op, "rb").read()
    off = 0
    n, = struct.unpack_from("<I", data, off)
    off += 4
    trees = []
    for _ in range(n):
        nn, npr = struct.unpack_from("<2I", data, off)
        off += 8
        tb = np.frombuffer(data, np.float32, 6, off).copy()
        off += 24
        md, ml = struct.unpack_from("<2i", data, off)
        off += 8
        cr, eb = struct.unpack_from("<2f", data, off)
        off += 8
        ob = np.frombuffer(data, np.float32, 6, off).copy()
        off += 24
        nodes = np.frombuffer(data, np.uint32, 2 * nn, off).reshape(nn, 2).copy()
        off += 8 * nn
        prims = np.frombuffer(data, np.uint32, npr, off).copy()
        off += 4 * npr
        trees.append(dict(nodes=nodes, prims=prims, tb=tb, max_depth=md, max_leaf=ml, cost_ratio=np.float32(cr),
                          ob=ob))
    nn, = struct.unpack_from("<I", data, off)
    off += 4
    raw = np.frombuffer(data, np.float32, 8 * nn, off).reshape(nn, 8)
    # harness record: bmin[3], bmax[3], left, right -> yr_object_node order
    otree = np.ascontiguousarray(raw[:, [0, 1, 2, 6, 3, 4, 5, 7]])
    return trees, otree


RAY_REC = np.dtype([("mode", "<u4"), ("object", "<u4"), ("frm", "<f4", 3), ("dir", "<f4", 3), ("dist", "<f4"),
                    ("l", "<f4", 3)])


def harness_rays(sc: scenes.Scene, recs: np.ndarray) -> np.ndarray:
    """Run ray records (RAY_REC) through the reference; returns (n,4) uint32."""
    with tempfile.TemporaryDirectory() as d:
        sp, rp, op = os.path.join(d, "s.yrs"), os.path.join(d, "r.bin"), os.path.join(d, "o.bin")
        scenes.write_yrs(sc, sp)
        with open(rp, "wb") as f:
            f.write(struct.pack("<I", recs.shape[0]))
            f.write(np.ascontiguousarray(recs, RAY_REC).tobytes())
        run_harness("rays", sp, rp, op)
        return np.fromfile(op, np.uint32).reshape(-1, 4)


def harness_render(sc: scenes.Scene, threads=1, crop=None):
    with tempfile.TemporaryDirectory() as d:
        sp, op = os.path.join(d, "s.yrs"), os.path.join(d, "o.bin")
        scenes.write_yrs(sc, sp)
        args = ["render", sp, op, threads] + (list(crop) if crop else [])
        out = run_harness(*args)
        img = np.fromfile(op, np.float32).reshape(sc.resy, sc.resx, 4)
    import json
    return img, json.loads(out.strip().splitlines()[-1])


ILLUM_REC = np.dtype([("light", "<u4"), ("m0", "<u4"), ("lcg", "<i4"), ("eye", "<f4", 3), ("frm", "<f4", 3),
                      ("dir", "<f4", 3)])
ILLUM_OUT = np.dtype([("hit", "<u4"), ("synced", "<u4"), ("rgb", "<f4", 3), ("nvals", "<u4"), ("vals", "<f4", 64)])


def harness_illum(sc: scenes.Scene, q: np.ndarray) -> np.ndarray:
    """One light's illuminate() per ILLUM_REC query in the reference, with
    the light's sample stream set from the query; returns ILLUM_OUT records."""
    with tempfile.TemporaryDirectory() as d:
        sp, qp, op = os.path.join(d, "s.yrs"), os.path.join(d, "q.bin"), os.path.join(d, "o.bin")
        scenes.write_yrs(sc, sp)
        with open(qp, "wb") as f:
            f.write(struct.pack("<I", q.shape[0]))
            f.write(np.ascontiguousarray(q, ILLUM_REC).tobytes())
        run_harness("illum", sp, qp, op)
        return np.fromfile(op, ILLUM_OUT)


def harness_instance_inverses(sc: scenes.Scene) -> dict:
    """{object index: 4x4 M^-1} of every reference, as referenceObject_t
    computes it."""
    with tempfile.TemporaryDirectory() as d:
        sp, op = os.path.join(d, "s.yrs"), os.path.join(d, "o.bin")
        scenes.write_yrs(sc, sp)
        run_harness("instmat", sp, op)
        data = open(op, "rb").read()
    n, = struct.unpack_from("<I", data, 0)
    out, off = {}, 4
    for _ in range(n):
        i, = struct.unpack_from("<I", data, off)
        out[i] = np.frombuffer(data, np.float32, 16, off + 4).reshape(4, 4).copy()
        off += 68
    return out


def harness_orco_matrices(sc: scenes.Scene) -> dict:
    """{object index: 4x4 backOrco} of every mesh whose orco matrix is set
    (any value: the reference makes those meshes through
    meshObject_t::transform and computes its own)."""
    with tempfile.TemporaryDirectory() as d:
        sp, op = os.path.join(d, "s.yrs"), os.path.join(d, "o.bin")
        scenes.write_yrs(sc, sp)
        run_harness("orcomat", sp, op)
        data = open(op, "rb").read()
    n, = struct.unpack_from("<I", data, 0)
    out, off = {}, 4
    for _ in range(n):
        i, = struct.unpack_from("<I", data, off)
        out[i] = np.frombuffer(data, np.float32, 16, off + 4).reshape(4, 4).copy()
        off += 68
    return out


def harness_camera(sc: scenes.Scene) -> np.ndarray:
    with tempfile.TemporaryDirectory() as d:
        sp, op = os.path.join(d, "s.yrs"), os.path.join(d, "o.bin")
        scenes.write_yrs(sc, sp)
        run_harness("camera", sp, op)
        return np.fromfile(op, np.float32).reshape(sc.resy, sc.resx, 3)


# ------------------------------------------------------------------- rays
def random_rays(sc: scenes.Scene, n: int, seed: int, spread=1.0) -> np.ndarray:
    """Rays from around the camera / scene towards random scene points,
    as yr_ray records (n, 8) float32."""
    rng = np.random.default_rng(seed)
    allv = np.concatenate([m.verts for m in sc.meshes])
    lo, hi = allv.min(0), allv.max(0)
    c = (lo + hi) / 2
    ext = (hi - lo) / 2 * 1.2
    org = c + rng.uniform(-1, 1, (n, 3)) * ext * spread
    tgt = c + rng.uniform(-1, 1, (n, 3)) * ext * 0.5
    d = tgt - org
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = org
    rays[:, 3] = -1.0
    rays[:, 4:7] = d
    return rays
