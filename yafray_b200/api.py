"""Python host interface over the C ABI (include/yr.h).

Mirrors the reference's front door for this path: a scene is assembled from
meshes, shaders and lights (yafrayInterface_t::addObject_trimesh /
addLight / addCamera, interface/external.h:144-183), then rendered
(yafrayInterface_t::render, interface_impl.cc:677-835) or queried ray by ray
(scene_t::firstHit / isShadowed, scene.cc:107-185, 688-721).  All compute
runs in the CUDA library; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional

import numpy as np

from . import abi, scenes


class DeviceScene:
    """A scene uploaded to one GPU (yr_scene_create)."""

    def __init__(self, sc: scenes.Scene, device: int = 0, trees=None):
        """trees: optional list (one entry per mesh, None = build here) of
        prebuilt kd-trees (pointers to abi.YrKdTree), e.g. from yr_kdtree_build
        or flattened from YafRay's own kdTree_t."""
        self.lib = abi.load()
        self.sc = sc
        self._keep = []
        objs = (abi.YrObjectDesc * len(sc.meshes))()
        for i, m in enumerate(sc.meshes):
            if m.is_instance:
                mat = np.ascontiguousarray(m.matrix, np.float32).reshape(16)
                self._keep.append(mat)
                objs[i].instance_matrix = mat.ctypes.data_as(C.POINTER(C.c_float))
                if m.inverse is not None:
                    inv = np.ascontiguousarray(m.inverse, np.float32).reshape(16)
                    self._keep.append(inv)
                    objs[i].instance_inverse = inv.ctypes.data_as(C.POINTER(C.c_float))
                objs[i].instance_of = m.instance_of
                continue
            v = np.ascontiguousarray(m.verts, np.float32)
            t = np.ascontiguousarray(m.tris, np.uint32)
            self._keep += [v, t]
            objs[i].verts = v.ctypes.data_as(C.POINTER(C.c_float))
            objs[i].nverts = v.shape[0]
            objs[i].tris = t.ctypes.data_as(C.POINTER(C.c_uint32))
            objs[i].ntris = t.shape[0]
            objs[i].shader = m.shader & 0xFFFFFFFF
            objs[i].cast_shadows = 1 if m.cast_shadows else 0
            objs[i].smooth_angle = float(m.smooth_angle)
            if trees is not None and trees[i] is not None:
                objs[i].tree = trees[i]
            if m.shader == abi.YR_PER_TRIANGLE:
                ts = np.ascontiguousarray(m.tri_shaders, np.uint32)
                self._keep.append(ts)
                objs[i].tri_shaders = ts.ctypes.data_as(C.POINTER(C.c_uint32))
            if m.uvs is not None:
                uv = np.ascontiguousarray(m.uvs, np.float32).reshape(-1, 6)
                assert uv.shape[0] == t.shape[0]
                self._keep.append(uv)
                objs[i].uvs = uv.ctypes.data_as(C.POINTER(C.c_float))
            if m.orco is not None:
                om = np.ascontiguousarray(m.orco, np.float32).reshape(16)
                self._keep.append(om)
                objs[i].orco_matrix = om.ctypes.data_as(C.POINTER(C.c_float))
        shaders = (abi.YrShaderDesc * len(sc.shaders))(*sc.shaders)
        lights = (abi.YrLightDesc * max(1, len(sc.lights)))(*sc.lights)
        desc = abi.YrSceneDesc()
        desc.objects = objs
        desc.nobjects = len(sc.meshes)
        desc.shaders = shaders
        desc.nshaders = len(sc.shaders)
        desc.lights = lights
        desc.nlights = len(sc.lights)
        desc.camera = sc.camera
        desc.render = sc.render
        self._keep += [objs, shaders, lights, desc]
        h = C.c_void_p()
        abi.check(self.lib.yr_scene_create(C.byref(desc), device, C.byref(h)), "yr_scene_create")
        self.handle = h
        self._keep = [v for v in self._keep if isinstance(v, np.ndarray)]  # descriptors no longer needed

    def close(self):
        if getattr(self, "handle", None):
            self.lib.yr_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> abi.YrSceneInfo:
        inf = abi.YrSceneInfo()
        abi.check(self.lib.yr_scene_info_get(self.handle, C.byref(inf)), "yr_scene_info_get")
        return inf

    # ------------------------------------------------------------ rendering
    def render_into(self, out_ptr: int, on_host: bool = False, stream: int = 0) -> abi.YrRenderStats:
        st = abi.YrRenderStats()
        abi.check(self.lib.yr_render(self.handle, C.c_void_p(out_ptr), int(on_host), C.byref(st),
                                     C.c_void_p(stream)), "yr_render")
        return st

    def render(self) -> np.ndarray:
        """Render to a host RGBA float image (resy, resx, 4)."""
        img = np.zeros((self.sc.resy, self.sc.resx, 4), np.float32)
        self.last_stats = self.render_into(img.ctypes.data, on_host=True)
        return img

    def render_progressive(self, on_pixels, wave_pixels: int = 0, img: np.ndarray = None):
        """Render wave by wave into a host RGBA image (yr_render_progressive):
        on_pixels(first, count) is called after each wave with the region
        pixels it finished (row-major in the render region); returning False
        stops the render.  Returns (image, status): status 0, or
        YR_ERR_CANCELLED when the callback stopped it."""
        if img is None:
            img = np.zeros((self.sc.resy, self.sc.resx, 4), np.float32)
        assert img.dtype == np.float32 and img.flags["C_CONTIGUOUS"] and img.shape == (self.sc.resy, self.sc.resx, 4)
        errors = []

        def cb(user, first, count):
            try:
                return 1 if on_pixels(int(first), int(count)) is not False else 0
            except Exception as ex:  # stop the render, raise after the call
                errors.append(ex)
                return 0

        fn = abi.PIXELS_FN(cb)
        st = abi.YrRenderStats()
        rc = self.lib.yr_render_progressive(self.handle, C.c_void_p(img.ctypes.data), int(wave_pixels), fn, None,
                                            C.byref(st), None)
        if errors:
            raise errors[0]
        if rc not in (0, 7):  # YR_OK, YR_ERR_CANCELLED
            abi.check(rc, "yr_render_progressive")
        self.last_stats = st
        return img, rc

    # ------------------------------------------------------------- adjoint
    def param_count(self) -> int:
        return int(self.lib.yr_param_count(self.handle))

    def params_get(self) -> np.ndarray:
        out = np.zeros(max(1, self.param_count()), np.float32)
        abi.check(self.lib.yr_params_get(self.handle, out.ctypes.data_as(C.POINTER(C.c_float))), "yr_params_get")
        return out[:self.param_count()]

    def params_set(self, params) -> None:
        p = np.ascontiguousarray(params, np.float32)
        assert p.shape == (self.param_count(),)
        abi.check(self.lib.yr_params_set(self.handle, p.ctypes.data_as(C.POINTER(C.c_float))), "yr_params_set")

    def backward(self, image_ptr: int, target_ptr: int, dparams_ptr: int, loss_scale: float = 1.0,
                 stream: int = 0) -> float:
        """Gradient of loss_scale * sum over pixels and RGB of (image - target)^2
        with respect to the parameter vector, written to dparams_ptr (device,
        param_count floats).  image: this scene's forward render (device RGBA).
        Returns the loss."""
        d = abi.YrBackwardDesc()
        d.target = target_ptr
        d.image = image_ptr
        d.loss_scale = float(loss_scale)
        loss = C.c_float(0.0)
        abi.check(self.lib.yr_backward(self.handle, C.byref(d), C.c_void_p(dparams_ptr), C.byref(loss),
                                       C.c_void_p(stream)), "yr_backward")
        return float(loss.value)

    def set_params(self, shaders=None, lights=None):
        sh = (abi.YrShaderDesc * len(shaders))(*shaders) if shaders is not None else None
        li = (abi.YrLightDesc * len(lights))(*lights) if lights is not None else None
        abi.check(self.lib.yr_scene_set_params(self.handle, sh, li), "yr_scene_set_params")


def trace_closest(ds: DeviceScene, rays_dev_ptr: int, n: int, hits_dev_ptr: int, shadow_only=False, stream=0):
    abi.check(ds.lib.yr_trace_closest(ds.handle, C.c_void_p(rays_dev_ptr), n, C.c_void_p(hits_dev_ptr),
                                      int(shadow_only), C.c_void_p(stream)), "yr_trace_closest")


def trace_shadow(ds: DeviceScene, rays_dev_ptr: int, n: int, occ_dev_ptr: int, stream=0):
    abi.check(ds.lib.yr_trace_shadow(ds.handle, C.c_void_p(rays_dev_ptr), n, C.c_void_p(occ_dev_ptr),
                                     C.c_void_p(stream)), "yr_trace_shadow")


def render_batch(dss: List[DeviceScene], out_ptrs: List[int], block_size: int = 0, queue_tile: int = 0,
                 use_graph: bool = True, stream: int = 0, mode: int = 0, streams: int = 0):
    """Render several scenes of one GPU as one launch (yr_render_batch).
    out_ptrs: device RGBA float images, one per scene.  mode: 0 = autotuned,
    abi.YR_BATCH_TILES (persistent tile kernel; block_size / queue_tile 0 =
    autotuned) or abi.YR_BATCH_WAVES (per-scene wavefronts on `streams`
    concurrent streams in one CUDA graph; 0 = autotuned).  Returns (stats,
    params used)."""
    lib = abi.load()
    n = len(dss)
    hs = (C.c_void_p * n)(*[d.handle.value for d in dss])
    outs = (C.c_void_p * n)(*out_ptrs)
    p = abi.YrBatchParams(int(block_size), int(queue_tile), int(use_graph), 0, int(mode), int(streams))
    st = abi.YrRenderStats()
    abi.check(lib.yr_render_batch(hs, n, outs, C.byref(p), C.byref(st), C.c_void_p(stream)), "yr_render_batch")
    return st, p


def backward_batch(dss: List[DeviceScene], image_ptrs: List[int], target_ptrs: List[int], grad_ptrs: List[int],
                   loss_scale: float = 1.0, streams: int = 0, stream: int = 0) -> np.ndarray:
    """One optimisation step of several scenes as one CUDA graph
    (yr_backward_batch): renders scene i into image_ptrs[i], then writes its
    gradient to grad_ptrs[i].  Returns the losses."""
    lib = abi.load()
    n = len(dss)
    hs = (C.c_void_p * n)(*[d.handle.value for d in dss])
    descs = (abi.YrBackwardDesc * n)()
    for i in range(n):
        descs[i].image = image_ptrs[i]
        descs[i].target = target_ptrs[i]
        descs[i].loss_scale = float(loss_scale)
    gp = (C.c_void_p * n)(*grad_ptrs)
    losses = np.zeros(n, np.float32)
    abi.check(lib.yr_backward_batch(hs, n, descs, gp, losses.ctypes.data_as(C.POINTER(C.c_float)), int(streams),
                                    C.c_void_p(stream)), "yr_backward_batch")
    return losses


def kdtrees_gpu(meshes, params: Optional[abi.YrKdTreeParams] = None, device: int = 0) -> List[dict]:
    """kd-trees of several meshes built on one GPU (yr_kdtree_build_gpu):
    per mesh a dict of nodes ((n, 2) uint32: word, flags), prims, tb (tree
    bound), max_depth, max_leaf, cost_ratio -- the host build's trees."""
    lib = abi.load()
    keep = []
    arr = (abi.YrKdTreeMesh * len(meshes))()
    for i, m in enumerate(meshes):
        v = np.ascontiguousarray(m.verts, np.float32)
        t = np.ascontiguousarray(m.tris, np.uint32)
        keep += [v, t]
        arr[i].verts = v.ctypes.data_as(C.POINTER(C.c_float))
        arr[i].nverts = v.shape[0]
        arr[i].tris = t.ctypes.data_as(C.POINTER(C.c_uint32))
        arr[i].ntris = t.shape[0]
    outs = (C.POINTER(abi.YrKdTree) * len(meshes))()
    abi.check(lib.yr_kdtree_build_gpu(arr, len(meshes), C.byref(params) if params is not None else None, device,
                                      outs), "yr_kdtree_build_gpu")
    res = []
    for p in outs:
        tr = p.contents
        nodes = np.ctypeslib.as_array(C.cast(tr.nodes, C.POINTER(C.c_uint32)), (2 * tr.nnodes,)).reshape(-1, 2).copy()
        prims = np.ctypeslib.as_array(tr.prims, (max(tr.nprims, 1),))[:tr.nprims].copy()
        res.append(dict(nodes=nodes, prims=prims, tb=np.array(tr.bound[:], np.float32), max_depth=tr.max_depth,
                        max_leaf=tr.max_leaf_size, cost_ratio=np.float32(tr.cost_ratio)))
        lib.yr_kdtree_free(p)
    return res


def encode_image(rgba: np.ndarray, fmt: str = "tga", alpha: bool = False) -> bytes:
    """The bytes YafRay's TGA (outTga_t) or Radiance HDR (outHDR_t) writer
    produces for this float RGBA image (rows top first)."""
    img = np.ascontiguousarray(rgba, np.float32)
    h, w = img.shape[:2]
    lib = abi.load()
    f = {"tga": abi.YR_IMAGE_TGA, "hdr": abi.YR_IMAGE_HDR}[fmt]
    flags = abi.YR_IMAGE_ALPHA if alpha else 0
    fp = img.ctypes.data_as(C.POINTER(C.c_float))
    n = C.c_size_t(0)
    abi.check(lib.yr_image_encode(f, fp, w, h, flags, None, 0, C.byref(n)), "yr_image_encode")
    out = (C.c_uint8 * n.value)()
    abi.check(lib.yr_image_encode(f, fp, w, h, flags, out, n.value, C.byref(n)), "yr_image_encode")
    return bytes(out)


def write_image(path: str, rgba: np.ndarray, fmt: str = "tga", alpha: bool = False) -> None:
    """Write a render as YafRay's loader would (TGA or HDR)."""
    with open(path, "wb") as f:
        f.write(encode_image(rgba, fmt, alpha))
