"""Python host mirror of the reference's hot-path interfaces, over the C ABI.

    Context            one psy_ctx (a CUDA device + uploaded scene)
    Tracer             Tracer::trace (reference tracer/tracer.hpp:76)
    LightTree          LightTree::sample (reference accel/light_tree.cpp:30)
    PathTraceIntegrator PathTraceIntegrator::integrate
                       (reference integrator/path_trace_integrator.hpp:103-126)

Scenes are the psychopath_cpp_b200.scene model (or .psy files through
scene.read_psy); ``flatten`` turns one into the C ABI's psy_scene_desc.
Every call goes through libpsy_b200.so; a missing library raises.
"""
from __future__ import annotations

import ctypes as C
import time
from typing import Dict, List, Optional, Tuple

import numpy as np

from . import _abi
from .scene import (Assembly, BicubicPatch, BilinearPatch, RectangleLight, Scene, Sphere, SphereLight,
                    SurfaceShader)

F32 = np.float32

HIT_FIELDS = {  # name -> (dtype, per-ray width)
    "hit": (np.uint8, 1), "id": (np.uint64, 1), "t": (np.float32, 1), "uv": (np.float32, 2),
    "p": (np.float32, 3), "n": (np.float32, 3), "dpdu": (np.float32, 3), "dpdv": (np.float32, 3),
    "dndu": (np.float32, 3), "dndv": (np.float32, 3), "backfacing": (np.uint8, 1),
    "light_pdf": (np.float32, 1), "offset": (np.float32, 3), "space": (np.float32, 16),
    "closure": (np.uint8, 1), "closure_color": (np.float32, 3),
}


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


# --------------------------------------------------------------------------
# Scene flattening
# --------------------------------------------------------------------------

def flatten(scene: Scene):
    """Returns (SceneDesc, keepalive) for psy_scene_upload."""
    keep: List = []
    asm_order: List[Assembly] = []

    def collect(a: Assembly):
        asm_order.append(a)
        for sub in a.assemblies.values():
            collect(sub)

    collect(scene.root)
    asm_index = {id(a): i for i, a in enumerate(asm_order)}
    shader_list: List[SurfaceShader] = []
    shader_index: Dict[int, int] = {}

    def shader_id(sh: Optional[SurfaceShader]) -> int:
        if sh is None:
            return -1
        if id(sh) not in shader_index:
            shader_index[id(sh)] = len(shader_list)
            shader_list.append(sh)
        return shader_index[id(sh)]

    asm_descs = (_abi.AssemblyDesc * len(asm_order))()
    for ai, a in enumerate(asm_order):
        obj_names = list(a.objects.keys())
        sub_names = list(a.assemblies.keys())
        obj_pos = {name: i for i, name in enumerate(obj_names)}
        sub_pos = {name: i for i, name in enumerate(sub_names)}
        objs = (_abi.ObjectDesc * max(1, len(obj_names)))()
        for oi, name in enumerate(obj_names):
            ob = a.objects[name]
            if isinstance(ob, Sphere):
                data = np.concatenate([ob.location, [ob.radius]]).astype(F32)
                kind, n0, n1, n2 = _abi.PSY_OBJ_SPHERE, 1, 0, 0
            elif isinstance(ob, BilinearPatch):
                data = ob.verts.reshape(-1).astype(F32)
                kind, n0, n1, n2 = _abi.PSY_OBJ_BILINEAR, ob.verts.shape[0], 0, 0
            elif isinstance(ob, BicubicPatch):
                data = ob.verts.reshape(-1).astype(F32)
                kind, n0, n1, n2 = _abi.PSY_OBJ_BICUBIC, ob.verts.shape[0], 0, 0
            elif isinstance(ob, SphereLight):
                data = np.concatenate([ob.locations.ravel(), ob.radii.ravel(), ob.colors.ravel()]).astype(F32)
                kind, n0, n1, n2 = (_abi.PSY_OBJ_SPHERE_LIGHT, ob.locations.shape[0], ob.radii.shape[0],
                                    ob.colors.shape[0])
            elif isinstance(ob, RectangleLight):
                data = np.concatenate([ob.dimensions.ravel(), ob.colors.ravel()]).astype(F32)
                kind, n0, n1, n2 = _abi.PSY_OBJ_RECT_LIGHT, ob.dimensions.shape[0], ob.colors.shape[0], 0
            else:
                raise TypeError("unsupported object %r" % type(ob))
            data = np.ascontiguousarray(data)
            keep.append(data)
            objs[oi] = _abi.ObjectDesc(kind, n0, n1, n2, data.ctypes.data_as(_abi.fp))
        xforms: List[np.ndarray] = []
        insts = (_abi.InstanceDesc * max(1, len(a.instances)))()
        for ii, inst in enumerate(a.instances):
            if inst.data in obj_pos:
                kind, didx = _abi.PSY_INSTANCE_OBJECT, obj_pos[inst.data]
            elif inst.data in sub_pos:
                kind, didx = _abi.PSY_INSTANCE_ASSEMBLY, sub_pos[inst.data]
            else:
                raise KeyError("instance of unknown data %r" % inst.data)
            sh = a.shader_of(inst)
            insts[ii] = _abi.InstanceDesc(kind, didx, len(xforms), len(inst.transforms), shader_id(sh))
            xforms.extend(inst.transforms)
        xf = np.ascontiguousarray(np.array(xforms, dtype=F32).reshape(-1)) if xforms else np.zeros(16, F32)
        children = np.array([asm_index[id(a.assemblies[n])] for n in sub_names] or [0], dtype=np.uint32)
        keep += [objs, insts, xf, children]
        asm_descs[ai] = _abi.AssemblyDesc(len(obj_names), objs, len(a.instances), insts, len(xforms),
                                          xf.ctypes.data_as(_abi.fp), len(sub_names),
                                          children.ctypes.data_as(_abi.u32p))
    shaders = (_abi.ShaderDesc * max(1, len(shader_list)))()
    kinds = {"Lambert": _abi.PSY_SHADER_LAMBERT, "Emit": _abi.PSY_SHADER_EMIT, "GTR": _abi.PSY_SHADER_GTR}
    for si, sh in enumerate(shader_list):
        shaders[si] = _abi.ShaderDesc(kinds[sh.kind], (C.c_float * 3)(*[float(c) for c in sh.color]),
                                      float(sh.roughness), float(sh.tail_shape), float(sh.fresnel))
    cam = scene.camera
    cx = np.ascontiguousarray(np.array(cam.transforms, dtype=F32).reshape(-1))
    fovs = np.ascontiguousarray(cam.fovs_radians())
    aps = np.ascontiguousarray(np.array(cam.aperture_radii or [0.0], dtype=F32))
    foc = np.ascontiguousarray(np.array(cam.focus_distances or [1.0], dtype=F32))
    keep += [asm_descs, shaders, cx, fovs, aps, foc]
    d = _abi.SceneDesc()
    d.cam_transform_count = len(cam.transforms)
    d.cam_transforms = cx.ctypes.data_as(_abi.fp)
    d.cam_fov_count = len(fovs)
    d.cam_fovs = fovs.ctypes.data_as(_abi.fp)
    d.cam_aperture_count = len(cam.aperture_radii)
    d.cam_aperture_radii = aps.ctypes.data_as(_abi.fp)
    d.cam_focus_count = len(cam.focus_distances)
    d.cam_focus_distances = foc.ctypes.data_as(_abi.fp)
    for k in range(3):
        d.background[k] = float(scene.background[k])
    d.dice_rate = float(F32(scene.dicing_rate if scene.dicing_rate is not None else 0.25))
    d.min_upoly_size = float(F32(0.00001))
    d.assembly_count = len(asm_order)
    d.assemblies = asm_descs
    d.shader_count = len(shader_list)
    d.shaders = shaders
    return d, keep


class PsyFile:
    """A .psy scene file read by the library (psy_file_parse), in place of
    the reference's Parser::parse_scene (parser/parser.cpp:37-662): its
    scene description and render settings.  Context.upload_flat(f.flat())
    uploads it; build_bvh4_records / build_light_tree take it too.  `frame`
    picks the file's Scene node (parse_next_frame reads them in order; past
    the last one raises PsyError with code PSY_ERR_NO_SCENE)."""

    def __init__(self, text: str, frame: int = 0):
        self.L = _abi.load()
        data = text.encode() if isinstance(text, str) else bytes(text)
        h = C.c_void_p()
        err = C.create_string_buffer(512)
        rc = self.L.psy_file_parse(data, len(data), frame, C.byref(h), err, len(err))
        if rc != 0:
            raise _abi.PsyError(rc, err.value.decode())
        self.h = h
        s = _abi.RenderSettings()
        self.L.psy_file_render_settings(h, C.byref(s))
        self.settings = {k: int(getattr(s, k)) for k in ("width", "height", "spp", "seed")}
        self.output_path = (s.output_path or b"").decode()

    @classmethod
    def read(cls, path: str, frame: int = 0) -> "PsyFile":
        with open(path) as f:
            return cls(f.read(), frame)

    @property
    def desc(self):
        """The scene description; it keeps this reader (and the memory it
        points into) alive."""
        d = self.L.psy_file_scene_desc(self.h).contents
        d._owner = self
        return d

    def flat(self):
        """(SceneDesc, keepalive), the form flatten() returns."""
        return self.desc, self

    def close(self):
        if getattr(self, "h", None):
            self.L.psy_file_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --------------------------------------------------------------------------
# Context and reference-named wrappers
# --------------------------------------------------------------------------

class Context:
    """A psy_ctx on one CUDA device."""

    def __init__(self, device: int = 0):
        self.L = _abi.load()
        h = C.c_void_p()
        rc = self.L.psy_ctx_create(device, C.byref(h))
        if rc != 0:
            raise _abi.PsyError(rc, "psy_ctx_create(%d) failed" % device)
        self.h = h
        self.device = device
        self.scene: Optional[Scene] = None

    def close(self):
        if getattr(self, "h", None):
            self.L.psy_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, rc: int):
        if rc != 0:
            raise _abi.PsyError(rc, self.L.psy_last_error(self.h).decode())

    def upload(self, scene: Scene, gpu_bvh: bool = False) -> float:
        """psy_scene_upload; gpu_bvh builds the root's traversal BVH4 and light
        tree on the device (psy_scene_upload_ex with PSY_UPLOAD_GPU_BVH).
        Returns the seconds spent in the library call (scene build and copy
        to the device, without this module's flattening of `scene`)."""
        dt = self.upload_flat(flatten(scene), gpu_bvh)
        self.scene = scene
        return dt

    def upload_flat(self, flat, gpu_bvh: bool = False) -> float:
        """upload() of a scene already flattened (flatten(scene)), for a scene
        uploaded more than once; returns the library call's seconds."""
        desc, _keep = flat
        t0 = time.perf_counter()
        if gpu_bvh:
            self.check(self.L.psy_scene_upload_ex(self.h, C.byref(desc), _abi.PSY_UPLOAD_GPU_BVH))
        else:
            self.check(self.L.psy_scene_upload(self.h, C.byref(desc)))
        return time.perf_counter() - t0

    def stats(self) -> dict:
        s = _abi.SceneStats()
        self.check(self.L.psy_scene_stats_get(self.h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in _abi.SceneStats._fields_}

    def sync(self, stream=None):
        self.check(self.L.psy_sync(self.h, stream))

    def trace_counters(self) -> dict:
        """Traversal work counters of the last render on this context
        (psy_profile_counters): {"closest": {...}, "occlusion": {...}}."""
        c, o = _abi.TraceCounters(), _abi.TraceCounters()
        self.check(self.L.psy_profile_counters(self.h, C.byref(c), C.byref(o)))
        return {"closest": c.as_dict(), "occlusion": o.as_dict()}

    MATH_FUNCTIONS = ("sin", "cos", "acos", "asin", "exp")

    def math_check(self, fn: str, x: np.ndarray) -> np.ndarray:
        """The device's float `fn` (one of MATH_FUNCTIONS) of every element
        of `x` (psy_math_check): the restatements of the host C library's
        sincosf / acosf / asinf / expf that the shading kernels use."""
        x = np.ascontiguousarray(x, np.float32).ravel()
        out = np.empty_like(x)
        fp = C.POINTER(C.c_float)
        self.check(self.L.psy_math_check(self.h, self.MATH_FUNCTIONS.index(fn), x.size, x.ctypes.data_as(fp),
                                         out.ctypes.data_as(fp)))
        return out


def _check(L, rc: int, what: str):
    if rc != 0:
        raise _abi.PsyError(rc, what)


def build_bvh4_records(scene: Scene, assembly: int = 0) -> dict:
    """Host-only: the BVH4 node records the builder produces for one
    assembly, in the reference's BVH4::Node form (psy_build_bvh4)."""
    L = _abi.load()
    desc, keep = scene.flat() if isinstance(scene, PsyFile) else flatten(scene)
    n = C.c_uint64()
    _check(L, L.psy_build_bvh4(C.byref(desc), assembly, C.byref(n), None, None, None, None), "psy_build_bvh4")
    k = n.value
    b = np.zeros((k, 24), F32)
    ch = np.zeros((k, 3), np.uint64)
    ts = np.zeros(k, np.uint32)
    di = np.zeros(k, np.uint64)
    _check(L, L.psy_build_bvh4(C.byref(desc), assembly, C.byref(n), b.ctypes.data_as(_abi.fp),
                               ch.ctypes.data_as(_abi.u64p), ts.ctypes.data_as(_abi.u32p),
                               di.ctypes.data_as(_abi.u64p)), "psy_build_bvh4")
    del keep
    return {"bounds": b, "child": ch, "ts": ts, "data_index": di}


def build_light_tree(scene: Scene, assembly: int = 0) -> dict:
    """Host-only: the light tree the builder produces for one assembly
    (psy_build_light_tree), in the reference's LightTree node form."""
    L = _abi.load()
    desc, keep = scene.flat() if isinstance(scene, PsyFile) else flatten(scene)
    n, nb, lc = C.c_uint64(), C.c_uint64(), C.c_uint64()
    te = C.c_float()
    _check(L, L.psy_build_light_tree(C.byref(desc), assembly, C.byref(n), C.byref(nb), None, None, None,
                                     C.byref(lc), C.byref(te)), "psy_build_light_tree")
    meta = np.zeros((n.value, 6), np.uint64)
    en = np.zeros(n.value, F32)
    bb = np.zeros((max(nb.value, 1), 6), F32)
    _check(L, L.psy_build_light_tree(C.byref(desc), assembly, C.byref(n), C.byref(nb),
                                     meta.ctypes.data_as(_abi.u64p), en.ctypes.data_as(_abi.fp),
                                     bb.ctypes.data_as(_abi.fp), C.byref(lc), C.byref(te)), "psy_build_light_tree")
    del keep
    return {"meta": meta, "energy": en, "bounds": bb[:nb.value], "light_count": lc.value,
            "total_energy": te.value}


def _ray_soa_host(rays: dict) -> Tuple[_abi.RaySoA, list]:
    keep = []

    def a(name, dtype, shape):
        arr = np.ascontiguousarray(np.asarray(rays[name], dtype=dtype).reshape(shape))
        keep.append(arr)
        return arr.ctypes.data_as(C.c_void_p)

    n = len(rays["time"])
    r = _abi.RaySoA(a("o", F32, (n, 3)), a("d", F32, (n, 3)), a("odx", F32, (n, 3)), a("ody", F32, (n, 3)),
                    a("ddx", F32, (n, 3)), a("ddy", F32, (n, 3)), a("time", F32, (n,)),
                    a("type", np.uint16, (n,)) if "type" in rays else None)
    return r, keep


class Tracer:
    """Tracer::trace over a ray stream (reference tracer/tracer.cpp:38-121)."""

    def __init__(self, ctx: Context):
        self.ctx = ctx

    def trace(self, rays: dict, fields=("hit", "id", "t", "uv")) -> Dict[str, np.ndarray]:
        """Host-array form (psy_trace_host): returns the requested
        Intersection fields as numpy arrays."""
        n = len(rays["time"])
        rs, keep = _ray_soa_host(rays)
        out = {}
        hs = _abi.HitSoA()
        for f in fields:
            dt, w = HIT_FIELDS[f]
            arr = np.zeros((n, w) if w > 1 else (n,), dt)
            out[f] = arr
            setattr(hs, f, arr.ctypes.data_as(C.c_void_p))
        self.ctx.check(self.ctx.L.psy_trace_host(self.ctx.h, C.byref(rs), n, C.byref(hs)))
        return out

    def trace_noalloc(self, rays: dict, fields=("hit", "id", "t", "uv"), stream=None) -> Dict[str, np.ndarray]:
        """psy_trace_host_noalloc: as trace(), staged in the library's
        fixed-size device array (at most _abi.PSY_NOALLOC_MAX_RAYS rays per
        call).  fields=None passes no hit arrays at all (hits = NULL)."""
        n = len(rays["time"])
        rs, keep = _ray_soa_host(rays)
        out = {}
        hs = _abi.HitSoA()
        for f in fields or ():
            dt, w = HIT_FIELDS[f]
            arr = np.zeros((n, w) if w > 1 else (n,), dt)
            out[f] = arr
            setattr(hs, f, arr.ctypes.data_as(C.c_void_p))
        self.ctx.check(self.ctx.L.psy_trace_host_noalloc(self.ctx.h, C.byref(rs), n,
                                                         C.byref(hs) if fields is not None else None, stream))
        return out

    def trace_device(self, rays: dict, hits: dict, stream=None) -> None:
        """Device form (psy_trace): `rays` and `hits` map field names to
        CUDA tensors (anything with .data_ptr()); stream-ordered."""
        n = int(rays["time"].shape[0])

        def p(t):
            return None if t is None else C.c_void_p(t.data_ptr())

        rs = _abi.RaySoA(p(rays["o"]), p(rays["d"]), p(rays["odx"]), p(rays["ody"]), p(rays["ddx"]),
                         p(rays["ddy"]), p(rays["time"]), p(rays.get("type")))
        hs = _abi.HitSoA()
        for f, t in hits.items():
            setattr(hs, f, p(t))
        self.ctx.check(self.ctx.L.psy_trace(self.ctx.h, C.byref(rs), n, C.byref(hs), stream))


def _torch():
    import torch
    return torch


class LightTree:
    """LightTree::sample over a batch of queries (reference accel/light_tree.cpp:30-96)."""

    def __init__(self, ctx: Context):
        self.ctx = ctx

    def sample(self, q: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
        """q: (n, 15) float32 rows n u v pos(3) nor(3) d(3) wavelength time (pad).
        Returns (out (n, 14) in the oracle's layout: to_light(3) spec(4)
        hero selection_pdf light_pdf light_count pad(3), ids (n,))."""
        torch = _torch()
        dev = torch.device("cuda", self.ctx.device)
        q = np.ascontiguousarray(q, np.float32).reshape(-1, 15)
        n = q.shape[0]
        cols = {"n": q[:, 0], "u": q[:, 1], "v": q[:, 2], "pos": q[:, 3:6], "nor": q[:, 6:9], "d": q[:, 9:12],
                "wavelength": q[:, 12], "time": q[:, 13]}
        dq = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in cols.items()}
        out = {"to_light": torch.zeros((n, 3), dtype=torch.float32, device=dev),
               "spec": torch.zeros((n, 4), dtype=torch.float32, device=dev),
               "selection_pdf": torch.zeros(n, dtype=torch.float32, device=dev),
               "light_pdf": torch.zeros(n, dtype=torch.float32, device=dev),
               "id": torch.zeros(n, dtype=torch.int64, device=dev)}
        qs = _abi.LightQuerySoA(*[C.c_void_p(dq[k].data_ptr()) for k in
                                  ("n", "u", "v", "pos", "nor", "d", "wavelength", "time")])
        os_ = _abi.LightSampleSoA(*[C.c_void_p(out[k].data_ptr()) for k in
                                    ("to_light", "spec", "selection_pdf", "light_pdf", "id")])
        self.ctx.check(self.ctx.L.psy_light_sample(self.ctx.h, C.byref(qs), n, C.byref(os_), None))
        self.ctx.sync()
        res = np.zeros((n, 14), np.float32)
        res[:, 0:3] = out["to_light"].cpu().numpy()
        res[:, 3:7] = out["spec"].cpu().numpy()
        res[:, 7] = q[:, 12]
        res[:, 8] = out["selection_pdf"].cpu().numpy()
        res[:, 9] = out["light_pdf"].cpu().numpy()
        return res, out["id"].cpu().numpy().view(np.uint64)


class PathTraceIntegrator:
    """PathTraceIntegrator (reference integrator/path_trace_integrator.hpp:103-126).

    integrate() renders the context's scene and returns the film's per-pixel
    XYZ sums (h, w, 3) and sample counts (h, w), as the reference's Film
    accumulates them."""

    def __init__(self, ctx: Context, width: int, height: int, spp: int, seed: int = 1, path_length: int = 4,
                 stream_paths: int = 0, block_size: int = 0):
        self.ctx = ctx
        self.desc = _abi.RenderDesc(width, height, spp, seed, path_length, stream_paths, block_size)
        self.stats = _abi.RenderStats()

    @classmethod
    def for_scene(cls, ctx: Context, scene: Scene, **kw):
        args = dict(width=scene.res_x, height=scene.res_y, spp=scene.spp, seed=scene.seed)
        args.update(kw)
        return cls(ctx, **args)

    def integrate_device(self, xyz, counts=None, stream=None, with_stats: bool = True) -> None:
        """Accumulates into device tensors xyz (h*w*3 float32) and counts
        (h*w int32/uint32), stream-ordered.  With with_stats the call also
        synchronises the stream and fills self.stats (rays, launches)."""
        self.ctx.check(self.ctx.L.psy_render(self.ctx.h, C.byref(self.desc), C.c_void_p(xyz.data_ptr()),
                                             C.c_void_p(counts.data_ptr()) if counts is not None else None,
                                             C.byref(self.stats) if with_stats else None, stream))

    def integrate(self) -> Tuple[np.ndarray, np.ndarray]:
        torch = _torch()
        dev = torch.device("cuda", self.ctx.device)
        w, h = self.desc.width, self.desc.height
        xyz = torch.zeros(h * w * 3, dtype=torch.float32, device=dev)
        cnt = torch.zeros(h * w, dtype=torch.int32, device=dev)
        self.integrate_device(xyz, cnt)
        self.ctx.sync()
        return xyz.cpu().numpy().reshape(h, w, 3), cnt.cpu().numpy().reshape(h, w).astype(np.uint32)


class Film:
    """The film of a render (the reference's Film, film/film.hpp): per-pixel
    XYZ sums and sample counts as psy_render accumulates them, its 8-bit
    sRGB image (psy_film_srgb8, Film::scanline_image_8bbc) and the image
    files the reference writes with OpenImageIO (renderer/renderer.cpp:24-42;
    OpenImageIO is absent, so PPM for the 8-bit image and PFM for the mean
    XYZ are written here)."""

    def __init__(self, ctx: Context, xyz, counts, width: int, height: int):
        self.ctx, self.xyz, self.counts, self.width, self.height = ctx, xyz, counts, width, height

    def srgb8(self, dither_seed: Optional[int] = 0, stream=None):
        """(h, w, 3) uint8 device tensor; dither_seed None = no dither."""
        torch = _torch()
        out = torch.empty(self.height * self.width * 3, dtype=torch.uint8, device=self.xyz.device)
        self.ctx.check(self.ctx.L.psy_film_srgb8(self.ctx.h, C.c_void_p(self.xyz.data_ptr()),
                                                 C.c_void_p(self.counts.data_ptr()), self.width, self.height,
                                                 0 if dither_seed is None else 1, int(dither_seed or 0) & 0xffffffff,
                                                 C.c_void_p(out.data_ptr()), stream))
        return out.view(self.height, self.width, 3)

    def write_ppm(self, path: str, dither_seed: Optional[int] = 0) -> None:
        """Binary PPM (P6) of the 8-bit sRGB image, scanlines top to bottom."""
        rgb = self.srgb8(dither_seed).cpu().numpy()
        with open(path, "wb") as f:
            f.write(b"P6\n%d %d\n255\n" % (self.width, self.height))
            f.write(np.ascontiguousarray(rgb).tobytes())

    def write_pfm(self, path: str) -> None:
        """PFM (little-endian, three channels) of the mean XYZ per pixel
        (0 where no sample landed), rows bottom to top as PFM stores them."""
        x = self.xyz.detach().cpu().numpy().reshape(self.height, self.width, 3).astype(np.float32)
        c = self.counts.detach().cpu().numpy().reshape(self.height, self.width, 1).astype(np.float32)
        mean = np.where(c > 0, x / np.maximum(c, 1), 0.0).astype("<f4")
        with open(path, "wb") as f:
            f.write(b"PF\n%d %d\n-1.0\n" % (self.width, self.height))
            f.write(np.ascontiguousarray(mean[::-1]).tobytes())


def read_ppm(path: str) -> np.ndarray:
    """Reads a binary PPM (P6, maxval 255) written by Film.write_ppm."""
    with open(path, "rb") as f:
        data = f.read()
    parts = data.split(b"\n", 3)
    assert parts[0] == b"P6" and parts[2] == b"255"
    w, h = (int(v) for v in parts[1].split())
    return np.frombuffer(parts[3], np.uint8).reshape(h, w, 3)


class BatchRenderer:
    """Many renders of different scenes in one stream of waves
    (psy_render_batch).  `entries` are dicts with `scene` (a Context holding
    the uploaded scene), `width`, `height`, `spp`, `seed` and `path_length`.
    Films are device tensors owned by this object, accumulated by each
    render() call."""

    def __init__(self, ctx: Context, entries: List[dict], stream_paths: int = 0, block_size: int = 0,
                 use_graph: bool = True):
        torch = _torch()
        dev = torch.device("cuda", ctx.device)
        self.ctx = ctx
        self.entries = entries
        n = len(entries)
        self.films = [torch.zeros(e["height"] * e["width"] * 3, dtype=torch.float32, device=dev) for e in entries]
        self.counts = [torch.zeros(e["height"] * e["width"], dtype=torch.int32, device=dev) for e in entries]
        self._scenes = (C.c_void_p * n)(*[e["scene"].h.value for e in entries])
        self._renders = (_abi.RenderDesc * n)(*[
            _abi.RenderDesc(e["width"], e["height"], e["spp"], e.get("seed", 1), e.get("path_length", 4), 0, 0)
            for e in entries])
        self._xyz = (C.c_void_p * n)(*[f.data_ptr() for f in self.films])
        self._cnt = (C.c_void_p * n)(*[c.data_ptr() for c in self.counts])
        self.desc = _abi.BatchDesc(n, C.cast(self._scenes, C.POINTER(C.c_void_p)),
                                   C.cast(self._renders, C.POINTER(_abi.RenderDesc)),
                                   C.cast(self._xyz, C.POINTER(C.c_void_p)), C.cast(self._cnt, C.POINTER(C.c_void_p)),
                                   stream_paths, block_size, 1 if use_graph else 0)
        self.stats = _abi.RenderStats()

    @property
    def paths(self) -> int:
        return sum(e["width"] * e["height"] * e["spp"] for e in self.entries)

    def zero(self) -> None:
        for f in self.films:
            f.zero_()
        for c in self.counts:
            c.zero_()

    def render(self, stream=None, with_stats: bool = True) -> None:
        self.ctx.check(self.ctx.L.psy_render_batch(self.ctx.h, C.byref(self.desc),
                                                   C.byref(self.stats) if with_stats else None, stream))

    def autotune(self, spp_divisor: int = 16) -> dict:
        t = _abi.BatchTuning()
        self.ctx.check(self.ctx.L.psy_batch_autotune(self.ctx.h, C.byref(self.desc), spp_divisor, C.byref(t)))
        return {"stream_paths": t.stream_paths, "block_size": t.block_size, "ms": t.ms, "trials": t.trials}

    def images(self) -> List[Tuple[np.ndarray, np.ndarray]]:
        _torch().cuda.synchronize(self.ctx.device)
        out = []
        for e, f, c in zip(self.entries, self.films, self.counts):
            out.append((f.cpu().numpy().reshape(e["height"], e["width"], 3),
                        c.cpu().numpy().reshape(e["height"], e["width"]).astype(np.uint32)))
        return out


def flat_indices(scene: Scene) -> Tuple[Dict[int, int], Dict[Tuple[int, str], int], int, int]:
    """The scene indices flatten() gives shaders and objects: shader index by
    id(SurfaceShader), object index by (assembly position, object name), and
    the two counts.  Assemblies are numbered depth first from the root."""
    asm_order: List[Assembly] = []

    def collect(a: Assembly):
        asm_order.append(a)
        for sub in a.assemblies.values():
            collect(sub)

    collect(scene.root)
    shaders: Dict[int, int] = {}
    objects: Dict[Tuple[int, str], int] = {}
    for ai, a in enumerate(asm_order):
        for name in a.objects:
            objects[(ai, name)] = len(objects)
        for inst in a.instances:
            sh = a.shader_of(inst)
            if sh is not None and id(sh) not in shaders:
                shaders[id(sh)] = len(shaders)
    return shaders, objects, len(shaders), len(objects)


class DiffRenderer:
    """Differentiable render of the context's scene (psy_render_diff) and its
    path-replay adjoint (psy_render_adjoint).  shader_param / object_param
    map scene shaders and objects (flat_indices order) to parameter indices
    (-1 = fixed): a shader gets 4 albedo basis weights, a light one emission
    scale.  shader_scale_param (optional) instead gives a shader one
    parameter that scales its RGB albedo."""

    def __init__(self, ctx: Context, width: int, height: int, spp: int, shader_param, object_param,
                 param_count: int, seed: int = 1, path_length: int = 4, stream_paths: int = 0,
                 shader_scale_param=None):
        self.ctx = ctx
        self.desc = _abi.RenderDesc(width, height, spp, seed, path_length, stream_paths, 0)
        self.param_count = int(param_count)
        self._sp = np.ascontiguousarray(np.asarray(shader_param, np.int32))
        self._op = np.ascontiguousarray(np.asarray(object_param, np.int32))
        self._ss = (np.ascontiguousarray(np.asarray(shader_scale_param, np.int32))
                    if shader_scale_param is not None else np.zeros(0, np.int32))
        self.stats = _abi.RenderStats()

    def _diff(self, params) -> _abi.DiffDesc:
        assert params.dtype == _torch().float32 and params.is_cuda and params.numel() == self.param_count
        return _abi.DiffDesc(self.param_count, C.cast(C.c_void_p(params.data_ptr()), _abi.fp),
                             len(self._sp), self._sp.ctypes.data_as(C.POINTER(C.c_int32)),
                             len(self._op), self._op.ctypes.data_as(C.POINTER(C.c_int32)),
                             len(self._ss), self._ss.ctypes.data_as(C.POINTER(C.c_int32)))

    def forward(self, params, xyz=None, counts=None, stream=None, with_stats: bool = False):
        """Film sums (h*w*3) and counts (h*w) of one render, as device tensors."""
        torch = _torch()
        dev = torch.device("cuda", self.ctx.device)
        n = self.desc.width * self.desc.height
        if xyz is None:
            xyz = torch.zeros(n * 3, dtype=torch.float32, device=dev)
        if counts is None:
            counts = torch.zeros(n, dtype=torch.int32, device=dev)
        d = self._diff(params)
        self.ctx.check(self.ctx.L.psy_render_diff(self.ctx.h, C.byref(self.desc), C.byref(d),
                                                  C.c_void_p(xyz.data_ptr()), C.c_void_p(counts.data_ptr()),
                                                  C.byref(self.stats) if with_stats else None, stream))
        return xyz, counts

    def adjoint(self, params, dl_dxyz, grad=None, stream=None, with_stats: bool = False):
        """Adds dL/dparams to grad (a new zero tensor when None) and returns it."""
        torch = _torch()
        if grad is None:
            grad = torch.zeros(self.param_count, dtype=torch.float32, device=params.device)
        dl = dl_dxyz.contiguous().to(torch.float32)
        d = self._diff(params)
        self.ctx.check(self.ctx.L.psy_render_adjoint(self.ctx.h, C.byref(self.desc), C.byref(d),
                                                     C.c_void_p(dl.data_ptr()), C.c_void_p(grad.data_ptr()),
                                                     C.byref(self.stats) if with_stats else None, stream))
        return grad
