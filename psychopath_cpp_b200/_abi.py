"""ctypes declarations of the C ABI in include/psy_b200.h.

The shared library is the in-tree build psychopath_cpp_b200/lib/libpsy_b200.so.
Loading fails loudly when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libpsy_b200.so")

PSY_OK = 0
PSY_ERR_ARG = -1
PSY_ERR_OOM = -2
PSY_ERR_DEVICE = -3
PSY_ERR_TIMEOUT = -4
PSY_ERR_STACK_OVERFLOW = -5
PSY_ERR_NAN = -6
PSY_ERR_NO_SCENE = -7

PSY_OBJ_SPHERE, PSY_OBJ_BILINEAR, PSY_OBJ_BICUBIC, PSY_OBJ_SPHERE_LIGHT, PSY_OBJ_RECT_LIGHT = 0, 1, 2, 3, 4
PSY_INSTANCE_OBJECT, PSY_INSTANCE_ASSEMBLY = 0, 1
PSY_SHADER_LAMBERT, PSY_SHADER_EMIT, PSY_SHADER_GTR = 0, 1, 2
PSY_RAY_CAMERA, PSY_RAY_DIFFUSE, PSY_RAY_OCCLUSION = 1, 2, 32

HEADER_PATH = os.path.join(os.path.dirname(HERE), "include", "psy_b200.h")


def header_define(name: str) -> int:
    """An integer #define of include/psy_b200.h, read from the header itself
    so that the binding and the library cannot disagree."""
    import re
    with open(HEADER_PATH) as f:
        m = re.search(r"^#define\s+%s\s+(\d+)u?\b" % re.escape(name), f.read(), re.M)
    if not m:
        raise KeyError(name)
    return int(m.group(1))


PSY_NOALLOC_MAX_RAYS = header_define("PSY_NOALLOC_MAX_RAYS")
PSY_UPLOAD_GPU_BVH = header_define("PSY_UPLOAD_GPU_BVH")

fp = C.POINTER(C.c_float)
u8p = C.POINTER(C.c_uint8)
u16p = C.POINTER(C.c_uint16)
u32p = C.POINTER(C.c_uint32)
u64p = C.POINTER(C.c_uint64)


class ObjectDesc(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("n0", C.c_uint32), ("n1", C.c_uint32), ("n2", C.c_uint32), ("data", fp)]


class InstanceDesc(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("data_index", C.c_uint32), ("transform_index", C.c_uint32),
                ("transform_count", C.c_uint32), ("shader", C.c_int32)]


class AssemblyDesc(C.Structure):
    _fields_ = [("object_count", C.c_uint32), ("objects", C.POINTER(ObjectDesc)),
                ("instance_count", C.c_uint32), ("instances", C.POINTER(InstanceDesc)),
                ("transform_count", C.c_uint32), ("transforms", fp),
                ("child_count", C.c_uint32), ("children", u32p)]


class ShaderDesc(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("color", C.c_float * 3), ("roughness", C.c_float),
                ("tail_shape", C.c_float), ("fresnel", C.c_float)]


class SceneDesc(C.Structure):
    _fields_ = [("cam_transform_count", C.c_uint32), ("cam_transforms", fp),
                ("cam_fov_count", C.c_uint32), ("cam_fovs", fp),
                ("cam_aperture_count", C.c_uint32), ("cam_aperture_radii", fp),
                ("cam_focus_count", C.c_uint32), ("cam_focus_distances", fp),
                ("background", C.c_float * 3), ("dice_rate", C.c_float), ("min_upoly_size", C.c_float),
                ("assembly_count", C.c_uint32), ("assemblies", C.POINTER(AssemblyDesc)),
                ("shader_count", C.c_uint32), ("shaders", C.POINTER(ShaderDesc))]


class SceneStats(C.Structure):
    _fields_ = [("assemblies", C.c_uint32), ("instances", C.c_uint32), ("objects", C.c_uint32),
                ("bvh4_nodes", C.c_uint32), ("light_nodes", C.c_uint32), ("lights", C.c_uint32),
                ("device_bytes", C.c_uint64), ("gpu_bvh4_nodes", C.c_uint32), ("gpu_light_nodes", C.c_uint32)]


class RenderSettings(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("spp", C.c_uint32), ("seed", C.c_uint32),
                ("output_path", C.c_char_p)]


class RaySoA(C.Structure):
    _fields_ = [("o", C.c_void_p), ("d", C.c_void_p), ("odx", C.c_void_p), ("ody", C.c_void_p),
                ("ddx", C.c_void_p), ("ddy", C.c_void_p), ("time", C.c_void_p), ("type", C.c_void_p)]


class HitSoA(C.Structure):
    _fields_ = [(name, C.c_void_p) for name in
                ("hit", "id", "t", "uv", "p", "n", "dpdu", "dpdv", "dndu", "dndv", "backfacing", "light_pdf",
                 "offset", "space", "closure", "closure_color")]


class LightQuerySoA(C.Structure):
    _fields_ = [(name, C.c_void_p) for name in ("n", "u", "v", "pos", "nor", "d", "wavelength", "time")]


class LightSampleSoA(C.Structure):
    _fields_ = [(name, C.c_void_p) for name in ("to_light", "spec", "selection_pdf", "light_pdf", "id")]


class RenderDesc(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("spp", C.c_uint32), ("seed", C.c_uint32),
                ("path_length", C.c_uint32), ("stream_paths", C.c_uint32), ("block_size", C.c_uint32)]


class DiffDesc(C.Structure):
    _fields_ = [("param_count", C.c_uint32), ("params", C.POINTER(C.c_float)), ("shader_count", C.c_uint32),
                ("shader_param", C.POINTER(C.c_int32)), ("object_count", C.c_uint32),
                ("object_param", C.POINTER(C.c_int32)), ("shader_scale_count", C.c_uint32),
                ("shader_scale_param", C.POINTER(C.c_int32))]


class BatchDesc(C.Structure):
    _fields_ = [("count", C.c_uint32), ("scenes", C.POINTER(C.c_void_p)), ("renders", C.POINTER(RenderDesc)),
                ("xyz", C.POINTER(C.c_void_p)), ("counts", C.POINTER(C.c_void_p)), ("stream_paths", C.c_uint32),
                ("block_size", C.c_uint32), ("use_graph", C.c_uint32)]


class BatchTuning(C.Structure):
    _fields_ = [("stream_paths", C.c_uint32), ("block_size", C.c_uint32), ("ms", C.c_float), ("trials", C.c_uint32)]


class RenderStats(C.Structure):
    _fields_ = [("paths", C.c_uint64), ("rays", C.c_uint64), ("launches", C.c_uint32), ("waves", C.c_uint32),
                ("occlusion_rays", C.c_uint64)]


class TraceCounters(C.Structure):
    _fields_ = [("rays", C.c_uint64), ("node_visits", C.c_uint64), ("leaf_visits", C.c_uint64),
                ("patch_iterations", C.c_uint64), ("warp_steps", C.c_uint64), ("lane_steps", C.c_uint64)]

    def as_dict(self) -> dict:
        return {name: int(getattr(self, name)) for name, _ in self._fields_}


# every symbol declared in include/psy_b200.h
EXPORTED = ["psy_ctx_create", "psy_ctx_destroy", "psy_last_error", "psy_version", "psy_scene_upload",
            "psy_scene_upload_ex",
            "psy_scene_stats_get", "psy_build_bvh4", "psy_build_light_tree", "psy_trace", "psy_trace_host", "psy_sync",
            "psy_trace_host_noalloc", "psy_render_batch", "psy_batch_autotune", "psy_render_diff",
            "psy_render_adjoint", "psy_profile_enable", "psy_profile_read", "psy_profile_counters",
            "psy_light_sample", "psy_render", "psy_film_srgb8", "psy_math_check", "psy_file_parse",
            "psy_file_scene_desc", "psy_file_render_settings", "psy_file_free"]

_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("psychopath_cpp_b200: %s is missing; run `python -m psychopath_cpp_b200.build`" % LIB_PATH)
    L = C.CDLL(LIB_PATH)
    L.psy_ctx_create.argtypes = [C.c_int, C.POINTER(C.c_void_p)]
    L.psy_ctx_destroy.argtypes = [C.c_void_p]
    L.psy_ctx_destroy.restype = None
    L.psy_last_error.argtypes = [C.c_void_p]
    L.psy_last_error.restype = C.c_char_p
    L.psy_version.restype = C.c_char_p
    L.psy_scene_upload.argtypes = [C.c_void_p, C.POINTER(SceneDesc)]
    if hasattr(L, "psy_scene_upload_ex"):
        L.psy_scene_upload_ex.argtypes = [C.c_void_p, C.POINTER(SceneDesc), C.c_uint32]
    L.psy_scene_stats_get.argtypes = [C.c_void_p, C.POINTER(SceneStats)]
    L.psy_build_bvh4.argtypes = [C.POINTER(SceneDesc), C.c_uint32, u64p, fp, u64p, u32p, u64p]
    L.psy_build_light_tree.argtypes = [C.POINTER(SceneDesc), C.c_uint32, u64p, u64p, u64p, fp, fp, u64p, fp]
    L.psy_trace.argtypes = [C.c_void_p, C.POINTER(RaySoA), C.c_uint32, C.POINTER(HitSoA), C.c_void_p]
    L.psy_trace_host.argtypes = [C.c_void_p, C.POINTER(RaySoA), C.c_uint32, C.POINTER(HitSoA)]
    L.psy_sync.argtypes = [C.c_void_p, C.c_void_p]
    if hasattr(L, "psy_profile_enable"):
        L.psy_profile_enable.argtypes = [C.c_void_p, C.c_int]
        L.psy_profile_read.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_uint32)]
    if hasattr(L, "psy_profile_counters"):
        L.psy_profile_counters.argtypes = [C.c_void_p, C.POINTER(TraceCounters), C.POINTER(TraceCounters)]
    if hasattr(L, "psy_render_diff"):
        L.psy_render_diff.argtypes = [C.c_void_p, C.POINTER(RenderDesc), C.POINTER(DiffDesc), C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p]
        L.psy_render_adjoint.argtypes = [C.c_void_p, C.POINTER(RenderDesc), C.POINTER(DiffDesc), C.c_void_p,
                                         C.c_void_p, C.c_void_p, C.c_void_p]
    if hasattr(L, "psy_render_batch"):
        L.psy_render_batch.argtypes = [C.c_void_p, C.POINTER(BatchDesc), C.c_void_p, C.c_void_p]
        L.psy_batch_autotune.argtypes = [C.c_void_p, C.POINTER(BatchDesc), C.c_uint32, C.POINTER(BatchTuning)]
    if hasattr(L, "psy_trace_host_noalloc"):
        L.psy_trace_host_noalloc.argtypes = [C.c_void_p, C.POINTER(RaySoA), C.c_uint32, C.POINTER(HitSoA),
                                             C.c_void_p]
    if hasattr(L, "psy_light_sample"):
        L.psy_light_sample.argtypes = [C.c_void_p, C.POINTER(LightQuerySoA), C.c_uint32,
                                       C.POINTER(LightSampleSoA), C.c_void_p]
    if hasattr(L, "psy_math_check"):
        L.psy_math_check.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, fp, fp]
    if hasattr(L, "psy_film_srgb8"):
        L.psy_film_srgb8.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_int, C.c_uint32,
                                     C.c_void_p, C.c_void_p]
    if hasattr(L, "psy_render"):
        L.psy_render.argtypes = [C.c_void_p, C.POINTER(RenderDesc), C.c_void_p, C.c_void_p,
                                 C.POINTER(RenderStats), C.c_void_p]
    if hasattr(L, "psy_file_parse"):
        L.psy_file_parse.argtypes = [C.c_char_p, C.c_size_t, C.c_uint32, C.POINTER(C.c_void_p), C.c_char_p,
                                     C.c_size_t]
        L.psy_file_scene_desc.argtypes = [C.c_void_p]
        L.psy_file_scene_desc.restype = C.POINTER(SceneDesc)
        L.psy_file_render_settings.argtypes = [C.c_void_p, C.POINTER(RenderSettings)]
        L.psy_file_free.argtypes = [C.c_void_p]
        L.psy_file_free.restype = None
    _lib = L
    return L


class PsyError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__("psy error %d: %s" % (code, msg))
        self.code = code
