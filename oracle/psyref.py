"""Test infrastructure: ctypes wrapper over oracle/_ref/libpsyref.so, the
reference renderer's own code compiled from its sources (see oracle/Makefile).

Only tests/, the smoke check and the benchmark's CPU-baseline leg use this,
and only as the checker or the timed CPU baseline, never as the product.
"""
from __future__ import annotations

import ctypes as C
import os
import tempfile
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libpsyref.so")
# The same reference build with tracer/tracer.cpp replaced by the reference-side
# bridge (oracle/ref/psy_bridge.cpp): its Tracer::trace calls libpsy_b200.
BRIDGED_LIB_PATH = os.path.join(HERE, "_ref", "libpsyref_bridged.so")

_libs = {}


def available(bridged: bool = False) -> bool:
    return os.path.exists(BRIDGED_LIB_PATH if bridged else LIB_PATH)


def lib(bridged: bool = False):
    """The reference build (or its bridged form, whose tracer runs on the
    B200 library at `psy_lib`, set with set_bridge_library first)."""
    if bridged not in _libs:
        path = BRIDGED_LIB_PATH if bridged else LIB_PATH
        if not os.path.exists(path):
            raise RuntimeError("%s is not built (make -C oracle %s)" % (path, "bridged" if bridged else "ref"))
        L = C.CDLL(path)
        vp, sz, fp, u64p, u32p, u8p, u16p, dp = (C.c_void_p, C.c_size_t, C.POINTER(C.c_float),
                                                  C.POINTER(C.c_uint64), C.POINTER(C.c_uint32),
                                                  C.POINTER(C.c_uint8), C.POINTER(C.c_uint16),
                                                  C.POINTER(C.c_double))
        L.psyref_load.restype = vp
        L.psyref_load.argtypes = [C.c_char_p]
        L.psyref_free.argtypes = [vp]
        L.psyref_info.argtypes = [vp] + [C.POINTER(C.c_int)] * 4
        L.psyref_get_dice_rate.restype = C.c_float
        L.psyref_set_dice_rate.argtypes = [C.c_float]
        L.psyref_render.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, fp, u32p, u64p, dp]
        L.psyref_trace.restype = C.c_double
        L.psyref_trace.argtypes = [vp, sz, fp, u16p, C.c_int, sz, u8p, u64p, fp]
        L.psyref_light_sample.argtypes = [vp, sz, fp, fp, u64p]
        L.psyref_camera_ray.argtypes = [vp, sz, fp, fp]
        L.psyref_halton.argtypes = [sz, u32p, u32p, fp]
        L.psyref_sampler.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, fp, u32p]
        L.psyref_eval.argtypes = [C.c_int, sz, fp, C.c_int, fp, C.c_int]
        L.psyref_film_srgb8.argtypes = [fp, u32p, C.c_int, C.c_int, u8p]
        L.psyref_assembly_count.restype = C.c_int
        L.psyref_assembly_count.argtypes = [vp]
        L.psyref_bvh4_node_count.restype = sz
        L.psyref_bvh4_node_count.argtypes = [vp, C.c_int]
        L.psyref_bvh4_nodes.argtypes = [vp, C.c_int, fp, u64p, u32p, u64p]
        L.psyref_lighttree_node_count.restype = sz
        L.psyref_lighttree_node_count.argtypes = [vp, C.c_int]
        L.psyref_lighttree_bounds_count.restype = sz
        L.psyref_lighttree_bounds_count.argtypes = [vp, C.c_int]
        L.psyref_lighttree_nodes.argtypes = [vp, C.c_int, u64p, fp, fp]
        L.psyref_lighttree_totals.argtypes = [vp, C.c_int, u64p, fp]
        if bridged:
            L.psy_bridge_set_library.argtypes = [C.c_char_p]
        _libs[bridged] = L
    return _libs[bridged]


def set_bridge_library(psy_lib_path: str) -> None:
    """Which libpsy_b200.so the bridged reference traces with."""
    lib(True).psy_bridge_set_library(psy_lib_path.encode())


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t)) if a is not None else None


def rays_to_flat(rays: dict) -> np.ndarray:
    n = len(rays["time"])
    flat = np.empty((n, 19), np.float32)
    flat[:, 0:3] = rays["o"]
    flat[:, 3:6] = rays["d"]
    flat[:, 6:9] = rays["odx"]
    flat[:, 9:12] = rays["ody"]
    flat[:, 12:15] = rays["ddx"]
    flat[:, 15:18] = rays["ddy"]
    flat[:, 18] = rays["time"]
    return flat


class RefScene:
    """A parsed and finalized reference Scene."""

    def __init__(self, psy_path: Optional[str] = None, scene=None, bridged: bool = False):
        self.bridged = bridged
        L = self.L = lib(bridged)
        tmp = None
        if psy_path is None:
            fd, tmp = tempfile.mkstemp(suffix=".psy")
            with os.fdopen(fd, "w") as f:
                f.write(scene.to_psy())
            psy_path = tmp
        # The reference parser writes DicingRate into a global; reset it first.
        L.psyref_set_dice_rate(0.25)
        self.h = L.psyref_load(psy_path.encode())
        if tmp:
            os.unlink(tmp)
        if not self.h:
            raise RuntimeError("reference parser failed on %s" % psy_path)
        a = [C.c_int() for _ in range(4)]
        L.psyref_info(self.h, *[C.byref(x) for x in a])
        self.res_x, self.res_y, self.spp, self.seed = [x.value for x in a]
        self.dice_rate = L.psyref_get_dice_rate()

    def close(self):
        if self.h:
            self.L.psyref_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _use(self):
        self.L.psyref_set_dice_rate(self.dice_rate)

    def render(self, threads: int = 0, spp: int = 0, path_length: int = 4, seed: int = -1):
        """Returns (xyz sums [h,w,3], counts [h,w], rays_shot, seconds)."""
        self._use()
        threads = threads or os.cpu_count() or 1
        xyz = np.zeros((self.res_y, self.res_x, 3), np.float32)
        cnt = np.zeros((self.res_y, self.res_x), np.uint32)
        rays = C.c_uint64()
        secs = C.c_double()
        self.L.psyref_render(self.h, threads, spp, path_length, seed, _p(xyz, C.c_float), _p(cnt, C.c_uint32),
                            C.byref(rays), C.byref(secs))
        return xyz, cnt, rays.value, secs.value

    def trace(self, rays: dict, threads: int = 0, chunk: int = 65536, full: bool = True):
        """Tracer::trace on SoA world rays; returns dict(hit, id, out[, seconds])."""
        self._use()
        flat = np.ascontiguousarray(rays_to_flat(rays))
        types = np.ascontiguousarray(rays["type"].astype(np.uint16))
        n = flat.shape[0]
        hit = np.zeros(n, np.uint8)
        ids = np.zeros(n, np.uint64)
        out = np.zeros((n, 48), np.float32) if full else None
        secs = self.L.psyref_trace(self.h, n, _p(flat, C.c_float), _p(types, C.c_uint16), threads or os.cpu_count(),
                                  chunk, _p(hit, C.c_uint8), _p(ids, C.c_uint64), _p(out, C.c_float))
        res = {"hit": hit, "id": ids, "seconds": secs}
        if full:
            res["out"] = out
            res["t"] = out[:, 0].copy()
            res["uv"] = out[:, 1:3].copy()
        return res

    def light_sample(self, q: np.ndarray):
        q = np.ascontiguousarray(q, np.float32).reshape(-1, 15)
        out = np.zeros((q.shape[0], 14), np.float32)
        ids = np.zeros(q.shape[0], np.uint64)
        self.L.psyref_light_sample(self.h, q.shape[0], _p(q, C.c_float), _p(out, C.c_float), _p(ids, C.c_uint64))
        return out, ids

    def camera_rays(self, args: np.ndarray) -> np.ndarray:
        args = np.ascontiguousarray(args, np.float32).reshape(-1, 7)
        out = np.zeros((args.shape[0], 19), np.float32)
        self.L.psyref_camera_ray(self.h, args.shape[0], _p(args, C.c_float), _p(out, C.c_float))
        return out

    def assembly_count(self) -> int:
        return self.L.psyref_assembly_count(self.h)

    def bvh4_nodes(self, assembly: int = 0):
        n = self.L.psyref_bvh4_node_count(self.h, assembly)
        b = np.zeros((n, 24), np.float32)
        ch = np.zeros((n, 3), np.uint64)
        ts = np.zeros(n, np.uint32)
        di = np.zeros(n, np.uint64)
        if n:
            self.L.psyref_bvh4_nodes(self.h, assembly, _p(b, C.c_float), _p(ch, C.c_uint64), _p(ts, C.c_uint32),
                                    _p(di, C.c_uint64))
        return {"bounds": b, "child": ch, "ts": ts, "data_index": di}

    def light_tree(self, assembly: int = 0):
        n = self.L.psyref_lighttree_node_count(self.h, assembly)
        nb = self.L.psyref_lighttree_bounds_count(self.h, assembly)
        meta = np.zeros((n, 6), np.uint64)
        en = np.zeros(n, np.float32)
        bb = np.zeros((max(nb, 1), 6), np.float32)
        if n:
            self.L.psyref_lighttree_nodes(self.h, assembly, _p(meta, C.c_uint64), _p(en, C.c_float),
                                         _p(bb, C.c_float))
        cnt = C.c_uint64()
        tot = C.c_float()
        self.L.psyref_lighttree_totals(self.h, assembly, C.byref(cnt), C.byref(tot))
        return {"meta": meta, "energy": en, "bounds": bb[:nb], "light_count": cnt.value, "total_energy": tot.value}


def halton(dims, idx) -> np.ndarray:
    dims = np.ascontiguousarray(dims, np.uint32)
    idx = np.ascontiguousarray(idx, np.uint32)
    out = np.zeros(len(dims), np.float32)
    lib().psyref_halton(len(dims), _p(dims, C.c_uint32), _p(idx, C.c_uint32), _p(out, C.c_float))
    return out


def sampler(x, y, s, seed, count):
    out = np.zeros(count, np.float32)
    off = C.c_uint32()
    lib().psyref_sampler(x, y, s, seed, count, _p(out, C.c_float), C.byref(off))
    return out, off.value


def eval_fn(fn: int, inputs: np.ndarray, out_stride: int) -> np.ndarray:
    inputs = np.ascontiguousarray(inputs, np.float32)
    n, k = inputs.shape
    out = np.zeros((n, out_stride), np.float32)
    lib().psyref_eval(fn, n, _p(inputs, C.c_float), k, _p(out, C.c_float), out_stride)
    return out


def film_srgb8(xyz: np.ndarray, counts: np.ndarray) -> np.ndarray:
    """Film::scanline_image_8bbc of a film with these sums (h, w, 3) and
    counts (h, w), with the reference film's own (clock-seeded) dither."""
    h, w = counts.shape
    xyz = np.ascontiguousarray(xyz, np.float32)
    counts = np.ascontiguousarray(counts, np.uint32)
    out = np.zeros((h, w, 3), np.uint8)
    lib().psyref_film_srgb8(_p(xyz, C.c_float), _p(counts, C.c_uint32), w, h, _p(out, C.c_uint8))
    return out
