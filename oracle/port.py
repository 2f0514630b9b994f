"""Test infrastructure: ctypes wrapper over oracle/_build/libpsyoracle.so, the
plain-C restatement of the reference's ray tracing (oracle/c/psy_port.c).

Only tests/, the smoke check and the benchmark's CPU-baseline leg use it,
as the checker.  Scenes are passed in the C ABI's flattened form.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libpsyoracle.so")

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-C", HERE, "port"], check=True, capture_output=True)
        from psychopath_cpp_b200 import _abi
        L = C.CDLL(LIB_PATH)
        fp = C.POINTER(C.c_float)
        L.psyport_box_hit.argtypes = [fp, fp, fp, fp, C.c_float, fp, fp]
        L.psyport_box_hit.restype = C.c_int
        L.psyport_id_push.argtypes = [C.c_uint64, C.c_uint64, C.c_int]
        L.psyport_id_push.restype = C.c_uint64
        L.psyport_trace.argtypes = [C.POINTER(_abi.SceneDesc), C.POINTER(_abi.RaySoA), C.c_uint32, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_void_p]
        L.psyport_libm.argtypes = [C.c_int, C.c_uint32, fp, fp]
        L.psyport_libm.restype = C.c_int
        _lib = L
    return _lib


def trace(scene, rays: dict) -> dict:
    """Brute-force trace of SoA host rays; returns hit, id, t, uv."""
    from psychopath_cpp_b200 import _abi, api
    desc, keep = api.flatten(scene)
    n = len(rays["time"])
    arrs = {k: np.ascontiguousarray(np.asarray(rays[k], np.float32)) for k in ("o", "d", "odx", "ody", "ddx", "ddy",
                                                                                "time")}
    types = np.ascontiguousarray(np.asarray(rays.get("type", np.full(n, 2)), np.uint16))
    rs = _abi.RaySoA(*[arrs[k].ctypes.data_as(C.c_void_p) for k in ("o", "d", "odx", "ody", "ddx", "ddy", "time")],
                     types.ctypes.data_as(C.c_void_p))
    out = {"hit": np.zeros(n, np.uint8), "id": np.zeros(n, np.uint64), "t": np.zeros(n, np.float32),
           "uv": np.zeros((n, 2), np.float32)}
    lib().psyport_trace(C.byref(desc), C.byref(rs), n, out["hit"].ctypes.data_as(C.c_void_p),
                        out["id"].ctypes.data_as(C.c_void_p), out["t"].ctypes.data_as(C.c_void_p),
                        out["uv"].ctypes.data_as(C.c_void_p))
    del keep
    return out


def box_hit(lo, hi, o, d, tmax=float("inf")):
    """BBox::intersect_ray of the restatement: (hit, t0, t1)."""
    f = C.c_float * 3
    t0, t1 = C.c_float(), C.c_float()
    h = lib().psyport_box_hit(f(*lo), f(*hi), f(*o), f(*d), tmax, C.byref(t0), C.byref(t1))
    return bool(h), t0.value, t1.value


def id_push(idv: int, sub: int, bits: int) -> int:
    return int(lib().psyport_id_push(idv, sub, bits))


LIBM_FUNCTIONS = ("sin", "cos", "acos", "asin", "exp")


def libm(fn: str, x: np.ndarray) -> np.ndarray:
    """The host C library's float `fn` (sincosf / acosf / asinf / expf, as
    the reference's std:: calls of a float resolve) of every element."""
    x = np.ascontiguousarray(x, np.float32).ravel()
    out = np.empty_like(x)
    fp = C.POINTER(C.c_float)
    rc = lib().psyport_libm(LIBM_FUNCTIONS.index(fn), x.size, x.ctypes.data_as(fp), out.ctypes.data_as(fp))
    assert rc == 0
    return out
