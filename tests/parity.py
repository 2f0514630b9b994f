"""Shared helpers for parity tests: seeded ray streams and hit comparison.

Parity bar (per ray): closest-hit instance ids bit-exact except near-ties
whose hit distances differ by under 1e-6 relative; hit t and uv within 4 ulp;
occlusion results (hit / no hit) identical.
"""
from __future__ import annotations

import numpy as np

T_ULP = 4
UV_ULP = 4
NEAR_TIE_REL = 1e-6


def ulp_diff(a, b) -> np.ndarray:
    """Distance in units in the last place between float32 arrays."""
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    ia = a.view(np.int32).astype(np.int64)
    ib = b.view(np.int32).astype(np.int64)
    ia = np.where(ia < 0, np.int64(-2**31) - ia, ia)
    ib = np.where(ib < 0, np.int64(-2**31) - ib, ib)
    d = np.abs(ia - ib)
    both_inf = np.isinf(a) & np.isinf(b) & (np.sign(a) == np.sign(b))
    return np.where(both_inf, 0, d)


def random_rays(n: int, lo, hi, seed: int, occl_frac: float = 0.0, width: float = 0.0,
                spread: float = 0.001) -> dict:
    """Rays with origins uniform in the box [lo, hi], uniform directions,
    and camera-like differentials (zero origin width, direction spread)."""
    rng = np.random.default_rng(seed)
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    o = lo + rng.uniform(0, 1, (n, 3)) * (hi - lo)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    occl = rng.uniform(0, 1, n) < occl_frac
    # occlusion rays: finite segments (the reference's shadow rays span t in [0,1))
    seg = rng.uniform(0.5, 8.0, n)
    d = np.where(occl[:, None], d * seg[:, None], d)
    f = np.float32
    z = np.zeros((n, 3), f)
    odx = z.copy()
    ody = z.copy()
    if width > 0:
        odx[:, 0] = width
        ody[:, 1] = width
    ddx = np.zeros((n, 3), f)
    ddy = np.zeros((n, 3), f)
    ddx[:, 0] = spread
    ddy[:, 1] = spread
    return {"o": o.astype(f), "d": d.astype(f), "odx": odx, "ody": ody, "ddx": ddx, "ddy": ddy,
            "time": rng.uniform(0, 1, n).astype(f),
            "type": np.where(occl, 32, 2).astype(np.uint16)}


def concat_rays(*rs) -> dict:
    return {k: np.concatenate([r[k] for r in rs]) for k in rs[0]}


def compare_trace(ref: dict, mine: dict, types: np.ndarray, uv_mask=None) -> dict:
    """Compares reference (oracle) and CUDA hits; returns counts of each
    kind of disagreement plus the near-tie count.

    `uv_mask` selects the rays whose uv is compared.  The reference leaves
    Intersection fields that a closer hit does not write (uv of a light hit,
    light_pdf of a surface hit) holding values from farther candidates, so
    uv is only meaningful for surface hits."""
    occl = types == 32
    rh = ref["hit"].astype(bool)
    mh = mine["hit"].astype(bool)
    rep = {"n": int(len(types)), "hit_mismatch": int((rh != mh).sum()),
           "occl_mismatch": int(((rh != mh) & occl).sum())}
    both = rh & mh & ~occl
    rt = ref["t"][both]
    mt = mine["t"][both]
    ids_eq = ref["id"][both] == mine["id"][both]
    rel = np.abs(rt.astype(np.float64) - mt.astype(np.float64)) / np.maximum(np.abs(rt.astype(np.float64)), 1e-30)
    near_tie = (~ids_eq) & (rel < NEAR_TIE_REL)
    rep["closest_hits"] = int(both.sum())
    rep["id_mismatch"] = int((~ids_eq & ~near_tie).sum())
    rep["near_ties"] = int(near_tie.sum())
    tu = ulp_diff(rt[ids_eq], mt[ids_eq])
    rep["t_ulp_max"] = int(tu.max()) if tu.size else 0
    rep["t_over"] = int((tu > T_ULP).sum())
    if "uv" in ref and "uv" in mine:
        sel = ids_eq if uv_mask is None else ids_eq & uv_mask[both]
        uu = ulp_diff(ref["uv"][both][sel], mine["uv"][both][sel])
        rep["uv_ulp_max"] = int(uu.max()) if uu.size else 0
        rep["uv_over"] = int((uu > UV_ULP).sum())
    return rep


def assert_parity(rep: dict, allow_near_ties: float = 1e-3):
    assert rep["hit_mismatch"] == 0, rep
    assert rep["id_mismatch"] == 0, rep
    assert rep["near_ties"] <= max(2, allow_near_ties * rep["closest_hits"]), rep
    assert rep["t_over"] == 0, rep
    assert rep.get("uv_over", 0) == 0, rep
