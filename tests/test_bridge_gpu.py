"""The drop-in, executed: the reference's own PathTraceIntegrator::integrate
(integrator/path_trace_integrator.cpp:282-384) rendering through a
Tracer::trace that calls psy_trace_host (oracle/ref/psy_bridge.cpp, built as
oracle/_ref/libpsyref_bridged.so with tracer/tracer.cpp left out), against
the same integrator with the reference's own tracer.

Everything but the trace is the reference's code on both sides, so the films
differ only where a traced hit differs (ids exact, t/uv within 4 ulp,
Intersection geometry within a few ulp): per-pixel relative RMSE <= 1e-3,
equal sample counts, equal ray counts.
"""
import multiprocessing as mp
import os
import queue as queue_mod

import numpy as np
import pytest

from psychopath_cpp_b200 import _abi, scenes

pytestmark = pytest.mark.gpu

CASES = {
    "plain": ("plain_scene", {"seed": 1, "res": (80, 60), "spp": 16}, 16, 4),
    "instanced": ("many_light_scene", {"seed": 7, "res": (48, 27), "spp": 8, "n_patches": 80, "n_groups": 40,
                                       "n_lights": 500}, 8, 6),
    "motion": ("motion_patch_scene", {"seed": 1, "res": (64, 48), "spp": 8}, 8, 4),
}


def _child(q, kind, kw, spp, path_length, bridged, psy_lib):
    from oracle import psyref
    if bridged:
        psyref.set_bridge_library(psy_lib)
    sc = getattr(scenes, kind)(**kw)
    ref = psyref.RefScene(scene=sc, bridged=bridged)
    x, c, rays, _ = ref.render(threads=os.cpu_count() or 1, spp=spp, path_length=path_length, seed=sc.seed)
    q.put((x, c, rays))


def _render(kind, kw, spp, path_length, bridged, limit_s=600):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_child, args=(q, kind, kw, spp, path_length, bridged, _abi.LIB_PATH))
    p.start()
    try:
        out = q.get(timeout=limit_s)
    except queue_mod.Empty:
        out = None
    if out is None:
        p.kill()
    p.join()
    return out


@pytest.fixture(scope="module")
def bridged_available(ref_available):
    from oracle import psyref
    if not psyref.available(bridged=True):
        pytest.skip("oracle/_ref/libpsyref_bridged.so not built (make -C oracle bridged)")
    return True


@pytest.mark.parametrize("case", sorted(CASES))
def test_reference_integrator_on_b200_trace(bridged_available, case):
    kind, kw, spp, pl = CASES[case]
    ref = _render(kind, kw, spp, pl, bridged=False)
    mine = _render(kind, kw, spp, pl, bridged=True)
    assert ref is not None and mine is not None
    rx, rc, rrays = ref
    bx, bc, brays = mine
    assert (rc == bc).all()
    assert rrays == brays, (rrays, brays)
    a = bx[..., 1].astype(np.float64)
    b = rx[..., 1].astype(np.float64)
    m = b > 1e-6 * b.max()
    err = float(np.sqrt(np.mean(((a[m] - b[m]) / b[m]) ** 2)))
    assert m.sum() > 0.1 * m.size  # lit pixels (most of the instanced frame is sky)
    assert err <= 1e-3, err
