"""Parity at the benchmark configurations' own sizes and on the headline
scene itself, against the reference's own code (oracle/_ref).

* The 4,194,304-ray stream against the 256x256 bilinear heightfield (the
  trace benchmark, whole): per-ray parity (ids bit-exact, t/uv within 4 ulp).
* The plain scene at 320x240, 16 spp, 4 segments (the CPU-runnable render,
  whole): per-pixel relative RMSE <= 1e-5 and the reference's ray count.
* The 720p benchmark scene at full density (2,000 bicubic patches, 500
  instanced motion-blurred sphere groups, 10,000 sphere lights, depth of
  field, camera motion, 6 segments) on a 64x36 frame at 1024 spp:
  per-pixel relative RMSE <= 1e-3, the image bar at 1024 spp, and in fact
  <= 1e-5 with the reference's exact ray count (and so at 8 and 64 spp).

The reference renders run in spawned child processes with a time limit: on
some sampler seeds a ray with NaN differentials makes the reference's patch
bisection run without end (it does at seeds 1, 2, 5 and 6 of the 64x36x1024
frame), so the headline test takes the first of a fixed list of seeds whose
reference render finishes.
"""
import multiprocessing as mp
import os
import queue as queue_mod

import numpy as np
import pytest

from psychopath_cpp_b200 import api, scenes
from tests import parity

pytestmark = pytest.mark.gpu

IMAGE_REL_RMSE = 1e-3
# renders here reproduce the reference path for path (the device restates
# the host C library's float math): what is left is film summation order
STRICT_REL_RMSE = 1e-5
HEADLINE_SEEDS = (3, 4, 7, 8)


def rel_rmse(mine, ref):
    """Per-pixel relative RMSE over pixels with signal (luminance Y)."""
    a = mine[..., 1].astype(np.float64)
    b = ref[..., 1].astype(np.float64)
    m = b > 1e-6 * max(b.max(), 1e-30)
    return float(np.sqrt(np.mean(((a[m] - b[m]) / b[m]) ** 2))), int(m.sum())


def _scene(kind, kw):
    return getattr(scenes, kind)(**kw)


def _ref_child(q, kind, kw, spp, path_length, seed):
    from oracle import psyref
    ref = psyref.RefScene(scene=_scene(kind, kw))
    x, c, rays, secs = ref.render(threads=os.cpu_count() or 1, spp=spp, path_length=path_length, seed=seed)
    q.put((x, c, rays))


def ref_render_bounded(kind, kw, spp, path_length, seed, limit_s):
    """The reference's PathTraceIntegrator::integrate in a spawned child
    (no CUDA state inherited); None when it does not finish in time."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_ref_child, args=(q, kind, kw, spp, path_length, seed))
    p.start()
    try:
        out = q.get(timeout=limit_s)
    except queue_mod.Empty:
        out = None
    if out is None:
        p.kill()
    p.join()
    return out


def _render_ours(ctx, sc, spp, path_length, seed):
    ctx.upload(sc)
    integ = api.PathTraceIntegrator(ctx, sc.res_x, sc.res_y, spp, seed=seed, path_length=path_length)
    x, c = integ.integrate()
    return x, c, int(integ.stats.rays)


def test_trace_benchmark_stream_full_size(ctx, ref_available):
    """All 4,194,304 rays of the trace benchmark against the 256x256
    heightfield: the reference's Tracer::trace and psy_trace_host agree ray
    for ray."""
    from oracle import psyref
    sc = scenes.heightfield_scene(256, seed=7)
    rays = scenes.heightfield_rays(4194304, n=256, seed=11)
    ref = psyref.RefScene(scene=sc).trace(rays, threads=os.cpu_count() or 1, chunk=65536)
    del ref["out"]
    ctx.upload(sc)
    mine = api.Tracer(ctx).trace(rays, fields=("hit", "id", "t", "uv"))
    rep = parity.compare_trace(ref, mine, rays["type"])
    parity.assert_parity(rep)
    assert rep["closest_hits"] > 3_000_000, rep


def test_plain_render_full_size(ctx, ref_available):
    """The plain scene at its configured 320x240, 16 spp, 4 segments."""
    kw = {"seed": 1}
    sc = _scene("plain_scene", kw)
    assert (sc.res_x, sc.res_y, sc.spp) == (320, 240, 16)
    out = ref_render_bounded("plain_scene", kw, 16, 4, 1, 600)
    assert out is not None, "reference render did not finish"
    rx, rc, rrays = out
    mx, mc, mrays = _render_ours(ctx, sc, 16, 4, 1)
    assert (rc == mc).all()
    err, npx = rel_rmse(mx, rx)
    assert npx > 50000
    assert err <= STRICT_REL_RMSE, err
    assert int(rrays) == int(mrays), (rrays, mrays)


def _headline_kw(res):
    return {"seed": 3, "res": res, "spp": 1}


@pytest.mark.parametrize("spp", [8, 64])
def test_headline_scene_low_spp(ctx, ref_available, spp):
    """The benchmark scene at full density, 64x36, at 8 and 64 spp (seed 3):
    the same sample sequences in both renderers, path for path."""
    kw = _headline_kw((64, 36))
    out = ref_render_bounded("many_light_scene", kw, spp, 6, HEADLINE_SEEDS[0], 600)
    assert out is not None, "reference render did not finish"
    rx, rc, rrays = out
    mx, mc, mrays = _render_ours(ctx, _scene("many_light_scene", kw), spp, 6, HEADLINE_SEEDS[0])
    assert (rc == mc).all()
    err, npx = rel_rmse(mx, rx)
    assert npx > 1500
    assert err <= STRICT_REL_RMSE, err
    assert int(rrays) == int(mrays), (rrays, mrays)


def test_headline_scene_1024spp(ctx, ref_available):
    """The north-star image bar on the benchmark scene itself: 64x36 at
    1024 spp, 6 segments, per-pixel relative RMSE <= 1e-3."""
    kw = _headline_kw((64, 36))
    out, seed = None, None
    for s in HEADLINE_SEEDS:
        out = ref_render_bounded("many_light_scene", kw, 1024, 6, s, 300)
        if out is not None:
            seed = s
            break
    assert out is not None, "the reference render stalled on every seed tried"
    rx, rc, rrays = out
    mx, mc, mrays = _render_ours(ctx, _scene("many_light_scene", kw), 1024, 6, seed)
    assert (rc == mc).all()
    err, npx = rel_rmse(mx, rx)
    assert npx > 1500
    assert err <= IMAGE_REL_RMSE, (seed, err)
    # and path for path: the stated bar with two orders of magnitude to spare
    assert err <= STRICT_REL_RMSE, (seed, err)
    assert int(rrays) == int(mrays), (rrays, mrays)
