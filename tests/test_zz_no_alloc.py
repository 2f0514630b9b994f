"""psy_trace_host_noalloc against psy_trace_host: identical results on two
calls in a row (a full-capacity call, then a smaller one with another field
set, so nothing of the first call may leak into the second), and a clear
error for a request beyond the fixed capacity.  Collected last so that it
also runs after every other GPU test in the same process."""
import numpy as np
import pytest

from psychopath_cpp_b200 import _abi, api, scenes
from tests import parity

pytestmark = pytest.mark.gpu

MAX_RAYS = _abi.PSY_NOALLOC_MAX_RAYS  # read from include/psy_b200.h
ALL_FIELDS = tuple(api.HIT_FIELDS)


def _same(a: dict, b: dict):
    assert a.keys() == b.keys()
    for k in a:
        assert a[k].dtype == b[k].dtype and a[k].shape == b[k].shape, k
        np.testing.assert_array_equal(a[k].view(np.uint8), b[k].view(np.uint8), err_msg=k)


def test_noalloc_matches_trace_host_on_consecutive_calls(ctx):
    sc = scenes.plain_scene(seed=5)
    ctx.upload(sc)
    tr = api.Tracer(ctx)
    first = parity.random_rays(MAX_RAYS, (-8, -8, -1), (8, 8, 8), seed=21, occl_frac=0.3, width=0.01)
    a0 = tr.trace(first, fields=ALL_FIELDS)
    b0 = tr.trace_noalloc(first, fields=ALL_FIELDS)
    _same(a0, b0)
    assert int(a0["hit"].sum()) > 1000

    second = parity.random_rays(20000, (-6, -6, 0), (6, 6, 6), seed=22, occl_frac=0.5, width=0.02)
    fields = ("hit", "id", "t", "n", "closure")
    a1 = tr.trace(second, fields=fields)
    b1 = tr.trace_noalloc(second, fields=fields)
    _same(a1, b1)


def test_noalloc_patch_scene(ctx):
    sc = scenes.heightfield_scene(n=64, seed=3)
    ctx.upload(sc)
    tr = api.Tracer(ctx)
    for seed, count in ((1, 40000), (2, 3000)):
        rays = scenes.heightfield_rays(count, n=64, seed=seed)
        _same(tr.trace(rays, fields=("hit", "id", "t", "uv", "p")),
              tr.trace_noalloc(rays, fields=("hit", "id", "t", "uv", "p")))


def test_noalloc_rejects_more_than_capacity(ctx):
    sc = scenes.plain_scene(seed=5)
    ctx.upload(sc)
    rays = parity.random_rays(MAX_RAYS + 1, (-8, -8, -1), (8, 8, 8), seed=23)
    with pytest.raises(_abi.PsyError) as e:
        api.Tracer(ctx).trace_noalloc(rays)
    assert e.value.code == _abi.PSY_ERR_ARG
    assert "capacity" in str(e.value)


def test_noalloc_hit_id_t_only_and_no_hits(ctx):
    """Only hit, id and t requested (no geometry epilogue), and a call with
    no hit arrays at all (hits = NULL), each against psy_trace_host."""
    sc = scenes.many_light_scene(3, res=(32, 18), spp=1, n_patches=60, n_groups=20, n_lights=200)
    ctx.upload(sc)
    tr = api.Tracer(ctx)
    rays = parity.random_rays(30000, (-6, -5, 0.0), (6, 5, 4), seed=31, occl_frac=0.4, width=0.01)
    fields = ("hit", "id", "t")
    _same(tr.trace(rays, fields=fields), tr.trace_noalloc(rays, fields=fields))
    assert tr.trace_noalloc(rays, fields=None) == {}
    # the array still serves a full call after the call without hits
    _same(tr.trace(rays, fields=ALL_FIELDS), tr.trace_noalloc(rays, fields=ALL_FIELDS))


def test_noalloc_zero_rays_is_a_warm_up(ctx):
    """n = 0 only makes the fixed array resident: it succeeds and returns
    empty results."""
    rays = parity.random_rays(1, (0, 0, 0), (1, 1, 1), seed=1)
    empty = {k: v[:0] for k, v in rays.items()}
    out = api.Tracer(ctx).trace_noalloc(empty, fields=("hit", "id", "t"))
    assert all(v.shape[0] == 0 for v in out.values())
