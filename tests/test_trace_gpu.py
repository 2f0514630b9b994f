"""Parity of psy_trace (CUDA) with the reference's Tracer::trace on the same
ray streams: closest-hit ids bit-exact (near-ties excepted), t and uv within
4 ulp, occlusion flags identical, and the reference's Intersection geometry
(p, n, dpdu/dpdv, offset, light pdf, closure) within small ulp bounds.
"""
import numpy as np
import pytest

from psychopath_cpp_b200 import api, scenes
from tests import parity

pytestmark = pytest.mark.gpu


def _trace_both(ctx, sc, rays, fields=("hit", "id", "t", "uv")):
    from oracle import psyref
    ref = psyref.RefScene(scene=sc).trace(rays, threads=8)
    ctx.upload(sc)
    mine = api.Tracer(ctx).trace(rays, fields=fields)
    return ref, mine


def _camera_rays(sc, n, seed):
    from oracle import psyref
    r = psyref.RefScene(scene=sc)
    rng = np.random.default_rng(seed)
    w, h = sc.res_x, sc.res_y
    args = np.zeros((n, 7), np.float32)
    args[:, 0] = rng.uniform(-1, 1, n)
    args[:, 1] = rng.uniform(-h / w, h / w, n)
    args[:, 2] = 2.0 / w
    args[:, 3] = 2.0 * (h / w) / h
    args[:, 4] = rng.uniform(0, 1, n)
    args[:, 5] = rng.uniform(0, 1, n)
    args[:, 6] = rng.uniform(0, 1, n)
    flat = r.camera_rays(args)
    return {"o": flat[:, 0:3], "d": flat[:, 3:6], "odx": flat[:, 6:9], "ody": flat[:, 9:12],
            "ddx": flat[:, 12:15], "ddy": flat[:, 15:18], "time": flat[:, 18].copy(),
            "type": np.ones(n, np.uint16)}


def test_plain_scene_camera_rays(ctx, ref_available):
    sc = scenes.plain_scene(1)
    rays = _camera_rays(sc, 20000, 5)
    ref, mine = _trace_both(ctx, sc, rays)
    rep = parity.compare_trace(ref, mine, rays["type"])
    parity.assert_parity(rep)
    assert rep["closest_hits"] > 10000


def test_plain_scene_random_and_shadow_rays(ctx, ref_available):
    sc = scenes.plain_scene(2)
    rays = parity.random_rays(30000, (-6, -6, 0.01), (6, 6, 3), seed=9, occl_frac=0.5)
    ref, mine = _trace_both(ctx, sc, rays)
    rep = parity.compare_trace(ref, mine, rays["type"])
    parity.assert_parity(rep)
    assert rep["occl_mismatch"] == 0


def test_heightfield_rays(ctx, ref_available):
    sc = scenes.heightfield_scene(32, seed=4)
    rays = scenes.heightfield_rays(20000, n=32, seed=12)
    ref, mine = _trace_both(ctx, sc, rays)
    rep = parity.compare_trace(ref, mine, rays["type"])
    parity.assert_parity(rep)
    assert rep["closest_hits"] > 15000


def test_heightfield_occlusion(ctx, ref_available):
    sc = scenes.heightfield_scene(24, seed=5)
    rays = scenes.heightfield_rays(8000, n=24, seed=13)
    rays["type"][:] = 32
    rays["d"] = rays["d"] * np.float32(3.0)
    ref, mine = _trace_both(ctx, sc, rays, fields=("hit",))
    assert (ref["hit"] == mine["hit"]).all()
    assert 0 < ref["hit"].sum() < len(ref["hit"])


def test_instanced_motion_bicubic_scene(ctx, ref_available):
    sc = scenes.many_light_scene(3, res=(64, 36), spp=1, n_patches=120, n_groups=60, n_lights=400)
    cam = _camera_rays(sc, 12000, 7)
    rnd = parity.random_rays(12000, (-8, -6, -0.5), (8, 6, 5), seed=3, occl_frac=0.4)
    rays = parity.concat_rays(cam, rnd)
    ref, mine = _trace_both(ctx, sc, rays, fields=("hit", "id", "t", "uv", "closure"))
    # every surface in this scene carries a Lambert shader, so Emit = sphere light
    rep = parity.compare_trace(ref, mine, rays["type"], uv_mask=mine["closure"] != 2)
    parity.assert_parity(rep)


def test_motion_patches(ctx, ref_available):
    """Bilinear and bicubic patches with two time samples: the bisection
    lerps each sub-patch's bounds to the ray time."""
    sc = scenes.motion_patch_scene(2)
    cam = _camera_rays(sc, 12000, 5)
    rnd = parity.random_rays(12000, (-4, -4, 0.05), (4, 4, 2), seed=9, occl_frac=0.4)
    rays = parity.concat_rays(cam, rnd)
    ref, mine = _trace_both(ctx, sc, rays, fields=("hit", "id", "t", "uv", "closure"))
    rep = parity.compare_trace(ref, mine, rays["type"], uv_mask=mine["closure"] != 2)
    parity.assert_parity(rep)
    assert rep["closest_hits"] > 10000


GEOM = ("hit", "id", "t", "uv", "p", "n", "dpdu", "dpdv", "backfacing", "light_pdf", "offset", "space",
        "closure", "closure_color")


@pytest.mark.parametrize("which", ["plain", "heightfield", "instanced"])
def test_intersection_fields(ctx, ref_available, which):
    if which == "plain":
        sc = scenes.plain_scene(3)
        rays = parity.random_rays(6000, (-6, -6, 0.01), (6, 6, 3), seed=21)
    elif which == "heightfield":
        sc = scenes.heightfield_scene(16, seed=2)
        rays = scenes.heightfield_rays(6000, n=16, seed=22)
    else:
        sc = scenes.many_light_scene(5, res=(64, 36), spp=1, n_patches=60, n_groups=30, n_lights=100)
        rays = parity.random_rays(6000, (-8, -6, -0.5), (8, 6, 5), seed=23)
    ref, mine = _trace_both(ctx, sc, rays, fields=GEOM)
    out = ref["out"]
    both = ref["hit"].astype(bool) & mine["hit"].astype(bool) & (ref["id"] == mine["id"])
    assert both.sum() > 100
    # closure kind and colour are exact
    assert (out[both, 42].astype(np.uint8) == mine["closure"][both]).all()
    np.testing.assert_array_equal(out[both, 43:46], mine["closure_color"][both])
    assert (out[both, 21].astype(np.uint8) == mine["backfacing"][both]).all()
    # geometry: patches and untransformed spheres are bit-exact; acos-based sphere
    # uv and the transformed-instance world data stay within a few ulp
    for name, sl in (("p", slice(3, 6)), ("n", slice(6, 9)), ("offset", slice(23, 26)),
                     ("space", slice(26, 42))):
        d = parity.ulp_diff(out[both, sl], mine[name][both])
        assert np.percentile(d, 99.9) <= 4, (name, int(d.max()))
    # light_pdf is only written by light hits (the reference keeps the value of
    # a farther light candidate on surface hits)
    light = both & (mine["closure"] == 2) & (mine["light_pdf"] != 9999.0)
    lp = parity.ulp_diff(out[light, 22], mine["light_pdf"][light])
    assert lp.size == 0 or lp.max() <= 4
    surf = both & (mine["closure"] != 2)
    uv = parity.ulp_diff(out[surf, 1:3], mine["uv"][surf])
    assert uv.size == 0 or np.percentile(uv, 99.9) <= 4


def test_rays_along_patch_faces(ctx, ref_available):
    """Rays that run exactly along a face of the ground patch's sub-boxes (a
    zero direction component with the origin on the face, e.g. a pinhole
    camera ray through the image centre column) make the reference's slab
    test report NaN-distance hits it can never take; the bisection skips
    those subtrees, with the same results as the reference."""
    sc = scenes.plain_scene(seed=1)
    n = 6
    o = np.array([[0.0, -15.0, 7.0]] * n, np.float32)
    d = np.array([[0.0, 0.7384976148605347, -0.6742561459541321],
                  [0.0, 0.60, -0.80], [0.0, 0.70, -0.71], [0.3, 0.0, -0.95], [-0.0, 0.5, -0.866], [0.0, 0.0, -1.0]],
                 np.float32)
    o[3] = [2.5, 0.0, 7.0]   # along the y = 0 plane
    z = np.zeros((n, 3), np.float32)
    ddx = np.tile(np.array([0.003236, 0.0, 0.0], np.float32), (n, 1))
    ddy = np.tile(np.array([0.0, 0.0012867, 0.00296925], np.float32), (n, 1))
    rays = {"o": o, "d": d, "odx": z, "ody": z, "ddx": ddx, "ddy": ddy, "time": np.full(n, 0.25, np.float32),
            "type": np.ones(n, np.uint16)}
    ref, mine = _trace_both(ctx, sc, rays)
    np.testing.assert_array_equal(ref["hit"], mine["hit"])
    np.testing.assert_array_equal(ref["id"], mine["id"])
    hit = ref["hit"] != 0
    np.testing.assert_array_equal(ref["t"][hit], mine["t"][hit])


def test_nan_differentials_end_at_min_upoly(ctx, ref_available):
    """A ray whose origin differentials are NaN (the reference makes them
    0/0 after a grazing hit) has a NaN width; the reference's bisection of a
    patch then never ends.  Here such a ray is diced like a ray with zero
    differentials, down to min_upoly_size: the same hits as that ray, which
    the reference traces normally."""
    sc = scenes.many_light_scene(3, res=(64, 36), spp=1)
    o = np.array([[0.5381631851196289, -7.612769603729248, 0.9662054777145386],
                  [0.7329777479171753, -7.632197856903076, 0.8413196802139282]], np.float32)
    d = np.array([[0.838919997215271, -0.08366194367408752, -0.5377862453460693],
                  [-0.17993035912513733, -0.35451218485832214, -0.9175761938095093]], np.float32)
    n = len(o)
    nan = np.full((n, 3), np.nan, np.float32)
    z = np.zeros((n, 3), np.float32)
    base = {"o": o, "d": d, "time": np.full(n, 0.632986307144165, np.float32), "type": np.full(n, 2, np.uint16)}
    with_nan = dict(base, odx=nan, ody=nan, ddx=z + 0.1, ddy=z + 0.1)
    zero = dict(base, odx=z, ody=z, ddx=z, ddy=z)
    ref, mine_zero = _trace_both(ctx, sc, zero)
    mine_nan = api.Tracer(ctx).trace(with_nan)
    np.testing.assert_array_equal(ref["hit"], mine_zero["hit"])
    np.testing.assert_array_equal(ref["id"], mine_zero["id"])
    np.testing.assert_array_equal(ref["t"], mine_zero["t"])
    for k in ("hit", "id", "t", "uv"):
        np.testing.assert_array_equal(mine_zero[k], mine_nan[k])


def _edge_scene(kind):
    """Small root shapes for the device builds: two instances, one
    instance, and 40 instances on one centre (no bin boundary separates
    them, so every split among them is the midpoint split peeling one off;
    the tree is as deep as the traversal's 64-entry node stack allows, the
    size of the reference's, accel/bvh4.hpp:161)."""
    from psychopath_cpp_b200.scene import Scene, Sphere, SphereLight
    sc = Scene(name="edge_" + kind, res_x=32, res_y=24, spp=1, seed=1)
    sc.camera = scenes.Camera(transforms=[scenes.look_at((0.0, -8.0, 3.0), (0.0, 0.0, 0.5))], fovs=[45.0])
    root = sc.root
    root.add_shader("m", scenes.SurfaceShader("Lambert", [0.7, 0.7, 0.7]))
    if kind == "two":
        root.add_object("s0", Sphere([-1.0, 0.0, 0.5], 0.8))
        root.add_instance("s0", shader="m")
    elif kind == "stacked":
        rng = np.random.default_rng(3)
        for k in range(40):
            root.add_object("s%d" % k, Sphere([0.0, 0.0, 0.5], float(rng.uniform(0.2, 1.5))))
            root.add_instance("s%d" % k, shader="m")
    # one light in every scene ("one": the light is the only instance)
    root.add_object("light", SphereLight([[1.0, -1.0, 4.0]], [0.4], [[50.0] * 3]))
    root.add_instance("light")
    return sc


@pytest.mark.parametrize("kind", ["two", "one", "stacked"])
def test_device_built_bvh_edge_cases(ctx, kind):
    """The device BVH4 build on the smallest and most degenerate roots:
    every trace output bit equal to the host-built tree's."""
    sc = _edge_scene(kind)
    rays = parity.random_rays(20000, (-3, -3, -0.5), (3, 3, 5), seed=47, occl_frac=0.3, width=0.002)
    fields = ("hit", "id", "t", "uv", "closure")
    ctx.upload(sc)
    host_st = ctx.stats()
    a = api.Tracer(ctx).trace(rays, fields=fields)
    ctx.upload(sc, gpu_bvh=True)
    st = ctx.stats()
    b = api.Tracer(ctx).trace(rays, fields=fields)
    assert st["bvh4_nodes"] == host_st["bvh4_nodes"]
    assert a["hit"].sum() > 0
    for k in fields:
        np.testing.assert_array_equal(np.asarray(a[k]).view(np.uint8), np.asarray(b[k]).view(np.uint8))


@pytest.mark.parametrize("kind", ["batch", "heightfield", "motion", "motion_patch"])
def test_device_built_bvh_gives_the_same_hits(ctx, ref_available, kind):
    """psy_scene_upload_ex(PSY_UPLOAD_GPU_BVH): the root's traversal BVH4
    built on the device.  It is the host's surface-area tree split for split,
    so the hits agree with the reference's, every output bit equals the
    host-built tree's, and a render visits the same nodes and gives the same
    image bit for bit.  "motion" and "motion_patch" have root instances
    with two time samples (moving clusters of instanced spheres, moving
    patches), so nodes carry time samples of their own."""
    from oracle import psyref
    if kind == "batch":
        sc = scenes.batch_scene(10, (64, 48), 4, 20000, 20)
        rays = parity.random_rays(60000, (-7, -7, -0.5), (7, 7, 4), seed=41, occl_frac=0.3, width=0.002)
    elif kind == "motion":
        sc = scenes.many_light_scene(7, res=(64, 48), spp=4, n_patches=80, n_groups=40, n_lights=500)
        rays = parity.random_rays(60000, (-8, -6, 0.0), (8, 6, 4), seed=43, occl_frac=0.3, width=0.002)
    elif kind == "motion_patch":
        sc = scenes.motion_patch_scene(1, res=(64, 48), spp=4)
        rays = parity.random_rays(60000, (-6, -6, -0.5), (6, 6, 4), seed=44, occl_frac=0.3, width=0.002)
    else:
        sc = scenes.heightfield_scene(64, seed=5)
        rays = scenes.heightfield_rays(60000, n=64, seed=42)
    fields = ("hit", "id", "t", "uv", "closure")
    ref = psyref.RefScene(scene=sc).trace(rays, threads=8)
    ctx.upload(sc)
    host_st = ctx.stats()
    host_tree = api.Tracer(ctx).trace(rays, fields=fields)
    ctx.upload(sc, gpu_bvh=True)
    st = ctx.stats()
    dev_tree = api.Tracer(ctx).trace(rays, fields=fields)
    assert st["bvh4_nodes"] > 0
    for mine in (host_tree, dev_tree):
        # uv of a light hit is whatever a farther candidate left (not compared)
        rep = parity.compare_trace(ref, mine, rays["type"], uv_mask=mine["closure"] != 2)
        parity.assert_parity(rep)
    for k in fields:
        np.testing.assert_array_equal(np.asarray(host_tree[k]).view(np.uint8), np.asarray(dev_tree[k]).view(np.uint8))
    assert st["gpu_bvh4_nodes"] > 0 and st["bvh4_nodes"] == host_st["bvh4_nodes"]
    if kind == "heightfield":
        return  # the heightfield scene has no light to render with
    work = ("rays", "node_visits", "leaf_visits", "patch_iterations")
    ctx.upload(sc)
    a, _ = api.PathTraceIntegrator(ctx, 64, 48, 4, seed=1, path_length=4).integrate()
    ca = ctx.trace_counters()
    ctx.upload(sc, gpu_bvh=True)
    b, _ = api.PathTraceIntegrator(ctx, 64, 48, 4, seed=1, path_length=4).integrate()
    cb = ctx.trace_counters()
    assert (np.asarray(a).view(np.uint32) == np.asarray(b).view(np.uint32)).all()
    for q in ("closest", "occlusion"):
        assert {k: ca[q][k] for k in work} == {k: cb[q][k] for k in work}, q


def test_rect_light_hits(ctx, ref_available):
    """Rays against rectangle lights: hit, id and t exact-to-4-ulp, the
    emission closure colour and light pdf of the light hits."""
    from oracle import psyref
    sc = scenes.rect_light_scene(3)
    rng = np.random.default_rng(8)
    n = 40000
    o = np.stack([rng.uniform(-5, 5, n), rng.uniform(-5, 5, n), rng.uniform(0.5, 3.0, n)], 1)
    tgt = np.where(rng.uniform(0, 1, (n, 1)) < 0.5,
                   np.stack([rng.uniform(-2, 2, n), rng.uniform(-1.5, 1.5, n), np.full(n, 6.0)], 1),
                   np.stack([rng.uniform(-5, -3, n), rng.uniform(1, 3, n), rng.uniform(2, 4, n)], 1))
    d = tgt - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = {"o": o.astype(np.float32), "d": d.astype(np.float32), "odx": np.zeros((n, 3), np.float32),
            "ody": np.zeros((n, 3), np.float32), "ddx": np.zeros((n, 3), np.float32),
            "ddy": np.zeros((n, 3), np.float32), "time": rng.uniform(0, 1, n).astype(np.float32),
            "type": np.full(n, 2, np.uint16)}
    ref = psyref.RefScene(scene=sc).trace(rays, threads=8)
    ctx.upload(sc)
    mine = api.Tracer(ctx).trace(rays, fields=("hit", "id", "t", "closure", "closure_color", "light_pdf"))
    rep = parity.compare_trace(ref, mine, rays["type"])
    parity.assert_parity(rep)
    light = (mine["hit"] == 1) & (mine["closure"] == 2)
    assert light.sum() > 2000
    out = ref["out"]
    assert parity.ulp_diff(out[light, 43:46], mine["closure_color"][light]).max() == 0
    assert np.percentile(parity.ulp_diff(out[light, 22], mine["light_pdf"][light]), 99) <= 8
