"""psy_render_batch: many renders of different scenes in shared waves give
every film exactly the samples psy_render gives it on its own (same sampler
sequence, same per-pixel order), whatever the wave length, block size or
graph use; the autotuner picks a configuration from its sweep."""
import numpy as np
import pytest

from psychopath_cpp_b200 import api, scenes

pytestmark = pytest.mark.gpu

CFGS = [  # (seed, res, spp, prims, lights)
    (0, (48, 40), 8, 30, 1),
    (1, (64, 64), 3, 400, 5),
    (2, (17, 23), 16, 12, 2),
    (3, (96, 54), 5, 2000, 40),
    (4, (33, 31), 11, 150, 100),
]


@pytest.fixture(scope="module")
def batch_scenes():
    ctxs = []
    for seed, res, spp, prims, lights in CFGS:
        c = api.Context(0)
        c.upload(scenes.batch_scene(seed, res, spp, prims, lights))
        ctxs.append(c)
    yield ctxs
    for c in ctxs:
        c.close()


def _entries(ctxs):
    return [{"scene": c, "width": res[0], "height": res[1], "spp": spp, "seed": seed + 1, "path_length": 4}
            for c, (seed, res, spp, _, _) in zip(ctxs, CFGS)]


def _plain(ctxs):
    out = []
    for c, (seed, res, spp, _, _) in zip(ctxs, CFGS):
        xyz, cnt = api.PathTraceIntegrator(c, res[0], res[1], spp, seed=seed + 1, path_length=4).integrate()
        out.append((xyz, cnt))
    return out


@pytest.mark.parametrize("stream_paths,block,graph", [(0, 0, True), (4096, 64, False), (1000, 256, True),
                                                       (1 << 20, 128, False)])
def test_batch_films_equal_plain_renders(batch_scenes, stream_paths, block, graph):
    plain = _plain(batch_scenes)
    owner = api.Context(0)
    b = api.BatchRenderer(owner, _entries(batch_scenes), stream_paths=stream_paths, block_size=block,
                          use_graph=graph)
    b.render()
    total = sum(r[0] * r[1] * s for _, r, s, _, _ in CFGS)
    assert b.stats.paths == total
    assert b.stats.rays >= total
    for (xyz, cnt), (bx, bc) in zip(plain, b.images()):
        np.testing.assert_array_equal(cnt, bc)
        np.testing.assert_array_equal(xyz.view(np.uint32), bx.view(np.uint32))
    owner.close()


def test_batch_graph_replay_accumulates(batch_scenes):
    plain = _plain(batch_scenes)
    owner = api.Context(0)
    b = api.BatchRenderer(owner, _entries(batch_scenes), stream_paths=8192, use_graph=True)
    b.render()
    b.render(with_stats=False)  # replays the captured graph
    for (xyz, cnt), (bx, bc) in zip(plain, b.images()):
        np.testing.assert_array_equal(cnt * 2, bc)
        np.testing.assert_allclose(bx, xyz * 2, rtol=1e-6, atol=0)
    owner.close()


def test_batch_autotune(batch_scenes):
    owner = api.Context(0)
    b = api.BatchRenderer(owner, _entries(batch_scenes), use_graph=False)
    t = b.autotune(spp_divisor=2)
    assert t["trials"] == 27  # waves of 2^14..2^22 paths x blocks of 64, 128, 256
    assert t["stream_paths"] in [1 << k for k in range(14, 23)]
    assert t["block_size"] in (64, 128, 256)
    assert t["ms"] > 0
    # the batch's own films are untouched by tuning, and a render with the
    # tuned configuration matches the plain renders
    for bx, bc in b.images():
        assert not bx.any() and not bc.any()
    b.render()
    for (xyz, cnt), (bx, bc) in zip(_plain(batch_scenes), b.images()):
        np.testing.assert_array_equal(xyz.view(np.uint32), bx.view(np.uint32))
    owner.close()


def test_batch_mixing_flat_and_instanced_scenes():
    """A batch whose scenes need different traversal variants (one flat, one
    with nested motion-blurred instances and bicubic patches) runs on the
    variant covering both; every film still equals its plain render."""
    entries, plain, ctxs = [], [], []
    specs = [(scenes.batch_scene(9, (40, 30), 6, 300, 3), (40, 30), 6, 4),
             (scenes.many_light_scene(7, res=(36, 20), spp=4, n_patches=60, n_groups=20, n_lights=200), (36, 20), 4, 6)]
    for sc, res, spp, L in specs:
        c = api.Context(0)
        c.upload(sc)
        ctxs.append(c)
        plain.append(api.PathTraceIntegrator(c, res[0], res[1], spp, seed=3, path_length=L).integrate())
        entries.append({"scene": c, "width": res[0], "height": res[1], "spp": spp, "seed": 3, "path_length": L})
    owner = api.Context(0)
    b = api.BatchRenderer(owner, entries, stream_paths=2048, use_graph=False)
    b.render()
    for (xyz, cnt), (bx, bc) in zip(plain, b.images()):
        np.testing.assert_array_equal(cnt, bc)
        np.testing.assert_array_equal(xyz.view(np.uint32), bx.view(np.uint32))
    for c in ctxs + [owner]:
        c.close()
