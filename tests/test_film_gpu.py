"""Film output (psy_film_srgb8, Film::scanline_image_8bbc in the reference,
film/film.hpp:173-225) and the image files written from it.

* Without dither, each channel is the reference's XYZ_to_sRGB_E of the mean
  XYZ (color/color.hpp:425-439) scaled to [0, 255], clamped and truncated:
  equal to the value built from the reference's own conversion, except where
  the device's powf and the host's differ in the last place right at an
  integer boundary (at most 0.1% of the channels, by one).
* The reference's own image (with its film's clock-seeded dither in
  [-0.5, 0.5)) is within one step of the undithered one everywhere, and
  pixels without samples show the same grey checkerboard.
* The PPM written from the film reads back as the same bytes.
"""
import os

import numpy as np
import pytest

from psychopath_cpp_b200 import api, scenes

pytestmark = pytest.mark.gpu


def _film(ctx, w=96, h=64, seed=3):
    import torch
    rng = np.random.default_rng(seed)
    counts = rng.integers(0, 9, (h, w)).astype(np.uint32)
    counts[rng.uniform(0, 1, (h, w)) < 0.15] = 0   # pixels without samples
    mean = rng.uniform(0, 1.4, (h, w, 3)).astype(np.float32) * rng.uniform(0, 1, (h, w, 1)).astype(np.float32)
    xyz = (mean * counts[..., None]).astype(np.float32)
    dx = torch.from_numpy(xyz.reshape(-1).copy()).cuda()
    dc = torch.from_numpy(counts.reshape(-1).astype(np.int32)).cuda()
    return api.Film(ctx, dx, dc, w, h), xyz, counts


def test_srgb8_matches_reference_conversion(ctx, ref_available):
    from oracle import psyref
    film, xyz, counts = _film(ctx)
    mine = film.srgb8(dither_seed=None).cpu().numpy()
    h, w = counts.shape
    has = counts > 0
    mean = np.zeros_like(xyz)
    mean[has] = xyz[has] / counts[has][:, None].astype(np.float32)
    srgb = psyref.eval_fn(9, mean.reshape(-1, 3), 3).reshape(h, w, 3)
    ys, xs = np.mgrid[0:h, 0:w]
    checker = np.where(((ys % 32) < 16) ^ ((xs % 32) < 16), np.float32(0.5), np.float32(0.35))
    v = np.where(has[..., None], srgb, checker[..., None]) * np.float32(255)
    expect = np.clip(v, 0, 255).astype(np.uint8)
    diff = np.abs(mine.astype(int) - expect.astype(int))
    assert diff.max() <= 1
    assert (diff > 0).mean() <= 1e-3, (diff > 0).mean()
    assert (mine[~has] == expect[~has]).all()
    # the reference's own image, with its dither, is within one step
    ref = psyref.film_srgb8(xyz, counts)
    assert np.abs(ref.astype(int) - mine.astype(int)).max() <= 1
    dithered = film.srgb8(dither_seed=7).cpu().numpy()
    assert np.abs(dithered.astype(int) - mine.astype(int)).max() <= 1
    assert (dithered != mine).mean() > 0.05


def test_rendered_film_to_ppm(ctx, tmp_path):
    sc = scenes.plain_scene(1, res=(64, 48), spp=4)
    ctx.upload(sc)
    import torch
    integ = api.PathTraceIntegrator.for_scene(ctx, sc)
    xyz = torch.zeros(64 * 48 * 3, device="cuda")
    cnt = torch.zeros(64 * 48, dtype=torch.int32, device="cuda")
    integ.integrate_device(xyz, cnt)
    ctx.sync()
    film = api.Film(ctx, xyz, cnt, 64, 48)
    path = os.path.join(str(tmp_path), "frame.ppm")
    film.write_ppm(path, dither_seed=1)
    back = api.read_ppm(path)
    np.testing.assert_array_equal(back, film.srgb8(dither_seed=1).cpu().numpy())
    assert back.mean() > 5
