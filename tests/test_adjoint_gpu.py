"""Differentiable render and its path-replay adjoint.

* With no parameters bound the differentiable render is the plain render,
  bit for bit; doubling every light's emission scale doubles the film
  exactly (power-of-two scaling).
* The adjoint is the exact derivative of the Monte Carlo estimator for fixed
  random numbers, so it is checked against central finite differences
  (h = 1e-3) of the same estimator on 16 random parameters: relative error
  below 1e-2.  (The finite differences of a fixed-seed estimator need no
  high sample count; 4096 spp would only bring both closer to the expected
  gradient.)
* The emission-scale gradient is checked against a reference gradient built
  from the reference CPU renderer: the image is linear in each scale, so
  dL/ds_i = sum_p 2 I_p I_p^(i) for L = sum_p I_p^2, with I^(i) the
  reference's render with light i alone.  Both sides are Monte Carlo
  estimates; tolerance 5e-2 relative.
"""
import numpy as np
import pytest

from psychopath_cpp_b200 import api, scenes
from tests import diff_util

pytestmark = pytest.mark.gpu


def _setup(ctx, res=(64, 64), spp=16, seed=1):
    import torch
    sc = scenes.adjoint_scene(seed, res=res, spp=spp)
    ctx.upload(sc)
    sp, op, count = diff_util.layout(sc)
    assert count == 64 * 4 + 8
    r = api.DiffRenderer(ctx, res[0], res[1], spp, sp, op, count, seed=1, path_length=4)
    p0 = torch.from_numpy(diff_util.initial_params(sc, sp, op, count)).cuda()
    return sc, r, p0, sp, op, count


def test_diff_render_reduces_to_plain(ctx):
    import torch
    sc, r, p0, sp, op, count = _setup(ctx)
    plain_xyz, plain_cnt = api.PathTraceIntegrator(ctx, 64, 64, 16, seed=1, path_length=4).integrate()
    none = api.DiffRenderer(ctx, 64, 64, 16, np.full_like(sp, -1), np.full_like(op, -1), count, seed=1)
    xyz, cnt = none.forward(p0)
    np.testing.assert_array_equal(plain_xyz.reshape(-1).view(np.uint32), xyz.cpu().numpy().view(np.uint32))
    lights_only = api.DiffRenderer(ctx, 64, 64, 16, np.full_like(sp, -1), op, count, seed=1)
    x1, _ = lights_only.forward(p0)
    p2 = p0.clone()
    p2[op[op >= 0]] = 2.0
    x2, _ = lights_only.forward(p2)
    np.testing.assert_array_equal((x1 * 2).cpu().numpy(), x2.cpu().numpy())


def _loss(xyz, cnt, target):
    import torch
    img = xyz.double().view(-1, 3) / cnt.double().clamp(min=1).view(-1, 1)
    return ((img - target) ** 2).sum()


def test_adjoint_matches_central_differences(ctx):
    import torch
    sc, r, p0, sp, op, count = _setup(ctx, res=(96, 96), spp=32)
    rng = np.random.default_rng(4)
    # target image: rendered from perturbed parameters
    pt = p0 + torch.from_numpy(rng.normal(0.0, 0.1, count).astype(np.float32)).cuda()
    tx, tc = r.forward(pt)
    target = (tx.double().view(-1, 3) / tc.double().clamp(min=1).view(-1, 1)).detach()
    Fn = diff_util.render_fn()
    params = p0.clone().requires_grad_(True)
    xyz = Fn.apply(params, r)
    cnt = torch.full((96 * 96,), 32, dtype=torch.int32, device="cuda")
    loss = _loss(xyz, cnt, target)
    loss.backward()
    g = params.grad.double().cpu().numpy()
    h = 1e-3
    idx = rng.choice(np.arange(count), 16, replace=False)
    # include some emission scales and the most influential albedo weights
    idx[:4] = np.arange(count - 8, count - 4)
    idx[4:8] = np.argsort(-np.abs(g[:count - 8]))[:4]
    fd = []
    for i in idx:
        pp = p0.clone()
        pp[i] += h
        lp = _loss(*r.forward(pp), target).item()
        pm = p0.clone()
        pm[i] -= h
        lm = _loss(*r.forward(pm), target).item()
        fd.append((lp - lm) / (2 * h))
    fd = np.array(fd)
    scale = np.abs(g).max()
    err = np.abs(g[idx] - fd) / np.maximum(np.abs(fd), 1e-3 * scale)
    assert np.all(err < 1e-2), list(zip(idx, g[idx], fd, err))


def test_emission_gradient_matches_reference(ctx, ref_available):
    import torch
    from oracle import psyref
    res, spp = (48, 48), 256
    sc, r, p0, sp, op, count = _setup(ctx, res=res, spp=spp)
    xyz, cnt = r.forward(p0)
    img = xyz.double().view(-1, 3) / cnt.double().view(-1, 1)
    # L = sum I^2: dL/d(film sums) = 2 I / count
    dl = (2.0 * img / cnt.double().view(-1, 1)).float().reshape(-1)
    g = r.adjoint(p0, dl).double().cpu().numpy()
    # reference: the image with one light alone, per light
    ref_full = psyref.RefScene(scene=sc).render(threads=0, spp=spp, path_length=4, seed=1)
    full = ref_full[0].reshape(-1, 3).astype(np.float64) / np.maximum(ref_full[1].reshape(-1, 1), 1)
    lights = sorted((n for n in sc.root.objects if n.startswith("light")), key=lambda n: int(n[5:]))
    ref_g = []
    for name in lights:
        solo = scenes.adjoint_scene(1, res=res, spp=spp)
        for other in lights:
            if other != name:
                solo.root.objects[other].colors[:] = 0.0
        out = psyref.RefScene(scene=solo).render(threads=0, spp=spp, path_length=4, seed=1)
        part = out[0].reshape(-1, 3).astype(np.float64) / np.maximum(out[1].reshape(-1, 1), 1)
        ref_g.append((2.0 * full * part).sum())
    ref_g = np.array(ref_g)
    mine = g[count - 8:]
    rel = np.abs(mine - ref_g) / np.abs(ref_g).max()
    assert np.all(rel < 5e-2), list(zip(mine, ref_g, rel))
