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


def _central_fd(r, p0, idx, target, h=1e-3):
    fd = []
    for i in idx:
        pp = p0.clone()
        pp[i] += h
        lp = _loss(*r.forward(pp), target).item()
        pm = p0.clone()
        pm[i] -= h
        lm = _loss(*r.forward(pm), target).item()
        fd.append((lp - lm) / (2 * h))
    return np.array(fd)


def test_adjoint_at_zero_valued_parameters(ctx):
    """A black albedo (all four weights 0) and a light scaled to 0 still get
    their gradient: the derivative for one factor is the product of the
    others, never a division by the factor."""
    import torch
    sc, r, p0, sp, op, count = _setup(ctx, res=(64, 64), spp=32)
    rng = np.random.default_rng(7)
    pt = p0 + torch.from_numpy(rng.normal(0.0, 0.1, count).astype(np.float32)).cuda()
    tx, tc = r.forward(pt)
    target = (tx.double().view(-1, 3) / tc.double().clamp(min=1).view(-1, 1)).detach()
    p = p0.clone()
    lights = np.arange(count - 8, count)
    p[int(lights[0])] = 0.0                       # one light switched off
    shaders, _, _, _ = api.flat_indices(sc)
    # the four largest spheres get black albedos
    big = sorted((n for n in sc.root.objects if n.startswith("sphere")),
                 key=lambda n: -float(sc.root.objects[n].radius))[:4]
    zeroed = []
    for name in big:
        w = int(sp[shaders[id(sc.root.shaders["mat" + name[6:]])]])
        p[w:w + 4] = 0.0
        zeroed += list(range(w, w + 4))
    xyz, cnt = r.forward(p)
    img = xyz.double().view(-1, 3) / cnt.double().view(-1, 1)
    g = r.adjoint(p, (2.0 * (img - target) / cnt.double().view(-1, 1)).float().reshape(-1)).double().cpu().numpy()
    idx = np.array([int(lights[0])] + zeroed[:8])
    fd = _central_fd(r, p, idx, target)
    assert np.all(np.abs(fd) > 0), fd
    err = np.abs(g[idx] - fd) / np.maximum(np.abs(fd), 1e-3 * np.abs(fd).max())
    assert np.all(err < 1e-2), list(zip(idx, g[idx], fd, err))


def test_adjoint_config_size(ctx):
    """The differentiable-render configuration: 256x256, 4 segments, 256
    albedo weights + 8 emission scales, target from N(0, 0.1)-perturbed
    parameters; the adjoint of the 4096-spp estimator against central
    differences (h = 1e-3) of that estimator on 16 random parameters."""
    import torch
    res, spp = (256, 256), 4096
    sc, r, p0, sp, op, count = _setup(ctx, res=res, spp=spp)
    rng = np.random.default_rng(11)
    pt = p0 + torch.from_numpy(rng.normal(0.0, 0.1, count).astype(np.float32)).cuda()
    tx, tc = r.forward(pt)
    target = (tx.double().view(-1, 3) / tc.double().clamp(min=1).view(-1, 1)).detach()
    xyz, cnt = r.forward(p0)
    img = xyz.double().view(-1, 3) / cnt.double().view(-1, 1)
    dl = (2.0 * (img - target) / cnt.double().view(-1, 1)).float().reshape(-1)
    g = r.adjoint(p0, dl).double().cpu().numpy()
    idx = rng.choice(np.arange(count), 16, replace=False)
    fd = _central_fd(r, p0, idx, target)
    scale = np.abs(g).max()
    err = np.abs(g[idx] - fd) / np.maximum(np.abs(fd), 1e-3 * scale)
    assert np.all(err < 1e-2), list(zip(idx, g[idx], fd, err))


def test_albedo_scale_gradient_matches_reference(ctx, ref_available):
    """Albedo gradients pinned to the reference renderer: a parameter that
    scales a shader's RGB albedo is the reference's albedo with its colour
    scaled (the spectral upsampling is linear in the colour's magnitude, and
    the reference's light selection does not read the albedo, so its paths
    stay the same).  Central differences of reference renders with the
    colour scaled by 1 +- h give the reference gradient of L = sum I^2."""
    import torch
    from oracle import psyref
    res, spp, h = (48, 48), 256, 1e-2
    sc = scenes.adjoint_scene(1, res=res, spp=spp)
    ctx.upload(sc)
    shaders, objects, ns, no = api.flat_indices(sc)
    chosen = ["ground_mat"] + sorted((n for n in sc.root.objects if n.startswith("sphere")),
                                      key=lambda n: -float(sc.root.objects[n].radius))[:4]
    chosen = [c if c == "ground_mat" else "mat" + c[6:] for c in chosen]
    ss = np.full(ns, -1, np.int32)
    for k, name in enumerate(chosen):
        ss[shaders[id(sc.root.shaders[name])]] = k
    r = api.DiffRenderer(ctx, res[0], res[1], spp, np.full(ns, -1, np.int32), np.full(no, -1, np.int32), len(chosen),
                         seed=1, path_length=4, shader_scale_param=ss)
    p = torch.ones(len(chosen), dtype=torch.float32, device="cuda")
    xyz, cnt = r.forward(p)
    plain, _ = api.PathTraceIntegrator(ctx, res[0], res[1], spp, seed=1, path_length=4).integrate()
    np.testing.assert_array_equal(plain.reshape(-1).view(np.uint32), xyz.cpu().numpy().view(np.uint32))
    img = xyz.double().view(-1, 3) / cnt.double().view(-1, 1)
    g = r.adjoint(p, (2.0 * img / cnt.double().view(-1, 1)).float().reshape(-1)).double().cpu().numpy()

    def ref_loss(name, f):
        s2 = scenes.adjoint_scene(1, res=res, spp=spp)
        s2.root.shaders[name].color = s2.root.shaders[name].color * np.float32(f)
        x, c, _, _ = psyref.RefScene(scene=s2).render(threads=0, spp=spp, path_length=4, seed=1)
        im = x.reshape(-1, 3).astype(np.float64) / np.maximum(c.reshape(-1, 1), 1)
        return (im ** 2).sum()

    ref_g = np.array([(ref_loss(n, 1 + h) - ref_loss(n, 1 - h)) / (2 * h) for n in chosen])
    rel = np.abs(g - ref_g) / np.abs(ref_g).max()
    assert np.all(rel < 1e-2), list(zip(chosen, g, ref_g, rel))
