"""Test-side helpers for the differentiable render: the parameter layout of
the adjoint scene and a torch.autograd.Function over psy_render_diff /
psy_render_adjoint (used by the tests only)."""
import numpy as np

from psychopath_cpp_b200 import api


def layout(scene):
    """shader_param, object_param and the parameter count: 4 albedo weights
    per sphere shader ("mat*"), one emission scale per light object."""
    shaders, objects, ns, no = api.flat_indices(scene)
    root = scene.root
    sp = np.full(ns, -1, np.int32)
    op = np.full(no, -1, np.int32)
    count = 0
    names = sorted((n for n in root.shaders if n.startswith("mat")), key=lambda n: int(n[3:]))
    for name in names:
        sh = root.shaders[name]
        if id(sh) in shaders:
            sp[shaders[id(sh)]] = count
            count += 4
    lights = sorted((n for n in root.objects if n.startswith("light")), key=lambda n: int(n[5:]))
    for name in lights:
        op[objects[(0, name)]] = count
        count += 1
    return sp, op, count


def initial_params(scene, sp, op, count):
    """Weights that give roughly each sphere's grey RGB albedo; unit scales."""
    shaders, _, _, _ = api.flat_indices(scene)
    p = np.zeros(count, np.float32)
    for name, sh in scene.root.shaders.items():
        if id(sh) in shaders and sp[shaders[id(sh)]] >= 0:
            p[sp[shaders[id(sh)]]:sp[shaders[id(sh)]] + 4] = 0.8 * float(sh.color[0])
    for o in op:
        if o >= 0:
            p[o] = 1.0
    return p


def render_fn():
    import torch

    class RenderFn(torch.autograd.Function):
        """Film sums as a function of the parameters; backward is the adjoint."""

        @staticmethod
        def forward(ctx, params, renderer):
            xyz, counts = renderer.forward(params)
            torch.cuda.synchronize()
            ctx.renderer = renderer
            ctx.save_for_backward(params)
            ctx.counts = counts
            return xyz

        @staticmethod
        def backward(ctx, grad_xyz):
            params, = ctx.saved_tensors
            g = ctx.renderer.adjoint(params, grad_xyz.contiguous())
            torch.cuda.synchronize()
            return g, None

    return RenderFn
