"""Seeded synthetic workloads with the shapes of the benchmark configurations.

No public scene set exists for the reference renderer, so every workload is
generated from a seed:

* ``plain_scene``      320x240, 16 spp, 4 path segments: one 20x20 ground
                       bilinear patch, 64 Lambert spheres (r ~ U(0.2,0.6),
                       centres ~ U([-5,5]^2 x [0,2])), one sphere light
                       (r 0.5, colour 100), pinhole camera.
* ``heightfield_scene`` + ``heightfield_rays``: 256x256 bilinear-patch
                       heightfield (fBm, 4 octaves, amplitude 0.5), one
                       instance per patch, and 4M SoA rays from a box above
                       it, cosine-distributed about -z, half Morton-sorted
                       (coherent) and half shuffled (incoherent), with a
                       constant ray width that dices patches to 8x8 cells.
* ``many_light_scene`` 1280x720, 64 spp, 6 segments: 2,000 bicubic patches
                       on a wavy surface (control points jittered N(0,0.1)),
                       500 sphere groups instanced through 3 assembly levels
                       with 2-sample transform motion, 10,000 sphere lights
                       (r 0.05, power log-uniform [1,1000]), depth of field
                       (aperture 0.05) and camera motion.
* ``motion_patch_scene`` bilinear and bicubic patches with two time samples
                       (patch motion), for parity tests.
* ``batch_scenes``     48 renders of random size/spp/light count.
"""
from __future__ import annotations

import math
from typing import List, Tuple

import numpy as np

from .scene import (Assembly, BicubicPatch, BilinearPatch, Camera, Scene, Sphere, SphereLight,
                    SurfaceShader)


def look_at(pos, target, up=(0.0, 0.0, 1.0)) -> np.ndarray:
    """Camera-to-world matrix in the reference's row-vector convention
    (rows: camera x, y, z axes and position; the camera looks down +z)."""
    pos = np.asarray(pos, np.float64)
    fwd = np.asarray(target, np.float64) - pos
    fwd /= np.linalg.norm(fwd)
    right = np.cross(fwd, np.asarray(up, np.float64))
    right /= np.linalg.norm(right)
    upv = np.cross(right, fwd)
    m = np.eye(4)
    m[0, :3], m[1, :3], m[2, :3], m[3, :3] = right, upv, fwd, pos
    return m.astype(np.float32)


def _rot(axis, angle) -> np.ndarray:
    axis = np.asarray(axis, np.float64)
    axis = axis / np.linalg.norm(axis)
    x, y, z = axis
    c, s = math.cos(angle), math.sin(angle)
    C = 1 - c
    # row-vector rotation (v' = v @ R)
    return np.array([[c + x * x * C, x * y * C + z * s, x * z * C - y * s],
                     [y * x * C - z * s, c + y * y * C, y * z * C + x * s],
                     [z * x * C + y * s, z * y * C - x * s, c + z * z * C]])


def placement(rot_axis, angle, translate, scale=1.0) -> np.ndarray:
    """World-to-local instance matrix for a local-to-world placement
    (the reference's instance transforms map parent space into the
    instance's space, reference tracer/tracer.cpp:142-156)."""
    m = np.eye(4)
    m[:3, :3] = _rot(rot_axis, angle) * scale
    m[3, :3] = translate
    return np.linalg.inv(m).astype(np.float32)


# --------------------------------------------------------------------------
# Plain renderer scene
# --------------------------------------------------------------------------

def plain_scene(seed: int = 1, res=(320, 240), spp: int = 16, n_spheres: int = 64,
                light_power: float = 100.0, light_radius: float = 0.5, fov: float = 45.0) -> Scene:
    rng = np.random.default_rng(seed)
    sc = Scene(name="plain_%d" % seed, res_x=res[0], res_y=res[1], spp=spp, seed=1)
    sc.camera = Camera(transforms=[look_at((0.0, -15.0, 7.0), (0.0, 0.0, 0.5))], fovs=[fov])
    root = sc.root
    ground_alb = rng.uniform(0.2, 0.8)
    root.add_shader("ground_mat", SurfaceShader("Lambert", [ground_alb] * 3))
    root.add_object("ground", BilinearPatch([[-10, -10, 0], [10, -10, 0], [-10, 10, 0], [10, 10, 0]]))
    root.add_instance("ground", shader="ground_mat")
    for i in range(n_spheres):
        r = rng.uniform(0.2, 0.6)
        c = [rng.uniform(-5, 5), rng.uniform(-5, 5), rng.uniform(0, 2)]
        alb = rng.uniform(0.2, 0.8)
        root.add_shader("mat%d" % i, SurfaceShader("Lambert", [alb] * 3))
        root.add_object("sphere%d" % i, Sphere(c, r))
        root.add_instance("sphere%d" % i, shader="mat%d" % i)
    root.add_object("light", SphereLight([[0.0, 0.0, 6.0]], [light_radius], [[light_power] * 3]))
    root.add_instance("light")
    return sc


def adjoint_scene(seed: int = 1, res=(256, 256), spp: int = 32, n_spheres: int = 64, n_lights: int = 8,
                  light_power: float = 100.0) -> Scene:
    """The plain scene's geometry with n_lights sphere lights (total power
    light_power) spread over a ring above it: the differentiable-render
    workload (per-sphere albedo basis weights and per-light emission scales)."""
    sc = plain_scene(seed, res=res, spp=spp, n_spheres=n_spheres)
    root = sc.root
    del root.objects["light"]
    root.instances = [i for i in root.instances if i.data != "light"]
    for k in range(n_lights):
        a = 2.0 * math.pi * k / n_lights
        p = [4.0 * math.cos(a), 4.0 * math.sin(a), 5.5 + 0.5 * math.sin(3 * a)]
        root.add_object("light%d" % k, SphereLight([p], [0.35], [[light_power / n_lights] * 3]))
        root.add_instance("light%d" % k)
    return sc


def gtr_scene(seed: int = 1, res=(96, 72), spp: int = 16, n_spheres: int = 24) -> Scene:
    """The plain scene with GTR microfacet shaders (GTRClosure,
    shading/surface_closure.hpp:339-608) on the ground and on most spheres:
    roughness from mirror (0, a delta closure) to 0.8, tail shapes on both
    sides of 1, Fresnel factors 0..1; the rest Lambert; one sphere light."""
    rng = np.random.default_rng(seed)
    sc = Scene(name="gtr_%d" % seed, res_x=res[0], res_y=res[1], spp=spp, seed=1)
    sc.camera = Camera(transforms=[look_at((0.0, -15.0, 7.0), (0.0, 0.0, 0.5))], fovs=[45.0])
    root = sc.root
    root.add_shader("ground_mat", SurfaceShader("GTR", [0.7, 0.65, 0.6], roughness=0.35, tail_shape=2.0, fresnel=0.5))
    root.add_object("ground", BilinearPatch([[-10, -10, 0], [10, -10, 0], [-10, 10, 0], [10, 10, 0]]))
    root.add_instance("ground", shader="ground_mat")
    roughs = [0.0, 0.02, 0.1, 0.3, 0.6, 0.8]
    for i in range(n_spheres):
        col = [rng.uniform(0.2, 0.9), rng.uniform(0.2, 0.9), rng.uniform(0.2, 0.9)]
        if i % 4 == 3:
            root.add_shader("mat%d" % i, SurfaceShader("Lambert", col))
        else:
            root.add_shader("mat%d" % i, SurfaceShader("GTR", col, roughness=roughs[i % len(roughs)],
                                                       tail_shape=[0.5, 1.0, 2.0, 4.0][i % 4],
                                                       fresnel=rng.uniform(0.0, 1.0)))
        root.add_object("sphere%d" % i, Sphere([rng.uniform(-5, 5), rng.uniform(-5, 5), rng.uniform(0, 2)],
                                               rng.uniform(0.2, 0.6)))
        root.add_instance("sphere%d" % i, shader="mat%d" % i)
    root.add_object("light", SphereLight([[1.0, -1.0, 6.0]], [0.5], [[100.0] * 3]))
    root.add_instance("light")
    return sc


def rect_light_scene(seed: int = 1, res=(96, 72), spp: int = 16, n_spheres: int = 24) -> Scene:
    """The plain scene's geometry lit by rectangle lights instead of a
    sphere light: one overhead (3 x 1.5, facing down through an instance
    transform), one tilted panel (1 x 2.5) to the side, with the
    reference's own rectangle-light arithmetic, including its upper y bound
    of half the x dimension."""
    from .scene import RectangleLight
    rng = np.random.default_rng(seed)
    sc = Scene(name="rect_light_%d" % seed, res_x=res[0], res_y=res[1], spp=spp, seed=1)
    sc.camera = Camera(transforms=[look_at((0.0, -15.0, 7.0), (0.0, 0.0, 0.5))], fovs=[45.0])
    root = sc.root
    root.add_shader("ground_mat", SurfaceShader("Lambert", [0.6, 0.55, 0.5]))
    root.add_object("ground", BilinearPatch([[-10, -10, 0], [10, -10, 0], [-10, 10, 0], [10, 10, 0]]))
    root.add_instance("ground", shader="ground_mat")
    for i in range(n_spheres):
        root.add_shader("mat%d" % i, SurfaceShader("Lambert", [rng.uniform(0.2, 0.8)] * 3))
        root.add_object("sphere%d" % i, Sphere([rng.uniform(-5, 5), rng.uniform(-5, 5), rng.uniform(0, 2)],
                                               rng.uniform(0.2, 0.6)))
        root.add_instance("sphere%d" % i, shader="mat%d" % i)
    root.add_object("panel", RectangleLight([[3.0, 1.5]], [[60.0, 60.0, 55.0]]))
    root.add_instance("panel", [placement((1.0, 0.0, 0.0), math.pi, (0.0, 0.0, 6.0))])
    root.add_object("side", RectangleLight([[1.0, 2.5]], [[30.0, 35.0, 40.0]]))
    root.add_instance("side", [placement((0.3, 1.0, 0.2), 1.2, (-4.0, 2.0, 3.0))])
    return sc


# --------------------------------------------------------------------------
# Heightfield trace microbenchmark
# --------------------------------------------------------------------------

def _value_noise(rng, size: int, freq: int) -> np.ndarray:
    """Bilinearly interpolated lattice noise sampled on a (size+1)^2 grid."""
    lat = rng.uniform(-1.0, 1.0, size=(freq + 2, freq + 2))
    xs = np.linspace(0.0, freq, size + 1)
    i = np.floor(xs).astype(int)
    f = xs - i
    f = f * f * (3 - 2 * f)
    a = lat[i][:, i]
    b = lat[i + 1][:, i]
    c = lat[i][:, i + 1]
    d = lat[i + 1][:, i + 1]
    fx = f[:, None]
    fy = f[None, :]
    return (a * (1 - fx) + b * fx) * (1 - fy) + (c * (1 - fx) + d * fx) * fy


def fbm_heights(n: int, seed: int, octaves: int = 4, amplitude: float = 0.5, base_freq: int = 8) -> np.ndarray:
    rng = np.random.default_rng(seed)
    h = np.zeros((n + 1, n + 1))
    amp, norm = 1.0, 0.0
    for o in range(octaves):
        h += amp * _value_noise(rng, n, base_freq * (2 ** o))
        norm += amp
        amp *= 0.5
    return (h / norm * amplitude).astype(np.float32)


def heightfield_scene(n: int = 256, seed: int = 7, dicing_rate: float = 0.25) -> Scene:
    """n x n unit bilinear patches over [0,n]^2, one object + instance each."""
    h = fbm_heights(n, seed)
    sc = Scene(name="heightfield_%d" % n, res_x=64, res_y=64, spp=1, seed=1, dicing_rate=dicing_rate)
    sc.camera = Camera(transforms=[look_at((n / 2, -n / 2, n / 2), (n / 2, n / 2, 0))], fovs=[45.0])
    root = sc.root
    root.add_shader("mat", SurfaceShader("Lambert", [0.5, 0.5, 0.5]))
    for y in range(n):
        for x in range(n):
            v = [[x, y, h[y, x]], [x + 1, y, h[y, x + 1]], [x, y + 1, h[y + 1, x]], [x + 1, y + 1, h[y + 1, x + 1]]]
            name = "p%d_%d" % (x, y)
            root.add_object(name, BilinearPatch(v))
            root.add_instance(name, shader="mat")
    return sc


def _morton2(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    def part(v):
        v = v.astype(np.uint64) & np.uint64(0xFFFF)
        v = (v | (v << np.uint64(8))) & np.uint64(0x00FF00FF)
        v = (v | (v << np.uint64(4))) & np.uint64(0x0F0F0F0F)
        v = (v | (v << np.uint64(2))) & np.uint64(0x33333333)
        v = (v | (v << np.uint64(1))) & np.uint64(0x55555555)
        return v
    return part(x) | (part(y) << np.uint64(1))


def heightfield_rays(count: int, n: int = 256, seed: int = 11, width: float = 0.6) -> dict:
    """SoA world rays above the heightfield (float32 arrays of length count).

    Ray width: odx=(w,0,0), ody=(0,w,0), ddx=ddy=0 gives a constant width w
    (reference basics/ray.hpp:207-252 with utils/utils.hpp:443-456), so with
    dicing rate 0.25 the leaf threshold is 0.25*w (0.15 for w=0.6): unit
    patches dice to 8x8 cells, more where the height varies."""
    rng = np.random.default_rng(seed)
    ox = rng.uniform(0.0, n, count)
    oy = rng.uniform(0.0, n, count)
    oz = rng.uniform(2.0, 4.0, count)
    # cosine-weighted directions about -z
    u1, u2 = rng.uniform(0, 1, count), rng.uniform(0, 1, count)
    r = np.sqrt(u1)
    phi = 2 * np.pi * u2
    dx, dy, dz = r * np.cos(phi), r * np.sin(phi), -np.sqrt(np.maximum(0.0, 1.0 - u1))
    half = count // 2
    # first half: coherent (Morton order of origin cell and direction octant)
    key = _morton2(np.floor(ox[:half]).astype(np.int64), np.floor(oy[:half]).astype(np.int64))
    octant = ((dx[:half] > 0).astype(np.uint64) | ((dy[:half] > 0).astype(np.uint64) << np.uint64(1)))
    order = np.lexsort((key, octant))
    # second half: incoherent (random order)
    perm = rng.permutation(count - half) + half
    idx = np.concatenate([order, perm])
    f = np.float32
    z = np.zeros(count, f)
    return {
        "o": np.stack([ox[idx], oy[idx], oz[idx]], 1).astype(f),
        "d": np.stack([dx[idx], dy[idx], dz[idx]], 1).astype(f),
        "odx": np.stack([np.full(count, width), z, z], 1).astype(f),
        "ody": np.stack([z, np.full(count, width), z], 1).astype(f),
        "ddx": np.zeros((count, 3), f),
        "ddy": np.zeros((count, 3), f),
        "time": np.zeros(count, f),
        "type": np.full(count, 1, np.uint16),
    }


# --------------------------------------------------------------------------
# Many-light 720p render
# --------------------------------------------------------------------------

def _bezier_surface_patch(x0, y0, size, rng, jitter) -> np.ndarray:
    pts = []
    for j in range(4):
        for i in range(4):
            x = x0 + size * i / 3.0
            y = y0 + size * j / 3.0
            z = 0.4 * math.sin(0.7 * x) * math.cos(0.5 * y)
            pts.append([x, y, z])
    pts = np.array(pts) + rng.normal(0.0, jitter, size=(16, 3))
    return pts.astype(np.float32)


def motion_patch_scene(seed: int = 1, res=(96, 72), spp: int = 8, n: int = 6) -> Scene:
    """Patches that move and deform while the shutter is open: an n x n grid
    of alternating bilinear and bicubic patches, each with two time samples
    (the second sample shifted by up to 0.3 and its control points jittered
    by N(0, 0.05)), over a static ground patch, with a few Lambert spheres
    and one sphere light; pinhole camera without motion."""
    rng = np.random.default_rng(seed)
    sc = Scene(name="motion_patch_%d" % seed, res_x=res[0], res_y=res[1], spp=spp, seed=1)
    sc.camera = Camera(transforms=[look_at((0.0, -9.0, 6.0), (0.0, 0.0, 0.3))], fovs=[50.0])
    root = sc.root
    root.add_shader("ground", SurfaceShader("Lambert", [0.5, 0.5, 0.5]))
    root.add_object("ground", BilinearPatch([[-8, -8, 0], [8, -8, 0], [-8, 8, 0], [8, 8, 0]]))
    root.add_instance("ground", shader="ground")
    size = 6.0 / n
    for j in range(n):
        for i in range(n):
            k = j * n + i
            x0, y0 = -3.0 + i * size, -3.0 + j * size
            shift = np.array([rng.uniform(-0.3, 0.3), rng.uniform(-0.3, 0.3), rng.uniform(0.0, 0.3)])
            if k % 2 == 0:
                z = rng.uniform(0.3, 0.9, 4)
                v0 = np.array([[x0, y0, z[0]], [x0 + size, y0, z[1]], [x0, y0 + size, z[2]],
                               [x0 + size, y0 + size, z[3]]])
                v1 = v0 + shift + rng.normal(0.0, 0.05, (4, 3))
                obj = BilinearPatch(np.stack([v0, v1]))
            else:
                v0 = _bezier_surface_patch(x0, y0, size, rng, 0.1) + np.array([0.0, 0.0, 0.6])
                v1 = v0 + shift + rng.normal(0.0, 0.05, (16, 3))
                obj = BicubicPatch(np.stack([v0, v1]))
            alb = rng.uniform(0.3, 0.8)
            root.add_shader("m%d" % k, SurfaceShader("Lambert", [alb, 0.5, 1.0 - alb]))
            root.add_object("p%d" % k, obj)
            root.add_instance("p%d" % k, shader="m%d" % k)
    for i in range(4):
        c = [rng.uniform(-3, 3), rng.uniform(-3, 3), rng.uniform(1.2, 1.8)]
        root.add_shader("s%d" % i, SurfaceShader("Lambert", [0.7] * 3))
        root.add_object("sphere%d" % i, Sphere(c, rng.uniform(0.2, 0.4)))
        root.add_instance("sphere%d" % i, shader="s%d" % i)
    root.add_object("light", SphereLight([[1.0, -1.0, 5.0]], [0.6], [[80.0] * 3]))
    root.add_instance("light")
    return sc


def many_light_scene(seed: int = 3, res=(1280, 720), spp: int = 64, n_patches: int = 2000,
                     n_groups: int = 500, spheres_per_group: int = 10, n_lights: int = 10000,
                     light_radius: float = 0.05, aperture: float = 0.05) -> Scene:
    rng = np.random.default_rng(seed)
    sc = Scene(name="many_light_%d" % seed, res_x=res[0], res_y=res[1], spp=spp, seed=1)
    cam0 = look_at((0.0, -32.0, 14.0), (0.0, 0.0, 0.0))
    cam1 = look_at((0.6, -31.5, 14.0), (0.0, 0.0, 0.0))
    sc.camera = Camera(transforms=[cam0, cam1], fovs=[50.0], aperture_radii=[aperture],
                       focus_distances=[float(np.linalg.norm([0.0, -32.0, 14.0]))])
    root = sc.root
    # ground of bicubic patches: a cols x rows grid of unit-size patches
    cols = int(math.ceil(math.sqrt(n_patches * 1.25)))
    rows = int(math.ceil(n_patches / cols))
    psize = 1.0
    root.add_shader("ground", SurfaceShader("Lambert", [0.6, 0.6, 0.6]))
    k = 0
    for j in range(rows):
        for i in range(cols):
            if k >= n_patches:
                break
            x0 = (i - cols / 2) * psize
            y0 = (j - rows / 2) * psize
            name = "bp%d" % k
            root.add_object(name, BicubicPatch(_bezier_surface_patch(x0, y0, psize, rng, 0.1)))
            root.add_instance(name, shader="ground")
            k += 1
    # three-level sphere groups: root -> cluster (2-sample motion) -> group -> spheres
    groups_per_cluster = 5
    clusters = max(1, n_groups // groups_per_cluster)
    group = Assembly()
    for s in range(spheres_per_group):
        group.add_object("s%d" % s, Sphere(rng.uniform(-0.8, 0.8, 3), rng.uniform(0.1, 0.35)))
        group.add_instance("s%d" % s)
    cluster = Assembly()
    cluster.add_assembly("group", group)
    for g in range(groups_per_cluster):
        ax = rng.normal(size=3)
        cluster.add_shader("gmat%d" % g, SurfaceShader("Lambert", [rng.uniform(0.1, 0.9)] * 3))
        cluster.add_instance("group", [placement(ax, rng.uniform(0, 6.28), rng.uniform(-2.5, 2.5, 3))],
                             shader="gmat%d" % g)
    root.add_assembly("cluster", cluster)
    half_w = cols * psize / 2
    half_h = rows * psize / 2
    for c in range(clusters):
        t = np.array([rng.uniform(-half_w * 0.8, half_w * 0.8), rng.uniform(-half_h * 0.8, half_h * 0.8),
                      rng.uniform(2.0, 4.0)])
        ax = rng.normal(size=3)
        ang = rng.uniform(0, 6.28)
        m0 = placement(ax, ang, t)
        m1 = placement(ax, ang + 0.05, t + rng.normal(0.0, 0.15, 3))
        root.add_instance("cluster", [m0, m1])
    # many small sphere lights over the scene bounds
    for li in range(n_lights):
        p = [rng.uniform(-half_w, half_w), rng.uniform(-half_h, half_h), rng.uniform(0.5, 8.0)]
        power = math.exp(rng.uniform(math.log(1.0), math.log(1000.0)))
        root.add_object("l%d" % li, SphereLight([p], [light_radius], [[power] * 3]))
        root.add_instance("l%d" % li)
    return sc


# --------------------------------------------------------------------------
# Batched renders
# --------------------------------------------------------------------------

def batch_scene(seed: int, res: Tuple[int, int], spp: int, n_prims: int, n_lights: int) -> Scene:
    rng = np.random.default_rng(1000 + seed)
    sc = Scene(name="batch_%d" % seed, res_x=res[0], res_y=res[1], spp=spp, seed=seed + 1)
    sc.camera = Camera(transforms=[look_at((0.0, -15.0, 7.0), (0.0, 0.0, 0.5))], fovs=[45.0])
    root = sc.root
    n_patches = max(1, n_prims // 10)
    n_spheres = max(0, n_prims - n_patches)
    side = int(math.ceil(math.sqrt(n_patches)))
    cell = 20.0 / side
    k = 0
    for j in range(side):
        for i in range(side):
            if k >= n_patches:
                break
            x0, y0 = -10 + i * cell, -10 + j * cell
            z = rng.uniform(-0.05, 0.05, 4)
            root.add_shader("pm%d" % k, SurfaceShader("Lambert", [rng.uniform(0.1, 0.9)] * 3))
            root.add_object("p%d" % k, BilinearPatch([[x0, y0, z[0]], [x0 + cell, y0, z[1]],
                                                      [x0, y0 + cell, z[2]], [x0 + cell, y0 + cell, z[3]]]))
            root.add_instance("p%d" % k, shader="pm%d" % k)
            k += 1
    for i in range(n_spheres):
        root.add_shader("sm%d" % i, SurfaceShader("Lambert", [rng.uniform(0.1, 0.9)] * 3))
        root.add_object("s%d" % i, Sphere([rng.uniform(-5, 5), rng.uniform(-5, 5), rng.uniform(0, 2)],
                                          rng.uniform(0.02, 0.6) if n_spheres < 1000 else rng.uniform(0.01, 0.1)))
        root.add_instance("s%d" % i, shader="sm%d" % i)
    for li in range(n_lights):
        p = [rng.uniform(-6, 6), rng.uniform(-6, 6), rng.uniform(3, 8)]
        root.add_object("l%d" % li, SphereLight([p], [rng.uniform(0.1, 0.5)], [[100.0 / n_lights * 10] * 3]))
        root.add_instance("l%d" % li)
    return sc


def batch_configs(count: int = 48, seed: int = 0) -> List[dict]:
    rng = np.random.default_rng(seed)
    cfgs = []
    for i in range(count):
        w = int(rng.integers(64, 1025))
        h = int(rng.integers(64, 769))
        cfgs.append({"seed": i, "res": (w, h), "spp": int(rng.integers(8, 129)),
                     "n_prims": int(rng.integers(10, 50001)), "n_lights": int(rng.integers(1, 101))})
    return cfgs
