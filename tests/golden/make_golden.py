"""Generates the golden fixtures under tests/golden/ from the reference
renderer itself (oracle/_ref/libpsyref.so, built from the reference's
sources by oracle/Makefile).

    python tests/golden/make_golden.py

Every fixture stores the seeded inputs and the reference's outputs, so the
CPU tests (oracle restatement, host builder) and GPU tests run without the
reference build.  Scenes are regenerated from their seeds by
psychopath_cpp_b200.scenes; each fixture records the generator arguments.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import psyref  # noqa: E402
from psychopath_cpp_b200 import scenes  # noqa: E402
from tests import parity  # noqa: E402

SCENES = {
    "plain": ("plain_scene", {"seed": 1}),
    "heightfield": ("heightfield_scene", {"n": 16, "seed": 2}),
    "instanced": ("many_light_scene", {"seed": 5, "res": [64, 36], "spp": 1, "n_patches": 40, "n_groups": 20,
                                       "n_lights": 100}),
    "motion": ("motion_patch_scene", {"seed": 2, "n": 4}),
}


def make_scene(name):
    fn, kw = SCENES[name]
    kw = dict(kw)
    if "res" in kw:
        kw["res"] = tuple(kw["res"])
    return getattr(scenes, fn)(**kw)


def rays_for(name):
    if name == "plain":
        return parity.random_rays(2048, (-6, -6, 0.01), (6, 6, 3), seed=31, occl_frac=0.3)
    if name == "heightfield":
        return scenes.heightfield_rays(2048, n=16, seed=32)
    if name == "motion":
        return parity.random_rays(2048, (-4, -4, 0.05), (4, 4, 2), seed=34, occl_frac=0.3)
    return parity.random_rays(2048, (-8, -6, -0.5), (8, 6, 5), seed=33, occl_frac=0.3)


def save(name, **arrays):
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)


def main():
    assert psyref.available(), "build oracle/_ref first (make -C oracle ref)"
    meta = {"scenes": SCENES}
    for name in SCENES:
        sc = make_scene(name)
        ref = psyref.RefScene(scene=sc)
        rays = rays_for(name)
        res = ref.trace(rays, threads=4)
        out = res["out"]
        save("trace_" + name, **{"ray_" + k: v for k, v in rays.items()}, hit=res["hit"], id=res["id"],
             t=res["t"], uv=res["uv"], p=out[:, 3:6], n=out[:, 6:9], closure=out[:, 42].astype(np.uint8),
             closure_color=out[:, 43:46], backfacing=out[:, 21].astype(np.uint8))
        recs = {}
        for a in range(ref.assembly_count()):
            b = ref.bvh4_nodes(a)
            lt = ref.light_tree(a)
            for k, v in b.items():
                recs["bvh%d_%s" % (a, k)] = v
            for k in ("meta", "energy", "bounds"):
                recs["lt%d_%s" % (a, k)] = lt[k]
            recs["lt%d_totals" % a] = np.array([lt["light_count"], lt["total_energy"]], np.float64)
        save("accel_" + name, assemblies=np.array(ref.assembly_count()), **recs)
    # sampler: Halton for every dimension, and whole Sampler sequences
    rng = np.random.default_rng(41)
    dims = np.repeat(np.arange(256, dtype=np.uint32), 32)
    idx = rng.integers(0, 2 ** 32, size=dims.size, dtype=np.uint64).astype(np.uint32)
    idx[:256] = np.arange(256, dtype=np.uint32)
    save("halton", dims=dims, idx=idx, value=psyref.halton(dims, idx))
    seqs, offs, args = [], [], []
    for k in range(64):
        x, y, s, seed = (int(v) for v in rng.integers(0, 2000, 4))
        vals, off = psyref.sampler(x, y, s, seed, 40)
        seqs.append(vals)
        offs.append(off)
        args.append((x, y, s, seed))
    save("sampler", args=np.array(args, np.uint32), offset=np.array(offs, np.uint32), values=np.array(seqs))
    # scalar helpers (psyref_eval)
    n = 4096
    rgb = rng.uniform(0, 2, (n, 3)).astype(np.float32)
    rgb[:64] = rng.uniform(0, 1, (64, 1)).astype(np.float32)  # greys
    wl = rng.uniform(380, 700, n).astype(np.float32)
    spec_in = np.concatenate([rgb, wl[:, None]], 1)
    spec = psyref.eval_fn(0, spec_in, 4)
    xyz = psyref.eval_fn(1, np.concatenate([spec, wl[:, None]], 1), 3)
    p = rng.uniform(0, 1, (n, 1)).astype(np.float32)
    logit = psyref.eval_fn(2, p, 1)
    sq = rng.uniform(-1, 1, (n, 2)).astype(np.float32)
    circ = psyref.eval_fn(3, sq, 2)
    uv = rng.uniform(0, 1, (n, 2)).astype(np.float32)
    hemi = psyref.eval_fn(4, uv, 3)
    sl = np.stack([rng.uniform(-1, 1, n), rng.uniform(0, 1, n)], 1).astype(np.float32)
    lamb = psyref.eval_fn(5, sl, 1)
    save("scalar", spec_in=spec_in, spec=spec, xyz=xyz, logit_in=p, logit=logit, circ_in=sq, circ=circ,
         hemi_in=uv, hemi=hemi, lambert_in=sl, lambert=lamb)
    # a small film
    sc = scenes.plain_scene(1, res=(32, 24), spp=16)
    xyzf, cnt, rays_shot, _ = psyref.RefScene(scene=sc).render(threads=4, spp=16, path_length=4, seed=1)
    save("render_plain_32x24", xyz=xyzf, counts=cnt, rays=np.array(rays_shot))
    with open(os.path.join(HERE, "README.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "source": "oracle/_ref (reference built from source)",
                   **meta}, f, indent=1)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
