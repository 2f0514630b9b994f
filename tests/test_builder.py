"""Host scene builder (the Assembly::finalize step) against the reference's
own builds: BVH4 node records and light trees, from golden fixtures made by
the reference, and live against oracle/_ref when it is built."""
import os

import numpy as np
import pytest

from psychopath_cpp_b200 import _abi, api, scenes
from tests import parity
from tests.golden import make_golden

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _record_kinds(child, ts):
    """Leaf and inner-node head records of a BVH4 record array; the extra
    time-sample records of an inner node follow its head."""
    leaf = np.zeros(len(ts), bool)
    head = np.zeros(len(ts), bool)
    i = 0
    while i < len(ts):
        if child[i, 0] == 0:
            leaf[i] = True
            i += 1
        else:
            head[i] = True
            i += max(int(ts[i]), 1)
    return leaf, head


def _compare_bvh4(ref, mine, transformed: bool):
    assert ref["ts"].shape == mine["ts"].shape
    np.testing.assert_array_equal(ref["ts"], mine["ts"])
    np.testing.assert_array_equal(ref["child"], mine["child"])
    leaf, _ = _record_kinds(ref["child"], ref["ts"])
    np.testing.assert_array_equal(ref["data_index"][leaf], mine["data_index"][leaf])
    inner = ~leaf
    if not inner.any():
        return
    rb = ref["bounds"][inner]
    mb = mine["bounds"][inner]
    # instance bounds (transformed) go through Matrix44::inverse, restated
    # lane for lane with this CPU's approximate reciprocal: exact as well
    assert parity.ulp_diff(rb, mb).max() == 0, (transformed, int(parity.ulp_diff(rb, mb).max()))


@pytest.mark.parametrize("name", ["plain", "heightfield", "instanced", "motion"])
def test_bvh4_matches_reference_golden(name):
    g = np.load(os.path.join(GOLDEN, "accel_%s.npz" % name))
    sc = make_golden.make_scene(name)
    for a in range(int(g["assemblies"])):
        ref = {k: g["bvh%d_%s" % (a, k)] for k in ("bounds", "child", "ts", "data_index")}
        mine = api.build_bvh4_records(sc, a)
        _compare_bvh4(ref, mine, transformed=(name == "instanced"))


@pytest.mark.parametrize("name", ["plain", "instanced"])
def test_light_tree_matches_reference_golden(name):
    g = np.load(os.path.join(GOLDEN, "accel_%s.npz" % name))
    sc = make_golden.make_scene(name)
    for a in range(int(g["assemblies"])):
        mine = api.build_light_tree(sc, a)
        np.testing.assert_array_equal(g["lt%d_meta" % a], mine["meta"])
        np.testing.assert_array_equal(g["lt%d_energy" % a], mine["energy"])
        np.testing.assert_array_equal(g["lt%d_bounds" % a], mine["bounds"])
        tot = g["lt%d_totals" % a]
        assert mine["light_count"] == int(tot[0])
        assert np.float32(mine["total_energy"]) == np.float32(tot[1])


def test_builder_matches_live_reference(ref_available):
    from oracle import psyref
    for sc, transformed in ((scenes.plain_scene(7), False), (scenes.batch_scene(3, (64, 64), 8, 900, 9), False),
                            (scenes.many_light_scene(9, res=(32, 18), spp=1, n_patches=30, n_groups=15,
                                                     n_lights=250), True)):
        ref = psyref.RefScene(scene=sc)
        for a in range(ref.assembly_count()):
            _compare_bvh4(ref.bvh4_nodes(a), api.build_bvh4_records(sc, a), transformed)
            lt = ref.light_tree(a)
            ml = api.build_light_tree(sc, a)
            np.testing.assert_array_equal(lt["meta"], ml["meta"])
            np.testing.assert_array_equal(lt["energy"], ml["energy"])


def test_degenerate_and_empty_assemblies():
    # coincident centroids exercise the builder's partition order; an empty
    # sub-assembly and an assembly with one instance exercise the edge cases
    from psychopath_cpp_b200.scene import Assembly, Scene, Sphere, SphereLight, SurfaceShader
    sc = Scene(res_x=8, res_y=8)
    root = sc.root
    root.add_shader("m", SurfaceShader("Lambert", [0.5, 0.5, 0.5]))
    for i in range(9):
        root.add_object("s%d" % i, Sphere([0, 0, 0], 0.5 + 0.01 * i))
        root.add_instance("s%d" % i, shader="m")
    empty = Assembly()
    root.add_assembly("empty", empty)
    root.add_instance("empty")
    single = Assembly()
    single.add_object("l", SphereLight([[1, 2, 3]], [0.25], [[5, 5, 5]]))
    single.add_instance("l")
    root.add_assembly("single", single)
    root.add_instance("single")
    recs = api.build_bvh4_records(sc, 0)
    assert len(recs["ts"]) > 0
    assert len(api.build_bvh4_records(sc, 1)["ts"]) == 0
    assert len(api.build_bvh4_records(sc, 2)["ts"]) == 1  # a lone leaf
    lt = api.build_light_tree(sc, 0)
    assert lt["light_count"] == 1
    from oracle import psyref
    if psyref.available():
        ref = psyref.RefScene(scene=sc)
        for a in range(3):
            _compare_bvh4(ref.bvh4_nodes(a), api.build_bvh4_records(sc, a), False)


def test_malformed_descriptions_are_rejected():
    import ctypes as C
    L = _abi.load()
    sc = scenes.plain_scene(1)
    desc, keep = api.flatten(sc)
    n = C.c_uint64()
    ok = L.psy_build_bvh4(C.byref(desc), 0, C.byref(n), None, None, None, None)
    assert ok == 0
    # instance pointing past the object list
    inst = desc.assemblies[0].instances
    saved = inst[0].data_index
    inst[0].data_index = 10 ** 6
    assert L.psy_build_bvh4(C.byref(desc), 0, C.byref(n), None, None, None, None) == _abi.PSY_ERR_ARG
    inst[0].data_index = saved
    # non-finite geometry
    obj = desc.assemblies[0].objects[0]
    saved_ptr = obj.data
    bad = np.array([np.nan] * 12, np.float32)
    obj.data = bad.ctypes.data_as(_abi.fp)
    assert L.psy_build_bvh4(C.byref(desc), 0, C.byref(n), None, None, None, None) == _abi.PSY_ERR_ARG
    obj.data = saved_ptr
    # no camera transform
    desc.cam_transform_count = 0
    assert L.psy_build_bvh4(C.byref(desc), 0, C.byref(n), None, None, None, None) == _abi.PSY_ERR_ARG
    del keep


def _two_ended_partition(v, pred):
    """std::partition on random-access iterators as libstdc++ writes it (the
    order the reference's BVH and light-tree splits leave their elements in)."""
    v = list(v)
    first, last = 0, len(v)
    while True:
        while first != last and pred(v[first]):
            first += 1
        if first == last:
            return v, first
        last -= 1
        while first != last and not pred(v[last]):
            last -= 1
        if first == last:
            return v, first
        v[first], v[last] = v[last], v[first]
        first += 1


def _closed_form_partition(v, pred):
    """The device builds' warp partition: with m elements satisfying the
    predicate, exchange the k-th one failing it among the first m positions
    (from the front) with the k-th one satisfying it among the others (from
    the back)."""
    v = list(v)
    m = sum(1 for x in v if pred(x))
    front = [i for i in range(m) if not pred(v[i])]
    back = [j for j in range(len(v) - 1, m - 1, -1) if pred(v[j])]
    assert len(front) == len(back)
    for i, j in zip(front, back):
        v[i], v[j] = v[j], v[i]
    return v, m


def test_closed_form_partition_is_the_two_ended_loop():
    """The element order (and partition point) of the device builds' warp
    partition equals libstdc++'s two-ended loop, on ragged and empty inputs,
    all-true and all-false predicates and heavy duplicates."""
    rng = np.random.default_rng(5)
    cases = [([], 1), ([(3, 0)], 1), ([(3, 0)], 5)]
    for trial in range(3000):
        n = int(rng.integers(1, 100))
        cases.append(([(int(rng.integers(0, 8)), k) for k in range(n)], int(rng.integers(0, 9))))
    for v, th in cases:
        pred = lambda x, th=th: x[0] < th
        assert _two_ended_partition(v, pred) == _closed_form_partition(v, pred), (v, th)


def test_library_reader_matches_reference_parser(ref_available, tmp_path):
    """The library's .psy reader (psy_file_parse) against the reference's
    own parser (Parser::parse_next_frame, in oracle/_ref) on the same files:
    the same BVH4 records and light trees in every assembly, for generated
    scenes, the hand-written file and a file that repeats a light's name
    with another power (the reference finds the first definition)."""
    from oracle import psyref
    from tests.test_scene_format import HAND_WRITTEN
    repeated = r"""
    Scene $s { RenderSettings { Resolution [8 6] SamplesPerPixel [1] }
      Camera { Fov [40] Transform [1 0 0 0 0 1 0 0 0 0 1 0 0 0 -5 1] }
      Assembly {
        SurfaceShader $m { Type [Lambert] Color [0.5 0.5 0.5] }
        SphereLight $l { Location [0 0 4] Radius [0.5] Color [3 3 3] }
        SphereLight $l { Location [1 0 4] Radius [0.5] Color [30 30 30] }
        SphereLight $k { Location [2 0 4] Radius [0.25] Color [5 5 5] }
        Sphere $a { Radius [1] }
        Instance { Data [$a] SurfaceShaderBind [$m] }
        Instance { Data [$l] }
        Instance { Data [$k] }
      }
    }"""
    texts = [HAND_WRITTEN, repeated,
             scenes.many_light_scene(9, res=(32, 18), spp=1, n_patches=30, n_groups=15, n_lights=250).to_psy(),
             scenes.motion_patch_scene(1, n=3).to_psy(),
             scenes.rect_light_scene(1, res=(8, 6), spp=1, n_spheres=3).to_psy()]
    for i, txt in enumerate(texts):
        path = tmp_path / ("s%d.psy" % i)
        path.write_text(txt)
        ref = psyref.RefScene(psy_path=str(path))
        mine = api.PsyFile(txt)
        for a in range(ref.assembly_count()):
            _compare_bvh4(ref.bvh4_nodes(a), api.build_bvh4_records(mine, a), True)
            lt = ref.light_tree(a)
            ml = api.build_light_tree(mine, a)
            np.testing.assert_array_equal(lt["meta"], ml["meta"])
            np.testing.assert_array_equal(lt["energy"], ml["energy"])
            np.testing.assert_array_equal(lt["bounds"], ml["bounds"])
