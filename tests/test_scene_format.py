"""The .psy writer and reader (the reference's scene format, parser/parser.cpp)."""
import numpy as np
import pytest

from psychopath_cpp_b200 import scene as S
from psychopath_cpp_b200 import scenes


def test_float_formatting_round_trips_through_float32():
    rng = np.random.default_rng(0)
    vals = np.concatenate([rng.normal(size=2000) * 10.0 ** rng.integers(-8, 6, 2000),
                           [0.0, -0.0, 1e-30, 3.4e38, 0.1, 1 / 3]]).astype(np.float32)
    for v in vals:
        s = S.fmt_f32(v)
        assert "e" not in s.lower()  # the reference's float pattern has no exponent
        assert np.float32(float(s)) == v


@pytest.mark.parametrize("make", [lambda: scenes.plain_scene(1),
                                  lambda: scenes.heightfield_scene(8),
                                  lambda: scenes.many_light_scene(2, res=(32, 18), spp=2, n_patches=12,
                                                                  n_groups=10, n_lights=20),
                                  lambda: scenes.motion_patch_scene(1, n=3),
                                  lambda: scenes.rect_light_scene(1, res=(8, 6), spp=1, n_spheres=3)])
def test_write_parse_round_trip(make):
    sc = make()
    txt = sc.to_psy()
    back = S.parse_psy(txt)
    assert back.to_psy() == txt
    assert back.res_x == sc.res_x and back.spp == sc.spp and back.seed == sc.seed
    # per-object time samples survive (patch motion: two Vertices blocks)
    for name, obj in sc.root.objects.items():
        if hasattr(obj, "verts"):
            assert back.root.objects[name].verts.shape == obj.verts.shape


def test_parser_handles_comments_escapes_and_defaults():
    txt = r"""
    # a comment
    Scene $s { RenderSettings { Resolution [4 3] SamplesPerPixel [2] Seed [9] DicingRate [0.5] }
      Camera { Fov [40] Transform [1 0 0 0 0 1 0 0 0 0 1 0 0 0 -5 1] }
      World { BackgroundShader { Type [Color] Color [0.1 0.2 0.3] } }
      Assembly {
        SurfaceShader $m\ x { Type [Lambert] Color [0.5 0.5 0.5] }
        Sphere $b { Location [1 2 3] }    # radius defaults to 0.5
        Instance { Data [$b] SurfaceShaderBind [$m\ x] }
      }
    }"""
    sc = S.parse_psy(txt)
    assert (sc.res_x, sc.res_y, sc.spp, sc.seed) == (4, 3, 2, 9)
    assert sc.dicing_rate == np.float32(0.5)
    assert sc.root.objects["b"].radius == np.float32(0.5)
    assert sc.root.instances[0].shader == "m x"
    np.testing.assert_array_equal(sc.background, np.float32([0.1, 0.2, 0.3]))


@pytest.mark.parametrize("bad", [
    "Scene $s { Assembly { Instance { Data [$missing] } } }",
    "Scene $s { Assembly { Sphere $a { Radius [1] } Instance { Data [$a] SurfaceShaderBind [$nope] } } }",
    "Scene $s { Assembly { Sphere $a { Radius [1] }",
    "Scene $s { Assembly { SurfaceShader $m { Color [1 1 1] } } }",
    "Nothing here",
])
def test_malformed_files_raise(bad):
    with pytest.raises(S.PsyParseError):
        S.parse_psy(bad)


def test_film_pfm_round_trip(tmp_path):
    """Film.write_pfm: mean XYZ per pixel, rows bottom to top, little-endian."""
    import torch
    from psychopath_cpp_b200 import api
    rng = np.random.default_rng(2)
    w, h = 7, 5
    xyz = rng.uniform(0, 3, (h, w, 3)).astype(np.float32)
    cnt = rng.integers(0, 4, (h, w)).astype(np.int32)
    film = api.Film(None, torch.from_numpy(xyz.reshape(-1)), torch.from_numpy(cnt.reshape(-1)), w, h)
    path = str(tmp_path / "f.pfm")
    film.write_pfm(path)
    data = open(path, "rb").read()
    header, rest = data.split(b"\n", 3)[:3], data.split(b"\n", 3)[3]
    assert header == [b"PF", b"7 5", b"-1.0"]
    img = np.frombuffer(rest, "<f4").reshape(h, w, 3)[::-1]
    expect = np.where(cnt[..., None] > 0, xyz / np.maximum(cnt[..., None], 1), 0)
    np.testing.assert_allclose(img, expect, rtol=1e-6)


# --------------------------------------------------------------------------
# The library's own .psy reader (psy_file_parse) against this module's
# reader + flatten(): the same scene description, field by field.
# --------------------------------------------------------------------------

def _f32s(ptr, n):
    return np.ctypeslib.as_array(ptr, shape=(n,)).copy() if n else np.zeros(0, np.float32)


def _obj_floats(o):
    k = o.kind
    if k == 0:
        return 4 * o.n0
    if k == 1:
        return 12 * o.n0
    if k == 2:
        return 48 * o.n0
    if k == 3:
        return 3 * o.n0 + o.n1 + 3 * o.n2
    return 2 * o.n0 + 3 * o.n1


def _desc_dict(d):
    """Every value a scene description holds, as plain Python data."""
    out = {"cam_transforms": _f32s(d.cam_transforms, 16 * d.cam_transform_count).tolist(),
           "cam_fovs": _f32s(d.cam_fovs, d.cam_fov_count).tolist(),
           "cam_apertures": _f32s(d.cam_aperture_radii, d.cam_aperture_count).tolist(),
           "cam_focus": _f32s(d.cam_focus_distances, d.cam_focus_count).tolist(),
           "background": list(d.background), "dice_rate": d.dice_rate, "min_upoly_size": d.min_upoly_size,
           "assemblies": [], "shaders": []}
    for ai in range(d.assembly_count):
        a = d.assemblies[ai]
        objs = []
        for oi in range(a.object_count):
            o = a.objects[oi]
            objs.append((o.kind, o.n0, o.n1, o.n2, _f32s(o.data, _obj_floats(o)).view(np.uint32).tolist()))
        insts = [(a.instances[i].kind, a.instances[i].data_index, a.instances[i].transform_index,
                  a.instances[i].transform_count, a.instances[i].shader) for i in range(a.instance_count)]
        out["assemblies"].append({"objects": objs, "instances": insts,
                                  "transforms": _f32s(a.transforms, 16 * a.transform_count).view(np.uint32).tolist(),
                                  "children": [a.children[i] for i in range(a.child_count)]})
    for si in range(d.shader_count):
        s = d.shaders[si]
        out["shaders"].append((s.kind, list(s.color), s.roughness, s.tail_shape, s.fresnel))
    return out


SCENE_MAKERS = [lambda: scenes.plain_scene(1),
                lambda: scenes.heightfield_scene(8),
                lambda: scenes.many_light_scene(2, res=(32, 18), spp=2, n_patches=12, n_groups=10, n_lights=20),
                lambda: scenes.motion_patch_scene(1, n=3),
                lambda: scenes.rect_light_scene(1, res=(8, 6), spp=1, n_spheres=3),
                lambda: scenes.gtr_scene(1, res=(8, 6), spp=1, n_spheres=4),
                lambda: scenes.batch_scene(3, (16, 12), 2, 300, 5)]


@pytest.mark.parametrize("make", SCENE_MAKERS)
def test_library_reader_matches_python_reader(make):
    from psychopath_cpp_b200 import api
    txt = make().to_psy()
    sc = S.parse_psy(txt)
    mine = api.PsyFile(txt)
    py_desc, keep = api.flatten(sc)
    assert _desc_dict(mine.desc) == _desc_dict(py_desc)
    assert mine.settings == {"width": sc.res_x, "height": sc.res_y, "spp": sc.spp, "seed": sc.seed}
    # the host builders see the same scene
    a = api.build_bvh4_records(sc, 0)
    b = api.build_bvh4_records(mine, 0)
    for k in a:
        np.testing.assert_array_equal(np.asarray(a[k]), np.asarray(b[k]))
    la, lb = api.build_light_tree(sc, 0), api.build_light_tree(mine, 0)
    for k in la:
        np.testing.assert_array_equal(np.asarray(la[k]), np.asarray(lb[k]))


HAND_WRITTEN = r"""
# comments, escapes, defaults and partial matrices
Scene $s { RenderSettings { Resolution [4 3] SamplesPerPixel [2] Seed [9] DicingRate [0.5] }
  Camera { Fov [40] Fov [50.] ApertureRadius [0.1] FocalDistance [7]
           Transform [1 0 0 0 0 1 0 0 0 0 1 0 0 0 -5 1] Transform [2 0 0] }
  World { BackgroundShader { Type [Color] Color [0.1 0.2] } }
  Assembly {
    SurfaceShader $m\ x { Type [Lambert] Color [0.5 0.5 0.5] }
    SurfaceShader $g { Type [GTR] Color [0.3] Roughness [0.4] TailShape [1.5] Fresnel [0.7] }
    Sphere $b { Location [1 2 3] }
    Sphere $c { Radius [-1.25] Location [-1 -2] }
    SphereLight $l { Location [0 0 4] Location [0 1 4] Radius [0.3] Color [5 5 5] Color [6 6 6] }
    RectangleLight $r { Dimensions [2] Color [1 2 3] }
    BilinearPatch $p { Vertices [0 0 0  1 0 0  0 1 0  1 1 0.5] }
    Assembly $sub {
      Sphere $inner { Radius [0.2] }
      SurfaceShader $g { Type [Emit] Color [9 9 9] }
      Instance { Data [$inner] SurfaceShaderBind [$g] }
      Instance { Data [$inner] SurfaceShaderBind [$m\ x] Transform [1 0 0 0 0 1 0 0 0 0 1 0 3 0 0 1] }
    }
    Instance { Data [$b] SurfaceShaderBind [$m\ x] }
    Instance { Data [$c] SurfaceShaderBind [$g] Transform [1 0 0 0 0 1 0 0 0 0 1 0 0 0 1 1]
               Transform [1 0 0 0 0 1 0 0 0 0 1 0 0 0 2 1] }
    Instance { Data [$l] }
    Instance { Data [$r] Transform [1 0 0 0 0 0 1 0 0 -1 0 0 0 0 5 1] }
    Instance { Data [$p] SurfaceShaderBind [$m\ x] }
    Instance { Data [$sub] }
  }
}"""


def test_library_reader_hand_written_file():
    """Comments, escaped names, float forms ("50.", "-1.25"), partial
    colours and matrices filled from the defaults, a shader of the nested
    assembly's own hiding the enclosing one's and one found in the
    enclosing assembly, motion transforms, every object kind, a nested
    assembly."""
    from psychopath_cpp_b200 import api
    sc = S.parse_psy(HAND_WRITTEN)
    mine = api.PsyFile(HAND_WRITTEN)
    py_desc, keep = api.flatten(sc)
    d = _desc_dict(mine.desc)
    assert d == _desc_dict(py_desc)
    assert mine.settings == {"width": 4, "height": 3, "spp": 2, "seed": 9}
    assert d["dice_rate"] == np.float32(0.5)
    # Transform [2 0 0]: the rest of the identity
    assert d["cam_transforms"][16:] == [2.0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1]
    assert d["background"] == pytest.approx([0.1, 0.2, 0.0])
    assert len(d["assemblies"]) == 2 and d["assemblies"][0]["children"] == [1]
    # the nested assembly's $g is its own Emit shader; $m x the root's
    sub = d["assemblies"][1]["instances"]
    assert d["shaders"][sub[0][4]][0] == 1 and d["shaders"][sub[1][4]][0] == 0


@pytest.mark.parametrize("bad", [
    "Scene $s { Assembly { Instance { Data [$missing] } } }",
    "Scene $s { Assembly { Sphere $a { Radius [1] } Instance { Data [$a] SurfaceShaderBind [$nope] } } }",
    "Scene $s { Assembly { Sphere $a { Radius [1] }",
    "Scene $s { Assembly { SurfaceShader $m { Color [1 1 1] } } }",
    "Scene $s { Assembly { SubdivisionSurface $q { } } }",
    "Scene $s { Assembly { Sphere $a { Radius [1 } } }",
    "Scene $s } }",
    "Nothing here",
    "",
])
def test_library_reader_rejects_malformed_files(bad):
    from psychopath_cpp_b200 import _abi, api
    with pytest.raises(_abi.PsyError) as e:
        api.PsyFile(bad)
    assert e.value.code == _abi.PSY_ERR_ARG and str(e.value).split(": ", 1)[1]


@pytest.mark.parametrize("make", SCENE_MAKERS)
def test_library_reader_reads_back_the_written_scene(make):
    """The writer's file read by the library gives the scene's own
    description (floats are written so that they read back exactly)."""
    from psychopath_cpp_b200 import api
    sc = make()
    d, keep = api.flatten(sc)
    assert _desc_dict(api.PsyFile(sc.to_psy()).desc) == _desc_dict(d)


def test_library_reader_frames():
    """A file of several Scene nodes read frame by frame, as the reference's
    parse_next_frame reads them; past the last frame, PSY_ERR_NO_SCENE."""
    from psychopath_cpp_b200 import _abi, api
    a = scenes.plain_scene(1, res=(8, 6), spp=1, n_spheres=3)
    b = scenes.rect_light_scene(1, res=(10, 4), spp=3, n_spheres=2)
    txt = a.to_psy() + "\n" + b.to_psy()
    for frame, sc in enumerate((a, b)):
        f = api.PsyFile(txt, frame)
        d, keep = api.flatten(sc)
        assert _desc_dict(f.desc) == _desc_dict(d)
        assert f.settings["width"] == sc.res_x and f.settings["spp"] == sc.spp
    with pytest.raises(_abi.PsyError) as e:
        api.PsyFile(txt, 2)
    assert e.value.code == _abi.PSY_ERR_NO_SCENE


def test_library_reader_binds_names_as_the_reference():
    """Name rules of the reference's Assembly and parser (scene/assembly.hpp:
    104-157, parser/parser.cpp:298-323): a repeated name keeps every
    definition and finds the first; an instance binds the shader of that
    name defined so far (here the enclosing assembly's, as the nested one's
    comes later); names match as written."""
    from psychopath_cpp_b200 import _abi, api
    txt = r"""
    Scene $s { Assembly {
      SurfaceShader $g { Type [Lambert] Color [0.1 0.2 0.3] }
      SurfaceShader $g { Type [Lambert] Color [0.9 0.9 0.9] }
      Sphere $a { Radius [1] }
      Sphere $a { Radius [2] }
      SphereLight $l { Location [0 0 4] Radius [0.5] Color [3 3 3] }
      Assembly $sub {
        Sphere $b { Radius [0.5] }
        Instance { Data [$b] SurfaceShaderBind [$g] }
        SurfaceShader $g { Type [Emit] Color [7 7 7] }
        Instance { Data [$b] SurfaceShaderBind [$g] }
      }
      Instance { Data [$a] SurfaceShaderBind [$g] }
      Instance { Data [$l] }
      Instance { Data [$sub] }
    } }"""
    d = _desc_dict(api.PsyFile(txt).desc)
    root, sub = d["assemblies"]
    assert len(root["objects"]) == 3 and root["instances"][0][1] == 0       # the first $a
    assert np.uint32(root["objects"][0][4][3]).view(np.float32) == 1.0
    first_g = d["shaders"][root["instances"][0][4]]
    assert first_g[0] == 0 and first_g[1] == pytest.approx([0.1, 0.2, 0.3])  # the first $g
    assert sub["instances"][0][4] == root["instances"][0][4]                # the root's $g, read so far
    assert d["shaders"][sub["instances"][1][4]][0] == 1                     # then the nested Emit $g
    with pytest.raises(_abi.PsyError):
        api.PsyFile("Scene $s { Assembly { Sphere $a { Radius [1] } Instance { Data [a] } } }")
    # the Python reader binds and resolves names the same way
    sc = S.parse_psy(txt)
    py_desc, keep = api.flatten(sc)
    pd = _desc_dict(py_desc)
    assert [i[4] for i in pd["assemblies"][1]["instances"]] == [i[4] for i in sub["instances"]]
    assert [pd["shaders"][i[4]] for i in pd["assemblies"][1]["instances"]] == \
        [d["shaders"][i[4]] for i in sub["instances"]]


def test_library_reader_output_path_and_defaults():
    """Output Path as the reference takes it (the text between the first
    and last double quote, quotes removed) and its render-setting defaults
    (parser/parser.cpp:61-76): 1 x 1 pixels, 1 sample, seed 1."""
    from psychopath_cpp_b200 import api
    f = api.PsyFile('Scene $s { Output { Path ["out/a"b".png"] } Assembly { } }')
    assert f.output_path == "out/ab.png"
    assert f.settings == {"width": 1, "height": 1, "spp": 1, "seed": 1}
    assert api.PsyFile("Scene $s { Assembly { } }").output_path == ""
