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
