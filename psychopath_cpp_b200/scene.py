"""Scene description mirroring the reference renderer's scene types.

The classes follow the reference's scene/assembly model
(reference scene/scene.hpp:33-53, scene/assembly.hpp:26-330,
object/sphere.hpp, object/bilinear.hpp, object/bicubic.hpp,
lights/sphere_light.hpp, shading/surface_shader.hpp, basics/camera.hpp):
a Scene holds a camera, a background colour and a root Assembly; an
Assembly holds shaders, objects, sub-assemblies and the instances that place
them (with optional motion transforms and a bound surface shader).

Two serialisations are provided:

* ``Scene.to_psy()`` writes the reference's ``.psy`` text format
  (reference parser/parser.cpp:37-662).  Every number is written as the
  shortest positional decimal that reads back to the same float32, because
  the reference parser's float pattern (parser/parser.cpp:31) accepts no
  exponent and converts with ``std::stof``.
* ``parse_psy(text)`` reads that format back into a Scene (a restatement of
  the reference's DataTree + Parser for the node types on the hot path).

All geometric values are stored as float32, exactly as the reference holds
them after parsing.
"""
from __future__ import annotations

import re
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Union

import numpy as np

F32 = np.float32


def _f32(x) -> np.ndarray:
    return np.asarray(x, dtype=np.float32)


def fmt_f32(x) -> str:
    """Shortest positional decimal that ``std::stof`` reads back as ``x``."""
    v = F32(x)
    if not np.isfinite(v):
        raise ValueError("non-finite value cannot be written to .psy: %r" % (x,))
    s = np.format_float_positional(v, unique=True, trim="-")
    if F32(float(s)) != v:  # guard against double-rounding on read-back
        s = np.format_float_positional(v, precision=12, unique=False, trim="-")
        if F32(float(s)) != v:
            raise ValueError("cannot round-trip %r" % (x,))
    return s


def _fmt_list(vals) -> str:
    return " ".join(fmt_f32(v) for v in np.asarray(vals, dtype=np.float32).ravel())


# --------------------------------------------------------------------------
# Scene element types
# --------------------------------------------------------------------------


@dataclass
class SurfaceShader:
    """Lambert / Emit / GTR shader (reference shading/surface_shader.hpp:28-72)."""

    kind: str = "Lambert"
    color: np.ndarray = field(default_factory=lambda: _f32([0.9, 0.9, 0.9]))
    roughness: float = 0.1
    tail_shape: float = 2.0
    fresnel: float = 0.25

    def __post_init__(self):
        self.color = _f32(self.color).reshape(3)


@dataclass
class Sphere:
    """Sphere with one time sample (the parser gives spheres no motion,
    reference parser/parser.cpp:629-662)."""

    location: np.ndarray = field(default_factory=lambda: _f32([0, 0, 0]))
    radius: float = 0.5

    def __post_init__(self):
        self.location = _f32(self.location).reshape(3)
        self.radius = F32(self.radius)


@dataclass
class BilinearPatch:
    """Bilinear patch, verts shaped (time_samples, 4, 3), ordered
    v1 v2 / v3 v4 as in reference object/bilinear.hpp:15-21."""

    verts: np.ndarray

    def __post_init__(self):
        self.verts = _f32(self.verts).reshape(-1, 4, 3)


@dataclass
class BicubicPatch:
    """Bicubic Bezier patch, verts shaped (time_samples, 16, 3), row-major
    4x4 control grid as in reference object/bicubic.hpp:15-25."""

    verts: np.ndarray

    def __post_init__(self):
        self.verts = _f32(self.verts).reshape(-1, 16, 3)


@dataclass
class SphereLight:
    """Sphere light with per-time-sample locations, radii and colours
    (reference lights/sphere_light.hpp:15-57)."""

    locations: np.ndarray
    radii: np.ndarray
    colors: np.ndarray

    def __post_init__(self):
        self.locations = _f32(self.locations).reshape(-1, 3)
        self.radii = _f32(self.radii).reshape(-1)
        self.colors = _f32(self.colors).reshape(-1, 3)


@dataclass
class RectangleLight:
    """Rectangle light in its local xy plane, centred on the origin, with
    per-time-sample dimensions (x, y) and colours (reference
    lights/rectangle_light.hpp:16-40, parser/parser.cpp:597-632)."""

    dimensions: np.ndarray
    colors: np.ndarray

    def __post_init__(self):
        self.dimensions = _f32(self.dimensions).reshape(-1, 2)
        self.colors = _f32(self.colors).reshape(-1, 3)


SceneObject = Union[Sphere, BilinearPatch, BicubicPatch, SphereLight, RectangleLight]


@dataclass
class Instance:
    """Placement of an object or sub-assembly (reference scene/assembly.hpp:26-66).

    ``transforms`` are world-to-local 4x4 matrices in the reference's
    row-vector convention, one per motion time sample."""

    data: str
    transforms: List[np.ndarray] = field(default_factory=list)
    shader: Optional[str] = None
    # the shader bound when the instance was read from a file: the one of
    # that name defined so far, as the reference binds it
    # (parser/parser.cpp:298-323); None: looked up by name when flattened
    bound: Optional["SurfaceShader"] = field(default=None, repr=False, compare=False)

    def __post_init__(self):
        self.transforms = [_f32(t).reshape(4, 4) for t in self.transforms]


@dataclass
class Assembly:
    """Shaders, objects, sub-assemblies and instances, in declaration order."""

    shaders: Dict[str, SurfaceShader] = field(default_factory=dict)
    objects: Dict[str, SceneObject] = field(default_factory=dict)
    assemblies: Dict[str, "Assembly"] = field(default_factory=dict)
    instances: List[Instance] = field(default_factory=list)
    parent: Optional["Assembly"] = None

    def add_shader(self, name: str, shader: SurfaceShader) -> str:
        self.shaders[name] = shader
        return name

    def add_object(self, name: str, obj: SceneObject) -> str:
        self.objects[name] = obj
        return name

    def add_assembly(self, name: str, asm: "Assembly") -> str:
        asm.parent = self
        self.assemblies[name] = asm
        return name

    def add_instance(self, data: str, transforms: Sequence = (), shader: Optional[str] = None) -> Instance:
        inst = Instance(data, list(transforms), shader)
        self.instances.append(inst)
        return inst

    def shader_of(self, inst: "Instance") -> Optional[SurfaceShader]:
        """The shader an instance of this assembly renders with."""
        if inst.bound is not None:
            return inst.bound
        return self.find_shader(inst.shader) if inst.shader is not None else None

    def find_shader(self, name: str) -> Optional[SurfaceShader]:
        """Shader lookup through the parent chain
        (reference scene/assembly.hpp:113-121)."""
        a: Optional[Assembly] = self
        while a is not None:
            if name in a.shaders:
                return a.shaders[name]
            a = a.parent
        return None


@dataclass
class Camera:
    """Camera time samples (reference basics/camera.hpp:22-64).

    ``fovs`` are in degrees, as written in .psy files; the reference parser
    converts them with ``(3.1415926536f/180.0f) * value`` in float."""

    transforms: List[np.ndarray] = field(default_factory=lambda: [np.eye(4, dtype=np.float32)])
    fovs: List[float] = field(default_factory=lambda: [45.0])
    aperture_radii: List[float] = field(default_factory=list)
    focus_distances: List[float] = field(default_factory=list)

    def __post_init__(self):
        self.transforms = [_f32(t).reshape(4, 4) for t in self.transforms]
        self.fovs = [F32(f) for f in self.fovs]
        self.aperture_radii = [F32(f) for f in self.aperture_radii]
        self.focus_distances = [F32(f) for f in self.focus_distances]

    def fovs_radians(self) -> np.ndarray:
        k = F32(3.1415926536) / F32(180.0)
        return np.array([F32(k * f) for f in self.fovs], dtype=np.float32)


@dataclass
class Scene:
    name: str = "scene"
    res_x: int = 64
    res_y: int = 64
    spp: int = 1
    seed: int = 1
    dicing_rate: Optional[float] = None
    camera: Camera = field(default_factory=Camera)
    background: np.ndarray = field(default_factory=lambda: _f32([0, 0, 0]))
    root: Assembly = field(default_factory=Assembly)

    def __post_init__(self):
        self.background = _f32(self.background).reshape(3)

    # ------------------------------------------------------------------
    def to_psy(self) -> str:
        out: List[str] = []
        w = out.append
        w("Scene $%s {\n" % self.name)
        w("\tRenderSettings {\n")
        w("\t\tResolution [%d %d]\n" % (self.res_x, self.res_y))
        w("\t\tSamplesPerPixel [%d]\n" % self.spp)
        if self.dicing_rate is not None:
            w("\t\tDicingRate [%s]\n" % fmt_f32(self.dicing_rate))
        w("\t\tSeed [%d]\n" % self.seed)
        w("\t}\n")
        cam = self.camera
        w("\tCamera {\n")
        for f in cam.fovs:
            w("\t\tFov [%s]\n" % fmt_f32(f))
        for f in cam.focus_distances:
            w("\t\tFocalDistance [%s]\n" % fmt_f32(f))
        for f in cam.aperture_radii:
            w("\t\tApertureRadius [%s]\n" % fmt_f32(f))
        for t in cam.transforms:
            w("\t\tTransform [%s]\n" % _fmt_list(t))
        w("\t}\n")
        w("\tWorld {\n\t\tBackgroundShader {\n\t\t\tType [Color]\n")
        w("\t\t\tColor [%s]\n\t\t}\n\t}\n" % _fmt_list(self.background))
        self._write_assembly(self.root, None, 1, w)
        w("}\n")
        return "".join(out)

    @staticmethod
    def _write_assembly(asm: Assembly, name: Optional[str], depth: int, w) -> None:
        ind = "\t" * depth
        w("%sAssembly%s {\n" % (ind, (" $" + name) if name else ""))
        ind2 = ind + "\t"
        for sname, sh in asm.shaders.items():
            w("%sSurfaceShader $%s {\n" % (ind2, sname))
            w("%s\tType [%s]\n" % (ind2, sh.kind))
            w("%s\tColor [%s]\n" % (ind2, _fmt_list(sh.color)))
            if sh.kind == "GTR":
                w("%s\tRoughness [%s]\n" % (ind2, fmt_f32(sh.roughness)))
                w("%s\tTailShape [%s]\n" % (ind2, fmt_f32(sh.tail_shape)))
                w("%s\tFresnel [%s]\n" % (ind2, fmt_f32(sh.fresnel)))
            w("%s}\n" % ind2)
        for sub_name, sub in asm.assemblies.items():
            Scene._write_assembly(sub, sub_name, depth + 1, w)
        for oname, obj in asm.objects.items():
            if isinstance(obj, Sphere):
                w("%sSphere $%s {\n%s\tLocation [%s]\n%s\tRadius [%s]\n%s}\n"
                  % (ind2, oname, ind2, _fmt_list(obj.location), ind2, fmt_f32(obj.radius), ind2))
            elif isinstance(obj, BilinearPatch):
                w("%sBilinearPatch $%s {\n" % (ind2, oname))
                for ts in obj.verts:
                    w("%s\tVertices [%s]\n" % (ind2, _fmt_list(ts)))
                w("%s}\n" % ind2)
            elif isinstance(obj, BicubicPatch):
                w("%sBicubicPatch $%s {\n" % (ind2, oname))
                for ts in obj.verts:
                    w("%s\tVertices [%s]\n" % (ind2, _fmt_list(ts)))
                w("%s}\n" % ind2)
            elif isinstance(obj, SphereLight):
                w("%sSphereLight $%s {\n" % (ind2, oname))
                for c in obj.colors:
                    w("%s\tColor [%s]\n" % (ind2, _fmt_list(c)))
                for r in obj.radii:
                    w("%s\tRadius [%s]\n" % (ind2, fmt_f32(r)))
                for loc in obj.locations:
                    w("%s\tLocation [%s]\n" % (ind2, _fmt_list(loc)))
                w("%s}\n" % ind2)
            elif isinstance(obj, RectangleLight):
                w("%sRectangleLight $%s {\n" % (ind2, oname))
                for c in obj.colors:
                    w("%s\tColor [%s]\n" % (ind2, _fmt_list(c)))
                for d in obj.dimensions:
                    w("%s\tDimensions [%s]\n" % (ind2, _fmt_list(d)))
                w("%s}\n" % ind2)
            else:
                raise TypeError("unsupported object %r" % (type(obj),))
        for inst in asm.instances:
            w("%sInstance {\n%s\tData [$%s]\n" % (ind2, ind2, inst.data))
            for t in inst.transforms:
                w("%s\tTransform [%s]\n" % (ind2, _fmt_list(t)))
            if inst.shader is not None:
                w("%s\tSurfaceShaderBind [$%s]\n" % (ind2, inst.shader))
            w("%s}\n" % ind2)
        w("%s}\n" % ind)

    def write_psy(self, path: str) -> None:
        with open(path, "w") as f:
            f.write(self.to_psy())


# --------------------------------------------------------------------------
# .psy reader
# --------------------------------------------------------------------------

# Same number patterns as the reference parser (parser/parser.cpp:28-29).
_RE_INT = re.compile(r"-?[0-9]+")
_RE_FLOAT = re.compile(r"-?[0-9]+[.]?[0-9]*")


class PsyParseError(ValueError):
    pass


@dataclass
class _Node:
    type: str
    name: str = ""
    leaf: Optional[str] = None
    children: List["_Node"] = field(default_factory=list)


def _tokenize(text: str):
    """Tokens of the DataTree format (reference parser/data_tree.cpp:177-400):
    TYPE identifiers, $NAMEs (with backslash escapes), { } and [leaf] bodies."""
    i, n = 0, len(text)
    toks = []
    while i < n:
        c = text[i]
        if c.isspace():
            i += 1
        elif c == "#":
            while i < n and text[i] != "\n":
                i += 1
        elif c in "{}":
            toks.append((c, c))
            i += 1
        elif c == "[":
            i += 1
            buf = []
            while i < n and text[i] != "]":
                if text[i] == "\\" and i + 1 < n:
                    buf.append(text[i + 1])
                    i += 2
                else:
                    buf.append(text[i])
                    i += 1
            if i >= n:
                raise PsyParseError("unterminated leaf contents")
            i += 1
            toks.append(("LEAF", "".join(buf).strip()))
        elif c == "$":
            buf = ["$"]
            i += 1
            while i < n:
                if text[i] == "\\" and i + 1 < n:
                    buf.append(text[i + 1])
                    i += 2
                elif text[i].isspace() or text[i] in "{}[]#$":
                    break
                else:
                    buf.append(text[i])
                    i += 1
            toks.append(("NAME", "".join(buf)))
        else:
            j = i
            while j < n and not (text[j].isspace() or text[j] in "{}[]#$"):
                j += 1
            if j == i:
                raise PsyParseError("unexpected character %r" % c)
            toks.append(("TYPE", text[i:j]))
            i = j
    return toks


def _build_tree(toks) -> _Node:
    root = _Node("ROOT")
    stack = [root]
    i = 0
    while i < len(toks):
        kind, val = toks[i]
        if kind == "}":
            if len(stack) == 1:
                raise PsyParseError("unbalanced '}'")
            stack.pop()
            i += 1
            continue
        if kind != "TYPE":
            raise PsyParseError("expected a type name, got %r" % (val,))
        node = _Node(val)
        i += 1
        if i < len(toks) and toks[i][0] == "NAME":
            node.name = toks[i][1]
            i += 1
        if i >= len(toks):
            raise PsyParseError("unexpected end of file after %r" % val)
        if toks[i][0] == "LEAF":
            node.leaf = toks[i][1]
            i += 1
            stack[-1].children.append(node)
        elif toks[i][0] == "{":
            i += 1
            stack[-1].children.append(node)
            stack.append(node)
        else:
            raise PsyParseError("expected '{' or '[' after %r" % val)
    if len(stack) != 1:
        raise PsyParseError("unbalanced '{'")
    return root


def _floats(s: str, limit: Optional[int] = None) -> List[np.float32]:
    vals = [F32(float(m)) for m in _RE_FLOAT.findall(s)]
    return vals[:limit] if limit is not None else vals


def _ints(s: str) -> List[int]:
    return [int(m) for m in _RE_INT.findall(s)]


def _matrix(s: str) -> np.ndarray:
    m = np.eye(4, dtype=np.float32).ravel()
    vals = _floats(s, 16)
    m[: len(vals)] = vals
    return m.reshape(4, 4)


def _color(s: str, default=(0.0, 0.0, 0.0)) -> np.ndarray:
    c = _f32(default).copy()
    vals = _floats(s, 3)
    c[: len(vals)] = vals
    return c


def _parse_assembly(node: _Node, parent: Optional[Assembly]) -> Assembly:
    """An Assembly node.  A repeated name keeps its first definition, as
    the reference's name maps do (scene/assembly.hpp:104-157)."""
    asm = Assembly(parent=parent)
    for ch in node.children:
        t = ch.type
        key = ch.name[1:]
        if ((t in ("BilinearPatch", "BicubicPatch", "Sphere", "SphereLight", "RectangleLight") and key in asm.objects)
                or (t == "SurfaceShader" and key in asm.shaders) or (t == "Assembly" and key in asm.assemblies)):
            continue
        if t == "Assembly":
            asm.add_assembly(ch.name[1:], _parse_assembly(ch, asm))
        elif t == "BilinearPatch":
            vs = [_floats(c.leaf, 12) for c in ch.children if c.type == "Vertices"]
            asm.add_object(ch.name[1:], BilinearPatch(np.array(vs, dtype=np.float32)))
        elif t == "BicubicPatch":
            vs = [_floats(c.leaf, 48) for c in ch.children if c.type == "Vertices"]
            asm.add_object(ch.name[1:], BicubicPatch(np.array(vs, dtype=np.float32)))
        elif t == "Sphere":
            loc, rad = _f32([0, 0, 0]), F32(0.5)
            for c in ch.children:
                if c.type == "Radius":
                    v = _floats(c.leaf, 1)
                    if v:
                        rad = v[0]
                elif c.type == "Location":
                    loc = _color(c.leaf)
            asm.add_object(ch.name[1:], Sphere(loc, rad))
        elif t == "SurfaceShader":
            kind = next((c.leaf for c in ch.children if c.type == "Type"), None)
            if kind is None:
                raise PsyParseError("surface shader without a type")
            sh = SurfaceShader(kind, _f32([0.9, 0.9, 0.9]))
            for c in ch.children:
                if c.type == "Color":
                    sh.color = _color(c.leaf, (0.9, 0.9, 0.9))
                elif c.type == "Roughness":
                    sh.roughness = _floats(c.leaf, 1)[0]
                elif c.type == "TailShape":
                    sh.tail_shape = _floats(c.leaf, 1)[0]
                elif c.type == "Fresnel":
                    sh.fresnel = _floats(c.leaf, 1)[0]
            asm.add_shader(ch.name[1:], sh)
        elif t == "SphereLight":
            cols, rads, locs = [], [], []
            for c in ch.children:
                if c.type == "Color":
                    cols.append(_color(c.leaf))
                elif c.type == "Radius":
                    v = _floats(c.leaf, 1)
                    if v:
                        rads.append(v[0])
                elif c.type == "Location":
                    locs.append(_color(c.leaf))
            if not locs:
                locs = [_f32([0, 0, 0])]
            asm.add_object(ch.name[1:], SphereLight(np.array(locs), np.array(rads, dtype=np.float32), np.array(cols)))
        elif t == "RectangleLight":
            cols, dims = [], []
            for c in ch.children:
                if c.type == "Color":
                    cols.append(_color(c.leaf))
                elif c.type == "Dimensions":
                    v = _floats(c.leaf, 2)
                    dims.append([v[0] if len(v) > 0 else 1.0, v[1] if len(v) > 1 else 1.0])
            asm.add_object(ch.name[1:], RectangleLight(np.array(dims, dtype=np.float32), np.array(cols)))
        elif t == "Instance":
            data, xf, shader = "", [], None
            for c in ch.children:
                if c.type == "Transform":
                    xf.append(_matrix(c.leaf))
                elif c.type == "Data":
                    data = c.leaf
                elif c.type == "SurfaceShaderBind":
                    shader = c.leaf
            data = data[1:] if data.startswith("$") else data
            if shader is not None:
                shader = shader[1:] if shader.startswith("$") else shader
                if asm.find_shader(shader) is None:
                    raise PsyParseError("instance binds unknown shader %r" % shader)
            if data not in asm.objects and data not in asm.assemblies:
                raise PsyParseError("instance of unknown data %r" % data)
            asm.add_instance(data, xf, shader).bound = asm.find_shader(shader) if shader is not None else None
        elif t in ("RectangleLight", "SubdivisionSurface"):
            raise PsyParseError("%s is outside the supported hot path" % t)
    return asm


def parse_psy(text: str) -> Scene:
    """Parses the first Scene of a .psy document (reference parser/parser.cpp:37-184)."""
    tree = _build_tree(_tokenize(text))
    snode = next((c for c in tree.children if c.type == "Scene"), None)
    if snode is None:
        raise PsyParseError("no Scene node")
    sc = Scene(name=snode.name[1:] if snode.name else "scene")
    for node in snode.children:
        if node.type == "RenderSettings":
            for c in node.children:
                if c.type == "Resolution":
                    v = _ints(c.leaf)
                    if len(v) >= 1:
                        sc.res_x = v[0]
                    if len(v) >= 2:
                        sc.res_y = v[1]
                elif c.type == "SamplesPerPixel":
                    sc.spp = _ints(c.leaf)[0]
                elif c.type == "DicingRate":
                    sc.dicing_rate = _floats(c.leaf, 1)[0]
                elif c.type == "Seed":
                    sc.seed = _ints(c.leaf)[0]
        elif node.type == "Camera":
            cam = Camera(transforms=[], fovs=[])
            for c in node.children:
                if c.type == "Fov":
                    cam.fovs.append(_floats(c.leaf, 1)[0])
                elif c.type == "FocalDistance":
                    cam.focus_distances.append(_floats(c.leaf, 1)[0])
                elif c.type == "ApertureRadius":
                    cam.aperture_radii.append(_floats(c.leaf, 1)[0])
                elif c.type == "Transform":
                    cam.transforms.append(_matrix(c.leaf))
            sc.camera = cam
        elif node.type == "World":
            for c in node.children:
                if c.type == "BackgroundShader":
                    kind = next((d.leaf for d in c.children if d.type == "Type"), None)
                    if kind is None:
                        raise PsyParseError("background shader without a type")
                    if kind == "Color":
                        for d in c.children:
                            if d.type == "Color":
                                sc.background = _color(d.leaf)
        elif node.type == "Assembly":
            sc.root = _parse_assembly(node, None)
    return sc


def read_psy(path: str) -> Scene:
    with open(path) as f:
        return parse_psy(f.read())
