"""Generates spectral_table.inc, the RGB->spectrum upsampling grid of
Hanika, Jakob & Dachsbacher, "Physically Meaningful Rendering using
Tristimulus Colours" (2015), in this project's own layout.

The grid (12x14 cells over the rotated xy chromaticity plane, 5 nm spectra
over 380-780 nm normalised to X+Y+Z = 1) is published data; the reference
renderer vendors it as color/spectra_xyz_5nm_380_780_0.97.h.  Spectral
parity with the reference needs exactly the same float values, so this
script reads that header and re-emits the numbers, converted the way a C
compiler converts them: unsuffixed literals as double then float, `f`
literals directly to the nearest float.

    python psychopath_cpp_b200/csrc/gen_spectral_table.py <path to spectra_xyz_5nm_380_780_0.97.h>
"""
from __future__ import annotations

import os
import re
import sys
from fractions import Fraction

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "spectral_table.inc")

NUM = re.compile(r"-?(?:\d+\.\d*|\.\d+|\d+)(?:[eE][-+]?\d+)?f?")


def to_f32(tok: str) -> np.float32:
    """C semantics: `1.5f` rounds the decimal straight to float; `1.5`
    rounds to double first and the double is then converted to float."""
    if tok.endswith("f"):
        exact = Fraction(tok[:-1])
        c = np.float32(float(tok[:-1]))
        best = c
        best_d = abs(Fraction(float(c)) - exact)
        for cand in (np.nextafter(c, np.float32(np.inf)), np.nextafter(c, np.float32(-np.inf))):
            d = abs(Fraction(float(cand)) - exact)
            if d < best_d or (d == best_d and (int(cand.view(np.uint32)) & 1) == 0):
                best, best_d = cand, d
        return np.float32(best)
    return np.float32(float(tok))


def block(text: str, name: str) -> str:
    i = text.index(name)
    j = text.index("{", i)
    depth, k = 0, j
    while True:
        if text[k] == "{":
            depth += 1
        elif text[k] == "}":
            depth -= 1
            if depth == 0:
                return text[j:k + 1]
        k += 1


def scalar(text: str, name: str) -> str:
    m = re.search(name + r"\s*=\s*([^;]+);", text)
    return m.group(1).strip()


def main(path: str) -> None:
    text = open(path).read()
    text = re.sub(r"//[^\n]*", "", text)
    width = int(scalar(text, "spectrum_grid_width"))
    height = int(scalar(text, "spectrum_grid_height"))
    nsamp = int(scalar(text, "spectrum_num_samples"))
    smin = to_f32(scalar(text, "spectrum_sample_min"))
    smax = to_f32(scalar(text, "spectrum_sample_max"))
    eer = to_f32(scalar(text, "equal_energy_reflectance"))
    m_uv = [to_f32(t) for t in NUM.findall(block(text, "spectrum_mat_xy_to_uv[]"))]
    assert len(m_uv) == 6
    cells_txt = block(text, "spectrum_grid[] =")
    cells = re.findall(r"\{\s*(-?\d+)\s*,\s*(-?\d+)\s*,\s*\{([^}]*)\}\s*\}", cells_txt)
    assert len(cells) == width * height, len(cells)
    pts_txt = block(text, "spectrum_data_points[] =")
    pts = re.findall(r"\{\s*\{([^}]*)\}\s*,\s*\{([^}]*)\}\s*,\s*\{([^}]*)\}\s*\}", pts_txt)
    out = []
    w = out.append
    w("/* Generated by gen_spectral_table.py from the published Hanika et al. (2015)\n"
      " * RGB->spectrum grid; do not edit.  Layout: cell records, then per data\n"
      " * point its uv coordinate and %d spectral samples. */\n" % nsamp)
    w("#define PSY_SPEC_GRID_W %d\n#define PSY_SPEC_GRID_H %d\n#define PSY_SPEC_SAMPLES %d\n" % (width, height, nsamp))
    w("#define PSY_SPEC_POINTS %d\n" % len(pts))
    w("#ifndef PSY_SPEC_QUAL\n#define PSY_SPEC_QUAL\n#endif\n")
    def f(v):
        return "%.9ef" % float(v) if np.isfinite(v) else "0.0f"
    w("PSY_SPEC_QUAL static const float psy_spec_sample_min = %s;\nPSY_SPEC_QUAL static const float psy_spec_sample_max = %s;\n" % (f(smin), f(smax)))
    w("PSY_SPEC_QUAL static const float psy_spec_equal_energy_reflectance = %s;\n" % f(eer))
    w("PSY_SPEC_QUAL static const float psy_spec_xy_to_uv[6] = {%s};\n" % ", ".join(f(v) for v in m_uv))
    w("/* inside, num_points, idx[6] */\nPSY_SPEC_QUAL static const int psy_spec_cells[%d][8] = {\n" % (width * height))
    for inside, num, idx in cells:
        ids = [int(x) for x in idx.split(",")]
        assert len(ids) == 6
        w("  {%s, %s, %s},\n" % (inside, num, ", ".join(str(i) for i in ids)))
    w("};\n")
    w("PSY_SPEC_QUAL static const float psy_spec_point_uv[%d][2] = {\n" % len(pts))
    for _, uv, _ in pts:
        vals = [to_f32(t) for t in NUM.findall(uv)]
        w("  {%s},\n" % ", ".join(f(v) for v in vals))
    w("};\n")
    w("PSY_SPEC_QUAL static const float psy_spec_point_spectrum[%d][%d] = {\n" % (len(pts), nsamp))
    for _, _, sp in pts:
        vals = [to_f32(t) for t in NUM.findall(sp)]
        assert len(vals) == nsamp, len(vals)
        w("  {%s},\n" % ", ".join(f(v) for v in vals))
    w("};\n")
    with open(OUT, "w") as fh:
        fh.write("".join(out))
    print("wrote", OUT, len(pts), "points")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: gen_spectral_table.py <reference>/color/spectra_xyz_5nm_380_780_0.97.h")
    main(sys.argv[1])
