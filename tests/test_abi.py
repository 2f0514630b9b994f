"""The C ABI library: it loads, exports every function include/psy_b200.h
declares, and reports errors through return codes (no GPU needed)."""
import ctypes as C
import os
import re

import pytest

from psychopath_cpp_b200 import _abi

HEADER = os.path.join(os.path.dirname(os.path.dirname(__file__)), "include", "psy_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(psy_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_expected_surface():
    fns = declared_functions()
    for f in ("psy_trace", "psy_scene_upload", "psy_render", "psy_light_sample"):
        assert f in fns
    assert set(_abi.EXPORTED) <= set(fns)


def test_library_exports_every_declared_symbol():
    L = _abi.load()
    missing = [f for f in declared_functions() if not hasattr(L, f)]
    assert not missing, missing


def test_version_and_null_arguments():
    L = _abi.load()
    assert L.psy_version().startswith(b"psy_b200")
    assert L.psy_ctx_create(0, None) == _abi.PSY_ERR_ARG
    assert L.psy_last_error(None) == b"no context"
    assert L.psy_scene_upload(None, None) == _abi.PSY_ERR_ARG
    assert L.psy_trace(None, None, 0, None, None) == _abi.PSY_ERR_ARG
    assert L.psy_sync(None, None) == _abi.PSY_ERR_ARG


def test_context_creation_without_a_device_fails_cleanly():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a CUDA device is present")
    except ImportError:
        pass
    L = _abi.load()
    h = C.c_void_p()
    assert L.psy_ctx_create(0, C.byref(h)) == _abi.PSY_ERR_DEVICE
    assert not h.value


# ctypes mirror -> the header's struct it mirrors
_MIRRORS = {
    "ObjectDesc": "psy_object_desc", "InstanceDesc": "psy_instance_desc", "AssemblyDesc": "psy_assembly_desc",
    "ShaderDesc": "psy_shader_desc", "SceneDesc": "psy_scene_desc", "SceneStats": "psy_scene_stats",
    "RaySoA": "psy_ray_soa", "HitSoA": "psy_hit_soa", "LightQuerySoA": "psy_light_query_soa",
    "LightSampleSoA": "psy_light_sample_soa", "RenderDesc": "psy_render_desc", "DiffDesc": "psy_diff_desc",
    "BatchDesc": "psy_batch_desc", "BatchTuning": "psy_batch_tuning", "RenderStats": "psy_render_stats",
    "TraceCounters": "psy_trace_counters", "RenderSettings": "psy_render_settings",
}


def test_ctypes_mirrors_match_the_header_layout(tmp_path):
    """Every ctypes structure has the size and field offsets that a C
    compiler gives the header's struct of the same field names."""
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "psy_b200.h"', "int main(void) {"]
    expect = []
    for py, cn in _MIRRORS.items():
        cls = getattr(_abi, py)
        lines.append('printf("%%zu\\n", sizeof(%s));' % cn)
        expect.append(C.sizeof(cls))
        for f in cls._fields_:
            lines.append('printf("%%zu\\n", offsetof(%s, %s));' % (cn, f[0]))
            expect.append(getattr(cls, f[0]).offset)
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    assert got == expect


C_CONSUMER = r"""
#include <stdio.h>
#include <stdlib.h>
#include "psy_b200.h"
int main(int argc, char** argv) {
    FILE* fp = fopen(argv[1], "rb");
    if (!fp) return 2;
    fseek(fp, 0, SEEK_END);
    long n = ftell(fp);
    fseek(fp, 0, SEEK_SET);
    char* text = (char*)malloc((size_t)n);
    if (fread(text, 1, (size_t)n, fp) != (size_t)n) return 3;
    fclose(fp);
    psy_file_scene* f = NULL;
    char err[256];
    if (psy_file_parse(text, (size_t)n, 0, &f, err, sizeof err) != PSY_OK) { printf("error %s\n", err); return 4; }
    const psy_scene_desc* d = psy_file_scene_desc(f);
    psy_render_settings rs;
    psy_file_render_settings(f, &rs);
    uint64_t nodes = 0;
    if (psy_build_bvh4(d, 0, &nodes, NULL, NULL, NULL, NULL) != PSY_OK) return 5;
    printf("%u %u %u %u %u %u %llu\n", rs.width, rs.height, rs.spp, d->assembly_count,
           d->assemblies[0].instance_count, d->shader_count, (unsigned long long)nodes);
    psy_file_free(f);
    free(text);
    return 0;
}
"""


def test_c_program_reads_a_scene_file(tmp_path):
    """The C ABI from plain C (no Python in between): a program compiled by
    gcc against include/psy_b200.h and linked to the library reads a .psy
    file and builds its root BVH4 on the host, with the Python path's
    counts."""
    import shutil
    import subprocess
    from psychopath_cpp_b200 import api, scenes
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    L = _abi.load()
    lib = L._name
    sc = scenes.many_light_scene(2, res=(32, 18), spp=2, n_patches=12, n_groups=10, n_lights=20)
    path = tmp_path / "s.psy"
    sc.write_psy(str(path))
    src = tmp_path / "consumer.c"
    src.write_text(C_CONSUMER)
    exe = tmp_path / "consumer"
    libdir = os.path.dirname(lib)
    subprocess.run(["gcc", "-std=c99", "-I", os.path.dirname(HEADER), str(src), "-o", str(exe), lib,
                    "-Wl,-rpath," + libdir], check=True)
    out = subprocess.run([str(exe), str(path)], check=True, capture_output=True, text=True).stdout.split()
    d, keep = api.flatten(sc)
    nodes = api.build_bvh4_records(sc, 0)["ts"].shape[0]
    assert [int(x) for x in out] == [sc.res_x, sc.res_y, sc.spp, d.assembly_count, d.assemblies[0].instance_count,
                                     d.shader_count, nodes]
