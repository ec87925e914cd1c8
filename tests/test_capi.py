"""The C ABI library: it loads without a GPU, exports every function include/mrt_cuda.h declares,
and the ctypes mirror has the C struct layout (checked against the compiler).  CPU only."""
import ctypes
import os
import re
import subprocess

import pytest

from mobileraytracer_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "mrt_cuda.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mrt_\w+)\s*\(", src)))


def test_library_loads_and_exports_every_declared_symbol():
    lib = capi.load()
    names = declared_functions()
    assert len(names) >= 16
    for n in names:
        assert hasattr(lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", capi.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (mrt_\w+)", out))
    assert set(names) <= exported
    assert set(capi.EXPORTED_SYMBOLS) <= exported


STRUCTS = ["MrtMaterial", "MrtLightDesc", "MrtSceneDesc", "MrtAccelOpts", "MrtRay", "MrtHit", "MrtCamera",
           "MrtRenderOpts", "MrtRenderStats", "MrtBatchOpts", "MrtBatchJob", "MrtBatchStats", "MrtServeOpts",
           "MrtServeStats"]


def test_struct_layouts_match_the_header(tmp_path):
    prog = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{HEADER}"', "int main(void){"]
    for s in STRUCTS:
        prog.append(f'printf("{s} %zu\\n", sizeof({s}));')
        for fname, _ in getattr(capi, s)._fields_:
            prog.append(f'printf("{s}.{fname} %zu\\n", offsetof({s}, {fname}));')
    prog.append("return 0;}")
    c = tmp_path / "layout.c"
    c.write_text("\n".join(prog))
    exe = tmp_path / "layout"
    subprocess.run(["/usr/bin/gcc", "-o", str(exe), str(c)], check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True).stdout.splitlines())
    for s in STRUCTS:
        t = getattr(capi, s)
        assert int(got[s]) == ctypes.sizeof(t), s
        for fname, _ in t._fields_:
            assert int(got[f"{s}.{fname}"]) == getattr(t, fname).offset, f"{s}.{fname}"


def test_context_without_gpu_fails_loudly():
    """No GPU: creating a context reports an error status instead of computing on the CPU."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import mobileraytracer_b200 as m
    with pytest.raises(m.MrtError):
        m.Context(0)


def test_hit_id_encoding():
    assert capi.hit_id(capi.MRT_PRIM_TRIANGLE, 5) == (2 << 30) | 5
    assert capi.hit_id(capi.MRT_PRIM_PLANE, 0) == 0
    assert capi.MRT_HIT_NONE >> 30 == 3


def test_render_flag_constants_match_the_header():
    src = open(HEADER).read()
    m = re.search(r"#define MRT_RENDER_SHADE_QUEUES (\d+)u", src)
    assert m and int(m.group(1)) == capi.MRT_RENDER_SHADE_QUEUES
