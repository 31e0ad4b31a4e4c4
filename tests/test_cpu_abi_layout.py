"""The ctypes mirrors of the C ABI's structs (oidn-protoray_b200/prt_types.py) against
include/prt_cuda.h: a C program compiled with the host compiler prints sizeof and offsetof of
every field the mirror declares, and both must agree, so that a field added to one side only
(or reordered, or retyped) fails here rather than as a shifted read on the device."""
import ctypes as C
import pathlib
import shutil
import subprocess

import pytest

import prt_types as T

ROOT = pathlib.Path(__file__).resolve().parents[1]

MIRRORS = [("prt_mesh", T.Mesh), ("prt_material", T.Material), ("prt_texture", T.Texture),
           ("prt_env_desc", T.EnvDesc), ("prt_scene_desc", T.SceneDesc), ("prt_scene_stats", T.SceneStats),
           ("prt_camera_desc", T.CameraDesc), ("prt_renderer_desc", T.RendererDesc),
           ("prt_render_stats", T.RenderStats), ("prt_batch_item", T.BatchItem), ("prt_tuning", T.Tuning)]


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    d = tmp_path_factory.mktemp("abi")
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "prt_cuda.h"', "int main(void) {"]
    for cname, py in MIRRORS:
        lines.append(f'  printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for field, _ in py._fields_:
            lines.append(f'  printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["  return 0;", "}"]
    src = d / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = d / "layout"
    subprocess.run([cc, "-std=c99", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    layout = {}
    for line in out.splitlines():
        cname, key, value = line.split()
        layout[(cname, key)] = int(value)
    return layout


@pytest.mark.parametrize("cname,py", MIRRORS, ids=[m[0] for m in MIRRORS])
def test_mirror_matches_the_header(c_layout, cname, py):
    assert C.sizeof(py) == c_layout[(cname, "sizeof")], cname
    for field, _ in py._fields_:
        assert getattr(py, field).offset == c_layout[(cname, field)], (cname, field)
