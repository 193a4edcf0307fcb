"""CPU test of the public structs' layouts: the ctypes mirrors in rq/__init__.py
against the C headers.  A C program built from include/*.h prints every
struct's size and each mirrored field's offset; both must equal ctypes'.  A
field added to a header struct without its mirror (or the reverse) changes
the size, so a caller of the Python API would otherwise read past the struct."""
import ctypes as C
import os
import shutil
import subprocess

import pytest

import rq

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# C struct -> its mirror class in rq
MIRRORS = {
    "rq_trace_tuning": "TraceTuning",
    "rq_camera_tuning": "CameraTuning",
    "rq_bvh_info": "BvhInfo",
    "rq_mesh_desc": "MeshDesc",
    "rq_instance": "Instance",
    "rq_batch_tuning": "BatchTuning",
    "rq_camera": "Camera",
    "rq_light": "Light",
    "rq_shade_params": "ShadeParams",
    "rq_reflect_params": "ReflectParams",
    "rq_ao_depth_params": "AoDepthParams",
    "rq_radv_check": "RadvCheck",
    "rq_radv_layout": "RadvLayout",
    "rq_server_config": "ServerConfig",
    "rq_request": "Request",
    "rq_completion": "Completion",
    "rq_server_stats": "ServerStats",
}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_ctypes_mirrors_match_the_headers(tmp_path):
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "rq.h"', '#include "rq_serve.h"',
             '#include "rq_layouts.h"', "int main(void) {"]
    for cname, pyname in MIRRORS.items():
        cls = getattr(rq, pyname)
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for field, _ in cls._fields_:
            lines.append(f'printf("{cname}.{field} %zu\\n", offsetof({cname}, {field}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    exe = tmp_path / "layout"
    src.write_text("\n".join(lines))
    r = subprocess.run(["gcc", "-std=c11", "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = dict(line.split() for line in out if line)
    for cname, pyname in MIRRORS.items():
        cls = getattr(rq, pyname)
        assert int(got[cname]) == C.sizeof(cls), (cname, int(got[cname]), C.sizeof(cls))
        for field, _ in cls._fields_:
            assert int(got[f"{cname}.{field}"]) == getattr(cls, field).offset, (cname, field)
