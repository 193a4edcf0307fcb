"""CPU tests of the C ABI: librq.so loads (no GPU needed to load it) and
exports every entry point include/*.h declares; host-only entry points
(layout planner, scene generators) work without a device."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import rq

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(inc, fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s*(rq_[a-z0-9_]+)\s*\(", text, re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    assert "rq_build" in names and "rq_trace" in names and "rq_build_radv" in names
    assert len(names) >= 25


def test_library_exports_every_declared_symbol():
    lib = rq.lib()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_mirror_binds_every_symbol():
    bound = {name for name, _, _ in rq.SIGNATURES}
    assert set(declared_functions()) <= bound


def test_no_device_is_reported_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("device present")
    h = C.c_void_p()
    assert rq.lib().rq_ctx_create(0, C.byref(h)) == rq.RQ_ERR_NO_DEVICE


def test_radv_layout_matches_reference_goldens():
    import json
    g = json.load(open(os.path.join(ROOT, "tests", "golden", "radv_layouts.json")))
    for n, want in g.items():
        got = rq.radv_layout(int(n))
        assert got["total_boxes"] == want["total_boxes"]
        assert got["num_levels"] == want["num_levels"]
        assert got["counts"] == want["counts"] and got["offsets"] == want["offsets"]
        assert got["total_size"] == want["total_size"]


def test_scene_grid_shapes_and_determinism():
    pos, idx = rq.scene_grid(64, 32, seed=0)
    assert pos.shape == (65 * 33, 3) and idx.shape == (4096, 3)
    pos2, idx2 = rq.scene_grid(64, 32, seed=0)
    assert np.array_equal(pos, pos2) and np.array_equal(idx, idx2)
    pos3, _ = rq.scene_grid(64, 32, seed=1)
    assert not np.array_equal(pos, pos3)
    # winding of generate_dynamic_grid_mesh: (v00, v10, v01), (v10, v11, v01)
    assert idx[0].tolist() == [0, 1, 65] and idx[1].tolist() == [1, 66, 65]
    # jitter sigma 0.01 around the height field
    x, y, z = pos[:, 0], pos[:, 1], pos[:, 2]
    resid = z - 0.2 * np.sin(3 * x) * np.cos(3 * y)
    assert 0.008 < resid.std() < 0.012


def test_scene_rays_down():
    r = rq.scene_rays_down(1000, seed=0)
    assert r.shape == (1000, 8)
    assert np.allclose(np.linalg.norm(r[:, 4:7], axis=1), 1.0, atol=1e-6)
    assert np.all(r[:, 2] == 2.0) and np.all(r[:, 6] < 0)


def test_status_strings_cover_every_status():
    names = {rq.RQ_OK: "ok", rq.RQ_ERR_BUDGET: "memory budget exceeded", rq.RQ_ERR_CANCELLED: "request cancelled"}
    for code, text in names.items():
        assert rq.lib().rq_status_string(code).decode() == text
    assert rq.lib().rq_status_string(11).decode() == "unknown status"


def test_server_refuses_bad_configs_without_a_device():
    # configuration checks run before any device call
    bad = [dict(mode=7), dict(max_leaf=0), dict(slots=0), dict(slots=9), dict(max_wave_requests=2000),
           dict(rebuild=True)]
    for kw in bad:
        with pytest.raises(rq.ServeError) as e:
            rq.Server(**kw)
        assert e.value.status == rq.RQ_ERR_INVALID_ARG, kw


def test_server_mesh_bytes_is_host_only():
    b = rq.Server.mesh_bytes(1000, 2000)
    assert b >= 12 * 1000 + 12 * 2000 + 2000 * (64 + 48 + 8 + 128)


def test_noalloc_radv_checks_arguments_before_any_device_call():
    # misaligned or missing buffers and oversized counts are refused on the
    # host: these pointers are never dereferenced and no CUDA call is made
    L = rq.lib()
    f = L.rq_build_radv_noalloc
    big = C.c_uint64(1 << 40)
    assert f(C.c_void_p(0x1002), 1, C.c_void_p(0x10000), big, None) == rq.RQ_ERR_INVALID_ARG
    assert f(C.c_void_p(0x1000), 1, C.c_void_p(0x10008), big, None) == rq.RQ_ERR_INVALID_ARG
    assert f(None, 1, C.c_void_p(0x10000), big, None) == rq.RQ_ERR_INVALID_ARG
    assert f(C.c_void_p(0x1000), 0, C.c_void_p(0x10000), big, None) == rq.RQ_ERR_INVALID_ARG
    assert f(C.c_void_p(0x1000), rq.RADV_NOALLOC_MAX_TRIANGLES + 1, C.c_void_p(0x10000), big,
             None) == rq.RQ_ERR_UNSUPPORTED
    assert f(C.c_void_p(0x1000), 5, C.c_void_p(0x10000), C.c_uint64(100), None) == rq.RQ_ERR_SIZE
