"""The C++ wrapper include/rq_software_bvh.hpp, compiled and run the way a
reference call site uses it (tests/cpp/software_bvh_wrapper.cpp:
SoftwareBVH::build + SoftwareBVH4::fromBVH2 on a SceneMesh-shaped mesh,
common/software_bvh.hpp:35,193).  The CPU test compiles it; the GPU tests link
it against librq.so and check its bytes: the median split against the
reference's own trees (committed fixtures, and the live reference where
oracle/_ref is built), the default split against the ctypes binding, and the
empty mesh against the reference's result for it."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import pyoracle as O
import rq
from test_gpu_median import check, tie_free_soup

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "software_bvh_wrapper.cpp")
PKG = os.path.join(ROOT, "rdna2-accel-raster_b200")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
GOLD = os.path.join(ROOT, "tests", "golden", "ref_median_soups.npz")
CXX = shutil.which("g++")

needs_cxx = pytest.mark.skipif(CXX is None, reason="needs g++")


def compile_args():
    return [CXX, "-std=c++20", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), "-I",
            os.path.join(CUDA, "include")]


@needs_cxx
def test_wrapper_compiles(tmp_path):
    obj = tmp_path / "w.o"
    r = subprocess.run(compile_args() + ["-c", SRC, "-o", str(obj)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert obj.stat().st_size > 0


@pytest.fixture(scope="module")
def wrapper(tmp_path_factory):
    if CXX is None:
        pytest.skip("needs g++")
    exe = tmp_path_factory.mktemp("wrapper") / "software_bvh_wrapper"
    cmd = compile_args() + [SRC, "-o", str(exe), "-L", PKG, "-lrq", "-L", os.path.join(CUDA, "lib64"), "-lcudart",
                            f"-Wl,-rpath,{PKG}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return str(exe)


def run(exe, tmp_path, pos, idx, max_leaf, median, mode=None):
    """mode: 0 Morton, 1 median (from `median`), 2 the reference's call shape
    (no engine argument)."""
    mesh = tmp_path / "mesh.bin"
    with open(mesh, "wb") as f:
        np.array([len(pos), idx.size], np.uint32).tofile(f)
        np.ascontiguousarray(pos, np.float32).tofile(f)
        np.ascontiguousarray(idx, np.uint32).tofile(f)
    out = str(tmp_path / "out")
    mode = (1 if median else 0) if mode is None else mode
    r = subprocess.run([exe, str(mesh), out, str(max_leaf), str(mode)], capture_output=True, text=True, timeout=120)
    if r.returncode:
        return r.returncode, r.stderr
    rd = lambda ext, dt: np.fromfile(out + ext, dtype=dt)  # noqa: E731
    return 0, (rd(".nodes2", rq.BVH2_NODE), rd(".tris", rq.TRIANGLE), rd(".nodes4", rq.BVH4_NODE),
               rd(".perm", np.uint32))


@pytest.mark.gpu
def test_wrapper_median_equals_reference_fixtures(wrapper, tmp_path):
    g = np.load(GOLD)
    for key in sorted(k for k in g.files if k.startswith("pos_")):
        tag = key[4:]
        pos = g[key]
        rc, res = run(wrapper, tmp_path, pos, np.arange(len(pos), dtype=np.uint32), int(g[f"leaf_{tag}"]), True)
        assert rc == 0, res
        n2, tris, n4, _ = res
        check(n2, tris, n4, g[f"nodes2_{tag}"].view(rq.BVH2_NODE), g[f"tris_{tag}"].view(rq.TRIANGLE),
              g[f"nodes4_{tag}"].view(rq.BVH4_NODE))


@pytest.mark.gpu
@pytest.mark.skipif(not O.have_ref(), reason="needs oracle/_ref")
def test_wrapper_median_equals_reference_live(wrapper, tmp_path):
    pos = tie_free_soup(20000, 31)
    idx = np.arange(len(pos), dtype=np.uint32)[::-1].copy()  # indexed, triangles reversed
    rc, res = run(wrapper, tmp_path, pos, idx, 4, True)
    assert rc == 0, res
    check(*res[:3], *O.ref_build(pos, idx, 4))


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 2], ids=["engine_argument", "reference_call_shape"])
def test_wrapper_morton_equals_binding(ctx, wrapper, tmp_path, mode):
    # mode 2 calls SoftwareBVH::build(mesh, 4) / SoftwareBVH4::fromBVH2(bvh)
    # exactly as the reference's microbench_main.cpp:175,185 does
    import torch
    pos, idx = rq.scene_grid(96, 64, seed=5)
    rc, res = run(wrapper, tmp_path, pos, idx.reshape(-1), 4, False, mode)
    assert rc == 0, res
    b = rq.Bvh.build(ctx, torch.from_numpy(pos).cuda(), torch.from_numpy(idx.view(np.int32)).cuda())
    ctx.sync_check()
    n2, tris, n4, perm = b.download()
    b.destroy()
    assert res[0].tobytes() == n2.tobytes() and res[1].tobytes() == tris.tobytes()
    assert res[2].tobytes() == n4.tobytes() and np.array_equal(res[3], perm)


@pytest.mark.gpu
def test_wrapper_empty_mesh_like_reference(wrapper, tmp_path):
    # the reference's SoftwareBVH::build + fromBVH2 of an empty mesh: one leaf
    # of no triangles over the box (FLT_MAX, -FLT_MAX); 4-wide slot 0 holds it
    big = np.float32(np.finfo(np.float32).max)
    e2 = np.zeros(1, rq.BVH2_NODE)
    e2["aabb_min"], e2["aabb_max"], e2["left_child"], e2["right_child"] = big, -big, -1, 0
    e4 = np.zeros(1, rq.BVH4_NODE)
    for lo, hi in (("min_x", "max_x"), ("min_y", "max_y"), ("min_z", "max_z")):
        e4[lo][0, 0], e4[hi][0, 0] = big, -big
    e4["child_index"][0, 0] = -1
    if O.have_ref():
        r2, _, r4 = O.ref_build(np.zeros((0, 3), np.float32), np.zeros(0, np.uint32), 4)
        assert r2.tobytes() == e2.tobytes() and r4.tobytes() == e4.tobytes()
    for median in (False, True):
        rc, res = run(wrapper, tmp_path, np.zeros((0, 3), np.float32), np.zeros(0, np.uint32), 4, median)
        assert rc == 0, res
        assert res[0].tobytes() == e2.tobytes() and len(res[1]) == 0 and res[2].tobytes() == e4.tobytes()


@pytest.mark.gpu
def test_wrapper_reports_library_errors(wrapper, tmp_path):
    pos, idx = rq.scene_grid(8, 8, seed=1)
    rc, err = run(wrapper, tmp_path, pos, idx.reshape(-1), 17, False)  # max_leaf outside 1..16
    assert rc == 1 and "rq::Error" in err and "max_leaf" in err
