"""CPU tests of the oracle's frame pieces and workload generators (no GPU):

  - the oracle's copy of the workload generators (height-field grid, look-at
    camera, the 1080p frame's lights and shading parameters) gives the same
    bytes as the engine's host generators, so a process that builds the
    frame from the oracle alone (the benchmark's reference arm) traces the
    same frame;
  - the rays the oracle emits (camera, shadow/AO, reflection, depth AO)
    reproduce its own frame results when traced one by one;
  - refit and permutation recovery are consistent with Oracle B."""
import ctypes as C

import numpy as np
import pytest

import pyoracle as O
import rq
from rq import workloads as W


def cam_bytes(cam):
    return C.string_at(C.addressof(cam), C.sizeof(cam))


@pytest.mark.parametrize("q", [(1, 1), (64, 32), (300, 200)])
def test_oracle_scene_grid_matches_engine_generator(q):
    a = O.scene_grid(*q, seed=7)
    b = rq.scene_grid(*q, seed=7)
    assert a[0].tobytes() == b[0].tobytes() and a[1].tobytes() == b[1].tobytes()


def test_shadow_frame_inputs_match_the_engine_workload():
    pos, idx, cam, params = O.shadow_frame_inputs()
    p2, i2 = W.shadow_mesh()
    assert pos.tobytes() == p2.tobytes() and idx.tobytes() == i2.tobytes()
    assert len(idx) == 2499848
    assert cam_bytes(cam) == cam_bytes(W.shadow_camera())
    assert cam_bytes(params) == cam_bytes(W.shadow_params())


def test_camera_look_at_matches_engine():
    for eye, fov, w, h in (((0.0, 0.0, 3.0), 19.5, 1920, 1080), ((1.0, -2.0, 1.5), 45.0, 320, 240)):
        a = O.camera_look_at(eye, (0.0, 0.0, 0.0), (0.0, 1.0, 0.0) if eye[0] == 0 else (0.0, 0.0, 1.0), fov, w, h,
                             jitter=True, seed=3)
        b = rq.camera_look_at(eye, (0.0, 0.0, 0.0), (0.0, 1.0, 0.0) if eye[0] == 0 else (0.0, 0.0, 1.0), fov, w, h,
                              jitter=True, seed=3)
        assert cam_bytes(a) == cam_bytes(b)


@pytest.fixture(scope="module")
def small_frame():
    pos, idx = O.scene_grid(96, 96, seed=1)
    o = O.lbvh_build(pos.reshape(-1), idx.reshape(-1))
    w, h = 160, 90
    cam = O.camera_look_at(O.SHADOW_EYE, O.SHADOW_TARGET, O.SHADOW_UP, O.SHADOW_FOVY, w, h)
    g = O.render_gbuffer(o["nodes4"], o["tris"], o["sorted"], cam)
    return pos, idx, o, cam, g, w, h


def test_emitted_camera_rays_reproduce_gbuffer(small_frame):
    pos, idx, o, cam, g, w, h = small_frame
    rays = O.camera_rays(cam)
    hits, _, _ = O.trace_bvh4(o["nodes4"], o["tris"], o["sorted"], rays, 0)
    assert np.array_equal(hits["hit"], (g["vis"] > 0).astype(np.uint32))
    assert np.array_equal(np.where(hits["hit"] == 1, hits["primitive_id"] + 1, 0), g["vis"])
    assert hits["t"].tobytes() == g["t"].tobytes()


def test_emitted_shade_rays_reproduce_mask_and_ao(small_frame):
    pos, idx, o, cam, g, w, h = small_frame
    params = O.shade_params(w, h, O.shadow_lights(16), ao_spp=3, ao_tmax=0.5)
    mask, ao, nrays = O.render_shadow_ao(o["nodes4"], o["tris"], g, params)
    px = np.arange(w * h, dtype=np.uint32)
    rays, rpx, slot = O.shade_rays(g, params, px)
    assert len(rays) == nrays
    hits, _, _ = O.trace_bvh4(o["nodes4"], o["tris"], o["sorted"], rays, 1)
    m2 = np.zeros(w * h, np.uint32)
    un = np.zeros(w * h, np.float32)
    lit = hits["hit"] == 0
    light = slot < 32
    np.bitwise_or.at(m2, rpx[light & lit], (np.uint32(1) << slot[light & lit]).astype(np.uint32))
    np.add.at(un, rpx[~light & lit], np.float32(1.0))
    assert np.array_equal(m2, mask)
    want_ao = np.where(g["vis"] > 0, un / np.float32(3.0), np.float32(1.0)).astype(np.float32)
    assert want_ao.tobytes() == ao.tobytes()


def test_reflection_rays_reproduce_hits(small_frame):
    pos, idx, o, cam, g, w, h = small_frame
    rp = O.reflect_params(cam)
    hits, rays = O.render_reflect(o["nodes4"], o["tris"], o["sorted"], g, rp, want_rays=True)
    vis = g["vis"] > 0
    h2, _, _ = O.trace_bvh4(o["nodes4"], o["tris"], o["sorted"], rays[vis], 0)
    assert h2.tobytes() == hits[vis].tobytes()
    assert (hits["hit"][~vis] == 0).all()
    # rays leave the surface on the camera's side, at unit length
    d = rays["dir"][vis].astype(np.float64)
    assert np.allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-5)
    nrm = g["nrm"][vis].astype(np.float64)
    assert (np.einsum("ij,ij->i", d, nrm) >= -1e-6).all()
    assert 0.0 < hits["hit"][vis].mean() < 1.0


def test_depth_ao_rays_reproduce_ao(small_frame):
    pos, idx, o, cam, g, w, h = small_frame
    vp = rq.view_proj_of(cam)
    depth = O.gbuffer_depth(g, vp)
    for spp in (0, 1, 4):
        ap = O.ao_depth_params(cam, spp=spp, max_distance=0.5)
        ao, nrays = O.render_ao_depth(o["nodes4"], o["tris"], depth, ap)
        rays, rpx = O.ao_depth_rays(depth, ap, np.arange(w * h, dtype=np.uint32))
        assert len(rays) == nrays == int((depth < 1.0).sum()) * max(1, spp)
        hits, _, _ = O.trace_bvh4(o["nodes4"], o["tris"], o["sorted"], rays, 1)
        un = np.zeros(w * h, np.float32)
        np.add.at(un, rpx[hits["hit"] == 0], np.float32(1.0))
        want = np.where(depth < 1.0, un / np.float32(max(1, spp)), np.float32(1.0)).astype(np.float32)
        assert want.tobytes() == ao.tobytes(), spp
    # the reconstructed surface agrees with the G-buffer's to the depth
    # buffer's precision, and the normal faces the camera
    ap = O.ao_depth_params(cam, spp=1)
    rays, rpx = O.ao_depth_rays(depth, ap, np.arange(w * h, dtype=np.uint32))
    org = rays["org"].astype(np.float64)
    gp = g["pos"][rpx].astype(np.float64)
    gn = g["nrm"][rpx].astype(np.float64)
    surf = org - 0.03 * ((org - gp) / np.linalg.norm(org - gp, axis=1, keepdims=True))
    assert np.median(np.linalg.norm(surf - gp, axis=1)) < 1e-3
    # AO from depth needs no G-buffer: background depth gives AO 1
    d1 = np.ones_like(depth)
    ao1, n1 = O.render_ao_depth(o["nodes4"], o["tris"], d1, ap)
    assert n1 == 0 and (ao1 == 1.0).all()


def test_refit_of_unmoved_mesh_is_the_build():
    pos, idx = O.scene_grid(50, 40, seed=5)
    o = O.lbvh_build(pos.reshape(-1), idx.reshape(-1))
    tris, n2, n4 = O.refit(pos, idx, o["sorted"], o["nodes2"], o["nodes4"])
    assert tris.tobytes() == o["tris"].tobytes()
    assert n2.tobytes() == o["nodes2"].tobytes() and n4.tobytes() == o["nodes4"].tobytes()


def test_refit_of_moved_mesh_bounds_its_leaves():
    pos, idx = O.scene_grid(40, 40, seed=6)
    o = O.lbvh_build(pos.reshape(-1), idx.reshape(-1))
    moved = pos.copy()
    moved[:, 2] += np.float32(0.3) * np.sin(moved[:, 0] * 4).astype(np.float32)
    tris, n2, n4 = O.refit(moved, idx, o["sorted"], o["nodes2"], o["nodes4"])
    assert np.array_equal(n2["left_child"], o["nodes2"]["left_child"])
    v = np.stack([tris["v0"][:, :3], tris["v1"][:, :3], tris["v2"][:, :3]], 1)
    root = n2[0]
    assert np.array_equal(root["aabb_min"], v.min((0, 1))) and np.array_equal(root["aabb_max"], v.max((0, 1)))
    assert not np.array_equal(n2["aabb_max"], o["nodes2"]["aabb_max"])


def test_recover_perm_inverts_the_leaf_order():
    pos, idx = O.scene_grid(60, 30, seed=2)
    o = O.lbvh_build(pos.reshape(-1), idx.reshape(-1))
    assert np.array_equal(O.recover_perm(o["tris"], pos, idx), o["sorted"])
    dup = np.concatenate([idx, idx[:1]])
    with pytest.raises(AssertionError):
        O.recover_perm(o["tris"], pos, dup)


@pytest.mark.parametrize("n,max_leaf", [(1, 4), (7, 4), (1500, 4), (5000, 2), (3000, 8)])
def test_oracle_sah_subtree_build_invariants(n, max_leaf):
    # the LBVH with SAH-rebuilt subtrees: a permutation of the triangles in
    # leaf order, every node's range contiguous and its box the union of its
    # leaves, leaves of at most max_leaf, Morton keys and sort as the LBVH's
    from conftest import soup
    v = soup(n, 900 + n).reshape(-1)
    o = O.lbvh_sah_build(v, None, max_leaf, 1024)
    ol = O.lbvh_build(v, None, max_leaf)
    assert np.array_equal(o["codes"], ol["codes"]) and np.array_equal(o["sorted"], ol["sorted"])
    assert np.array_equal(np.sort(o["perm"]), np.arange(n, dtype=np.uint32))
    tri = v.reshape(-1, 3, 3)[o["perm"]]
    assert np.array_equal(o["tris"]["v0"][:, :3], tri[:, 0])
    lo, hi = tri.min(1), tri.max(1)
    n2 = o["nodes2"]

    def walk(k):
        nd = n2[k]
        if nd["left_child"] < 0:
            f, c = ~int(nd["left_child"]), int(nd["right_child"])
            assert 1 <= c <= max_leaf
            rng = (f, f + c)
        else:
            a, b = walk(int(nd["left_child"])), walk(int(nd["right_child"]))
            assert a[1] == b[0] and int(nd["left_child"]) == k + 1
            rng = (a[0], b[1])
        assert np.array_equal(nd["aabb_min"], lo[rng[0]:rng[1]].min(0))
        assert np.array_equal(nd["aabb_max"], hi[rng[0]:rng[1]].max(0))
        return rng

    assert walk(0) == (0, n)


def test_oracle_sah_subtrees_need_fewer_node_visits():
    pos, idx = O.scene_grid(300, 300, seed=1)
    o = O.lbvh_sah_build(pos.reshape(-1), idx.reshape(-1), 4, 1024)
    ol = O.lbvh_build(pos.reshape(-1), idx.reshape(-1))
    w, h = 160, 90
    cam = O.camera_look_at(O.SHADOW_EYE, O.SHADOW_TARGET, O.SHADOW_UP, O.SHADOW_FOVY, w, h)
    g = O.render_gbuffer(ol["nodes4"], ol["tris"], ol["sorted"], cam)
    params = O.shade_params(w, h, O.shadow_lights(16), ao_spp=1, ao_tmax=0.5)
    rays, _, _ = O.shade_rays(g, params, np.arange(w * h, dtype=np.uint32))
    hs, _, ss = O.trace_bvh4(o["nodes4"], o["tris"], o["perm"], rays, 1, want_stats=True)
    hl, _, sl = O.trace_bvh4(ol["nodes4"], ol["tris"], ol["sorted"], rays, 1, want_stats=True)
    assert np.array_equal(hs["hit"], hl["hit"])  # any-hit results do not depend on the tree
    assert ss["box_tests"].mean() < 0.95 * sl["box_tests"].mean()
