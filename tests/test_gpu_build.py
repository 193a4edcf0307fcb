"""GPU parity of the BVH build through the C ABI.

Bit-exact against Oracle B (the CPU LBVH restatement): Morton keys, sort
permutation, binary nodes, leaf-ordered triangles, 4-wide nodes.  The 4-wide
collapse is also checked byte-for-byte against the reference's own
SoftwareBVH4::fromBVH2 on the reference's own SoftwareBVH (imported)."""
import numpy as np
import pytest
import torch

import pyoracle as O
import rq
from conftest import soup

pytestmark = pytest.mark.gpu


def gpu_build(ctx, pos, idx, max_leaf=4):
    p = torch.from_numpy(np.ascontiguousarray(pos, np.float32)).cuda()
    i = torch.from_numpy(np.ascontiguousarray(idx, np.uint32).view(np.int32)).cuda() if idx is not None else None
    b = rq.Bvh.build(ctx, p, i, max_leaf=max_leaf)
    ctx.sync_check()
    return b


def assert_same_as_oracle(ctx, pos, idx, max_leaf=4):
    b = gpu_build(ctx, pos, idx, max_leaf)
    n2, tr, n4, perm = b.download()
    keys, ids = b.download_sort()
    o = O.lbvh_build(np.ascontiguousarray(pos, np.float32).reshape(-1), idx.reshape(-1) if idx is not None else None,
                     max_leaf)
    n = len(o["sorted"])
    assert np.array_equal(ids, o["sorted"]), "sort permutation"
    assert np.array_equal(perm, o["sorted"])
    assert np.array_equal(keys, o["codes"][o["sorted"]]), "Morton keys"
    assert len(n2) == len(o["nodes2"]) and n2.tobytes() == o["nodes2"].tobytes(), "binary nodes"
    assert tr.tobytes() == o["tris"].tobytes(), "leaf-ordered triangles"
    assert len(n4) == len(o["nodes4"]) and n4.tobytes() == o["nodes4"].tobytes(), "4-wide nodes"
    assert b.info()["depth4"] == o["depth4"]
    b.destroy()
    return n


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 7, 16, 17, 33, 100, 1000, 4097])
def test_soup_parity_small(ctx, n):
    assert_same_as_oracle(ctx, soup(n, 100 + n), None)


@pytest.mark.parametrize("max_leaf", [1, 2, 4, 8, 16])
def test_max_leaf_parity(ctx, max_leaf):
    assert_same_as_oracle(ctx, soup(3000, 5), None, max_leaf)


def test_grid_parity_plain_config(ctx):
    # the plain workload's mesh: 64x32 quads, 4,096 triangles, seed 0
    pos, idx = rq.scene_grid(64, 32, seed=0)
    assert assert_same_as_oracle(ctx, pos, idx) == 4096


def test_duplicate_codes_parity(ctx):
    # many identical centroids -> equal Morton codes, split by sorted index
    v = np.tile(soup(1, 9), (700, 1)).astype(np.float32)
    v[::3] += np.float32(1e-3) * (np.arange(700)[:, None] % 3)
    assert_same_as_oracle(ctx, v, None)


def test_large_soup_parity(ctx):
    assert_same_as_oracle(ctx, soup(300000, 11), None)


@pytest.mark.parametrize("n", [255, 256, 257, 511, 512, 513, 1023, 1025, 2049, 65537])
def test_block_boundary_sizes_parity(ctx, n):
    # sizes around the refit kernel's 256-leaf blocks and the collapse's
    # one-block top levels
    assert_same_as_oracle(ctx, soup(n, 700 + n), None)


def test_repeated_in_place_rebuilds_parity(ctx):
    # one handle rebuilt in place over changing inputs (larger, smaller, larger
    # again): every build equals the oracle's, so no scratch state of an
    # earlier build leaks into a later one
    b = None
    for k, n in enumerate((20000, 513, 70000, 4097, 70000)):
        pos = soup(n, 900 + k)
        p = torch.from_numpy(pos).cuda()
        b = rq.Bvh.build(ctx, p, None, into=b) if b is not None else rq.Bvh.build(ctx, p, None)
        ctx.sync_check()
        n2, tr, n4, perm = b.download()
        o = O.lbvh_build(pos.reshape(-1), None, 4)
        assert n2.tobytes() == o["nodes2"].tobytes() and n4.tobytes() == o["nodes4"].tobytes(), n
        assert tr.tobytes() == o["tris"].tobytes() and np.array_equal(perm, o["sorted"]), n
    b.destroy()


def test_reference_terrain_parity(ctx):
    d = np.load(__file__.replace("test_gpu_build.py", "golden/ref_terrain1000.npz"))
    assert_same_as_oracle(ctx, d["pos"], d["idx"])


def test_collapse_matches_reference_bytes(ctx):
    # SoftwareBVH from the reference (fixture) -> import -> GPU collapse ->
    # identical bytes to the reference's SoftwareBVH4::fromBVH2.
    d = np.load(__file__.replace("test_gpu_build.py", "golden/ref_terrain1000.npz"))
    n2 = torch.from_numpy(d["nodes2"].view(np.int32).copy()).cuda()
    tr = torch.from_numpy(d["tris"].view(np.int32).copy()).cuda()
    b = rq.Bvh.import2(ctx, n2, tr)
    b.collapse4()
    ctx.sync_check()
    _, _, n4, _ = b.download()
    assert n4.tobytes() == d["nodes4"].tobytes()
    b.destroy()


@pytest.mark.skipif(not O.have_ref(), reason="needs oracle/_ref")
@pytest.mark.parametrize("target", [64, 4096, 100000, 1000000])
def test_collapse_matches_reference_bytes_live(ctx, target):
    pos, idx = O.ref_terrain(target)
    n2r, trr, n4r = O.ref_build(pos, idx)
    b = rq.Bvh.import2(ctx, torch.from_numpy(n2r.view(np.int32).copy()).cuda(),
                       torch.from_numpy(trr.view(np.int32).copy()).cuda())
    b.collapse4()
    ctx.sync_check()
    _, _, n4, _ = b.download()
    assert n4.tobytes() == n4r.tobytes()
    b.destroy()


def test_rebuild_in_place_and_refit(ctx):
    pos, idx = rq.scene_grid(64, 32, seed=0)
    p = torch.from_numpy(pos).cuda()
    i = torch.from_numpy(idx.view(np.int32)).cuda()
    b = rq.Bvh.build(ctx, p, i)
    n4_before = b.download()[2]
    # deform, then refit: topology kept, boxes and triangles follow the vertices
    q = torch.empty_like(p)
    rq.deform_wave(ctx, p, q, 0.7, 0.05, 1.0)
    b.refit(q, i)
    ctx.sync_check()
    n2, tr, n4, perm = b.download()
    qh = q.cpu().numpy()
    tri = qh[idx[perm]]
    assert np.array_equal(tr["v0"][:, :3], tri[:, 0]) and np.array_equal(tr["v2"][:, :3], tri[:, 2])
    # every binary node box is the union of its leaves' triangle boxes
    lo = tri.min(1)
    hi = tri.max(1)
    for k in range(len(n2)):
        nd = n2[k]
        if nd["left_child"] < 0:
            f, c = ~int(nd["left_child"]), int(nd["right_child"])
            assert np.array_equal(nd["aabb_min"], lo[f:f + c].min(0))
            assert np.array_equal(nd["aabb_max"], hi[f:f + c].max(0))
        else:
            l, r = n2[nd["left_child"]], n2[nd["right_child"]]
            assert np.array_equal(nd["aabb_min"], np.minimum(l["aabb_min"], r["aabb_min"]))
            assert np.array_equal(nd["aabb_max"], np.maximum(l["aabb_max"], r["aabb_max"]))
    # the 4-wide tree keeps its topology and every slot box is the union of
    # what lies below it in the refitted geometry
    assert np.array_equal(n4["child_index"], n4_before["child_index"])
    assert np.array_equal(n4["child_count"], n4_before["child_count"])

    def box4(i):
        mn, mx = np.full(3, np.inf, np.float32), np.full(3, -np.inf, np.float32)
        nd = n4[i]
        for k in range(4):
            cc, ci = int(nd["child_count"][k]), int(nd["child_index"][k])
            if cc == 0:
                continue
            if cc < 0:
                cmn, cmx = box4(ci)
            else:
                cmn, cmx = lo[~ci:~ci + cc].min(0), hi[~ci:~ci + cc].max(0)
            got_mn = np.array([nd["min_x"][k], nd["min_y"][k], nd["min_z"][k]])
            got_mx = np.array([nd["max_x"][k], nd["max_y"][k], nd["max_z"][k]])
            assert np.array_equal(got_mn, cmn) and np.array_equal(got_mx, cmx)
            mn, mx = np.minimum(mn, cmn), np.maximum(mx, cmx)
        return mn, mx

    box4(0)
    # a rebuild in place on the deformed mesh equals a fresh build
    rq.Bvh.build(ctx, q, i, into=b)
    ctx.sync_check()
    o = O.lbvh_build(qh.reshape(-1), idx.reshape(-1))
    n2b, _, n4b, _ = b.download()
    assert n2b.tobytes() == o["nodes2"].tobytes() and n4b.tobytes() == o["nodes4"].tobytes()
    b.destroy()


def test_deform_matches_oracle_sin(ctx):
    pos, _ = rq.scene_grid(64, 32, seed=0)
    p = torch.from_numpy(pos).cuda()
    q = torch.empty_like(p)
    rq.deform_wave(ctx, p, q, 1.3, 0.05, 1.0)
    got = q.cpu().numpy()
    arg = (np.float32(1.3) + np.float32(1.0) * pos[:, 0]).astype(np.float32)
    s = np.array([O.sincos(float(a))[0] for a in arg], np.float32)
    want = (pos[:, 2] + np.float32(0.05) * s).astype(np.float32)
    assert np.array_equal(got[:, 2], want) and np.array_equal(got[:, :2], pos[:, :2])


def test_deform_step_advances_device_time(ctx):
    pos, _ = rq.scene_grid(100, 100, seed=2)
    p = torch.from_numpy(pos).cuda()
    q = torch.empty_like(p)
    want = torch.empty_like(p)
    state = torch.zeros(2, dtype=torch.int32, device="cuda")
    state[0] = int(np.float32(0.3).view(np.int32))
    for k in range(3):
        rq.deform_wave_step(ctx, p, q, state, 0.1)
        t = np.float32(0.3)
        for _ in range(k):
            t = np.float32(t + np.float32(0.1))
        rq.deform_wave(ctx, p, want, float(t), 0.05, 1.0)
        assert torch.equal(q, want), k
    assert int(state[1].item()) == 0


def test_bad_arguments_fail_loudly(ctx):
    p = torch.zeros(9, dtype=torch.float32, device="cuda")
    with pytest.raises(rq.RqError) as e:
        rq.Bvh.build(ctx, p, None, max_leaf=0)
    assert e.value.status == rq.RQ_ERR_INVALID_ARG
    with pytest.raises(rq.RqError):
        rq.Bvh.build(ctx, p, None, max_leaf=17)
