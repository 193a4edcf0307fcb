"""GPU parity of the median-split build (rq_build with RQ_BUILD_MEDIAN)
against the reference's own SoftwareBVH::build (common/software_bvh.hpp,
compiled from its sources into oracle/_ref) on inputs whose centroid values
never repeat on an axis (then nth_element's left and right sets are unique):
binary nodes byte for byte, each leaf's triangles as a set, and the 4-wide
collapse byte for byte against the reference's fromBVH2.  Committed fixtures
(tests/golden/ref_median_soups.npz, the reference's output) stand in where
the reference library is not built."""
import os

import numpy as np
import pytest
import torch

import pyoracle as O
import rq
from conftest import soup

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_median_soups.npz")


def tie_free_soup(n, seed):
    """A random soup with the triangles whose float32 centroid ((p0+p1)+p2)/3
    repeats a value on some axis removed."""
    v = soup(n, seed).reshape(-1, 3, 3)
    c = ((v[:, 0] + v[:, 1]) + v[:, 2]) / np.float32(3.0)
    keep = np.ones(len(v), bool)
    for a in range(3):
        _, inv, cnt = np.unique(c[:, a], return_inverse=True, return_counts=True)
        keep &= cnt[inv] == 1
    return np.ascontiguousarray(v[keep].reshape(-1, 3))


def gpu_median(ctx, pos, max_leaf):
    p = torch.from_numpy(pos).cuda()
    b = rq.Bvh.build(ctx, p, None, max_leaf=max_leaf, median=True)
    ctx.sync_check()
    out = b.download()
    b.destroy()
    return out  # nodes2, tris, nodes4, perm


def check(n2g, trg, n4g, n2r, trr, n4r):
    assert len(n2g) == len(n2r)
    assert n2g.tobytes() == n2r.tobytes(), "binary nodes"
    for nd in n2r[n2r["left_child"] < 0]:
        f, c = ~int(nd["left_child"]), int(nd["right_child"])
        a = np.sort(trg[f:f + c].view(np.uint8).reshape(c, -1), axis=0)
        b = np.sort(trr[f:f + c].view(np.uint8).reshape(c, -1), axis=0)
        assert np.array_equal(a, b), "leaf triangle sets"
    assert n4g.tobytes() == n4r.tobytes(), "4-wide nodes"


@pytest.mark.skipif(not O.have_ref(), reason="needs oracle/_ref")
@pytest.mark.parametrize("n,seed,max_leaf", [(1, 1, 4), (2, 2, 4), (5, 3, 4), (17, 4, 1), (100, 5, 4),
                                             (1000, 6, 8), (4097, 7, 4), (100000, 8, 4)])
def test_median_matches_reference_live(ctx, n, seed, max_leaf):
    pos = tie_free_soup(n, seed)
    idx = np.arange(len(pos), dtype=np.uint32)
    n2r, trr, n4r = O.ref_build(pos, idx, max_leaf)
    n2g, trg, n4g, perm = gpu_median(ctx, pos, max_leaf)
    check(n2g, trg, n4g, n2r, trr, n4r)
    # the permutation names the triangles written in leaf order
    v = pos.reshape(-1, 3, 3)
    assert np.array_equal(trg["v0"][:, :3], v[perm, 0]) and np.array_equal(trg["v2"][:, :3], v[perm, 2])


def test_median_matches_reference_fixtures(ctx):
    g = np.load(GOLD)
    for key in sorted(k for k in g.files if k.startswith("pos_")):
        tag = key[4:]
        max_leaf = int(g[f"leaf_{tag}"])
        n2g, trg, n4g, _ = gpu_median(ctx, g[key], max_leaf)
        check(n2g, trg, n4g, g[f"nodes2_{tag}"].view(rq.BVH2_NODE), g[f"tris_{tag}"].view(rq.TRIANGLE),
              g[f"nodes4_{tag}"].view(rq.BVH4_NODE))


def test_median_traces_like_lbvh(ctx):
    # another tree over the same triangles: identical closest hits (hit
    # flags, primitive ids, t) except exact-t ties
    pos, idx = rq.scene_grid(64, 32, seed=0)
    p = torch.from_numpy(pos).cuda()
    i = torch.from_numpy(idx.view(np.int32)).cuda()
    bm = rq.Bvh.build(ctx, p, i, median=True)
    bl = rq.Bvh.build(ctx, p, i)
    rays = torch.from_numpy(rq.scene_rays_down(65536, seed=2)).cuda()
    hm = rq.hits_numpy(rq.trace(ctx, bm, rays)[0])
    hl = rq.hits_numpy(rq.trace(ctx, bl, rays)[0])
    assert np.array_equal(hm["hit"], hl["hit"]) and hm["t"].tobytes() == hl["t"].tobytes()
    assert (hm["primitive_id"] != hl["primitive_id"]).mean() < 1e-4
    bm.destroy()
    bl.destroy()


def test_median_build_replayed_from_a_graph(ctx):
    # the median build is stream-ordered (it launches every level a split can
    # reach and reads each level's size on the device), so a rebuild can be
    # captured in a CUDA graph beside an LBVH rebuild and replayed after the
    # vertices move; each replay equals a build outside the graph
    pos_a = tie_free_soup(30000, 61)
    n = len(pos_a) // 3
    pos_b = tie_free_soup(40000, 62)[: 3 * n]
    p = torch.from_numpy(pos_a).cuda()
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        bm = rq.Bvh.build(ctx, p, None, median=True, stream=side)  # arrays and scratch before the capture
        bl = rq.Bvh.build(ctx, p, None, stream=side)
        side.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=side):
            rq.Bvh.build(ctx, p, None, median=True, into=bm, stream=side)
            rq.Bvh.build(ctx, p, None, into=bl, stream=side)
    for pos in (pos_b, pos_a):
        p.copy_(torch.from_numpy(pos))
        g.replay()
        torch.cuda.synchronize()
        ctx.sync_check()
        got_m, got_l = bm.download(), bl.download()
        want_m = gpu_median(ctx, pos, 4)
        o = O.lbvh_build(pos.reshape(-1), None)
        for a, b in zip(got_m, want_m):
            assert a.tobytes() == b.tobytes()
        assert got_l[0].tobytes() == o["nodes2"].tobytes() and got_l[2].tobytes() == o["nodes4"].tobytes()
    del g
    bm.destroy()
    bl.destroy()
