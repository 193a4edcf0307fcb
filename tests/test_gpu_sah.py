"""GPU parity of the LBVH with SAH-rebuilt subtrees (rq_build with
RQ_BUILD_SAH) against the oracle's statement of the same build
(orc_lbvh_sah_build): Morton keys, leaf-order permutation, binary nodes,
leaf-ordered triangles and 4-wide nodes byte for byte, at sizes around the
1,024 triangles a block rebuilds in shared memory (larger nodes are split by
the node queue first), the 16,384-triangle subtree limit, the one-subtree case
and the 32-triangle switch from 16 to 8 bins, for every leaf size,
degenerate inputs (equal centroids), trees past the depth cap, a grid mesh,
and a refit; traversal on
the rebuilt tree bit-exact with the oracle's traversal of it."""
import numpy as np
import pytest
import torch

import pyoracle as O
import rq
from conftest import soup

pytestmark = pytest.mark.gpu


def sah_build(ctx, pos, idx=None, max_leaf=4):
    p = torch.from_numpy(np.ascontiguousarray(pos, np.float32)).cuda()
    i = torch.from_numpy(np.ascontiguousarray(idx, np.uint32).view(np.int32)).cuda() if idx is not None else None
    b = rq.Bvh.build(ctx, p, i, max_leaf=max_leaf, sah=True)
    ctx.sync_check()
    return b


def assert_same_as_oracle(ctx, pos, idx, max_leaf=4):
    b = sah_build(ctx, pos, idx, max_leaf)
    n2, tr, n4, perm = b.download()
    keys, ids = b.download_sort()
    o = O.lbvh_sah_build(np.ascontiguousarray(pos, np.float32).reshape(-1),
                         None if idx is None else np.ascontiguousarray(idx).reshape(-1), max_leaf, rq.SAH_SUBTREE_MAX)
    assert np.array_equal(keys, o["codes"][o["sorted"]]), "Morton keys"
    assert np.array_equal(perm, o["perm"]) and np.array_equal(ids, o["perm"]), "leaf-order permutation"
    assert len(n2) == len(o["nodes2"]) and n2.tobytes() == o["nodes2"].tobytes(), "binary nodes"
    assert tr.tobytes() == o["tris"].tobytes(), "leaf-ordered triangles"
    assert len(n4) == len(o["nodes4"]) and n4.tobytes() == o["nodes4"].tobytes(), "4-wide nodes"
    assert b.info()["depth4"] == o["depth4"]
    b.destroy()
    return o


@pytest.mark.parametrize("n", [1, 2, 3, 5, 17, 31, 32, 33, 64, 65, 100, 1000, 1023, 1024, 1025, 2049, 4097, 16383,
                               16384, 16385, 50000, 65537, 300000])
def test_sah_soup_parity(ctx, n):
    assert_same_as_oracle(ctx, soup(n, 300 + n), None)


@pytest.mark.parametrize("n", [33, 65, 700])
def test_sah_bin_count_boundary(ctx, n):
    # leaves of one triangle: every node is split, so nodes of 33 triangles
    # (16 bins) and of 32 (8 bins) meet under each other
    assert_same_as_oracle(ctx, soup(n, 900 + n), None, max_leaf=1)


@pytest.mark.parametrize("max_leaf", [1, 2, 4, 8, 16])
def test_sah_max_leaf_parity(ctx, max_leaf):
    assert_same_as_oracle(ctx, soup(6000, 7), None, max_leaf)


def test_sah_grid_parity_and_fewer_visits(ctx):
    pos, idx = rq.scene_grid(200, 160, seed=1)
    o = assert_same_as_oracle(ctx, pos, idx)
    ol = O.lbvh_build(pos.reshape(-1), idx.reshape(-1))
    assert len(o["nodes4"]) < len(ol["nodes4"])


def test_sah_degenerate_centroids(ctx):
    # every centroid equal: no axis has an extent, every split is the middle
    v = np.tile(soup(1, 9), (3000, 1)).astype(np.float32)
    assert_same_as_oracle(ctx, v, None)
    # equal centroids on one axis only
    w = soup(5000, 10)
    w[:, 2] = np.float32(0.5)
    assert_same_as_oracle(ctx, w, None)


@pytest.mark.parametrize("n, ratio", [(200, 1.25), (3000, 1.012)])
def test_sah_depth_cap(ctx, n, ratio):
    # small triangles spaced geometrically along x: the cheapest split cuts off
    # the few farthest ones, so the tree runs past the depth cap (24 levels)
    # and continues with middle splits; at 3,000 triangles the node queue
    # takes the first levels
    x = (ratio ** np.arange(n, dtype=np.float64)).astype(np.float32)
    v = np.zeros((n, 9), np.float32)
    v[:, 0] = x
    v[:, 3] = x + np.float32(0.1)
    v[:, 6] = x
    v[:, 7] = np.float32(0.1)
    o = assert_same_as_oracle(ctx, v, None)
    assert o["depth4"] > 12


def test_sah_trace_bit_exact_and_refit(ctx):
    pos, idx = rq.scene_grid(128, 96, seed=2)
    b = sah_build(ctx, pos, idx)
    n2, tr, n4, perm = b.download()
    rays_np = rq.scene_rays_down(100000, spread=0.5, seed=5)
    rays = torch.from_numpy(rays_np).cuda()
    for flags in (0, 1, 2, 3):
        hits, _, stats = rq.trace(ctx, b, rays, flags=flags, stats=True)
        oh, _, os_ = O.trace_bvh4(n4, tr, perm, rays_np.view(O.RAY).reshape(-1), flags, want_stats=True)
        assert rq.hits_numpy(hits).tobytes() == oh.tobytes(), flags
        assert rq.stats_numpy(stats).tobytes() == os_.tobytes(), flags
    # refit after a deformation equals the oracle's refit of this topology
    p = torch.from_numpy(pos).cuda()
    q = torch.empty_like(p)
    i = torch.from_numpy(idx.view(np.int32)).cuda()
    rq.deform_wave(ctx, p, q, 0.9, 0.05, 1.0)
    b.refit(q, i)
    ctx.sync_check()
    n2f, trf, n4f, permf = b.download()
    otr, on2, on4 = O.refit(q.cpu().numpy(), idx, perm, n2, n4)
    assert trf.tobytes() == otr.tobytes() and n2f.tobytes() == on2.tobytes() and n4f.tobytes() == on4.tobytes()
    b.destroy()


def test_sah_in_place_rebuilds_switch_modes(ctx):
    # one handle rebuilt as LBVH, SAH, LBVH: each equals its oracle
    pos = soup(20000, 44)
    p = torch.from_numpy(pos).cuda()
    b = rq.Bvh.build(ctx, p, None)
    for sah in (True, False, True):
        rq.Bvh.build(ctx, p, None, sah=sah, into=b)
        ctx.sync_check()
        n2, tr, n4, perm = b.download()
        o = O.lbvh_sah_build(pos.reshape(-1), None, 4, rq.SAH_SUBTREE_MAX) if sah else O.lbvh_build(pos.reshape(-1), None)
        assert n2.tobytes() == o["nodes2"].tobytes() and n4.tobytes() == o["nodes4"].tobytes(), sah
    with pytest.raises(rq.RqError):
        rq.Bvh.build(ctx, p, None, sah=True, median=True)
    b.destroy()
