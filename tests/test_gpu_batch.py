"""GPU parity of the batched form: one persistent launch builds many meshes,
one launch traces rays of all of them.  Every mesh's bytes must equal a
separate rq_build of that mesh (itself bit-exact with the oracle), and every
hit must equal a separate rq_trace on that mesh."""
import numpy as np
import pytest
import torch

import pyoracle as O
import rq
from rq import workloads as W

pytestmark = pytest.mark.gpu


def make_batch(ctx, sizes, seed=5):
    pos, idx, descs = W.batched_meshes(sizes, seed=seed)
    p = torch.from_numpy(pos).cuda()
    i = torch.from_numpy(idx.view(np.int32)).cuda()
    b = rq.Batch(ctx, descs)
    b.build(p, i)
    ctx.sync_check()
    return pos, idx, descs, p, i, b


SIZES = [2, 4, 6, 64, 100, 998, 4096, 20000, 65536, 3, 130]


def test_batch_bytes_equal_separate_builds(ctx):
    pos, idx, descs, p, i, b = make_batch(ctx, SIZES)
    for m, (vo, nv, to, nt) in enumerate(descs):
        pm, im = pos[vo:vo + nv], idx[to:to + nt]
        s = rq.Bvh.build(ctx, torch.from_numpy(pm).cuda(), torch.from_numpy(im.view(np.int32)).cuda())
        got = b.download(m)
        want = s.download()
        for g, w, name in zip(got, want, ("nodes2", "tris", "nodes4", "perm")):
            assert g.tobytes() == w.tobytes(), f"mesh {m} ({nt} triangles): {name} differs"
        assert b.info(m)["depth4"] == s.info()["depth4"]
        s.destroy()
    # and one mesh against the oracle directly
    vo, nv, to, nt = descs[7]
    o = O.lbvh_build(pos[vo:vo + nv].reshape(-1), idx[to:to + nt].reshape(-1))
    n2, tr, n4, pm = b.download(7)
    assert n2.tobytes() == o["nodes2"].tobytes() and n4.tobytes() == o["nodes4"].tobytes()
    b.destroy()


def test_batch_rebuild_is_stable(ctx):
    pos, idx, descs, p, i, b = make_batch(ctx, SIZES)
    first = [b.download(m) for m in range(len(descs))]
    b.build(p, i)
    ctx.sync_check()
    for m in range(len(descs)):
        assert all(x.tobytes() == y.tobytes() for x, y in zip(first[m], b.download(m)))
    b.destroy()


@pytest.mark.parametrize("tri_flags", [0, rq.RQ_TRI_MT])
def test_batch_trace_equals_separate_traces(ctx, tri_flags):
    pos, idx, descs, p, i, b = make_batch(ctx, SIZES)
    rays, mesh, flags = W.batched_rays(descs, 500, 700, seed=11)
    rays_t = torch.from_numpy(rays).cuda()
    hits, stats = b.trace(rays_t, torch.from_numpy(mesh.view(np.int32)).cuda(),
                          torch.from_numpy(flags.view(np.int32)).cuda(), flags=tri_flags, stats=True)
    h = rq.hits_numpy(hits)
    st = rq.stats_numpy(stats)
    for m, (vo, nv, to, nt) in enumerate(descs):
        s = rq.Bvh.build(ctx, torch.from_numpy(pos[vo:vo + nv]).cuda(),
                         torch.from_numpy(idx[to:to + nt].view(np.int32)).cuda())
        sel = np.nonzero(mesh == m)[0]
        for f in (0, 1):
            part = sel[flags[sel] == f]
            hh, _, ss = rq.trace(ctx, s, torch.from_numpy(rays[part]).cuda(), flags=f | tri_flags, stats=True)
            assert rq.hits_numpy(hh).tobytes() == h[part].tobytes(), (m, f)
            assert rq.stats_numpy(ss).tobytes() == st[part].tobytes(), (m, f)
        s.destroy()
    assert 0.3 < h["hit"].mean() < 0.9
    b.destroy()


def test_batched_workload_sampled(ctx):
    # the batched configuration's 512 meshes (log-uniform 64..65,536), one build
    sizes = W.batched_sizes(512, seed=2)
    pos, idx, descs, p, i, b = make_batch(ctx, sizes, seed=2)
    rng = np.random.default_rng(1)
    for m in rng.choice(len(descs), 6, replace=False):
        vo, nv, to, nt = descs[m]
        o = O.lbvh_build(pos[vo:vo + nv].reshape(-1), idx[to:to + nt].reshape(-1))
        n2, tr, n4, pm = b.download(int(m))
        assert n2.tobytes() == o["nodes2"].tobytes() and n4.tobytes() == o["nodes4"].tobytes(), m
    # the same batch built with clusters for its large meshes: every mesh's
    # bytes unchanged, and the largest against the oracle
    want = [b.download(m) for m in range(len(descs))]
    for bt, cl, min_tris in ((1024, 2, 16384), (512, 4, 8192)):
        b.set_tuning({"build_threads": bt, "build_blocks": b.tuning()["max_build_blocks"], "build_cluster": cl,
                      "cluster_min_tris": min_tris})
        b.build(p, i)
        ctx.sync_check()
        for m in range(len(descs)):
            assert all(x.tobytes() == y.tobytes() for x, y in zip(want[m], b.download(m))), (bt, cl, m)
    m = int(np.argmax(sizes))
    vo, nv, to, nt = descs[m]
    o = O.lbvh_build(pos[vo:vo + nv].reshape(-1), idx[to:to + nt].reshape(-1))
    n2, tr, n4, pm = b.download(m)
    assert n2.tobytes() == o["nodes2"].tobytes() and n4.tobytes() == o["nodes4"].tobytes(), m
    b.destroy()


def test_batch_rejects_bad_descriptors(ctx):
    with pytest.raises(rq.RqError):
        rq.Batch(ctx, [(0, 3, 0, 2), (0, 3, 1, 2)])  # overlapping triangle ranges
    with pytest.raises(rq.RqError):
        rq.Batch(ctx, [(0, 3, 0, 0)])  # empty mesh


def test_every_launch_shape_gives_identical_results(ctx):
    pos, idx, descs, p, i, b = make_batch(ctx, SIZES)
    rays, mesh, flags = W.batched_rays(descs, 300, 300, seed=12)
    rays_t = torch.from_numpy(rays).cuda()
    mesh_t = torch.from_numpy(mesh.view(np.int32)).cuda()
    flags_t = torch.from_numpy(flags.view(np.int32)).cuda()
    want_tree = [b.download(m) for m in range(len(descs))]
    depths = [b.info(m)["depth4"] for m in range(len(descs))]
    want_hits = b.trace(rays_t, mesh_t, flags_t)[0].cpu().numpy()
    base = b.tuning()
    assert base["build_cluster"] == 1
    assert base["build_threads"] == 512 and base["trace_threads"] == 128 and base["max_build_blocks"] >= 1
    for bt, blocks in ((256, 1), (1024, 3), (512, base["max_build_blocks"])):
        b.set_tuning({"build_threads": bt, "build_blocks": blocks, "build_cluster": 1})
        b.build(p, i)
        ctx.sync_check()
        for m in range(len(descs)):
            assert all(x.tobytes() == y.tobytes() for x, y in zip(want_tree[m], b.download(m))), (bt, blocks, m)
    # thread-block clusters: every mesh (threshold 0, the 2-triangle ones
    # included), the large ones only, and grids that round down to whole
    # clusters or hold fewer blocks than one cluster
    for bt, blocks, cl, min_tris in ((1024, 8, 2, 0), (256, 8, 4, 0), (512, 5, 2, 1000), (1024, 11, 4, 20000),
                                     (512, base["max_build_blocks"], 4, 4096), (256, 1, 4, 0)):
        b.set_tuning({"build_threads": bt, "build_blocks": blocks, "build_cluster": cl, "cluster_min_tris": min_tris})
        b.build(p, i)
        ctx.sync_check()
        for m in range(len(descs)):
            got = b.download(m)
            assert all(x.tobytes() == y.tobytes() for x, y in zip(want_tree[m], got)), (bt, blocks, cl, min_tris, m)
        assert [b.info(m)["depth4"] for m in range(len(descs))] == depths
    for tt in (64, 128, 256):
        for chunk in (32, 64):
            for cap in (0, 64, 80):
                b.set_tuning({"trace_threads": tt, "trace_chunk": chunk, "trace_reg_cap": cap, "stack_entries": 128})
                got = b.trace(rays_t, mesh_t, flags_t)[0].cpu().numpy()
                ctx.sync_check()
                assert got.tobytes() == want_hits.tobytes(), (tt, chunk, cap)
    with pytest.raises(rq.RqError):
        b.set_tuning({"trace_threads": 96})
    with pytest.raises(rq.RqError):
        b.set_tuning({"build_cluster": 3})
    b.destroy()


def test_autotune_keeps_a_measured_shape(ctx):
    pos, idx, descs, p, i, b = make_batch(ctx, SIZES)
    rays, mesh, flags = W.batched_rays(descs, 200, 200, seed=13)
    rays_t = torch.from_numpy(rays).cuda()
    mesh_t = torch.from_numpy(mesh.view(np.int32)).cuda()
    flags_t = torch.from_numpy(flags.view(np.int32)).cuda()
    want = b.trace(rays_t, mesh_t, flags_t)[0].cpu().numpy()
    shape, trials = b.autotune(p, i, rays_t, mesh_t, flags_t, reps=2)
    builds = [t for t in trials if t["build_ms"] > 0]
    traces = [t for t in trials if t["trace_ms"] > 0]
    # 3 block sizes x 2 chunks x budgets {none, 64, 80}, plus 72 at 64 and 128 threads, then 4 refill
    # thresholds for the fastest of those
    assert len(traces) == 26 and len(builds) >= 3
    assert shape["build_ms"] == min(t["build_ms"] for t in builds)
    assert shape["trace_ms"] == min(t["trace_ms"] for t in traces)
    assert shape["stack_entries"] >= 3 * (max(b.info(m)["depth4"] for m in range(len(descs))) + 2) + 1
    got = b.trace(rays_t, mesh_t, flags_t)[0].cpu().numpy()
    assert got.tobytes() == want.tobytes()
    b.destroy()
