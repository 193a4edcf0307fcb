"""GPU parity of two-level scenes (rq_tlas_build / rq_tlas_trace): rotated,
scaled and translated instances of shared BLAS handles, closest and any hit,
both triangle tests and cull masks, bit-exact with the oracle's statement of
the same build and traversal; one identity instance equals rq_trace."""
import numpy as np
import pytest
import torch

import pyoracle as O
import rq
from rq import workloads as W

pytestmark = pytest.mark.gpu


def random_transform(rng):
    q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
    a = q @ np.diag(rng.uniform(0.5, 2.0, 3))
    t = rng.uniform(-5.0, 5.0, 3)
    return np.hstack([a, t[:, None]]).astype(np.float32)


def scene(ctx, seed=3):
    rng = np.random.default_rng(seed)
    meshes = [rq.scene_grid(*W.grid_for_triangles(t), seed=70 + k) for k, t in enumerate([2000, 8000, 500])]
    blas = [rq.Bvh.build(ctx, torch.from_numpy(p).cuda(), torch.from_numpy(i.view(np.int32)).cuda())
            for p, i in meshes]
    host = [b.download() for b in blas]  # nodes2, tris, nodes4, perm
    insts = [(random_transform(rng), 1000 + k, [0x1, 0x2, 0xFF][k % 3], k % 3) for k in range(24)]
    return blas, host, insts


def rays_in_box(n, seed):
    rng = np.random.default_rng(seed)
    r = np.zeros(n, rq.RAY)
    r["org"] = rng.uniform(-8, 8, (n, 3))
    d = rng.standard_normal((n, 3))
    r["dir"] = d / np.linalg.norm(d, axis=1, keepdims=True)
    r["tmin"] = 0.0
    r["tmax"] = 1e30
    return r


@pytest.mark.parametrize("flags", [0, rq.RQ_TRACE_ANY, rq.RQ_TRI_MT, rq.RQ_TRACE_ANY | rq.RQ_TRI_MT])
def test_tlas_matches_oracle(ctx, flags):
    blas, host, insts = scene(ctx)
    t = rq.Tlas(ctx, [(x, i, m, blas[b]) for x, i, m, b in insts])
    rays = rays_in_box(50000, 5)
    rt = torch.from_numpy(rays.view(np.float32).reshape(-1, 8)).cuda()
    for cull in (0xFF, 0x1):
        got = rq.hits_numpy(t.trace(rt, flags=flags, cull_mask=cull))
        ctx.sync_check()
        want = O.tlas_trace([(h[2], h[1], h[3]) for h in host], [b for _, _, _, b in insts],
                            [x for x, _, _, _ in insts], [i for _, i, _, _ in insts], [m for _, _, m, _ in insts],
                            rays, flags=flags, cull=cull)
        assert got.tobytes() == want.tobytes(), (flags, cull)
        hit = got["hit"] == 1
        assert 0.02 < hit.mean() < 0.95
        seen = set(got["instance_id"][hit].tolist())
        if cull == 0x1:
            assert seen <= {1000 + k for k in range(24) if k % 3 != 1}
        else:
            assert len(seen) > 12
    t.destroy()
    for b in blas:
        b.destroy()


def test_identity_instance_equals_plain_trace(ctx):
    pos, idx = rq.scene_grid(64, 32, seed=0)
    b = rq.Bvh.build(ctx, torch.from_numpy(pos).cuda(), torch.from_numpy(idx.view(np.int32)).cuda())
    eye = np.hstack([np.eye(3), np.zeros((3, 1))]).astype(np.float32)
    t = rq.Tlas(ctx, [(eye, 7, 0xFF, b)])
    rays = torch.from_numpy(rq.scene_rays_down(65536, seed=1)).cuda()
    for flags in (0, rq.RQ_TRACE_ANY):
        a = rq.hits_numpy(t.trace(rays, flags=flags))
        p, _, _ = rq.trace(ctx, b, rays, flags=flags)
        p = rq.hits_numpy(p)
        assert np.array_equal(a["hit"], p["hit"]) and np.array_equal(a["primitive_id"], p["primitive_id"])
        assert a["t"].tobytes() == p["t"].tobytes()
        assert (a["instance_id"][a["hit"] == 1] == 7).all()
    t.destroy()
    b.destroy()


def test_tlas_rejects_bad_instances(ctx):
    pos, idx = rq.scene_grid(8, 8, seed=0)
    b = rq.Bvh.build(ctx, torch.from_numpy(pos).cuda(), torch.from_numpy(idx.view(np.int32)).cuda())
    with pytest.raises(rq.RqError):
        rq.Tlas(ctx, [(np.zeros((3, 4), np.float32), 0, 0xFF, b)])  # singular
    with pytest.raises(rq.RqError):
        rq.Tlas(ctx, [])
    b.destroy()
