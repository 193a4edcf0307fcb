"""GPU tests of the serving loop (include/rq_serve.h).

Every request's result must be the same in the mix (batched mode: many
requests per launch, several launches in flight, meshes evicted and rebuilt
under a tight budget) as alone (rq_build + rq_gen_mesh_rays + rq_trace on
that mesh), as in plain mode, and — for small requests — as the oracle's
build and traversal on the same rays, bit for bit."""
import numpy as np
import pytest
import torch

import pyoracle as O
import rq
from rq import workloads as W

pytestmark = pytest.mark.gpu

SIZES = [64, 200, 2000, 9000, 30000, 100000]


def catalogue():
    meshes = []
    for m, t in enumerate(SIZES):
        qx, qy = W.grid_for_triangles(t)
        meshes.append(rq.scene_grid(qx, qy, seed=400 + m))
    return meshes


def request_mix(meshes, n=48, seed=7):
    """(mesh, kind, rays, seed, flags) tuples covering every kind, counts
    below, at and above 32-id boundaries, and caller-buffer rays."""
    rng = np.random.default_rng(seed)
    counts = [1, 31, 32, 33, 1000, 40000] + list(rng.integers(1, 20000, n - 6))
    out = []
    for i, c in enumerate(counts):
        mesh = int(rng.integers(0, len(meshes)))
        kind = [rq.RQ_RAYS_SHADOW, rq.RQ_RAYS_AO, rq.RQ_RAYS_CLOSEST, rq.RQ_RAYS_BUFFER][i % 4]
        out.append((mesh, kind, int(c), 1000 + i, rq.RQ_TRACE_ANY if i % 8 == 3 else rq.RQ_TRACE_CLOSEST))
    return out


def buffer_rays(i, count):
    r = rq.scene_rays_down(count, seed=9000 + i)
    return torch.from_numpy(r).cuda()


def alone(ctx, mesh, kind, count, seed, flags, rays_buf):
    pos, idx = mesh
    p = torch.from_numpy(pos).cuda()
    ix = torch.from_numpy(idx.view(np.int32)).cuda()
    b = rq.Bvh.build(ctx, p, ix)
    if kind == rq.RQ_RAYS_BUFFER:
        rays, anyf = rays_buf, None
        hits, _, _ = rq.trace(ctx, b, rays, flags=flags)
    else:
        rays, anyf = rq.gen_mesh_rays(ctx, p, ix, kind, seed, count)
        hits, _, _ = rq.trace(ctx, b, rays, flags=rq.RQ_TRACE_CLOSEST if kind == rq.RQ_RAYS_CLOSEST else rq.RQ_TRACE_ANY)
    ctx.sync_check()
    b.destroy()
    return hits.cpu().numpy(), rays


def serve(meshes, reqs, bufs, **cfg):
    srv = rq.Server(**cfg)
    ids = [srv.add_mesh(p, i) for p, i in meshes]
    outs = [torch.full((c, 4), -7, dtype=torch.int32, device="cuda") for (_, _, c, _, _) in reqs]
    tickets = []
    for k, (m, kind, c, seed, flags) in enumerate(reqs):
        r = srv.request(ids[m], kind, c, outs[k], seed=seed, rays=bufs.get(k), flags=flags, user=k)
        tickets.append(srv.submit(r))
    comp = srv.completions()
    stats = srv.stats()
    srv.close()
    torch.cuda.synchronize()
    return [o.cpu().numpy() for o in outs], comp, tickets, stats


def test_generated_rays_match_oracle(ctx):
    pos, idx = rq.scene_grid(40, 30, seed=11)
    p = torch.from_numpy(pos).cuda()
    ix = torch.from_numpy(idx.view(np.int32)).cuda()
    for kind in (rq.RQ_RAYS_SHADOW, rq.RQ_RAYS_AO, rq.RQ_RAYS_CLOSEST):
        rays, anyf = rq.gen_mesh_rays(ctx, p, ix, kind, 77, 20000)
        want, wany = O.gen_mesh_rays(pos, idx, kind, 77, 20000)
        assert rays.cpu().numpy().tobytes() == want.tobytes(), kind
        assert np.array_equal(anyf.cpu().numpy().astype(np.uint32), wany)


def test_served_equals_alone_plain_and_oracle(ctx):
    meshes = catalogue()
    reqs = request_mix(meshes)
    bufs = {k: buffer_rays(k, c) for k, (_, kind, c, _, _) in enumerate(reqs) if kind == rq.RQ_RAYS_BUFFER}
    # budget: room for the largest mesh and a little more, so the mix evicts
    budget = rq.Server.mesh_bytes(*[len(x) for x in meshes[-1]]) + rq.Server.mesh_bytes(*[len(x) for x in meshes[-2]])
    got, comp, tickets, st = serve(meshes, reqs, bufs, budget_bytes=budget, slots=3, max_wave_requests=16,
                                   max_wave_rays=60000)
    assert all(comp[t]["status"] == rq.RQ_OK for t in tickets), [comp[t]["status"] for t in tickets]
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["launches"] > 1 and st["max_requests_per_launch"] > 1
    assert st["evictions"] > 0 and st["peak_resident_bytes"] <= budget
    plain, pcomp, ptickets, pst = serve(meshes, reqs, bufs, mode=rq.RQ_SERVE_PLAIN)
    assert pst["launches"] == len(reqs) and pst["max_requests_per_launch"] == 1
    rebuilt, _, _, rst = serve(meshes, reqs, bufs, mode=rq.RQ_SERVE_PLAIN, rebuild=True)
    assert rst["builds"] == len(reqs)  # first use builds, every later use rebuilds
    with pytest.raises(rq.ServeError):
        rq.Server(rebuild=True)  # batched mode keeps resident BVHs
    oracle_checked = 0
    for k, (m, kind, c, seed, flags) in enumerate(reqs):
        want, rays = alone(ctx, meshes[m], kind, c, seed, flags, bufs.get(k))
        assert got[k].tobytes() == want.tobytes(), f"request {k}: mix differs from alone"
        assert plain[k].tobytes() == want.tobytes(), f"request {k}: plain differs from alone"
        assert rebuilt[k].tobytes() == want.tobytes(), f"request {k}: plain with rebuilds differs from alone"
        if c <= 2000 and SIZES[m] <= 9000 and oracle_checked < 8:
            pos, idx = meshes[m]
            o = O.lbvh_build(pos.reshape(-1), idx.reshape(-1))
            rr = rq.rays_numpy(rays)
            anyhit = flags == rq.RQ_TRACE_ANY if kind == rq.RQ_RAYS_BUFFER else kind != rq.RQ_RAYS_CLOSEST
            oh, _, _ = O.trace_bvh4(o["nodes4"], o["tris"], o["sorted"], rr, flags=1 if anyhit else 0)
            assert got[k].view(np.uint8).tobytes() == oh.tobytes(), f"request {k}: differs from the oracle"
            oracle_checked += 1
    assert oracle_checked >= 4


def test_mesh_over_budget_fails_its_requests_only(ctx):
    meshes = catalogue()[:3]
    small = rq.Server.mesh_bytes(*[len(x) for x in meshes[1]])
    srv = rq.Server(budget_bytes=small)
    ids = [srv.add_mesh(p, i) for p, i in meshes]
    h = [torch.empty((100, 4), dtype=torch.int32, device="cuda") for _ in range(3)]
    t = [srv.submit(srv.request(ids[k], rq.RQ_RAYS_SHADOW, 100, h[k], seed=k)) for k in range(3)]
    comp = srv.completions()
    srv.close()
    assert comp[t[0]]["status"] == rq.RQ_OK and comp[t[1]]["status"] == rq.RQ_OK
    assert comp[t[2]]["status"] == rq.RQ_ERR_BUDGET


def test_invalid_requests_are_refused(ctx):
    pos, idx = rq.scene_grid(4, 4, seed=1)
    srv = rq.Server()
    mid = srv.add_mesh(pos, idx)
    h = torch.empty((10, 4), dtype=torch.int32, device="cuda")
    for req in (srv.request(mid + 1, rq.RQ_RAYS_AO, 10, h), srv.request(mid, 9, 10, h),
                srv.request(mid, rq.RQ_RAYS_AO, 0, h), srv.request(mid, rq.RQ_RAYS_BUFFER, 10, h)):
        with pytest.raises(rq.ServeError) as e:
            srv.submit(req)
        assert e.value.status == rq.RQ_ERR_INVALID_ARG
    with pytest.raises(rq.ServeError):
        srv.add_mesh(pos, np.full_like(idx, len(pos)))
    srv.close()


def test_replay_timestamps(ctx):
    meshes = catalogue()[:4]
    srv = rq.Server()
    ids = [srv.add_mesh(p, i) for p, i in meshes]
    outs = [torch.empty((500, 4), dtype=torch.int32, device="cuda") for _ in range(40)]
    reqs = [srv.request(ids[k % 4], rq.RQ_RAYS_AO, 500, outs[k], seed=k) for k in range(40)]
    arrival = np.arange(40) * 1e-3
    t0 = srv.now()
    tickets = srv.replay(reqs, arrival)
    comp = srv.completions()
    srv.close()
    ts = np.array([comp[t]["t_submit"] for t in tickets]) - t0
    assert np.all(np.diff(ts) > 0) and abs(ts[-1] - ts[0] - 0.039) < 0.01
    for t in tickets:
        c = comp[t]
        assert c["status"] == rq.RQ_OK and c["t_submit"] <= c["t_admit"] <= c["t_done"]
