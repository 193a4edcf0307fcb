"""Failure handling without a GPU fault.

A bounded device wait on a flag that nothing sets runs out, the context
reports RQ_ERR_DEVICE_TIMEOUT and stays usable.  The serving loop turns
host-injected allocation and launch failures and cancellations into
per-request statuses and keeps serving; the other requests' results are
unchanged."""
import numpy as np
import pytest
import torch

import rq
from rq import workloads as W

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_context_survives(ctx):
    flag = torch.zeros(1, dtype=torch.int32, device="cuda")
    ctx.debug_wait_timeout(flag, 2000)  # about 0.2 ms of polls; nothing sets the flag
    with pytest.raises(rq.RqError) as e:
        ctx.sync_check()
    assert e.value.status == rq.RQ_ERR_DEVICE_TIMEOUT
    ctx.sync_check()  # reading the error word cleared it
    flag.fill_(1)
    ctx.debug_wait_timeout(flag, 2000)  # the word already left 0: no wait
    ctx.sync_check()
    pos, idx = rq.scene_grid(16, 16, seed=1)
    b = rq.Bvh.build(ctx, torch.from_numpy(pos).cuda(), torch.from_numpy(idx.view(np.int32)).cuda())
    hits, _, _ = rq.trace(ctx, b, torch.from_numpy(rq.scene_rays_down(1000, seed=2)).cuda())
    ctx.sync_check()
    assert (rq.hits_numpy(hits)["hit"] == 1).any()
    b.destroy()
    with pytest.raises(rq.RqError):
        ctx.debug_wait_timeout(flag, 1 << 21)


def small_meshes():
    return [rq.scene_grid(*W.grid_for_triangles(t), seed=50 + k) for k, t in enumerate([200, 3000, 20000])]


def alone(ctx, mesh, kind, count, seed):
    pos, idx = mesh
    p = torch.from_numpy(pos).cuda()
    ix = torch.from_numpy(idx.view(np.int32)).cuda()
    b = rq.Bvh.build(ctx, p, ix)
    rays, _ = rq.gen_mesh_rays(ctx, p, ix, kind, seed, count)
    hits, _, _ = rq.trace(ctx, b, rays, flags=rq.RQ_TRACE_CLOSEST if kind == rq.RQ_RAYS_CLOSEST else rq.RQ_TRACE_ANY)
    ctx.sync_check()
    b.destroy()
    return hits.cpu().numpy()


@pytest.mark.parametrize("mode", [rq.RQ_SERVE_PLAIN, rq.RQ_SERVE_BATCHED])
def test_injected_allocation_failure_fails_one_request(ctx, mode):
    meshes = small_meshes()
    srv = rq.Server(mode=mode)
    ids = [srv.add_mesh(p, i) for p, i in meshes]
    srv.inject_fault(rq.RQ_FAULT_ALLOC, 1)
    outs = [torch.empty((500, 4), dtype=torch.int32, device="cuda") for _ in range(6)]
    t = [srv.submit(srv.request(ids[k % 3], rq.RQ_RAYS_AO, 500, outs[k], seed=k)) for k in range(6)]
    comp = srv.completions()
    st = srv.stats()
    srv.close()
    status = [comp[x]["status"] for x in t]
    assert status.count(rq.RQ_ERR_OOM) == 1 and status.count(rq.RQ_OK) == 5, status
    assert st["failed"] == 1 and st["completed"] == 5
    for k in range(6):
        if status[k] == rq.RQ_OK:
            assert outs[k].cpu().numpy().tobytes() == alone(ctx, meshes[k % 3], rq.RQ_RAYS_AO, 500, k).tobytes()


def test_injected_launch_failure_fails_its_launch_only(ctx):
    meshes = small_meshes()
    srv = rq.Server(mode=rq.RQ_SERVE_PLAIN)
    ids = [srv.add_mesh(p, i) for p, i in meshes]
    srv.inject_fault(rq.RQ_FAULT_LAUNCH, 1)
    outs = [torch.empty((700, 4), dtype=torch.int32, device="cuda") for _ in range(4)]
    t = [srv.submit(srv.request(ids[k % 3], rq.RQ_RAYS_SHADOW, 700, outs[k], seed=k)) for k in range(4)]
    comp = srv.completions()
    srv.close()
    assert comp[t[0]]["status"] == rq.RQ_ERR_CUDA
    for k in range(1, 4):
        assert comp[t[k]]["status"] == rq.RQ_OK
        assert outs[k].cpu().numpy().tobytes() == alone(ctx, meshes[k % 3], rq.RQ_RAYS_SHADOW, 700, k).tobytes()


def test_cancel_before_admission(ctx):
    meshes = small_meshes()
    srv = rq.Server(mode=rq.RQ_SERVE_PLAIN)
    ids = [srv.add_mesh(p, i) for p, i in meshes]
    outs = [torch.empty((200000, 4), dtype=torch.int32, device="cuda") for _ in range(40)]
    t = [srv.submit(srv.request(ids[2], rq.RQ_RAYS_SHADOW, 200000, outs[k], seed=k)) for k in range(40)]
    for x in t[20:]:
        srv.cancel(x)
    with pytest.raises(rq.ServeError):
        srv.cancel(10 ** 9)
    comp = srv.completions()
    srv.close()
    status = [comp[x]["status"] for x in t]
    assert all(s == rq.RQ_OK for s in status[:20])
    assert all(s in (rq.RQ_OK, rq.RQ_ERR_CANCELLED) for s in status[20:])
    assert status[20:].count(rq.RQ_ERR_CANCELLED) >= 10
