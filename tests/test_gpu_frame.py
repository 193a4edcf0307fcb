"""GPU parity of the fused ray-generation kernels (G-buffer primary rays,
shadow rays, AO rays) against the oracle's statement of the same frame:
bit-exact G-buffer, light masks, AO values and ray counts, on a full small
frame and on a pixel sample of the full 1080p shadows + AO workload."""
import numpy as np
import pytest
import torch

import pyoracle as O
import rq
from rq import workloads as W

pytestmark = pytest.mark.gpu


def build(ctx, pos, idx):
    return rq.Bvh.build(ctx, torch.from_numpy(pos).cuda(), torch.from_numpy(idx.view(np.int32)).cuda())


def frame(ctx, b, cam, params):
    gb = rq.render_gbuffer(ctx, b, cam)
    counter = torch.zeros(4, dtype=torch.int64, device="cuda")
    mask, ao = rq.render_shadow_ao(ctx, b, gb, params, counter=counter)
    ctx.sync_check()
    return gb, mask, ao, int(counter[0])


@pytest.mark.parametrize("flags", [0, rq.RQ_TRI_MT])
def test_small_frame_bit_exact(ctx, flags):
    pos, idx = rq.scene_grid(128, 128, seed=1)
    b = build(ctx, pos, idx)
    n2, tr, n4, perm = b.download()
    w, h = 320, 180
    cam = W.shadow_camera(w, h, flags=flags)
    params = rq.shade_params(w, h, W.shadow_lights(16), ao_spp=2, ao_tmax=0.5, flags=flags)
    gb, mask, ao, rays = frame(ctx, b, cam, params)
    og = O.render_gbuffer(n4, tr, perm, cam)
    gbn = gb.cpu().numpy().view(rq.GBUFFER_PX).reshape(-1)
    assert gbn.tobytes() == og.tobytes()
    assert (gbn["vis"] > 0).all(), "the camera sees only the mesh"
    om, oa, orays = O.render_shadow_ao(n4, tr, og, params)
    assert np.array_equal(mask.cpu().numpy().astype(np.uint32), om)
    assert ao.cpu().numpy().tobytes() == oa.tobytes()
    assert rays == orays
    # some pixels are shadowed or occluded, most are lit
    lit = np.unpackbits(om.view(np.uint8)).mean() * 32 / 16
    assert 0.5 < lit < 1.0 and 0.0 < oa.mean() < 1.0
    b.destroy()


def test_jittered_primary_rays_bit_exact(ctx):
    pos, idx = rq.scene_grid(256, 256, seed=3)
    b = build(ctx, pos, idx)
    n2, tr, n4, perm = b.download()
    cam = W.visibility_camera(400, 240, jitter=True, seed=3)
    gb = rq.render_gbuffer(ctx, b, cam)
    og = O.render_gbuffer(n4, tr, perm, cam)
    assert gb.cpu().numpy().view(rq.GBUFFER_PX).reshape(-1).tobytes() == og.tobytes()
    cam0 = W.visibility_camera(400, 240, jitter=False)
    gb0 = rq.render_gbuffer(ctx, b, cam0).cpu().numpy().view(rq.GBUFFER_PX).reshape(-1)
    assert not np.array_equal(gb0["vis"], og["vis"])  # jitter moves the samples
    b.destroy()


def test_full_1080p_workload_sampled(ctx):
    # the benchmarked frame: 2,499,848 triangles, 1920x1080, 16 lights, AO
    pos, idx = W.shadow_mesh()
    assert len(idx) == 2499848
    b = build(ctx, pos, idx)
    cam = W.shadow_camera()
    params = W.shadow_params()
    gb, mask, ao, rays = frame(ctx, b, cam, params)
    n2, tr, n4, perm = b.download()
    rng = np.random.default_rng(0)
    pixels = rng.choice(1920 * 1080, 4000, replace=False).astype(np.uint32)
    og = O.render_gbuffer(n4, tr, perm, cam, pixels)
    gbn = gb.cpu().numpy().view(rq.GBUFFER_PX).reshape(-1)
    assert gbn[pixels].tobytes() == og.tobytes()
    assert (gbn["vis"] > 0).all()
    om, oa, _ = O.render_shadow_ao(n4, tr, gbn, params, pixels)
    assert np.array_equal(mask.cpu().numpy().astype(np.uint32)[pixels], om)
    assert ao.cpu().numpy()[pixels].tobytes() == oa.tobytes()
    # ray count: up to 16 shadow rays (lights behind the local surface are
    # skipped; the sigma-0.01 jitter on a 0.0018-spaced grid makes the surface
    # rough) and one AO ray per pixel
    assert 0.6 * 16 * 1920 * 1080 < rays <= 17 * 1920 * 1080
    b.destroy()


def test_every_shadow_launch_shape_gives_identical_results(ctx):
    from rq import tune as T
    pos, idx = rq.scene_grid(96, 96, seed=4)
    b = build(ctx, pos, idx)
    w, h = 256, 144
    cam = W.shadow_camera(w, h)
    params = rq.shade_params(w, h, W.shadow_lights(16), ao_spp=2, ao_tmax=0.5)
    gb = rq.render_gbuffer(ctx, b, cam)
    base = ctx.trace_tuning()
    assert base == {"threads": 128, "chunk": 32, "reg_cap": 80, "top_levels": 0, "speculative": 0, "refill_min": 1,
                    "leaf_batch": 0}
    want_m, want_a = [x.cpu().numpy() for x in rq.render_shadow_ao(ctx, b, gb, params)]
    for t, c, r, top, spec in T.SHADE_SHAPES:
        ctx.set_trace_tuning(t, c, r, top, spec)
        m, a = rq.render_shadow_ao(ctx, b, gb, params)
        ctx.sync_check()
        assert np.array_equal(m.cpu().numpy(), want_m) and a.cpu().numpy().tobytes() == want_a.tobytes(), (t, c, r, top, spec)
    for refill in (0, 8, 16, 32):
        ctx.set_trace_tuning(64, 64, 64, 0, 0, refill)
        m, a = rq.render_shadow_ao(ctx, b, gb, params)
        ctx.sync_check()
        assert np.array_equal(m.cpu().numpy(), want_m) and a.cpu().numpy().tobytes() == want_a.tobytes(), refill
    # in-loop refill: rays finish and lanes refill inside the node loop
    for t, c, r in T.INLOOP_SHAPES:
        for refill, lb in ((1, 1), (8, 8), (16, 4), (4, 32)):
            ctx.set_trace_tuning(t, c, r, 0, 1, refill, lb)
            m, a = rq.render_shadow_ao(ctx, b, gb, params)
            ctx.sync_check()
            assert np.array_equal(m.cpu().numpy(), want_m) and a.cpu().numpy().tobytes() == want_a.tobytes(), (
                t, c, r, refill, lb)
    with pytest.raises(rq.RqError):
        ctx.set_trace_tuning(128, 32, 0, 0, 0, 1, 8)  # in-loop refill needs a speculative shape
    with pytest.raises(rq.RqError):
        ctx.set_trace_tuning(128, 64, 64, 0, 1, 8, 33)
    with pytest.raises(rq.RqError):
        ctx.set_trace_tuning(96, 32, 0)
    with pytest.raises(rq.RqError):
        ctx.set_trace_tuning(64, 64, 64, 0, 0, 33)
    ctx.set_trace_tuning(**base)
    b.destroy()


def test_ao_blur_chain_bit_exact(ctx):
    # frame -> AO -> depth -> horizontal blur -> vertical blur, against the
    # oracle's statement of shaders/bilateral_blur.comp
    pos, idx = rq.scene_grid(128, 128, seed=1)
    b = build(ctx, pos, idx)
    n2, tr, n4, perm = b.download()
    w, h = 320, 180
    cam = W.shadow_camera(w, h)
    params = rq.shade_params(w, h, W.shadow_lights(16), ao_spp=4, ao_tmax=0.5)
    gb, mask, ao, _ = frame(ctx, b, cam, params)
    vp = rq.view_proj_of(cam)
    depth = rq.gbuffer_depth(ctx, gb, vp)
    d_want = O.gbuffer_depth(gb.cpu().numpy().view(rq.GBUFFER_PX).reshape(-1), vp)
    assert depth.cpu().numpy().tobytes() == d_want.tobytes()
    dn = depth.cpu().numpy()
    assert 0.0 < dn.min() and dn.max() < 1.0, "every pixel sees the mesh"
    for thr in (1e-4, 5e-3, 1.0):
        hpass = rq.blur_ao(ctx, ao, depth, w, h, 1, 0, thr)
        vpass = rq.blur_ao(ctx, hpass, depth, w, h, 0, 1, thr)
        ctx.sync_check()
        oh = O.blur_ao(ao.cpu().numpy(), d_want, w, h, 1, 0, thr)
        ov = O.blur_ao(oh, d_want, w, h, 0, 1, thr)
        assert hpass.cpu().numpy().tobytes() == oh.tobytes(), thr
        assert vpass.cpu().numpy().tobytes() == ov.tobytes(), thr
    # background pixels (depth 1) pass through unchanged
    d1 = torch.ones_like(depth)
    same = rq.blur_ao(ctx, ao, d1, w, h, 1, 0, 0.01)
    assert torch.equal(same, ao)
    with pytest.raises(rq.RqError):
        rq.blur_ao(ctx, ao, depth, w, h, 1, 1, 0.01)
    b.destroy()


def wide_camera(w, h, flags=0):
    # looks past the mesh edge at the horizon: part of the image is empty
    return rq.camera_look_at((0.0, -2.2, 0.9), (0.0, 0.0, 0.0), (0.0, 0.0, 1.0), 50.0, w, h, flags=flags)


@pytest.mark.parametrize("flags", [0, rq.RQ_TRI_MT])
@pytest.mark.parametrize("view", ["shadow", "wide"])
def test_reflection_rays_bit_exact(ctx, flags, view):
    # tiled_lighting_ra.comp:91-113: R = reflect(normalize(P - cam), N) from
    # P + 0.04 N over [0.02, 100], closest hit, one record per pixel
    pos, idx = rq.scene_grid(128, 128, seed=1)
    b = build(ctx, pos, idx)
    n2, tr, n4, perm = b.download()
    w, h = 320, 180
    cam = W.shadow_camera(w, h, flags=flags) if view == "shadow" else wide_camera(w, h, flags)
    gb = rq.render_gbuffer(ctx, b, cam)
    hits = rq.render_reflect(ctx, b, gb, rq.reflect_params(cam, flags=flags))
    ctx.sync_check()
    gbn = gb.cpu().numpy().view(rq.GBUFFER_PX).reshape(-1)
    oh = O.render_reflect(n4, tr, perm, gbn, O.reflect_params(cam, flags=flags))
    hn = rq.hits_numpy(hits)
    assert hn.tobytes() == oh.tobytes()
    vis = gbn["vis"] > 0
    assert 0.0 < hn["hit"][vis].mean() < 1.0
    if view == "wide":
        assert (~vis).any() and (hn["hit"][~vis] == 0).all() and (hn["primitive_id"][~vis] == 0xFFFFFFFF).all()
    b.destroy()


@pytest.mark.parametrize("flags", [0, rq.RQ_TRI_MT])
@pytest.mark.parametrize("view", ["shadow", "wide"])
def test_depth_ao_bit_exact(ctx, flags, view):
    # rq_ao.comp from the depth buffer: position from depth x invViewProj,
    # normal from the right and upper neighbours, AO 1 at depth >= 1
    pos, idx = rq.scene_grid(128, 128, seed=1)
    b = build(ctx, pos, idx)
    n2, tr, n4, perm = b.download()
    w, h = 320, 180
    cam = W.shadow_camera(w, h) if view == "shadow" else wide_camera(w, h)
    gb = rq.render_gbuffer(ctx, b, cam)
    depth = rq.gbuffer_depth(ctx, gb, rq.view_proj_of(cam))
    dn = depth.cpu().numpy()
    for spp in (0, 1, 3):
        ap = rq.ao_depth_params(cam, spp=spp, max_distance=0.5, flags=flags)
        counters = torch.zeros(4, dtype=torch.int64, device="cuda")
        ao = rq.render_ao_depth(ctx, b, depth, ap, counters=counters)
        ctx.sync_check()
        oa, orays = O.render_ao_depth(n4, tr, dn, O.ao_depth_params(cam, spp=spp, max_distance=0.5, flags=flags))
        assert ao.cpu().numpy().tobytes() == oa.tobytes(), spp
        assert int(counters[0]) == orays
    if view == "wide":
        assert (dn >= 1.0).any() and (oa[dn >= 1.0] == 1.0).all()
    assert 0.0 < oa[dn < 1.0].mean() < 1.0
    with pytest.raises(rq.RqError):
        rq.render_ao_depth(ctx, b, depth, rq.ao_depth_params(cam, spp=33))
    b.destroy()


def test_every_camera_schedule_gives_identical_gbuffers(ctx):
    # one ray per thread or the refilling engine with in-loop refill, every
    # refill threshold and leaf batch: the same G-buffer bytes (closest hit,
    # jittered, both triangle tests)
    pos, idx = rq.scene_grid(160, 120, seed=6)
    b = build(ctx, pos, idx)
    base = ctx.camera_tuning()
    assert base == {"engine": 0, "refill_min": 1, "leaf_batch": 32}
    for flags in (0, rq.RQ_TRI_MT):
        cam = W.visibility_camera(320, 200, jitter=True, seed=8, flags=flags)
        want = rq.render_gbuffer(ctx, b, cam).cpu().numpy()
        for refill, lb in ((1, 32), (1, 1), (8, 8), (16, 4), (32, 16)):
            ctx.set_camera_tuning(1, refill, lb)
            got = rq.render_gbuffer(ctx, b, cam)
            ctx.sync_check()
            assert got.cpu().numpy().tobytes() == want.tobytes(), (flags, refill, lb)
        ctx.set_camera_tuning(**base)
    with pytest.raises(rq.RqError):
        ctx.set_camera_tuning(2, 1, 1)
    b.destroy()
