"""GPU parity of the RADV image build (fast_bvh_builder.comp) and of the
RADV-image traversal standing in for rayQueryEXT.

Bit-exact against Oracle C for any size; the reference's own known-answer
tests (src/main.cpp) replayed on the GPU image: the forged one-triangle KAT
(t = 5, barycentrics (0.25, 0.5), miss at (10,10,0)) and the centroid-ray
verification over generate_dynamic_grid_mesh(N, 1.25) for N = 64..4096."""
import numpy as np
import pytest
import torch

import pyoracle as O
import rq
from conftest import soup

pytestmark = pytest.mark.gpu

GRIDS = __file__.replace("test_gpu_radv.py", "golden/ref_dynamic_grids.npz")


def radv_gpu(ctx, tri9):
    t = torch.from_numpy(np.ascontiguousarray(tri9, np.float32).reshape(-1)).cuda()
    img = rq.build_radv(ctx, t)
    ctx.sync_check()
    return img


# 256 / 257 triangles: one block (each lane its own triangle) or two staged
# blocks; 131,072 / 131,073 and 4,194,300 / 4,194,304: the subtree per block
# grows from 64 to 256 and from 256 to 1,024 leaf boxes
@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 63, 64, 65, 255, 256, 257, 1023, 1024, 1025, 4096, 4097, 4100,
                               16385, 100000, 131072, 131073, 1 << 20, 1208321, 4194300, 4194304])
def test_radv_bytes_match_oracle(ctx, n):
    tri9 = soup(n, 40 + n).reshape(-1)
    img = radv_gpu(ctx, tri9).cpu().numpy()
    ref = O.radv_build(tri9)
    assert len(img) == len(ref)
    bad = np.nonzero(img != ref)[0]
    assert len(bad) == 0, f"first differing byte {bad[:8]}"


def rays_plus_z(origins, tmin=0.1, tmax=20.0):
    r = np.zeros((len(origins), 8), np.float32)
    r[:, 0:3] = origins
    r[:, 3] = tmin
    r[:, 6] = 1.0
    r[:, 7] = tmax
    return r


def test_forged_single_triangle_kat(ctx):
    # src/main.cpp:269-313, 410-413: V=(-2,-2,5),(2,-2,5),(0,2,5); ray from the
    # origin along +z hits at t=5 with barycentrics (0.25, 0.5); (10,10,0) misses.
    tri9 = np.array([-2, -2, 5, 2, -2, 5, 0, 2, 5], np.float32)
    img = radv_gpu(ctx, tri9)
    rays = torch.from_numpy(rays_plus_z(np.array([[0, 0, 0], [10, 10, 0]], np.float32), 0.0, 100.0)).cuda()
    for flags in (rq.RQ_TRI_WATERTIGHT, rq.RQ_TRI_MT):
        hits, bary = rq.trace_radv(ctx, img, rays, flags=flags, bary=True)
        h = rq.hits_numpy(hits)
        b = bary.cpu().numpy()
        assert h["hit"][0] == 1 and abs(h["t"][0] - 5.0) < 1e-3
        assert abs(b[0, 0] - 0.25) < 1e-3 and abs(b[0, 1] - 0.5) < 1e-3
        assert h["hit"][1] == 0 and h["t"][1] == -1.0 and h["primitive_id"][1] == 0xFFFFFFFF


@pytest.mark.parametrize("n", [64, 256, 1024, 4096])
def test_builder_centroid_verification(ctx, n):
    # src/main.cpp:1002-1106: for each triangle a +z ray from (cx, cy, 0),
    # tmin 0.1, tmax 20, must hit with |t - cz| < 1e-2; a ray at (10,10,0) misses.
    g = np.load(GRIDS)
    tri9, cen = g[f"tri9_{n}"], g[f"cen_{n}"].reshape(-1, 3)
    img = radv_gpu(ctx, tri9)
    org = np.concatenate([np.c_[cen[:, 0], cen[:, 1], np.zeros(n, np.float32)], [[10, 10, 0]]]).astype(np.float32)
    rays_np = rays_plus_z(org)
    rays = torch.from_numpy(rays_np).cuda()
    for flags in (0, rq.RQ_TRI_MT):
        h = rq.hits_numpy(rq.trace_radv(ctx, img, rays, flags=flags)[0])
        assert np.all(h["hit"][:n] == 1)
        assert np.all(np.abs(h["t"][:n] - cen[:, 2]) < 1e-2)
        assert h["hit"][n] == 0
        # and the whole result equals the oracle's RADV traversal
        oh, _ = O.trace_radv(radv_gpu(ctx, tri9).cpu().numpy(), rays_np.view(O.RAY).reshape(-1), flags)
        assert h.tobytes() == oh.tobytes()


@pytest.mark.parametrize("flags", [0, 1, 2, 3])
def test_radv_trace_matches_oracle(ctx, flags):
    pos, idx = rq.scene_grid(64, 32, seed=0)
    tri9 = pos[idx].reshape(-1).astype(np.float32)
    img = radv_gpu(ctx, tri9)
    rays_np = rq.scene_rays_down(20000, seed=5)
    h, b = rq.trace_radv(ctx, img, torch.from_numpy(rays_np).cuda(), flags=flags, bary=True)
    oh, ob = O.trace_radv(img.cpu().numpy(), rays_np.view(O.RAY).reshape(-1), flags, want_bary=True)
    assert rq.hits_numpy(h).tobytes() == oh.tobytes()
    assert b.cpu().numpy().reshape(-1).tobytes() == ob.tobytes()


def test_radv_size_errors(ctx):
    t = torch.zeros(9 * 8, dtype=torch.float32, device="cuda")
    small = torch.empty(rq.radv_size(8) - 1, dtype=torch.uint8, device="cuda")
    with pytest.raises(rq.RqError) as e:
        rq.build_radv(ctx, t, image=small)
    assert e.value.status == rq.RQ_ERR_SIZE


def test_device_images_describe_like_the_reference(ctx):
    import json
    grids = np.load(GRIDS)
    dumps = json.load(open(GRIDS.replace("ref_dynamic_grids.npz", "radv_dumps.json")))
    for n, text in dumps.items():
        img = radv_gpu(ctx, grids[f"tri9_{n}"])
        assert rq.radv_describe(img.cpu().numpy().tobytes()) == text, n


@pytest.mark.parametrize("n", [1, 2, 5, 64, 4097, 100000])
def test_validate_clean_images(ctx, n):
    tri9 = np.random.default_rng(n).standard_normal(9 * n).astype(np.float32)
    img = radv_gpu(ctx, tri9)
    r = rq.radv_validate(ctx, img)
    lay = rq.radv_layout(n)
    assert r["header_ok"] == 1 and r["box_nodes"] == lay["total_boxes"] and r["triangle_nodes"] == n
    assert r["box_children"] == lay["total_boxes"] - 1 and r["triangle_children"] == n
    for k in ("bad_offsets", "bad_boxes", "box_refs_wrong", "triangle_refs_wrong", "ids_wrong"):
        assert r[k] == 0, (k, r)


def test_validate_reports_damage(ctx):
    n = 1000
    tri9 = np.random.default_rng(7).standard_normal(9 * n).astype(np.float32)
    img = radv_gpu(ctx, tri9)
    host = img.cpu().numpy()
    leaf = int(host[96:104].view(np.uint64)[0])

    def check(mutate):
        h = host.copy()
        mutate(h)
        return rq.radv_validate(ctx, torch.from_numpy(h).cuda())

    # a root child id that points past the image: counted, never read
    r = check(lambda h: h.__setitem__(slice(196, 200), np.frombuffer((0x7ffffff8 | 5).to_bytes(4, "little"), np.uint8)))
    assert r["bad_offsets"] >= 1 and r["box_refs_wrong"] >= 1
    # a moved vertex in the first triangle node: its parent's box no longer fits
    r = check(lambda h: h.__setitem__(slice(leaf, leaf + 4), np.frombuffer(np.float32(99.0).tobytes(), np.uint8)))
    assert r["bad_boxes"] >= 1 and r["bad_offsets"] == 0
    # two triangle nodes with the same id
    r = check(lambda h: h.__setitem__(slice(leaf + 64 + 48, leaf + 64 + 52), h[leaf + 48:leaf + 52].copy()))
    assert r["ids_wrong"] == 2
    # a header whose leaf region runs past the image
    r = check(lambda h: h.__setitem__(slice(96, 104), np.frombuffer(np.uint64(len(h)).tobytes(), np.uint8)))
    assert r["header_ok"] == 0


@pytest.mark.parametrize("n", [5, 4097, 100000, 400000, 4500000])
def test_radv_refit_equals_rebuild(ctx, n):
    # rq_refit_radv after the vertices move: the bytes of a fresh build on the
    # new vertices (and of the oracle's image of them)
    a = soup(n, 300 + n).reshape(-1)
    moved = (a + np.float32(0.25) * np.sin(np.arange(a.size, dtype=np.float32))).astype(np.float32)
    img = radv_gpu(ctx, a)
    rq.refit_radv(ctx, torch.from_numpy(moved).cuda(), img)
    ctx.sync_check()
    assert np.array_equal(img.cpu().numpy(), O.radv_build(moved))


def test_radv_refit_of_another_count_is_reported(ctx):
    # an image built for 100 triangles refitted as 64: the header check
    # reports it on the next rq_ctx_check; the context stays usable
    img = radv_gpu(ctx, soup(100, 5).reshape(-1))
    tri64 = torch.from_numpy(soup(64, 6).reshape(-1)).cuda()
    rq.refit_radv(ctx, tri64, img)
    with pytest.raises(rq.RqError) as ei:
        ctx.sync_check()
    assert ei.value.status == rq.RQ_ERR_STATE
    out = radv_gpu(ctx, soup(64, 6).reshape(-1))  # later calls work
    assert np.array_equal(out.cpu().numpy(), O.radv_build(soup(64, 6).reshape(-1)))


@pytest.mark.parametrize("n", [1000, 20000, 600000])
def test_radv_builds_replayed_from_a_graph(ctx, n):
    # multi-block builds leave their finishing ticket ready for the next
    # launch: builds replayed back to back from a CUDA graph all finish
    tri9 = soup(n, 500 + n).reshape(-1)
    t = torch.from_numpy(np.ascontiguousarray(tri9)).cuda()
    img = torch.empty(rq.radv_size(n), dtype=torch.uint8, device="cuda")
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        rq.build_radv(ctx, t, img)  # scratch allocated before the capture
        side.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=side):
            for _ in range(3):
                rq.build_radv(ctx, t, img)
    ref = O.radv_build(tri9)
    for _ in range(2):
        img.fill_(0xAB)
        g.replay()
        torch.cuda.synchronize()
        ctx.sync_check()
        assert np.array_equal(img.cpu().numpy(), ref)
    del g
