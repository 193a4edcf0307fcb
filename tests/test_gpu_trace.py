"""GPU parity of the traversal kernels through the C ABI.

  - rq_trace (engine traversal): bit-exact against the oracle's statement of
    the same traversal on the same tree (hits, t bits, barycentrics, stats),
    for closest/any hit and watertight/Moller-Trumbore triangles;
  - rq_trace against the reference pipeline (the reference's own SoftwareBVH
    tree + the restated software_bvh_bvh4.comp traversal): identical hit flags
    and closest-hit primitive IDs except rays that graze a shared edge, which
    are counted and must stay under 1e-5 of the rays; t within 1e-6 relative;
  - rq_trace_ref_bvh4 / rq_trace_ref_bvh2 (the reference shaders' own
    semantics) and the procedural ray generator: bit-exact against the oracle,
    and the published SW BVH4 statistics reproduced on the GPU."""
import json
import os

import numpy as np
import pytest
import torch

import pyoracle as O
import rq
from parity_util import assert_t_close, graze_report

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def build_plain(ctx, seed=0):
    pos, idx = rq.scene_grid(64, 32, seed=seed)
    b = rq.Bvh.build(ctx, torch.from_numpy(pos).cuda(), torch.from_numpy(idx.view(np.int32)).cuda())
    return pos, idx, b


@pytest.mark.parametrize("flags", [0, 1, 2, 3])
def test_trace_bit_exact_vs_oracle(ctx, flags):
    # plain workload: 4,096 triangles, 65,536 downward rays (seed 0)
    pos, idx, b = build_plain(ctx)
    n2, tr, n4, perm = b.download()
    rays_np = rq.scene_rays_down(65536, seed=0)
    rays = torch.from_numpy(rays_np).cuda()
    hits, bary, stats = rq.trace(ctx, b, rays, flags=flags, bary=True, stats=True)
    ctx.sync_check()
    oh, ob, os_ = O.trace_bvh4(n4, tr, perm, rays_np.view(O.RAY).reshape(-1), flags, want_bary=True,
                               want_stats=True)
    h = rq.hits_numpy(hits)
    assert h.tobytes() == oh.tobytes()
    assert bary.cpu().numpy().reshape(-1).tobytes() == ob.tobytes()
    assert rq.stats_numpy(stats).tobytes() == os_.tobytes()
    # the lean variant (no barycentrics / stats) returns the same hits
    h2, _, _ = rq.trace(ctx, b, rays, flags=flags)
    assert rq.hits_numpy(h2).tobytes() == oh.tobytes()
    # rays leave the 2x2 footprint at the sides: about 72 % hit
    assert 0.6 < h["hit"].mean() < 0.85
    b.destroy()


def test_trace_larger_mesh_vs_oracle(ctx):
    pos, idx = rq.scene_grid(512, 512, seed=1)
    b = rq.Bvh.build(ctx, torch.from_numpy(pos).cuda(), torch.from_numpy(idx.view(np.int32)).cuda())
    n2, tr, n4, perm = b.download()
    rays_np = rq.scene_rays_down(200000, spread=0.6, seed=3)
    for flags in (0, 1):
        hits, _, _ = rq.trace(ctx, b, torch.from_numpy(rays_np).cuda(), flags=flags)
        oh, _, _ = O.trace_bvh4(n4, tr, perm, rays_np.view(O.RAY).reshape(-1), flags)
        assert rq.hits_numpy(hits).tobytes() == oh.tobytes()
    b.destroy()


@pytest.mark.parametrize("flags", [rq.RQ_TRI_MT, rq.RQ_TRI_WATERTIGHT])
def test_closest_hit_vs_reference_pipeline(ctx, flags, have_ref):
    if not have_ref:
        pytest.skip("needs oracle/_ref (the reference's SoftwareBVH)")
    pos, idx, b = build_plain(ctx)
    n = 1 << 20
    rays_np = rq.scene_rays_down(n, seed=7)
    hits, _, _ = rq.trace(ctx, b, torch.from_numpy(rays_np).cuda(), flags=flags)
    ours = rq.hits_numpy(hits)
    n2r, trr, n4r = O.ref_build(pos.reshape(-1), idx.reshape(-1))
    perm_r = O.recover_perm(trr, pos.reshape(-1), idx.reshape(-1))
    st, rh = O.trace_ref_bvh4(n4r, trr, rays_np.view(O.RAY).reshape(-1))
    ref_prim = np.where(rh["hit"] == 1, perm_r[np.minimum(rh["primitive_id"], len(perm_r) - 1)], 0xFFFFFFFF)
    dis, kinds, unexplained = graze_report(pos, idx, rays_np, ours["hit"], ours["primitive_id"], rh["hit"], ref_prim,
                                           ours_t=ours["t"], ref_t=rh["t"])
    assert len(unexplained) == 0, unexplained[:10]
    assert len(dis) < 1e-5 * n, (len(dis), kinds)
    both = (ours["hit"] == 1) & (rh["hit"] == 1) & (ours["primitive_id"] == ref_prim)
    assert_t_close(ours["t"], rh["t"], both)
    b.destroy()


def test_any_hit_flags_vs_reference_pipeline(ctx, have_ref):
    if not have_ref:
        pytest.skip("needs oracle/_ref")
    pos, idx, b = build_plain(ctx)
    rays_np = rq.scene_rays_down(1 << 18, spread=0.5, seed=9)
    rays_np[:, 7] = 2.0  # shorter rays: part of them stop before the surface
    hits, _, _ = rq.trace(ctx, b, torch.from_numpy(rays_np).cuda(), flags=rq.RQ_TRACE_ANY | rq.RQ_TRI_MT)
    ours = rq.hits_numpy(hits)
    n2r, trr, n4r = O.ref_build(pos.reshape(-1), idx.reshape(-1))
    _, rh = O.trace_ref_bvh4(n4r, trr, rays_np.view(O.RAY).reshape(-1))
    mism = int((ours["hit"] != rh["hit"]).sum())
    assert mism < 1e-5 * len(rays_np) + 1
    assert 0.05 < ours["hit"].mean() < 0.95
    b.destroy()


def test_procedural_rays_bit_exact(ctx):
    for coh in (1, 0):
        g = rq.gen_rays_procedural(ctx, [0, 50, -45], [0, 0, 5], 100000, coh)
        o = O.gen_rays_procedural([0, 50, -45], [0, 0, 5], 100000, coh)
        assert g.cpu().numpy().tobytes() == o.tobytes()


def ref_fixture():
    d = np.load(os.path.join(GOLDEN, "ref_terrain1000.npz"))
    return d, d["nodes2"].view(O.BVH2_NODE), d["tris"].view(O.TRIANGLE), d["nodes4"].view(O.BVH4_NODE)


def test_reference_bvh4_semantics_bit_exact(ctx):
    d, n2, tr, n4 = ref_fixture()
    t_n4 = torch.from_numpy(d["nodes4"].copy()).cuda()
    t_tr = torch.from_numpy(d["tris"].copy()).cuda()
    for coh in (1, 0):
        rays = rq.gen_rays_procedural(ctx, [0, 50, -45], [0, 0, 5], 1 << 18, coh)
        st, hits = rq.trace_ref_bvh4(ctx, t_n4, t_tr, rays)
        ost, oh = O.trace_ref_bvh4(n4, tr, rq.rays_numpy(rays))
        assert rq.stats_numpy(st).tobytes() == ost.tobytes()
        assert rq.hits_numpy(hits).tobytes() == oh.tobytes()


def test_reference_bvh2_semantics_bit_exact(ctx):
    d, n2, tr, n4 = ref_fixture()
    t_n2 = torch.from_numpy(d["nodes2"].copy()).cuda()
    t_tr = torch.from_numpy(d["tris"].copy()).cuda()
    for coh, eps in ((1, 0.001), (0, 0.01)):
        rays = rq.gen_rays_procedural(ctx, [0, 50, -45], [0, 0, 5], 1 << 18, coh)
        f = rq.trace_ref_bvh2(ctx, t_n2, t_tr, rays, eps).cpu().numpy().astype(np.uint32)
        of = O.trace_ref_bvh2(n2, tr, rq.rays_numpy(rays), eps)
        assert np.array_equal(f, of)


def test_published_statistics_on_gpu(ctx):
    # results/exp0_ray_stats.csv, 968 triangles x 1,048,576 procedural rays
    g = json.load(open(os.path.join(GOLDEN, "exp0_ray_stats.json")))
    rows = {(r["tris"], r["pattern"]): r for r in g["rows"]}
    d, n2, tr, n4 = ref_fixture()
    t_n4 = torch.from_numpy(d["nodes4"].copy()).cuda()
    t_tr = torch.from_numpy(d["tris"].copy()).cuda()
    for pattern, coh in (("Coherent", 1), ("Incoherent", 0)):
        rays = rq.gen_rays_procedural(ctx, [0, 50, -45], [0, 0, 5], 1 << 20, coh)
        st = rq.stats_numpy(rq.trace_ref_bvh4(ctx, t_n4, t_tr, rays)[0])
        ref = rows[(968, pattern)]
        assert abs(int(st["hit"].sum()) - ref["sw_hit_pct"] / 100 * 1048576) <= 12
        assert abs(st["box_tests"].mean() / ref["box_tests"] - 1) < 0.025
        assert abs(st["tri_tests"].mean() / ref["tri_tests"] - 1) < 0.025


def test_import4_reference_tree_trace(ctx):
    # the reference's own 4-wide tree, imported, traced by the engine kernel
    d, n2, tr, n4 = ref_fixture()
    perm = O.recover_perm(tr, d["pos"], d["idx"])
    b = rq.Bvh.import4(ctx, torch.from_numpy(d["nodes4"].copy()).cuda(), torch.from_numpy(d["tris"].copy()).cuda(),
                       torch.from_numpy(perm.view(np.int32)).cuda())
    rays = rq.gen_rays_procedural(ctx, [0, 50, -45], [0, 0, 5], 1 << 17, 0)
    rn = rq.rays_numpy(rays)
    for flags in (0, 1, 2, 3):
        h, _, _ = rq.trace(ctx, b, rays, flags=flags)
        oh, _, _ = O.trace_bvh4(n4, tr, perm, rn, flags)
        assert rq.hits_numpy(h).tobytes() == oh.tobytes()
    b.destroy()


def test_empty_and_degenerate_rays(ctx):
    pos, idx, b = build_plain(ctx)
    n2, tr, n4, perm = b.download()
    r = rq.scene_rays_down(64, seed=1)
    r[0, 4:7] = [0, 0, -1]          # axis-aligned direction (zero components)
    r[1, 7] = r[1, 3]               # tmax == tmin: empty interval
    r[2, 4:7] = [1, 0, 0]           # parallel to the height field
    r[3, 0:3] = [5, 5, 2]           # outside the mesh
    hits, _, _ = rq.trace(ctx, b, torch.from_numpy(r).cuda(), flags=0)
    oh, _, _ = O.trace_bvh4(n4, tr, perm, r.view(O.RAY).reshape(-1), 0)
    h = rq.hits_numpy(hits)
    assert h.tobytes() == oh.tobytes()
    assert h["hit"][1] == 0 and h["hit"][3] == 0 and h["hit"][0] == 1
    # zero rays is a no-op
    z = torch.empty((0, 8), dtype=torch.float32, device="cuda")
    rq.trace(ctx, b, z)
    b.destroy()
