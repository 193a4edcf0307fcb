"""Launch-shape table written by the autotuner.

`python -m rq.tune --out FILE` times, on the device:
  - the 1080p shadows + AO frame's traversal (rq_render_shadow_ao) in every
    block size x refill chunk x register budget, with and without staged top
    levels and speculative traversal, then the refill threshold, then the
    in-loop refill shapes x refill threshold x leaf batch (median of 5 runs
    each);
  - the batched workload (512 deforming grids, 4,096 any-hit + 4,096
    closest-hit rays per mesh) through rq_batch_autotune: every build block
    size x blocks per SM, every traversal block size x chunk x register budget;
and writes the chosen shapes and every measured candidate as JSON.  The
committed copy (tuning_b200.json beside this file) is what the benchmark and
callers load with `lookup` / `lookup_shadow`; a workload missing from it is
tuned at run time.
"""
import argparse
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE = os.path.join(HERE, "tuning_b200.json")


def workload_key(descs, rays_per_mesh):
    """Key of a batched workload: mesh count, total and largest triangle count,
    rays per mesh."""
    tris = [d[3] for d in descs]
    return f"meshes={len(descs)},tris={sum(tris)},max={max(tris)},rays_per_mesh={rays_per_mesh}"


def load(path=TABLE):
    if not os.path.exists(path):
        return {}
    with open(path) as f:
        return json.load(f)


def lookup(key, path=TABLE):
    """The committed shape for a workload key, or None."""
    e = load(path).get("entries", {}).get(key)
    return e["shape"] if e else None


# (threads, refill chunk, register budget, staged top levels, speculative)
SHADE_SHAPES = ([(t, c, r, 0, 0) for t in (64, 128, 256) for c in (32, 64) for r in (0, 64, 80)]
                + [(t, c, 80, 4, 0) for t in (64, 128, 256) for c in (32, 64)]
                + [(t, c, 80, 0, 1) for t in (64, 128, 256) for c in (32, 64)]
                + [(t, c, 72, 0, s) for t in (64, 128) for c in (32, 64) for s in (0, 1)]
                + [(t, 64, 64, 0, 1) for t in (64, 128, 256)])
# second stage: the refill threshold (idle lanes out of 32), with and without
# speculation, for the fastest block size / chunk / register budgets
REFILL_MINS = (4, 8, 12, 16, 20, 24)
REFILL_TOP = 4
# third stage: in-loop refill (speculative shapes): (threads, chunk, register
# budget) x refill threshold x leaf batch
INLOOP_SHAPES = [(64, 32, 64), (64, 64, 64), (128, 32, 64), (128, 64, 64), (256, 32, 64), (256, 64, 64),
                 (128, 64, 72), (256, 64, 72)]
INLOOP_REFILL = (4, 8, 12, 16)
INLOOP_LEAF_BATCH = (4, 8, 12, 16, 24)
SHAPE_KEYS = ("threads", "chunk", "reg_cap", "top_levels", "speculative", "refill_min", "leaf_batch")


def shadow_key(ntri, params, sah=False):
    return (f"shadow_ao:tris={ntri},{params.width}x{params.height},lights={params.num_lights},"
            f"ao_spp={params.ao_spp}" + (",build=sah" if sah else ""))


def tune_shadow(ctx, bvh, gbuf, params, reps=5):
    """Time rq_render_shadow_ao in every launch shape (median of `reps` after
    one warm-up run) and keep the fastest on the context.  Returns (shape,
    trials)."""
    import statistics
    import torch
    import rq
    n = params.width * params.height
    mask = torch.empty(n, dtype=torch.int32, device="cuda")
    ao = torch.empty(n, dtype=torch.float32, device="cuda")
    trials = []

    def timed(t, c, r, top, spec, refill, leaf_batch=0):
        ctx.set_trace_tuning(t, c, r, top, spec, refill, leaf_batch)
        rq.render_shadow_ao(ctx, bvh, gbuf, params, mask, ao)
        ms = []
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            rq.render_shadow_ao(ctx, bvh, gbuf, params, mask, ao)
            b.record()
            b.synchronize()
            ms.append(a.elapsed_time(b))
        ctx.sync_check()
        trials.append({"threads": t, "chunk": c, "reg_cap": r, "top_levels": top, "speculative": spec,
                       "refill_min": refill, "leaf_batch": leaf_batch, "ms": statistics.median(ms)})

    for t, c, r, top, spec in SHADE_SHAPES:
        timed(t, c, r, top, spec, 1)
    bases = []
    for s in sorted(trials, key=lambda x: x["ms"]):
        b = (s["threads"], s["chunk"], s["reg_cap"], s["top_levels"])
        if b not in bases:
            bases.append(b)
    for t, c, r, top in bases[:REFILL_TOP]:
        for spec in (0, 1):
            if (t, c, r, top, spec) not in SHADE_SHAPES:
                continue
            for refill in REFILL_MINS:
                timed(t, c, r, top, spec, refill)
    for t, c, r in INLOOP_SHAPES:
        for refill in INLOOP_REFILL:
            for lb in INLOOP_LEAF_BATCH:
                timed(t, c, r, 0, 1, refill, lb)
    best = min(trials, key=lambda x: x["ms"])
    ctx.set_trace_tuning(**{k: best.get(k, 0) for k in SHAPE_KEYS})
    return {k: best.get(k, 0) for k in SHAPE_KEYS}, trials


CAMERA_REFILL = (1, 4, 8, 16)
CAMERA_LEAF_BATCH = (4, 8, 16, 32)


def tune_camera(ctx, bvh, cam, reps=5):
    """Time rq_render_gbuffer on one ray per thread and on the refilling
    engine (refill threshold x leaf batch); keep the fastest.  Returns
    (schedule, trials)."""
    import statistics
    import torch
    import rq
    gbuf = torch.empty((cam.width * cam.height, 8), dtype=torch.int32, device="cuda")
    trials = []

    def timed(engine, refill, lb):
        ctx.set_camera_tuning(engine, refill, lb)
        rq.render_gbuffer(ctx, bvh, cam, gbuf)
        ms = []
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            rq.render_gbuffer(ctx, bvh, cam, gbuf)
            b.record()
            b.synchronize()
            ms.append(a.elapsed_time(b))
        ctx.sync_check()
        trials.append({"engine": engine, "refill_min": refill, "leaf_batch": lb, "ms": statistics.median(ms)})

    timed(0, 1, 32)
    for refill in CAMERA_REFILL:
        for lb in CAMERA_LEAF_BATCH:
            timed(1, refill, lb)
    best = min(trials, key=lambda x: x["ms"])
    keys = ("engine", "refill_min", "leaf_batch")
    ctx.set_camera_tuning(**{k: best[k] for k in keys})
    return {k: best[k] for k in keys}, trials


def lookup_camera(key, path=TABLE):
    e = load(path).get("camera", {}).get(key)
    return e["shape"] if e else None


def lookup_shadow(key, path=TABLE):
    e = load(path).get("shadow", {}).get(key)
    return e["shape"] if e else None


def tune_batched(ctx, descs, pos, idx, rays, mesh, flags, reps=5):
    import rq
    b = rq.Batch(ctx, descs)
    shape, trials = b.autotune(pos, idx, rays, mesh, flags, reps=reps)
    b.destroy()
    return shape, trials


def main():
    import numpy as np
    import torch
    import rq
    from rq import workloads as W

    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--only", choices=["shadow", "batched"], help="tune one workload, keep the other's entry")
    ap.add_argument("--build", choices=["lbvh", "sah"], default="sah", help="the frame's build for the shadow tuning")
    args = ap.parse_args()
    ctx = rq.Context(0)
    table = load(args.out) if os.path.exists(args.out) else {}
    table.setdefault("device", torch.cuda.get_device_name(0))
    if args.only != "batched":
        tune_frame(ctx, table, args)
    if args.only != "shadow":
        tune_batch_entry(ctx, table, args)
    with open(args.out, "w") as fo:
        json.dump(table, fo, indent=1)


def tune_frame(ctx, table, args):
    import numpy as np
    import torch
    import rq
    from rq import workloads as W
    # the 1080p shadows + AO frame
    pos, idx = W.shadow_mesh()
    p = torch.from_numpy(pos).cuda()
    i = torch.from_numpy(idx.view(np.int32)).cuda()
    sah = args.build == "sah"
    bvh = rq.Bvh.build(ctx, p, i, sah=sah)
    params = W.shadow_params()
    gbuf = rq.render_gbuffer(ctx, bvh, W.shadow_camera())
    shape, trials = tune_shadow(ctx, bvh, gbuf, params, args.reps)
    table.setdefault("shadow", {})[shadow_key(len(idx), params, sah)] = {
        "workload": ("1080p shadows + AO frame (2.5M-triangle grid, seed 1, 16 lights, 1 AO ray)"
                     + (", LBVH with SAH-rebuilt subtrees" if sah else ", LBVH")),
        "shape": shape, "ms": min(t["ms"] for t in trials), "trials": trials}
    print(json.dumps({"shadow_shape": shape, "ms": min(t["ms"] for t in trials)}))
    cshape, ctrials = tune_camera(ctx, bvh, W.shadow_camera(), args.reps)
    table.setdefault("camera", {})[shadow_key(len(idx), params, sah)] = {
        "workload": "1080p frame's primary rays (the shadows + AO frame's camera)",
        "shape": cshape, "ms": min(t["ms"] for t in ctrials), "trials": ctrials}
    print(json.dumps({"camera_schedule": cshape, "ms": min(t["ms"] for t in ctrials)}))
    bvh.destroy()


def tune_batch_entry(ctx, table, args):
    import numpy as np
    import torch
    import rq
    from rq import workloads as W
    sizes = W.batched_sizes(512, seed=2)
    pos, idx, descs = W.batched_meshes(sizes, seed=2)
    rays, mesh, flags = W.batched_rays(descs, 4096, 4096, seed=2)
    p = torch.from_numpy(pos).cuda()
    i = torch.from_numpy(idx.view(np.int32)).cuda()
    r = torch.from_numpy(rays).cuda()
    m = torch.from_numpy(mesh.view(np.int32)).cuda()
    f = torch.from_numpy(flags.view(np.int32)).cuda()
    shape, trials = tune_batched(ctx, descs, p, i, r, m, f, args.reps)
    table.setdefault("entries", {})
    table["entries"][workload_key(descs, 8192)] = {
        "workload": "batched: 512 grids (seed 2), 4,096 any-hit + 4,096 closest-hit rays per mesh",
        "shape": {k: shape[k] for k in rq.Batch.TUNING_KEYS},
        "build_ms": shape["build_ms"], "trace_ms": shape["trace_ms"],
        "trials": trials,
    }
    print(json.dumps({"shape": table["entries"][workload_key(descs, 8192)]["shape"],
                      "build_ms": shape["build_ms"], "trace_ms": shape["trace_ms"]}))


if __name__ == "__main__":
    main()
