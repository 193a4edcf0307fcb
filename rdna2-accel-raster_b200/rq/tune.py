"""Launch-shape table of the batched form, written by the autotuner.

`python -m rq.tune --out FILE` builds the batched workload (512 deforming
grids, 4,096 any-hit + 4,096 closest-hit rays per mesh), runs
rq_batch_autotune on it (every build block size x blocks per SM, every
traversal block size x refill chunk x register cap, median of 5 timed runs
each) and writes the chosen shapes and all measured candidates as JSON.  The
committed copy (tuning_b200.json beside this file) is what the benchmark and
callers load with `lookup`; a workload missing from it is tuned at run time.
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
    args = ap.parse_args()
    ctx = rq.Context(0)
    sizes = W.batched_sizes(512, seed=2)
    pos, idx, descs = W.batched_meshes(sizes, seed=2)
    rays, mesh, flags = W.batched_rays(descs, 4096, 4096, seed=2)
    p = torch.from_numpy(pos).cuda()
    i = torch.from_numpy(idx.view(np.int32)).cuda()
    r = torch.from_numpy(rays).cuda()
    m = torch.from_numpy(mesh.view(np.int32)).cuda()
    f = torch.from_numpy(flags.view(np.int32)).cuda()
    shape, trials = tune_batched(ctx, descs, p, i, r, m, f, args.reps)
    table = load(args.out) if os.path.exists(args.out) else {}
    table.setdefault("device", torch.cuda.get_device_name(0))
    table.setdefault("entries", {})
    table["entries"][workload_key(descs, 8192)] = {
        "workload": "batched: 512 grids (seed 2), 4,096 any-hit + 4,096 closest-hit rays per mesh",
        "shape": {k: shape[k] for k in rq.Batch.TUNING_KEYS},
        "build_ms": shape["build_ms"], "trace_ms": shape["trace_ms"],
        "trials": trials,
    }
    with open(args.out, "w") as fo:
        json.dump(table, fo, indent=1)
    print(json.dumps({"shape": table["entries"][workload_key(descs, 8192)]["shape"],
                      "build_ms": shape["build_ms"], "trace_ms": shape["trace_ms"]}))


if __name__ == "__main__":
    main()
