#!/usr/bin/env python
"""Benchmark of the ray-query engine on one B200 (or N replicas).

Default workload — the 1080p shadows + AO frame: a 2,499,848-triangle
height-field grid (1118x1118 quads, seed 1), per step a full LBVH rebuild
(Morton codes, onesweep radix sort, Karras hierarchy, refit, 4-wide
collapse), 2,073,600 primary closest-hit rays into a G-buffer, then 16
any-hit shadow rays and 1 cosine AO ray per pixel generated and traced in one
kernel.  value = rays traced per step / step time (Mrays/s); the per-frame
build rate (Mtris/s) and the any-hit rate are reported beside it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun) every rank runs an independent replica of the frame:
the path has no exchange step, so there is no collective on the data path;
the barrier and the max-over-ranks step time use the process group only.

--impl reference times the reference's CPU implementation of the path on the
host cores: the reference's own SoftwareBVH::build + SoftwareBVH4::fromBVH2
(compiled from its sources into oracle/_ref, single-threaded as written) and
the CPU statement of the frame's rays (the reference has no CPU traversal)
on all host threads, over a bounded pixel sample, projected to the frame.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "rdna2-accel-raster_b200"))

WIDTH, HEIGHT = 1920, 1080
METRIC = "Mrays/s + BVH Mtris/s on 1 B200; p50/p99 request latency batched vs plain"
# kernels launched by one step of the frame: the build — centroids, morton,
# hist, hist_scan, 4 onesweep passes, karras, then leaves, the top refit,
# scan, emit (plain LBVH) or per-position boxes, SAH roots, the node queue
# above the block size, the block subtrees, scan, emit (SAH subtrees), then
# collapse: 14 or 16 — then G-buffer, shadow/AO and the shade finish (3)
BUILD_KERNELS = {"lbvh": 14, "sah": 16}
FRAME_KERNELS = 3


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-sample", type=int, default=200000, help="pixels in the CPU baseline sample")
    ap.add_argument("--build", choices=["lbvh", "sah"], default="sah",
                    help="the frame's per-step build: plain LBVH, or LBVH with SAH-rebuilt subtrees (RQ_BUILD_SAH)")
    ap.add_argument("--serve-catalogue", type=int, default=256,
                    help="meshes in the serving catalogue (fewer for a small profiling case)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the visibility / batched / serving workloads")
    ap.add_argument("--extra", choices=["visibility", "batched", "serving", "radv"],
                    help="run only this workload (--steps frames / steps / x50 ms of arrivals) and print its JSON")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # nvidia-smi takes longer to start than a short timed region lasts:
            # wait for its first sample, then drop it (taken before the load)
            t0 = time.time()
            while not self.lines and time.time() - t0 < 5.0 and self.proc.poll() is None:
                time.sleep(0.01)
            self.skip = len(self.lines)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines[getattr(self, "skip", 0):]:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    elif torch.cuda.is_available():  # (the CPU reference arm runs without one)
        torch.cuda.set_device(0)
    return world, rank, local, pg


def barrier(pg):
    if pg is not None:
        pg.barrier()


def _pg_device(pg):
    """Tensor device of the process group's backend (gloo: CPU, nccl: GPU)."""
    return "cpu" if pg.get_backend() == "gloo" else "cuda"


def max_over_ranks(pg, x):
    import torch
    if pg is None:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=_pg_device(pg))
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(pg, x):
    import torch
    if pg is None:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=_pg_device(pg))
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


def replica_line(pg, rank, world, ms_local, rays_local):
    """Whole-job figures of N independent replicas: the step time is the
    slowest rank's, the work is every rank's; rank 0 reports."""
    ms = max_over_ranks(pg, ms_local)
    rays = sum_over_ranks(pg, rays_local)
    return {"ms_per_step": ms, "value": rays / (ms * 1e-3) / 1e6, "n_gpus": world} if rank == 0 else None


def read_profile(name, key):
    """A `key: value` figure from a committed ncu summary (profiles/<name>.md),
    e.g. traffic_bytes_per_launch (DRAM read + write bytes of one launch)."""
    path = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(path):
        return None
    for ln in open(path):
        if ln.strip().startswith(key + ":"):
            try:
                return float(ln.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


def read_traffic(name):
    return read_profile(name, "traffic_bytes_per_launch")


def frame_config(world):
    """The workload description both arms print (the measured counts of a
    frame go to the line's `frame` key)."""
    return {
        "workload": ("1080p shadows + AO: 2,499,848-triangle grid (1118x1118 quads, seed 1), per-frame BVH "
                     "rebuild, 1920x1080 primary rays, 16 any-hit shadow rays + 1 SPP AO (tmax 0.5) per pixel"),
        "triangles": 2499848, "width": WIDTH, "height": HEIGHT, "lights": 16, "ao_spp": 1,
        "l2": "inputs larger than L2: the per-step rebuild writes ~0.2 GB of nodes and triangles",
        "parallelism": "replicas" if world > 1 else "single",
    }


def cpu_frame_sample(O, pos, idx, cam, params, sample, threads, seed, gfull):
    """One step of the CPU path of the frame: the reference's own
    SoftwareBVH::build + SoftwareBVH4::fromBVH2 on the full mesh
    (oracle/_ref, single-threaded as written; Oracle B where the reference
    library is absent), then the frame's primary, shadow and AO rays at
    `sample` random pixels traced on `threads` host threads by the CPU
    statement of the traversal (the reference has no CPU traversal).
    Returns the measured times and the frame throughput they project to."""
    import numpy as np
    t0 = time.perf_counter()
    if O.have_ref():
        n2, tr, n4 = O.ref_build(pos.reshape(-1), idx.reshape(-1))
        kind = "reference"
    else:
        b = O.lbvh_build(pos.reshape(-1), idx.reshape(-1))
        n2, tr, n4 = b["nodes2"], b["tris"], b["nodes4"]
        kind = "port"
    build_s = time.perf_counter() - t0
    rng = np.random.default_rng(seed)
    pixels = np.sort(rng.choice(WIDTH * HEIGHT, sample, replace=False)).astype(np.uint32)
    t0 = time.perf_counter()
    g = O.render_gbuffer(n4, tr, None, cam, pixels)
    gfull[pixels] = g
    _, _, sec_rays = O.render_shadow_ao(n4, tr, gfull, params, pixels)
    trace_s = time.perf_counter() - t0
    rays_sample = sample + sec_rays
    npix = WIDTH * HEIGHT
    frame_rays = rays_sample * npix / sample
    frame_s = build_s + trace_s * npix / sample
    return dict(value=frame_rays / frame_s / 1e6, build_s=build_s, trace_s=trace_s, rays_sample=rays_sample,
                frame_s=frame_s, frame_rays=frame_rays, kind=kind, cores=threads, triangles=len(idx),
                build_mtris=len(idx) / build_s / 1e6, trace_mrays=rays_sample / trace_s / 1e6)


def cpu_inputs():
    """The frame's inputs made by the oracle's generators alone (no engine
    library is loaded): positions, indices, camera, shading parameters."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as O
    return (O,) + O.shadow_frame_inputs(WIDTH, HEIGHT)


def cpu_sample_text(r, sample):
    return (f"per step: reference SoftwareBVH::build + fromBVH2 on the full mesh ({r['build_s']:.2f} s, 1 thread "
            f"as written, {r['build_mtris']:.2f} Mtris/s) + the frame's primary, shadow and AO rays at {sample} "
            f"random pixels ({r['rays_sample']} rays, {r['trace_mrays']:.2f} Mrays/s on {r['cores']} threads); "
            f"value = the frame's rays / (build time + the sample's trace time scaled to {WIDTH}x{HEIGHT})")


def run_reference(args, world, rank, pg):
    """The reference arm: the CPU implementation of the path on the host
    cores, rank 0 only.  Each step is measured whole (reference build + the
    sampled rays); the frame throughput is projected from the step's two
    measured parts, and the projection is stated in its own key."""
    if rank != 0:
        return
    import numpy as np
    O, pos, idx, cam, params = cpu_inputs()
    threads = os.cpu_count() or 1
    gfull = np.zeros(WIDTH * HEIGHT, O.GBUFFER_PX)
    step_ms, vals, frame_ms, last = [], [], [], None
    for s in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        r = cpu_frame_sample(O, pos, idx, cam, params, args.cpu_sample, threads, 123 + s, gfull)
        dt = time.perf_counter() - t0
        if s >= args.warmup:
            step_ms.append(dt * 1e3)
            vals.append(r["value"])
            frame_ms.append(r["frame_s"] * 1e3)
            last = r
    v = statistics.median(vals)
    pct = (lambda q: float(np.percentile(vals, q)))
    line = {
        "impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": "Mrays/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(statistics.median(step_ms), 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": frame_config(world),
        "projection": {"frame_ms": round(statistics.median(frame_ms), 1),
                       "build_ms": round(1e3 * last["build_s"], 1),
                       "sample_trace_ms": round(1e3 * last["trace_s"], 1),
                       "sample_pixels": args.cpu_sample, "frame_pixels": WIDTH * HEIGHT,
                       "frame_rays": round(last["frame_rays"]),
                       "method": ("ms_per_step is the measured step (full build + sampled rays); value = frame "
                                  "rays / (measured build + measured sample trace x frame pixels / sample pixels)")},
        "cpu_baseline": {"value": round(v, 3), "unit": "Mrays/s", "cores": threads, "kind": last["kind"],
                         "sample": cpu_sample_text(last, args.cpu_sample),
                         "p5": round(pct(5), 3), "p50": round(pct(50), 3), "p95": round(pct(95), 3)},
        "e2e": {"value": round(v, 3), "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, world, rank, local, pg):
    import numpy as np
    import torch
    import rq
    from rq import workloads as W

    ctx = rq.Context(local)
    sah = args.build == "sah"
    pos, idx = W.shadow_mesh()
    ntri = len(idx)
    cam = W.shadow_camera()
    params = W.shadow_params()
    npx = WIDTH * HEIGHT
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)

    # device-resident inputs and outputs
    p_d = torch.from_numpy(pos).to(dev)
    i_d = torch.from_numpy(idx.view(np.int32)).to(dev)
    gbuf = torch.empty((npx, 8), dtype=torch.int32, device=dev)
    mask = torch.empty(npx, dtype=torch.int32, device=dev)
    ao = torch.empty(npx, dtype=torch.float32, device=dev)
    counters = torch.zeros(4, dtype=torch.int64, device=dev)
    bvh = rq.Bvh.build(ctx, p_d, i_d, sah=sah)

    def step(count=None):
        rq.Bvh.build(ctx, p_d, i_d, into=bvh, sah=sah)
        rq.render_gbuffer(ctx, bvh, cam, gbuf)
        rq.render_shadow_ao(ctx, bvh, gbuf, params, mask, ao, count)

    # ray count of one frame (deterministic): primary + shadow + AO
    counters.zero_()
    step(counters)
    ctx.sync_check()
    sec_rays = int(counters[0].item())
    frame_rays = npx + sec_rays
    hits = int((gbuf[:, 3] != 0).sum().item())

    # launch shape of the shadow/AO traversal: committed autotuner table,
    # else tuned now (untimed)
    from rq import tune as T
    skey = T.shadow_key(len(idx), params, sah)
    sshape = T.lookup_shadow(skey)
    if sshape is not None:
        ctx.set_trace_tuning(**sshape)
        shade_tuning = {"source": "committed table rq/tuning_b200.json", **sshape}
    else:
        sshape, strials = T.tune_shadow(ctx, bvh, gbuf, params, reps=3)
        shade_tuning = {"source": f"autotuned in this run ({len(strials)} shapes timed)", **sshape}
    cshape = T.lookup_camera(skey)
    if cshape is not None:
        ctx.set_camera_tuning(**cshape)
        camera_tuning = {"source": "committed table rq/tuning_b200.json", **cshape}
    else:
        camera_tuning = {"source": "default (one ray per thread)", **ctx.camera_tuning()}

    # node / triangle tests per any-hit ray, for the algorithmic bytes
    cp = rq.shade_params(WIDTH, HEIGHT, W.shadow_lights(16), ao_spp=1, ao_tmax=0.5,
                         flags=rq.RQ_SHADE_COUNT_TESTS)
    counters.zero_()
    rq.render_shadow_ao(ctx, bvh, gbuf, cp, mask, ao, counters)
    ctx.sync_check()
    c = counters.cpu().numpy()
    v_node = c[1] / 4.0 / max(1, c[0])
    v_tri = c[2] / max(1, c[0])
    info = bvh.info()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)

    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4 * args.steps + 2)]
    barrier(pg)
    torch.cuda.synchronize(dev)
    with ClockSampler(local) as clk:
        ev[0].record(stream)
        for s in range(args.steps):
            e0, e1, e2, e3 = ev[1 + 4 * s: 5 + 4 * s]
            e0.record(stream)
            rq.Bvh.build(ctx, p_d, i_d, into=bvh, sah=sah)
            e1.record(stream)
            rq.render_gbuffer(ctx, bvh, cam, gbuf)
            e2.record(stream)
            rq.render_shadow_ao(ctx, bvh, gbuf, params, mask, ao, None)
            e3.record(stream)
        ev[-1].record(stream)
        torch.cuda.synchronize(dev)
    barrier(pg)
    ctx.sync_check()
    total_ms = ev[0].elapsed_time(ev[-1])
    build_ms = [ev[1 + 4 * s].elapsed_time(ev[2 + 4 * s]) for s in range(args.steps)]
    prim_ms = [ev[2 + 4 * s].elapsed_time(ev[3 + 4 * s]) for s in range(args.steps)]
    shade_ms = [ev[3 + 4 * s].elapsed_time(ev[4 + 4 * s]) for s in range(args.steps)]
    agg = replica_line(pg, rank, world, total_ms / args.steps, frame_rays)
    ms_step = agg["ms_per_step"] if agg else total_ms / args.steps
    value = agg["value"] if agg else 0.0

    # end to end through the C ABI with host buffers: H2D of the mesh from
    # pinned memory, the frame, D2H of the light masks and AO values
    pos_h = torch.from_numpy(pos).pin_memory()
    idx_h = torch.from_numpy(idx.view(np.int32)).pin_memory()
    mask_h = torch.empty(npx, dtype=torch.int32).pin_memory()
    ao_h = torch.empty(npx, dtype=torch.float32).pin_memory()
    h2d = pos_h.numel() * 4 + idx_h.numel() * 4
    d2h = mask_h.numel() * 4 + ao_h.numel() * 4

    def e2e_step():
        p_d.copy_(pos_h, non_blocking=True)
        i_d.copy_(idx_h, non_blocking=True)
        step()
        mask_h.copy_(mask, non_blocking=True)
        ao_h.copy_(ao, non_blocking=True)

    for _ in range(max(3, args.warmup)):
        e2e_step()
    torch.cuda.synchronize(dev)
    barrier(pg)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(args.steps):
        e2e_step()
    b.record(stream)
    torch.cuda.synchronize(dev)
    barrier(pg)
    e2e_ms = max_over_ranks(pg, a.elapsed_time(b) / args.steps)
    e2e_value = sum_over_ranks(pg, frame_rays) / (e2e_ms * 1e-3) / 1e6
    serial_mask, serial_ao = mask_h.clone(), ao_h.clone()

    # the same calls with the copies overlapped, as a streaming caller runs
    # them: two device sets of inputs and results; on a copy stream, frame
    # f+1's mesh upload and frame f's result download run while the compute
    # stream works on the next frame.  Every copy stays inside the timed region.
    cs = torch.cuda.Stream(dev)
    p2, i2 = [p_d, torch.empty_like(p_d)], [i_d, torch.empty_like(i_d)]
    m2, a2 = [mask, torch.empty_like(mask)], [ao, torch.empty_like(ao)]

    def pipelined(n):
        up = [torch.cuda.Event(), torch.cuda.Event()]
        used, out = [None, None], [None, None]
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        cs.wait_stream(stream)

        def upload(f):
            k = f % 2
            with torch.cuda.stream(cs):
                if used[k] is not None:
                    cs.wait_event(used[k])  # the build that read this set is done
                p2[k].copy_(pos_h, non_blocking=True)
                i2[k].copy_(idx_h, non_blocking=True)
                up[k].record(cs)

        upload(0)
        for f in range(n):
            k = f % 2
            if f + 1 < n:
                upload(f + 1)
            stream.wait_event(up[k])
            if out[k] is not None:
                stream.wait_event(out[k])  # this result set has been downloaded
            rq.Bvh.build(ctx, p2[k], i2[k], into=bvh, sah=sah)
            used[k] = torch.cuda.Event()
            used[k].record(stream)
            rq.render_gbuffer(ctx, bvh, cam, gbuf)
            rq.render_shadow_ao(ctx, bvh, gbuf, params, m2[k], a2[k], None)
            done = torch.cuda.Event()
            done.record(stream)
            with torch.cuda.stream(cs):
                cs.wait_event(done)
                mask_h.copy_(m2[k], non_blocking=True)
                ao_h.copy_(a2[k], non_blocking=True)
                out[k] = torch.cuda.Event()
                out[k].record(cs)
        stream.wait_stream(cs)
        t1.record(stream)
        return t0, t1

    pipelined(max(3, args.warmup))
    torch.cuda.synchronize(dev)
    barrier(pg)
    t0, t1 = pipelined(args.steps)
    torch.cuda.synchronize(dev)
    barrier(pg)
    pipe_ms = max_over_ranks(pg, t0.elapsed_time(t1) / args.steps)
    pipe_value = sum_over_ranks(pg, frame_rays) / (pipe_ms * 1e-3) / 1e6
    pipe_equal = bool(torch.equal(mask_h, serial_mask) and torch.equal(ao_h, serial_ao))
    ctx.sync_check()

    # the AO consumer after the frame: depth from the G-buffer, then the
    # horizontal and vertical passes of the depth-aware blur (not part of the
    # frame step above; timed on its own)
    vp = rq.view_proj_of(cam)
    depth = rq.gbuffer_depth(ctx, gbuf, vp)
    tmp, blurred = torch.empty_like(ao), torch.empty_like(ao)

    def blur_chain():
        rq.gbuffer_depth(ctx, gbuf, vp, depth)
        rq.blur_ao(ctx, ao, depth, WIDTH, HEIGHT, 1, 0, 0.005, tmp)
        rq.blur_ao(ctx, tmp, depth, WIDTH, HEIGHT, 0, 1, 0.005, blurred)

    for _ in range(3):
        blur_chain()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(20):
        blur_chain()
    b.record(stream)
    torch.cuda.synchronize(dev)
    blur_ms = a.elapsed_time(b) / 20
    # compulsory bytes per pixel: G-buffer 32 B in + depth 4 B out, then per
    # pass AO and depth 4 + 4 B in and 4 B out (the other taps hit in cache)
    blur = {"workload": "AO depth + 2-pass bilateral blur at 1920x1080", "ms": round(blur_ms, 4),
            "gb_per_s_compulsory": round(npx * (36 + 2 * 12) / (blur_ms * 1e-3) / 1e9, 1)}

    # the reference's median-split topology (RQ_BUILD_MEDIAN) on the same
    # mesh: stream-ordered (one round of launches per possible tree level, no
    # host synchronisation), timed with CUDA events
    med = rq.Bvh.build(ctx, p_d, i_d, median=True)
    torch.cuda.synchronize(dev)
    med_ms = []
    for _ in range(5):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        rq.Bvh.build(ctx, p_d, i_d, median=True, into=med)
        b.record(stream)
        b.synchronize()
        med_ms.append(a.elapsed_time(b))
    ctx.sync_check()
    med_info = med.info()
    med.destroy()
    median_build = {"workload": "median-split build of the frame mesh (2,499,848 triangles) + 4-wide collapse",
                    "ms": round(min(med_ms), 2), "mtris_per_s": round(len(idx) / min(med_ms) / 1e3, 1),
                    "nodes2": med_info["num_nodes2"], "depth4": med_info["depth4"]}

    bvh.destroy()
    del p_d, i_d, gbuf, mask, ao, depth, tmp, blurred
    refbench = run_reference_benchmarks(ctx, dev) if not args.no_extra else None
    radv_build = run_radv_build(ctx, dev, load_peaks()) if not args.no_extra else None
    vis = run_visibility(ctx, dev, stream) if not args.no_extra else None
    batched = run_batched(ctx, dev) if not args.no_extra else None
    serving = run_serving(dev) if not args.no_extra else None

    if rank != 0:
        return
    peaks = load_peaks()
    hbm = peaks.get("hbm_gbs", 6650.0)
    shade_med = statistics.median(shade_ms)
    # algorithmic bytes of the shadow/AO launch: G-buffer read (32 B/pixel),
    # mask + AO written (8 B/pixel), per ray the 128-B nodes and 48-B
    # triangles its traversal visits (mean counts measured above)
    alg_bytes = npx * (32 + 8) + sec_rays * (128.0 * v_node + 48.0 * v_tri)
    achieved = alg_bytes / (shade_med * 1e-3) / 1e9
    # compulsory I/O alone: the G-buffer pixel in (32 B) and the result word out (8 B)
    comp_bytes = npx * (32 + 8)
    comp_gbs = comp_bytes / (shade_med * 1e-3) / 1e9
    traffic = read_traffic("k_shadow_ao_1080p.md")
    # what binds the kernel, from the same capture: instruction issue and L1
    binding = {k: read_profile("k_shadow_ao_1080p.md", k) for k in
               ("issue_active_frac", "l1tex_busy_frac", "lanes_per_instruction", "dram_frac")}
    clocks = clk.summary()
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        import numpy as np
        O, cpos, cidx, ccam, cparams = cpu_inputs()
        r = cpu_frame_sample(O, cpos, cidx, ccam, cparams, args.cpu_sample, os.cpu_count() or 1, 123,
                             np.zeros(WIDTH * HEIGHT, O.GBUFFER_PX))
        cpu = {"value": round(r["value"], 3), "unit": "Mrays/s", "cores": r["cores"], "kind": r["kind"],
               "sample": cpu_sample_text(r, args.cpu_sample)}
    line = {
        "metric": METRIC,
        "value": round(value, 2),
        "unit": "Mrays/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_step, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": frame_config(world),
        "build_mode": ("LBVH with SAH-rebuilt subtrees of at most 16,384 triangles (RQ_BUILD_SAH)" if sah
                       else "LBVH (Karras hierarchy, Morton order)"),
        "frame": {"triangles": ntri, "rays_per_step": frame_rays, "primary_rays": npx, "secondary_rays": sec_rays,
                  "primary_hits": hits},
        "build_mtris_per_s": round(ntri / statistics.median(build_ms) / 1e3, 1),
        "build_ms": round(statistics.median(build_ms), 4),
        "primary_mrays_per_s": round(npx / statistics.median(prim_ms) / 1e3, 1),
        "anyhit_mrays_per_s": round(sec_rays / shade_med / 1e3, 1),
        "shadow_ao_ms": round(shade_med, 4),
        "bvh": {"nodes4": info["num_nodes4"], "depth4": info["depth4"], "nodes2": info["num_nodes2"],
                "node_visits_per_anyhit_ray": round(v_node, 3), "tri_tests_per_anyhit_ray": round(v_tri, 3)},
        "e2e": {"value": round(pipe_value, 2), "unit": "Mrays/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": round(pipe_ms, 4),
                "mode": ("C ABI calls with pinned host buffers; per frame H2D of the mesh (positions + indices) "
                         "and D2H of the light masks and AO; copies on a second stream overlap the neighbouring "
                         "frames' compute (two device sets)"),
                "results_equal_serial": pipe_equal,
                "serial": {"value": round(e2e_value, 2), "ms_per_step": round(e2e_ms, 4),
                           "mode": "the same calls and copies on one stream, nothing overlapped"}},
        "roofline": {"bound": "hbm", "kernel": "k_shadow_ao", "achieved": round(achieved, 1), "peak": hbm,
                     "unit": "GB/s", "frac": round(achieved / hbm, 4), "traffic": traffic,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if "hbm_gbs" in peaks else "fallback",
                     "algorithmic_bytes_per_launch": round(alg_bytes),
                     "binding": dict(binding, source="profiles/k_shadow_ao_1080p.md (ncu, same kernel and frame)",
                                     what=("the algorithmic bytes are consumed from L1/L2: the kernel is bound by "
                                           "instruction issue and the L1, not by HBM (dram_frac)")),
                     "compulsory": {"bytes_per_launch": comp_bytes, "achieved": round(comp_gbs, 2),
                                    "frac": round(comp_gbs / hbm, 5),
                                    "what": "G-buffer pixel in (32 B) + light mask / AO word out (8 B); rays are "
                                            "generated in the kernel, so no ray or hit record crosses HBM"}},
        "cpu_baseline": cpu,
        "clocks": clocks,
        "gpu_launches": (BUILD_KERNELS[args.build] + FRAME_KERNELS) * args.steps,
        "shadow_tuning": shade_tuning,
        "camera_tuning": camera_tuning,
        "ao_blur": blur,
        "median_build": median_build,
        "reference_benchmarks": refbench,
        "radv_build": radv_build,
        "visibility": vis,
        "batched": batched,
        "serving": serving,
    }
    print(json.dumps(line), flush=True)
    ctx.close()


def load_peaks():
    """The measured HBM copy bandwidth and GEMM peaks of this GPU model, if present."""
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    return json.load(open(pk)) if os.path.exists(pk) else {}


def percentile(xs, q):
    import numpy as np
    return float(np.percentile(np.asarray(xs, dtype=np.float64), q))


def run_batched(ctx, dev, steps=200, plain_steps=20):
    """Batched builds: 512 deforming grids, triangle counts log-uniform in
    [64, 65536] (seed 2), 4,096 any-hit + 4,096 closest-hit rays per mesh.
    Batched: one deformation launch, one persistent build launch and one
    traversal launch per step, captured in a CUDA graph and replayed.  Plain:
    the same work as per-mesh rq_build + rq_trace calls (captured too when the
    driver allows, else eager).  Per-step device time p50 / p99."""
    import numpy as np
    import torch
    import rq
    from rq import workloads as W

    sizes = W.batched_sizes(512, seed=2)
    pos, idx, descs = W.batched_meshes(sizes, seed=2)
    ntri = len(idx)
    base = torch.from_numpy(pos).to(dev)
    cur = torch.empty_like(base)
    i_d = torch.from_numpy(idx.view(np.int32)).to(dev)
    rays, mesh, flags = W.batched_rays(descs, 4096, 4096, seed=2)
    nrays = len(rays)
    rays_d = torch.from_numpy(rays).to(dev)
    mesh_d = torch.from_numpy(mesh.view(np.int32)).to(dev)
    flags_d = torch.from_numpy(flags.view(np.int32)).to(dev)
    hits_b = torch.empty((nrays, 4), dtype=torch.int32, device=dev)
    hits_p = torch.empty((nrays, 4), dtype=torch.int32, device=dev)
    state = torch.zeros(2, dtype=torch.int32, device=dev)
    dt = W.DEFORM_DT

    batch = rq.Batch(ctx, descs)
    # launch shapes: the committed autotuner table, else tune now (untimed)
    from rq import tune as T
    key = T.workload_key(descs, 8192)
    shape = T.lookup(key)
    if shape is not None:
        batch.set_tuning(shape)
        tuning = {"source": "committed table rq/tuning_b200.json", **shape}
    else:
        got, trials = batch.autotune(base, i_d, rays_d, mesh_d, flags_d, hits=hits_b, reps=3)
        tuning = {"source": f"autotuned in this run ({len(trials)} shapes timed)",
                  **{k: got[k] for k in rq.Batch.TUNING_KEYS}}

    def bstep():
        rq.deform_wave_step(ctx, base, cur, state, dt, W.DEFORM_AMP, W.DEFORM_FREQ)
        batch.build(cur, i_d)
        batch.trace(rays_d, mesh_d, flags_d, hits=hits_b)

    handles = []
    for (vo, nv, to, nt) in descs:
        handles.append(rq.Bvh.build(ctx, cur[vo:vo + nv], i_d[to:to + nt]))

    def pstep():
        rq.deform_wave_step(ctx, base, cur, state, dt, W.DEFORM_AMP, W.DEFORM_FREQ)
        for m, (vo, nv, to, nt) in enumerate(descs):
            h = handles[m]
            rq.Bvh.build(ctx, cur[vo:vo + nv], i_d[to:to + nt], into=h)
            r0 = m * 8192
            rq.trace(ctx, h, rays_d[r0:r0 + 4096], flags=rq.RQ_TRACE_ANY, hits=hits_p[r0:r0 + 4096])
            rq.trace(ctx, h, rays_d[r0 + 4096:r0 + 8192], flags=rq.RQ_TRACE_CLOSEST, hits=hits_p[r0 + 4096:r0 + 8192])

    def capture(fn):
        side = torch.cuda.Stream(dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(side):
            fn()
        torch.cuda.current_stream(dev).wait_stream(side)
        torch.cuda.synchronize(dev)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            fn()
        return g

    def timed(run, n):
        evs = [torch.cuda.Event(enable_timing=True) for _ in range(n + 1)]
        s = torch.cuda.current_stream(dev)
        torch.cuda.synchronize(dev)
        evs[0].record(s)
        for k in range(n):
            run()
            evs[k + 1].record(s)
        torch.cuda.synchronize(dev)
        return [evs[k].elapsed_time(evs[k + 1]) for k in range(n)]

    for _ in range(3):
        bstep()
    gb = capture(bstep)
    state.zero_()
    bms = timed(gb.replay, steps)
    ctx.sync_check()
    # the same step through per-mesh calls; then check the hits agree
    for _ in range(2):
        pstep()
    plain_mode = "graph"
    try:
        gp = capture(pstep)
        prun = gp.replay
    except Exception as exc:  # capture refused: time the eager calls
        plain_mode = f"eager ({type(exc).__name__})"
        torch.cuda.synchronize(dev)
        prun = pstep
    state.zero_()
    pms = timed(prun, plain_steps)
    ctx.sync_check()
    state.zero_()
    gb.replay()
    state.zero_()
    prun()
    torch.cuda.synchronize(dev)
    equal = bool(torch.equal(hits_b, hits_p))
    out = {
        "workload": ("batched: 512 deforming grids, triangle counts log-uniform in [64, 65536] (seed 2), rebuilt "
                     "every step; 4,096 any-hit + 4,096 closest-hit rays per mesh; one persistent build launch and "
                     "one traversal launch per step in a CUDA graph"),
        "meshes": len(descs), "triangles_per_step": ntri, "rays_per_step": nrays,
        "batched": {"p50_ms": round(percentile(bms, 50), 4), "p99_ms": round(percentile(bms, 99), 4),
                    "mtris_per_s": round(ntri / percentile(bms, 50) / 1e3, 1),
                    "mrays_per_s": round(nrays / percentile(bms, 50) / 1e3, 1), "steps": steps},
        "plain": {"p50_ms": round(percentile(pms, 50), 4), "p99_ms": round(percentile(pms, 99), 4),
                  "mtris_per_s": round(ntri / percentile(pms, 50) / 1e3, 1),
                  "mrays_per_s": round(nrays / percentile(pms, 50) / 1e3, 1), "steps": plain_steps,
                  "mode": plain_mode},
        "speedup_p50": round(percentile(pms, 50) / percentile(bms, 50), 2),
        "hits_equal": equal,
        "tuning": tuning,
    }
    del gb
    for h in handles:
        h.destroy()
    batch.destroy()
    return out


def run_serving(dev, duration_s=2.0, catalogue=256):
    """Serving: Poisson 2,000 requests/s for `duration_s` (seed 4) over a
    catalogue of 256 height-field meshes with triangle counts log-uniform in
    [64, 1M]; rays per request log-uniform in [1k, 2M]; 50 % shadow, 30 % AO,
    20 % closest hit, rays generated inside the traversal launch.  BVHs stay
    resident (120 GB budget, LRU eviction); every mesh is built once before
    the timed stream.  Batched: up to 1,024 requests / 16M rays per launch,
    4 launches in flight.  Plain: one request per launch, one in flight.
    Latency = completion seen by the host - submission at the arrival time.
    Also a saturation run (every request at t=0) for throughput, and a sweep
    of arrival rates (the same requests, arrival times scaled) giving p50 /
    p99 per rate and the highest rate each mode sustains under a p99 bound."""
    import numpy as np
    import torch
    import rq
    from rq import workloads as W

    sizes = W.serving_catalogue(catalogue, seed=4)
    meshes = [W.serving_mesh(sizes, m, seed=4) for m in range(catalogue)]
    t_arr, mesh, kind, nrays, seeds = W.serving_requests(catalogue, duration_s, seed=4)
    n = len(t_arr)
    ring = 1 << 27  # hit slots reused round-robin (results are left on the device)
    hits = torch.empty((ring, 4), dtype=torch.int32, device=dev)
    offs, o = [], 0
    for c in nrays:
        if o + c > ring:
            o = 0
        offs.append(o)
        o += int(c)
    base = hits.data_ptr()

    def make_reqs(srv, ids):
        return [rq.Request(ids[int(mesh[i])], int(kind[i]), int(nrays[i]), int(seeds[i]), 0, 0, None,
                           base + 16 * offs[i], i) for i in range(n)]

    rates = (1000, 2000, 4000, 6000, 8000, 12000, 16000, 24000)

    def run_stream(srv, reqs, arrivals):
        tickets = srv.replay(reqs, arrivals)
        comp = srv.completions()
        lat = np.array([comp[t]["t_done"] - comp[t]["t_submit"] for t in tickets])
        t_first = min(comp[t]["t_submit"] for t in tickets)
        t_last = max(comp[t]["t_done"] for t in tickets)
        ok = all(comp[t]["status"] == 0 for t in tickets)
        return lat, t_first, t_last, ok

    def one(mode, rebuild=False):
        cfg = dict(mode=mode, budget_bytes=120 << 30, slots=4, max_wave_rays=1 << 24, max_wave_requests=1024,
                   rebuild=rebuild)
        srv = rq.Server(**cfg)
        ids = [srv.add_mesh(p, i) for p, i in meshes]
        # warm the resident cache: one 1,000-ray request per mesh
        t0 = srv.now()
        for m in range(catalogue):
            srv.submit(rq.Request(ids[m], 3, 1000, 1, 0, 0, None, base, 0))
        warm = srv.completions()
        t_warm = srv.now() - t0
        st0 = srv.stats()
        reqs = make_reqs(srv, ids)
        tickets = srv.replay(reqs, t_arr)
        comp = srv.completions()
        st1 = srv.stats()
        lat = np.array([comp[t]["t_done"] - comp[t]["t_submit"] for t in tickets])
        ok = all(comp[t]["status"] == 0 for t in tickets) and all(c["status"] == 0 for c in warm.values())
        t_first = min(comp[t]["t_submit"] for t in tickets)
        t_last = max(comp[t]["t_done"] for t in tickets)
        stream = {"p50_ms": round(float(np.percentile(lat, 50)) * 1e3, 3),
                  "p99_ms": round(float(np.percentile(lat, 99)) * 1e3, 3),
                  "mean_ms": round(float(lat.mean()) * 1e3, 3),
                  "mrays_per_s": round(float(nrays.sum()) / (t_last - t_first) / 1e6, 1),
                  "requests_per_s": round(n / (t_last - t_first), 1),
                  "launches": int(st1["launches"] - st0["launches"]),
                  "requests_per_launch": round(n / max(1, st1["launches"] - st0["launches"]), 2),
                  "all_ok": bool(ok)}
        # saturation: the same requests, all at t = 0
        tickets = srv.replay(reqs, np.zeros(n))
        comp = srv.completions()
        t_first = min(comp[t]["t_submit"] for t in tickets)
        t_last = max(comp[t]["t_done"] for t in tickets)
        lat = np.array([comp[t]["t_done"] - comp[t]["t_submit"] for t in tickets])
        sat = {"makespan_ms": round((t_last - t_first) * 1e3, 2),
               "mrays_per_s": round(float(nrays.sum()) / (t_last - t_first) / 1e6, 1),
               "requests_per_s": round(n / (t_last - t_first), 1),
               "p50_ms": round(float(np.percentile(lat, 50)) * 1e3, 3),
               "p99_ms": round(float(np.percentile(lat, 99)) * 1e3, 3)}
        # arrival-rate sweep: the same requests, arrivals scaled to each rate
        sweep = []
        for r in rates:
            s0 = srv.stats()
            lat, t_first, t_last, ok_r = run_stream(srv, reqs, t_arr * (W.SERVE_RATE / r))
            s1 = srv.stats()
            sweep.append({"rate": r, "p50_ms": round(float(np.percentile(lat, 50)) * 1e3, 3),
                          "p99_ms": round(float(np.percentile(lat, 99)) * 1e3, 3),
                          "mrays_per_s": round(float(nrays.sum()) / (t_last - t_first) / 1e6, 1),
                          "requests_per_s": round(n / (t_last - t_first), 1),
                          "requests_per_launch": round(n / max(1, s1["launches"] - s0["launches"]), 2),
                          "all_ok": bool(ok_r)})
        st = srv.stats()
        srv.close()
        return {"stream": stream, "saturation": sat, "sweep": sweep, "warm_build_s": round(t_warm, 3),
                "resident_gb": round(st["peak_resident_bytes"] / 1e9, 2), "builds": int(st["builds"])}

    b = one(rq.RQ_SERVE_BATCHED)
    p = one(rq.RQ_SERVE_PLAIN)
    pr = one(rq.RQ_SERVE_PLAIN, rebuild=True)
    torch.cuda.synchronize(dev)

    def sustained(m, bound_ms):
        """Highest swept rate whose p99 stays within the bound and whose
        achieved request rate keeps up with the offered one (within 10 %)."""
        ok = [x for x in m["sweep"] if x["p99_ms"] <= bound_ms and x["requests_per_s"] >= 0.9 * x["rate"]]
        return max((x["rate"] for x in ok), default=None)

    at_p99 = []
    for bound in (1.0, 2.0, 5.0, 10.0, 20.0):
        rb, rp, rr = sustained(b, bound), sustained(p, bound), sustained(pr, bound)
        at_p99.append({"p99_bound_ms": bound, "batched_rate": rb, "plain_rate": rp, "plain_rebuild_rate": rr,
                       "batched_over_plain": round(rb / rp, 2) if rb and rp else None,
                       "batched_over_plain_rebuild": round(rb / rr, 2) if rb and rr else None})
    return {
        "workload": (f"serving: Poisson {W.SERVE_RATE:.0f} req/s for {duration_s:g} s (seed 4, {n} requests), "
                     f"{catalogue} resident height-field meshes with triangle counts log-uniform in [64, 1M] "
                     f"(mean {sizes.mean() / 1e3:.1f}k), rays log-uniform in [1k, 2M] (mean {nrays.mean() / 1e3:.1f}k), "
                     "50% shadow / 30% AO / 20% closest hit generated in the launch; 120 GB budget"),
        "requests": n, "rays": int(nrays.sum()), "catalogue_triangles": int(sizes.sum()),
        "batched": b, "plain": p, "plain_rebuild": pr,
        "plain_modes": ("plain: one request per launch, one launch in flight, BVHs resident; plain_rebuild: the "
                        "same with the request's BVH rebuilt before its trace (per-request build + trace)"),
        "stream_p99_ratio_plain_over_batched": round(p["stream"]["p99_ms"] / b["stream"]["p99_ms"], 2),
        "stream_p99_ratio_plain_rebuild_over_batched": round(pr["stream"]["p99_ms"] / b["stream"]["p99_ms"], 2),
        "saturation_throughput_ratio": round(b["saturation"]["mrays_per_s"] / p["saturation"]["mrays_per_s"], 2),
        "saturation_throughput_ratio_vs_plain_rebuild": round(
            b["saturation"]["mrays_per_s"] / pr["saturation"]["mrays_per_s"], 2),
        "sweep_rates": list(rates),
        "sustained_at_p99": at_p99,
        "sustained_how": ("for each p99 bound, the highest swept arrival rate (same requests, arrivals scaled) at "
                          "which the mode's p99 stays within the bound and its achieved request rate is at least "
                          "90 % of the offered rate; ratios are served (batched) over plain at the same bound"),
    }


def run_reference_benchmarks(ctx, dev):
    """The reference's own micro-benchmarks of this path, on the B200, beside the figures the
    reference published for an RX 6700 XT (Vulkan): the fast RADV builder at N = 64 ... 4,096
    (README.md:48-51) and the SW BVH4 traversal of 1,048,576 procedural rays, coherent and
    incoherent, at 968 / 99,458 / 999,698 triangles (results/exp0_throughput.csv).  The terrain
    is a height field of this repository with the reference's triangle counts and extent (Y up,
    100 units wide), not the reference's own terrain; the rays come from the reference's
    generators (camera (0, 50, -45) looking at (0, 0, 5)).  CUDA-event medians."""
    import numpy as np
    import torch
    import rq

    def timed(fn, reps):
        fn()
        ms = []
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            b.synchronize()
            ms.append(a.elapsed_time(b))
        return statistics.median(ms)

    # the builder's device time: 50 builds captured in a CUDA graph and replayed, so that the
    # host's per-call launch cost (larger than these kernels) does not count, as the
    # reference's GPU timestamps do not count its host
    radv = {}
    published_radv = {64: 9.41, 256: 5.14, 1024: 15.59, 4096: 80.35}
    side = torch.cuda.Stream(dev)
    for n in (64, 256, 1024, 4096):
        rng = np.random.default_rng(n)
        tri9 = torch.from_numpy(rng.uniform(-1, 1, size=9 * n).astype(np.float32)).to(dev)
        img = torch.empty(rq.radv_size(n), dtype=torch.uint8, device=dev)
        with torch.cuda.stream(side):
            rq.build_radv(ctx, tri9, img)  # scratch allocated before the capture
            side.synchronize()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=side):
                for _ in range(50):
                    rq.build_radv(ctx, tri9, img)
        ctx.sync_check()
        us = 1e3 * timed(g.replay, 20) / 50
        del g
        radv[str(n)] = {"us": round(us, 2), "reference_rx6700xt_us": published_radv[n]}
    published_sw = {968: (1839.7, 1197.7), 99458: (883.5, 67.5), 999698: (447.4, 27.7)}
    sw = {}
    for q, n in ((22, 968), (223, 99458), (707, 999698)):
        pos, idx = rq.scene_grid(q, q, amp=0.05, seed=7)
        pos = np.ascontiguousarray(np.stack([50.0 * pos[:, 0], 50.0 * pos[:, 2], 50.0 * pos[:, 1]], 1),
                                   dtype=np.float32)
        p = torch.from_numpy(pos).to(dev)
        i = torch.from_numpy(idx.view(np.int32)).to(dev)
        b = rq.Bvh.build(ctx, p, i)
        n2, tr, n4, _ = b.download()
        t_n4 = torch.from_numpy(n4.view(np.uint8).copy()).to(dev)
        t_tr = torch.from_numpy(tr.view(np.uint8).copy()).to(dev)
        row = {}
        for name, coh in (("coherent", 1), ("incoherent", 0)):
            rays = rq.gen_rays_procedural(ctx, [0, 50, -45], [0, 0, 5], 1 << 20, coh)
            hits = torch.empty((1 << 20, 4), dtype=torch.int32, device=dev)
            ms_ref = timed(lambda: rq.trace_ref_bvh4(ctx, t_n4, t_tr, rays), 20)
            ms_eng = timed(lambda: rq.trace(ctx, b, rays, rq.RQ_TRI_MT, hits=hits), 20)
            row[name] = {"published_arithmetic_mrays_per_s": round((1 << 20) / ms_ref / 1e3, 1),
                         "engine_mrays_per_s": round((1 << 20) / ms_eng / 1e3, 1),
                         "reference_rx6700xt_mrays_per_s": published_sw[n][0 if coh else 1]}
        sw[str(n)] = row
        b.destroy()
    torch.cuda.synchronize(dev)
    return {"fast_bvh_builder": radv, "sw_bvh4_traversal": sw,
            "note": ("reference figures: RX 6700 XT through Vulkan, as published; ours: this B200. "
                     "published_arithmetic = k_ref4 (software_bvh_bvh4.comp restated, closest hit, "
                     "Moller-Trumbore); engine = rq_trace closest hit with the same triangle test")}


def run_radv_build(ctx, dev, peaks, reps=50, meshes=None):
    """The fast builder (fast_bvh_builder.comp, rq_build_radv) at the frame's and the visibility
    workload's triangle counts: the meshes' triangles as a vertex soup (9 floats each), one image
    rebuilt per launch.  Algorithmic bytes per launch = 36 B per triangle read + the whole image
    written (64 B triangle nodes, 128 B box nodes, 192 B header); both exceed L2 (126 MB).
    CUDA-event median over `reps` back-to-back builds."""
    import numpy as np
    import torch
    import rq
    from rq import workloads as W

    hbm = peaks.get("hbm_gbs", 6650.0)
    out = {}
    for name, mesh in (meshes or (("frame_2.5M", W.shadow_mesh), ("visibility_8.3M", W.visibility_mesh))):
        pos, idx = mesh()
        n = len(idx)
        tri9 = torch.from_numpy(pos).to(dev)[torch.from_numpy(idx.astype(np.int64)).to(dev)].reshape(-1)
        tri9 = tri9.contiguous()
        img = torch.empty(rq.radv_size(n), dtype=torch.uint8, device=dev)
        for _ in range(3):
            rq.build_radv(ctx, tri9, img)
        ms = []
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            rq.build_radv(ctx, tri9, img)
            b.record()
            ms.append((a, b))
        torch.cuda.synchronize(dev)
        ctx.sync_check()
        med = statistics.median(a.elapsed_time(b) for a, b in ms)
        alg = 36 * n + rq.radv_size(n)
        gbs = alg / med / 1e6
        out[name] = {"triangles": n, "us": round(1e3 * med, 2), "mtris_per_s": round(n / med / 1e3, 1),
                     "algorithmic_bytes": alg, "achieved_gbs": round(gbs, 1), "frac_of_hbm": round(gbs / hbm, 4)}
        del tri9, img
    return out


def run_visibility(ctx, dev, stream, frames=200):
    """Subpixel visibility: 8,323,200 triangles (2040x2040 quads, seed 3) deforming
    every frame (z = z0 + 0.05 sin(0.1 f + x)); 1920x1080 jittered primary rays
    per frame; the BVH either fully rebuilt or refitted each frame."""
    import numpy as np
    import torch
    import rq
    from rq import workloads as W

    pos, idx = W.visibility_mesh()
    ntri = len(idx)
    base = torch.from_numpy(pos).to(dev)
    cur = torch.empty_like(base)
    i_d = torch.from_numpy(idx.view(np.int32)).to(dev)
    gbuf = torch.empty((WIDTH * HEIGHT, 8), dtype=torch.int32, device=dev)
    rq.deform_wave(ctx, base, cur, W.deform_time(0), W.DEFORM_AMP, W.DEFORM_FREQ)
    bvh = rq.Bvh.build(ctx, cur, i_d)
    out = {"workload": ("subpixel visibility: 8,323,200-triangle grid (2040x2040 quads, seed 3) deformed every "
                        "frame, 1920x1080 jittered closest-hit primary rays, 200 frames per mode"),
           "triangles": ntri, "frames": frames}
    for mode in ("rebuild", "refit"):
        rq.deform_wave(ctx, base, cur, W.deform_time(0), W.DEFORM_AMP, W.DEFORM_FREQ)
        rq.Bvh.build(ctx, cur, i_d, into=bvh)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3 * frames + 1)]
        torch.cuda.synchronize(dev)
        ev[0].record(stream)
        for f in range(frames):
            rq.deform_wave(ctx, base, cur, W.deform_time(f), W.DEFORM_AMP, W.DEFORM_FREQ)
            if mode == "rebuild":
                rq.Bvh.build(ctx, cur, i_d, into=bvh)
            else:
                bvh.refit(cur, i_d)
            ev[3 * f + 1].record(stream)
            cam = W.visibility_camera(seed=3 + f)
            rq.render_gbuffer(ctx, bvh, cam, gbuf)
            ev[3 * f + 2].record(stream)
            ev[3 * f + 3].record(stream)
        torch.cuda.synchronize(dev)
        ctx.sync_check()
        total = ev[0].elapsed_time(ev[-1])
        upd = [(ev[3 * f].elapsed_time(ev[3 * f + 1])) for f in range(1, frames)]
        trc = [ev[3 * f + 1].elapsed_time(ev[3 * f + 2]) for f in range(frames)]
        hits = int((gbuf[:, 3] != 0).sum().item())
        out[mode] = {"ms_per_frame": round(total / frames, 4),
                     "update_ms": round(statistics.median(upd), 4),
                     "trace_ms": round(statistics.median(trc), 4),
                     "trace_ms_last_frame": round(trc[-1], 4),
                     "mrays_per_s": round(WIDTH * HEIGHT / (total / frames) / 1e3, 1),
                     "update_mtris_per_s": round(ntri / statistics.median(upd) / 1e3, 1),
                     "primary_hits_last_frame": hits}
    bvh.destroy()
    return out


def run_extra(args):
    """One secondary workload alone (for profiling): its JSON object."""
    import torch
    import rq
    dev = torch.device("cuda", 0)
    ctx = rq.Context(0)
    if args.extra == "visibility":
        out = run_visibility(ctx, dev, torch.cuda.current_stream(dev), frames=max(1, args.steps))
    elif args.extra == "batched":
        out = run_batched(ctx, dev, steps=max(1, args.steps), plain_steps=1)
    elif args.extra == "radv":
        from rq import workloads as W
        out = run_radv_build(ctx, dev, load_peaks(), reps=max(1, args.steps),
                             meshes=(("frame_2.5M", W.shadow_mesh),))
    else:
        out = run_serving(dev, duration_s=max(0.05, args.steps * 0.05), catalogue=args.serve_catalogue)
    print(json.dumps({"extra": args.extra, **out}))


def main():
    args = parse()
    if args.extra:
        run_extra(args)
        return
    world, rank, local, pg = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank, pg)
        else:
            run_ours(args, world, rank, local, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
