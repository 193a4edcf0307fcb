"""Synthetic workloads of the benchmark configurations, defined once for the
benchmark and the tests.  All inputs are generated on the host from seeds.

  plain        64x32-quad grid (4,096 triangles) on [-1,1]^2, height
               0.2*sin(3x)*cos(3y) + N(0, 0.01) per vertex (seed 0); 65,536
               closest-hit rays from z=2, origins U([-1,1]^2), directions
               normalize(U(-0.3,0.3), U(-0.3,0.3), -1)
  shadows      1118x1118 quads (2,499,848 triangles), same height field,
               seed 1; 1920x1080 primary rays from a camera that sees only the
               mesh; 16 point lights U([-1,1]^2 x [2,2.5]) (seed 1, radius
               100, so every light is in range); 1 SPP AO rays, tmax 0.5
  visibility   2040x2040 quads (8,323,200 triangles), seed 3; 1920x1080
               jittered primary rays; per-frame deformation z += 0.05*sin(t+x)
  batched      512 grids with triangle counts log-uniform in [64, 65,536]
               (seed 2); 4,096 any-hit and 4,096 closest-hit rays per mesh
  serving      Poisson arrivals at 2,000 requests/s (seed 4); mesh sizes
               log-uniform in [64, 1M] triangles, ray batches log-uniform in
               [1k, 2M], kinds 50 % shadow / 30 % AO / 20 % closest hit
"""
import math

import numpy as np

from . import camera_look_at, scene_grid, scene_rays_down, shade_params

AMP, FREQ, SIGMA = 0.2, 3.0, 0.01


def plain_mesh():
    return scene_grid(64, 32, seed=0)


def plain_rays(n=65536, seed=0):
    return scene_rays_down(n, -1.0, 1.0, -1.0, 1.0, 2.0, 0.3, 0.01, 1000.0, seed)


def shadow_mesh():
    return scene_grid(1118, 1118, seed=1)


def shadow_camera(width=1920, height=1080, flags=0):
    return camera_look_at((0.0, -0.6, 2.6), (0.0, 0.0, 0.0), (0.0, 0.0, 1.0), 20.0, width, height, flags=flags)


def shadow_lights(n=16, seed=1):
    rng = np.random.default_rng(seed)
    xy = rng.uniform(-1.0, 1.0, size=(n, 2))
    z = rng.uniform(2.0, 2.5, size=n)
    return [(float(xy[k, 0]), float(xy[k, 1]), float(z[k]), 100.0) for k in range(n)]


def shadow_params(width=1920, height=1080, flags=0):
    return shade_params(width, height, shadow_lights(16), ao_spp=1, ao_tmax=0.5, flags=flags)


def visibility_mesh(q=2040):
    return scene_grid(q, q, seed=3)


def visibility_camera(width=1920, height=1080, jitter=True, seed=3, flags=0):
    """Straight down from z=3 with a 19.5 degree vertical field: every pixel
    stays on the mesh even where it dips to z=-0.25, and about 47 % of the
    grid (1.9 triangles per pixel at 2040x2040 quads) is in view."""
    return camera_look_at((0.0, 0.0, 3.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 19.5, width, height, jitter=jitter,
                          seed=seed, flags=flags)


DEFORM_AMP, DEFORM_FREQ, DEFORM_DT = 0.05, 1.0, 0.1


def deform_time(frame):
    """Frame f of a deformation sequence: z = z0 + 0.05*sin(0.1*f + x)."""
    return DEFORM_DT * frame


def log_uniform_int(rng, lo, hi, size):
    return np.exp(rng.uniform(math.log(lo), math.log(hi), size=size)).astype(np.int64)


def batched_sizes(count=512, seed=2):
    """Triangle counts log-uniform in [64, 65536], rounded to whole quads."""
    rng = np.random.default_rng(seed)
    t = log_uniform_int(rng, 64, 65536, count)
    return np.maximum(64, t // 2 * 2)


def grid_for_triangles(t):
    """Quad grid (qx, qy) with 2*qx*qy close to t triangles."""
    q = max(1, int(t) // 2)
    qx = max(1, int(math.sqrt(q)))
    qy = max(1, q // qx)
    return qx, qy


def batched_meshes(sizes, seed=2):
    """Concatenate one height-field grid per requested triangle count (mesh m
    seeded seed*100003 + m).  Returns float32 [V,3] positions, uint32 [T,3]
    mesh-local indices and the (vertex_offset, num_vertices, triangle_offset,
    num_triangles) of every mesh."""
    pos_l, idx_l, descs = [], [], []
    v_off = t_off = 0
    for m, t in enumerate(sizes):
        qx, qy = grid_for_triangles(t)
        p, i = scene_grid(qx, qy, seed=seed * 100003 + m)
        pos_l.append(p)
        idx_l.append(i)
        descs.append((v_off, len(p), t_off, len(i)))
        v_off += len(p)
        t_off += len(i)
    return np.concatenate(pos_l), np.concatenate(idx_l), descs


def batched_rays(descs, per_mesh_any=4096, per_mesh_closest=4096, seed=2):
    """Downward random rays per mesh (as the plain workload's): the first
    per_mesh_any of each mesh are any-hit, the rest closest-hit.  Returns
    float32 [R,8] rays, uint32 mesh index per ray, uint32 flags per ray."""
    k = per_mesh_any + per_mesh_closest
    rays = scene_rays_down(len(descs) * k, -1.0, 1.0, -1.0, 1.0, 2.0, 0.3, 0.01, 1000.0, seed)
    mesh = np.repeat(np.arange(len(descs), dtype=np.uint32), k)
    flags = np.tile(np.r_[np.ones(per_mesh_any, np.uint32), np.zeros(per_mesh_closest, np.uint32)], len(descs))
    return rays, mesh, flags


# ------------------------------------------------------------------ serving
SERVE_RATE = 2000.0          # requests per second (Poisson)
SERVE_MIX = (0.5, 0.3, 0.2)  # shadow, AO, closest hit


def serving_catalogue(count=256, seed=4):
    """Triangle counts of the served meshes, log-uniform in [64, 1M]; mesh m
    is the height-field grid seeded seed*100003 + m.  A request draws its mesh
    uniformly from the catalogue, so request meshes are log-uniform in
    [64, 1M] too, and each mesh is reused by many requests."""
    rng = np.random.default_rng(seed)
    return np.maximum(64, log_uniform_int(rng, 64, 1 << 20, count) // 2 * 2)


def serving_mesh(sizes, m, seed=4):
    qx, qy = grid_for_triangles(sizes[m])
    return scene_grid(qx, qy, seed=seed * 100003 + m)


def serving_requests(n_meshes, duration_s=2.0, rate=SERVE_RATE, seed=4):
    """Poisson arrivals at `rate` over `duration_s`: arrival times (s), mesh
    index, kind (1 shadow, 2 AO, 3 closest), ray count log-uniform in
    [1000, 2M], per-request seed."""
    rng = np.random.default_rng(seed + 1)
    gaps = rng.exponential(1.0 / rate, size=int(rate * duration_s * 1.5) + 16)
    t = np.cumsum(gaps)
    t = t[t < duration_s]
    n = len(t)
    mesh = rng.integers(0, n_meshes, n)
    kind = rng.choice([1, 2, 3], size=n, p=list(SERVE_MIX))
    rays = log_uniform_int(rng, 1000, 2_000_000, n)
    return t, mesh, kind, rays, np.arange(n, dtype=np.uint32) + 1
