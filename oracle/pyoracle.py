"""ctypes bindings for the oracle — TEST INFRASTRUCTURE, not product code.

Loads oracle/_build/liboracle.so (the CPU restatement in oracle.cpp) and,
when present, oracle/_ref/libref.so (the reference's own SoftwareBVH,
createTessellatedTerrain, compute_tree_layout and generate_dynamic_grid_mesh,
compiled from the reference sources by oracle/Makefile).

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs import this.
Every array crossing the boundary is a C-contiguous numpy array.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref.so")

# numpy mirrors of include/rq_layouts.h
BVH2_NODE = np.dtype([("aabb_min", "<f4", 3), ("left_child", "<i4"), ("aabb_max", "<f4", 3), ("right_child", "<i4")])
TRIANGLE = np.dtype([("v0", "<f4", 4), ("v1", "<f4", 4), ("v2", "<f4", 4)])
BVH4_NODE = np.dtype([("min_x", "<f4", 4), ("max_x", "<f4", 4), ("min_y", "<f4", 4), ("max_y", "<f4", 4),
                      ("min_z", "<f4", 4), ("max_z", "<f4", 4), ("child_index", "<i4", 4), ("child_count", "<i4", 4)])
RAY = np.dtype([("org", "<f4", 3), ("tmin", "<f4"), ("dir", "<f4", 3), ("tmax", "<f4")])
HIT = np.dtype([("hit", "<u4"), ("t", "<f4"), ("instance_id", "<u4"), ("primitive_id", "<u4")])
STATS = np.dtype([("hit", "<u4"), ("box_tests", "<u4"), ("tri_tests", "<u4"), ("pad", "<u4")])
assert BVH2_NODE.itemsize == 32 and TRIANGLE.itemsize == 48 and BVH4_NODE.itemsize == 128
assert RAY.itemsize == 32 and HIT.itemsize == 16 and STATS.itemsize == 16

_P = C.c_void_p


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_P)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError("oracle library missing: run `make -C oracle`")
        L = C.CDLL(ORACLE_SO)
        L.orc_lbvh_build.argtypes = [_P, C.c_uint32, _P, C.c_uint32, C.c_uint32, _P, _P, _P, _P, _P, _P, _P, _P]
        L.orc_lbvh_build.restype = C.c_int
        L.orc_lbvh_sah_build.argtypes = [_P, C.c_uint32, _P, C.c_uint32, C.c_uint32, C.c_uint32, _P, _P, _P, _P, _P,
                                         _P, _P, _P, _P]
        L.orc_lbvh_sah_build.restype = C.c_int
        L.orc_collapse4.argtypes = [_P, C.c_uint32, _P, _P, _P]
        L.orc_collapse4.restype = C.c_int
        L.orc_radv_build.argtypes = [_P, C.c_uint32, _P]
        L.orc_radv_build.restype = C.c_int
        L.orc_trace_ref_bvh4.argtypes = [_P, _P, _P, C.c_uint32, _P, _P, _P, C.c_int]
        L.orc_trace_ref_bvh2.argtypes = [_P, _P, _P, C.c_uint32, C.c_float, _P, C.c_int]
        L.orc_trace_bvh4.argtypes = [_P, _P, _P, _P, C.c_uint32, C.c_uint32, _P, _P, _P, C.c_int]
        L.orc_trace_radv.argtypes = [_P, _P, C.c_uint32, C.c_uint32, _P, _P, C.c_int]
        L.orc_gen_rays_procedural.argtypes = [_P, _P, C.c_uint32, C.c_uint32, _P]
        L.orc_sincos.argtypes = [C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.orc_gen_mesh_rays.argtypes = [_P, _P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, _P, _P]
        L.orc_gbuffer_depth.argtypes = [_P, C.c_uint32, _P, _P]
        L.orc_blur_ao.argtypes = [_P, _P, _P, C.c_uint32, C.c_uint32, C.c_int, C.c_int, C.c_float]
        L.orc_tlas_trace.argtypes = [_P, _P, _P, _P, _P, _P, _P, C.c_uint32, _P, C.c_uint32, C.c_uint32,
                                     C.c_uint32, _P, C.c_int]
        L.orc_render_gbuffer.argtypes = [_P, _P, _P, _P, _P, C.c_uint32, _P, C.c_int]
        L.orc_render_shadow_ao.argtypes = [_P, _P, _P, _P, _P, C.c_uint32, _P, _P, _P, C.c_int]
        L.orc_camera_rays.argtypes = [_P, _P, C.c_uint32, _P]
        L.orc_shade_rays.argtypes = [_P, _P, _P, C.c_uint32, _P, _P, _P, C.c_uint64, _P]
        L.orc_render_reflect.argtypes = [_P, _P, _P, _P, _P, _P, C.c_uint32, _P, _P, C.c_int]
        L.orc_render_ao_depth.argtypes = [_P, _P, _P, _P, _P, C.c_uint32, _P, _P, C.c_int]
        L.orc_ao_depth_rays.argtypes = [_P, _P, _P, C.c_uint32, _P, _P, C.c_uint64, _P]
        L.orc_refit.argtypes = [_P, _P, _P, C.c_uint32, _P, _P, C.c_uint32, _P, C.c_uint32]
        L.orc_recover_perm.argtypes = [_P, C.c_uint32, _P, _P, C.c_uint32, _P]
        L.orc_recover_perm.restype = C.c_int
        L.orc_scene_grid.argtypes = [C.c_uint32, C.c_uint32, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float,
                                     C.c_float, C.c_float, C.c_uint64, _P, _P]
        L.orc_scene_grid.restype = C.c_int
        L.orc_camera_look_at.argtypes = [_P, _P, _P, C.c_float, C.c_uint32, C.c_uint32, _P]
        L.orc_camera_look_at.restype = C.c_int
        _lib = L
    return _lib


def have_ref():
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        if not have_ref():
            raise RuntimeError("reference library missing: run `make -C oracle` where the reference tree exists")
        R = C.CDLL(REF_SO)
        R.ref_build.argtypes = [_P, C.c_uint32, _P, C.c_uint32, C.c_uint32, C.c_int]
        R.ref_build.restype = _P
        R.ref_collapse.argtypes = [_P, C.c_uint32, _P, C.c_uint32]
        R.ref_collapse.restype = _P
        R.ref_counts.argtypes = [_P, _P, _P, _P]
        R.ref_copy.argtypes = [_P, _P, _P, _P]
        R.ref_free.argtypes = [_P]
        R.ref_terrain.argtypes = [C.c_uint32, C.c_float, _P, _P, _P, _P]
        R.ref_tree_layout.argtypes = [C.c_uint32, _P, _P, _P, _P, _P]
        R.ref_dynamic_grid.argtypes = [C.c_uint32, C.c_float, C.c_float, _P, _P]
        R.ref_dump_bvh_structure.argtypes = [_P, C.c_size_t, _P, C.c_size_t]
        R.ref_dump_bvh_structure.restype = C.c_size_t
        _ref = R
    return _ref


def threads():
    return max(1, os.cpu_count() or 1)


# ------------------------------------------------------------- Oracle B --

def lbvh_build(pos, idx, max_leaf=4, stride_floats=3):
    """Oracle B.  pos: float32 vertex array; idx: uint32 (3 per tri) or None.
    Returns dict with codes, sorted ids, nodes2, tris, nodes4, depth4."""
    pos = np.ascontiguousarray(pos, dtype=np.float32)
    if idx is not None:
        idx = np.ascontiguousarray(idx, dtype=np.uint32)
        n = idx.size // 3
    else:
        n = (pos.size // stride_floats) // 3
    codes = np.empty(n, np.uint32)
    srt = np.empty(n, np.uint32)
    nodes2 = np.empty(2 * n, BVH2_NODE)
    tris = np.empty(n, TRIANGLE)
    nodes4 = np.empty(max(1, n), BVH4_NODE)
    n2 = np.zeros(1, np.uint32)
    n4 = np.zeros(1, np.uint32)
    d4 = np.zeros(1, np.uint32)
    rc = lib().orc_lbvh_build(_ptr(pos), stride_floats, _ptr(idx), n, max_leaf, _ptr(codes), _ptr(srt),
                              _ptr(nodes2), _ptr(n2), _ptr(tris), _ptr(nodes4), _ptr(n4), _ptr(d4))
    assert rc == 0
    return dict(codes=codes, sorted=srt, nodes2=nodes2[: n2[0]].copy(), tris=tris,
                nodes4=nodes4[: n4[0]].copy(), depth4=int(d4[0]))


def lbvh_sah_build(pos, idx, max_leaf=4, sah_max=1024, stride_floats=3):
    """LBVH with SAH-rebuilt subtrees of at most sah_max primitives.  Returns
    dict with codes, sorted ids, perm (leaf order -> original), nodes2,
    tris, nodes4, depth4."""
    pos = np.ascontiguousarray(pos, dtype=np.float32)
    if idx is not None:
        idx = np.ascontiguousarray(idx, dtype=np.uint32)
        n = idx.size // 3
    else:
        n = (pos.size // stride_floats) // 3
    codes = np.empty(n, np.uint32)
    srt = np.empty(n, np.uint32)
    perm = np.empty(n, np.uint32)
    nodes2 = np.empty(2 * n, BVH2_NODE)
    tris = np.empty(n, TRIANGLE)
    nodes4 = np.empty(max(1, n), BVH4_NODE)
    n2 = np.zeros(1, np.uint32)
    n4 = np.zeros(1, np.uint32)
    d4 = np.zeros(1, np.uint32)
    rc = lib().orc_lbvh_sah_build(_ptr(pos), stride_floats, _ptr(idx), n, max_leaf, sah_max, _ptr(codes), _ptr(srt),
                                  _ptr(nodes2), _ptr(n2), _ptr(tris), _ptr(perm), _ptr(nodes4), _ptr(n4), _ptr(d4))
    assert rc == 0
    return dict(codes=codes, sorted=srt, perm=perm, nodes2=nodes2[: n2[0]].copy(), tris=tris,
                nodes4=nodes4[: n4[0]].copy(), depth4=int(d4[0]))


def collapse4(nodes2):
    nodes2 = np.ascontiguousarray(nodes2)
    out = np.empty(max(1, len(nodes2)), BVH4_NODE)
    n4 = np.zeros(1, np.uint32)
    d4 = np.zeros(1, np.uint32)
    lib().orc_collapse4(_ptr(nodes2), len(nodes2), _ptr(out), _ptr(n4), _ptr(d4))
    return out[: n4[0]].copy(), int(d4[0])


# ------------------------------------------------------------- Oracle C --

def radv_size(n):
    counts = [(n + 3) // 4]
    while counts[-1] > 1:
        counts.append((counts[-1] + 3) // 4)
    return 192 + 128 * sum(counts) + 64 * n


def radv_build(tri9):
    tri9 = np.ascontiguousarray(tri9, dtype=np.float32)
    n = tri9.size // 9
    img = np.empty(radv_size(n), np.uint8)
    assert lib().orc_radv_build(_ptr(tri9), n, _ptr(img)) == 0
    return img


# ------------------------------------------------------------ traversal --

def trace_ref_bvh4(nodes4, tris, rays, return_dropped=False):
    """software_bvh_bvh4.comp as published: (stats, hits[, dropped]) where
    dropped counts the pushes per ray its 24-entry stack could not hold."""
    rays = np.ascontiguousarray(rays)
    stats = np.empty(len(rays), STATS)
    hits = np.empty(len(rays), HIT)
    dropped = np.empty(len(rays), np.uint32) if return_dropped else None
    lib().orc_trace_ref_bvh4(_ptr(np.ascontiguousarray(nodes4)), _ptr(np.ascontiguousarray(tris)), _ptr(rays),
                             len(rays), _ptr(stats), _ptr(hits), _ptr(dropped), threads())
    return (stats, hits, dropped) if return_dropped else (stats, hits)


def trace_ref_bvh2(nodes2, tris, rays, t_eps=0.001):
    rays = np.ascontiguousarray(rays)
    flags = np.empty(len(rays), np.uint32)
    lib().orc_trace_ref_bvh2(_ptr(np.ascontiguousarray(nodes2)), _ptr(np.ascontiguousarray(tris)), _ptr(rays),
                             len(rays), t_eps, _ptr(flags), threads())
    return flags


def trace_bvh4(nodes4, tris, perm, rays, flags=0, want_bary=False, want_stats=False):
    rays = np.ascontiguousarray(rays)
    hits = np.empty(len(rays), HIT)
    bary = np.empty(2 * len(rays), np.float32) if want_bary else None
    stats = np.empty(len(rays), STATS) if want_stats else None
    perm = None if perm is None else np.ascontiguousarray(perm, dtype=np.uint32)
    lib().orc_trace_bvh4(_ptr(np.ascontiguousarray(nodes4)), _ptr(np.ascontiguousarray(tris)), _ptr(perm),
                         _ptr(rays), len(rays), flags, _ptr(hits), _ptr(bary), _ptr(stats), threads())
    return hits, bary, stats


def trace_radv(img, rays, flags=0, want_bary=False):
    rays = np.ascontiguousarray(rays)
    hits = np.empty(len(rays), HIT)
    bary = np.empty(2 * len(rays), np.float32) if want_bary else None
    lib().orc_trace_radv(_ptr(np.ascontiguousarray(img)), _ptr(rays), len(rays), flags, _ptr(hits), _ptr(bary),
                         threads())
    return hits, bary


def tlas_trace(blas, blas_of, transforms, ids, masks, rays, flags=0, cull=0xFF):
    """Two-level scene traversal.  blas: list of (nodes4, tris, perm) arrays;
    instance i uses blas[blas_of[i]] with the row-major 3x4 transforms[i]."""
    keep = [tuple(np.ascontiguousarray(x) for x in b) for b in blas]
    nodes = np.array([k[0].ctypes.data for k in keep], np.uint64)
    tris = np.array([k[1].ctypes.data for k in keep], np.uint64)
    perm = np.array([k[2].ctypes.data for k in keep], np.uint64)
    bo = np.ascontiguousarray(blas_of, np.uint32)
    xf = np.ascontiguousarray(transforms, np.float32).reshape(-1)
    ids = np.ascontiguousarray(ids, np.uint32)
    masks = np.ascontiguousarray(masks, np.uint32)
    rays = np.ascontiguousarray(rays)
    hits = np.empty(len(rays), HIT)
    lib().orc_tlas_trace(_ptr(nodes), _ptr(tris), _ptr(perm), _ptr(bo), _ptr(xf), _ptr(ids), _ptr(masks), len(bo),
                         _ptr(rays), len(rays), flags, cull, _ptr(hits), threads())
    return hits


def gbuffer_depth(gbuf, view_proj):
    g = np.ascontiguousarray(gbuf)
    vp = np.ascontiguousarray(view_proj, np.float32).reshape(-1)
    d = np.empty(len(g), np.float32)
    lib().orc_gbuffer_depth(_ptr(g), len(g), _ptr(vp), _ptr(d))
    return d


def blur_ao(ao, depth, w, h, dx, dy, threshold):
    a = np.ascontiguousarray(ao, np.float32)
    d = np.ascontiguousarray(depth, np.float32)
    out = np.empty(w * h, np.float32)
    lib().orc_blur_ao(_ptr(a), _ptr(d), _ptr(out), w, h, dx, dy, threshold)
    return out


def gen_mesh_rays(pos, idx, kind, seed, count):
    """Rays of a generated serving request (kind 1 shadow, 2 AO, 3 closest)
    and their any-hit flags."""
    pos = np.ascontiguousarray(pos, np.float32)
    idx = np.ascontiguousarray(idx, np.uint32)
    rays = np.empty(count, RAY)
    anyf = np.empty(count, np.uint32)
    lib().orc_gen_mesh_rays(_ptr(pos), _ptr(idx), len(idx.reshape(-1)) // 3, kind, seed, count, _ptr(rays),
                            _ptr(anyf))
    return rays, anyf


def gen_rays_procedural(cam, look, count, coherent):
    rays = np.empty(count, RAY)
    c = np.asarray(cam, np.float32)
    l = np.asarray(look, np.float32)
    lib().orc_gen_rays_procedural(_ptr(c), _ptr(l), count, 1 if coherent else 0, _ptr(rays))
    return rays


GBUFFER_PX = np.dtype([("pos", "<f4", 3), ("vis", "<u4"), ("nrm", "<f4", 3), ("t", "<f4")])


def render_gbuffer(nodes4, tris, perm, cam, pixels=None):
    """cam: a Camera (this module's or rq's) ctypes structure; pixels: uint32
    indices or None."""
    import ctypes as CC
    L = lib()
    npix = cam.width * cam.height if pixels is None else len(pixels)
    out = np.empty(npix, GBUFFER_PX)
    px = None if pixels is None else np.ascontiguousarray(pixels, np.uint32)
    L.orc_render_gbuffer(_ptr(np.ascontiguousarray(nodes4)), _ptr(np.ascontiguousarray(tris)),
                         _ptr(None if perm is None else np.ascontiguousarray(perm, np.uint32)),
                         CC.cast(CC.byref(cam), _P), _ptr(px), npix, _ptr(out), threads())
    return out


def render_shadow_ao(nodes4, tris, gbuf_full, params, pixels=None):
    import ctypes as CC
    L = lib()
    npix = params.width * params.height if pixels is None else len(pixels)
    mask = np.empty(npix, np.uint32)
    ao = np.empty(npix, np.float32)
    rays = np.zeros(1, np.uint64)
    px = None if pixels is None else np.ascontiguousarray(pixels, np.uint32)
    L.orc_render_shadow_ao(_ptr(np.ascontiguousarray(nodes4)), _ptr(np.ascontiguousarray(tris)),
                           _ptr(np.ascontiguousarray(gbuf_full)), CC.cast(CC.byref(params), _P), _ptr(px), npix,
                           _ptr(mask), _ptr(ao), _ptr(rays), threads())
    return mask, ao, int(rays[0])


def sincos(x):
    s, c = C.c_float(), C.c_float()
    lib().orc_sincos(float(x), C.byref(s), C.byref(c))
    return s.value, c.value


# ------------------------------------------------------------ reference --

def ref_terrain(target, size=100.0):
    R = ref()
    nv, ni = np.zeros(1, np.uint32), np.zeros(1, np.uint32)
    R.ref_terrain(target, size, None, None, _ptr(nv), _ptr(ni))
    pos = np.empty(3 * int(nv[0]), np.float32)
    idx = np.empty(int(ni[0]), np.uint32)
    R.ref_terrain(target, size, _ptr(pos), _ptr(idx), _ptr(nv), _ptr(ni))
    return pos, idx


def ref_build(pos, idx, max_leaf=4, collapse=True):
    """The reference's SoftwareBVH::build (+ SoftwareBVH4::fromBVH2)."""
    R = ref()
    pos = np.ascontiguousarray(pos, dtype=np.float32)
    idx = np.ascontiguousarray(idx, dtype=np.uint32)
    h = R.ref_build(_ptr(pos), pos.size // 3, _ptr(idx), idx.size // 3, max_leaf, 1 if collapse else 0)
    assert h
    try:
        n2, nt, n4 = np.zeros(1, np.uint32), np.zeros(1, np.uint32), np.zeros(1, np.uint32)
        R.ref_counts(h, _ptr(n2), _ptr(nt), _ptr(n4))
        nodes2 = np.empty(int(n2[0]), BVH2_NODE)
        tris = np.empty(int(nt[0]), TRIANGLE)
        nodes4 = np.empty(int(n4[0]), BVH4_NODE)
        R.ref_copy(h, _ptr(nodes2), _ptr(tris), _ptr(nodes4) if n4[0] else None)
    finally:
        R.ref_free(h)
    return nodes2, tris, nodes4


def ref_collapse(nodes2, tris):
    R = ref()
    nodes2 = np.ascontiguousarray(nodes2)
    tris = np.ascontiguousarray(tris)
    h = R.ref_collapse(_ptr(nodes2), len(nodes2), _ptr(tris), len(tris))
    try:
        n2, nt, n4 = np.zeros(1, np.uint32), np.zeros(1, np.uint32), np.zeros(1, np.uint32)
        R.ref_counts(h, _ptr(n2), _ptr(nt), _ptr(n4))
        nodes4 = np.empty(int(n4[0]), BVH4_NODE)
        R.ref_copy(h, None, None, _ptr(nodes4))
    finally:
        R.ref_free(h)
    return nodes4


def ref_tree_layout(n):
    R = ref()
    tb, nl, ts = np.zeros(1, np.uint32), np.zeros(1, np.uint32), np.zeros(1, np.uint32)
    counts, offs = np.zeros(32, np.uint32), np.zeros(32, np.uint32)
    R.ref_tree_layout(n, _ptr(tb), _ptr(nl), _ptr(ts), _ptr(counts), _ptr(offs))
    L = int(nl[0])
    return dict(total_boxes=int(tb[0]), num_levels=L, total_size=int(ts[0]),
                counts=counts[:L].tolist(), offsets=offs[:L].tolist())


def ref_dynamic_grid(n, time_val=0.0, extent=2.0):
    R = ref()
    tri9 = np.empty(9 * n, np.float32)
    cen = np.empty(3 * n, np.float32)
    R.ref_dynamic_grid(n, time_val, extent, _ptr(tri9), _ptr(cen))
    return tri9, cen


def ref_dump_bvh_structure(image):
    """The reference's text dump of a RADV image (bytes / uint8 array)."""
    R = ref()
    img = np.ascontiguousarray(np.frombuffer(bytes(image), np.uint8))
    n = R.ref_dump_bvh_structure(_ptr(img), len(img), None, 0)
    buf = C.create_string_buffer(n + 1)
    R.ref_dump_bvh_structure(_ptr(img), len(img), buf, n + 1)
    return buf.value.decode()


def recover_perm(tris_leaf_order, pos, idx):
    """The reference discards the leaf-order permutation
    (common/software_bvh.hpp:60-63); recover it by matching the 9 float bit
    patterns of every leaf triangle to the input triangles.  Asserts unique."""
    tl = np.ascontiguousarray(tris_leaf_order)
    pos = np.ascontiguousarray(pos, np.float32).reshape(-1)
    idx = np.ascontiguousarray(idx, np.uint32).reshape(-1)
    perm = np.empty(len(tl), np.uint32)
    rc = lib().orc_recover_perm(_ptr(tl), len(tl), _ptr(pos), _ptr(idx), idx.size // 3, _ptr(perm))
    assert rc == 0, "input triangles are not unique by vertex bits, or a leaf triangle is not an input triangle"
    return perm


# ------------------------------------------------------- frame ray makers --

class Camera(C.Structure):
    """rq_camera (include/rq.h)."""
    _fields_ = [("inv_view_proj", C.c_float * 16), ("cam_pos", C.c_float * 3), ("width", C.c_uint32),
                ("height", C.c_uint32), ("jitter", C.c_uint32), ("seed", C.c_uint32), ("tmin", C.c_float),
                ("tmax", C.c_float), ("flags", C.c_uint32)]


class Light(C.Structure):
    _fields_ = [("pos", C.c_float * 3), ("radius", C.c_float)]


class ShadeParams(C.Structure):
    """rq_shade_params (include/rq.h)."""
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("num_lights", C.c_uint32), ("ao_spp", C.c_uint32),
                ("ao_tmax", C.c_float), ("ao_tmin", C.c_float), ("ao_bias", C.c_float), ("shadow_tmin", C.c_float),
                ("shadow_bias", C.c_float), ("flags", C.c_uint32), ("lights", Light * 32)]


class ReflectParams(C.Structure):
    """rq_reflect_params (include/rq.h)."""
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("cam_pos", C.c_float * 3), ("tmin", C.c_float),
                ("tmax", C.c_float), ("bias", C.c_float), ("flags", C.c_uint32)]


class AoDepthParams(C.Structure):
    """rq_ao_depth_params (include/rq.h)."""
    _fields_ = [("inv_view_proj", C.c_float * 16), ("cam_pos", C.c_float * 3), ("width", C.c_uint32),
                ("height", C.c_uint32), ("spp", C.c_uint32), ("max_distance", C.c_float), ("tmin", C.c_float),
                ("bias", C.c_float), ("flags", C.c_uint32)]


def _ref_of(s):
    return C.cast(C.byref(s), _P)


def scene_grid(qx, qy, x0=-1.0, x1=1.0, y0=-1.0, y1=1.0, amp=0.2, freq=3.0, sigma=0.01, seed=0):
    """The benchmark's height-field grid, generated by the oracle's own copy of
    the generator: float32 [V,3] positions, uint32 [T,3] indices."""
    pos = np.empty(((qx + 1) * (qy + 1), 3), np.float32)
    idx = np.empty((2 * qx * qy, 3), np.uint32)
    assert lib().orc_scene_grid(qx, qy, x0, x1, y0, y1, amp, freq, sigma, seed, _ptr(pos), _ptr(idx)) == 0
    return pos, idx


def camera_look_at(eye, target, up, fovy_deg, width, height, jitter=False, seed=0, flags=0):
    cam = Camera()
    f3 = C.c_float * 3
    assert lib().orc_camera_look_at(C.cast(f3(*eye), _P), C.cast(f3(*target), _P), C.cast(f3(*up), _P), fovy_deg,
                                    width, height, _ref_of(cam)) == 0
    cam.jitter, cam.seed, cam.flags = (1 if jitter else 0), seed, flags
    return cam


def shade_params(width, height, lights, ao_spp=1, ao_tmax=0.5, flags=0):
    p = ShadeParams()
    p.width, p.height, p.num_lights, p.ao_spp = width, height, len(lights), ao_spp
    p.ao_tmax, p.ao_tmin, p.ao_bias = ao_tmax, 0.01, 0.03
    p.shadow_tmin, p.shadow_bias, p.flags = 0.01, 0.04, flags
    for k, (x, y, z, r) in enumerate(lights):
        p.lights[k].pos[0], p.lights[k].pos[1], p.lights[k].pos[2], p.lights[k].radius = x, y, z, r
    return p


def reflect_params(cam, flags=0, tmin=0.02, tmax=100.0, bias=0.04):
    p = ReflectParams()
    p.width, p.height = cam.width, cam.height
    for k in range(3):
        p.cam_pos[k] = cam.cam_pos[k]
    p.tmin, p.tmax, p.bias, p.flags = tmin, tmax, bias, flags
    return p


def ao_depth_params(cam, spp=1, max_distance=0.5, flags=0, tmin=0.01, bias=0.03):
    p = AoDepthParams()
    for k in range(16):
        p.inv_view_proj[k] = cam.inv_view_proj[k]
    for k in range(3):
        p.cam_pos[k] = cam.cam_pos[k]
    p.width, p.height, p.spp, p.max_distance = cam.width, cam.height, spp, max_distance
    p.tmin, p.bias, p.flags = tmin, bias, flags
    return p


# The 1080p shadows + AO frame (the benchmark's headline workload), built
# here from the oracle's generators so a process can set it up without the
# engine.  The same constants define it in the engine's workload module; a
# CPU test checks that both give the same bytes.
SHADOW_QUADS, SHADOW_SEED = 1118, 1
SHADOW_EYE, SHADOW_TARGET, SHADOW_UP, SHADOW_FOVY = (0.0, -0.6, 2.6), (0.0, 0.0, 0.0), (0.0, 0.0, 1.0), 20.0


def shadow_lights(n=16, seed=1):
    rng = np.random.default_rng(seed)
    xy = rng.uniform(-1.0, 1.0, size=(n, 2))
    z = rng.uniform(2.0, 2.5, size=n)
    return [(float(xy[k, 0]), float(xy[k, 1]), float(z[k]), 100.0) for k in range(n)]


def shadow_frame_inputs(width=1920, height=1080):
    """(positions, indices, camera, shade params) of the 1080p frame."""
    pos, idx = scene_grid(SHADOW_QUADS, SHADOW_QUADS, seed=SHADOW_SEED)
    cam = camera_look_at(SHADOW_EYE, SHADOW_TARGET, SHADOW_UP, SHADOW_FOVY, width, height)
    params = shade_params(width, height, shadow_lights(16), ao_spp=1, ao_tmax=0.5)
    return pos, idx, cam, params


def camera_rays(cam, pixels=None):
    npix = cam.width * cam.height if pixels is None else len(pixels)
    px = None if pixels is None else np.ascontiguousarray(pixels, np.uint32)
    rays = np.empty(npix, RAY)
    lib().orc_camera_rays(_ref_of(cam), _ptr(px), npix, _ptr(rays))
    return rays


def shade_rays(gbuf_full, params, pixels):
    """The frame's secondary rays of the listed pixels, in casting order:
    (rays, index into pixels, slot: light k or 32 + AO sample)."""
    g = np.ascontiguousarray(gbuf_full)
    px = np.ascontiguousarray(pixels, np.uint32)
    cap = len(px) * (params.num_lights + params.ao_spp)
    rays = np.empty(max(1, cap), RAY)
    rpx = np.empty(max(1, cap), np.uint32)
    slot = np.empty(max(1, cap), np.uint32)
    cnt = np.zeros(1, np.uint64)
    lib().orc_shade_rays(_ptr(g), _ref_of(params), _ptr(px), len(px), _ptr(rays), _ptr(rpx), _ptr(slot), cap,
                         _ptr(cnt))
    n = int(cnt[0])
    return rays[:n].copy(), rpx[:n].copy(), slot[:n].copy()


def render_reflect(nodes4, tris, perm, gbuf_full, params, pixels=None, want_rays=False):
    g = np.ascontiguousarray(gbuf_full)
    npix = params.width * params.height if pixels is None else len(pixels)
    px = None if pixels is None else np.ascontiguousarray(pixels, np.uint32)
    hits = np.empty(npix, HIT)
    rays = np.empty(npix, RAY) if want_rays else None
    lib().orc_render_reflect(_ptr(np.ascontiguousarray(nodes4)), _ptr(np.ascontiguousarray(tris)),
                             _ptr(None if perm is None else np.ascontiguousarray(perm, np.uint32)), _ptr(g),
                             _ref_of(params), _ptr(px), npix, _ptr(hits), _ptr(rays), threads())
    return (hits, rays) if want_rays else hits


def render_ao_depth(nodes4, tris, depth, params, pixels=None):
    d = np.ascontiguousarray(depth, np.float32)
    npix = params.width * params.height if pixels is None else len(pixels)
    px = None if pixels is None else np.ascontiguousarray(pixels, np.uint32)
    ao = np.empty(npix, np.float32)
    rays = np.zeros(1, np.uint64)
    lib().orc_render_ao_depth(_ptr(np.ascontiguousarray(nodes4)), _ptr(np.ascontiguousarray(tris)), _ptr(d),
                              _ref_of(params), _ptr(px), npix, _ptr(ao), _ptr(rays), threads())
    return ao, int(rays[0])


def ao_depth_rays(depth, params, pixels):
    d = np.ascontiguousarray(depth, np.float32)
    px = np.ascontiguousarray(pixels, np.uint32)
    cap = len(px) * max(1, params.spp)
    rays = np.empty(max(1, cap), RAY)
    rpx = np.empty(max(1, cap), np.uint32)
    cnt = np.zeros(1, np.uint64)
    lib().orc_ao_depth_rays(_ptr(d), _ref_of(params), _ptr(px), len(px), _ptr(rays), _ptr(rpx), cap, _ptr(cnt))
    n = int(cnt[0])
    return rays[:n].copy(), rpx[:n].copy()


def refit(pos, idx, perm, nodes2, nodes4):
    """Boxes and leaf triangles of a built tree moved to new vertex
    positions, topology kept: (tris, nodes2, nodes4) as new arrays."""
    pos = np.ascontiguousarray(pos, np.float32).reshape(-1)
    idx = np.ascontiguousarray(idx, np.uint32).reshape(-1)
    perm = np.ascontiguousarray(perm, np.uint32)
    n2 = np.array(nodes2, copy=True)
    n4 = np.array(nodes4, copy=True)
    tris = np.empty(len(perm), TRIANGLE)
    lib().orc_refit(_ptr(pos), _ptr(idx), _ptr(perm), len(perm), _ptr(tris), _ptr(n2), len(n2), _ptr(n4), len(n4))
    return tris, n2, n4
