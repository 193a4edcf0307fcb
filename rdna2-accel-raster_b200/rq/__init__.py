"""Python host mirror of librq's C ABI (include/rq.h), through ctypes.

The engine itself is librq.so (C++ host + sm_100a CUDA kernels).  This module
binds it for tests, benchmarks and Python callers: device buffers are torch
CUDA tensors, passed as raw pointers.  There is no CPU or PyTorch fallback —
loading fails loudly when librq.so is missing or no sm_100 device exists.

Layouts (include/rq_layouts.h):
  rays  float32 [n, 8]: origin xyz, tmin, direction xyz, tmax   (rq_ray)
  hits  int32   [n, 4]: hit, t (float bits), instance id, primitive id (rq_hit)
  stats int32   [n, 4]: hit, box tests, triangle tests, 0        (rq_ray_stats)
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(HERE), "librq.so")

RQ_OK = 0
RQ_ERR_INVALID_ARG = 1
RQ_ERR_SIZE = 2
RQ_ERR_CUDA = 3
RQ_ERR_OOM = 4
RQ_ERR_DEVICE_TIMEOUT = 5
RQ_ERR_UNSUPPORTED = 6
RQ_ERR_BUDGET = 7
RQ_ERR_NO_DEVICE = 8
RQ_ERR_STATE = 9
RQ_ERR_CANCELLED = 10
RQ_FAULT_ALLOC = 1
RQ_FAULT_LAUNCH = 2

RQ_BUILD_BVH4 = 1
RQ_BUILD_MEDIAN = 2
RQ_BUILD_SAH = 4
SAH_SUBTREE_MAX = 16384
RQ_TRACE_CLOSEST = 0
RQ_TRACE_ANY = 1
RQ_TRI_WATERTIGHT = 0
RQ_TRI_MT = 2
RQ_SHADE_COUNT_TESTS = 16

# numpy mirrors of the byte layouts
BVH2_NODE = np.dtype([("aabb_min", "<f4", 3), ("left_child", "<i4"), ("aabb_max", "<f4", 3), ("right_child", "<i4")])
TRIANGLE = np.dtype([("v0", "<f4", 4), ("v1", "<f4", 4), ("v2", "<f4", 4)])
BVH4_NODE = np.dtype([("min_x", "<f4", 4), ("max_x", "<f4", 4), ("min_y", "<f4", 4), ("max_y", "<f4", 4),
                      ("min_z", "<f4", 4), ("max_z", "<f4", 4), ("child_index", "<i4", 4), ("child_count", "<i4", 4)])
RAY = np.dtype([("org", "<f4", 3), ("tmin", "<f4"), ("dir", "<f4", 3), ("tmax", "<f4")])
HIT = np.dtype([("hit", "<u4"), ("t", "<f4"), ("instance_id", "<u4"), ("primitive_id", "<u4")])
STATS = np.dtype([("hit", "<u4"), ("box_tests", "<u4"), ("tri_tests", "<u4"), ("pad", "<u4")])


class RqError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"rq status {status}: {msg}")
        self.status = status


class BvhInfo(C.Structure):
    _fields_ = [("num_triangles", C.c_uint32), ("num_nodes2", C.c_uint32), ("num_nodes4", C.c_uint32),
                ("depth4", C.c_uint32), ("max_leaf", C.c_uint32), ("stack_bound", C.c_uint32),
                ("device_bytes", C.c_uint64)]


class RadvCheck(C.Structure):
    _fields_ = [("header_ok", C.c_uint32), ("reserved", C.c_uint32)] + [
        (k, C.c_uint64) for k in ("box_nodes", "triangle_nodes", "box_children", "triangle_children", "bad_offsets",
                                  "bad_boxes", "box_refs_wrong", "triangle_refs_wrong", "ids_wrong")]


class RadvLayout(C.Structure):
    _fields_ = [("num_triangles", C.c_uint32), ("total_boxes", C.c_uint32), ("num_levels", C.c_uint32),
                ("total_as_size_lo", C.c_uint32), ("total_as_size", C.c_uint64),
                ("level_offsets", C.c_uint32 * 16), ("level_counts", C.c_uint32 * 16)]


class Camera(C.Structure):
    _fields_ = [("inv_view_proj", C.c_float * 16), ("cam_pos", C.c_float * 3), ("width", C.c_uint32),
                ("height", C.c_uint32), ("jitter", C.c_uint32), ("seed", C.c_uint32), ("tmin", C.c_float),
                ("tmax", C.c_float), ("flags", C.c_uint32)]


class Light(C.Structure):
    _fields_ = [("pos", C.c_float * 3), ("radius", C.c_float)]


MAX_LIGHTS = 32


class ShadeParams(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("num_lights", C.c_uint32), ("ao_spp", C.c_uint32),
                ("ao_tmax", C.c_float), ("ao_tmin", C.c_float), ("ao_bias", C.c_float), ("shadow_tmin", C.c_float),
                ("shadow_bias", C.c_float), ("flags", C.c_uint32), ("lights", Light * MAX_LIGHTS)]


class ReflectParams(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("cam_pos", C.c_float * 3), ("tmin", C.c_float),
                ("tmax", C.c_float), ("bias", C.c_float), ("flags", C.c_uint32)]


class AoDepthParams(C.Structure):
    _fields_ = [("inv_view_proj", C.c_float * 16), ("cam_pos", C.c_float * 3), ("width", C.c_uint32),
                ("height", C.c_uint32), ("spp", C.c_uint32), ("max_distance", C.c_float), ("tmin", C.c_float),
                ("bias", C.c_float), ("flags", C.c_uint32)]


GBUFFER_PX = np.dtype([("pos", "<f4", 3), ("vis", "<u4"), ("nrm", "<f4", 3), ("t", "<f4")])


class MeshDesc(C.Structure):
    _fields_ = [("vertex_offset", C.c_uint32), ("num_vertices", C.c_uint32), ("triangle_offset", C.c_uint32),
                ("num_triangles", C.c_uint32)]


class Instance(C.Structure):
    _fields_ = [("transform", C.c_float * 12), ("instance_id", C.c_uint32), ("mask", C.c_uint32),
                ("blas", C.c_void_p)]


class CameraTuning(C.Structure):
    _fields_ = [("engine", C.c_uint32), ("refill_min", C.c_uint32), ("leaf_batch", C.c_uint32)]


class TraceTuning(C.Structure):
    _fields_ = [("threads", C.c_uint32), ("chunk", C.c_uint32), ("reg_cap", C.c_uint32), ("top_levels", C.c_uint32),
                ("speculative", C.c_uint32), ("refill_min", C.c_uint32), ("leaf_batch", C.c_uint32)]


class BatchTuning(C.Structure):
    _fields_ = [("build_threads", C.c_uint32), ("build_blocks", C.c_uint32), ("trace_threads", C.c_uint32),
                ("trace_chunk", C.c_uint32), ("trace_reg_cap", C.c_uint32), ("trace_blocks_per_sm", C.c_uint32),
                ("stack_entries", C.c_uint32), ("max_build_blocks", C.c_uint32), ("build_ms", C.c_float),
                ("trace_ms", C.c_float), ("trace_refill_min", C.c_uint32), ("build_cluster", C.c_uint32),
                ("cluster_min_tris", C.c_uint32)]


class ServerConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_uint64), ("mode", C.c_uint32), ("slots", C.c_uint32),
                ("max_wave_rays", C.c_uint32), ("max_wave_requests", C.c_uint32), ("max_leaf", C.c_uint32),
                ("trace_flags", C.c_uint32), ("rebuild", C.c_uint32)]


class Request(C.Structure):
    _fields_ = [("mesh", C.c_uint32), ("kind", C.c_uint32), ("num_rays", C.c_uint32), ("seed", C.c_uint32),
                ("flags", C.c_uint32), ("reserved", C.c_uint32), ("rays", C.c_void_p), ("hits", C.c_void_p),
                ("user", C.c_uint64)]


class Completion(C.Structure):
    _fields_ = [("ticket", C.c_uint64), ("user", C.c_uint64), ("status", C.c_int32), ("built", C.c_uint32),
                ("t_submit", C.c_double), ("t_admit", C.c_double), ("t_done", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in ("submitted", "completed", "failed", "launches", "builds", "evictions",
                                          "rays", "resident_bytes", "peak_resident_bytes",
                                          "max_requests_per_launch", "max_launches_in_flight")]


_P = C.c_void_p
_U32 = C.c_uint32
# (name, restype, argtypes) for every entry point in include/rq.h
SIGNATURES = [
    ("rq_ctx_create", C.c_int, [C.c_int, C.POINTER(_P)]),
    ("rq_ctx_destroy", C.c_int, [_P]),
    ("rq_status_string", C.c_char_p, [C.c_int]),
    ("rq_ctx_last_error", C.c_char_p, [_P]),
    ("rq_ctx_check", C.c_int, [_P, _P]),
    ("rq_ctx_scratch_bytes", C.c_uint64, [_P]),
    ("rq_ctx_trace_tuning_get", C.c_int, [_P, C.POINTER(TraceTuning)]),
    ("rq_ctx_trace_tuning_set", C.c_int, [_P, C.POINTER(TraceTuning)]),
    ("rq_ctx_camera_tuning_get", C.c_int, [_P, C.POINTER(CameraTuning)]),
    ("rq_ctx_camera_tuning_set", C.c_int, [_P, C.POINTER(CameraTuning)]),
    ("rq_debug_wait_timeout", C.c_int, [_P, _P, _U32, _P]),
    ("rq_scene_grid", C.c_int, [_U32, _U32, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float,
                                C.c_float, C.c_uint64, _P, _P]),
    ("rq_scene_rays_down", C.c_int, [_U32, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float,
                                     C.c_float, C.c_float, C.c_uint64, _P]),
    ("rq_deform_wave", C.c_int, [_P, _P, _P, _U32, C.c_float, C.c_float, C.c_float, _P]),
    ("rq_deform_wave_step", C.c_int, [_P, _P, _P, _U32, _P, C.c_float, C.c_float, C.c_float, _P]),
    ("rq_build", C.c_int, [_P, _P, _U32, _U32, _P, _U32, _U32, _U32, C.POINTER(_P), _P]),
    ("rq_collapse4", C.c_int, [_P, _P, _P]),
    ("rq_refit", C.c_int, [_P, _P, _P, _U32, _P, _P]),
    ("rq_bvh_import2", C.c_int, [_P, _P, _U32, _P, _P, _U32, C.POINTER(_P), _P]),
    ("rq_bvh_import4", C.c_int, [_P, _P, _U32, _P, _P, _U32, C.POINTER(_P), _P]),
    ("rq_bvh_info_get", C.c_int, [_P, C.POINTER(BvhInfo)]),
    ("rq_bvh_download", C.c_int, [_P, C.c_int, _P, _U32, _P, _U32, _P, _U32, _P, _U32]),
    ("rq_bvh_download_sort", C.c_int, [_P, C.c_int, _P, _P, _U32]),
    ("rq_bvh_destroy", C.c_int, [_P]),
    ("rq_trace", C.c_int, [_P, _P, _P, _U32, _U32, _P, _P, _P, _P]),
    ("rq_trace_ref_bvh4", C.c_int, [_P, _P, _P, _P, _U32, _P, _P, _P]),
    ("rq_trace_ref_bvh2", C.c_int, [_P, _P, _P, _P, _U32, C.c_float, _P, _P]),
    ("rq_gen_rays_procedural", C.c_int, [_P, _P, _P, _U32, _U32, _P, _P]),
    ("rq_camera_look_at", C.c_int, [_P, _P, _P, C.c_float, _U32, _U32, C.POINTER(Camera)]),
    ("rq_render_gbuffer", C.c_int, [_P, _P, C.POINTER(Camera), _P, _P]),
    ("rq_render_shadow_ao", C.c_int, [_P, _P, _P, C.POINTER(ShadeParams), _P, _P, _P, _P]),
    ("rq_render_reflect", C.c_int, [_P, _P, _P, C.POINTER(ReflectParams), _P, _P]),
    ("rq_render_ao_depth", C.c_int, [_P, _P, _P, C.POINTER(AoDepthParams), _P, _P, _P]),
    ("rq_gbuffer_depth", C.c_int, [_P, _P, _U32, _P, _P, _P]),
    ("rq_blur_ao", C.c_int, [_P, _P, _P, _P, _U32, _U32, C.c_int, C.c_int, C.c_float, _P]),
    ("rq_radv_layout_get", C.c_int, [_U32, C.POINTER(RadvLayout)]),
    ("rq_radv_size", C.c_uint64, [_U32]),
    ("rq_build_radv", C.c_int, [_P, _P, _U32, _P, C.c_uint64, _P]),
    ("rq_refit_radv", C.c_int, [_P, _P, _U32, _P, C.c_uint64, _P]),
    ("rq_trace_radv", C.c_int, [_P, _P, C.c_uint64, _P, _U32, _U32, _P, _P, _P]),
    ("rq_radv_describe", C.c_int, [_P, C.c_uint64, _P, C.c_uint64, C.POINTER(C.c_uint64)]),
    ("rq_radv_validate", C.c_int, [_P, _P, C.c_uint64, C.POINTER(RadvCheck), _P]),
    ("rq_build_radv_noalloc", C.c_int, [_P, _U32, _P, C.c_uint64, _P]),
    ("rq_batch_create", C.c_int, [_P, C.POINTER(MeshDesc), _U32, _U32, C.POINTER(_P)]),
    ("rq_batch_build", C.c_int, [_P, _P, _P, _U32, _P, _P]),
    ("rq_batch_trace", C.c_int, [_P, _P, _P, _P, _P, _U32, _U32, _P, _P, _P]),
    ("rq_batch_info_get", C.c_int, [_P, _U32, C.POINTER(BvhInfo)]),
    ("rq_batch_download", C.c_int, [_P, _U32, C.c_int, _P, _U32, _P, _U32, _P, _U32, _P, _U32]),
    ("rq_batch_destroy", C.c_int, [_P]),
    ("rq_tlas_build", C.c_int, [_P, C.POINTER(Instance), _U32, C.POINTER(_P), _P]),
    ("rq_tlas_trace", C.c_int, [_P, _P, _P, _U32, _U32, _U32, _P, _P]),
    ("rq_tlas_destroy", C.c_int, [_P]),
    ("rq_batch_tuning_get", C.c_int, [_P, C.POINTER(BatchTuning)]),
    ("rq_batch_tuning_set", C.c_int, [_P, C.POINTER(BatchTuning)]),
    ("rq_batch_autotune", C.c_int, [_P, _P, _P, _U32, _P, _P, _P, _P, _U32, _P, _U32, C.POINTER(BatchTuning), _U32,
                                    C.POINTER(_U32), _P]),
    # include/rq_serve.h
    ("rq_server_create", C.c_int, [C.c_int, C.POINTER(ServerConfig), C.POINTER(_P)]),
    ("rq_server_destroy", C.c_int, [_P]),
    ("rq_server_add_mesh", C.c_int, [_P, _P, _U32, _P, _U32, C.POINTER(_U32)]),
    ("rq_server_mesh_bytes", C.c_uint64, [_U32, _U32]),
    ("rq_server_submit", C.c_int, [_P, C.POINTER(Request), C.POINTER(C.c_uint64)]),
    ("rq_server_replay", C.c_int, [_P, C.POINTER(Request), _P, _U32, _P]),
    ("rq_server_poll", C.c_int, [_P, C.POINTER(Completion), _U32, C.POINTER(_U32)]),
    ("rq_server_drain", C.c_int, [_P, _U32]),
    ("rq_server_now", C.c_double, [_P]),
    ("rq_server_stats_get", C.c_int, [_P, C.POINTER(ServerStats)]),
    ("rq_server_last_error", C.c_char_p, [_P]),
    ("rq_gen_mesh_rays", C.c_int, [_P, _P, _P, _U32, _U32, _U32, _U32, _P, _P, _P]),
    ("rq_server_cancel", C.c_int, [_P, C.c_uint64]),
    ("rq_server_inject_fault", C.c_int, [_P, _U32, _U32]),
]

RQ_RAYS_BUFFER = 0
RQ_RAYS_SHADOW = 1
RQ_RAYS_AO = 2
RQ_RAYS_CLOSEST = 3
RQ_SERVE_BATCHED = 0
RQ_SERVE_PLAIN = 1

RADV_NOALLOC_MAX_TRIANGLES = 1 << 24

_lib = None


def lib():
    """Load librq.so (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"librq.so not built at {LIB_PATH}: run `make -C rdna2-accel-raster_b200/csrc`")
        L = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _ptr(t):
    """Raw pointer of a torch tensor or numpy array (None -> NULL)."""
    if t is None:
        return None
    if isinstance(t, np.ndarray):
        return t.ctypes.data_as(_P)
    return _P(t.data_ptr())


def _count(t, item_bytes):
    """Number of `item_bytes` records in a tensor/array, whatever its dtype."""
    nbytes = t.nbytes if isinstance(t, np.ndarray) else t.numel() * t.element_size()
    if nbytes % item_bytes:
        raise ValueError(f"buffer of {nbytes} bytes is not a whole number of {item_bytes}-byte records")
    return nbytes // item_bytes


def _stream(stream):
    if stream is None:
        import torch
        return _P(torch.cuda.current_stream().cuda_stream)
    if isinstance(stream, int):
        return _P(stream)
    return _P(stream.cuda_stream)


class Context:
    """An rq_ctx on one CUDA device (owns scratch memory)."""

    def __init__(self, device=0):
        h = _P()
        rc = lib().rq_ctx_create(device, C.byref(h))
        if rc != RQ_OK:
            raise RqError(rc, lib().rq_status_string(rc).decode())
        self.h = h
        self.device = device

    def close(self):
        if self.h:
            lib().rq_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, rc, what=""):
        if rc != RQ_OK:
            msg = lib().rq_ctx_last_error(self.h).decode() if self.h else ""
            raise RqError(rc, f"{what}: {lib().rq_status_string(rc).decode()} ({msg})")

    def sync_check(self, stream=None):
        """Synchronise and raise if a device-side bounded wait failed."""
        self.check(lib().rq_ctx_check(self.h, _stream(stream)), "device error word")

    def scratch_bytes(self):
        return int(lib().rq_ctx_scratch_bytes(self.h))

    def trace_tuning(self):
        """Launch shape of the shadow/AO traversal (rq_trace_tuning)."""
        t = TraceTuning()
        self.check(lib().rq_ctx_trace_tuning_get(self.h, C.byref(t)), "rq_ctx_trace_tuning_get")
        return {"threads": t.threads, "chunk": t.chunk, "reg_cap": t.reg_cap, "top_levels": t.top_levels,
                "speculative": t.speculative, "refill_min": t.refill_min, "leaf_batch": t.leaf_batch}

    def debug_wait_timeout(self, flag, limit, stream=None):
        """One bounded device wait on flag (int32 CUDA tensor) leaving 0."""
        self.check(lib().rq_debug_wait_timeout(self.h, _ptr(flag), limit, _stream(stream)), "rq_debug_wait_timeout")

    def set_trace_tuning(self, threads=128, chunk=32, reg_cap=80, top_levels=0, speculative=0, refill_min=1,
                         leaf_batch=0):
        t = TraceTuning(threads, chunk, reg_cap, top_levels, speculative, refill_min, leaf_batch)
        self.check(lib().rq_ctx_trace_tuning_set(self.h, C.byref(t)), "rq_ctx_trace_tuning_set")

    def camera_tuning(self):
        t = CameraTuning()
        self.check(lib().rq_ctx_camera_tuning_get(self.h, C.byref(t)), "rq_ctx_camera_tuning_get")
        return {"engine": t.engine, "refill_min": t.refill_min, "leaf_batch": t.leaf_batch}

    def set_camera_tuning(self, engine=0, refill_min=1, leaf_batch=32):
        t = CameraTuning(engine, refill_min, leaf_batch)
        self.check(lib().rq_ctx_camera_tuning_set(self.h, C.byref(t)), "rq_ctx_camera_tuning_set")


class Bvh:
    """An rq_bvh handle (device-resident BVH in the reference layouts)."""

    def __init__(self, ctx, handle):
        self.ctx = ctx
        self.h = handle

    @staticmethod
    def build(ctx, pos, idx=None, max_leaf=4, bvh4=True, stride_bytes=12, stream=None, into=None, median=False,
              sah=False):
        """pos: float32 CUDA tensor of vertices; idx: int32/uint32 CUDA tensor
        [T, 3] or None (non-indexed: 3 consecutive vertices per triangle).
        median: the reference's median-split topology (RQ_BUILD_MEDIAN);
        sah: the LBVH with SAH-rebuilt subtrees (RQ_BUILD_SAH)."""
        nverts = _count(pos, 4) * 4 // stride_bytes
        ntri = _count(idx, 12) if idx is not None else nverts // 3
        h = _P(into.h.value) if into is not None else _P()
        flags = (RQ_BUILD_BVH4 if bvh4 else 0) | (RQ_BUILD_MEDIAN if median else 0) | (RQ_BUILD_SAH if sah else 0)
        rc = lib().rq_build(ctx.h, _ptr(pos), stride_bytes, nverts, _ptr(idx), ntri, max_leaf, flags, C.byref(h),
                            _stream(stream))
        ctx.check(rc, "rq_build")
        if into is not None:
            into.h = h
            return into
        return Bvh(ctx, h)

    @staticmethod
    def import2(ctx, nodes2, tris, perm=None, stream=None):
        h = _P()
        rc = lib().rq_bvh_import2(ctx.h, _ptr(nodes2), _count(nodes2, 32), _ptr(tris), _ptr(perm),
                                  _count(tris, 48), C.byref(h), _stream(stream))
        ctx.check(rc, "rq_bvh_import2")
        return Bvh(ctx, h)

    @staticmethod
    def import4(ctx, nodes4, tris, perm=None, stream=None):
        h = _P()
        rc = lib().rq_bvh_import4(ctx.h, _ptr(nodes4), _count(nodes4, 128), _ptr(tris), _ptr(perm),
                                  _count(tris, 48), C.byref(h), _stream(stream))
        ctx.check(rc, "rq_bvh_import4")
        return Bvh(ctx, h)

    def collapse4(self, stream=None):
        self.ctx.check(lib().rq_collapse4(self.ctx.h, self.h, _stream(stream)), "rq_collapse4")

    def refit(self, pos, idx=None, stride_bytes=12, stream=None):
        self.ctx.check(lib().rq_refit(self.ctx.h, self.h, _ptr(pos), stride_bytes, _ptr(idx), _stream(stream)),
                       "rq_refit")

    def info(self):
        inf = BvhInfo()
        self.ctx.check(lib().rq_bvh_info_get(self.h, C.byref(inf)), "rq_bvh_info_get")
        return {k: getattr(inf, k) for k, _ in BvhInfo._fields_}

    def download(self):
        """Host copies: nodes2, tris, nodes4, perm as numpy structured arrays."""
        inf = self.info()
        n2 = np.empty(inf["num_nodes2"], BVH2_NODE)
        tr = np.empty(inf["num_triangles"], TRIANGLE)
        n4 = np.empty(inf["num_nodes4"], BVH4_NODE)
        pm = np.empty(inf["num_triangles"], np.uint32)
        rc = lib().rq_bvh_download(self.h, 1, _ptr(n2), len(n2), _ptr(tr), len(tr), _ptr(n4), len(n4), _ptr(pm),
                                   len(pm))
        self.ctx.check(rc, "rq_bvh_download")
        return n2, tr, n4, pm

    def download_sort(self):
        inf = self.info()
        keys = np.empty(inf["num_triangles"], np.uint32)
        ids = np.empty(inf["num_triangles"], np.uint32)
        self.ctx.check(lib().rq_bvh_download_sort(self.h, 1, _ptr(keys), _ptr(ids), len(keys)), "download_sort")
        return keys, ids

    def destroy(self):
        if self.h:
            lib().rq_bvh_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


class Tlas:
    """An rq_tlas handle: instances of Bvh handles under a top-level BVH."""

    def __init__(self, ctx, instances, stream=None):
        """instances: sequence of (transform 3x4 row-major (12 floats), instance_id, mask, Bvh)."""
        arr = (Instance * len(instances))()
        for k, (xf, iid, mask, bvh) in enumerate(instances):
            arr[k].transform = (C.c_float * 12)(*[float(x) for x in np.asarray(xf, np.float32).reshape(-1)])
            arr[k].instance_id = iid
            arr[k].mask = mask
            arr[k].blas = bvh.h
        h = _P()
        ctx.check(lib().rq_tlas_build(ctx.h, arr, len(instances), C.byref(h), _stream(stream)), "rq_tlas_build")
        self.ctx, self.h, self._blas = ctx, h, [x[3] for x in instances]

    def trace(self, rays, flags=0, cull_mask=0xFF, hits=None, stream=None):
        n = _count(rays, 32)
        hits = hits if hits is not None else _empty_i32(n, 4, rays.device)
        self.ctx.check(lib().rq_tlas_trace(self.ctx.h, self.h, _ptr(rays), n, flags, cull_mask, _ptr(hits),
                                           _stream(stream)), "rq_tlas_trace")
        return hits

    def destroy(self):
        if self.h:
            lib().rq_tlas_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


class Batch:
    """An rq_batch handle: many meshes' BVHs, built by one launch."""

    def __init__(self, ctx, meshes, max_leaf=4):
        """meshes: sequence of (vertex_offset, num_vertices, triangle_offset, num_triangles)."""
        arr = (MeshDesc * len(meshes))(*[MeshDesc(*m) for m in meshes])
        h = _P()
        ctx.check(lib().rq_batch_create(ctx.h, arr, len(meshes), max_leaf, C.byref(h)), "rq_batch_create")
        self.ctx, self.h, self.meshes = ctx, h, list(meshes)

    def build(self, pos, idx, stride_bytes=12, stream=None):
        self.ctx.check(lib().rq_batch_build(self.ctx.h, self.h, _ptr(pos), stride_bytes, _ptr(idx), _stream(stream)),
                       "rq_batch_build")

    def trace(self, rays, ray_mesh, ray_flags=None, flags=0, hits=None, stats=False, stream=None):
        import torch
        n = _count(rays, 32)
        hits = hits if hits is not None else _empty_i32(n, 4, rays.device)
        s = _empty_i32(n, 4, rays.device) if stats else None
        rc = lib().rq_batch_trace(self.ctx.h, self.h, _ptr(rays), _ptr(ray_mesh), _ptr(ray_flags), n, flags,
                                  _ptr(hits), _ptr(s), _stream(stream))
        self.ctx.check(rc, "rq_batch_trace")
        return hits, s

    TUNING_KEYS = ("build_threads", "build_blocks", "trace_threads", "trace_chunk", "trace_reg_cap",
                   "trace_blocks_per_sm", "stack_entries", "trace_refill_min", "build_cluster", "cluster_min_tris")

    def tuning(self):
        t = BatchTuning()
        self.ctx.check(lib().rq_batch_tuning_get(self.h, C.byref(t)), "rq_batch_tuning_get")
        return {k: getattr(t, k) for k, _ in BatchTuning._fields_}

    def set_tuning(self, shape):
        """shape: dict with (a subset of) TUNING_KEYS."""
        t = BatchTuning()
        lib().rq_batch_tuning_get(self.h, C.byref(t))
        for k in self.TUNING_KEYS:
            if k in shape:
                setattr(t, k, int(shape[k]))
        self.ctx.check(lib().rq_batch_tuning_set(self.h, C.byref(t)), "rq_batch_tuning_set")

    def autotune(self, pos, idx, rays, ray_mesh, ray_flags=None, hits=None, reps=5, stride_bytes=12, stream=None):
        """Time every build and traversal shape on these inputs; keep the
        fastest.  Returns (chosen shape, list of measured candidates)."""
        n = _count(rays, 32)
        hits = hits if hits is not None else _empty_i32(n, 4, rays.device)
        cap = 256
        trials = (BatchTuning * cap)()
        cnt = _U32()
        rc = lib().rq_batch_autotune(self.ctx.h, self.h, _ptr(pos), stride_bytes, _ptr(idx), _ptr(rays),
                                     _ptr(ray_mesh), _ptr(ray_flags), n, _ptr(hits), reps, trials, cap,
                                     C.byref(cnt), _stream(stream))
        self.ctx.check(rc, "rq_batch_autotune")
        tr = [{k: getattr(trials[i], k) for k, _ in BatchTuning._fields_} for i in range(min(cap, cnt.value))]
        return self.tuning(), tr

    def info(self, m):
        inf = BvhInfo()
        self.ctx.check(lib().rq_batch_info_get(self.h, m, C.byref(inf)), "rq_batch_info_get")
        return {k: getattr(inf, k) for k, _ in BvhInfo._fields_}

    def download(self, m):
        inf = self.info(m)
        n2 = np.empty(inf["num_nodes2"], BVH2_NODE)
        tr = np.empty(inf["num_triangles"], TRIANGLE)
        n4 = np.empty(inf["num_nodes4"], BVH4_NODE)
        pm = np.empty(inf["num_triangles"], np.uint32)
        rc = lib().rq_batch_download(self.h, m, 1, _ptr(n2), len(n2), _ptr(tr), len(tr), _ptr(n4), len(n4),
                                     _ptr(pm), len(pm))
        self.ctx.check(rc, "rq_batch_download")
        return n2, tr, n4, pm

    def destroy(self):
        if self.h:
            lib().rq_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def _empty_i32(n, cols, device):
    import torch
    return torch.empty((n, cols), dtype=torch.int32, device=device)


def trace(ctx, bvh, rays, flags=0, bary=False, stats=False, hits=None, stream=None):
    """rays: float32 CUDA tensor [n, 8].  Returns (hits int32 [n,4], bary, stats)."""
    import torch
    n = _count(rays, 32)
    dev = rays.device
    hits = hits if hits is not None else _empty_i32(n, 4, dev)
    b = torch.empty((n, 2), dtype=torch.float32, device=dev) if bary else None
    s = _empty_i32(n, 4, dev) if stats else None
    rc = lib().rq_trace(ctx.h, bvh.h, _ptr(rays), n, flags, _ptr(hits), _ptr(b), _ptr(s), _stream(stream))
    ctx.check(rc, "rq_trace")
    return hits, b, s


def trace_ref_bvh4(ctx, nodes4, tris, rays, stream=None):
    n = _count(rays, 32)
    st = _empty_i32(n, 4, rays.device)
    hits = _empty_i32(n, 4, rays.device)
    rc = lib().rq_trace_ref_bvh4(ctx.h, _ptr(nodes4), _ptr(tris), _ptr(rays), n, _ptr(st), _ptr(hits),
                                 _stream(stream))
    ctx.check(rc, "rq_trace_ref_bvh4")
    return st, hits


def trace_ref_bvh2(ctx, nodes2, tris, rays, t_eps=0.001, stream=None):
    import torch
    n = _count(rays, 32)
    flags = torch.empty(n, dtype=torch.int32, device=rays.device)
    rc = lib().rq_trace_ref_bvh2(ctx.h, _ptr(nodes2), _ptr(tris), _ptr(rays), n, t_eps, _ptr(flags),
                                 _stream(stream))
    ctx.check(rc, "rq_trace_ref_bvh2")
    return flags


def gen_rays_procedural(ctx, cam, look, count, coherent, device="cuda", stream=None):
    import torch
    rays = torch.empty((count, 8), dtype=torch.float32, device=device)
    c = (C.c_float * 3)(*cam)
    l = (C.c_float * 3)(*look)
    rc = lib().rq_gen_rays_procedural(ctx.h, C.cast(c, _P), C.cast(l, _P), count, 1 if coherent else 0,
                                      _ptr(rays), _stream(stream))
    ctx.check(rc, "rq_gen_rays_procedural")
    return rays


def radv_layout(n):
    L = RadvLayout()
    rc = lib().rq_radv_layout_get(n, C.byref(L))
    if rc != RQ_OK:
        raise RqError(rc, "rq_radv_layout_get")
    lv = L.num_levels
    return dict(total_boxes=L.total_boxes, num_levels=lv, total_size=int(L.total_as_size),
                counts=list(L.level_counts[:lv]), offsets=list(L.level_offsets[:lv]))


def radv_size(n):
    return int(lib().rq_radv_size(n))


def build_radv(ctx, tri9, image=None, stream=None):
    import torch
    n = _count(tri9, 36)
    size = radv_size(n)
    if image is None:
        image = torch.empty(size, dtype=torch.uint8, device=tri9.device)
    rc = lib().rq_build_radv(ctx.h, _ptr(tri9), n, _ptr(image), _count(image, 1), _stream(stream))
    ctx.check(rc, "rq_build_radv")
    return image


def refit_radv(ctx, tri9, image, stream=None):
    """Refit an image in place after its vertices moved (same triangle count)."""
    rc = lib().rq_refit_radv(ctx.h, _ptr(tri9), _count(tri9, 36), _ptr(image), _count(image, 1), _stream(stream))
    ctx.check(rc, "rq_refit_radv")
    return image


def radv_describe(image):
    """Text of a RADV image held on the host (bytes or a uint8 array), as the
    reference's decoder prints it.  Host only: no device needed."""
    img = np.ascontiguousarray(np.frombuffer(bytes(image), np.uint8))
    n = C.c_uint64()
    rc = lib().rq_radv_describe(_ptr(img), len(img), None, 0, C.byref(n))
    if rc:
        raise RqError(rc, "rq_radv_describe")
    buf = C.create_string_buffer(n.value + 1)
    rc = lib().rq_radv_describe(_ptr(img), len(img), buf, n.value + 1, C.byref(n))
    if rc:
        raise RqError(rc, "rq_radv_describe")
    return buf.value.decode()


def radv_validate(ctx, image, stream=None):
    """Device-side decode and invariant counts of a RADV image (uint8 CUDA tensor)."""
    out = RadvCheck()
    ctx.check(lib().rq_radv_validate(ctx.h, _ptr(image), _count(image, 1), C.byref(out), _stream(stream)),
              "rq_radv_validate")
    return {k: getattr(out, k) for k, _ in RadvCheck._fields_ if k != "reserved"}


def trace_radv(ctx, image, rays, flags=0, bary=False, stream=None):
    import torch
    n = _count(rays, 32)
    hits = _empty_i32(n, 4, rays.device)
    b = torch.empty((n, 2), dtype=torch.float32, device=rays.device) if bary else None
    rc = lib().rq_trace_radv(ctx.h, _ptr(image), image.numel(), _ptr(rays), n, flags, _ptr(hits), _ptr(b),
                             _stream(stream))
    ctx.check(rc, "rq_trace_radv")
    return hits, b


def scene_grid(qx, qy, x0=-1.0, x1=1.0, y0=-1.0, y1=1.0, amp=0.2, freq=3.0, sigma=0.01, seed=0):
    """Height-field grid on the host: float32 [V,3] positions, uint32 [T,3] indices."""
    pos = np.empty(((qx + 1) * (qy + 1), 3), np.float32)
    idx = np.empty((2 * qx * qy, 3), np.uint32)
    rc = lib().rq_scene_grid(qx, qy, x0, x1, y0, y1, amp, freq, sigma, seed, _ptr(pos), _ptr(idx))
    if rc != RQ_OK:
        raise RqError(rc, "rq_scene_grid")
    return pos, idx


def scene_rays_down(n, x0=-1.0, x1=1.0, y0=-1.0, y1=1.0, z=2.0, spread=0.3, tmin=0.01, tmax=1000.0, seed=0):
    """Downward rays on the host as float32 [n, 8] (the plain workload's rays)."""
    rays = np.empty((n, 8), np.float32)
    rc = lib().rq_scene_rays_down(n, x0, x1, y0, y1, z, spread, tmin, tmax, seed, _ptr(rays))
    if rc != RQ_OK:
        raise RqError(rc, "rq_scene_rays_down")
    return rays


def deform_wave(ctx, base, out, t, amp=0.05, freq=1.0, stream=None):
    rc = lib().rq_deform_wave(ctx.h, _ptr(base), _ptr(out), base.numel() // 3, t, amp, freq, _stream(stream))
    ctx.check(rc, "rq_deform_wave")
    return out


def camera_look_at(eye, target, up, fovy_deg, width, height, jitter=False, seed=0, flags=0):
    cam = Camera()
    f3 = C.c_float * 3
    rc = lib().rq_camera_look_at(C.cast(f3(*eye), _P), C.cast(f3(*target), _P), C.cast(f3(*up), _P), fovy_deg,
                                 width, height, C.byref(cam))
    if rc != RQ_OK:
        raise RqError(rc, "rq_camera_look_at")
    cam.jitter = 1 if jitter else 0
    cam.seed = seed
    cam.flags = flags
    return cam


def shade_params(width, height, lights, ao_spp=1, ao_tmax=0.5, flags=0):
    """lights: sequence of (x, y, z, radius)."""
    p = ShadeParams()
    p.width, p.height, p.num_lights, p.ao_spp = width, height, len(lights), ao_spp
    p.ao_tmax, p.ao_tmin, p.ao_bias = ao_tmax, 0.01, 0.03
    p.shadow_tmin, p.shadow_bias, p.flags = 0.01, 0.04, flags
    for k, (x, y, z, r) in enumerate(lights):
        p.lights[k].pos[0], p.lights[k].pos[1], p.lights[k].pos[2], p.lights[k].radius = x, y, z, r
    return p


def render_gbuffer(ctx, bvh, cam, gbuf=None, stream=None):
    """Primary rays -> G-buffer as int32 [H*W, 8] CUDA tensor (rq_gbuffer_px)."""
    import torch
    if gbuf is None:
        gbuf = torch.empty((cam.width * cam.height, 8), dtype=torch.int32, device="cuda")
    ctx.check(lib().rq_render_gbuffer(ctx.h, bvh.h, C.byref(cam), _ptr(gbuf), _stream(stream)), "rq_render_gbuffer")
    return gbuf


def reflect_params(cam, flags=0, tmin=0.02, tmax=100.0, bias=0.04):
    """Reflection rays of shaders/tiled_lighting_ra.comp:91-113 for a camera's
    G-buffer (tmin 0.02, tmax 100, offset 0.04 as the shader)."""
    p = ReflectParams()
    p.width, p.height = cam.width, cam.height
    for k in range(3):
        p.cam_pos[k] = cam.cam_pos[k]
    p.tmin, p.tmax, p.bias, p.flags = tmin, tmax, bias, flags
    return p


def render_reflect(ctx, bvh, gbuf, params, hits=None, stream=None):
    """Closest-hit reflection ray per G-buffer pixel -> int32 [H*W, 4] hit
    records (rq_hit) as a CUDA tensor."""
    import torch
    npix = params.width * params.height
    if hits is None:
        hits = torch.empty((npix, 4), dtype=torch.int32, device=gbuf.device)
    ctx.check(lib().rq_render_reflect(ctx.h, bvh.h, _ptr(gbuf), C.byref(params), _ptr(hits), _stream(stream)),
              "rq_render_reflect")
    return hits


def ao_depth_params(cam, spp=1, max_distance=0.5, flags=0, tmin=0.01, bias=0.03):
    """rq_ao.comp's push constants for a camera (inv_view_proj, cam_pos,
    resolution) with its fixed tmin 0.01 and 0.03 normal offset."""
    p = AoDepthParams()
    for k in range(16):
        p.inv_view_proj[k] = cam.inv_view_proj[k]
    for k in range(3):
        p.cam_pos[k] = cam.cam_pos[k]
    p.width, p.height, p.spp, p.max_distance = cam.width, cam.height, spp, max_distance
    p.tmin, p.bias, p.flags = tmin, bias, flags
    return p


def render_ao_depth(ctx, bvh, depth, params, ao=None, counters=None, stream=None):
    """rq_ao.comp from a depth buffer (float32 CUDA tensor, width*height) ->
    float32 AO per pixel."""
    import torch
    if ao is None:
        ao = torch.empty(params.width * params.height, dtype=torch.float32, device=depth.device)
    ctx.check(lib().rq_render_ao_depth(ctx.h, bvh.h, _ptr(depth), C.byref(params), _ptr(ao), _ptr(counters),
                                       _stream(stream)), "rq_render_ao_depth")
    return ao


def view_proj_of(cam):
    """Forward view-projection (column-major float32[16]) of a camera, the
    inverse of its inv_view_proj computed in double precision."""
    inv = np.array(cam.inv_view_proj, np.float64).reshape(4, 4).T
    return np.ascontiguousarray(np.linalg.inv(inv).T.reshape(-1), np.float32)


def gbuffer_depth(ctx, gbuf, view_proj, depth=None, stream=None):
    """G-buffer (int32 [n,8] CUDA tensor) -> float32 [n] depth z/w (1.0 for misses)."""
    import torch
    n = _count(gbuf, 32)
    depth = depth if depth is not None else torch.empty(n, dtype=torch.float32, device=gbuf.device)
    vp = np.ascontiguousarray(view_proj, np.float32)
    ctx.check(lib().rq_gbuffer_depth(ctx.h, _ptr(gbuf), n, _ptr(vp), _ptr(depth), _stream(stream)), "rq_gbuffer_depth")
    return depth


def blur_ao(ctx, ao, depth, width, height, dir_x, dir_y, threshold, out=None, stream=None):
    """One pass of the depth-aware AO blur (float32 CUDA tensors of width*height)."""
    import torch
    out = out if out is not None else torch.empty_like(ao)
    ctx.check(lib().rq_blur_ao(ctx.h, _ptr(ao), _ptr(depth), _ptr(out), width, height, dir_x, dir_y, threshold,
                               _stream(stream)), "rq_blur_ao")
    return out


def render_shadow_ao(ctx, bvh, gbuf, params, mask=None, ao=None, counter=None, stream=None):
    import torch
    n = params.width * params.height
    mask = mask if mask is not None else torch.empty(n, dtype=torch.int32, device="cuda")
    ao = ao if ao is not None else torch.empty(n, dtype=torch.float32, device="cuda")
    rc = lib().rq_render_shadow_ao(ctx.h, bvh.h, _ptr(gbuf), C.byref(params), _ptr(mask), _ptr(ao), _ptr(counter),
                                   _stream(stream))
    ctx.check(rc, "rq_render_shadow_ao")
    return mask, ao


def deform_wave_step(ctx, base, out, state, dt, amp=0.05, freq=1.0, stream=None):
    """state: int32 CUDA tensor of 2 (t as float bits, work word)."""
    rc = lib().rq_deform_wave_step(ctx.h, _ptr(base), _ptr(out), base.numel() // 3, _ptr(state), dt, amp, freq,
                                   _stream(stream))
    ctx.check(rc, "rq_deform_wave_step")
    return out


def hits_numpy(hits_tensor):
    """int32 [n,4] CUDA tensor -> numpy HIT structured array."""
    return hits_tensor.cpu().numpy().view(HIT).reshape(-1)


def stats_numpy(stats_tensor):
    return stats_tensor.cpu().numpy().view(STATS).reshape(-1)


def rays_numpy(rays_tensor):
    return rays_tensor.cpu().numpy().view(RAY).reshape(-1)


def gen_mesh_rays(ctx, pos, idx, kind, seed, count, stream=None):
    """The rays a generated serving request of `kind` traces on the mesh
    (pos float32 [V,3], idx int32/uint32 [T,3] CUDA tensors): float32 [count,8]
    rays and int32 [count] any-hit flags."""
    import torch
    rays = torch.empty((count, 8), dtype=torch.float32, device=pos.device)
    anyf = torch.empty(count, dtype=torch.int32, device=pos.device)
    ntri = _count(idx, 12) if idx is not None else 0
    rc = lib().rq_gen_mesh_rays(ctx.h, _ptr(pos), _ptr(idx), ntri, kind, seed, count, _ptr(rays), _ptr(anyf),
                                _stream(stream))
    ctx.check(rc, "rq_gen_mesh_rays")
    return rays, anyf


class ServeError(RqError):
    pass


class Server:
    """An rq_server (include/rq_serve.h): a request loop with resident BVHs,
    a memory budget and coalesced traversal launches."""

    def __init__(self, device=0, budget_bytes=120 << 30, mode=RQ_SERVE_BATCHED, slots=4, max_wave_rays=1 << 24,
                 max_wave_requests=1024, max_leaf=4, trace_flags=0, rebuild=False):
        cfg = ServerConfig(budget_bytes, mode, slots, max_wave_rays, max_wave_requests, max_leaf, trace_flags,
                           1 if rebuild else 0)
        h = _P()
        rc = lib().rq_server_create(device, C.byref(cfg), C.byref(h))
        if rc:
            raise ServeError(rc, f"rq_server_create: {lib().rq_status_string(rc).decode()}")
        self.h = h
        self._keep = []

    def _check(self, rc, what):
        if rc:
            err = lib().rq_server_last_error(self.h).decode()
            raise ServeError(rc, f"{what}: {lib().rq_status_string(rc).decode()} {err}")

    @staticmethod
    def mesh_bytes(num_vertices, num_triangles):
        return int(lib().rq_server_mesh_bytes(num_vertices, num_triangles))

    def add_mesh(self, pos, idx):
        """pos float32 [V,3], idx uint32 [T,3] host arrays -> mesh id."""
        pos = np.ascontiguousarray(pos, np.float32)
        idx = np.ascontiguousarray(idx, np.uint32)
        mid = _U32()
        self._check(lib().rq_server_add_mesh(self.h, _ptr(pos), len(pos.reshape(-1)) // 3, _ptr(idx),
                                             len(idx.reshape(-1)) // 3, C.byref(mid)), "rq_server_add_mesh")
        return mid.value

    @staticmethod
    def request(mesh, kind, num_rays, hits, seed=0, rays=None, flags=0, user=0):
        """hits: int32 [num_rays,4] CUDA tensor (kept alive by the caller)."""
        return Request(mesh, kind, num_rays, seed, flags, 0, _ptr(rays).value if rays is not None else None,
                       _ptr(hits).value, user)

    def submit(self, req):
        t = C.c_uint64()
        self._check(lib().rq_server_submit(self.h, C.byref(req), C.byref(t)), "rq_server_submit")
        return t.value

    def replay(self, reqs, arrival):
        """Submit reqs[i] at arrival[i] seconds from now (ascending); returns tickets."""
        n = len(reqs)
        arr = (Request * n)(*reqs)
        at = np.ascontiguousarray(arrival, np.float64)
        tickets = np.zeros(n, np.uint64)
        self._check(lib().rq_server_replay(self.h, arr, _ptr(at), n, _ptr(tickets)), "rq_server_replay")
        return tickets

    def poll(self, capacity=4096):
        out = (Completion * capacity)()
        n = _U32()
        self._check(lib().rq_server_poll(self.h, out, capacity, C.byref(n)), "rq_server_poll")
        return [out[i] for i in range(n.value)]

    def drain(self, timeout_ms=120000):
        self._check(lib().rq_server_drain(self.h, timeout_ms), "rq_server_drain")

    def completions(self):
        """Drain, then every completion as a dict keyed by ticket."""
        self.drain()
        res = {}
        while True:
            got = self.poll()
            if not got:
                break
            for c in got:
                res[c.ticket] = {k: getattr(c, k) for k, _ in Completion._fields_}
        return res

    def now(self):
        return lib().rq_server_now(self.h)

    def cancel(self, ticket):
        self._check(lib().rq_server_cancel(self.h, int(ticket)), "rq_server_cancel")

    def inject_fault(self, kind, count=1):
        self._check(lib().rq_server_inject_fault(self.h, kind, count), "rq_server_inject_fault")

    def stats(self):
        s = ServerStats()
        self._check(lib().rq_server_stats_get(self.h, C.byref(s)), "rq_server_stats_get")
        return {k: getattr(s, k) for k, _ in ServerStats._fields_}

    def close(self):
        if self.h:
            lib().rq_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
