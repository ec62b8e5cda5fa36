"""voxelengine3.0_b200 — B200-native voxel ray pipeline (RayPass, bounce/shade
loop, AccumPass, AvgPass of AnghelusAndrei/VoxelEngine3.0).

This module binds the native library ``libve.so`` (C ABI: include/ve.h) with
ctypes and mirrors the reference's host interface:

* ``OctreeCPU``   — src/octree_cpu.hpp:9-57 (insert / remove / lookup /
  insertBox / insertSphere / raycast)
* ``Octree``      — src/renderer/octree.hpp:14-98 (set / applyEdits /
  findGpuSlot, node words in the reference layout)
* ``camera_ubo``  — Camera::UpdateUBO, src/renderer/camera.cpp:39-50
* ``FrameConfig`` — core::FrameConfig, src/renderer/core.hpp:83-158
* ``Renderer``    — src/renderer/renderer.hpp:9-129 (``run`` renders one frame)

There is no CPU fallback: every render call runs the CUDA kernels of
libve.so, and loading fails loudly when the library is missing.
"""
from __future__ import annotations

import ctypes
import dataclasses
import math
import os
from typing import Dict, Iterable, List, Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libve.so")
HEADER_PATH = os.path.join(os.path.dirname(_HERE), "include", "ve.h")

VE_OK = 0
VE_ERR_INVALID = -1
VE_ERR_CUDA = -2
VE_ERR_NOMEM = -3
VE_ERR_CAPACITY = -4
VE_ERR_NOT_FOUND = -5
VE_ERR_TIMEOUT = -6
VE_ERR_STATE = -7

RENDER_DEFAULT, RENDER_STRUCTURE, RENDER_ALBEDO, RENDER_NORMAL, RENDER_VOXELID, RENDER_VARIANCE = range(6)
SCENE_KEEP_NORMALS = 1
FRAME_TIMING = 1
FRAME_COUNT_FETCH = 2
FRAME_PATH_RGB = 4
FRAME_LEARNED = 8
FRAME_TERMINATE_HASH = 16
FRAME_TRAIN = 32
FRAME_SCHEDULED = 64
FRAME_EMISSIVE = 128
FRAME_LBUFFER = 256
FRAME_SPLIT = 512
FRAME_ASYNC_OUTPUTS = 1024
SPLIT_RECORD_BYTES = 32  # ve_split_record
RESTIR_ENABLE = 1
RESTIR_TEMPORAL = 2
RESTIR_SPATIAL = 4
RAYCAST_FULL_WALK = 1
CFG_NO_GRAPHS = 1
CFG_PIPELINE = 2
SERVER_FIFO = 1


class VeError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"ve error {code}: {msg}")
        self.code = code


# ---------------------------------------------------------------------------
# ctypes structures (include/ve.h)
# ---------------------------------------------------------------------------
class RendererConfigC(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("hash_log2", ctypes.c_uint32), ("hash_probes", ctypes.c_uint32),
                ("flags", ctypes.c_uint32)]


class FrameConfigC(ctypes.Structure):
    _fields_ = [("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("spp", ctypes.c_uint32),
                ("bounces", ctypes.c_uint32), ("primary_controlchecks", ctypes.c_uint32),
                ("bounce_controlchecks", ctypes.c_uint32), ("reconstruction_radius", ctypes.c_uint32),
                ("render_type", ctypes.c_uint32), ("frame_index", ctypes.c_uint32),
                ("sun_dir", ctypes.c_float * 3), ("sun_intensity", ctypes.c_float), ("sky", ctypes.c_float * 3),
                ("decay", ctypes.c_float), ("variance_norm", ctypes.c_float), ("flags", ctypes.c_uint32),
                ("weight_pixels", ctypes.c_float), ("weight_variance", ctypes.c_float),
                ("pixels_norm", ctypes.c_float), ("top_fraction", ctypes.c_float), ("mid_fraction", ctypes.c_float),
                ("min_samples", ctypes.c_uint32), ("shading_budget", ctypes.c_uint32),
                ("restir", ctypes.c_uint32), ("restir_m", ctypes.c_uint32),
                ("restir_spatial_neighbors", ctypes.c_uint32), ("restir_max_m", ctypes.c_uint32),
                ("restir_spatial_radius", ctypes.c_float),
                ("time", ctypes.c_uint32), ("update_time", ctypes.c_uint32),
                ("disable_stale_reset", ctypes.c_uint32), ("sample_cap_direct", ctypes.c_uint32),
                ("sample_cap_indirect", ctypes.c_uint32), ("firefly_k", ctypes.c_float),
                ("firefly_floor", ctypes.c_float), ("row_begin", ctypes.c_uint32), ("row_end", ctypes.c_uint32)]


class ViewC(ctypes.Structure):
    _fields_ = [("scene_id", ctypes.c_int32), ("camera", ctypes.c_float * 16), ("frame", FrameConfigC)]


class FrameOutputsC(ctypes.Structure):
    _fields_ = [("gbuffer", ctypes.c_void_p), ("voxel_id", ctypes.c_void_p), ("hit_node", ctypes.c_void_p),
                ("rgb", ctypes.c_void_p), ("mapped", ctypes.c_void_p), ("path_rgb", ctypes.c_void_p),
                ("mapped8", ctypes.c_void_p)]


class LaunchConfigC(ctypes.Structure):
    _fields_ = [("trace_blocks_per_sm", ctypes.c_uint32), ("shade_blocks_per_sm", ctypes.c_uint32),
                ("refill_threshold", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class FrameStatsC(ctypes.Structure):
    _fields_ = [("rays_primary", ctypes.c_uint64), ("rays_bounce", ctypes.c_uint64),
                ("rays_shadow", ctypes.c_uint64), ("fetch_nodes", ctypes.c_uint64), ("paths", ctypes.c_uint64),
                ("deposits", ctypes.c_uint64), ("deposits_dropped", ctypes.c_uint64), ("dda_steps", ctypes.c_uint64),
                ("fetch_nodes_trace", ctypes.c_uint64), ("dda_steps_trace", ctypes.c_uint64),
                ("h2d_bytes", ctypes.c_uint64), ("d2h_bytes", ctypes.c_uint64), ("frames", ctypes.c_uint64),
                ("ms_total", ctypes.c_float), ("ms_primary", ctypes.c_float), ("ms_trace", ctypes.c_float),
                ("ms_shade", ctypes.c_float), ("ms_resolve", ctypes.c_float), ("ms_decay", ctypes.c_float),
                ("trace_launches", ctypes.c_uint32), ("kernel_launches", ctypes.c_uint32),
                ("cache_capacity", ctypes.c_uint64), ("nrc_queries", ctypes.c_uint64),
                ("nrc_hash_terminated", ctypes.c_uint64), ("nrc_samples", ctypes.c_uint64),
                ("scheduled_voxels", ctypes.c_uint64), ("scheduled_paths", ctypes.c_uint64),
                ("ms_learned", ctypes.c_float), ("reserved", ctypes.c_uint32),
                ("emissive_lights", ctypes.c_uint64), ("nee_emissive", ctypes.c_uint64),
                ("restir_commits", ctypes.c_uint64), ("shadow_shared", ctypes.c_uint64)]


class ServerConfigC(ctypes.Structure):
    _fields_ = [("pixel_capacity", ctypes.c_uint64), ("path_capacity", ctypes.c_uint64),
                ("max_requests", ctypes.c_uint32), ("flags", ctypes.c_uint32),
                ("step_path_budget", ctypes.c_uint64), ("max_bypass_ms", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32)]


class RequestInfoC(ctypes.Structure):
    _fields_ = [("request_id", ctypes.c_uint64), ("submit_s", ctypes.c_double), ("admit_s", ctypes.c_double),
                ("done_s", ctypes.c_double), ("pixels", ctypes.c_uint64), ("paths", ctypes.c_uint64)]


class ServerStatsC(ctypes.Structure):
    _fields_ = [(k, ctypes.c_uint64) for k in ("completed", "admitted", "queued", "in_flight", "max_in_flight",
                                               "steps", "pool_bytes", "scene_bytes", "rays")]


class NrcConfigC(ctypes.Structure):
    _fields_ = [("log2_table", ctypes.c_uint32), ("base_resolution", ctypes.c_uint32),
                ("max_resolution", ctypes.c_uint32), ("train_samples", ctypes.c_uint32),
                ("learning_rate", ctypes.c_float), ("beta1", ctypes.c_float), ("beta2", ctypes.c_float),
                ("eps", ctypes.c_float), ("fallback_threshold", ctypes.c_float), ("flags", ctypes.c_uint32),
                ("seed", ctypes.c_uint64)]


_P = ctypes.c_void_p
_U32 = ctypes.c_uint32
_U64 = ctypes.c_uint64
_I32 = ctypes.c_int32
_F = ctypes.c_float
_PTR = ctypes.POINTER

_SIGNATURES = {
    "ve_version": ([], ctypes.c_char_p),
    "ve_last_error": ([], ctypes.c_char_p),
    "ve_octree_cpu_create": ([_U32, _PTR(_P)], ctypes.c_int),
    "ve_octree_cpu_destroy": ([_P], ctypes.c_int),
    "ve_octree_cpu_insert": ([_P, _U32, _U32, _U32, _U32], ctypes.c_int),
    "ve_octree_cpu_insert_many": ([_P, _P, _U64], ctypes.c_int),
    "ve_octree_cpu_remove": ([_P, _U32, _U32, _U32], ctypes.c_int),
    "ve_octree_cpu_lookup": ([_P, _U32, _U32, _U32, _PTR(ctypes.c_int64)], ctypes.c_int),
    "ve_octree_cpu_insert_box": ([_P, _P, _P, _U32], ctypes.c_int),
    "ve_octree_cpu_insert_sphere": ([_P, _P, _F, _U32], ctypes.c_int),
    "ve_octree_cpu_raycast": ([_P, _P, _P, _U32, _PTR(ctypes.c_int), _P], ctypes.c_int),
    "ve_octree_create": ([_U32, _PTR(_P)], ctypes.c_int),
    "ve_octree_destroy": ([_P], ctypes.c_int),
    "ve_octree_set": ([_P, _P], ctypes.c_int),
    "ve_octree_apply_edits": ([_P, _P, _P, _U64, _PTR(_U64)], ctypes.c_int),
    "ve_octree_last_changed": ([_P, _PTR(_P), _PTR(_U64)], ctypes.c_int),
    "ve_octree_find_gpu_slot": ([_P, _P, _U32, _U32, _U32, _PTR(_U32)], ctypes.c_int),
    "ve_octree_info": ([_P, _PTR(_U32), _PTR(_U32), _PTR(_U32)], ctypes.c_int),
    "ve_octree_words": ([_P, _PTR(_P), _PTR(_U64)], ctypes.c_int),
    "ve_terrain_build": ([_U32, _U32, _U64, _U32, _PTR(_P), _PTR(_U64)], ctypes.c_int),
    "ve_words_data": ([_P, _PTR(_P), _PTR(_U64)], ctypes.c_int),
    "ve_words_free": ([_P], ctypes.c_int),
    "ve_terrain_voxels": ([_U32, _U32, _U64, _P, _U64, _PTR(_U64)], ctypes.c_int),
    "ve_terrain_materials": ([_U64, _P], ctypes.c_int),
    "ve_camera_ubo": ([_P, _P, _F, _F, _P], ctypes.c_int),
    "ve_ctx_create": ([_PTR(RendererConfigC), _PTR(_P)], ctypes.c_int),
    "ve_ctx_destroy": ([_P], ctypes.c_int),
    "ve_ctx_stream": ([_P, _PTR(_P)], ctypes.c_int),
    "ve_ctx_synchronize": ([_P], ctypes.c_int),
    "ve_ctx_join": ([_P], ctypes.c_int),
    "ve_scene_upload": ([_P, _P, _U64, _U32, _U32, _PTR(_I32)], ctypes.c_int),
    "ve_scene_release": ([_P, _I32], ctypes.c_int),
    "ve_scene_apply_edits": ([_P, _I32, _P, _P, _U64, _U32], ctypes.c_int),
    "ve_scene_download": ([_P, _I32, _P, _U64, _PTR(_U64)], ctypes.c_int),
    "ve_scene_footprint": ([_P, _I32, _PTR(_U64)], ctypes.c_int),
    "ve_scene_clip_box": ([_P, _I32, _P, _P, _PTR(_U32)], ctypes.c_int),
    "ve_raycast_batch": ([_P, _I32, _P, _P, _U64, _U32, _U32, _P], ctypes.c_int),
    "ve_lbuffer_dump": ([_P, _I32, _P, _U64, _PTR(_U64)], ctypes.c_int),
    "ve_set_materials": ([_P, _P, _U32], ctypes.c_int),
    "ve_cache_reset": ([_P, _I32], ctypes.c_int),
    "ve_cache_dump": ([_P, _I32, _P, _P, _P, _U64, _PTR(_U64)], ctypes.c_int),
    "ve_render": ([_P, _PTR(ViewC), _PTR(FrameOutputsC)], ctypes.c_int),
    "ve_render_batch": ([_P, _PTR(ViewC), _U32, _P], ctypes.c_int),
    "ve_get_stats": ([_P, _PTR(FrameStatsC)], ctypes.c_int),
    "ve_get_total_stats": ([_P, _PTR(FrameStatsC)], ctypes.c_int),
    "ve_fill_normals_noalloc": ([_P, _U64, _U32, _P], ctypes.c_int),
    "ve_get_launch_config": ([_P, _PTR(LaunchConfigC)], ctypes.c_int),
    "ve_nrc_create": ([_P, _PTR(NrcConfigC), _PTR(_P)], ctypes.c_int),
    "ve_nrc_destroy": ([_P], ctypes.c_int),
    "ve_nrc_param_counts": ([_P, _PTR(_U64), _PTR(_U64)], ctypes.c_int),
    "ve_nrc_get_params": ([_P, _P, _P], ctypes.c_int),
    "ve_nrc_set_params": ([_P, _P, _P], ctypes.c_int),
    "ve_nrc_infer": ([_P, _P, _U32, _P], ctypes.c_int),
    "ve_nrc_gradients": ([_P, _P, _P, _U32, _P, _P, _PTR(ctypes.c_float)], ctypes.c_int),
    "ve_nrc_train": ([_P, _P, _P, _U32, _PTR(ctypes.c_float)], ctypes.c_int),
    "ve_scene_set_nrc": ([_P, ctypes.c_int, _P], ctypes.c_int),
    "ve_scene_build": ([_P, _P, _U64, _U32, _U32, _PTR(ctypes.c_int32), _PTR(_U64)], ctypes.c_int),
    "ve_scene_refresh": ([_P, ctypes.c_int32, _P, _U64, _U32], ctypes.c_int),
    "ve_scene_normal_mode": ([_P, ctypes.c_int32, _U32], ctypes.c_int),
    "ve_nrc_stats": ([_P, _PTR(ctypes.c_float), _PTR(_U64), _PTR(_U64)], ctypes.c_int),
    "ve_server_create": ([_P, _PTR(ServerConfigC), _PTR(_P)], ctypes.c_int),
    "ve_server_submit": ([_P, _PTR(ViewC), _P, _P, _PTR(_U64)], ctypes.c_int),
    "ve_server_wait": ([_P, _U64, _U32, _PTR(RequestInfoC)], ctypes.c_int),
    "ve_server_get_stats": ([_P, _PTR(ServerStatsC)], ctypes.c_int),
    "ve_server_destroy": ([_P], ctypes.c_int),
    "ve_split_export": ([_P, _I32, _P, _U64, _PTR(_U64)], ctypes.c_int),
    "ve_split_merge": ([_P, _I32, _P, _P, _U32, _U64, _PTR(_U64)], ctypes.c_int),
    "ve_split_resolve": ([_P, _PTR(ViewC), _PTR(FrameOutputsC)], ctypes.c_int),
    "ve_set_launch_config": ([_P, _PTR(LaunchConfigC)], ctypes.c_int),
    "ve_autotune": ([_P, _PTR(ViewC), _U32, _U32, _PTR(LaunchConfigC)], ctypes.c_int),
    "ve_reset_total_stats": ([_P], ctypes.c_int),
}

_lib: Optional[ctypes.CDLL] = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads libve.so (raises when it has not been built: there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"libve.so not found at {path}; build it with `python voxelengine3.0_b200/build.py` "
                          "or __graft_entry__.build()")
    lib = ctypes.CDLL(path)
    for name, (args, res) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def _check(rc: int) -> None:
    if rc != VE_OK:
        raise VeError(rc, load_library().ve_last_error().decode(errors="replace"))


def _ptr(a: Optional[np.ndarray]) -> Optional[int]:
    return None if a is None else a.ctypes.data


# ---------------------------------------------------------------------------
# host scene layer
# ---------------------------------------------------------------------------
class OctreeCPU:
    """Pointer sparse voxel octree with the reference's build API."""

    def __init__(self, depth: int):
        self._lib = load_library()
        self.depth = int(depth)
        h = _P()
        _check(self._lib.ve_octree_cpu_create(self.depth, ctypes.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.ve_octree_cpu_destroy(self._h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def insert(self, x: int, y: int, z: int, material: int) -> None:
        _check(self._lib.ve_octree_cpu_insert(self._h, x, y, z, material))

    def insert_many(self, xyzm: np.ndarray) -> None:
        a = np.ascontiguousarray(xyzm, dtype=np.uint32).reshape(-1, 4)
        _check(self._lib.ve_octree_cpu_insert_many(self._h, _ptr(a), a.shape[0]))

    def remove(self, x: int, y: int, z: int) -> None:
        _check(self._lib.ve_octree_cpu_remove(self._h, x, y, z))

    def lookup(self, x: int, y: int, z: int) -> int:
        m = ctypes.c_int64()
        _check(self._lib.ve_octree_cpu_lookup(self._h, x, y, z, ctypes.byref(m)))
        return m.value

    def insert_box(self, mn: Sequence[int], mx: Sequence[int], material: int) -> None:
        a = np.asarray(mn, np.uint32)
        b = np.asarray(mx, np.uint32)
        _check(self._lib.ve_octree_cpu_insert_box(self._h, _ptr(a), _ptr(b), material))

    def insert_sphere(self, centre: Sequence[float], radius: float, material: int) -> None:
        c = np.asarray(centre, np.float32)
        _check(self._lib.ve_octree_cpu_insert_sphere(self._h, _ptr(c), float(radius), material))

    def raycast(self, origin: Sequence[float], direction: Sequence[float], max_steps: int = 300):
        o = np.asarray(origin, np.float32)
        d = np.asarray(direction, np.float32)
        hit = ctypes.c_int()
        pos = np.zeros(3, np.uint32)
        _check(self._lib.ve_octree_cpu_raycast(self._h, _ptr(o), _ptr(d), max_steps, ctypes.byref(hit), _ptr(pos)))
        return (True, tuple(int(v) for v in pos)) if hit.value else (False, None)

    # reference-style names
    insertBox = insert_box
    insertSphere = insert_sphere


class Octree:
    """Node array in the reference layout (Octree::data)."""

    def __init__(self, depth: int):
        self._lib = load_library()
        self.depth = int(depth)
        h = _P()
        _check(self._lib.ve_octree_create(self.depth, ctypes.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.ve_octree_destroy(self._h)
            self._h = None

    def set(self, cpu: OctreeCPU) -> None:
        _check(self._lib.ve_octree_set(self._h, cpu.handle))

    def apply_edits(self, cpu: OctreeCPU) -> np.ndarray:
        """Octree::applyEdits; returns the slots whose words changed."""
        n = _U64()
        _check(self._lib.ve_octree_apply_edits(self._h, cpu.handle, None, 0, ctypes.byref(n)))
        p = _P()
        _check(self._lib.ve_octree_last_changed(self._h, ctypes.byref(p), ctypes.byref(n)))
        if n.value == 0:
            return np.zeros(0, np.uint32)
        return np.frombuffer((ctypes.c_uint32 * n.value).from_address(p.value), dtype=np.uint32).copy()

    def find_gpu_slot(self, cpu: OctreeCPU, pos: Sequence[int]) -> int:
        s = _U32()
        _check(self._lib.ve_octree_find_gpu_slot(self._h, cpu.handle, pos[0], pos[1], pos[2], ctypes.byref(s)))
        return s.value

    def info(self):
        size, cap, nv = _U32(), _U32(), _U32()
        _check(self._lib.ve_octree_info(self._h, ctypes.byref(size), ctypes.byref(cap), ctypes.byref(nv)))
        return size.value, cap.value, nv.value

    @property
    def size(self) -> int:
        return self.info()[0]

    @property
    def capacity(self) -> int:
        return self.info()[1]

    @property
    def num_voxels(self) -> int:
        return self.info()[2]

    def words(self) -> np.ndarray:
        """Copy of all `capacity` words (Octree::data)."""
        p = _P()
        n = _U64()
        _check(self._lib.ve_octree_words(self._h, ctypes.byref(p), ctypes.byref(n)))
        if n.value == 0:
            return np.zeros(0, np.uint32)
        buf = (ctypes.c_uint32 * n.value).from_address(p.value)
        return np.frombuffer(buf, dtype=np.uint32).copy()

    findGpuSlot = find_gpu_slot
    applyEdits = apply_edits


def terrain_words(depth: int, variant: int = 0, seed: int = 1, threads: int = 0):
    """Bulk-built node words of a seeded terrain scene; returns (words, n_voxels)."""
    lib = load_library()
    h = _P()
    nv = _U64()
    _check(lib.ve_terrain_build(depth, variant, seed, threads, ctypes.byref(h), ctypes.byref(nv)))
    try:
        p = _P()
        n = _U64()
        _check(lib.ve_words_data(h, ctypes.byref(p), ctypes.byref(n)))
        buf = (ctypes.c_uint32 * n.value).from_address(p.value)
        words = np.frombuffer(buf, dtype=np.uint32).copy()
    finally:
        lib.ve_words_free(h)
    return words, nv.value


def terrain_voxels(depth: int, variant: int = 0, seed: int = 1) -> np.ndarray:
    lib = load_library()
    n = _U64()
    _check(lib.ve_terrain_voxels(depth, variant, seed, None, 0, ctypes.byref(n)))
    out = np.zeros((n.value, 4), np.uint32)
    _check(lib.ve_terrain_voxels(depth, variant, seed, _ptr(out), n.value, ctypes.byref(n)))
    return out


def terrain_materials(seed: int = 1) -> np.ndarray:
    """128 std140 Material entries (64 B each) as a (128, 16) float32 view."""
    out = np.zeros((128, 16), np.float32)
    _check(load_library().ve_terrain_materials(seed, _ptr(out)))
    return out


def camera_ubo(position: Sequence[float], direction: Sequence[float], fov_deg: float, aspect: float) -> np.ndarray:
    p = np.asarray(position, np.float32)
    d = np.asarray(direction, np.float32)
    out = np.zeros(16, np.float32)
    _check(load_library().ve_camera_ubo(_ptr(p), _ptr(d), float(fov_deg), float(aspect), _ptr(out)))
    return out


def look_at(eye: Sequence[float], target: Sequence[float]) -> np.ndarray:
    """Unit view direction from eye toward target (float32, normalised in float64)."""
    d = np.asarray(target, np.float64) - np.asarray(eye, np.float64)
    return (d / np.linalg.norm(d)).astype(np.float32)


# ---------------------------------------------------------------------------
# frame configuration
# ---------------------------------------------------------------------------
SUN_DIR = tuple(float(v) for v in (np.array([0.3, 1.0, 0.2]) / np.linalg.norm([0.3, 1.0, 0.2])).astype(np.float32))


@dataclasses.dataclass
class FrameConfig:
    """core::FrameConfig subset read by the plain method + benchmark lighting."""
    width: int = 256
    height: int = 256
    spp: int = 1
    bounces: int = 1
    primary_controlchecks: int = 70
    bounce_controlchecks: int = 100
    reconstruction_radius: int = 10
    render_type: int = RENDER_DEFAULT
    frame_index: int = 0
    sun_dir: Sequence[float] = SUN_DIR
    sun_intensity: float = math.pi
    sky: Sequence[float] = (0.4, 0.4, 0.4)
    decay: float = 0.95
    variance_norm: float = 10000.0
    flags: int = 0
    # importance-aware scheduling (FRAME_SCHEDULED), core.hpp:95-112 defaults
    weight_pixels: float = 0.1
    weight_variance: float = 0.9
    pixels_norm: float = 100.0
    top_fraction: float = 0.30
    mid_fraction: float = 0.40
    min_samples: int = 1
    shading_budget: int = 131072
    # emissive NEE (FRAME_EMISSIVE), core.hpp:138-144 ReSTIR defaults
    restir: int = RESTIR_ENABLE | RESTIR_TEMPORAL | RESTIR_SPATIAL
    restir_m: int = 4
    restir_spatial_neighbors: int = 1
    restir_max_m: int = 24
    restir_spatial_radius: float = 2.75
    # dual-channel lBuffer (FRAME_LBUFFER), core.hpp:93-104, 150-157 defaults
    time: int = 0
    update_time: int = 0
    disable_stale_reset: int = 0
    sample_cap_direct: int = 16
    sample_cap_indirect: int = 64
    firefly_k: float = 1.0
    firefly_floor: float = 255.0
    # split frames (FRAME_SPLIT): this rank's band of rows
    row_begin: int = 0
    row_end: int = 0

    def to_c(self) -> FrameConfigC:
        c = FrameConfigC()
        for f in ("width", "height", "spp", "bounces", "primary_controlchecks", "bounce_controlchecks",
                  "reconstruction_radius", "render_type", "frame_index", "flags", "min_samples", "shading_budget",
                  "restir", "restir_m", "restir_spatial_neighbors", "restir_max_m", "time", "update_time",
                  "disable_stale_reset", "sample_cap_direct", "sample_cap_indirect", "row_begin", "row_end"):
            setattr(c, f, int(getattr(self, f)))
        for i in range(3):
            c.sun_dir[i] = float(self.sun_dir[i])
            c.sky[i] = float(self.sky[i])
        c.sun_intensity = float(self.sun_intensity)
        c.decay = float(self.decay)
        c.variance_norm = float(self.variance_norm)
        for f in ("weight_pixels", "weight_variance", "pixels_norm", "top_fraction", "mid_fraction",
                  "restir_spatial_radius", "firefly_k", "firefly_floor"):
            setattr(c, f, float(getattr(self, f)))
        return c


OUTPUT_KINDS = ("gbuffer", "voxel_id", "hit_node", "rgb", "mapped", "path_rgb", "mapped8")
# bytes per pixel of the per-pixel host outputs
IMAGE_BYTES = {"gbuffer": 16, "voxel_id": 4, "hit_node": 4, "rgb": 12, "mapped": 12, "mapped8": 4}


def _dev_ptr(buf) -> Optional[int]:
    """Device address of a tensor-like object (data_ptr()) or an integer."""
    if buf is None:
        return None
    if hasattr(buf, "data_ptr"):
        return int(buf.data_ptr())
    return int(buf)


def _alloc_outputs(fc: FrameConfig, want: Iterable[str]):
    npx = fc.width * fc.height
    arrays: Dict[str, np.ndarray] = {}
    for k in want:
        if k == "gbuffer":
            arrays[k] = np.zeros((fc.height, fc.width, 4), np.uint32)
        elif k in ("voxel_id", "hit_node"):
            arrays[k] = np.zeros((fc.height, fc.width), np.uint32)
        elif k in ("rgb", "mapped"):
            arrays[k] = np.zeros((fc.height, fc.width, 3), np.float32)
        elif k == "mapped8":
            arrays[k] = np.zeros((fc.height, fc.width, 4), np.uint8)
        elif k == "path_rgb":
            n = min(fc.shading_budget, 2 * npx) if fc.flags & FRAME_SCHEDULED else npx * fc.spp
            arrays[k] = np.zeros((n, 3), np.float32)
        else:
            raise ValueError(f"unknown output {k!r}")
    o = FrameOutputsC()
    for k, a in arrays.items():
        setattr(o, k, a.ctypes.data)
    return o, arrays


def _image_outputs(fc: FrameConfig, arrays: Dict[str, np.ndarray]) -> "FrameOutputsC":
    """FrameOutputsC over caller-owned full-size host images (name -> a
    C-contiguous array of IMAGE_BYTES[name] bytes per pixel)."""
    npx = fc.width * fc.height
    o = FrameOutputsC()
    for k, a in arrays.items():
        if k not in IMAGE_BYTES:
            raise ValueError(f"unknown output {k!r}")
        if not a.flags.c_contiguous or a.nbytes != IMAGE_BYTES[k] * npx:
            raise ValueError(f"output {k!r}: {IMAGE_BYTES[k] * npx} contiguous bytes expected")
        setattr(o, k, a.ctypes.data)
    return o


class Renderer:
    """The device renderer (one CUDA context stream, owned device memory)."""

    def __init__(self, device: int = 0, hash_log2: int = 22, hash_probes: int = 64, graphs: bool = True,
                 pipeline: bool = False):
        self._lib = load_library()
        cfg = RendererConfigC(device, hash_log2, hash_probes,
                              (0 if graphs else CFG_NO_GRAPHS) | (CFG_PIPELINE if pipeline else 0))
        h = _P()
        _check(self._lib.ve_ctx_create(ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self._children: List[object] = []
        self.hash_log2 = hash_log2
        self.scene: Optional[int] = None
        self.camera: Optional[np.ndarray] = None

    def close(self) -> None:
        for child in list(getattr(self, "_children", ())):
            child.close()
        if getattr(self, "_h", None):
            self._lib.ve_ctx_destroy(self._h)
            self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def stream(self) -> int:
        s = _P()
        _check(self._lib.ve_ctx_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    def synchronize(self) -> None:
        _check(self._lib.ve_ctx_synchronize(self._h))

    def join(self) -> None:
        """Orders work enqueued on `stream` from now on behind every frame
        rendered so far (pipelined frames run partly on a second stream)."""
        _check(self._lib.ve_ctx_join(self._h))

    def upload_scene(self, words: np.ndarray, depth: int, keep_normals: bool = False) -> int:
        w = np.ascontiguousarray(words, np.uint32)
        sid = _I32()
        _check(self._lib.ve_scene_upload(self._h, _ptr(w), w.size, depth, SCENE_KEEP_NORMALS if keep_normals else 0,
                                         ctypes.byref(sid)))
        return sid.value

    def build_scene(self, xyzm: np.ndarray, depth: int, keep_normals: bool = False) -> int:
        """GPU bulk build from (x, y, z, material) rows: the words of
        OctreeCPU.insert_many + Octree.set, built on the device."""
        v = np.ascontiguousarray(np.asarray(xyzm, np.uint32).reshape(-1, 4))
        sid = ctypes.c_int32()
        nw = _U64()
        _check(self._lib.ve_scene_build(self._h, _ptr(v) if v.size else None, v.shape[0], depth,
                                        1 if keep_normals else 0, ctypes.byref(sid), ctypes.byref(nw)))
        return sid.value

    def release_scene(self, scene_id: int) -> None:
        _check(self._lib.ve_scene_release(self._h, scene_id))

    def apply_edits(self, scene_id: int, slots: np.ndarray, words: np.ndarray, keep_normals: bool = False) -> None:
        s = np.ascontiguousarray(slots, np.uint32)
        w = np.ascontiguousarray(words, np.uint32)
        _check(self._lib.ve_scene_apply_edits(self._h, scene_id, _ptr(s), _ptr(w), s.size,
                                              SCENE_KEEP_NORMALS if keep_normals else 0))

    def refresh_scene(self, scene_id: int, positions: np.ndarray, keep_cache: bool = False) -> None:
        """Targeted refresh around edited positions (n x 3): leaf normals of
        their 3x3x3 neighbourhoods and, unless keep_cache, their radiance-cache
        entries."""
        p = np.ascontiguousarray(np.asarray(positions, np.uint32).reshape(-1, 3))
        _check(self._lib.ve_scene_refresh(self._h, scene_id, _ptr(p) if p.size else None, p.shape[0],
                                          1 if keep_cache else 0))

    def lbuffer_dump(self, scene_id: int) -> np.ndarray:
        """Occupied lBuffer slots, (n, 14) u32 rows {row, slot, 12 slot words}."""
        n = _U64()
        _check(self._lib.ve_lbuffer_dump(self._h, scene_id, None, 0, ctypes.byref(n)))
        out = np.zeros((n.value, 14), np.uint32)
        _check(self._lib.ve_lbuffer_dump(self._h, scene_id, _ptr(out), n.value, ctypes.byref(n)))
        return out

    def raycast_batch(self, scene_id: int, origins: np.ndarray, dirs: np.ndarray, controlchecks: int = 300,
                      full_walk: bool = False) -> np.ndarray:
        """Rays through the device DDA; (n, 8) u32 rows {status, hit node,
        material, x, y, z, size, checks}."""
        o = np.ascontiguousarray(origins, np.float32).reshape(-1, 3)
        d = np.ascontiguousarray(dirs, np.float32).reshape(-1, 3)
        if o.shape != d.shape:
            raise ValueError("origins and dirs differ in shape")
        out = np.zeros((o.shape[0], 8), np.uint32)
        _check(self._lib.ve_raycast_batch(self._h, scene_id, _ptr(o), _ptr(d), o.shape[0], controlchecks,
                                          RAYCAST_FULL_WALK if full_walk else 0, _ptr(out)))
        return out

    def set_normal_mode(self, scene_id: int, radius: int) -> None:
        """radius 0: 3x3x3 occupancy-gradient normals (the default); R >= 1:
        the reference's normal pass with normalPrecision = R (normal.comp's
        L2 ball).  Recomputes the scene's leaf normals."""
        _check(self._lib.ve_scene_normal_mode(self._h, scene_id, radius))

    def download_scene(self, scene_id: int) -> np.ndarray:
        n = _U64()
        _check(self._lib.ve_scene_download(self._h, scene_id, None, 0, ctypes.byref(n)))
        out = np.zeros(n.value, np.uint32)
        _check(self._lib.ve_scene_download(self._h, scene_id, _ptr(out), n.value, ctypes.byref(n)))
        return out

    def scene_footprint(self, scene_id: int) -> int:
        b = _U64()
        _check(self._lib.ve_scene_footprint(self._h, scene_id, ctypes.byref(b)))
        return b.value

    def clip_box(self, scene_id: int):
        """(lo, hi, bounded): the box bounce rays are clipped to (ve_scene_clip_box)."""
        lo = np.zeros(3, np.float32)
        hi = np.zeros(3, np.float32)
        b = ctypes.c_uint32()
        _check(self._lib.ve_scene_clip_box(self._h, scene_id, _ptr(lo), _ptr(hi), ctypes.byref(b)))
        return lo, hi, bool(b.value)

    def set_materials(self, materials: np.ndarray) -> None:
        m = np.ascontiguousarray(materials, np.float32).reshape(-1, 16)
        _check(self._lib.ve_set_materials(self._h, _ptr(m), m.shape[0]))

    def cache_reset(self, scene_id: int) -> None:
        _check(self._lib.ve_cache_reset(self._h, scene_id))

    def cache_dump(self, scene_id: int):
        n = _U64()
        _check(self._lib.ve_cache_dump(self._h, scene_id, None, None, None, 0, ctypes.byref(n)))
        vids = np.zeros(n.value, np.uint32)
        counts = np.zeros(n.value, np.uint32)
        vals = np.zeros((n.value, 5), np.float32)
        _check(self._lib.ve_cache_dump(self._h, scene_id, _ptr(vids), _ptr(counts), _ptr(vals), n.value,
                                       ctypes.byref(n)))
        return vids, counts, vals

    @staticmethod
    def make_view(scene_id: int, camera: np.ndarray, fc: FrameConfig) -> ViewC:
        v = ViewC()
        v.scene_id = scene_id
        cam = np.asarray(camera, np.float32).reshape(16)
        for i in range(16):
            v.camera[i] = float(cam[i])
        v.frame = fc.to_c()
        return v

    def render(self, scene_id: int, camera: np.ndarray, fc: FrameConfig,
               outputs: Iterable[str] = ("voxel_id", "rgb")) -> Dict[str, np.ndarray]:
        """One frame of one view; returns the requested host outputs."""
        view = self.make_view(scene_id, camera, fc)
        want = list(outputs)
        o, arrays = _alloc_outputs(fc, want)
        _check(self._lib.ve_render(self._h, ctypes.byref(view), ctypes.byref(o) if want else None))
        return arrays

    def render_into(self, scene_id: int, camera: np.ndarray, fc: FrameConfig, arrays: Dict[str, np.ndarray]) -> None:
        """One frame into caller-owned host arrays (name -> C-contiguous array
        of the output's size).  With FRAME_ASYNC_OUTPUTS the call returns once
        the frame is enqueued; the arrays (pinned memory for an asynchronous
        copy) hold the frame after synchronize()."""
        o = _image_outputs(fc, arrays)
        view = self.make_view(scene_id, camera, fc)
        _check(self._lib.ve_render(self._h, ctypes.byref(view), ctypes.byref(o)))

    def render_batch(self, views: Sequence[tuple], outputs: Iterable[str] = ("voxel_id", "rgb")):
        """views: sequence of (scene_id, camera, FrameConfig)."""
        arr = (ViewC * len(views))()
        want = list(outputs)
        outs = (FrameOutputsC * len(views))()
        results: List[Dict[str, np.ndarray]] = []
        for i, (sid, cam, fc) in enumerate(views):
            arr[i] = self.make_view(sid, cam, fc)
            o, arrays = _alloc_outputs(fc, want)
            outs[i] = o
            results.append(arrays)
        _check(self._lib.ve_render_batch(self._h, arr, len(views), outs if want else None))
        return results

    # split frames (one frame over several ranks; see dist.SplitFrame)
    def split_export(self, scene_id: int, out, cap: int) -> int:
        """Records of the last FRAME_SPLIT frame into device memory `out` (a
        tensor or an address, room for `cap` records of 32 B); returns the
        frame's record count."""
        n = _U64()
        _check(self._lib.ve_split_export(self._h, scene_id, _dev_ptr(out), cap, ctypes.byref(n)))
        return n.value

    def split_merge(self, scene_id: int, parts, counts: Sequence[int], stride: int) -> int:
        """Adds the ranks' records (device memory; part k at record k * stride)
        into the scene's cache in rank order; returns the records dropped."""
        c = np.ascontiguousarray(np.asarray(counts, np.uint64))
        d = _U64()
        _check(self._lib.ve_split_merge(self._h, scene_id, _dev_ptr(parts), _ptr(c) if c.size else None, c.size,
                                        stride, ctypes.byref(d)))
        return d.value

    def split_resolve(self, scene_id: int, camera: np.ndarray, fc: FrameConfig,
                      outputs: Iterable[str] = ("rgb",)) -> Dict[str, np.ndarray]:
        """AvgPass of the band of the last FRAME_SPLIT frame; full-size host
        images with the band's rows written."""
        view = self.make_view(scene_id, camera, fc)
        want = list(outputs)
        o, arrays = _alloc_outputs(fc, want)
        _check(self._lib.ve_split_resolve(self._h, ctypes.byref(view), ctypes.byref(o) if want else None))
        return arrays

    def split_resolve_into(self, scene_id: int, camera: np.ndarray, fc: FrameConfig,
                           arrays: Dict[str, np.ndarray]) -> None:
        """split_resolve into caller-owned full-size host arrays (the band's
        rows are written)."""
        o = _image_outputs(fc, arrays)
        view = self.make_view(scene_id, camera, fc)
        _check(self._lib.ve_split_resolve(self._h, ctypes.byref(view), ctypes.byref(o)))

    def launch_config(self) -> Dict[str, int]:
        c = LaunchConfigC()
        _check(self._lib.ve_get_launch_config(self._h, ctypes.byref(c)))
        return {k: getattr(c, k) for k, _ in LaunchConfigC._fields_}

    def set_launch_config(self, trace_blocks_per_sm: int = 0, shade_blocks_per_sm: int = 0,
                          refill_threshold: int = 0) -> None:
        """0 for any field keeps the library's default (occupancy maximum; refill at 20 idle lanes)."""
        c = LaunchConfigC(trace_blocks_per_sm, shade_blocks_per_sm, refill_threshold, 0)
        _check(self._lib.ve_set_launch_config(self._h, ctypes.byref(c)))

    def autotune(self, views: Sequence[tuple], frames_per_trial: int = 2) -> Dict[str, int]:
        """views: (scene_id, camera, FrameConfig) tuples; returns the chosen launch config."""
        arr = (ViewC * len(views))()
        for i, (sid, cam, fc) in enumerate(views):
            arr[i] = self.make_view(sid, cam, fc)
        best = LaunchConfigC()
        _check(self._lib.ve_autotune(self._h, arr, len(views), frames_per_trial, ctypes.byref(best)))
        return {k: getattr(best, k) for k, _ in LaunchConfigC._fields_}

    def stats(self) -> Dict[str, float]:
        """Counters and timings of the last render call."""
        s = FrameStatsC()
        _check(self._lib.ve_get_stats(self._h, ctypes.byref(s)))
        return {name: getattr(s, name) for name, _ in FrameStatsC._fields_}

    def total_stats(self) -> Dict[str, float]:
        """Counters summed over every render since reset_total_stats()."""
        s = FrameStatsC()
        _check(self._lib.ve_get_total_stats(self._h, ctypes.byref(s)))
        return {name: getattr(s, name) for name, _ in FrameStatsC._fields_}

    def reset_total_stats(self) -> None:
        _check(self._lib.ve_reset_total_stats(self._h))

    # Renderer::run (reference-shaped): renders the bound scene from the bound camera
    def set_scene(self, scene_id: int) -> None:
        self.scene = scene_id

    def set_camera(self, ubo: np.ndarray) -> None:
        self.camera = np.asarray(ubo, np.float32).reshape(16)

    def run(self, fc: FrameConfig, outputs: Iterable[str] = ("rgb",)) -> Dict[str, np.ndarray]:
        if self.scene is None or self.camera is None:
            raise VeError(VE_ERR_STATE, "run: bind a scene (set_scene) and a camera (set_camera) first")
        return self.render(self.scene, self.camera, fc, outputs)


class Server:
    """Render server with continuous batching over one Renderer's context."""

    def __init__(self, renderer: "Renderer", pixel_capacity: int, path_capacity: int, max_requests: int = 64,
                 fifo: bool = False, step_path_budget: int = 0, max_bypass_ms: int = 0):
        """fifo: strict first-come-first-served admission, each request's
        primary pass in one step.  Otherwise a step starts at most
        `step_path_budget` paths (0: 2^23) and admission may pass over a
        request that does not fit for up to `max_bypass_ms` (0: 50 ms)."""
        self._lib = load_library()
        self.renderer = renderer
        cfg = ServerConfigC(pixel_capacity, path_capacity, max_requests, SERVER_FIFO if fifo else 0,
                            step_path_budget, max_bypass_ms, 0)
        h = _P()
        _check(self._lib.ve_server_create(renderer._h, ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        renderer._children.append(self)
        self._buffers: Dict[int, tuple] = {}

    def submit(self, scene_id: int, camera: np.ndarray, fc: FrameConfig, want_vid: bool = True,
               want_rgb: bool = True, out_vid: Optional[np.ndarray] = None,
               out_rgb: Optional[np.ndarray] = None) -> int:
        """Queues one frame request.  Results land in freshly allocated arrays,
        or in `out_vid` (u32, >= W*H) / `out_rgb` (f32, >= 3*W*H) when given
        (e.g. views of pinned host memory); those must outlive the request."""
        view = Renderer.make_view(scene_id, camera, fc)
        npx = fc.width * fc.height
        vid = rgb = None
        if out_vid is not None:
            assert out_vid.dtype == np.uint32 and out_vid.size >= npx and out_vid.flags.c_contiguous
            vid = out_vid
        elif want_vid:
            vid = np.zeros((fc.height, fc.width), np.uint32)
        if out_rgb is not None:
            assert out_rgb.dtype == np.float32 and out_rgb.size >= 3 * npx and out_rgb.flags.c_contiguous
            rgb = out_rgb
        elif want_rgb:
            rgb = np.zeros((fc.height, fc.width, 3), np.float32)
        rid = _U64()
        _check(self._lib.ve_server_submit(self._h, ctypes.byref(view), _ptr(vid), _ptr(rgb), ctypes.byref(rid)))
        self._buffers[rid.value] = (vid, rgb)
        return rid.value

    def wait(self, request_id: int, timeout_ms: int = 120000) -> Dict[str, object]:
        info = RequestInfoC()
        _check(self._lib.ve_server_wait(self._h, request_id, timeout_ms, ctypes.byref(info)))
        vid, rgb = self._buffers.pop(request_id)
        return {"voxel_id": vid, "rgb": rgb, "submit_s": info.submit_s, "admit_s": info.admit_s,
                "done_s": info.done_s, "latency_s": info.done_s - info.submit_s, "pixels": info.pixels,
                "paths": info.paths}

    def stats(self) -> Dict[str, int]:
        st = ServerStatsC()
        _check(self._lib.ve_server_get_stats(self._h, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in ServerStatsC._fields_}

    def close(self) -> None:
        if getattr(self, "_h", None):
            rc = self._lib.ve_server_destroy(self._h)
            self._h = None
            if self in self.renderer._children:
                self.renderer._children.remove(self)
            _check(rc)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class LearnedCache:
    """Learned radiance cache (hash-grid encoding + 4 x 64 ReLU MLP, bf16
    tensor-core kernels) living on a Renderer's device.

    Inputs are float32 rows [px, py, pz, 0, nx_oct, ny_oct, vx_oct, vy_oct]:
    the voxel centre divided by the scene extent, the octahedral shading
    normal and the octahedral direction toward the previous path vertex."""

    LEVELS = 16
    WIDTH = 64
    LAYERS = 5

    def __init__(self, renderer: "Renderer", log2_table: int = 19, base_resolution: int = 16,
                 max_resolution: int = 2048, train_samples: int = 65536, learning_rate: float = 1e-2,
                 beta1: float = 0.9, beta2: float = 0.99, eps: float = 1e-8, fallback_threshold: float = 0.1,
                 seed: int = 1):
        self._lib = load_library()
        self.renderer = renderer
        self.log2_table = log2_table
        self.config = dict(log2_table=log2_table, base_resolution=base_resolution, max_resolution=max_resolution,
                           train_samples=train_samples, learning_rate=learning_rate, beta1=beta1, beta2=beta2,
                           eps=eps, fallback_threshold=fallback_threshold)
        cfg = NrcConfigC(log2_table, base_resolution, max_resolution, train_samples, learning_rate, beta1, beta2,
                         eps, fallback_threshold, 0, seed)
        h = _P()
        _check(self._lib.ve_nrc_create(renderer._h, ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        renderer._children.append(self)

    @staticmethod
    def _rows(inputs) -> np.ndarray:
        x = np.ascontiguousarray(np.asarray(inputs, np.float32))
        assert x.ndim == 2 and x.shape[1] == 8, "inputs are (n, 8) float32 rows"
        return x

    def param_counts(self):
        a, b = _U64(), _U64()
        _check(self._lib.ve_nrc_param_counts(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def get_params(self):
        nw, nt = self.param_counts()
        w = np.zeros(nw, np.float32)
        t = np.zeros(nt, np.float32)
        _check(self._lib.ve_nrc_get_params(self._h, w.ctypes.data, t.ctypes.data))
        return w.reshape(self.LAYERS, self.WIDTH, self.WIDTH), t.reshape(self.LEVELS, -1, 2)

    def set_params(self, weights: Optional[np.ndarray] = None, table: Optional[np.ndarray] = None) -> None:
        w = None if weights is None else np.ascontiguousarray(weights, np.float32)
        t = None if table is None else np.ascontiguousarray(table, np.float32)
        nw, nt = self.param_counts()
        assert w is None or w.size == nw
        assert t is None or t.size == nt
        _check(self._lib.ve_nrc_set_params(self._h, _ptr(w), _ptr(t)))

    def infer(self, inputs) -> np.ndarray:
        x = self._rows(inputs)
        out = np.zeros((x.shape[0], 3), np.float32)
        _check(self._lib.ve_nrc_infer(self._h, x.ctypes.data, x.shape[0], out.ctypes.data))
        return out

    def gradients(self, inputs, targets):
        x = self._rows(inputs)
        t = np.ascontiguousarray(np.asarray(targets, np.float32).reshape(x.shape[0], 3))
        nw, nt = self.param_counts()
        gw = np.zeros(nw, np.float32)
        gt = np.zeros(nt, np.float32)
        loss = ctypes.c_float()
        _check(self._lib.ve_nrc_gradients(self._h, x.ctypes.data, t.ctypes.data, x.shape[0], gw.ctypes.data,
                                          gt.ctypes.data, ctypes.byref(loss)))
        return gw.reshape(self.LAYERS, self.WIDTH, self.WIDTH), gt.reshape(self.LEVELS, -1, 2), loss.value

    def train(self, inputs, targets) -> float:
        x = self._rows(inputs)
        t = np.ascontiguousarray(np.asarray(targets, np.float32).reshape(x.shape[0], 3))
        loss = ctypes.c_float()
        _check(self._lib.ve_nrc_train(self._h, x.ctypes.data, t.ctypes.data, x.shape[0], ctypes.byref(loss)))
        return loss.value

    def attach(self, scene_id: int) -> None:
        _check(self._lib.ve_scene_set_nrc(self.renderer._h, scene_id, self._h))

    def stats(self) -> Dict[str, float]:
        """Loss and sample count of the last training step, steps taken."""
        loss, n, steps = ctypes.c_float(), _U64(), _U64()
        _check(self._lib.ve_nrc_stats(self._h, ctypes.byref(loss), ctypes.byref(n), ctypes.byref(steps)))
        return {"loss": loss.value, "samples": n.value, "steps": steps.value}

    def close(self) -> None:
        if getattr(self, "_h", None):
            if getattr(self.renderer, "_h", None):  # the context destroys its caches itself
                self._lib.ve_nrc_destroy(self._h)
            self._h = None
            if self in self.renderer._children:
                self.renderer._children.remove(self)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


__all__ = [
    "OctreeCPU", "Octree", "Renderer", "FrameConfig", "VeError", "camera_ubo", "look_at", "terrain_words",
    "terrain_voxels", "terrain_materials", "load_library", "SUN_DIR", "Server", "LearnedCache",
]
