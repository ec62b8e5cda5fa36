"""TEST INFRASTRUCTURE ONLY — ctypes bindings of the CPU oracle
(oracle/liboracle.so, a scalar restatement of the reference's ray pipeline)
and of the reference's own compiled octree code (oracle/_ref/libveref.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, always as the checker / the timed CPU baseline, never as the
product path.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libveref.so")

_P = ctypes.c_void_p
_U32 = ctypes.c_uint32
_U64 = ctypes.c_uint64


class FrameParams(ctypes.Structure):
    """ov_frame_params (same layout as the product's ve_frame_config)."""
    _fields_ = [("width", _U32), ("height", _U32), ("spp", _U32), ("bounces", _U32),
                ("primary_controlchecks", _U32), ("bounce_controlchecks", _U32),
                ("reconstruction_radius", _U32), ("render_type", _U32), ("frame_index", _U32),
                ("sun_dir", ctypes.c_float * 3), ("sun_intensity", ctypes.c_float), ("sky", ctypes.c_float * 3),
                ("decay", ctypes.c_float), ("variance_norm", ctypes.c_float), ("flags", _U32),
                ("weight_pixels", ctypes.c_float), ("weight_variance", ctypes.c_float),
                ("pixels_norm", ctypes.c_float), ("top_fraction", ctypes.c_float), ("mid_fraction", ctypes.c_float),
                ("min_samples", _U32), ("shading_budget", _U32),
                ("restir", _U32), ("restir_m", _U32), ("restir_spatial_neighbors", _U32), ("restir_max_m", _U32),
                ("restir_spatial_radius", ctypes.c_float),
                ("time", _U32), ("update_time", _U32), ("disable_stale_reset", _U32),
                ("sample_cap_direct", _U32), ("sample_cap_indirect", _U32),
                ("firefly_k", ctypes.c_float), ("firefly_floor", ctypes.c_float)]


class Stats(ctypes.Structure):
    _fields_ = [("rays_primary", _U64), ("rays_bounce", _U64), ("rays_shadow", _U64), ("fetch_restart", _U64),
                ("fetch_min", _U64), ("paths", _U64), ("deposits", _U64), ("steps", _U64),
                ("scheduled_voxels", _U64), ("scheduled_paths", _U64),
                ("emissive_lights", _U64), ("nee_emissive", _U64), ("restir_commits", _U64),
                ("shadow_shared", _U64)]


def build_oracle(force: bool = False) -> str:
    srcs = [os.path.join(HERE, f) for f in ("ve_oracle.cpp", "terrain_oracle.cpp", "ve_oracle.h")]
    if force or not os.path.exists(ORACLE_LIB) or any(os.path.getmtime(ORACLE_LIB) < os.path.getmtime(s)
                                                       for s in srcs):
        subprocess.check_call(["bash", os.path.join(HERE, "build_oracle.sh")])
    return ORACLE_LIB


def build_ref() -> Optional[str]:
    """Compiles the reference's octree code in place (needs the reference tree)."""
    subprocess.check_call(["bash", os.path.join(HERE, "build_ref.sh")])
    return REF_LIB if os.path.exists(REF_LIB) else None


def _np(dtype):
    return np.ctypeslib.ndpointer(dtype, flags="C_CONTIGUOUS")


class Oracle:
    def __init__(self):
        self.lib = ctypes.CDLL(build_oracle())
        L = self.lib
        L.oracle_build.restype = _U64
        L.oracle_build.argtypes = [_U32, _np(np.uint32), _U64, _np(np.uint32), _U64, ctypes.POINTER(_U32)]
        L.oracle_fill_normals.argtypes = [_np(np.uint32), _U64, _U32]
        L.oracle_fill_normals_mode.argtypes = [_np(np.uint32), _U64, _U32, ctypes.c_int, _U32]
        L.oracle_fill_normals_ball.restype = _U64
        L.oracle_fill_normals_ball.argtypes = [_np(np.uint32), _U64, _U32, _U32, _U32, _P, _U64]
        L.oracle_renderer_set_normal_codes.argtypes = [_P, _P, _U64]
        L.oracle_lookup_occupied.restype = ctypes.c_int
        L.oracle_lookup_occupied.argtypes = [_np(np.uint32), _U64, _U32, ctypes.c_int64, ctypes.c_int64,
                                             ctypes.c_int64]
        L.oracle_camera_ubo.argtypes = [_np(np.float32), _np(np.float32), ctypes.c_float, ctypes.c_float,
                                        _np(np.float32)]
        L.oracle_raycast.argtypes = [_np(np.uint32), _U64, _U32, _np(np.float32), _np(np.float32), _U32,
                                     _np(np.uint32), _P]
        L.oracle_raycast_batch.argtypes = [_np(np.uint32), _U64, _U32, _np(np.float32), _np(np.float32), _U64, _U32,
                                           _U32, _np(np.uint32)]
        L.oracle_pow_unit.argtypes = [_np(np.float32), _np(np.float32), _U64, _np(np.float32)]
        L.oracle_voxel_key.restype = _U32
        L.oracle_voxel_key.argtypes = [_U32, _U32, _U32]
        L.oracle_rand_seq.restype = _U32
        L.oracle_rand_seq.argtypes = [_U32, _U32, _np(np.float32)]
        L.oracle_sincos_turn.argtypes = [_np(np.float32), _U64, _np(np.float32), _np(np.float32)]
        L.oracle_shading_normal.argtypes = [_U32, _np(np.float32), _np(np.float32)]
        L.oracle_renderer_new.restype = _P
        L.oracle_renderer_free.argtypes = [_P]
        L.oracle_lb_apply.argtypes = [_np(np.uint32), _U64, ctypes.POINTER(FrameParams), _np(np.uint32)]
        L.oracle_lbuffer_dump.restype = _U64
        L.oracle_lbuffer_dump.argtypes = [_P, _P, _U64]
        L.oracle_cache_dump.restype = _U64
        L.oracle_cache_dump.argtypes = [_P, _P, _P, _P, _U64]
        L.oracle_render_frame.restype = ctypes.c_int
        L.oracle_render_frame.argtypes = [_P, _np(np.uint32), _U64, _U32, _np(np.float32), _U32,
                                          _np(np.float32), ctypes.POINTER(FrameParams), _U32, _U32, _U32,
                                          _P, _P, _P, _P, ctypes.POINTER(Stats)]

    # -- scene ------------------------------------------------------------
    def build(self, depth: int, xyzm: np.ndarray) -> np.ndarray:
        v = np.ascontiguousarray(xyzm, np.uint32).reshape(-1)
        n = v.size // 4
        nv = _U32()
        size = self.lib.oracle_build(depth, v, n, np.zeros(1, np.uint32), 0, ctypes.byref(nv))
        out = np.zeros(size, np.uint32)
        self.lib.oracle_build(depth, v, n, out, size, ctypes.byref(nv))
        return out

    def fill_normals(self, words: np.ndarray, depth: int, fast: bool = False, threads: int = 1) -> np.ndarray:
        """Leaf normal fields by tree-descent occupancy lookups, or (fast) by
        an occupancy bitmask of all leaves."""
        w = np.ascontiguousarray(words, np.uint32).copy()
        self.lib.oracle_fill_normals_mode(w, w.size, depth, 1 if fast else 0, threads)
        return w

    def fill_normals_ball(self, words: np.ndarray, depth: int, radius: int, threads: int = 1):
        """The reference's normal mode (normal.comp's L2 ball of `radius`):
        (words with the leaves' code indices, the sorted code table)."""
        w = np.ascontiguousarray(words, np.uint32).copy()
        n = self.lib.oracle_fill_normals_ball(w.copy(), w.size, depth, radius, threads, None, 0)
        codes = np.zeros(max(n, 1), np.uint32)
        self.lib.oracle_fill_normals_ball(w, w.size, depth, radius, threads, codes.ctypes.data, n)
        return w, codes[:n]

    def occupied(self, words, depth, x, y, z) -> bool:
        return bool(self.lib.oracle_lookup_occupied(np.ascontiguousarray(words, np.uint32), words.size, depth,
                                                    x, y, z))

    def camera_ubo(self, pos, direction, fov, aspect) -> np.ndarray:
        out = np.zeros(16, np.float32)
        self.lib.oracle_camera_ubo(np.asarray(pos, np.float32), np.asarray(direction, np.float32), fov, aspect, out)
        return out

    def raycast(self, words, depth, o, d, controlchecks):
        out = np.zeros(8, np.uint32)
        cnt = (ctypes.c_uint64 * 2)()
        self.lib.oracle_raycast(np.ascontiguousarray(words, np.uint32), words.size, depth,
                                np.asarray(o, np.float32), np.asarray(d, np.float32), controlchecks, out,
                                ctypes.cast(cnt, _P))
        return out, (cnt[0], cnt[1])

    def raycast_batch(self, words, depth, origins, dirs, controlchecks, threads=8):
        """(n, 8) u32 rows {status, id, material, x, y, z, size, checks}."""
        o = np.ascontiguousarray(origins, np.float32).reshape(-1, 3)
        d = np.ascontiguousarray(dirs, np.float32).reshape(-1, 3)
        w = np.ascontiguousarray(words, np.uint32)
        out = np.zeros((o.shape[0], 8), np.uint32)
        self.lib.oracle_raycast_batch(w, w.size, depth, o.reshape(-1), d.reshape(-1), o.shape[0], controlchecks,
                                      threads, out.reshape(-1))
        return out

    LB_WIDTH, LB_SLOTS, LB_STRIDE = 32768, 32, 12

    def lb_apply(self, records: np.ndarray, params, table: np.ndarray) -> None:
        """depositSampleDual of (n, 8) u32 records {vid, 0, d.rgb f32, e.rgb f32}
        in order, on `table` ((32768 * 32 * 12,) u32, modified in place)."""
        r = np.ascontiguousarray(records, np.uint32)
        self.lib.oracle_lb_apply(r.reshape(-1), r.shape[0], ctypes.byref(params), table)

    def pow_unit(self, x, e) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32)
        e = np.ascontiguousarray(e, np.float32)
        out = np.zeros_like(x)
        self.lib.oracle_pow_unit(x, e, x.size, out)
        return out

    def voxel_key(self, x, y, z) -> int:
        return self.lib.oracle_voxel_key(x, y, z)

    def rand_seq(self, state: int, n: int):
        out = np.zeros(n, np.float32)
        st = self.lib.oracle_rand_seq(state, n, out)
        return out, st

    def sincos_turn(self, u: np.ndarray):
        u = np.ascontiguousarray(u, np.float32)
        s = np.zeros_like(u)
        c = np.zeros_like(u)
        self.lib.oracle_sincos_turn(u, u.size, s, c)
        return s, c

    def shading_normal(self, word: int, ray_dir) -> np.ndarray:
        out = np.zeros(3, np.float32)
        self.lib.oracle_shading_normal(word, np.asarray(ray_dir, np.float32), out)
        return out


class OracleRenderer:
    """Frame-by-frame CPU renderer with an FP64 radiance cache."""

    def __init__(self, oracle: Oracle):
        self.o = oracle
        self.h = oracle.lib.oracle_renderer_new()

    def __del__(self):
        if getattr(self, "h", None):
            self.o.lib.oracle_renderer_free(self.h)
            self.h = None

    def render(self, words: np.ndarray, depth: int, materials: np.ndarray, camera: np.ndarray, params: FrameParams,
               threads: int = 1, rows: Optional[tuple] = None, want_path_rgb: bool = False, want_rgb: bool = True):
        W, H = params.width, params.height
        gbuf = np.zeros((H, W, 4), np.uint32)
        rgb = np.zeros((H, W, 3), np.float32) if want_rgb else None
        mapped = np.zeros((H, W, 3), np.float32) if want_rgb else None
        n_paths = min(params.shading_budget, 2 * W * H) if params.flags & 64 else W * H * params.spp
        path_rgb = np.zeros((n_paths, 3), np.float32) if want_path_rgb else None
        st = Stats()
        r0, r1 = rows if rows else (0, 0)
        w = np.ascontiguousarray(words, np.uint32)
        m = np.ascontiguousarray(materials, np.float32).reshape(-1)
        cam = np.ascontiguousarray(camera, np.float32).reshape(16)
        rc = self.o.lib.oracle_render_frame(
            self.h, w, w.size, depth, m, m.size // 16, cam, ctypes.byref(params), threads, r0, r1,
            gbuf.ctypes.data, None if rgb is None else rgb.ctypes.data,
            None if mapped is None else mapped.ctypes.data, None if path_rgb is None else path_rgb.ctypes.data,
            ctypes.byref(st))
        assert rc == 0
        stats = {k: getattr(st, k) for k, _ in Stats._fields_}
        return {"gbuffer": gbuf, "rgb": rgb, "mapped": mapped, "path_rgb": path_rgb, "stats": stats}

    def set_normal_codes(self, codes: Optional[np.ndarray]) -> None:
        """The code table of a ball-normal scene (None: a gradient-normal scene)."""
        c = np.ascontiguousarray(codes if codes is not None else np.zeros(0), np.uint32)
        self.o.lib.oracle_renderer_set_normal_codes(self.h, c.ctypes.data if c.size else None, c.size)

    def lbuffer(self) -> np.ndarray:
        """Occupied lBuffer slots, (n, 14) u32 rows {row, slot, 12 slot words}."""
        n = self.o.lib.oracle_lbuffer_dump(self.h, None, 0)
        out = np.zeros((n, 14), np.uint32)
        self.o.lib.oracle_lbuffer_dump(self.h, out.ctypes.data, n)
        return out

    def cache(self):
        n = self.o.lib.oracle_cache_dump(self.h, None, None, None, 0)
        vids = np.zeros(n, np.uint32)
        counts = np.zeros(n, np.uint64)
        vals = np.zeros((n, 5), np.float64)
        self.o.lib.oracle_cache_dump(self.h, vids.ctypes.data, counts.ctypes.data, vals.ctypes.data, n)
        return vids, counts, vals


class Reference:
    """The reference's own OctreeCPU / Octree compiled in place (oracle/_ref)."""

    def __init__(self, path: str = REF_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = ctypes.CDLL(path)
        L.ref_scene_new.restype = _P
        L.ref_scene_new.argtypes = [_U32]
        L.ref_scene_free.argtypes = [_P]
        L.ref_insert.argtypes = [_P, _U32, _U32, _U32, _U32]
        L.ref_insert_many.argtypes = [_P, _np(np.uint32), _U64]
        L.ref_remove.argtypes = [_P, _U32, _U32, _U32]
        L.ref_insert_box.argtypes = [_P, _np(np.uint32), _np(np.uint32), _U32]
        L.ref_insert_sphere.argtypes = [_P, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, _U32]
        L.ref_lookup.restype = ctypes.c_int64
        L.ref_lookup.argtypes = [_P, _U32, _U32, _U32]
        L.ref_set.restype = _U64
        L.ref_set.argtypes = [_P, _np(np.uint32), _U64, ctypes.POINTER(_U32), ctypes.POINTER(_U32)]
        L.ref_apply_edits.restype = _U64
        L.ref_apply_edits.argtypes = [_P, _np(np.uint32), _U64, ctypes.POINTER(_U32)]
        L.ref_find_gpu_slot.restype = _U32
        L.ref_find_gpu_slot.argtypes = [_P, _U32, _U32, _U32]
        L.ref_raycast.restype = ctypes.c_int
        L.ref_raycast.argtypes = [_P, _np(np.float32), _np(np.float32), _U32, _np(np.uint32)]
        self.lib = L

    def scene(self, depth: int) -> "RefScene":
        return RefScene(self, depth)


class RefScene:
    def __init__(self, ref: Reference, depth: int):
        self.L = ref.lib
        self.h = self.L.ref_scene_new(depth)
        self.cap = 1 << 26

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ref_scene_free(self.h)
            self.h = None

    def insert(self, x, y, z, m):
        self.L.ref_insert(self.h, x, y, z, m)

    def insert_many(self, xyzm):
        a = np.ascontiguousarray(xyzm, np.uint32).reshape(-1)
        self.L.ref_insert_many(self.h, a, a.size // 4)

    def remove(self, x, y, z):
        self.L.ref_remove(self.h, x, y, z)

    def insert_box(self, mn, mx, m):
        self.L.ref_insert_box(self.h, np.asarray(mn, np.uint32), np.asarray(mx, np.uint32), m)

    def insert_sphere(self, c, r, m):
        self.L.ref_insert_sphere(self.h, float(c[0]), float(c[1]), float(c[2]), float(r), m)

    def lookup(self, x, y, z) -> int:
        return int(self.L.ref_lookup(self.h, x, y, z))

    def set(self):
        """Octree::set; returns (data words [capacity], size, numVoxels)."""
        size = _U32()
        nv = _U32()
        n = self.L.ref_set(self.h, np.zeros(1, np.uint32), 0, ctypes.byref(size), ctypes.byref(nv))
        out = np.zeros(n, np.uint32)
        # set() is idempotent for an unchanged tree, so it can run again to copy out
        self.L.ref_set(self.h, out, n, ctypes.byref(size), ctypes.byref(nv))
        return out, size.value, nv.value

    def apply_edits(self):
        size = _U32()
        out = np.zeros(self.cap, np.uint32)
        n = self.L.ref_apply_edits(self.h, out, self.cap, ctypes.byref(size))
        return out[: min(n, self.cap)].copy(), size.value

    def find_gpu_slot(self, x, y, z) -> int:
        return int(self.L.ref_find_gpu_slot(self.h, x, y, z))

    def raycast(self, o, d, max_steps=300):
        pos = np.zeros(3, np.uint32)
        hit = self.L.ref_raycast(self.h, np.asarray(o, np.float32), np.asarray(d, np.float32), max_steps, pos)
        return (True, tuple(int(v) for v in pos)) if hit else (False, None)


def frame_params(fc) -> FrameParams:
    """FrameParams from the product's FrameConfig dataclass (same fields)."""
    p = FrameParams()
    for f in ("width", "height", "spp", "bounces", "primary_controlchecks", "bounce_controlchecks",
              "reconstruction_radius", "render_type", "frame_index", "flags"):
        setattr(p, f, int(getattr(fc, f)))
    for i in range(3):
        p.sun_dir[i] = float(fc.sun_dir[i])
        p.sky[i] = float(fc.sky[i])
    p.sun_intensity = float(fc.sun_intensity)
    p.decay = float(fc.decay)
    p.variance_norm = float(fc.variance_norm)
    for f in ("weight_pixels", "weight_variance", "pixels_norm", "top_fraction", "mid_fraction"):
        setattr(p, f, float(getattr(fc, f, FrameParams_defaults[f])))
    for f in ("min_samples", "shading_budget", "restir", "restir_m", "restir_spatial_neighbors", "restir_max_m",
              "time", "update_time", "disable_stale_reset", "sample_cap_direct", "sample_cap_indirect"):
        setattr(p, f, int(getattr(fc, f, FrameParams_defaults[f])))
    for f in ("restir_spatial_radius", "firefly_k", "firefly_floor"):
        setattr(p, f, float(getattr(fc, f, FrameParams_defaults[f])))
    return p


# core.hpp:95-112 scheduling defaults, for frame configs without those fields
FrameParams_defaults = {"weight_pixels": 0.1, "weight_variance": 0.9, "pixels_norm": 100.0, "top_fraction": 0.30,
                        "mid_fraction": 0.40, "min_samples": 1, "shading_budget": 131072,
                        # core.hpp:138-144 ReSTIR defaults (enable | temporal | spatial)
                        "restir": 7, "restir_m": 4, "restir_spatial_neighbors": 1, "restir_max_m": 24,
                        "restir_spatial_radius": 2.75,
                        # core.hpp:93-104, 150-157 lBuffer defaults
                        "time": 0, "update_time": 0, "disable_stale_reset": 0, "sample_cap_direct": 16,
                        "sample_cap_indirect": 64, "firefly_k": 1.0, "firefly_floor": 255.0}
