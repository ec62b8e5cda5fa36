"""TEST INFRASTRUCTURE ONLY — the benchmark workloads on the CPU side, built
without the product library: the terrain scene's node words
(oracle/terrain_oracle.cpp), its material table, the seeded orbit camera and
the frame parameters of the large workload.

The timed reference arm of bench.py (``--impl reference``) renders from these,
so that process maps only the oracle's libraries; tests check every item here
against the product's own workload definitions.
"""
from __future__ import annotations

import ctypes
import dataclasses
import math

import numpy as np

from .oracle import FrameParams, Oracle

_P = ctypes.c_void_p
_U32 = ctypes.c_uint32
_U64 = ctypes.c_uint64


@dataclasses.dataclass(frozen=True)
class Large:
    """depth-10 (1024^3) terrain with overhangs (variant 1, seed 1), 1920x1080,
    4 spp x 3 bounces, radiance cache 2^22 entries with decay 0.95, 64 frames
    on a circular orbit of radius 600 at height 300 around (512, 64, 512),
    vertical FOV 70 degrees, controlchecks 300 / 300."""
    depth: int = 10
    variant: int = 1
    seed: int = 1
    width: int = 1920
    height: int = 1080
    spp: int = 4
    bounces: int = 3
    frames: int = 64
    fov: float = 70.0
    hash_log2: int = 22
    primary_controlchecks: int = 300
    bounce_controlchecks: int = 300


LARGE = Large()

SUN_DIR = (np.array([0.3, 1.0, 0.2]) / np.linalg.norm([0.3, 1.0, 0.2])).astype(np.float32)


def _bind(orc: Oracle) -> None:
    L = orc.lib
    if getattr(L, "_terrain_bound", False):
        return
    L.oracle_terrain_build.restype = _P
    L.oracle_terrain_build.argtypes = [_U32, _U32, _U64, _U32, ctypes.POINTER(_U64), ctypes.POINTER(_U64)]
    L.oracle_terrain_data.restype = _P
    L.oracle_terrain_data.argtypes = [_P]
    L.oracle_terrain_free.argtypes = [_P]
    L.oracle_terrain_materials.argtypes = [_U64, _P]
    L._terrain_bound = True


def terrain_words(orc: Oracle, depth: int, variant: int = 0, seed: int = 1, threads: int = 0):
    """Node words (Octree::set order) of the seeded terrain; (words, n_voxels)."""
    _bind(orc)
    nw, nv = _U64(), _U64()
    h = orc.lib.oracle_terrain_build(depth, variant, seed, threads, ctypes.byref(nw), ctypes.byref(nv))
    if not h:
        raise ValueError(f"terrain depth {depth} variant {variant} does not fit the node layout")
    try:
        buf = (ctypes.c_uint32 * nw.value).from_address(orc.lib.oracle_terrain_data(h))
        words = np.frombuffer(buf, dtype=np.uint32).copy()
    finally:
        orc.lib.oracle_terrain_free(h)
    return words, nv.value


def terrain_materials(orc: Oracle, seed: int = 1) -> np.ndarray:
    """128 std140 Material entries as a (128, 16) float32 array."""
    _bind(orc)
    out = np.zeros((128, 16), np.float32)
    orc.lib.oracle_terrain_materials(seed, out.ctypes.data)
    return out


def orbit_camera(frame: int, n_frames: int = 64, seed: int = 1, radius: float = 600.0, height: float = 300.0):
    """Eye and unit view direction of orbit frame `frame`: start angle drawn
    from numpy's default_rng(seed), one turn per `n_frames` frames."""
    rng = np.random.default_rng(seed)
    theta0 = float(rng.uniform(0.0, 2.0 * math.pi))
    th = theta0 + 2.0 * math.pi * frame / n_frames
    eye = np.array([512.0 + radius * math.cos(th), height, 512.0 + radius * math.sin(th)])
    d = np.array([512.0, 64.0, 512.0]) - eye
    return eye.astype(np.float32), (d / np.linalg.norm(d)).astype(np.float32)


def large_camera(orc: Oracle, frame: int, w: Large = LARGE) -> np.ndarray:
    eye, d = orbit_camera(frame % w.frames, w.frames, w.seed)
    return orc.camera_ubo(eye, d, w.fov, w.width / w.height)


def large_params(frame: int, w: Large = LARGE, flags: int = 0) -> FrameParams:
    """Frame parameters of the large workload: sun normalize(0.3, 1, 0.2) with
    irradiance pi, sky 0.4, decay 0.95, reconstruction radius 10, DEFAULT render
    type; the scheduling / emissive / lBuffer knobs keep the reference's
    defaults (unused by the plain method)."""
    p = FrameParams()
    p.width, p.height, p.spp, p.bounces = w.width, w.height, w.spp, w.bounces
    p.primary_controlchecks, p.bounce_controlchecks = w.primary_controlchecks, w.bounce_controlchecks
    p.reconstruction_radius = 10
    p.render_type = 0
    p.frame_index = frame
    for i in range(3):
        p.sun_dir[i] = float(SUN_DIR[i])
        p.sky[i] = 0.4
    p.sun_intensity = math.pi
    p.decay = 0.95
    p.variance_norm = 10000.0
    p.flags = flags
    p.weight_pixels, p.weight_variance, p.pixels_norm = 0.1, 0.9, 100.0
    p.top_fraction, p.mid_fraction = 0.30, 0.40
    p.min_samples, p.shading_budget = 1, 131072
    p.restir, p.restir_m, p.restir_spatial_neighbors, p.restir_max_m = 7, 4, 1, 24
    p.restir_spatial_radius = 2.75
    p.time, p.update_time, p.disable_stale_reset = 0, 0, 0
    p.sample_cap_direct, p.sample_cap_indirect = 16, 64
    p.firefly_k, p.firefly_floor = 1.0, 255.0
    return p


def cpu_model() -> str:
    """The host CPU's model name from /proc/cpuinfo (or the platform string)."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform

    return platform.processor() or platform.machine()
