"""Benchmark workloads of the plain method (seeded, synthetic).

* ``small``: depth-7 (128^3) value-noise terrain, 256x256, vertical FOV 70,
  eye (64,120,-40) looking at (64,48,64), 1 spp x 1 bounce, 16 frames with a
  fixed camera, sun normalize(0.3,1,0.2), sky 0.4.
* ``large``: depth-10 (1024^3) terrain of the same family plus 3 octaves of
  3D overhang noise, 1920x1080, 4 spp x 3 bounces, radiance cache 2^22
  entries with decay 0.95, 64 frames on a seeded circular orbit of radius 600
  around the scene centre (eye height 300, looking at (512, 64, 512)).
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Tuple

import numpy as np


@dataclasses.dataclass
class Workload:
    name: str
    depth: int
    variant: int
    seed: int
    width: int
    height: int
    spp: int
    bounces: int
    frames: int
    fov: float
    hash_log2: int
    primary_controlchecks: int
    bounce_controlchecks: int


SMALL = Workload("small", depth=7, variant=0, seed=1, width=256, height=256, spp=1, bounces=1, frames=16,
                 fov=70.0, hash_log2=22, primary_controlchecks=70, bounce_controlchecks=100)
# controlchecks 300/300: a depth-10 scene is 8x the extent of the reference's
# depth-7 defaults (core.hpp:85-86 give 70/100 for its depth-8 demo).
LARGE = Workload("large", depth=10, variant=1, seed=1, width=1920, height=1080, spp=4, bounces=3, frames=64,
                 fov=70.0, hash_log2=22, primary_controlchecks=300, bounce_controlchecks=300)


def small_camera() -> Tuple[np.ndarray, np.ndarray]:
    eye = np.array([64.0, 120.0, -40.0], np.float32)
    target = np.array([64.0, 48.0, 64.0])
    d = target - eye.astype(np.float64)
    return eye, (d / np.linalg.norm(d)).astype(np.float32)


def orbit_camera(frame: int, n_frames: int = 64, seed: int = 1, radius: float = 600.0,
                 height: float = 300.0) -> Tuple[np.ndarray, np.ndarray]:
    """Seeded circular orbit around the depth-10 scene centre."""
    rng = np.random.default_rng(seed)
    theta0 = float(rng.uniform(0.0, 2.0 * math.pi))
    th = theta0 + 2.0 * math.pi * frame / n_frames
    eye = np.array([512.0 + radius * math.cos(th), height, 512.0 + radius * math.sin(th)])
    target = np.array([512.0, 64.0, 512.0])
    d = target - eye
    return eye.astype(np.float32), (d / np.linalg.norm(d)).astype(np.float32)


# Batching workload: 64 views over 4 resident octrees of depth 8, 9, 10, 10
# (seeded terrain with overhangs), resolutions drawn from BATCH_RESOLUTIONS,
# spp uniform 1-8, bounces uniform 1-4, random poses.
BATCH_RESOLUTIONS = [(128, 128), (256, 256), (640, 360), (1280, 720), (1920, 1080)]
BATCH_SCENES = [(8, 1, 11), (9, 1, 12), (10, 1, 13), (10, 1, 14)]  # (depth, variant, seed)


def random_pose(rng, depth: int) -> Tuple[np.ndarray, np.ndarray]:
    """Eye on a circle of radius 0.6 L at height 0.2-0.35 L, looking at the
    terrain centre (heights are 64 +- 48 at every depth)."""
    L = float(1 << depth)
    th = float(rng.uniform(0.0, 2.0 * math.pi))
    eye = np.array([L / 2 + 0.6 * L * math.cos(th), float(rng.uniform(0.2, 0.35)) * L, L / 2 + 0.6 * L * math.sin(th)])
    target = np.array([L / 2 + float(rng.uniform(-0.1, 0.1)) * L, 64.0, L / 2 + float(rng.uniform(-0.1, 0.1)) * L])
    d = target - eye
    return eye.astype(np.float32), (d / np.linalg.norm(d)).astype(np.float32)


def batching_views(n: int = 64, seed: int = 7) -> List[dict]:
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        sc = int(rng.integers(0, len(BATCH_SCENES)))
        w, h = BATCH_RESOLUTIONS[int(rng.integers(0, len(BATCH_RESOLUTIONS)))]
        eye, d = random_pose(rng, BATCH_SCENES[sc][0])
        out.append({"scene": sc, "width": w, "height": h, "spp": int(rng.integers(1, 9)),
                    "bounces": int(rng.integers(1, 5)), "eye": eye, "dir": d, "frame": i})
    return out


# Serving workload: 8 resident octrees of depth 8-11 (two per depth; depth 11
# is the "island" variant, the overhang terrain on the central 1024^2
# columns, because the full-extent depth-11 terrain needs more than 2^28 node
# slots), requests {scene uniform, resolution from BATCH_RESOLUTIONS, spp 1-16,
# bounces 1-4, seeded pose}.
SERVING_SCENES = [(8, 1, 31), (9, 1, 32), (10, 1, 33), (11, 2, 34), (8, 1, 35), (9, 1, 36), (10, 1, 37), (11, 2, 38)]


def serving_requests(n: int = 10000, seed: int = 5) -> List[dict]:
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        sc = int(rng.integers(0, len(SERVING_SCENES)))
        w, h = BATCH_RESOLUTIONS[int(rng.integers(0, len(BATCH_RESOLUTIONS)))]
        eye, d = random_pose(rng, SERVING_SCENES[sc][0])
        out.append({"scene": sc, "width": w, "height": h, "spp": int(rng.integers(1, 17)),
                    "bounces": int(rng.integers(1, 5)), "eye": eye, "dir": d, "frame": i})
    return out


def camera_sequence(w: Workload) -> List[Tuple[np.ndarray, np.ndarray]]:
    if w.name == "small":
        return [small_camera()] * w.frames
    return [orbit_camera(f, w.frames, w.seed) for f in range(w.frames)]


# ---------------------------------------------------------------------------
# The reference's default emissive scene: the Cornell box of
# src/voxelengine.cpp:82-142 (depth 8, camera of :41-46), for VE_FRAME_EMISSIVE.
# ---------------------------------------------------------------------------
CORNELL = Workload("cornell", depth=8, variant=0, seed=0, width=512, height=512, spp=1, bounces=3, frames=16,
                   fov=90.0, hash_log2=22, primary_controlchecks=70, bounce_controlchecks=120)
# material indices in MaterialPool::addMaterial order (index 0 is reserved)
CORNELL_EMISSIVE, CORNELL_RED, CORNELL_GREEN, CORNELL_WHITE, CORNELL_METALLIC, CORNELL_BLUE = 1, 2, 3, 4, 5, 6


def cornell_materials() -> np.ndarray:
    """128 std140 Material entries (64 B: color, specularColor, roughness,
    specular, metallic, emissive (int), emissiveIntensity) as (128, 16) f32."""
    out = np.zeros((128, 16), np.float32)
    mats = {  # color, specularColor, roughness, specular, metallic, emissive, intensity
        CORNELL_EMISSIVE: ((1, 1, 1, 0), (1, 1, 1, 1), 0.4, 0.03, 0.2, 1, 10.0),
        CORNELL_RED: ((1, 0, 0, 0), (0.8, 0.1, 0.1, 1), 0.1, 0.9, 0.2, 0, 0.0),
        CORNELL_GREEN: ((0, 1, 0, 0), (1, 1, 1, 1), 0.8, 0.1, 0.0, 0, 0.0),
        CORNELL_WHITE: ((1, 1, 1, 0), (1, 1, 1, 1), 0.6, 0.2, 0.0, 0, 0.0),
        CORNELL_METALLIC: ((0.8, 0.8, 0.8, 0), (1, 1, 1, 1), 0.15, 1.0, 0.7, 0, 0.0),
        CORNELL_BLUE: ((0, 0, 1, 0), (1, 1, 1, 1), 0.8, 0.1, 0.0, 0, 0.0),
    }
    for i, (col, spc, rough, spec, metal, emissive, intensity) in mats.items():
        out[i, 0:4] = col
        out[i, 4:8] = spc
        out[i, 8] = rough
        out[i, 9] = spec
        out[i, 10] = metal
        out[i, 11] = np.array([emissive], np.int32).view(np.float32)[0]
        out[i, 12] = intensity
    return out


def cornell_build(cpu, depth: int = 8) -> None:
    """The scene's insertSphere / insertBox calls, in their order, on an
    OctreeCPU-like object (ours or the reference's own)."""
    L = 1 << depth
    f = np.float32
    cpu.insert_sphere((f(L) / f(3), f(L) / f(3) - f(5), f(L) / f(2)), f(L) / f(4), CORNELL_METALLIC)
    cpu.insert_sphere((f(L) * f(3) / f(4) - f(5), f(L) * f(3) / f(4) - f(15), f(L) * f(3) / f(4) - f(5)), f(L) / f(4),
                      CORNELL_WHITE)
    cpu.insert_box((0, 0, 0), (L, 4, L), CORNELL_WHITE)            # floor
    cpu.insert_box((0, 0, 0), (4, L, L), CORNELL_GREEN)            # left wall
    cpu.insert_box((L - 4, 0, 0), (L, L, L), CORNELL_RED)          # right wall
    cpu.insert_box((0, 0, L - 4), (L, L, L), CORNELL_METALLIC)     # back wall (mirror)
    cpu.insert_box((0, L - 4, 0), (L, L, L), CORNELL_WHITE)        # ceiling
    cpu.insert_box((L // 4, L - 8, L // 4), (L * 3 // 4, L - 4, L * 3 // 4), CORNELL_EMISSIVE)  # light panel


def cornell_camera(depth: int = 8) -> Tuple[np.ndarray, np.ndarray]:
    """Camera::Config of src/voxelengine.cpp:41-46: (L/2, L/2, -L/2) looking +z."""
    h = float(1 << (depth - 1))
    return np.array([h, h, -h], np.float32), np.array([0.0, 0.0, 1.0], np.float32)
