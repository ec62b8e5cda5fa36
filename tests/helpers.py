"""Shared test helpers: package loading and the small benchmark scene."""
import functools
import importlib.util
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "voxelengine3.0_b200")


def package():
    """Imports the package directory (its name is not a Python identifier)."""
    if "ve_b200" in sys.modules:
        return sys.modules["ve_b200"]
    lib = os.path.join(PKG_DIR, "libve.so")
    if not os.path.exists(lib):
        spec_b = importlib.util.spec_from_file_location("ve_b200_build", os.path.join(PKG_DIR, "build.py"))
        b = importlib.util.module_from_spec(spec_b)
        spec_b.loader.exec_module(b)
        b.build()
    spec = importlib.util.spec_from_file_location("ve_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    m = importlib.util.module_from_spec(spec)
    sys.modules["ve_b200"] = m
    spec.loader.exec_module(m)
    return m


def workloads():
    package()
    import ve_b200.workloads as w  # noqa: E402

    return w


@functools.lru_cache(maxsize=None)
def terrain(depth, variant=0, seed=1):
    ve = package()
    words, nv = ve.terrain_words(depth, variant, seed)
    return words, nv


def small_setup():
    """(words, depth, materials, camera ubo, FrameConfig) of the small workload."""
    ve = package()
    w = workloads()
    S = w.SMALL
    words, _ = terrain(S.depth, S.variant, S.seed)
    mats = ve.terrain_materials(S.seed)
    eye, d = w.small_camera()
    cam = ve.camera_ubo(eye, d, S.fov, S.width / S.height)
    fc = ve.FrameConfig(width=S.width, height=S.height, spp=S.spp, bounces=S.bounces,
                        primary_controlchecks=S.primary_controlchecks,
                        bounce_controlchecks=S.bounce_controlchecks)
    return words, S.depth, mats, cam, fc


def random_voxels(rng, depth, density):
    L = 1 << depth
    n = max(1, int(L ** 3 * density))
    v = np.zeros((n, 4), np.uint32)
    v[:, :3] = rng.integers(0, L, (n, 3))
    v[:, 3] = rng.integers(1, 9, n)
    return v
