"""The oracle-side benchmark workloads (oracle/scenes.py, oracle/terrain_oracle.cpp)
equal the product's: the CPU reference arm renders the same scene, camera,
materials and frame parameters as the device arm without loading the product
library."""
import ctypes

import numpy as np
import pytest

import helpers


@pytest.mark.parametrize("depth,variant,seed", [(1, 0, 1), (2, 0, 1), (3, 1, 1), (4, 0, 1), (5, 1, 3), (6, 1, 1),
                                                (7, 0, 1), (7, 1, 2), (8, 1, 11)])
def test_terrain_words_equal_product(ve, oracle, depth, variant, seed):
    from oracle import scenes

    a, na = scenes.terrain_words(oracle, depth, variant, seed)
    b, nb = ve.terrain_words(depth, variant, seed)
    assert na == nb
    assert np.array_equal(a, b)


def test_terrain_words_equal_pointer_tree(oracle):
    """The pyramid emitter equals the oracle's pointer-tree Octree::set on the
    terrain's own voxel list (independent build path)."""
    from oracle import scenes

    ve = helpers.package()
    for depth, variant in ((4, 1), (6, 0)):
        vox = ve.terrain_voxels(depth, variant, 1)
        a, na = scenes.terrain_words(oracle, depth, variant, 1)
        b = oracle.build(depth, vox)
        assert na == vox.shape[0]
        assert np.array_equal(a, b[: a.size]) and not b[a.size:].any()


def test_terrain_words_equal_reference(oracle, ref):
    """... and the reference's own compiled OctreeCPU::insert + Octree::set."""
    from oracle import scenes

    ve = helpers.package()
    depth = 6
    vox = ve.terrain_voxels(depth, 1, 1)
    rs = ref.scene(depth)
    rs.insert_many(vox)
    data, size, nv = rs.set()
    a, na = scenes.terrain_words(oracle, depth, 1, 1)
    assert size == a.size and nv == na
    assert np.array_equal(data[:size], a)


def test_materials_camera_params_equal_product(ve, oracle):
    from oracle import scenes
    from oracle.oracle import FrameParams, frame_params

    w = helpers.workloads()
    W = w.LARGE
    assert np.array_equal(scenes.terrain_materials(oracle, W.seed).view(np.uint32),
                          ve.terrain_materials(W.seed).view(np.uint32))
    for f in (0, 1, 17, 63, 64):
        eye, d = w.orbit_camera(f % W.frames, W.frames, W.seed)
        c = ve.camera_ubo(eye, d, W.fov, W.width / W.height)
        assert np.array_equal(scenes.large_camera(oracle, f).view(np.uint32), c.view(np.uint32))
        fc = ve.FrameConfig(width=W.width, height=W.height, spp=W.spp, bounces=W.bounces, frame_index=f % W.frames,
                            primary_controlchecks=W.primary_controlchecks, bounce_controlchecks=W.bounce_controlchecks)
        a, b = scenes.large_params(f % W.frames), frame_params(fc)
        assert bytes(a) == bytes(b), f"frame {f}: frame parameters differ"
    assert ctypes.sizeof(FrameParams) == len(bytes(scenes.large_params(0)))
    L = scenes.LARGE
    for k in ("depth", "variant", "seed", "width", "height", "spp", "bounces", "frames", "fov", "hash_log2",
              "primary_controlchecks", "bounce_controlchecks"):
        assert getattr(L, k) == getattr(W, k), k


def test_cpu_model_reported():
    from oracle import scenes

    assert isinstance(scenes.cpu_model(), str) and scenes.cpu_model()
