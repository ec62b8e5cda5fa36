"""GPU bulk octree builder: the node words built on the device equal those of
OctreeCPU.insert (every voxel, in order) followed by Octree.set — the host
restatement that tests/test_host_scene.py pins against the reference's own
compiled octree code — word for word, including repeated positions (last
insert wins), empty and single-voxel scenes, and the bulk terrain builder."""
import numpy as np
import pytest

import helpers

pytestmark = pytest.mark.gpu


def host_words(ve, depth, xyzm):
    cpu = ve.OctreeCPU(depth)
    if len(xyzm):
        cpu.insert_many(xyzm)
    tree = ve.Octree(depth)
    tree.set(cpu)
    return tree.words()[: tree.size]


@pytest.fixture(scope="module")
def renderer(ve):
    r = ve.Renderer(hash_log2=12)
    yield r
    r.close()


def check(ve, r, depth, xyzm):
    ref = host_words(ve, depth, xyzm)
    sid = r.build_scene(xyzm, depth, keep_normals=True)
    got = r.download_scene(sid)
    r.release_scene(sid)
    assert got.size == ref.size, (got.size, ref.size)
    diff = np.nonzero(got != ref)[0]
    assert diff.size == 0, (diff[:10], got[diff[:10]], ref[diff[:10]])


@pytest.mark.parametrize("depth,density,seed", [(1, 0.5, 1), (2, 0.3, 2), (3, 0.2, 3), (4, 0.1, 4), (5, 0.05, 5),
                                                (6, 0.02, 6), (7, 0.01, 7), (8, 0.002, 8)])
def test_random_scenes_match_octree_set(ve, renderer, depth, density, seed):
    rng = np.random.default_rng(seed)
    v = helpers.random_voxels(rng, depth, density)
    # repeated positions with other materials: the last row wins
    if len(v) > 4:
        dup = v[rng.integers(0, len(v), len(v) // 4)].copy()
        dup[:, 3] = rng.integers(1, 128, len(dup))
        v = np.concatenate([v, dup])
    check(ve, renderer, depth, v)


def test_edge_scenes(ve, renderer):
    check(ve, renderer, 5, np.zeros((0, 4), np.uint32))
    check(ve, renderer, 5, np.array([[31, 0, 17, 127]], np.uint32))
    full = np.array([[x, y, z, 1 + (x + y + z) % 8] for x in range(8) for y in range(8) for z in range(8)], np.uint32)
    check(ve, renderer, 3, full)  # every node has 8 children: the 3-bit count wraps to 0


def test_terrain_matches_bulk_builder(ve, renderer):
    depth = 8
    vox = ve.terrain_voxels(depth, 1, 5)
    words, _ = ve.terrain_words(depth, 1, 5)
    sid = renderer.build_scene(vox, depth, keep_normals=True)
    got = renderer.download_scene(sid)
    renderer.release_scene(sid)
    assert got.size == words.size and np.array_equal(got, words)


def test_built_scene_renders_like_uploaded(ve, renderer):
    depth = 6
    vox = ve.terrain_voxels(depth, 1, 3)
    words, _ = ve.terrain_words(depth, 1, 3)
    renderer.set_materials(ve.terrain_materials(1))
    a = renderer.build_scene(vox, depth)
    b = renderer.upload_scene(words, depth)
    assert np.array_equal(renderer.download_scene(a), renderer.download_scene(b))  # normals included
    cam = ve.camera_ubo([32.0, 50.0, -20.0], [0.0, -0.5, 0.866], 70.0, 1.0)
    fc = ve.FrameConfig(width=64, height=64, spp=1, bounces=1)
    ra = renderer.render(a, cam, fc, outputs=("voxel_id", "gbuffer"))
    rb = renderer.render(b, cam, fc, outputs=("voxel_id", "gbuffer"))
    assert np.array_equal(ra["voxel_id"], rb["voxel_id"]) and np.array_equal(ra["gbuffer"], rb["gbuffer"])
    renderer.release_scene(a)
    renderer.release_scene(b)


def test_invalid_voxels_are_rejected(ve, renderer):
    with pytest.raises(ve.VeError):
        renderer.build_scene(np.array([[8, 0, 0, 1]], np.uint32), 3)
    with pytest.raises(ve.VeError):
        renderer.build_scene(np.array([[1, 0, 0, 0]], np.uint32), 3)
