"""Device edits: Octree::applyEdits words scattered on the device, then the
targeted refresh (normals of the edited voxels' 3x3x3 neighbourhoods, their
radiance-cache entries cleared) — the scene equals a fresh upload of the
edited tree with the full normal pass, and only the refreshed cache entries
are cleared."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def edited_tree(ve, rng, depth, n_remove, n_insert):
    vox = ve.terrain_voxels(depth, 1, 9)
    cpu = ve.OctreeCPU(depth)
    cpu.insert_many(vox)
    tree = ve.Octree(depth)
    tree.set(cpu)
    before = tree.words().copy()
    L = 1 << depth
    edited = []
    for v in vox[rng.choice(len(vox), n_remove, replace=False)]:
        cpu.remove(int(v[0]), int(v[1]), int(v[2]))
        edited.append(v[:3])
    for v in vox[rng.choice(len(vox), n_insert, replace=False)]:  # on top of existing voxels
        p = np.minimum(v[:3] + np.array([0, 1, 0], np.uint32), L - 1)
        cpu.insert(int(p[0]), int(p[1]), int(p[2]), int(rng.integers(1, 9)))
        edited.append(p)
    slots = tree.apply_edits(cpu)
    return before, tree.words(), slots, np.array(edited, np.uint32)


def test_targeted_refresh_matches_full_pass(ve):
    rng = np.random.default_rng(3)
    depth = 6
    before, after, slots, edited = edited_tree(ve, rng, depth, 40, 40)
    assert after.size == before.size, "the edit grew the array; pick fewer edits"
    r = ve.Renderer(hash_log2=14)
    try:
        sid = r.upload_scene(before, depth)
        r.apply_edits(sid, slots, after[slots], keep_normals=True)
        r.refresh_scene(sid, edited)
        got = r.download_scene(sid)
        full = r.upload_scene(after, depth)
        ref = r.download_scene(full)
        diff = np.nonzero(got != ref)[0]
        assert diff.size == 0, (diff[:10], got[diff[:10]], ref[diff[:10]])
        # the full-pass path of apply_edits gives the same words too
        sid3 = r.upload_scene(before, depth)
        r.apply_edits(sid3, slots, after[slots])
        assert np.array_equal(r.download_scene(sid3), ref)
    finally:
        r.close()


def test_refresh_clears_only_the_neighbourhood_cache_entries(ve, oracle):
    rng = np.random.default_rng(4)
    depth = 6
    vox = ve.terrain_voxels(depth, 1, 9)
    words, _ = ve.terrain_words(depth, 1, 9)
    r = ve.Renderer(hash_log2=16)
    try:
        r.set_materials(ve.terrain_materials(1))
        sid = r.upload_scene(words, depth)
        cam = ve.camera_ubo([32.0, 60.0, -30.0], [0.0, -0.6, 0.8], 70.0, 1.0)
        for f in range(3):
            r.render(sid, cam, ve.FrameConfig(width=96, height=96, spp=2, bounces=1, frame_index=f), outputs=())
        vids0, counts0, vals0 = r.cache_dump(sid)
        # visible voxels: the top of each column
        top = {}
        for x, y, z, _ in vox:
            if y >= top.get((x, z), (-1,))[0]:
                top[(x, z)] = (y,)
        cols = list(top.items())
        picked = np.array([[k[0], v[0], k[1]] for k, v in (cols[i] for i in rng.choice(len(cols), 30, replace=False))],
                          np.uint32)
        r.refresh_scene(sid, picked)
        vids1, counts1, vals1 = r.cache_dump(sid)
        assert np.array_equal(vids0, vids1)  # keys stay, probe chains intact
        cleared = set()
        L = 1 << depth
        for p in picked:
            for dx in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dz in (-1, 0, 1):
                        q = (int(p[0]) + dx, int(p[1]) + dy, int(p[2]) + dz)
                        if min(q) >= 0 and max(q) < L:
                            cleared.add(oracle.voxel_key(*q) + 1)
        hit = np.array([v in cleared for v in vids1])
        assert hit.any()
        assert np.all(counts1[hit] == 0) and np.all(vals1[hit] == 0)
        assert np.array_equal(counts1[~hit], counts0[~hit]) and np.array_equal(vals1[~hit], vals0[~hit])
        # the scene words (normals) were refreshed in place and are unchanged
        assert np.array_equal(r.download_scene(sid)[: words.size], r.download_scene(r.upload_scene(words, depth)))
    finally:
        r.close()
