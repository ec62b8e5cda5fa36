"""Host scene layer against the reference's own compiled octree code
(oracle/_ref: src/octree_cpu.cpp + src/renderer/octree.cpp built in place):
node words, slot order, applyEdits, findGpuSlot, lookup and raycast; and the
parallel terrain bulk builder against the OctreeCPU + Octree::set path."""
import numpy as np
import pytest

import helpers


def build_product(ve, depth, voxels):
    c = ve.OctreeCPU(depth)
    c.insert_many(voxels)
    o = ve.Octree(depth)
    o.set(c)
    return c, o


@pytest.mark.parametrize("depth,density,seed", [(1, 0.5, 0), (2, 0.3, 1), (3, 0.2, 2), (4, 0.05, 3),
                                                (5, 0.1, 4), (6, 0.01, 5), (7, 0.002, 6)])
def test_set_matches_reference_words(ve, ref, depth, density, seed):
    rng = np.random.default_rng(seed)
    v = helpers.random_voxels(rng, depth, density)
    rs = ref.scene(depth)
    rs.insert_many(v)
    rwords, rsize, rnv = rs.set()
    c, o = build_product(ve, depth, v)
    size, cap, nv = o.info()
    assert (size, nv) == (rsize, rnv)
    assert cap == rwords.size
    assert np.array_equal(o.words(), rwords)


def test_boxes_spheres_match_reference(ve, ref):
    depth = 6
    rs = ref.scene(depth)
    c = ve.OctreeCPU(depth)
    ops = [("box", (0, 0, 0), (64, 4, 64), 3), ("box", (0, 0, 0), (4, 64, 64), 2),
           ("sphere", (21.33, 16.3, 32.0), 16.0, 5), ("sphere", (43.0, 33.0, 43.0), 16.0, 4),
           ("box", (16, 56, 16), (48, 60, 48), 1), ("sphere", (0.5, 63.2, 10.0), 7.5, 6)]
    for op in ops:
        if op[0] == "box":
            rs.insert_box(op[1], op[2], op[3])
            c.insert_box(op[1], op[2], op[3])
        else:
            rs.insert_sphere(op[1], op[2], op[3])
            c.insert_sphere(op[1], op[2], op[3])
    rwords, rsize, rnv = rs.set()
    o = ve.Octree(depth)
    o.set(c)
    assert o.info()[:1] == (rsize,) and o.num_voxels == rnv
    assert np.array_equal(o.words(), rwords)


def test_lookup_and_find_gpu_slot_match_reference(ve, ref):
    rng = np.random.default_rng(7)
    depth = 5
    v = helpers.random_voxels(rng, depth, 0.08)
    rs = ref.scene(depth)
    rs.insert_many(v)
    rs.set()
    c, o = build_product(ve, depth, v)
    for p in rng.integers(0, 1 << depth, (500, 3)):
        x, y, z = (int(t) for t in p)
        assert c.lookup(x, y, z) == rs.lookup(x, y, z)
        assert o.find_gpu_slot(c, (x, y, z)) == rs.find_gpu_slot(x, y, z)
    assert c.lookup(1 << depth, 0, 0) == -1 == rs.lookup(1 << depth, 0, 0)


def test_apply_edits_matches_reference(ve, ref):
    rng = np.random.default_rng(11)
    depth = 5
    v = helpers.random_voxels(rng, depth, 0.05)
    rs = ref.scene(depth)
    rs.insert_many(v)
    rs.set()
    c, o = build_product(ve, depth, v)
    before = o.words()
    for rnd in range(4):
        for _ in range(60):
            x, y, z = (int(t) for t in rng.integers(0, 1 << depth, 3))
            if rng.random() < 0.5:
                m = int(rng.integers(1, 9))
                rs.insert(x, y, z, m)
                c.insert(x, y, z, m)
            else:
                rs.remove(x, y, z)
                c.remove(x, y, z)
        rwords, rsize = rs.apply_edits()
        changed = o.apply_edits(c)
        after = o.words()
        assert o.size == rsize
        assert np.array_equal(after, rwords[: after.size]) and not rwords[after.size:].any()
        # every word that differs from the previous upload is in the changed list
        n = min(before.size, after.size)
        diff = set(np.nonzero(before[:n] != after[:n])[0].tolist()) | set(range(n, after.size)) - set(
            np.nonzero(after[n:] == 0)[0] + n)
        assert diff <= set(changed.tolist())
        before = after


def test_remove_everything(ve, ref):
    depth = 3
    c = ve.OctreeCPU(depth)
    rs = ref.scene(depth)
    for p in [(1, 2, 3), (7, 7, 7), (0, 0, 0)]:
        c.insert(*p, 2)
        rs.insert(*p, 2)
    for p in [(1, 2, 3), (7, 7, 7), (0, 0, 0), (5, 5, 5)]:
        c.remove(*p)
        rs.remove(*p)
    assert c.lookup(1, 2, 3) == -1 == rs.lookup(1, 2, 3)


def test_raycast_matches_reference(ve, ref):
    rng = np.random.default_rng(3)
    depth = 6
    L = 1 << depth
    v = helpers.random_voxels(rng, depth, 0.01)
    rs = ref.scene(depth)
    rs.insert_many(v)
    c, _ = build_product(ve, depth, v)
    hits = 0
    for _ in range(2000):
        o = rng.uniform(-0.5 * L, 1.5 * L, 3).astype(np.float32)
        d = rng.normal(size=3)
        d = (d / np.linalg.norm(d)).astype(np.float32)
        if rng.random() < 0.1:  # axis-aligned directions (reciprocals of 0 -> inf)
            d = np.zeros(3, np.float32)
            d[rng.integers(0, 3)] = rng.choice([-1.0, 1.0])
        a = c.raycast(o, d, 300)
        b = rs.raycast(o, d, 300)
        assert a == b
        hits += a[0]
    assert hits > 100


@pytest.mark.parametrize("depth,variant,seed", [(4, 0, 1), (5, 1, 2), (6, 0, 3), (6, 1, 4), (7, 0, 1), (7, 1, 9)])
def test_terrain_bulk_builder_matches_octree_set(ve, depth, variant, seed):
    words, nv = ve.terrain_words(depth, variant, seed)
    vox = ve.terrain_voxels(depth, variant, seed)
    c, o = build_product(ve, depth, vox)
    assert nv == vox.shape[0] == o.num_voxels
    assert words.size == o.size
    assert np.array_equal(words, o.words()[: o.size])


def test_terrain_bulk_builder_matches_reference(ve, ref):
    depth = 6
    vox = ve.terrain_voxels(depth, 1, 5)
    rs = ref.scene(depth)
    rs.insert_many(vox)
    rwords, rsize, rnv = rs.set()
    words, nv = ve.terrain_words(depth, 1, 5)
    assert (words.size, nv) == (rsize, rnv)
    assert np.array_equal(words, rwords[:rsize])


def test_small_terrain_shape(ve):
    words, nv = ve.terrain_words(7, 0, 1)
    vox = ve.terrain_voxels(7, 0, 1)
    assert 500_000 < nv < 2_000_000
    assert vox[:, 3].min() == 1 and vox[:, 3].max() == 8
    # heights 64 + 32 fBm stay inside the domain
    assert vox[:, 1].max() < 127 and vox[:, 1].min() == 0


def test_camera_ubo_matches_oracle(ve, oracle):
    for eye, target, fov, aspect in [((64, 120, -40), (64, 48, 64), 70.0, 1.0),
                                     ((10, 300, 1100), (512, 64, 512), 70.0, 16 / 9),
                                     ((1, 2, 3), (4, 1, 9), 90.0, 0.5)]:
        d = ve.look_at(eye, target)
        a = ve.camera_ubo(eye, d, fov, aspect)
        b = oracle.camera_ubo(np.asarray(eye, np.float32), d, fov, aspect)
        assert np.array_equal(a, b)
        # basis: right _|_ dir, up _|_ dir, vertical FOV
        right, up = a[8:11].astype(np.float64), a[12:15].astype(np.float64)
        assert abs(right @ d) < 1e-5 and abs(up @ d) < 1e-5
        assert np.isclose(np.linalg.norm(up), np.tan(np.radians(fov / 2)), rtol=1e-5)


def test_materials_table(ve):
    m = ve.terrain_materials(1)
    assert m.shape == (128, 16)
    assert not m[0].any()
    alb = m[1:9, :3]
    assert (alb >= 0.2).all() and (alb <= 0.9).all()
    assert (m[1:9, 8] == 1.0).all() and (m[1:9, 10] == 0.0).all()  # roughness 1, metallic 0
    assert not m[9:].any()
