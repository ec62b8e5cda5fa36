"""The oracle's restatement of the reference's normal pass
(normal.comp:55-95 computeRefinedNormal + packNormalAccum, at the voxel's
even-aligned corner, normal.comp:147-152) against an independent numpy
transcription on small scenes."""
import numpy as np
import pytest

import helpers


def _pack(c):
    v = (np.float32(c) + np.float32(1.0)) * np.float32(511.0)  # float32, as the shader
    q = int(np.floor(np.float64(v) + 0.5))  # round half away from zero (v >= 0)
    return min(max(q, 0), 1022)


def _numpy_ball(words, depth, voxels, radius):
    L = 1 << depth
    occ = np.zeros((L, L, L), bool)
    occ[voxels[:, 0], voxels[:, 1], voxels[:, 2]] = True
    R = radius
    offs = [(dx, dy, dz) for dx in range(-R, R + 1) for dy in range(-R, R + 1) for dz in range(-R, R + 1)
            if (dx, dy, dz) != (0, 0, 0) and dx * dx + dy * dy + dz * dz <= R * R]
    codes = {}
    for x, y, z in voxels[:, :3]:
        cx, cy, cz = int(x) & ~1, int(y) & ~1, int(z) & ~1
        a = np.zeros(3, np.int64)
        for dx, dy, dz in offs:
            nx, ny, nz = cx + dx, cy + dy, cz + dz
            inside = 0 <= nx < L and 0 <= ny < L and 0 <= nz < L
            if not (inside and occ[nx, ny, nz]):
                a += (dx, dy, dz)
        acc = a.astype(np.float32)
        dot = (acc[0] * acc[0] + acc[1] * acc[1]) + acc[2] * acc[2]
        ln = np.sqrt(np.float32(dot))
        n = acc / ln if ln > np.float32(0.001) else np.array([0, 1, 0], np.float32)
        codes[(int(x), int(y), int(z))] = (_pack(n[0]) << 22) | (_pack(n[1]) << 12) | (_pack(n[2]) << 2)
    return codes


@pytest.mark.parametrize("radius", [1, 2, 3, 5])
def test_oracle_ball_normals_match_numpy(ve, oracle, radius):
    rng = np.random.default_rng(radius)
    depth = 4
    vox = helpers.random_voxels(rng, depth, 0.3)
    # a solid floor as well, so interior corners occur
    fl = np.array([(x, y, z, 2) for x in range(16) for y in range(3) for z in range(16)], np.uint32)
    vox = np.concatenate([vox, fl])
    c = ve.OctreeCPU(depth)
    c.insert_many(vox)
    o = ve.Octree(depth)
    o.set(c)
    words = o.words()[: o.size]
    uniq = np.unique(vox[:, :3], axis=0)
    want = _numpy_ball(words, depth, uniq, radius)
    got_words, table = oracle.fill_normals_ball(words, depth, radius, threads=2)
    assert list(table) == sorted(set(want.values()))
    for x, y, z in uniq:
        slot = o.find_gpu_slot(c, (int(x), int(y), int(z)))
        w = got_words[slot]
        assert (w >> 31) == 0 and (w & 0xFF) == (words[slot] & 0xFF)
        assert table[((w >> 8) & 0x7FFFFF) - 1] == want[(int(x), int(y), int(z))]
