"""Ray-by-ray parity of the device DDA (ve_raycast_batch) with the oracle's
restatement of Raycast / RaycastCounted (internal.glsl:297-400).

Every field is compared exactly: status (hit / left the volume / out of
controlchecks), hit node slot, material, integer position, node size and the
check count.  Ray sets stress the traversal's ties: origins on integer and
half-integer lattice points, directions with zero or equal components, rays
from outside the volume, grazing rays along faces, and short controlcheck
budgets that end rays mid-walk; both the top-table descent and the full
per-level walk are checked.
"""
import numpy as np
import pytest

import helpers


def ray_sets(rng, depth, n):
    L = float(1 << depth)
    sets = {}
    o = rng.uniform(0, L, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    sets["random"] = (o, d)
    # lattice origins, directions with ties (zero / equal components)
    o = rng.integers(0, 1 << depth, (n, 3)).astype(np.float32) + rng.choice([0.0, 0.5, 1.0], (n, 3))
    d = rng.choice([-1.0, -0.5, 0.0, 0.5, 1.0], (n, 3))
    d[np.abs(d).sum(1) == 0] = (1.0, 1.0, 1.0)
    sets["lattice"] = (o.astype(np.float32), d)
    # from outside the volume toward its interior
    c = rng.uniform(0, L, (n, 3))
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    o = c + u * L * rng.uniform(0.6, 2.0, (n, 1))
    sets["outside"] = (o.astype(np.float32), c - o)
    # grazing: origin on a face plane, direction in the plane (+ tiny tilt)
    o = rng.uniform(0, L, (n, 3))
    ax = rng.integers(0, 3, n)
    o[np.arange(n), ax] = np.round(o[np.arange(n), ax])
    d = rng.normal(size=(n, 3))
    d[np.arange(n), ax] = rng.choice([0.0, 1e-7, -1e-7], n)
    sets["grazing"] = (o.astype(np.float32), d)
    out = {}
    for k, (o, d) in sets.items():
        d = np.asarray(d, np.float64)
        d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
        out[k] = (np.asarray(o, np.float32), d)
    return out


def shading_rays(rng, words, depth, oracle, n):
    """Secondary rays as the bounce loop casts them: from hit voxel + 0.5 +
    shading normal, random hemisphere directions."""
    L = 1 << depth
    cam_o = rng.uniform(0, L, (n, 3)).astype(np.float32)
    cam_d = rng.normal(size=(n, 3))
    cam_d = (cam_d / np.linalg.norm(cam_d, axis=1, keepdims=True)).astype(np.float32)
    prim = oracle.raycast_batch(words, depth, cam_o, cam_d, 300)
    hit = prim[:, 0] == 0
    prim, cam_d = prim[hit], cam_d[hit]
    o = np.zeros((prim.shape[0], 3), np.float32)
    for i in range(prim.shape[0]):
        N = oracle.shading_normal(int(words[prim[i, 1]]), cam_d[i])
        o[i] = (prim[i, 3:6].astype(np.float32) + np.float32(0.5)) + N.astype(np.float32)
    d = rng.normal(size=o.shape)
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    return o, d


def test_oracle_batch_matches_single(oracle):
    words, depth, *_ = helpers.small_setup()
    words = oracle.fill_normals(words, depth)
    rng = np.random.default_rng(5)
    for name, (o, d) in ray_sets(rng, depth, 64).items():
        b = oracle.raycast_batch(words, depth, o, d, 100, threads=3)
        for i in range(o.shape[0]):
            s, _ = oracle.raycast(words, depth, o[i], d[i], 100)
            assert np.array_equal(b[i], s), (name, i)


@pytest.fixture(scope="module")
def scenes(ve, oracle):
    r = ve.Renderer(hash_log2=16)
    out = []
    words, depth, *_ = helpers.small_setup()
    out.append((r.upload_scene(words, depth), depth))
    rng = np.random.default_rng(11)
    for depth, density in ((5, 0.2), (8, 0.002), (9, 0.0005), (10, 0.00005)):
        xyzm = helpers.random_voxels(rng, depth, density)
        out.append((r.build_scene(xyzm, depth), depth))
    yield r, [(sid, r.download_scene(sid), depth) for sid, depth in out]
    r.close()


@pytest.mark.gpu
@pytest.mark.parametrize("full_walk", [False, True])
def test_device_rays_match_oracle(ve, oracle, scenes, full_walk):
    r, sc = scenes
    rng = np.random.default_rng(3 + int(full_walk))
    for sid, words, depth in sc:
        sets = ray_sets(rng, depth, 20000)
        sets["shading"] = shading_rays(rng, words, depth, oracle, 4000)
        for name, (o, d) in sets.items():
            for cc in (300, 7):
                dev = r.raycast_batch(sid, o, d, cc, full_walk=full_walk)
                ref = oracle.raycast_batch(words, depth, o, d, cc)
                bad = np.nonzero((dev != ref).any(1))[0]
                assert bad.size == 0, (depth, name, cc, bad[:5].tolist(), o[bad[:1]].tolist(), d[bad[:1]].tolist(),
                                       dev[bad[:1]].tolist(), ref[bad[:1]].tolist())


@pytest.mark.gpu
def test_depth10_terrain_rays_match_oracle(ve, oracle):
    """The benchmark's depth-10 terrain (77.6M node words): rays from the
    orbit camera's eye, from inside the volume and from surface points."""
    import ve_b200.workloads as wl

    W = wl.LARGE
    words, _ = ve.terrain_words(W.depth, W.variant, W.seed)
    r = ve.Renderer(hash_log2=16)
    try:
        sid = r.upload_scene(words, W.depth)
        dev_words = r.download_scene(sid)
        rng = np.random.default_rng(21)
        eye, _ = wl.orbit_camera(0, W.frames, W.seed)
        n = 20000
        target = rng.uniform((0.0, 0.0, 0.0), (1024.0, 128.0, 1024.0), (n, 3))
        d = target - np.float64(eye)
        d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
        sets = {"eye": (np.repeat(np.float32(eye)[None], n, 0), d)}
        sets.update(ray_sets(rng, W.depth, n))
        sets["shading"] = shading_rays(rng, dev_words, W.depth, oracle, 4000)
        for name, (o, dd) in sets.items():
            for full in (False, True):
                dev = r.raycast_batch(sid, o, dd, W.bounce_controlchecks, full_walk=full)
                ref = oracle.raycast_batch(dev_words, W.depth, o, dd, W.bounce_controlchecks)
                bad = np.nonzero((dev != ref).any(1))[0]
                assert bad.size == 0, (name, full, bad[:5].tolist())
                if name == "eye":
                    assert (ref[:, 0] == 0).mean() > 0.3  # rays from the eye toward the terrain hit it
    finally:
        r.close()


@pytest.mark.gpu
def test_bounce_ray_of_scheduled_path(ve, oracle, scenes):
    """A secondary ray of the small scene that passes within an ulp of cell
    edges (its fetch count changes under one-ulp perturbations)."""
    r, sc = scenes
    sid, words, depth = sc[0]
    o = np.array([[6.93634224, 69.3726883, 113.280853]], np.float32)
    d = np.array([[0.244187325, 0.567281604, -0.786488473]], np.float32)
    for full in (False, True):
        assert np.array_equal(r.raycast_batch(sid, o, d, 100, full_walk=full), oracle.raycast_batch(words, depth, o, d, 100))
