"""GPU parity: the CUDA pipeline (through the C ABI) against the CPU oracle.

Bars (per the plain method's contract):
  * GBuffer {checks, material, hit node, voxel id}: bit-exact;
  * every path's deposit value: bit-exact (same IEEE operation sequence);
  * per-voxel deposit counts in the radiance cache: exact;
  * cache sums and resolved radiance: within 1e-4 relative per pixel of the
    oracle's FP64 re-accumulation (absolute floor 1e-6).
"""
import numpy as np
import pytest

import helpers
from oracle.oracle import OracleRenderer, frame_params

pytestmark = pytest.mark.gpu

RTOL = 1e-4
ATOL = 1e-6


@pytest.fixture(scope="module")
def renderer(ve):
    r = ve.Renderer(hash_log2=20)
    yield r
    r.close()


@pytest.fixture(scope="module")
def small(ve, renderer):
    words, depth, mats, cam, fc = helpers.small_setup()
    renderer.set_materials(mats)
    sid = renderer.upload_scene(words, depth)
    return sid, words, depth, mats, cam, fc


def close_rel(a, b, rtol=RTOL, atol=ATOL):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b) <= rtol * np.abs(b) + atol


def test_device_normals_match_oracle(ve, renderer, oracle, small):
    sid, words, depth, *_ = small
    dev = renderer.download_scene(sid)
    ref = oracle.fill_normals(words, depth)
    assert np.array_equal(dev, ref)
    leaves = (ref & 1) == 0
    has_mat = ((ref >> 1) & 0x7F) != 0
    assert ((ref[leaves & has_mat] >> 31) == 1).all()


def run_both(ve, oracle, renderer, sid, words_dev, depth, mats, cam, fc, frames, orc=None, want=("gbuffer",)):
    orc = orc or OracleRenderer(oracle)
    outs = []
    for f in range(frames):
        fc.frame_index = f
        g = renderer.render(sid, cam, fc, outputs=want)
        st = renderer.stats()
        o = orc.render(words_dev, depth, mats, cam, frame_params(fc), threads=8,
                       want_path_rgb="path_rgb" in want)
        outs.append((g, st, o))
    return orc, outs


def test_single_frame_gbuffer_and_paths_exact(ve, renderer, oracle, small):
    sid, words, depth, mats, cam, fc = small
    renderer.cache_reset(sid)
    dev_words = renderer.download_scene(sid)
    fc = ve.FrameConfig(**{**fc.__dict__, "flags": ve.FRAME_PATH_RGB | ve.FRAME_COUNT_FETCH})
    _, outs = run_both(ve, oracle, renderer, sid, dev_words, depth, mats, cam, fc, 1,
                       want=("gbuffer", "path_rgb", "voxel_id", "hit_node"))
    g, st, o = outs[0]
    assert np.array_equal(g["gbuffer"], o["gbuffer"])
    assert np.array_equal(g["voxel_id"], o["gbuffer"][..., 3])
    assert np.array_equal(g["hit_node"], o["gbuffer"][..., 2])
    hit = o["gbuffer"][..., 3].reshape(-1) != 0
    assert hit.mean() > 0.3
    gp = g["path_rgb"].reshape(-1, 3)[hit]
    op = o["path_rgb"].reshape(-1, 3)[hit]
    assert np.array_equal(gp.view(np.uint32), op.view(np.uint32)), "per-path radiance differs bitwise"
    assert (op > 0).any()
    s = o["stats"]
    assert st["rays_primary"] == s["rays_primary"]
    assert st["rays_bounce"] == s["rays_bounce"]
    assert st["rays_shadow"] == s["rays_shadow"]
    assert st["shadow_shared"] == s["shadow_shared"]
    assert st["paths"] == s["paths"] == st["deposits"]
    assert st["deposits_dropped"] == 0
    # distinct-node fetches: the device descent reads each node of the walk once
    assert st["fetch_nodes"] == s["fetch_min"]
    assert st["dda_steps"] == s["steps"]


def test_shared_first_shadow_rays(ve, renderer, oracle, small):
    """A pixel's samples share their first sun shadow ray (same origin and
    direction): traced once, its result taken by every sample.  Per-path
    deposits stay bitwise equal, the walk is counted once on both sides."""
    sid, words, depth, mats, cam, fc = small
    renderer.cache_reset(sid)
    dev_words = renderer.download_scene(sid)
    fc = ve.FrameConfig(**{**fc.__dict__, "spp": 4, "bounces": 2,
                           "flags": ve.FRAME_PATH_RGB | ve.FRAME_COUNT_FETCH})
    _, outs = run_both(ve, oracle, renderer, sid, dev_words, depth, mats, cam, fc, 1,
                       want=("gbuffer", "path_rgb"))
    g, st, o = outs[0]
    assert np.array_equal(g["gbuffer"], o["gbuffer"])
    hit = np.repeat(o["gbuffer"][..., 3].reshape(-1) != 0, 4)
    assert np.array_equal(g["path_rgb"][hit].view(np.uint32), o["path_rgb"][hit].view(np.uint32))
    s = o["stats"]
    for k in ("rays_primary", "rays_bounce", "rays_shadow", "shadow_shared"):
        assert st[k] == s[k], k
    # three of every four first shadow rays of a lit pixel are shared
    assert s["shadow_shared"] > 0 and s["shadow_shared"] % 3 == 0
    assert st["fetch_nodes"] == s["fetch_min"]
    assert st["dda_steps"] == s["steps"]


def test_sixteen_frames_accumulation(ve, renderer, oracle, small):
    sid, words, depth, mats, cam, fc = small
    renderer.cache_reset(sid)
    dev_words = renderer.download_scene(sid)
    fc = ve.FrameConfig(**{**fc.__dict__})
    orc, outs = run_both(ve, oracle, renderer, sid, dev_words, depth, mats, cam, fc, 16,
                         want=("gbuffer", "rgb", "mapped", "mapped8"))
    for g, st, o in outs:
        assert np.array_equal(g["gbuffer"], o["gbuffer"])
    # cache: exact counts, FP32 sums vs FP64
    vids, counts, vals = renderer.cache_dump(sid)
    ovids, ocounts, ovals = orc.cache()
    assert np.array_equal(vids, ovids)
    assert np.array_equal(counts.astype(np.uint64), ocounts)
    assert close_rel(vals, ovals, rtol=2e-4).all()
    # resolved radiance per pixel
    g, st, o = outs[-1]
    ok = close_rel(g["rgb"], o["rgb"])
    frac_bad = 1.0 - ok.all(axis=-1).mean()
    assert frac_bad == 0.0, f"{frac_bad:.2e} of pixels beyond 1e-4 relative"
    assert close_rel(g["mapped"], o["mapped"]).all()
    # the displayed RGBA8 image: the device's mapped radiance stored exactly
    # (clamp, x 255, round to nearest), within one step of the oracle's
    m = np.clip(g["mapped"], np.float32(0), np.float32(1))
    assert np.array_equal(g["mapped8"][..., :3], (m * np.float32(255) + np.float32(0.5)).astype(np.uint8))
    assert (g["mapped8"][..., 3] == 255).all()
    om = np.floor(np.clip(o["mapped"], 0.0, 1.0) * 255.0 + 0.5)
    assert (np.abs(g["mapped8"][..., :3].astype(np.int32) - om.astype(np.int32)) <= 1).all()
    assert g["rgb"].max() > 0.05


@pytest.mark.parametrize("rtype", [1, 2, 3, 4, 5])
def test_render_types(ve, renderer, oracle, small, rtype):
    sid, words, depth, mats, cam, fc = small
    renderer.cache_reset(sid)
    dev_words = renderer.download_scene(sid)
    fc = ve.FrameConfig(**{**fc.__dict__, "render_type": rtype})
    _, outs = run_both(ve, oracle, renderer, sid, dev_words, depth, mats, cam, fc, 3, want=("gbuffer", "rgb"))
    g, st, o = outs[-1]
    assert np.array_equal(g["gbuffer"], o["gbuffer"])
    if rtype == 5:
        # VARIANCE view: E[L^2] - E[L]^2 cancels catastrophically, so the FP32
        # cache cannot hold 1e-4 relative against FP64; the display value
        # (in [0, 1]) is held to 1e-4 absolute instead.
        assert (np.abs(g["rgb"].astype(np.float64) - o["rgb"]) <= 1e-4).all()
    else:
        assert close_rel(g["rgb"], o["rgb"]).all()


def scene_from_voxels(ve, depth, voxels):
    c = ve.OctreeCPU(depth)
    c.insert_many(np.asarray(voxels, np.uint32).reshape(-1, 4))
    o = ve.Octree(depth)
    o.set(c)
    return o.words()[: o.size]


EDGE_CASES = {
    "single_voxel": (3, [(3, 4, 5, 2)], (4.5, 4.5, -10.0), (3.5, 4.5, 5.5)),
    "full_octant": (3, [(x, y, z, 1 + (x + y + z) % 8) for x in range(4) for y in range(4) for z in range(4)],
                    (12.0, 9.0, 13.0), (2.0, 2.0, 2.0)),
    # camera along +z, odd resolution: the centre row/column rays have exact
    # zero components (reciprocal +-inf in the slab tests)
    "axis_aligned": (4, [(x, y, 10 + (x * y) % 3, 3) for x in range(16) for y in range(16)], (8.0, 8.0, -6.0),
                     (8.0, 8.0, 10.0)),
    "inside_volume": (5, [(x, y, 0, 4) for x in range(32) for y in range(32)], (16.0, 16.0, 20.0),
                      (16.0, 16.0, 0.0)),
    "depth1": (1, [(0, 0, 0, 1), (1, 1, 1, 2)], (3.0, 3.0, -3.0), (1.0, 1.0, 1.0)),
    # a cube floating in an empty volume: most bounce rays leave the box of
    # the cells that can hold a voxel long before the volume's boundary
    "floating_cube": (6, [(x, y, z, 1 + (x + 2 * y + z) % 7) for x in range(28, 36) for y in range(27, 36)
                          for z in range(29, 36)], (20.0, 44.0, -14.0), (32.0, 31.0, 32.0)),
}


@pytest.mark.parametrize("case", sorted(EDGE_CASES))
@pytest.mark.parametrize("cc", [6, 70])
def test_edge_cases(ve, renderer, oracle, case, cc):
    depth, vox, eye, target = EDGE_CASES[case]
    words = scene_from_voxels(ve, depth, vox)
    mats = ve.terrain_materials(3)
    renderer.set_materials(mats)
    sid = renderer.upload_scene(words, depth)
    try:
        dev_words = renderer.download_scene(sid)
        assert np.array_equal(dev_words, oracle.fill_normals(words, depth))
        d = ve.look_at(eye, target)
        W, H = (41, 25) if case == "axis_aligned" else (40, 24)
        cam = ve.camera_ubo(np.asarray(eye, np.float32), d, 70.0, W / H)
        fc = ve.FrameConfig(width=W, height=H, spp=3, bounces=2, primary_controlchecks=cc,
                            bounce_controlchecks=cc, reconstruction_radius=3, flags=ve.FRAME_PATH_RGB)
        orc, outs = run_both(ve, oracle, renderer, sid, dev_words, depth, mats, cam, fc, 2,
                             want=("gbuffer", "rgb", "path_rgb"))
        for g, st, o in outs:
            assert np.array_equal(g["gbuffer"], o["gbuffer"])
            hit = o["gbuffer"][..., 3].reshape(-1) != 0
            hit = np.repeat(hit, fc.spp)
            assert np.array_equal(g["path_rgb"][hit].view(np.uint32), o["path_rgb"][hit].view(np.uint32))
            assert close_rel(g["rgb"], o["rgb"]).all()
        vids, counts, _ = renderer.cache_dump(sid)
        ovids, ocounts, _ = orc.cache()
        assert np.array_equal(vids, ovids) and np.array_equal(counts.astype(np.uint64), ocounts)
    finally:
        renderer.release_scene(sid)


def words_with_root_copies(depth, voxels):
    """Octree words whose root word (word 0, child block at word 8) is
    repeated in words 1..7.  A position with a coordinate equal to 2^D reads
    one of those at level 0, so the face {x = 2^D} holds the voxels of the
    plane x = 0, and likewise for y and z."""
    occ = {(int(x), int(y), int(z)): int(m) for x, y, z, m in voxels}
    words = [0] * 8

    def build(level, ox, oy, oz):
        size = 1 << (depth - level)
        if level == depth:
            return (occ.get((ox, oy, oz), 0) & 0x7F) << 1
        if not any(ox <= x < ox + size and oy <= y < oy + size and oz <= z < oz + size for x, y, z in occ):
            return 0
        block = len(words)
        words.extend([0] * 8)
        half = size >> 1
        for c in range(8):
            words[block + c] = build(level + 1, ox + ((c >> 2) & 1) * half, oy + ((c >> 1) & 1) * half,
                                     oz + (c & 1) * half)
        return (block << 4) | 1

    root = build(0, 0, 0, 0)
    words[0:8] = [root] * 8
    return np.asarray(words, np.uint32)


def test_clip_box(ve, renderer, oracle):
    """The box is the top-table cells holding voxels widened by one voxel, and
    no box applies when the faces at 2^D (read through root words 1..7) hold
    voxels."""
    cube = [(x, y, z, 2) for x in range(28, 36) for y in range(27, 36) for z in range(29, 35)]
    sid = renderer.upload_scene(scene_from_voxels(ve, 6, cube), 6)
    try:
        lo, hi, bounded = renderer.clip_box(sid)
        # depth 6: the table resolves all 6 levels above the leaves, cells of
        # 2 voxels (the cube spans x 28-35, y 27-35, z 29-34)
        assert bounded
        assert lo.tolist() == [27.0, 25.0, 27.0] and hi.tolist() == [37.0, 37.0, 37.0]
    finally:
        renderer.release_scene(sid)
    depth = 4
    inner = [(x, y, z, 1 + (x + y) % 5) for x in range(3, 9) for y in range(1, 7) for z in range(2, 12)]
    faces = inner + [(5, 0, 5, 3)]  # mirrored onto the face y = 16
    mats = ve.terrain_materials(3)
    renderer.set_materials(mats)
    for vox, want in ((inner, True), (faces, False)):
        words = words_with_root_copies(depth, vox)
        sid = renderer.upload_scene(words, depth)
        try:
            assert renderer.clip_box(sid)[2] == want
            dev_words = renderer.download_scene(sid)
            assert np.array_equal(dev_words, oracle.fill_normals(words, depth))
            eye = np.array([10.0, 9.0, 0.5], np.float32)
            cam = ve.camera_ubo(eye, ve.look_at(eye, (6.0, 3.0, 7.0)), 70.0, 40 / 24)
            fc = ve.FrameConfig(width=40, height=24, spp=4, bounces=3, primary_controlchecks=90,
                                bounce_controlchecks=90, flags=ve.FRAME_PATH_RGB)
            _, outs = run_both(ve, oracle, renderer, sid, dev_words, depth, mats, cam, fc, 1,
                               want=("gbuffer", "path_rgb"))
            g, st, ref = outs[0]
            assert np.array_equal(g["gbuffer"], ref["gbuffer"])
            hit = np.repeat(ref["gbuffer"][..., 3].reshape(-1) != 0, fc.spp)
            assert hit.mean() > 0.1
            assert np.array_equal(g["path_rgb"][hit].view(np.uint32), ref["path_rgb"][hit].view(np.uint32))
        finally:
            renderer.release_scene(sid)


def test_clip_box_follows_edits(ve, renderer, oracle):
    """Bounce rays end on leaving the box of the cells that can hold a voxel;
    edits that add voxels far outside it (a floor under a floating cube) must
    widen it, so paths then bounce off the floor exactly as in the oracle."""
    depth = 6
    cube = [(x, y, z, 1 + (x + y + z) % 7) for x in range(28, 36) for y in range(28, 36) for z in range(28, 36)]
    floor = [(x, 2, z, 3) for x in range(64) for z in range(64)]
    c = ve.OctreeCPU(depth)
    c.insert_many(np.asarray(cube + floor, np.uint32))
    o = ve.Octree(depth)
    o.set(c)
    for x, y, z, _ in floor:
        c.remove(x, y, z)
    o.apply_edits(c)
    mats = ve.terrain_materials(3)
    renderer.set_materials(mats)
    sid = renderer.upload_scene(o.words(), depth)
    eye = np.array([38.0, 40.0, 17.0], np.float32)
    cam = ve.camera_ubo(eye, ve.look_at(eye, (32.0, 30.0, 32.0)), 60.0, 48 / 32)
    fc = ve.FrameConfig(width=48, height=32, spp=4, bounces=3, primary_controlchecks=200,
                        bounce_controlchecks=200, flags=ve.FRAME_PATH_RGB)
    try:
        for step in range(2):
            if step == 1:
                for v in floor:
                    c.insert(*v)
                cap = o.capacity
                slots = o.apply_edits(c)
                assert o.capacity == cap  # the blocks freed above are reused: the edit path is taken
                renderer.apply_edits(sid, slots, o.words()[slots])
            lo, hi, bounded = renderer.clip_box(sid)
            # depth 6: cells of 2 voxels, widened by one voxel (the floor at
            # y = 2 lies in the cell of rows 2-3)
            assert bounded and lo[1] == (27.0 if step == 0 else 1.0) and hi[1] == 37.0
            renderer.cache_reset(sid)
            dev_words = renderer.download_scene(sid)
            assert np.array_equal(dev_words, oracle.fill_normals(o.words(), depth))
            _, outs = run_both(ve, oracle, renderer, sid, dev_words, depth, mats, cam, fc, 1,
                               want=("gbuffer", "path_rgb"))
            g, st, ref = outs[0]
            assert np.array_equal(g["gbuffer"], ref["gbuffer"])
            hit = np.repeat(ref["gbuffer"][..., 3].reshape(-1) != 0, fc.spp)
            assert hit.mean() > 0.1
            assert np.array_equal(g["path_rgb"][hit].view(np.uint32), ref["path_rgb"][hit].view(np.uint32))
            assert st["rays_bounce"] == ref["stats"]["rays_bounce"]
            assert st["rays_shadow"] == ref["stats"]["rays_shadow"]
    finally:
        renderer.release_scene(sid)


def test_batch_matches_single_views(ve, renderer, oracle, small):
    """Views of different sizes/spp/bounces over two scenes in one batch give
    the per-view results of separate renders."""
    sid, words, depth, mats, cam, fc = small
    words6, _ = helpers.terrain(6, 1, 4)
    sid6 = renderer.upload_scene(words6, 6)
    try:
        w = helpers.workloads()
        eye6 = np.array([32.0, 90.0, -20.0], np.float32)
        cam6 = ve.camera_ubo(eye6, ve.look_at(eye6, (32, 30, 32)), 60.0, 48 / 40)
        views = [(sid, cam, ve.FrameConfig(width=64, height=48, spp=2, bounces=1, flags=ve.FRAME_PATH_RGB)),
                 (sid6, cam6, ve.FrameConfig(width=48, height=40, spp=1, bounces=3, flags=ve.FRAME_PATH_RGB)),
                 (sid, cam, ve.FrameConfig(width=33, height=17, spp=3, bounces=2, frame_index=5,
                                           flags=ve.FRAME_PATH_RGB))]
        for s in (sid, sid6):
            renderer.cache_reset(s)
        batch = renderer.render_batch(views, outputs=("gbuffer", "path_rgb"))
        for (s, c, f), b in zip(views, batch):
            single = renderer.render(s, c, f, outputs=("gbuffer", "path_rgb"))
            assert np.array_equal(b["gbuffer"], single["gbuffer"])
            hit = np.repeat(single["gbuffer"][..., 3].reshape(-1) != 0, f.spp)
            assert hit.any() and not b["path_rgb"][~hit].any()
            assert np.array_equal(b["path_rgb"].view(np.uint32), single["path_rgb"].view(np.uint32))
    finally:
        renderer.release_scene(sid6)


def test_apply_edits_on_device(ve, renderer, oracle):
    depth = 5
    rng = np.random.default_rng(2)
    c = ve.OctreeCPU(depth)
    c.insert_many(helpers.random_voxels(rng, depth, 0.05))
    o = ve.Octree(depth)
    o.set(c)
    sid = renderer.upload_scene(o.words(), depth)
    try:
        for _ in range(3):
            for _ in range(40):
                x, y, z = (int(t) for t in rng.integers(0, 1 << depth, 3))
                if rng.random() < 0.6:
                    c.insert(x, y, z, int(rng.integers(1, 9)))
                else:
                    c.remove(x, y, z)
            old_cap = o.capacity
            slots = o.apply_edits(c)
            words = o.words()
            if o.capacity != old_cap:  # the array grew: re-upload, as glBufferData does
                renderer.release_scene(sid)
                sid = renderer.upload_scene(words, depth)
            else:
                renderer.apply_edits(sid, slots, words[slots])
            assert np.array_equal(renderer.download_scene(sid), oracle.fill_normals(words, depth))
    finally:
        renderer.release_scene(sid)


def test_large_frame_properties(ve, oracle):
    """Depth-10, 1920x1080, 4 spp x 3 bounces: sampled pixels against the
    oracle's single-ray DDA, and size-independent invariants."""
    w = helpers.workloads()
    L = w.LARGE
    words, nv = helpers.terrain(L.depth, L.variant, L.seed)
    mats = ve.terrain_materials(L.seed)
    eye, d = w.orbit_camera(0, L.frames, L.seed)
    cam = ve.camera_ubo(eye, d, L.fov, L.width / L.height)
    fc = ve.FrameConfig(width=L.width, height=L.height, spp=L.spp, bounces=L.bounces,
                        primary_controlchecks=L.primary_controlchecks, bounce_controlchecks=L.bounce_controlchecks,
                        flags=ve.FRAME_COUNT_FETCH)
    with ve.Renderer(hash_log2=L.hash_log2) as r:
        r.set_materials(mats)
        sid = r.upload_scene(words, L.depth)
        dev_words = r.download_scene(sid)
        out = r.render(sid, cam, fc, outputs=("gbuffer", "rgb"))
        st = r.stats()
        vids, counts, vals = r.cache_dump(sid)
    g = out["gbuffer"]
    hit = g[..., 3] != 0
    assert hit.mean() > 0.5
    assert np.array_equal(hit, g[..., 2] != 0)
    assert st["paths"] == int(hit.sum()) * L.spp
    assert st["deposits"] + st["deposits_dropped"] == st["paths"]
    assert st["deposits_dropped"] == 0
    assert int(counts.sum()) == st["deposits"]
    assert len(np.unique(g[..., 3][hit])) == len(vids)
    rng = np.random.default_rng(0)
    ys = rng.integers(0, L.height, 400)
    xs = rng.integers(0, L.width, 400)
    plane, right, up = cam[4:7], cam[8:11], cam[12:15]
    for x, y in zip(xs, ys):
        ndx = np.float32((np.float32(x) + np.float32(0.5)) / np.float32(L.width) * np.float32(2.0) - np.float32(1.0))
        ndy = np.float32((np.float32(y) + np.float32(0.5)) / np.float32(L.height) * np.float32(2.0) - np.float32(1.0))
        v = (plane + right * ndx) - up * ndy
        dd = (v / np.sqrt(np.float32((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]))).astype(np.float32)
        res, _ = oracle.raycast(dev_words, L.depth, cam[:3], dd, L.primary_controlchecks)
        assert g[y, x, 0] == res[7]
        if res[0] == 0:
            assert g[y, x, 2] == res[1] and g[y, x, 3] == oracle.voxel_key(res[3], res[4], res[5]) + 1
        else:
            assert g[y, x, 3] == 0


def test_graph_replay_matches_direct_launches(ve):
    """The frame's kernel sequence replayed from a captured CUDA graph gives
    the same results as direct launches (several frames, two batch shapes)."""
    words, depth, mats, cam, fc = helpers.small_setup()
    outs = []
    for graphs in (True, False):
        with ve.Renderer(hash_log2=18, graphs=graphs) as r:
            r.set_materials(mats)
            sid = r.upload_scene(words, depth)
            res = []
            for f in range(3):
                f1 = ve.FrameConfig(width=96, height=64, spp=2, bounces=2, frame_index=f, flags=ve.FRAME_PATH_RGB)
                res.append(r.render(sid, cam, f1, outputs=("gbuffer", "rgb", "path_rgb")))
                f2 = ve.FrameConfig(width=40, height=30, spp=1, bounces=1, frame_index=f)
                res.append(r.render_batch([(sid, cam, f2), (sid, cam, f1)], outputs=("gbuffer", "rgb"))[1])
            outs.append(res)
    for a, b in zip(*outs):
        for k in a:
            if k == "rgb":  # FP32 atomic accumulation order differs run to run
                assert close_rel(a[k], b[k], rtol=1e-5).all()
            else:
                assert np.array_equal(a[k].view(np.uint32), b[k].view(np.uint32)), k
