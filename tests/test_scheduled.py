"""Importance-aware voxel scheduling (VE_FRAME_SCHEDULED).

The reference's schedule/rank/threshold/emit compute passes
(src/renderer/shaders/schedule.comp, rank.comp, threshold.comp, emit.comp)
are GLSL and cannot run here; the oracle restates them (oracle/ve_oracle.cpp
schedule_frame) and is itself checked below against an independent numpy
restatement of the tier and threshold rules.  The device path is then held
to the oracle: bit-exact GBuffer, shade list (through the per-path deposit
values, which the list index seeds) and counters; exact cache counts;
radiance within 1e-4 relative.  Frames whose importance reads the cache's
variance compare the voxel count exactly and the path count within a small
tolerance: the device's FP32 cache and the oracle's FP64 one can put a voxel
on either side of a threshold bin.
"""
import numpy as np
import pytest

import helpers
from oracle.oracle import OracleRenderer, frame_params

RTOL = 1e-4
ATOL = 1e-6
BINS = 256


def sched_config(ve, fc, **kw):
    d = {**fc.__dict__, "flags": ve.FRAME_SCHEDULED}
    d.update(kw)
    return ve.FrameConfig(**d)


def numpy_schedule(vids, t_high, t_mid, fc):
    """Counts of the scheduling rules on a voxel-id image with variance
    weight 0: (voxels, paths, next t_high, next t_mid)."""
    v = vids.reshape(-1)
    v = v[v != 0]
    uniq, cnt = np.unique(v, return_counts=True)
    pn = np.clip(cnt.astype(np.float32) / np.float32(max(fc.pixels_norm, 1.0)), 0, 1).astype(np.float32)
    imp = (np.float32(fc.weight_pixels) * pn).astype(np.float32)
    n = np.where(imp >= t_high, 2, np.where(imp >= t_mid, 1, fc.min_samples))
    paths = min(int(n.sum()), fc.shading_budget, 2 * vids.size)
    bins = np.minimum((imp * np.float32(BINS)).astype(np.int64), BINS - 1)
    hist = np.bincount(bins, minlength=BINS)
    total = hist.sum()
    top = np.float32(min(max(fc.top_fraction, 0.0), 1.0))
    mid = np.float32(min(max(fc.mid_fraction, 0.0), 1.0 - top))
    top_n = int(top * np.float32(total))
    topmid_n = int(np.float32(top + mid) * np.float32(total))
    cum = np.cumsum(hist[::-1])
    hb = BINS - 1 - int(np.argmax(cum >= top_n)) if (cum >= top_n).any() else BINS - 1
    mb = BINS - 1 - int(np.argmax(cum >= topmid_n)) if (cum >= topmid_n).any() else BINS - 1
    return len(uniq), paths, np.float32(hb / BINS), np.float32(mb / BINS)


# ---------------------------------------------------------------------------
# CPU: the oracle's scheduling against the numpy restatement
# ---------------------------------------------------------------------------
def test_oracle_schedule_counts_and_thresholds(ve, oracle):
    words, depth, mats, cam, fc = helpers.small_setup()
    words = oracle.fill_normals(words, depth)
    fc = sched_config(ve, fc, weight_variance=0.0, pixels_norm=8.0)
    orc = OracleRenderer(oracle)
    t_high, t_mid = np.float32(np.inf), np.float32(-np.inf)
    prev = None
    for f in range(3):
        fc.frame_index = f
        o = orc.render(words, depth, mats, cam, frame_params(fc), threads=8)
        vids = o["gbuffer"][..., 3]
        nvox, npaths, t_high, t_mid = numpy_schedule(vids, t_high, t_mid, fc)
        st = o["stats"]
        assert st["scheduled_voxels"] == nvox > 100
        assert st["scheduled_paths"] == npaths == st["paths"]
        if f == 0:
            assert npaths == nvox  # first frame: every voxel in the middle tier
        else:
            assert npaths != nvox  # tiers from the previous frame's histogram
        prev = st
    assert prev is not None


def test_oracle_schedule_budget(ve, oracle):
    words, depth, mats, cam, fc = helpers.small_setup()
    words = oracle.fill_normals(words, depth)
    fc = sched_config(ve, fc, shading_budget=257)
    o = OracleRenderer(oracle).render(words, depth, mats, cam, frame_params(fc), threads=4, want_path_rgb=True)
    assert o["stats"]["scheduled_paths"] == 257 == o["stats"]["paths"]
    assert o["path_rgb"].shape == (257, 3)
    assert (o["path_rgb"] > 0).any()


def test_oracle_budget_cut_rotates(ve, oracle):
    """Over budget, the list starts at a per-frame rotation of the pixel
    order, so the voxels left out change from frame to frame."""
    words, depth, mats, cam, fc = helpers.small_setup()
    words = oracle.fill_normals(words, depth)
    fc = sched_config(ve, fc, shading_budget=1000)
    orc = OracleRenderer(oracle)
    for f in range(6):
        fc.frame_index = f
        o = orc.render(words, depth, mats, cam, frame_params(fc), threads=4)
        assert o["stats"]["scheduled_paths"] == 1000
    vids, counts, _ = orc.cache()
    assert vids.size > 2000  # without the rotation the same <= 1000 voxels would be shaded every frame


def test_oracle_schedule_thread_invariant(ve, oracle):
    words, depth, mats, cam, fc = helpers.small_setup()
    words = oracle.fill_normals(words, depth)
    fc = sched_config(ve, fc)
    a = OracleRenderer(oracle).render(words, depth, mats, cam, frame_params(fc), threads=1, want_path_rgb=True)
    b = OracleRenderer(oracle).render(words, depth, mats, cam, frame_params(fc), threads=7, want_path_rgb=True)
    assert np.array_equal(a["path_rgb"].view(np.uint32), b["path_rgb"].view(np.uint32))
    assert a["stats"] == b["stats"]


# ---------------------------------------------------------------------------
# GPU: the device path against the oracle
# ---------------------------------------------------------------------------
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
    return sid, renderer.download_scene(sid), depth, mats, cam, fc


def close_rel(a, b, rtol=RTOL, atol=ATOL):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b) <= rtol * np.abs(b) + atol


def frame_pair(renderer, orc, sid, words, depth, mats, cam, fc, want=("gbuffer", "path_rgb")):
    g = renderer.render(sid, cam, fc, outputs=want)
    st = renderer.stats()
    o = orc.render(words, depth, mats, cam, frame_params(fc), threads=8, want_path_rgb="path_rgb" in want)
    return g, st, o


def assert_frame_exact(g, st, o):
    assert np.array_equal(g["gbuffer"], o["gbuffer"])
    s = o["stats"]
    for k_dev, k_or in (("scheduled_voxels", "scheduled_voxels"), ("scheduled_paths", "scheduled_paths"),
                        ("paths", "paths"), ("rays_primary", "rays_primary"), ("rays_bounce", "rays_bounce"),
                        ("rays_shadow", "rays_shadow")):
        assert st[k_dev] == s[k_or], k_dev
    assert st["deposits"] == st["paths"]
    assert st["deposits_dropped"] == 0
    n = s["scheduled_paths"]
    if "path_rgb" in g:
        gp = g["path_rgb"][:n]
        op = o["path_rgb"][:n]
        assert np.array_equal(gp.view(np.uint32), op.view(np.uint32)), "per-path radiance differs bitwise"
        assert not g["path_rgb"][n:].any()


@pytest.mark.gpu
def test_first_frame_exact(ve, oracle, renderer, small):
    sid, words, depth, mats, cam, fc = small
    renderer.cache_reset(sid)
    fc = sched_config(ve, fc, flags=ve.FRAME_SCHEDULED | ve.FRAME_PATH_RGB)
    g, st, o = frame_pair(renderer, OracleRenderer(oracle), sid, words, depth, mats, cam, fc)
    assert_frame_exact(g, st, o)
    assert st["scheduled_paths"] == st["scheduled_voxels"] > 100
    vids, counts, _ = renderer.cache_dump(sid)
    assert set(vids.tolist()) == set(np.unique(o["gbuffer"][..., 3][o["gbuffer"][..., 3] != 0]).tolist())
    assert (counts == 1).all()


@pytest.mark.gpu
def test_tiers_follow_previous_thresholds(ve, oracle, renderer, small):
    """Variance weight 0: the tiers depend on pixel coverage and the carried
    thresholds only, so every frame is exact."""
    sid, words, depth, mats, cam, fc = small
    renderer.cache_reset(sid)
    fc = sched_config(ve, fc, flags=ve.FRAME_SCHEDULED | ve.FRAME_PATH_RGB, weight_variance=0.0, pixels_norm=8.0)
    orc = OracleRenderer(oracle)
    for f in range(4):
        fc.frame_index = f
        g, st, o = frame_pair(renderer, orc, sid, words, depth, mats, cam, fc,
                              want=("gbuffer", "path_rgb", "rgb", "mapped"))
        assert_frame_exact(g, st, o)
        if f > 0:
            assert st["scheduled_paths"] != st["scheduled_voxels"]
    vids, counts, vals = renderer.cache_dump(sid)
    ovids, ocounts, ovals = orc.cache()
    assert np.array_equal(vids, ovids)
    assert np.array_equal(counts.astype(np.uint64), ocounts)
    assert close_rel(vals, ovals, rtol=2e-4).all()
    assert close_rel(g["rgb"], o["rgb"]).all()
    assert close_rel(g["mapped"], o["mapped"]).all()


@pytest.mark.gpu
def test_variance_weighted_frames(ve, oracle, renderer, small):
    sid, words, depth, mats, cam, fc = small
    renderer.cache_reset(sid)
    fc = sched_config(ve, fc, variance_norm=50.0)
    orc = OracleRenderer(oracle)
    n2 = 0
    for f in range(4):
        fc.frame_index = f
        g, st, o = frame_pair(renderer, orc, sid, words, depth, mats, cam, fc, want=("gbuffer",))
        assert np.array_equal(g["gbuffer"], o["gbuffer"])
        s = o["stats"]
        assert st["scheduled_voxels"] == s["scheduled_voxels"]
        assert abs(st["scheduled_paths"] - s["scheduled_paths"]) <= max(2, 0.01 * s["scheduled_paths"])
        n2 += st["scheduled_paths"] - st["scheduled_voxels"]
    assert n2 != 0  # the variance moved voxels between tiers


@pytest.mark.gpu
def test_shading_budget(ve, oracle, renderer, small):
    sid, words, depth, mats, cam, fc = small
    renderer.cache_reset(sid)
    fc = sched_config(ve, fc, flags=ve.FRAME_SCHEDULED | ve.FRAME_PATH_RGB, shading_budget=1000)
    orc = OracleRenderer(oracle)
    for f in (0, 5, 6):  # rotation 0 and two others
        fc.frame_index = f
        g, st, o = frame_pair(renderer, orc, sid, words, depth, mats, cam, fc)
        assert_frame_exact(g, st, o)
        assert st["scheduled_paths"] == 1000 == st["paths"]
        assert g["path_rgb"].shape == (1000, 3)
    vids, counts, _ = renderer.cache_dump(sid)
    ovids, ocounts, _ = orc.cache()
    assert np.array_equal(vids, ovids)
    assert np.array_equal(counts.astype(np.uint64), ocounts)


@pytest.mark.gpu
def test_graph_replay_matches(ve, oracle, small):
    """The scheduled frame replays from a CUDA graph with the same results as
    the eager launch sequence."""
    sid0, words, depth, mats, cam, fc = small
    fc = sched_config(ve, fc, flags=ve.FRAME_SCHEDULED | ve.FRAME_PATH_RGB, weight_variance=0.0, pixels_norm=8.0)
    res = []
    for graphs in (True, False):
        with ve.Renderer(hash_log2=20, graphs=graphs) as r:
            r.set_materials(mats)
            sid = r.upload_scene(words, depth, keep_normals=True)
            out = []
            for f in range(3):
                fc.frame_index = f
                out.append(r.render(sid, cam, fc, outputs=("path_rgb",))["path_rgb"].copy())
            res.append(out)
    for a, b in zip(*res):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.gpu
def test_rejects_unsupported(ve, renderer, small):
    sid, words, depth, mats, cam, fc = small
    fc2 = sched_config(ve, fc)
    with pytest.raises(ve.VeError):
        renderer.render_batch([(sid, cam, fc2), (sid, cam, fc2)])
    with pytest.raises(ve.VeError):
        renderer.render(sid, cam, sched_config(ve, fc, flags=ve.FRAME_SCHEDULED | ve.FRAME_LEARNED))
    # the context stays usable
    renderer.render(sid, cam, fc2, outputs=("voxel_id",))
