"""VE_CFG_PIPELINE: consecutive plain frames alternate between two sets of
frame buffers on two streams; a frame's primary pass and first trace pass run
while the previous frame finishes, its radiance-cache work after the previous
frame's.  A pipelined renderer must give the frames, counters and radiance
cache of an unpipelined one: voxel ids and deposit counts exact, radiance
within 1e-4 relative (float cache sums differ only in atomic order), also
when other calls (cache reset, edits) and unpipelined frames come between
pipelined ones."""
import dataclasses

import numpy as np
import pytest

import helpers

pytestmark = pytest.mark.gpu


def close_rel(a, b, rtol=1e-4, atol=1e-6):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b) <= rtol * np.abs(b) + atol


@pytest.fixture(scope="module")
def pair(ve):
    words, depth, mats, cam, fc = helpers.small_setup()
    fc = dataclasses.replace(fc, bounces=max(fc.bounces, 2))
    out = []
    for pipe in (True, False):
        r = ve.Renderer(hash_log2=20, pipeline=pipe)
        r.set_materials(mats)
        out.append((r, r.upload_scene(words, depth)))
    yield out, cam, fc, words, depth
    for r, _ in out:
        r.close()


def orbit(ve, cam, k):
    """A slightly different camera per frame (the frames differ)."""
    c = np.array(cam, np.float32).copy()
    c[0] += 0.25 * k
    c[2] -= 0.15 * k
    return c


def compare_caches(rp, sp, rq, sq):
    v0, c0, x0 = rp.cache_dump(sp)
    v1, c1, x1 = rq.cache_dump(sq)
    assert np.array_equal(v0, v1)
    assert np.array_equal(c0, c1)
    assert close_rel(x0, x1, rtol=2e-4).all()


def test_pipelined_frames_equal_plain_frames(ve, pair):
    (rp, sp), (rq, sq) = pair[0]
    cam, fc = pair[1], pair[2]
    rp.cache_reset(sp)
    rq.cache_reset(sq)
    for f in range(8):
        ff = dataclasses.replace(fc, frame_index=f)
        a = rp.render(sp, orbit(ve, cam, f), ff, outputs=("voxel_id", "rgb"))
        b = rq.render(sq, orbit(ve, cam, f), ff, outputs=("voxel_id", "rgb"))
        assert np.array_equal(a["voxel_id"], b["voxel_id"]), f
        assert close_rel(a["rgb"], b["rgb"]).all(), f
        sa, sb = rp.stats(), rq.stats()
        for k in ("rays_primary", "rays_bounce", "rays_shadow", "paths", "deposits"):
            assert sa[k] == sb[k], (f, k)
    compare_caches(rp, sp, rq, sq)


def test_pipelined_frames_back_to_back(ve, pair):
    """Frames enqueued without waiting (no host outputs), then compared
    through the accumulated cache and the totals."""
    (rp, sp), (rq, sq) = pair[0]
    cam, fc = pair[1], pair[2]
    for r, s in ((rp, sp), (rq, sq)):
        r.cache_reset(s)
        r.reset_total_stats()
        for f in range(12):
            r.render(s, orbit(ve, cam, f), dataclasses.replace(fc, frame_index=f), outputs=())
        r.synchronize()
    ta, tb = rp.total_stats(), rq.total_stats()
    for k in ("rays_primary", "rays_bounce", "rays_shadow", "paths", "deposits"):
        assert ta[k] == tb[k], k
    compare_caches(rp, sp, rq, sq)
    # the last frame's image, rendered again after the sequence
    ff = dataclasses.replace(fc, frame_index=12)
    a = rp.render(sp, orbit(ve, cam, 12), ff, outputs=("voxel_id", "rgb"))
    b = rq.render(sq, orbit(ve, cam, 12), ff, outputs=("voxel_id", "rgb"))
    assert np.array_equal(a["voxel_id"], b["voxel_id"])
    assert close_rel(a["rgb"], b["rgb"]).all()


def test_calls_between_pipelined_frames(ve, pair):
    """A cache reset, unpipelined frames (fetch counting) and a scene edit
    between pipelined frames take effect in call order."""
    (rp, sp), (rq, sq) = pair[0]
    cam, fc, words, depth = pair[1], pair[2], pair[3], pair[4]
    dev = rp.download_scene(sp)
    # an edit that changes a voxel's material in both renderers
    leaf = int(np.nonzero(((dev & 1) == 0) & (((dev >> 1) & 0x7F) != 0))[0][5])
    new_word = np.array([(int(dev[leaf]) & ~0xFE) | (7 << 1)], np.uint32)
    for r, s in ((rp, sp), (rq, sq)):
        r.cache_reset(s)
        for f in range(5):
            r.render(s, orbit(ve, cam, f), dataclasses.replace(fc, frame_index=f), outputs=())
            if f == 1:
                r.cache_reset(s)
            if f == 2:
                r.render(s, orbit(ve, cam, f), dataclasses.replace(fc, frame_index=100, flags=ve.FRAME_COUNT_FETCH),
                         outputs=())
            if f == 3:
                r.apply_edits(s, np.array([leaf], np.uint32), new_word, keep_normals=True)
        r.synchronize()
    compare_caches(rp, sp, rq, sq)
    assert np.array_equal(rp.download_scene(sp), rq.download_scene(sq))
    # restore the scene for later tests
    for r, s in ((rp, sp), (rq, sq)):
        r.apply_edits(s, np.array([leaf], np.uint32), dev[leaf:leaf + 1], keep_normals=True)


def test_async_outputs_pipelined(ve, pair):
    """Displayed images copied while later frames render, with pipelining."""
    import torch

    (rp, sp), (rq, sq) = pair[0]
    cam, fc = pair[1], pair[2]
    rp.cache_reset(sp)
    rq.cache_reset(sq)
    H, W = fc.height, fc.width
    keep, outs = [], []
    for f in range(6):
        t8 = torch.empty((H, W, 4), dtype=torch.uint8, pin_memory=True)
        tv = torch.empty((H, W), dtype=torch.int32, pin_memory=True)
        keep += [t8, tv]
        outs.append({"mapped8": t8.numpy(), "voxel_id": tv.numpy().view(np.uint32)})
        rp.render_into(sp, orbit(ve, cam, f), dataclasses.replace(fc, frame_index=f, flags=ve.FRAME_ASYNC_OUTPUTS),
                       outs[-1])
    rp.synchronize()
    for f in range(6):
        ref = rq.render(sq, orbit(ve, cam, f), dataclasses.replace(fc, frame_index=f),
                        outputs=("voxel_id", "mapped8"))
        assert np.array_equal(outs[f]["voxel_id"], ref["voxel_id"]), f
        assert (np.abs(outs[f]["mapped8"].astype(np.int32) - ref["mapped8"].astype(np.int32)) <= 1).all(), f
