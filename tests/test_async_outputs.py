"""VE_FRAME_ASYNC_OUTPUTS: a frame's images are copied to host memory on the
context's copy stream while the next frame renders (two device image sets,
alternating).  Frames rendered back to back into pinned host arrays equal the
same frames rendered synchronously on a second context: voxel ids exact,
radiance within 1e-4 relative (the two caches' float sums differ only in
atomic order)."""
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
    rs = []
    for _ in range(2):
        r = ve.Renderer(hash_log2=20)
        r.set_materials(mats)
        rs.append((r, r.upload_scene(words, depth)))
    yield rs, cam, fc
    for r, _ in rs:
        r.close()


def pinned(shape, dtype):
    import torch

    tdtype = {np.uint32: torch.int32, np.uint8: torch.uint8, np.float32: torch.float32}[dtype]
    t = torch.empty(shape, dtype=tdtype, pin_memory=True)
    return t, t.numpy().view(dtype)


def quantize(mapped):
    """The RGBA8 store of (mapped, 1): clamp, x 255, round to nearest (float32 steps)."""
    m = np.clip(np.asarray(mapped, np.float32), np.float32(0), np.float32(1))
    return (m * np.float32(255) + np.float32(0.5)).astype(np.uint32).astype(np.uint8)


def test_async_frames_equal_sync_frames(ve, pair):
    (ra, sa), (rb, sb) = pair[0]
    cam, fc = pair[1], pair[2]
    ra.cache_reset(sa)
    rb.cache_reset(sb)
    H, W = fc.height, fc.width
    keep, outs = [], []
    for f in range(6):
        tv, v = pinned((H, W), np.uint32)
        tr, rgb = pinned((H, W, 3), np.float32)
        tm, mp = pinned((H, W, 3), np.float32)
        t8, m8 = pinned((H, W, 4), np.uint8)
        keep += [tv, tr, tm, t8]
        outs.append({"voxel_id": v, "rgb": rgb, "mapped": mp, "mapped8": m8})
        ff = dataclasses.replace(fc, frame_index=f, flags=ve.FRAME_ASYNC_OUTPUTS)
        ra.render_into(sa, cam, ff, outs[-1])
    ra.synchronize()
    for f in range(6):
        ref = rb.render(sb, cam, dataclasses.replace(fc, frame_index=f), outputs=("voxel_id", "rgb", "mapped"))
        assert np.array_equal(outs[f]["voxel_id"], ref["voxel_id"]), f
        assert close_rel(outs[f]["rgb"], ref["rgb"]).all(), f
        assert close_rel(outs[f]["mapped"], ref["mapped"]).all(), f
        # the displayed image: the frame's own mapped radiance stored as RGBA8
        assert np.array_equal(outs[f]["mapped8"][..., :3], quantize(outs[f]["mapped"])), f
        assert (outs[f]["mapped8"][..., 3] == 255).all()
    assert outs[-1]["rgb"].max() > 0.05
    # a synchronous frame after asynchronous ones writes the first image set
    g = ra.render(sa, cam, dataclasses.replace(fc, frame_index=6), outputs=("voxel_id",))
    h = rb.render(sb, cam, dataclasses.replace(fc, frame_index=6), outputs=("voxel_id",))
    assert np.array_equal(g["voxel_id"], h["voxel_id"])


def test_async_outputs_reject_gbuffer(ve, pair):
    (ra, sa), _ = pair[0]
    cam, fc = pair[1], pair[2]
    ff = dataclasses.replace(fc, flags=ve.FRAME_ASYNC_OUTPUTS)
    with pytest.raises(ve.VeError):
        ra.render(sa, cam, ff, outputs=("gbuffer",))
    with pytest.raises(ve.VeError):
        ra.render(sa, cam, dataclasses.replace(ff, flags=ve.FRAME_ASYNC_OUTPUTS | ve.FRAME_SPLIT, row_end=4),
                  outputs=("rgb",))
