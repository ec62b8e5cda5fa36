"""The launch autotuner (ve_autotune): it returns a legal launch shape, leaves
it in the context, and frames rendered under the tuned shape equal frames
rendered before tuning (GBuffer and every path's deposit bitwise; resolved
radiance within the FP32 atomic-order tolerance)."""
import numpy as np
import pytest

import helpers

pytestmark = pytest.mark.gpu


def _frames(r, views):
    out = []
    for sid, cam, fc in views:
        r.cache_reset(sid)
    for sid, cam, fc in views:
        out.append(r.render(sid, cam, fc, outputs=("gbuffer", "path_rgb", "rgb")))
    return out


def test_autotune_legal_and_result_preserving(ve):
    words, depth, mats, cam, _ = helpers.small_setup()
    words6, _ = helpers.terrain(6, 1, 4)
    eye6 = np.array([32.0, 90.0, -20.0], np.float32)
    cam6 = ve.camera_ubo(eye6, ve.look_at(eye6, (32, 30, 32)), 60.0, 96 / 64)
    with ve.Renderer(hash_log2=18) as r:
        r.set_materials(mats)
        sid = r.upload_scene(words, depth)
        sid6 = r.upload_scene(words6, 6)
        views = [(sid, cam, ve.FrameConfig(width=128, height=96, spp=2, bounces=3, frame_index=3,
                                           flags=ve.FRAME_PATH_RGB)),
                 (sid6, cam6, ve.FrameConfig(width=96, height=64, spp=1, bounces=2, frame_index=7,
                                             flags=ve.FRAME_PATH_RGB))]
        default = r.launch_config()
        before = _frames(r, views)
        best = r.autotune(views, frames_per_trial=1)
        assert 1 <= best["trace_blocks_per_sm"] <= 32
        assert 1 <= best["shade_blocks_per_sm"] <= 32
        assert 1 <= best["refill_threshold"] <= 32
        assert r.launch_config() == best
        after = _frames(r, views)
        # a shape set by hand is honoured and results still agree
        r.set_launch_config(1, 1, 4)
        assert r.launch_config()["trace_blocks_per_sm"] == 1 and r.launch_config()["refill_threshold"] == 4
        forced = _frames(r, views)
        r.set_launch_config(default["trace_blocks_per_sm"], default["shade_blocks_per_sm"],
                            default["refill_threshold"] or 12)
    for b, a, f, (s, c, fc) in zip(before, after, forced, views):
        hit = np.repeat(b["gbuffer"][..., 3].reshape(-1) != 0, fc.spp)
        assert hit.any()
        for other in (a, f):
            assert np.array_equal(other["gbuffer"], b["gbuffer"])
            assert np.array_equal(other["path_rgb"][hit].view(np.uint32), b["path_rgb"][hit].view(np.uint32))
            x, y = other["rgb"].astype(np.float64), b["rgb"].astype(np.float64)
            assert (np.abs(x - y) <= 1e-5 * np.abs(y) + 1e-6).all()
