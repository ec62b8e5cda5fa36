"""The reference's own normal mode (normal.comp:55-95, normalPrecision = R):
the device's leaf words and code table equal the oracle's at R = 1, 3 and 6
(the oracle's occupancy by tree descents, lookupOccupied), and frames
rendered with those normals equal the oracle's (GBuffer and every path's
deposit bitwise, resolved radiance within 1e-4)."""
import numpy as np
import pytest

import helpers
from oracle.oracle import OracleRenderer, frame_params

pytestmark = pytest.mark.gpu


def _ntab_from_words(words):
    idx = (words >> 8) & 0x7FFFFF
    leaf = ((words & 1) == 0) & (((words >> 1) & 0x7F) != 0)
    return idx[leaf]


@pytest.mark.parametrize("radius", [1, 3, 6])
def test_ball_normals_words_match_oracle(ve, oracle, radius):
    words, nv = helpers.terrain(6, 1, 1)
    with ve.Renderer(hash_log2=12) as r:
        sid = r.upload_scene(words, 6)
        grad = r.download_scene(sid)
        r.set_normal_mode(sid, radius)
        dev = r.download_scene(sid)
        want, codes = oracle.fill_normals_ball(words, 6, radius, threads=8)
        assert np.array_equal(dev, want)
        leaf_idx = _ntab_from_words(dev)
        assert leaf_idx.min() >= 1 and leaf_idx.max() == codes.size
        # back to the gradient mode: the upload's words again
        r.set_normal_mode(sid, 0)
        assert np.array_equal(r.download_scene(sid), grad)


def test_ball_normal_frames_match_oracle(ve, oracle):
    words, depth, mats, cam, fc = helpers.small_setup()
    with ve.Renderer(hash_log2=18) as r:
        r.set_materials(mats)
        sid = r.upload_scene(words, depth)
        r.set_normal_mode(sid, 6)
        dev_words = r.download_scene(sid)
        want, codes = oracle.fill_normals_ball(words, depth, 6, threads=8)
        assert np.array_equal(dev_words, want)
        orc = OracleRenderer(oracle)
        orc.set_normal_codes(codes)
        for f in range(3):
            c = ve.FrameConfig(**{**fc.__dict__, "width": 128, "height": 96, "spp": 2, "bounces": 3,
                                  "frame_index": f, "flags": ve.FRAME_PATH_RGB})
            g = r.render(sid, cam, c, outputs=("gbuffer", "rgb", "path_rgb"))
            o = orc.render(dev_words, depth, mats, cam, frame_params(c), threads=8, want_path_rgb=True)
            assert np.array_equal(g["gbuffer"], o["gbuffer"])
            hit = np.repeat(o["gbuffer"][..., 3].reshape(-1) != 0, c.spp)
            assert np.array_equal(g["path_rgb"][hit].view(np.uint32), o["path_rgb"][hit].view(np.uint32))
            x, y = g["rgb"].astype(np.float64), o["rgb"]
            assert (np.abs(x - y) <= 1e-4 * np.abs(y) + 1e-6).all()
        # the NORMAL view decodes the same table
        c = ve.FrameConfig(**{**fc.__dict__, "width": 64, "height": 48, "render_type": 3})
        g = r.render(sid, cam, c, outputs=("rgb",))
        o = orc.render(dev_words, depth, mats, cam, frame_params(c), threads=8)
        assert (np.abs(g["rgb"].astype(np.float64) - o["rgb"]) <= 1e-6).all()
        # targeted refresh is refused in the ball mode
        with pytest.raises(ve.VeError):
            r.refresh_scene(sid, np.array([[1, 2, 3]], np.uint32))
