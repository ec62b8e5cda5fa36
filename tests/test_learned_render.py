"""Learned radiance cache in the frame: without evidence it changes nothing,
training frames record samples and train, the hashed per-voxel cache ends
paths once it holds enough deposits, and a trained network lowers the error
against a 64-spp plain render at equal samples per pixel."""
import dataclasses

import numpy as np
import pytest

import helpers

pytestmark = pytest.mark.gpu

DEPTH = 8


@pytest.fixture(scope="module")
def scene(ve):
    w = helpers.workloads()
    r = ve.Renderer(hash_log2=20)
    r.set_materials(ve.terrain_materials(1))
    words, _ = helpers.terrain(DEPTH, 1, 41)
    sid = r.upload_scene(words, DEPTH)
    eye, d = w.random_pose(np.random.default_rng(11), DEPTH)
    yield r, sid, eye, d
    r.close()


def fc_of(ve, W, H, spp, frame, flags=0, bounces=3):
    return ve.FrameConfig(width=W, height=H, spp=spp, bounces=bounces, frame_index=frame, decay=1.0,
                          primary_controlchecks=200, bounce_controlchecks=200, flags=flags)


def rmse(img, ref, mask):
    e = (img - ref) ** 2 / (ref ** 2 + 0.01)
    return float(e[mask].mean())


def test_without_evidence_the_frame_is_plain(ve, scene):
    r, sid, eye, d = scene
    cam = ve.camera_ubo(eye, d, 70.0, 1.0)
    with ve.LearnedCache(r, log2_table=16, seed=2) as m:
        m.attach(sid)
        r.cache_reset(sid)
        lf = r.render(sid, cam, fc_of(ve, 128, 128, 1, 3, ve.FRAME_LEARNED))
        st = r.stats()
        assert st["nrc_queries"] == 0 and st["nrc_hash_terminated"] == 0
        r.cache_reset(sid)
        pf = r.render(sid, cam, fc_of(ve, 128, 128, 1, 3))
        assert np.array_equal(lf["voxel_id"], pf["voxel_id"])
        assert np.allclose(lf["rgb"], pf["rgb"], rtol=1e-4, atol=1e-6)


def test_training_frames_record_samples_and_train(ve, scene):
    r, sid, eye, d = scene
    cam = ve.camera_ubo(eye, d, 70.0, 1.0)
    with ve.LearnedCache(r, log2_table=16, train_samples=8192, seed=3) as m:
        m.attach(sid)
        losses = []
        for f in range(24):
            r.render(sid, cam, fc_of(ve, 192, 192, 2, 100 + f, ve.FRAME_TRAIN), outputs=())
            st = r.stats()
            assert 0 < st["nrc_samples"] <= 8192
            ms = m.stats()
            assert np.isfinite(ms["loss"]) and 0 < ms["samples"] <= st["nrc_samples"]
            losses.append(ms["loss"])
        assert m.stats()["steps"] == 24
        assert np.mean(losses[-6:]) < np.mean(losses[:3])


def test_hash_cache_ends_paths_once_filled(ve, scene):
    r, sid, eye, d = scene
    cam = ve.camera_ubo(eye, d, 70.0, 1.0)
    r.cache_reset(sid)
    for f in range(12):
        r.render(sid, cam, fc_of(ve, 192, 192, 4, 200 + f), outputs=())
    r.render(sid, cam, fc_of(ve, 192, 192, 4, 300), outputs=())
    plain = r.stats()
    r.render(sid, cam, fc_of(ve, 192, 192, 4, 300, ve.FRAME_TERMINATE_HASH), outputs=())
    term = r.stats()
    assert term["nrc_hash_terminated"] > 0.02 * term["paths"]
    assert term["rays_bounce"] < plain["rays_bounce"]
    assert term["rays_primary"] == plain["rays_primary"]


def test_trained_network_lowers_error_against_64spp(ve, scene):
    """At equal samples per pixel the learned cache replaces each path's
    random continuation past its second vertex by the network's estimate:
    the per-pixel variance across independent frames drops, and the error
    against a 64-spp plain render does not grow."""
    r, sid, eye, d = scene
    W = H = 192
    cam = ve.camera_ubo(eye, d, 70.0, 1.0)
    r.cache_reset(sid)
    ref = r.render(sid, cam, fc_of(ve, W, H, 64, 5000))
    mask = ref["voxel_id"] != 0
    with ve.LearnedCache(r, log2_table=18, train_samples=16384, seed=4) as m:
        m.attach(sid)
        for f in range(60):
            r.render(sid, cam, fc_of(ve, W, H, 4, 6000 + f, ve.FRAME_TRAIN), outputs=())
        imgs = {}
        for name, flags in (("plain", 0), ("learned", ve.FRAME_LEARNED)):
            imgs[name] = []
            for k in range(6):
                r.cache_reset(sid)
                imgs[name].append(r.render(sid, cam, fc_of(ve, W, H, 1, 7000 + k, flags))["rgb"])
                if flags:
                    assert r.stats()["nrc_queries"] > 0
        var = {k: float(np.stack(v).var(axis=0)[mask].mean()) for k, v in imgs.items()}
        err = {k: float(np.mean([rmse(i, ref["rgb"], mask) for i in v])) for k, v in imgs.items()}
        print("1 spp: per-pixel variance", var, "rMSE vs 64 spp", err)
        assert var["learned"] < 0.9 * var["plain"], var
        assert err["learned"] < 1.05 * err["plain"], err
