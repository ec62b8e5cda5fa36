"""Render server (continuous batching): each request's result is the same
alone and in a mix, late arrivals join while others are on the GPU, and
admission respects the pooled device memory."""
import dataclasses
import time

import numpy as np
import pytest

import helpers

pytestmark = pytest.mark.gpu


def close_rel(a, b, rtol=1e-4, atol=1e-6):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b) <= rtol * np.abs(b) + atol


@pytest.fixture(scope="module")
def world(ve):
    w = helpers.workloads()
    r = ve.Renderer(hash_log2=18)
    r.set_materials(ve.terrain_materials(1))
    scenes = []
    for i, (depth, variant, seed) in enumerate([(6, 1, 21), (7, 0, 22), (7, 1, 23), (6, 0, 24)]):
        words, _ = helpers.terrain(depth, variant, seed)
        scenes.append((r.upload_scene(words, depth), depth))
    rng = np.random.default_rng(3)
    reqs = []
    for i in range(8):
        sid, depth = scenes[i % 4]
        eye, d = w.random_pose(rng, depth)
        W, H = [(40, 32), (64, 48), (96, 64), (33, 17)][i % 4]
        cam = ve.camera_ubo(eye, d, 70.0, W / H)
        fc = ve.FrameConfig(width=W, height=H, spp=1 + i % 4, bounces=1 + i % 3, frame_index=i,
                            primary_controlchecks=200, bounce_controlchecks=200)
        reqs.append((sid, cam, fc))
    yield r, scenes, reqs
    r.close()


def reset(r, scenes):
    for sid, _ in scenes:
        r.cache_reset(sid)


def test_requests_alone_equal_requests_in_the_mix(ve, world):
    r, scenes, reqs = world
    distinct = reqs[:4]  # one request per scene: no shared radiance cache
    alone = []
    for sid, cam, fc in distinct:
        reset(r, scenes)
        with ve.Server(r, pixel_capacity=1 << 16, path_capacity=1 << 18, max_requests=8) as srv:
            alone.append(srv.wait(srv.submit(sid, cam, fc)))
    reset(r, scenes)
    with ve.Server(r, pixel_capacity=1 << 16, path_capacity=1 << 18, max_requests=8) as srv:
        ids = [srv.submit(*q) for q in distinct]
        mixed = [srv.wait(i) for i in ids]
    for a, b in zip(alone, mixed):
        assert np.array_equal(a["voxel_id"], b["voxel_id"])
        assert close_rel(a["rgb"], b["rgb"]).all()
        assert (a["voxel_id"] != 0).any()
    # and against the plain renderer (same frame, fresh caches)
    for (sid, cam, fc), a in zip(distinct, alone):
        reset(r, scenes)
        fc1 = dataclasses.replace(fc, decay=1.0)
        p = r.render(sid, cam, fc1, outputs=("voxel_id", "rgb"))
        assert np.array_equal(p["voxel_id"], a["voxel_id"])
        assert close_rel(p["rgb"], a["rgb"]).all()


def test_voxel_ids_equal_with_shared_scenes(ve, world):
    r, scenes, reqs = world
    with ve.Server(r, pixel_capacity=1 << 16, path_capacity=1 << 18, max_requests=8) as srv:
        ids = [srv.submit(*q) for q in reqs]
        mixed = [srv.wait(i) for i in ids]
    for q, m in zip(reqs, mixed):
        p = r.render(*q, outputs=("voxel_id",))
        assert np.array_equal(p["voxel_id"], m["voxel_id"])


def test_late_arrivals_overlap_with_requests_on_the_gpu(ve, world):
    r, scenes, reqs = world
    sid, depth = scenes[1]
    w = helpers.workloads()
    eye, d = w.random_pose(np.random.default_rng(9), depth)
    big = (sid, ve.camera_ubo(eye, d, 70.0, 1.0), ve.FrameConfig(width=1024, height=1024, spp=8, bounces=4,
                                                                   primary_controlchecks=200,
                                                                   bounce_controlchecks=200))
    with ve.Server(r, pixel_capacity=1 << 21, path_capacity=1 << 24, max_requests=16) as srv:
        b = srv.submit(*big)
        t_end = time.monotonic() + 10.0
        while srv.stats()["steps"] < 1 and time.monotonic() < t_end:  # the big request is on the GPU
            time.sleep(1e-4)
        small = [srv.submit(*q) for q in reqs[:4]]
        rs = [srv.wait(i) for i in small]
        rb = srv.wait(b)
        st = srv.stats()
    # the small requests arrived after the big one was admitted and joined it
    # on the GPU before it finished
    assert all(x["submit_s"] > rb["admit_s"] for x in rs)
    assert all(x["admit_s"] < rb["done_s"] for x in rs), ([x["admit_s"] for x in rs], rb)
    assert st["max_in_flight"] >= 2
    assert st["completed"] == 5


def test_admission_waits_for_pool_space(ve, world):
    r, scenes, reqs = world
    sid, cam, fc = reqs[2]  # 96 x 64 pixels
    with ve.Server(r, pixel_capacity=96 * 64 * 2, path_capacity=96 * 64 * 8, max_requests=8) as srv:
        ids = [srv.submit(sid, cam, fc) for _ in range(6)]
        out = [srv.wait(i) for i in ids]
        st = srv.stats()
        assert st["max_in_flight"] <= 2
        with pytest.raises(ve.VeError) as e:
            srv.submit(sid, cam, ve.FrameConfig(width=512, height=512))
        assert e.value.code == ve.VE_ERR_CAPACITY
    for o in out[1:]:
        assert np.array_equal(o["voxel_id"], out[0]["voxel_id"])


def test_step_budget_spreads_large_requests_without_changing_results(ve, world):
    """A request whose primary tiles are started a few per step (a tiny
    per-step path budget) gives the results of the whole-request primary pass."""
    r, scenes, reqs = world
    sid, cam, fc = reqs[2]  # 96 x 64, 24 tiles
    outs = []
    for kw in ({"fifo": True}, {"step_path_budget": 256 * fc.spp}, {"step_path_budget": 3 * 256 * fc.spp}):
        reset(r, scenes)
        with ve.Server(r, pixel_capacity=1 << 16, path_capacity=1 << 18, max_requests=8, **kw) as srv:
            outs.append(srv.wait(srv.submit(sid, cam, fc)))
            st = srv.stats()
        if "step_path_budget" in kw and kw["step_path_budget"] == 256 * fc.spp:
            assert st["steps"] >= 24  # one tile per step
    for o in outs[1:]:
        assert np.array_equal(o["voxel_id"], outs[0]["voxel_id"])
        assert close_rel(o["rgb"], outs[0]["rgb"]).all()


@pytest.mark.parametrize("fifo", [False, True])
def test_small_request_passes_a_large_one_that_does_not_fit(ve, world, fifo):
    """Pools that hold one large request and a small one: a second large
    request waits for space; a small request queued behind it is admitted
    first unless admission is strict first come first served."""
    r, scenes, reqs = world
    sid, depth = scenes[1]
    eye = np.array([64.0, 120.0, -40.0], np.float32)  # the terrain fills most of the view
    big_fc = ve.FrameConfig(width=256, height=256, spp=4, bounces=3, primary_controlchecks=200,
                            bounce_controlchecks=200)
    big = (sid, ve.camera_ubo(eye, ve.look_at(eye, (64, 48, 64)), 70.0, 1.0), big_fc)
    small = reqs[1]  # 64 x 48
    with ve.Server(r, pixel_capacity=256 * 256 + 256 * 128, path_capacity=1 << 22, max_requests=8, fifo=fifo,
                   max_bypass_ms=60000) as srv:
        a = srv.submit(*big)
        b = srv.submit(*big)
        c = srv.submit(*small)
        ra, rb, rc = srv.wait(a), srv.wait(b), srv.wait(c)
    assert (ra["voxel_id"] != 0).mean() > 0.3  # a takes several steps
    assert rb["admit_s"] >= ra["done_s"] - 1e-3  # b waited for a's pixels
    if fifo:
        assert rc["admit_s"] >= rb["admit_s"]
    else:
        assert rc["admit_s"] < rb["admit_s"]
        assert rc["done_s"] < rb["done_s"]
    assert np.array_equal(ra["voxel_id"], rb["voxel_id"])
