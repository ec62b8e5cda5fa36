"""Full-frame parity at the benchmark's own configuration: depth-10 terrain
(66.2M voxels, 77.6M node words), 1920x1080, 4 spp x 3 bounces, radiance cache
2^22 entries with decay 0.95, orbit frames 0 and 1 — the device (through the
C ABI, production kernels: top table, persistent trace) against the oracle
rendering from its own build of the scene (oracle/scenes.py).

Bars: node words (with the device's leaf normals) bit-exact; per frame the
whole GBuffer bit-exact, every hit path's deposit value bitwise, ray counts
per category exact; after both frames the radiance cache's voxel ids and
deposit counts exact, its FP32 sums within 2e-4 relative of the FP64 oracle,
and every pixel's resolved and tonemapped radiance within 1e-4 relative
(floor 1e-6)."""
import os

import numpy as np
import pytest

import helpers
from oracle.oracle import OracleRenderer

pytestmark = pytest.mark.gpu

RTOL = 1e-4
ATOL = 1e-6


def close_rel(a, b, rtol=RTOL, atol=ATOL):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b) <= rtol * np.abs(b) + atol


def test_large_two_frames_full_parity(ve, oracle):
    from oracle import scenes

    w = helpers.workloads()
    L = w.LARGE
    threads = os.cpu_count() or 1
    words, nv = ve.terrain_words(L.depth, L.variant, L.seed)
    owords, onv = scenes.terrain_words(oracle, L.depth, L.variant, L.seed, threads)
    assert nv == onv == 66190300 and words.size == owords.size == 77636105
    assert np.array_equal(words, owords)
    mats = ve.terrain_materials(L.seed)
    omats = scenes.terrain_materials(oracle, L.seed)
    normals = oracle.fill_normals(owords, L.depth, fast=True, threads=threads)
    orc = OracleRenderer(oracle)
    with ve.Renderer(hash_log2=L.hash_log2) as r:
        r.set_materials(mats)
        sid = r.upload_scene(words, L.depth)
        assert np.array_equal(r.download_scene(sid), normals), "device leaf normals differ from the oracle"
        for f in (0, 1):
            eye, d = w.orbit_camera(f, L.frames, L.seed)
            cam = ve.camera_ubo(eye, d, L.fov, L.width / L.height)
            fc = ve.FrameConfig(width=L.width, height=L.height, spp=L.spp, bounces=L.bounces, frame_index=f,
                                primary_controlchecks=L.primary_controlchecks,
                                bounce_controlchecks=L.bounce_controlchecks, flags=ve.FRAME_PATH_RGB)
            g = r.render(sid, cam, fc, outputs=("gbuffer", "rgb", "mapped", "path_rgb"))
            st = r.stats()
            o = orc.render(normals, L.depth, omats, scenes.large_camera(oracle, f), scenes.large_params(f, flags=4),
                           threads=threads, want_path_rgb=True)
            assert np.array_equal(g["gbuffer"], o["gbuffer"]), f"frame {f}: GBuffer differs"
            hit = np.repeat(o["gbuffer"][..., 3].reshape(-1) != 0, L.spp)
            assert hit.mean() > 0.5
            gp, op = g["path_rgb"][hit], o["path_rgb"][hit]
            bad = np.any(gp.view(np.uint32) != op.view(np.uint32), axis=1)
            assert not bad.any(), f"frame {f}: {int(bad.sum())} of {hit.sum()} paths differ bitwise"
            s = o["stats"]
            for k in ("rays_primary", "rays_bounce", "rays_shadow"):
                assert st[k] == s[k], f"frame {f}: {k} {st[k]} != {s[k]}"
            assert st["paths"] == s["paths"] == st["deposits"] == int(hit.sum())
            assert st["deposits_dropped"] == 0
        vids, counts, vals = r.cache_dump(sid)
    ovids, ocounts, ovals = orc.cache()
    assert np.array_equal(vids, ovids)
    assert np.array_equal(counts.astype(np.uint64), ocounts)
    assert close_rel(vals, ovals, rtol=2e-4).all()
    ok = close_rel(g["rgb"], o["rgb"]).all(axis=-1)
    assert ok.all(), f"{1.0 - ok.mean():.2e} of pixels beyond 1e-4 relative"
    assert close_rel(g["mapped"], o["mapped"]).all()
    assert g["rgb"].max() > 0.05
