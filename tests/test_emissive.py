"""Emissive-light NEE (VE_FRAME_EMISSIVE): the light registry, single-pick RIS
and ReSTIR DI with per-voxel reservoirs (reference src/shd/shade.comp:576-836)
on the reference's own Cornell box (src/voxelengine.cpp:82-142).

The GLSL cannot run here, so the oracle restates the shader code
(oracle/ve_oracle.cpp emissive_nee, commit_emissive) under the product's
deterministic registration and reservoir-commit rules.  The scene itself is
pinned against the reference's compiled OctreeCPU / Octree::set.  The device
is held to the oracle frame after frame: GBuffer, every path's deposit value
bit for bit (this exercises the registry, the reservoirs committed by earlier
frames and every random draw), the counters, cache counts, and radiance within
1e-4 relative.
"""
import numpy as np
import pytest

import helpers
from oracle.oracle import OracleRenderer, frame_params

RTOL = 1e-4
ATOL = 1e-6
W = H = 96


def cornell(ve, depth=8):
    import ve_b200.workloads as wl

    cpu = ve.OctreeCPU(depth)
    wl.cornell_build(cpu, depth)
    oc = ve.Octree(depth)
    oc.set(cpu)
    eye, d = wl.cornell_camera(depth)
    cam = ve.camera_ubo(eye, d, 90.0, 1.0)
    return oc.words(), wl.cornell_materials(), cam


def emissive_config(ve, **kw):
    d = dict(width=W, height=H, spp=2, bounces=3, primary_controlchecks=70, bounce_controlchecks=120,
             sky=(0.05, 0.05, 0.05), flags=ve.FRAME_EMISSIVE)
    d.update(kw)
    return ve.FrameConfig(**d)


# ---------------------------------------------------------------------------
# CPU
# ---------------------------------------------------------------------------
def test_cornell_scene_matches_reference_build(ve, ref):
    import ve_b200.workloads as wl

    words, _, _ = cornell(ve, 7)
    rs = ref.scene(7)
    wl.cornell_build(rs, 7)
    ref_words, size, n_voxels = rs.set()
    assert np.array_equal(words, ref_words)
    assert n_voxels > 100000


def test_pow_unit_accuracy(oracle):
    rng = np.random.default_rng(4)
    x = np.concatenate([rng.uniform(1e-3, 1.0, 200000), 1.0 - rng.uniform(0, 1e-2, 100000)]).astype(np.float32)
    e = rng.uniform(2.0, 20000.0, x.size).astype(np.float32)
    got = oracle.pow_unit(x, e).astype(np.float64)
    y = e.astype(np.float64) * np.log2(x.astype(np.float64))
    want = np.exp2(y)
    ok = want > 1e-30
    rel = np.abs(got[ok] - want[ok]) / want[ok]
    assert (rel <= 3e-7 * (1.0 + np.abs(y[ok]))).all()
    assert oracle.pow_unit(np.float32([1.0, 0.5]), np.float32([88.0, 2.0])).tolist() == [1.0, 0.25]


def test_oracle_registry_and_reservoirs(ve, oracle):
    words, mats, cam = cornell(ve)
    words = oracle.fill_normals(words, 8)
    orc = OracleRenderer(oracle)
    fc = emissive_config(ve)
    fc.frame_index = 0
    o0 = orc.render(words, 8, mats, cam, frame_params(fc), threads=8)
    s0 = o0["stats"]
    g = o0["gbuffer"]
    lit = np.unique(g[..., 3][(g[..., 1] == 1) & (g[..., 3] != 0)])
    assert s0["emissive_lights"] == min(lit.size, 4096) > 100
    assert s0["nee_emissive"] == 0 and s0["restir_commits"] == 0  # frame 0: no lights yet
    fc.frame_index = 1
    s1 = orc.render(words, 8, mats, cam, frame_params(fc), threads=8)["stats"]
    assert s1["nee_emissive"] > 1000
    assert s1["restir_commits"] > 1000
    # without ReSTIR only the single-pick estimator runs: no reservoirs
    orc2 = OracleRenderer(oracle)
    fc2 = emissive_config(ve, restir=0)
    for f in range(2):
        fc2.frame_index = f
        s = orc2.render(words, 8, mats, cam, frame_params(fc2), threads=8)["stats"]
    assert s["restir_commits"] == 0 and s["nee_emissive"] > 1000


def test_oracle_thread_invariant(ve, oracle):
    words, mats, cam = cornell(ve)
    words = oracle.fill_normals(words, 8)
    outs = []
    for threads in (1, 5):
        orc = OracleRenderer(oracle)
        fc = emissive_config(ve)
        res = []
        for f in range(3):
            fc.frame_index = f
            res.append(orc.render(words, 8, mats, cam, frame_params(fc), threads=threads, want_path_rgb=True))
        outs.append(res)
    for a, b in zip(*outs):
        assert np.array_equal(a["path_rgb"].view(np.uint32), b["path_rgb"].view(np.uint32))
        assert a["stats"] == b["stats"]


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def scene(ve):
    words, mats, cam = cornell(ve)
    r = ve.Renderer(hash_log2=20)
    r.set_materials(mats)
    sid = r.upload_scene(words, 8)
    yield r, sid, r.download_scene(sid), mats, cam
    r.close()


def close_rel(a, b, rtol=RTOL, atol=ATOL):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b) <= rtol * np.abs(b) + atol


def run_frames(ve, oracle, scene, fc, frames, want=("gbuffer", "path_rgb")):
    r, sid, words, mats, cam = scene
    r.cache_reset(sid)
    orc = OracleRenderer(oracle)
    out = []
    for f in range(frames):
        fc.frame_index = f
        g = r.render(sid, cam, fc, outputs=want)
        st = r.stats()
        o = orc.render(words, 8, mats, cam, frame_params(fc), threads=8, want_path_rgb="path_rgb" in want)
        out.append((g, st, o))
    return orc, out


def assert_exact(g, st, o, frame):
    assert np.array_equal(g["gbuffer"], o["gbuffer"]), frame
    s = o["stats"]
    for k in ("rays_primary", "rays_bounce", "rays_shadow", "paths", "emissive_lights", "nee_emissive",
              "restir_commits"):
        assert st[k] == s[k], (frame, k, st[k], s[k])
    hit = o["gbuffer"][..., 3].reshape(-1) != 0
    spp = g["path_rgb"].shape[0] // hit.size
    mask = np.repeat(hit, spp)
    gp = g["path_rgb"][mask].view(np.uint32)
    op = o["path_rgb"][mask].view(np.uint32)
    bad = np.nonzero((gp != op).any(1))[0]
    assert bad.size == 0, (frame, bad.size, bad[:5].tolist())


@pytest.mark.gpu
@pytest.mark.parametrize("restir", [7, 0, 1 | 2, 1 | 4], ids=["restir", "ris", "temporal", "spatial"])
def test_frames_match_oracle(ve, oracle, scene, restir):
    fc = emissive_config(ve, restir=restir, flags=ve.FRAME_EMISSIVE | ve.FRAME_PATH_RGB)
    orc, out = run_frames(ve, oracle, scene, fc, 4, want=("gbuffer", "path_rgb", "rgb"))
    for f, (g, st, o) in enumerate(out):
        assert_exact(g, st, o, f)
    assert out[-1][1]["nee_emissive"] > 1000
    if restir & 1:
        assert out[-1][1]["restir_commits"] > 1000
    r, sid = scene[0], scene[1]
    vids, counts, vals = r.cache_dump(sid)
    ovids, ocounts, ovals = orc.cache()
    assert np.array_equal(vids, ovids)
    assert np.array_equal(counts.astype(np.uint64), ocounts)
    assert close_rel(vals, ovals, rtol=2e-4).all()
    g, st, o = out[-1]
    assert close_rel(g["rgb"], o["rgb"]).all()
    assert g["rgb"].max() > 0.05


@pytest.mark.gpu
def test_scheduled_emissive_frames(ve, oracle, scene):
    fc = emissive_config(ve, flags=ve.FRAME_EMISSIVE | ve.FRAME_SCHEDULED | ve.FRAME_PATH_RGB)
    _, out = run_frames(ve, oracle, scene, fc, 3)
    for f, (g, st, o) in enumerate(out):
        assert np.array_equal(g["gbuffer"], o["gbuffer"])
        for k in ("scheduled_paths", "emissive_lights", "nee_emissive", "restir_commits", "rays_shadow"):
            assert st[k] == o["stats"][k], (f, k)
        n = o["stats"]["scheduled_paths"]
        assert np.array_equal(g["path_rgb"][:n].view(np.uint32), o["path_rgb"][:n].view(np.uint32)), f


@pytest.mark.gpu
def test_cache_reset_forgets_lights(ve, oracle, scene):
    r, sid, words, mats, cam = scene
    fc = emissive_config(ve)
    r.cache_reset(sid)
    for f in range(2):
        fc.frame_index = f
        r.render(sid, cam, fc, outputs=())
    assert r.stats()["emissive_lights"] > 0
    r.cache_reset(sid)
    fc.frame_index = 0
    r.render(sid, cam, fc, outputs=())
    st = r.stats()
    assert st["nee_emissive"] == 0  # the registry starts empty again
    o = OracleRenderer(oracle).render(words, 8, mats, cam, frame_params(fc), threads=8)
    assert st["emissive_lights"] == o["stats"]["emissive_lights"]


@pytest.mark.gpu
def test_rejects_cache_terminated_paths(ve, scene):
    r, sid, words, mats, cam = scene
    with pytest.raises(ve.VeError):
        r.render(sid, cam, emissive_config(ve, flags=ve.FRAME_EMISSIVE | ve.FRAME_TERMINATE_HASH))
    with pytest.raises(ve.VeError):
        r.render(sid, cam, emissive_config(ve, restir_m=65))
    r.render(sid, cam, emissive_config(ve), outputs=("voxel_id",))
