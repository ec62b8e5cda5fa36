"""The reference's dual-channel lBuffer AccumPass (VE_FRAME_LBUFFER):
depositSampleDual (src/shd/shade.comp:96-257) with per-channel halving at the
sample caps, the firefly clamp, the stale reset and least-recently-used slot
replacement; lookupVoxelAvg (src/shd/resolve.comp:109-148) and
lookupIndirectVariance (src/shd/rank.comp:66-87) read it.

The oracle's restatement is pinned against a plain-Python transcription of
the shader's deposit (below, written from the GLSL statement by statement) on
synthetic deposit streams that exercise every branch.  The device is held to
the oracle: GBuffer, per-path deposit values and counters exact, the whole
lBuffer (every occupied slot, all 12 words) exact, radiance within 1e-4.
"""
import struct

import numpy as np
import pytest

import helpers
from oracle.oracle import OracleRenderer, frame_params

W_ROWS, SLOTS, STRIDE = 32768, 32, 12
RTOL = 1e-4
ATOL = 1e-6


# ---------------------------------------------------------------------------
# plain-Python transcription of shade.comp depositSampleDual
# ---------------------------------------------------------------------------
def f32(x):
    return struct.unpack("f", struct.pack("f", x))[0]


def u32(x):
    return x & 0xFFFFFFFF


def pack_rgb_l2(rgb):
    u = [int(f32(min(max(c, 0.0), 1024.0) * 255.0)) for c in rgb]
    L = (u[0] + u[1] + u[2]) // 3
    return u + [u32(L * L)]


def deposit_sample_dual(img, vid, dir_rgb, ind_rgb, P):
    d = pack_rgb_l2(dir_rgb)
    e = pack_rgb_l2(ind_rgb)
    h = vid % (W_ROWS - 1) + 1
    row = img[h]
    candidate = (0xFFFFFFFF, 0, 0)
    for i in range(0, STRIDE * SLOTS, STRIDE):
        if row[i] == 0:  # imageAtomicCompSwap(.., 0, vid)
            row[i] = vid
        id_, slot_time = row[i], row[i + 11]
        if id_ != vid:
            if slot_time < candidate[0]:
                candidate = (slot_time, id_, i)
            continue
        if not P["disable_stale"] and slot_time != 0 and u32(slot_time + P["update_time"]) < P["time"]:
            reset_slot(row, i, vid, d, e, P["time"])
            return
        if row[i + 1] >= P["cap_dir"]:
            for k in range(1, 6):
                row[i + k] >>= 1
        if row[i + 6] >= P["cap_ind"]:
            for k in range(6, 11):
                row[i + k] >>= 1
        for base, c in ((i + 1, d), (i + 6, e)):
            n = row[base]
            if n > 4:
                mean_l = f32(f32(float(u32(row[base + 1] + row[base + 2] + row[base + 3]))) / f32(float(u32(3 * n))))
                sample_l = f32(f32(float(u32(c[0] + c[1] + c[2]))) / 3.0)
                m = f32(mean_l * P["k"])
                thresh = P["floor"] if m < P["floor"] else m
                if sample_l > thresh:
                    scale = f32(thresh / sample_l)
                    for k in range(3):
                        c[k] = int(f32(float(c[k]) * scale))
                    L = (c[0] + c[1] + c[2]) // 3
                    c[3] = u32(L * L)
        row[i + 1] = u32(row[i + 1] + 1)
        for k in range(4):
            row[i + 2 + k] = u32(row[i + 2 + k] + d[k])
        row[i + 6] = u32(row[i + 6] + 1)
        for k in range(4):
            row[i + 7 + k] = u32(row[i + 7 + k] + e[k])
        row[i + 11] = P["time"]
        return
    if candidate[0] != 0xFFFFFFFF:
        reset_slot(row, candidate[2], vid, d, e, P["time"])


def reset_slot(row, i, vid, d, e, time):
    row[i] = vid
    row[i + 1] = 1
    row[i + 2:i + 6] = d
    row[i + 6] = 1
    row[i + 7:i + 11] = e
    row[i + 11] = time


def synthetic_stream(rng, n, rows):
    """Deposits of many vids crowded into a few rows (collisions, evictions),
    with bright outliers (firefly clamp) and zero samples."""
    vids = []
    for r in rows:
        base = rng.integers(0, 1 << 12, 48)
        vids += [int(r + (W_ROWS - 1) * b) for b in base]  # vid % (W-1) + 1 == r + 1
    vids = np.array(vids, np.int64)
    recs = np.zeros((n, 8), np.uint32)
    pick = vids[rng.integers(0, vids.size, n)]
    recs[:, 0] = pick.astype(np.uint32)
    vals = rng.exponential(0.3, (n, 6)).astype(np.float32)
    vals[rng.random(n) < 0.05] *= 200.0
    vals[rng.random(n) < 0.1] = 0.0
    recs[:, 2:8] = vals.view(np.uint32)
    return recs


@pytest.mark.parametrize("stale", [False, True])
def test_oracle_deposit_matches_shader_transcription(oracle, stale):
    from oracle.oracle import FrameParams

    rng = np.random.default_rng(7 + int(stale))
    recs = synthetic_stream(rng, 6000, rows=[3, 900, 32000])
    P = FrameParams()
    P.sample_cap_direct, P.sample_cap_indirect = 16, 64
    P.firefly_k, P.firefly_floor = 1.0, 255.0
    P.disable_stale_reset = 0 if stale else 1
    P.update_time = 20
    table = np.zeros(W_ROWS * SLOTS * STRIDE, np.uint32)
    img = {}
    pp = {"cap_dir": 16, "cap_ind": 64, "k": f32(1.0), "floor": f32(255.0), "disable_stale": 0 if stale else 1,
          "update_time": 20}
    for chunk in range(6):  # advancing clock: stale slots get reset
        P.time = pp["time"] = 100 + 15 * chunk
        part = recs[chunk * 1000:(chunk + 1) * 1000]
        oracle.lb_apply(part, P, table)
        for r in part:
            vid = int(r[0])
            dv = r[2:5].view(np.float32).tolist()
            iv = r[5:8].view(np.float32).tolist()
            h = vid % (W_ROWS - 1) + 1
            img.setdefault(h, [0] * (SLOTS * STRIDE))
            deposit_sample_dual(img, vid, dv, iv, pp)
    t = table.reshape(W_ROWS, SLOTS * STRIDE)
    for h, row in img.items():
        assert t[h].tolist() == row, h
    occupied = t[:, 0::STRIDE] != 0
    assert occupied.sum() == sum(sum(1 for i in range(0, SLOTS * STRIDE, STRIDE) if row[i]) for row in img.values())
    assert (t[:, 1::STRIDE][occupied] <= 16).all() and (t[:, 6::STRIDE][occupied] <= 64).all()


def lb_config(ve, fc, **kw):
    d = {**fc.__dict__, "flags": ve.FRAME_LBUFFER | ve.FRAME_PATH_RGB}
    d.update(kw)
    return ve.FrameConfig(**d)


def test_oracle_lbuffer_frames(ve, oracle):
    words, depth, mats, cam, fc = helpers.small_setup()
    words = oracle.fill_normals(words, depth)
    outs = []
    for threads in (1, 6):
        orc = OracleRenderer(oracle)
        f = lb_config(ve, fc)
        for k in range(3):
            f.frame_index = k
            o = orc.render(words, depth, mats, cam, frame_params(f), threads=threads, want_path_rgb=True)
        outs.append((orc.lbuffer(), o))
    (l1, o1), (l2, o2) = outs
    assert np.array_equal(l1, l2)
    assert np.array_equal(o1["rgb"], o2["rgb"])
    assert l1.shape[0] > 1000
    dc, ic = l1[:, 3], l1[:, 8]
    assert (dc <= 16).all() and (ic <= 64).all() and (dc >= 1).all()


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def small(ve):
    words, depth, mats, cam, fc = helpers.small_setup()
    r = ve.Renderer(hash_log2=20)
    r.set_materials(mats)
    sid = r.upload_scene(words, depth)
    yield r, sid, r.download_scene(sid), depth, mats, cam, fc
    r.close()


def close_rel(a, b, rtol=RTOL, atol=ATOL):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b) <= rtol * np.abs(b) + atol


def run_pair(r, sid, words, depth, mats, cam, fcs, oracle, want=("gbuffer", "path_rgb", "rgb")):
    r.cache_reset(sid)
    orc = OracleRenderer(oracle)
    out = []
    for f in fcs:
        g = r.render(sid, cam, f, outputs=want)
        st = r.stats()
        o = orc.render(words, depth, mats, cam, frame_params(f), threads=8, want_path_rgb=True)
        out.append((g, st, o))
    return orc, out


def assert_frame(g, st, o, n_paths=None):
    assert np.array_equal(g["gbuffer"], o["gbuffer"])
    for k in ("rays_primary", "rays_bounce", "rays_shadow", "paths", "deposits"):
        assert st[k] == o["stats"][k], k
    gp, op = g["path_rgb"], o["path_rgb"]
    if n_paths is not None:
        gp, op = gp[:n_paths], op[:n_paths]
    assert np.array_equal(gp.view(np.uint32), op.view(np.uint32))


@pytest.mark.gpu
def test_frames_and_lbuffer_exact(ve, oracle, small):
    r, sid, words, depth, mats, cam, fc = small
    fcs = []
    for k in range(6):  # caps reached (direct cap 4), the clock advancing with stale resets
        f = lb_config(ve, fc, frame_index=k, spp=2, sample_cap_direct=4, sample_cap_indirect=8, time=10 * k,
                      update_time=15, disable_stale_reset=0)
        fcs.append(f)
    orc, out = run_pair(r, sid, words, depth, mats, cam, fcs, oracle)
    for g, st, o in out:
        assert_frame(g, st, o)
    dev, ref = r.lbuffer_dump(sid), orc.lbuffer()
    assert dev.shape == ref.shape and dev.shape[0] > 1000
    assert np.array_equal(dev, ref)
    g, st, o = out[-1]
    assert close_rel(g["rgb"], o["rgb"]).all()
    assert g["rgb"].max() > 0.05


@pytest.mark.gpu
def test_scheduled_lbuffer_frames(ve, oracle, small):
    """Scheduling ranks voxels by the lBuffer's own indirect variance
    (rank.comp), so the tiers and shade lists match exactly."""
    r, sid, words, depth, mats, cam, fc = small
    fcs = [lb_config(ve, fc, flags=ve.FRAME_LBUFFER | ve.FRAME_SCHEDULED | ve.FRAME_PATH_RGB, frame_index=k,
                     variance_norm=2000.0) for k in range(4)]
    orc, out = run_pair(r, sid, words, depth, mats, cam, fcs, oracle)
    n2 = 0
    for g, st, o in out:
        n = o["stats"]["scheduled_paths"]
        assert st["scheduled_paths"] == n and st["scheduled_voxels"] == o["stats"]["scheduled_voxels"]
        assert_frame(g, st, o, n_paths=n)
        n2 += n - st["scheduled_voxels"]
    assert n2 != 0
    assert np.array_equal(r.lbuffer_dump(sid), orc.lbuffer())


@pytest.mark.gpu
def test_emissive_lbuffer_frames(ve, oracle):
    import test_emissive as te

    words, mats, cam = te.cornell(ve)
    with ve.Renderer(hash_log2=20) as r:
        r.set_materials(mats)
        sid = r.upload_scene(words, 8)
        dw = r.download_scene(sid)
        fcs = [te.emissive_config(ve, flags=ve.FRAME_EMISSIVE | ve.FRAME_LBUFFER | ve.FRAME_PATH_RGB, frame_index=k)
               for k in range(3)]
        orc, out = run_pair(r, sid, dw, 8, mats, cam, fcs, oracle)
        for g, st, o in out:
            assert_frame(g, st, o)
        assert np.array_equal(r.lbuffer_dump(sid), orc.lbuffer())


@pytest.mark.gpu
def test_lbuffer_rejects(ve, small):
    r, sid, words, depth, mats, cam, fc = small
    f = lb_config(ve, fc)
    with pytest.raises(ve.VeError):
        r.render_batch([(sid, cam, f), (sid, cam, f)])
    with pytest.raises(ve.VeError):
        r.render(sid, cam, lb_config(ve, fc, flags=ve.FRAME_LBUFFER | ve.FRAME_TERMINATE_HASH))
    r.render(sid, cam, f, outputs=("voxel_id",))
