"""Split frames (VE_FRAME_SPLIT): one frame of one view rendered as bands of
rows by several ranks, whose cache deposits are exchanged once and merged in
rank order (ve_split_export / ve_split_merge / ve_split_resolve).

CPU: the host logic of dist.SplitFrame with world_size 1, 2 and 3 on the gloo
backend, over a numpy stand-in of the renderer — bands, the padded record
all-gather with unequal counts, the rank-order merge, the row gather.

GPU: two or three ranks emulated by renderer contexts on one device, each
rendering its band in turn (no kernel waits on another rank), with bands that
do not align with the 16-row tiles and AvgPass halos of 1 to 10 rows.
Against the oracle's unsplit frames: GBuffer rows and every path's deposit
value bit for bit, counters summed over the ranks exact, the merged cache's
counts exact and sums within 2e-4, the resolved image within 1e-4 relative
(1e-4 absolute for the variance view); and the ranks' caches bitwise
identical frame after frame.
"""
import dataclasses
import os
import socket
import sys

import numpy as np
import pytest

import helpers

# ---------------------------------------------------------------------------
# CPU: host logic over a stand-in renderer
# ---------------------------------------------------------------------------
H, W = 13, 6


def vid_map():
    y, x = np.mgrid[0:H, 0:W]
    v = (y // 3) * 4 + x // 2 + 1  # voxels span band boundaries
    v[(y * 7 + x * 3) % 11 == 0] = 0  # misses
    return v.astype(np.uint32)


class StandInRenderer:
    """The split-frame methods of Renderer on the host: a frame decays the
    cache and deposits one sample per band pixel into the pixel's voxel."""

    def __init__(self, decay=0.5):
        self.vids = vid_map()
        self.decay = np.float32(decay)
        self.cache = {}  # vid -> (count, float32[5] {l2, r, g, b, w})
        self.delta = {}

    def render(self, sid, cam, f, outputs=()):
        import ve_b200 as ve

        assert f.flags & ve.FRAME_SPLIT and 0 <= f.row_begin < f.row_end <= f.height
        for k in self.cache:
            n, s = self.cache[k]
            self.cache[k] = (n, s * self.decay)
        self.delta = {}
        for y in range(f.row_begin, f.row_end):
            for x in range(W):
                vid = int(self.vids[y, x])
                if not vid:
                    continue
                rgb = np.float32([(y * 31 + x * 17 + f.frame_index * 5) % 97, (y + x) % 13, x + 1]) / np.float32(50)
                l2 = np.float32(rgb.mean()) ** 2
                n, s = self.delta.get(vid, (0, np.zeros(5, np.float32)))
                self.delta[vid] = (n + 1, s + np.concatenate([[l2], rgb, [1.0]]).astype(np.float32))
        out = {}
        if "gbuffer" in outputs:
            g = np.zeros((f.height, W, 4), np.uint32)
            g[f.row_begin:f.row_end, :, 3] = self.vids[f.row_begin:f.row_end]
            out["gbuffer"] = g
        return out

    def split_export(self, sid, buf, cap):
        recs = np.zeros((len(self.delta), 8), np.uint32)
        for i, (vid, (n, s)) in enumerate(sorted(self.delta.items(), reverse=True)):
            recs[i, 0], recs[i, 1] = vid, n
            recs[i, 2:7] = s.view(np.uint32)
        m = min(len(recs), cap)
        buf[: 8 * m] = __import__("torch").from_numpy(recs[:m].reshape(-1).view(np.int32))
        return len(recs)

    def split_merge(self, sid, parts, counts, stride):
        a = parts.cpu().numpy().view(np.uint32).reshape(-1, 8)
        for k, c in enumerate(counts):
            for r in a[k * stride:k * stride + c]:
                n, s = self.cache.get(int(r[0]), (0, np.zeros(5, np.float32)))
                self.cache[int(r[0])] = (n + int(r[1]), s + r[2:7].view(np.float32))
        return 0

    def split_resolve(self, sid, cam, f, outputs=("rgb",)):
        rgb = np.zeros((f.height, W, 3), np.float32)
        for y in range(f.row_begin, f.row_end):
            for x in range(W):
                vid = int(self.vids[y, x])
                if vid:
                    n, s = self.cache[vid]
                    rgb[y, x] = s[1:4] / s[4]
        return {"rgb": rgb} if "rgb" in outputs else {}


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _frames(vd, dist, frames=3):
    import ve_b200 as ve

    r = StandInRenderer()
    sf = vd.SplitFrame(r, 0, dist, device="cpu")
    fc = ve.FrameConfig(width=W, height=H, spp=1)
    outs = []
    for f in range(frames):
        fc.frame_index = f
        outs.append(sf.render(None, fc, outputs=("rgb", "gbuffer")))
    cache = {k: (n, s.view(np.uint32).tolist()) for k, (n, s) in sorted(r.cache.items())}
    return outs, cache, dict(sf.last)


def _worker(rank, world, port, queue):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, os.path.join(helpers.ROOT, "tests"))
    import helpers as h

    h.package()
    import ve_b200.dist as vd

    try:
        dist = vd.init("gloo", timeout_s=30.0)
        outs, cache, last = _frames(vd, dist)
        queue.put((rank, outs, cache, last))
        vd.shutdown(dist)
    except Exception as e:  # pragma: no cover - reported to the parent
        queue.put((rank, "error", repr(e), None))


def _run(world):
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        r = q.get(timeout=180)
        out[r[0]] = r
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return out


def test_band_rows(ve):
    import ve_b200.dist as vd

    for h, world in ((13, 2), (13, 3), (1080, 8), (7, 7)):
        bands = [vd.band_rows(h, k, world) for k in range(world)]
        assert bands[0][0] == 0 and bands[-1][1] == h
        assert all(a[1] == b[0] for a, b in zip(bands, bands[1:]))
        assert max(b - a for a, b in bands) - min(b - a for a, b in bands) <= 1
    with pytest.raises(ValueError):
        vd.band_rows(3, 0, 4)


@pytest.mark.parametrize("world", [2, 3])
def test_split_frames_gloo(ve, world):
    import ve_b200.dist as vd

    ref_outs, ref_cache, _ = _frames(vd, None)
    res = _run(world)
    for rank in range(world):
        assert res[rank][1] != "error", res[rank][2]
    caches = [res[k][2] for k in range(world)]
    for c in caches[1:]:
        assert c == caches[0]  # every rank merged the same records in the same order
    assert sorted(caches[0]) == sorted(ref_cache)
    for vid, (n, bits) in caches[0].items():
        assert n == ref_cache[vid][0]
        got = np.array(bits, np.uint32).view(np.float32)
        want = np.array(ref_cache[vid][1], np.uint32).view(np.float32)
        assert np.allclose(got, want, rtol=1e-5, atol=1e-6)
    counts = res[0][3]["counts"]
    assert len(counts) == world and len(set(counts)) > 1  # unequal parts: the padded exchange
    for rank in range(world):
        lo, hi = vd.band_rows(H, rank, world)
        assert res[rank][3]["band"] == (lo, hi)
        for f, out in enumerate(res[rank][1]):
            assert np.array_equal(out["gbuffer"], ref_outs[f]["gbuffer"])
            assert np.allclose(out["rgb"], ref_outs[f]["rgb"], rtol=1e-5, atol=1e-6)
            assert np.array_equal(out["rgb"], res[0][1][f]["rgb"])


# ---------------------------------------------------------------------------
# GPU: ranks emulated by contexts on one device
# ---------------------------------------------------------------------------
RTOL = 1e-4
ATOL = 1e-6


def close_rel(a, b, rtol=RTOL, atol=ATOL):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b) <= rtol * np.abs(b) + atol


@pytest.fixture(scope="module")
def ranks(ve):
    words, depth, mats, cam, fc = helpers.small_setup()
    rs = []
    for _ in range(3):
        r = ve.Renderer(hash_log2=20)
        r.set_materials(mats)
        rs.append((r, r.upload_scene(words, depth)))
    yield rs, rs[0][0].download_scene(rs[0][1]), depth, mats, cam, fc
    for r, _ in rs:
        r.close()


def split_frame(ve, rs, cam, fc, world, want=("gbuffer", "path_rgb")):
    """One frame over `world` emulated ranks; returns the assembled outputs,
    each rank's counters and the merge's record counts."""
    import torch
    import ve_b200.dist as vd

    bands = [vd.band_rows(fc.height, k, world) for k in range(world)]
    cap = max(b - a for a, b in bands) * fc.width
    bufs, counts, stats, fcs, outs = [], [], [], [], []
    for k, (r, sid) in enumerate(rs[:world]):
        f = dataclasses.replace(fc, flags=fc.flags | ve.FRAME_SPLIT, row_begin=bands[k][0], row_end=bands[k][1])
        outs.append(r.render(sid, cam, f, outputs=[w for w in want if w in ("gbuffer", "path_rgb")]))
        stats.append(r.stats())
        buf = torch.empty(cap * 8, dtype=torch.int32, device="cuda")
        counts.append(r.split_export(sid, buf, cap))
        bufs.append(buf)
        fcs.append(f)
    stride = max(max(counts), 1)
    parts = torch.cat([b[: stride * 8] for b in bufs])
    torch.cuda.synchronize()
    img = {}
    for k, (r, sid) in enumerate(rs[:world]):
        assert r.split_merge(sid, parts, counts, stride) == 0
        outs[k].update(r.split_resolve(sid, cam, fcs[k], [w for w in want if w in ("rgb", "voxel_id", "mapped")]))
    for key in outs[0]:
        a = outs[0][key].copy()
        for k in range(1, world):
            lo, hi = bands[k]
            if key == "path_rgb":
                s = fc.spp * fc.width
                a[lo * s:hi * s] = outs[k][key][lo * s:hi * s]
            else:
                a[lo:hi] = outs[k][key][lo:hi]
        img[key] = a
    return img, stats, counts


@pytest.mark.gpu
@pytest.mark.parametrize("world,radius,rtype", [(2, 10, 0), (3, 3, 0), (3, 0, 5)],
                         ids=["2-ranks", "3-ranks-radius-3", "3-ranks-variance-view"])
def test_ranks_match_oracle(ve, oracle, ranks, world, radius, rtype):
    from oracle.oracle import OracleRenderer, frame_params

    rs, words, depth, mats, cam, fc = ranks
    for r, sid in rs:
        r.cache_reset(sid)
    fc = ve.FrameConfig(**{**fc.__dict__, "flags": ve.FRAME_PATH_RGB, "reconstruction_radius": radius,
                           "render_type": rtype})
    orc = OracleRenderer(oracle)
    for frame in range(3):
        fc.frame_index = frame
        img, stats, counts = split_frame(ve, rs, cam, fc, world, want=("gbuffer", "path_rgb", "rgb", "voxel_id"))
        o = orc.render(words, depth, mats, cam, frame_params(fc), threads=8, want_path_rgb=True)
        assert np.array_equal(img["gbuffer"], o["gbuffer"]), frame
        assert np.array_equal(img["voxel_id"], o["gbuffer"][..., 3]), frame
        hit = o["gbuffer"][..., 3].reshape(-1) != 0
        mask = np.repeat(hit, fc.spp)
        gp = img["path_rgb"][mask].view(np.uint32)
        op = o["path_rgb"][mask].view(np.uint32)
        assert np.array_equal(gp, op), frame
        s = o["stats"]
        for k in ("rays_primary", "rays_bounce", "rays_shadow", "paths"):
            assert sum(st[k] for st in stats) == s[k], (frame, k)
        assert sum(st["deposits"] for st in stats) == s["paths"]
        assert sum(counts) >= len(np.unique(o["gbuffer"][..., 3][o["gbuffer"][..., 3] != 0]))
        # every rank holds the same cache, bit for bit
        d0 = rs[0][0].cache_dump(rs[0][1])
        for r, sid in rs[1:world]:
            d1 = r.cache_dump(sid)
            for a, b in zip(d0, d1):
                assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), frame
        ovids, ocounts, ovals = orc.cache()
        assert np.array_equal(d0[0], ovids)
        assert np.array_equal(d0[1].astype(np.uint64), ocounts)
        assert close_rel(d0[2], ovals, rtol=2e-4).all()
        if rtype == 5:  # the VARIANCE view cancels catastrophically: 1e-4 absolute on the display value
            assert (np.abs(img["rgb"].astype(np.float64) - o["rgb"]) <= 1e-4).all(), frame
        else:
            assert close_rel(img["rgb"], o["rgb"]).all(), frame
    assert img["rgb"].max() > 0.05 or rtype != 0


@pytest.mark.gpu
def test_one_band_is_the_whole_frame(ve, ranks):
    rs, words, depth, mats, cam, fc = ranks
    (r0, s0), (r1, s1) = rs[:2]
    r0.cache_reset(s0)
    r1.cache_reset(s1)
    fc = ve.FrameConfig(**{**fc.__dict__})
    for frame in range(2):
        fc.frame_index = frame
        img, stats, _ = split_frame(ve, rs, cam, fc, 1, want=("gbuffer", "rgb"))
        ref = r1.render(s1, cam, fc, outputs=("gbuffer", "rgb"))
        st = r1.stats()
        assert np.array_equal(img["gbuffer"], ref["gbuffer"])
        for k in ("rays_primary", "rays_bounce", "rays_shadow", "paths", "deposits"):
            assert stats[0][k] == st[k], k
        assert close_rel(img["rgb"], ref["rgb"]).all()
    v0, c0, _ = r0.cache_dump(s0)
    v1, c1, _ = r1.cache_dump(s1)
    assert np.array_equal(v0, v1) and np.array_equal(c0, c1)


@pytest.mark.gpu
def test_split_rejects(ve, ranks):
    import torch

    rs, words, depth, mats, cam, fc = ranks
    r, sid = rs[0]
    f = dataclasses.replace(fc, flags=ve.FRAME_SPLIT, row_begin=0, row_end=fc.height // 2)
    with pytest.raises(ve.VeError):  # the image comes from split_resolve
        r.render(sid, cam, f, outputs=("rgb",))
    with pytest.raises(ve.VeError):
        r.render(sid, cam, dataclasses.replace(f, row_begin=5, row_end=5), outputs=())
    with pytest.raises(ve.VeError):
        r.render(sid, cam, dataclasses.replace(f, flags=ve.FRAME_SPLIT | ve.FRAME_SCHEDULED), outputs=())
    r.render(sid, cam, f, outputs=())
    buf = torch.zeros(64 * 8, dtype=torch.int32, device="cuda")
    host = np.zeros(64 * 8, np.int32)
    with pytest.raises(ve.VeError):  # host memory is refused
        r.split_export(sid, host.ctypes.data, 64)
    with pytest.raises(ve.VeError):  # past the end of the allocation
        r.split_export(sid, buf, 1 << 30)
    n = r.split_export(sid, buf, 64)
    assert n > 64
    with pytest.raises(ve.VeError):  # more records than the stride
        r.split_merge(sid, buf, [65], 64)
    with pytest.raises(ve.VeError):  # a stride whose part offsets would overflow
        r.split_merge(sid, buf, [1, 1], 1 << 62)
    with pytest.raises(ve.VeError):  # the resolve's view differs from the frame's
        r.split_resolve(sid, cam, dataclasses.replace(f, row_end=f.row_end + 1), ("rgb",))
    r.render(sid, cam, fc, outputs=())  # a plain frame ends the split state
    with pytest.raises(ve.VeError):
        r.split_export(sid, buf, 64)
