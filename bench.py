#!/usr/bin/env python
"""Benchmark of the plain method: Mrays/s at 1080p on a depth-10 octree.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one frame of the large workload: depth-10 (1024^3) seeded terrain
with overhangs (66.2M voxels, 77.6M node words), 1920x1080, 4 spp x 3 bounces,
radiance cache 2^22 entries, decay 0.95, camera on the seeded 64-frame orbit of
radius 600.  A ray is one DDA traversal (primary, bounce or sun shadow).

* ``value``: device-resident frames back to back (no host outputs, each a
  replay of the frame's CUDA graph), CUDA events on the renderer's stream
  around K frames, max over ranks.  The stage breakdown comes from the same
  frames rendered again with per-pass events (direct launches).
* ``e2e``: the same frames through the public API with each frame's result —
  its displayed RGBA8 image, final.frag's framebuffer store — read into pinned
  host memory and the per-frame view table uploaded; each frame's image is
  copied on the renderer's copy stream while the next frame renders
  (VE_FRAME_ASYNC_OUTPUTS, two alternating pinned images); events around all K
  steps and the last frame's copy.
* ``roofline``: the trace kernel (bounce + shadow DDA): algorithmic bytes
  (4 B per distinct node word read + 48 B ray state per traversal) over its
  CUDA-event time inside the timed frames, against the measured HBM copy
  bandwidth; ``roofline.l2`` sets the L2 bytes of the same kernel (ncu) over
  that time against the L2 byte peak, the yardstick for its L2-resident tree.
* ``cpu_baseline``: the scalar C++ oracle on the host cores (all threads),
  on a bounded band of rows of frame 0.

Multi-GPU (torchrun, one process per GPU): replicas — rank r renders its own
orbit frames; no collective on the data path ("scaling": "weak").
``--impl reference`` times the reference's path on the host CPU (the oracle
port of its GLSL passes; the reference has no runnable GPU path here).
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402


def load_package():
    import importlib.util

    pkg = os.path.join(ROOT, "voxelengine3.0_b200")
    if "ve_b200" in sys.modules:
        return sys.modules["ve_b200"]
    spec = importlib.util.spec_from_file_location("ve_b200", os.path.join(pkg, "__init__.py"),
                                                  submodule_search_locations=[pkg])
    m = importlib.util.module_from_spec(spec)
    sys.modules["ve_b200"] = m
    spec.loader.exec_module(m)
    return m


METRIC = "Mrays/s at 1080p depth-10 octree"


def measured_trace_traffic():
    """DRAM bytes per k_trace launch of this workload, measured by ncu on the
    960x540 reduced case and scaled to 1080p (profiles/k_trace_traffic.json):
    (bytes, source) or (None, None)."""
    p = os.path.join(ROOT, "profiles", "k_trace_traffic.json")
    try:
        d = json.load(open(p))
        return float(d["dram_bytes_per_launch_1080p"]), d.get("source")
    except (OSError, KeyError, ValueError):
        return None, None


def trace_l2_roofline(ms_per_launch):
    """The trace kernel against L2 instead of HBM (its node words and top
    table are mostly L2-resident): L2 bytes per launch from the same ncu
    capture as the DRAM traffic, over the live launch time, against the
    nominal L2 byte peak recorded with it.  None when the record is absent."""
    p = os.path.join(ROOT, "profiles", "k_trace_traffic.json")
    try:
        d = json.load(open(p))
        b, peak = float(d["lts_bytes_per_launch_1080p"]), float(d["l2_peak_gbs"])
    except (OSError, KeyError, ValueError):
        return None
    if not ms_per_launch:
        return None
    achieved = b / (ms_per_launch / 1e3) / 1e9
    return {"achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "bytes_per_launch": b, "peak_kind": d.get("l2_peak_source")}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9 and parts[1].replace(".", "").isdigit():
                    rows.append(parts)
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]), "reasons": reasons,
                "samples": len(rows)}


def frame_config(ve, W, f, flags=0):
    return ve.FrameConfig(width=W.width, height=W.height, spp=W.spp, bounces=W.bounces, frame_index=f,
                          primary_controlchecks=W.primary_controlchecks,
                          bounce_controlchecks=W.bounce_controlchecks, flags=flags)


def rays_of(st):
    return st["rays_primary"] + st["rays_bounce"] + st["rays_shadow"]


def cpu_baseline(ve, W, words, mats, budget_s):
    """Oracle on all host cores over whole frames of the orbit (frame 0 first;
    rows of it when one frame exceeds the budget), plus a 1-thread figure on
    a band of rows of frame 0 and the CPU model."""
    from oracle.oracle import Oracle, OracleRenderer
    from oracle import scenes

    orc = Oracle()
    threads = os.cpu_count() or 1
    cam = scenes.large_camera(orc, 0)
    fp = scenes.large_params(0)
    mid = W.height // 2
    rows = max(threads, 8)
    total_rays = 0
    total_t = 0.0
    while True:
        r0 = max(0, mid - rows // 2)
        rr = OracleRenderer(orc)
        t = time.perf_counter()
        out = rr.render(words, W.depth, mats, cam, fp, threads=threads, rows=(r0, r0 + rows), want_rgb=False)
        dt = time.perf_counter() - t
        s = out["stats"]
        total_rays, total_t = s["rays_primary"] + s["rays_bounce"] + s["rays_shadow"], dt
        if dt * 2.5 > budget_s or rows >= W.height:
            break
        rows = min(W.height, int(rows * max(2.0, budget_s / max(dt, 1e-3) * 0.5)))
    # one thread: a band of rows of frame 0 sized to about a fifth of the budget
    rows1 = 2
    while True:
        r1 = mid - rows1 // 2
        t = time.perf_counter()
        o1 = OracleRenderer(orc).render(words, W.depth, mats, cam, fp, threads=1, rows=(r1, r1 + rows1),
                                        want_rgb=False)
        dt1 = time.perf_counter() - t
        n1 = rays_of_oracle(o1["stats"])
        if dt1 * 2.5 > budget_s / 5 or rows1 >= W.height:
            break
        rows1 = min(W.height, rows1 * 2)
    return {"value": total_rays / total_t / 1e6, "unit": "Mrays/s", "cores": threads, "kind": "port",
            "sample": f"frame 0 rows {r0}-{r0 + rows - 1} of {W.width}x{W.height}, {W.spp} spp x {W.bounces} "
                      f"bounces, {total_rays} rays in {total_t:.1f} s",
            "threads_1": {"value": n1 / dt1 / 1e6, "unit": "Mrays/s", "cores": 1,
                          "sample": f"frame 0 rows {r1}-{r1 + rows1 - 1}, {n1} rays in {dt1:.1f} s"},
            "cpu_model": scenes.cpu_model(), "nproc": threads}


def large_config(n_voxels, n_words):
    """The workload description both arms print (identical by construction)."""
    return {"workload": "large: depth-10 (1024^3) terrain + overhangs, 1920x1080, 4 spp x 3 bounces, "
                        "hash 2^22, decay 0.95, orbit r=600 (one whole frame per step)",
            "voxels": int(n_voxels), "node_words": int(n_words), "controlchecks": [300, 300],
            "frames": "orbit frames 0, 1, 2, ... (warm-up first)",
            "l2": "inputs larger than L2 (310 MB node array, ~1 GB path state)",
            "parallelism": "replicas"}


def run_reference(args, rank, world):
    """The reference's path on the host CPU: the oracle port of its passes on
    all host threads, whole frames of the large workload, the same frames as
    rank 0 of the device arm.  Maps no product library: the scene, materials,
    camera and frame parameters come from oracle/ (oracle/scenes.py)."""
    if rank != 0:
        return 0
    from oracle.oracle import Oracle, OracleRenderer
    from oracle import scenes

    W = scenes.LARGE
    orc = Oracle()
    threads = os.cpu_count() or 1
    words, nv = scenes.terrain_words(orc, W.depth, W.variant, W.seed, threads)
    # normals as the device pass computes them (3x3x3 occupancy gradient)
    words = orc.fill_normals(words, W.depth, fast=True, threads=threads)
    mats = scenes.terrain_materials(orc, W.seed)
    rr = OracleRenderer(orc)

    def step(f):
        cam = scenes.large_camera(orc, f)
        t = time.perf_counter()
        out = rr.render(words, W.depth, mats, cam, scenes.large_params(f % W.frames), threads=threads)
        return time.perf_counter() - t, rays_of_oracle(out["stats"])

    for f in range(args.warmup):
        step(f)
    tt = 0.0
    rays = 0
    for i in range(args.steps):
        dt, n = step(args.warmup + i)
        tt += dt
        rays += n
    v = rays / tt / 1e6
    sample = (f"whole {W.width}x{W.height} frames {args.warmup}..{args.warmup + args.steps - 1} of the orbit "
              f"(after {args.warmup} warm-up frames), {W.spp} spp x {W.bounces} bounces, GBuffer + paths + "
              f"FP64 radiance cache + AvgPass, {rays} rays in {tt:.1f} s")
    line = {"metric": METRIC, "value": v, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": tt / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded value-noise terrain, seeded orbit camera)", "impl": "reference",
            "config": large_config(nv, words.size),
            "cpu_baseline": {"value": v, "unit": "Mrays/s", "cores": threads, "kind": "port", "sample": sample,
                             "cpu_model": scenes.cpu_model(), "nproc": threads},
            "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "rays_per_step": rays / args.steps}
    print(json.dumps(line), flush=True)
    return 0


def rays_of_oracle(s):
    return s["rays_primary"] + s["rays_bounce"] + s["rays_shadow"]


def run_batching(args, rank, world):
    """64 views (resolutions 128^2..1080p, spp 1-8, bounces 1-4, random poses)
    over 4 resident octrees of depth 8, 9, 10, 10: one batched wavefront per
    frame (one launch per kernel and bounce for all views, CUDA-graph replay,
    autotuned launch shapes) against 64 per-view plain renders."""
    import torch

    import ve_b200.dist as vd
    import ve_b200.workloads as wl

    ve = load_package()
    rank, world, local = vd.env_rank()
    dist = vd.init("nccl", timeout_s=300.0, device=local)
    torch.cuda.set_device(local)
    vs = wl.batching_views(64, seed=7 + rank)
    scene_words = []
    for depth, variant, seed in wl.BATCH_SCENES:
        w, nv = ve.terrain_words(depth, variant, seed)
        scene_words.append((w, depth, nv))
    results = {}
    for mode in ("batched", "per_view"):
        r = ve.Renderer(device=local, hash_log2=22, graphs=(mode == "batched"), pipeline=not args.no_pipeline)
        r.set_materials(ve.terrain_materials(1))
        sids = [r.upload_scene(w, d) for w, d, _ in scene_words]
        views = []
        for v in vs:
            cam = ve.camera_ubo(v["eye"], v["dir"], 70.0, v["width"] / v["height"])
            fc = ve.FrameConfig(width=v["width"], height=v["height"], spp=v["spp"], bounces=v["bounces"],
                                frame_index=v["frame"], primary_controlchecks=300, bounce_controlchecks=300)
            views.append((sids[v["scene"]], cam, fc))
        tuned = r.autotune(views, frames_per_trial=1) if mode == "batched" else r.launch_config()
        stream = torch.cuda.ExternalStream(r.stream, device=local)

        def frame():
            if mode == "batched":
                r.render_batch(views, outputs=())
            else:
                for v in views:
                    r.render(*v, outputs=())

        for _ in range(args.warmup):
            frame()
        r.synchronize()
        r.reset_total_stats()
        torch.cuda.synchronize(local)
        vd.barrier(dist)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            frame()
        r.join()  # the end event follows the second frame set's stream too
        e1.record(stream)
        e1.synchronize()
        ms = vd.max_over_ranks(e0.elapsed_time(e1), dist, f"cuda:{local}")
        tot = r.total_stats()
        rays = vd.sum_over_ranks(rays_of(tot), dist, f"cuda:{local}")
        results[mode] = {"mrays_s": rays / (ms / 1e3) / 1e6, "ms_per_frame": ms / args.steps,
                         "rays_per_frame": rays_of(tot) / args.steps, "launch_config": tuned,
                         "kernel_launches_per_frame": tot["kernel_launches"] / args.steps}
        r.close()
    if rank == 0:
        line = {"metric": "Mrays/s, 64-view batch over 4 octrees (depth 8/9/10/10)",
                "value": results["batched"]["mrays_s"], "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": results["batched"]["ms_per_frame"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded views)",
                "config": {"workload": "batching: 64 views, resolutions {128^2,256^2,640x360,1280x720,1920x1080}, "
                                       "spp 1-8, bounces 1-4, 4 octrees depth 8/9/10/10",
                           "pixels": int(sum(v["width"] * v["height"] for v in vs))},
                "batched": results["batched"], "per_view_plain": results["per_view"],
                "frame_pipeline": not args.no_pipeline,
                "speedup_vs_per_view": results["batched"]["mrays_s"] / results["per_view"]["mrays_s"]}
        print(json.dumps(line), flush=True)
    vd.shutdown(dist)
    return 0


def _pct(xs, q):
    xs = sorted(xs)
    if not xs:
        return None
    k = min(len(xs) - 1, max(0, int(math.ceil(q / 100.0 * len(xs))) - 1))
    return xs[k]


def run_serving(args, rank, world):
    """Render server under a Poisson request stream at 80% of its measured
    capacity: 8 resident octrees of depth 8-11, requests with resolutions
    128^2..1080p, spp 1-16, bounces 1-4.  Capacity is measured first in a
    closed loop (32 requests outstanding); the open-loop stream then submits
    args.requests requests with exponential inter-arrival gaps.  Results go
    to pinned host buffers.  Latency = completion - scheduled arrival.  Serial
    plain rendering (one ve_render per request, same outputs) of a bounded
    prefix of the same requests is the comparison."""
    import ctypes
    import queue
    import threading

    import torch

    import ve_b200.dist as vd
    import ve_b200.workloads as wl

    ve = load_package()
    rank, world, local = vd.env_rank()
    dist = vd.init("nccl", timeout_s=900.0, device=local)
    torch.cuda.set_device(local)
    r = ve.Renderer(device=local, hash_log2=22)
    r.set_materials(ve.terrain_materials(1))
    sids, scene_desc = [], []
    for depth, variant, seed in wl.SERVING_SCENES:
        w, nv = ve.terrain_words(depth, variant, seed)
        sids.append(r.upload_scene(w, depth))
        scene_desc.append({"depth": depth, "variant": variant, "voxels": int(nv), "node_words": int(len(w))})
        del w
    reqs = wl.serving_requests(args.requests, seed=5 + rank)
    jobs = []
    for q in reqs:
        cam = ve.camera_ubo(q["eye"], q["dir"], 70.0, q["width"] / q["height"])
        fc = ve.FrameConfig(width=q["width"], height=q["height"], spp=q["spp"], bounces=q["bounces"],
                            frame_index=q["frame"], primary_controlchecks=300, bounce_controlchecks=300, decay=1.0)
        jobs.append((sids[q["scene"]], cam, fc))
    max_px = max(w * h for w, h in wl.BATCH_RESOLUTIONS)
    n_buf = 48
    pool = queue.Queue()
    bufs = []
    for i in range(n_buf):
        hv = torch.empty(max_px, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
        hr = torch.empty(3 * max_px, dtype=torch.float32, pin_memory=True).numpy()
        bufs.append((hv, hr))
        pool.put(i)
    cfg = {"pixel_capacity": 8 * max_px, "path_capacity": 1 << 27, "max_requests": 64,
           "fifo": bool(args.serve_fifo), "step_path_budget": int(args.serve_budget)}
    srv = ve.Server(r, **cfg)
    st0 = srv.stats()

    def serve(order, arrivals):
        """Submits jobs[order[i]] at arrivals[i] (None: as soon as a buffer is
        free); returns per-request records and the wall time."""
        done = []
        inflight = queue.Queue()

        def waiter():
            while True:
                item = inflight.get()
                if item is None:
                    return
                rid, b, t_arr, j = item
                info = srv.wait(rid, timeout_ms=600000)
                pool.put(b)
                done.append((j, t_arr, info))

        th = threading.Thread(target=waiter)
        th.start()
        t0 = time.monotonic()
        s0 = srv.stats()["rays"]
        for i, j in enumerate(order):
            t_arr = None
            if arrivals is not None:
                t_arr = t0 + arrivals[i]
                dt = t_arr - time.monotonic()
                if dt > 0:
                    time.sleep(dt)
            b = pool.get()
            sid, cam, fc = jobs[j]
            hv, hr = bufs[b]
            rid = srv.submit(sid, cam, fc, out_vid=hv, out_rgb=hr)
            inflight.put((rid, b, t_arr, j))
        inflight.put(None)
        th.join()
        wall = time.monotonic() - t0
        return done, wall, srv.stats()["rays"] - s0

    # 1. capacity: closed loop, at most n_buf outstanding
    n_cap = min(len(jobs), args.capacity_requests)
    done, wall, rays = serve(list(range(n_cap)), None)
    capacity_rps = n_cap / wall
    cap_mrays = rays / wall / 1e6
    # 2. Poisson stream at 80% of capacity
    rate = 0.8 * capacity_rps
    rng = np.random.default_rng(99 + rank)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=len(jobs))).tolist()
    with ClockSampler(local) as clk:
        done, wall, rays = serve(list(range(len(jobs))), arrivals)
    lat = [info["done_s"] - t_arr for (_, t_arr, info) in done]
    svc = [info["done_s"] - info["admit_s"] for (_, _, info) in done]
    qwait = [info["admit_s"] - info["submit_s"] for (_, _, info) in done]
    stats = srv.stats()
    srv.close()
    # 3. serial plain rendering of a bounded prefix (ve_render per request)
    lib = ve.load_library()
    hv, hr = bufs[0]
    outs = ve.FrameOutputsC()
    outs.voxel_id = hv.ctypes.data
    outs.rgb = hr.ctypes.data
    r.reset_total_stats()
    t0 = time.monotonic()
    serial_lat = []
    n_serial = 0
    for j in range(len(jobs)):
        if n_serial >= args.serial_requests or time.monotonic() - t0 > args.serial_seconds:
            break
        sid, cam, fc = jobs[j]
        v = ve.Renderer.make_view(sid, cam, fc)
        t1 = time.monotonic()
        rc = lib.ve_render(r._h, ctypes.byref(v), ctypes.byref(outs))
        if rc != 0:
            raise RuntimeError(lib.ve_last_error().decode())
        serial_lat.append(time.monotonic() - t1)
        n_serial += 1
    serial_wall = time.monotonic() - t0
    serial_rays = rays_of(r.total_stats())
    # slowdown: a request's served latency over its latency rendered alone
    # (the serial pass above renders jobs[0..n_serial) one at a time)
    sd = [(info["done_s"] - t_arr) / serial_lat[j] for (j, t_arr, info) in done if j < n_serial]
    slowdown = {"requests": len(sd), "p50": _pct(sd, 50), "p90": _pct(sd, 90), "p99": _pct(sd, 99)} if sd else None
    # latency by request size (paths = pixels x spp)
    by_size = {}
    for name, lo, hi in (("small (< 2^18 paths)", 0, 1 << 18), ("medium", 1 << 18, 1 << 23),
                         ("large (>= 2^23 paths)", 1 << 23, 1 << 62)):
        ls = [info["done_s"] - t_arr for (j, t_arr, info) in done
              if lo <= jobs[j][2].width * jobs[j][2].height * jobs[j][2].spp < hi]
        if ls:
            by_size[name] = {"requests": len(ls), "p50": 1e3 * _pct(ls, 50), "p99": 1e3 * _pct(ls, 99)}
    r.close()
    mrays = rays / wall / 1e6
    line = {"metric": "served p50/p99 latency (Poisson at 80% of capacity) and Mrays/s",
            "value": mrays, "unit": "Mrays/s", "n_gpus": world, "steps": len(jobs), "warmup": n_cap,
            "ms_per_step": 1e3 * wall / len(jobs), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scenes, requests and arrivals)",
            "config": {"workload": "serving: 8 resident octrees depth 8/9/10/11 x2, resolutions "
                                   "{128^2,256^2,640x360,1280x720,1920x1080}, spp 1-16, bounces 1-4, "
                                   f"{len(jobs)} requests, Poisson at 80% of measured capacity",
                       "scenes": scene_desc, "server": cfg,
                       "hbm_budget_bytes": stats["pool_bytes"] + stats["scene_bytes"]},
            "latency_ms": {"p50": 1e3 * _pct(lat, 50), "p90": 1e3 * _pct(lat, 90), "p99": 1e3 * _pct(lat, 99),
                           "max": 1e3 * max(lat)},
            "service_ms": {"p50": 1e3 * _pct(svc, 50), "p99": 1e3 * _pct(svc, 99)},
            "queue_ms": {"p50": 1e3 * _pct(qwait, 50), "p99": 1e3 * _pct(qwait, 99)},
            "capacity": {"requests_per_s": capacity_rps, "mrays_s": cap_mrays, "requests": n_cap},
            "offered_requests_per_s": rate, "achieved_requests_per_s": len(jobs) / wall,
            "max_in_flight": stats["max_in_flight"], "server_steps": stats["steps"],
            "serial_plain": {"requests": n_serial, "mrays_s": serial_rays / serial_wall / 1e6,
                             "requests_per_s": n_serial / serial_wall,
                             "latency_ms_p50": 1e3 * _pct(serial_lat, 50),
                             "latency_ms_p99": 1e3 * _pct(serial_lat, 99)},
            "slowdown": slowdown,
            "latency_ms_by_size": by_size,
            "clocks": clk.summary()}
    lines = [None] * world
    if world > 1:
        import torch.distributed as td
        td.all_gather_object(lines, line)
    else:
        lines = [line]
    if rank == 0:
        if world > 1:
            line["value"] = sum(x["value"] for x in lines)
            line["per_rank_p99_ms"] = [x["latency_ms"]["p99"] for x in lines]
        print(json.dumps(line), flush=True)
    vd.shutdown(dist)
    return 0


class _EqualTime:
    """Image quality at equal device time on the depth-10 scene at 1080p,
    fixed camera: the reference image is a 64-spp plain render (16 frames x
    4 spp through the per-voxel cache, decay 1); each method renders frames
    from a fresh radiance cache until its device time (CUDA events inside the
    library, host copies excluded) reaches the budget, and its last image is
    scored by the relative MSE (img - ref)^2 / (ref^2 + 0.01) over hit pixels."""

    STATS = ("nrc_queries", "nrc_hash_terminated", "paths", "ms_learned", "ms_trace", "ms_shade", "ms_primary",
             "rays_bounce", "rays_shadow", "scheduled_voxels", "scheduled_paths")

    def __init__(self, ve, wl, local):
        W = self.W = wl.LARGE
        self.ve = ve
        words, _ = ve.terrain_words(W.depth, W.variant, W.seed)
        r = self.r = ve.Renderer(device=local, hash_log2=W.hash_log2)
        r.set_materials(ve.terrain_materials(W.seed))
        self.sid = r.upload_scene(words, W.depth)
        eye, d = wl.orbit_camera(0, W.frames, W.seed)
        self.cam = ve.camera_ubo(eye, d, W.fov, W.width / W.height)
        r.cache_reset(self.sid)
        for k in range(15):
            r.render(self.sid, self.cam, self.fc(90000 + k, 4), outputs=())
        ref = r.render(self.sid, self.cam, self.fc(90015, 4), outputs=("voxel_id", "rgb"))
        self.mask = ref["voxel_id"] != 0
        self.refrgb = ref["rgb"]

    def fc(self, frame, spp, flags=0, **kw):
        W = self.W
        return self.ve.FrameConfig(width=W.width, height=W.height, spp=spp, bounces=W.bounces, frame_index=frame,
                                   primary_controlchecks=W.primary_controlchecks,
                                   bounce_controlchecks=W.bounce_controlchecks, decay=1.0, flags=flags, **kw)

    def timed(self, frame, spp, flags, outputs=(), **kw):
        out = self.r.render(self.sid, self.cam, self.fc(frame, spp, flags | self.ve.FRAME_TIMING, **kw),
                            outputs=outputs)
        return out, self.r.stats()["ms_total"]

    def rmse(self, img):
        e = (img - self.refrgb) ** 2 / (self.refrgb ** 2 + 0.01)
        return float(e[self.mask].mean())

    def run(self, flags, budget_ms, max_frames, **kw):
        r = self.r
        # one untimed frame first: the method's kernels load and its buffers
        # are allocated outside the budget
        self.timed(19999, self.W.spp, flags & ~self.ve.FRAME_TRAIN, **kw)
        r.cache_reset(self.sid)
        t = 0.0
        n = 0
        img = None
        stats = {k: 0 for k in self.STATS}
        while n < max_frames:
            out, ms = self.timed(20000 + n, self.W.spp, flags, outputs=("rgb",), **kw)
            if budget_ms is not None and n > 0 and t + ms > budget_ms * 1.0001:
                break
            t += ms
            n += 1
            img = out["rgb"]  # the image after n frames (host copy outside the timed kernels)
            st = r.stats()
            for k in stats:
                stats[k] += st[k]
            if budget_ms is None and n >= max_frames:
                break
        return {"rmse": self.rmse(img), "frames": n, "ms": t, "spp": n * self.W.spp, **stats}


def run_learned(args, rank, world):
    """rMSE at equal time against a 64-spp plain render: the plain method,
    the hashed per-voxel cache ending paths at their second vertex, and the
    learned cache (trained online on 2^16 samples per frame over
    `--train-frames` plain frames, then ending paths at their second vertex,
    falling back to the hashed cache per cell).  The budget is the plain
    method's `--eq-frames` frames."""
    import torch

    import ve_b200.dist as vd
    import ve_b200.workloads as wl

    ve = load_package()
    rank, world, local = vd.env_rank()
    dist = vd.init("nccl", timeout_s=600.0, device=local)
    torch.cuda.set_device(local)
    H = _EqualTime(ve, wl, local)
    W, r = H.W, H.r

    # online training of the learned cache on plain frames
    m = ve.LearnedCache(r, log2_table=19, train_samples=65536, seed=1)
    m.attach(H.sid)
    train_ms = 0.0
    losses = []
    for f in range(args.train_frames):
        _, ms = H.timed(1000 + f, W.spp, ve.FRAME_TRAIN)
        train_ms += ms
        losses.append(m.stats()["loss"])

    plain = H.run(0, None, args.eq_frames)
    budget = plain["ms"]
    hashed = H.run(ve.FRAME_TERMINATE_HASH, budget, 64)
    learned_frozen = H.run(ve.FRAME_LEARNED, budget, 64)
    learned = H.run(ve.FRAME_LEARNED | ve.FRAME_TRAIN, budget, 64)
    line = {"metric": "rMSE at equal time vs 64-spp plain render (learned cache)", "value": learned["rmse"],
            "unit": "relative MSE", "n_gpus": world, "steps": learned["frames"], "warmup": args.train_frames,
            "ms_per_step": learned["ms"] / max(learned["frames"], 1), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "bf16 network / f32 tracer",
            "data": "synthetic (seeded terrain, fixed orbit camera)",
            "config": {"workload": "learned: depth-10 terrain 1920x1080, 4 spp x 3 bounces per frame, "
                                   "64-spp reference (16 x 4 spp through the per-voxel cache), equal device time",
                       "network": "hash grid 16 x 2 fp16 (2^19/level) + oct normal + oct view -> 4 x 64 ReLU -> 3",
                       "train_frames": args.train_frames, "train_samples_per_frame": 65536,
                       "budget_ms": budget},
            "plain": plain, "hash_terminated": hashed, "learned": learned,
            "learned_inference_only": learned_frozen,
            "train_ms_per_frame": train_ms / max(args.train_frames, 1),
            "train_loss_first_last": [losses[0] if losses else None, losses[-1] if losses else None]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    m.close()
    r.close()
    vd.shutdown(dist)
    return 0


def run_scheduled(args, rank, world):
    """Importance-aware voxel scheduling (rank/threshold/emit) against the
    plain per-pixel method at equal device time: rMSE against the 64-spp
    plain render, frames and paths per frame, for the default weights
    (pixels 0.1, variance 0.9, top 30 %, middle 40 %) at two shading budgets
    (131072, the reference's default, and 2 x pixels)."""
    import torch

    import ve_b200.dist as vd
    import ve_b200.workloads as wl

    ve = load_package()
    rank, world, local = vd.env_rank()
    dist = vd.init("nccl", timeout_s=600.0, device=local)
    torch.cuda.set_device(local)
    H = _EqualTime(ve, wl, local)
    W = H.W
    plain = H.run(0, None, args.eq_frames)
    budget = plain["ms"]
    out = {}
    for name, sb in (("budget_131072", 131072), ("budget_2x_pixels", 2 * W.width * W.height)):
        res = H.run(ve.FRAME_SCHEDULED, budget, 4096, shading_budget=sb)
        res["ms_per_frame"] = res["ms"] / max(res["frames"], 1)
        res["paths_per_frame"] = res["paths"] / max(res["frames"], 1)
        out[name] = res
    best = min(out.values(), key=lambda x: x["rmse"])
    line = {"metric": "rMSE at equal time vs 64-spp plain render (importance scheduling)", "value": best["rmse"],
            "unit": "relative MSE", "n_gpus": world, "steps": best["frames"], "warmup": 0,
            "ms_per_step": best["ms_per_frame"], "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded terrain, fixed orbit camera)",
            "config": {"workload": "scheduled: depth-10 terrain 1920x1080, 3 bounces, 64-spp reference, "
                                   "equal device time with the plain method's frames",
                       "plain_frames": args.eq_frames, "budget_ms": budget},
            "plain": plain, **out}
    if rank == 0:
        print(json.dumps(line), flush=True)
    H.r.close()
    vd.shutdown(dist)
    return 0


def run_lbuffer(args, rank, world):
    """The reference's dual-channel lBuffer AccumPass (VE_FRAME_LBUFFER,
    deterministic per-row application) against the FP32 per-voxel cache on
    the depth-10 1080p workload: device time per frame and rMSE against the
    64-spp plain render at equal device time."""
    import torch

    import ve_b200.dist as vd
    import ve_b200.workloads as wl

    ve = load_package()
    rank, world, local = vd.env_rank()
    dist = vd.init("nccl", timeout_s=600.0, device=local)
    torch.cuda.set_device(local)
    H = _EqualTime(ve, wl, local)
    plain = H.run(0, None, args.eq_frames)
    lb = H.run(ve.FRAME_LBUFFER, plain["ms"], 64)
    for res in (plain, lb):
        res["ms_per_frame"] = res["ms"] / max(res["frames"], 1)
    line = {"metric": "ms per frame, lBuffer AccumPass (depth-10 1080p, 4 spp x 3 bounces)",
            "value": lb["ms_per_frame"], "unit": "ms", "n_gpus": world, "steps": lb["frames"], "warmup": 1,
            "ms_per_step": lb["ms_per_frame"], "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 shading / u32 lBuffer", "data": "synthetic (seeded terrain, fixed orbit camera)",
            "config": {"workload": "lbuffer: depth-10 terrain 1920x1080, 4 spp x 3 bounces, caps 16/64, "
                                   "equal device time with the FP32-cache frames", "budget_ms": plain["ms"]},
            "fp32_cache": plain, "lbuffer": lb}
    if rank == 0:
        print(json.dumps(line), flush=True)
    H.r.close()
    vd.shutdown(dist)
    return 0


def run_emissive(args, rank, world):
    """The reference's Cornell box (depth 8, light panel of 65,536 emissive
    voxels, camera of its demo) at 1920x1080, 1 spp x 3 bounces, with
    VE_FRAME_EMISSIVE: throughput of ReSTIR-DI frames and of single-pick RIS
    frames, and rMSE against a 256-spp RIS reference (64 frames x 4 spp
    through the per-voxel cache, decay 1) at equal device time."""
    import torch

    import ve_b200.dist as vd
    import ve_b200.workloads as wl

    ve = load_package()
    rank, world, local = vd.env_rank()
    dist = vd.init("nccl", timeout_s=600.0, device=local)
    torch.cuda.set_device(local)
    C = wl.CORNELL
    cpu = ve.OctreeCPU(C.depth)
    wl.cornell_build(cpu, C.depth)
    oc = ve.Octree(C.depth)
    oc.set(cpu)
    r = ve.Renderer(device=local, hash_log2=C.hash_log2)
    r.set_materials(wl.cornell_materials())
    sid = r.upload_scene(oc.words(), C.depth)
    W, H = 1920, 1080
    eye, d = wl.cornell_camera(C.depth)
    cam = ve.camera_ubo(eye, d, C.fov, W / H)

    def fc(frame, spp, restir, timing=True):
        return ve.FrameConfig(width=W, height=H, spp=spp, bounces=C.bounces, frame_index=frame,
                              primary_controlchecks=C.primary_controlchecks,
                              bounce_controlchecks=C.bounce_controlchecks, sky=(0.05, 0.05, 0.05), decay=1.0,
                              flags=ve.FRAME_EMISSIVE | (ve.FRAME_TIMING if timing else 0), restir=restir)

    # reference: 64 frames x 4 spp of the single-pick estimator
    r.cache_reset(sid)
    for k in range(63):
        r.render(sid, cam, fc(50000 + k, 4, 0, False), outputs=())
    ref = r.render(sid, cam, fc(50063, 4, 0, False), outputs=("voxel_id", "rgb"))
    mask = ref["voxel_id"] != 0
    refrgb = ref["rgb"]

    def rmse(img):
        e = (img - refrgb) ** 2 / (refrgb ** 2 + 0.01)
        return float(e[mask].mean())

    def run(restir, budget_ms, max_frames):
        r.render(sid, cam, fc(59999, 1, restir), outputs=())  # kernels loaded, buffers allocated
        r.cache_reset(sid)
        t, n, rays, img = 0.0, 0, 0, None
        while n < max_frames:
            out = r.render(sid, cam, fc(60000 + n, 1, restir), outputs=("rgb",))
            st = r.stats()
            if budget_ms is not None and n > 0 and t + st["ms_total"] > budget_ms * 1.0001:
                break
            t += st["ms_total"]
            n += 1
            rays += st["rays_primary"] + st["rays_bounce"] + st["rays_shadow"]
            img = out["rgb"]
        return {"rmse": rmse(img), "frames": n, "ms": t, "ms_per_frame": t / max(n, 1),
                "mrays_s": rays / max(t, 1e-9) / 1e3, "lights": st["emissive_lights"],
                "nee_per_frame": st["nee_emissive"], "reservoirs_per_frame": st["restir_commits"]}

    restir = run(ve.RESTIR_ENABLE | ve.RESTIR_TEMPORAL | ve.RESTIR_SPATIAL, None, args.eq_frames * 4)
    ris = run(0, restir["ms"], 256)
    line = {"metric": "rMSE at equal time vs 256-spp render (Cornell box, emissive NEE)", "value": restir["rmse"],
            "unit": "relative MSE", "n_gpus": world, "steps": restir["frames"], "warmup": 1,
            "ms_per_step": restir["ms_per_frame"], "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "the reference's Cornell box scene (voxelengine.cpp:82-142)",
            "config": {"workload": "emissive: Cornell box depth 8 at 1920x1080, 1 spp x 3 bounces, "
                                   "256-spp single-pick RIS reference, equal device time",
                       "budget_ms": restir["ms"]},
            "restir_di": restir, "single_pick_ris": ris}
    if rank == 0:
        print(json.dumps(line), flush=True)
    r.close()
    vd.shutdown(dist)
    return 0


def run_build(args, rank, world):
    """GPU bulk octree build (voxel list -> Octree::set words on the device)
    against the host paths: OctreeCPU.insert + Octree.set (the reference's
    algorithm, restated) on a bounded depth, and the terrain bulk builder.
    Seconds per build; the words of every path are compared."""
    import torch

    import ve_b200.dist as vd
    import ve_b200.workloads as wl

    ve = load_package()
    rank, world, local = vd.env_rank()
    torch.cuda.set_device(local)
    W = wl.LARGE
    r = ve.Renderer(device=local, hash_log2=12)
    out = {}
    for depth in (8, W.depth):
        vox = ve.terrain_voxels(depth, W.variant, W.seed)
        words, _ = ve.terrain_words(depth, W.variant, W.seed)
        sid = r.build_scene(vox, depth, keep_normals=True)  # warm-up (module load, first allocations)
        r.release_scene(sid)
        ts = []
        for _ in range(max(args.steps, 3)):
            t0 = time.perf_counter()
            sid = r.build_scene(vox, depth, keep_normals=True)
            ts.append(time.perf_counter() - t0)
            got = r.download_scene(sid) if not ts[1:] else None
            r.release_scene(sid)
            if got is not None:
                assert np.array_equal(got, words), "GPU build differs from the bulk builder"
        t0 = time.perf_counter()
        ve.terrain_words(depth, W.variant, W.seed)
        t_bulk = time.perf_counter() - t0
        rec = {"voxels": int(len(vox)), "words": int(words.size), "gpu_build_s": statistics.median(ts),
               "host_bulk_builder_s": t_bulk}
        if depth <= 8:
            t0 = time.perf_counter()
            cpu = ve.OctreeCPU(depth)
            cpu.insert_many(vox)
            tree = ve.Octree(depth)
            tree.set(cpu)
            rec["host_octree_cpu_set_s"] = time.perf_counter() - t0
            assert np.array_equal(tree.words()[: tree.size], words)
        out[f"depth{depth}"] = rec
    r.close()
    big = out[f"depth{W.depth}"]
    line = {"metric": "GPU octree build, Mvoxels/s (voxel list -> Octree::set words)",
            "value": big["voxels"] / big["gpu_build_s"] / 1e6, "unit": "Mvoxels/s", "n_gpus": 1,
            "steps": max(args.steps, 3), "warmup": 1, "ms_per_step": 1e3 * big["gpu_build_s"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded terrain voxel lists)",
            "config": {"workload": "build: depth-8 and depth-10 terrain + overhangs, host voxel list in, "
                                   "device words out (host copy of the list included)"},
            "builds": out}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def run_split(args, rank, world):
    """Split frames: each 1080p frame of the large workload rendered by every
    rank on its band of rows, one all-gather of the frame's cache records
    (NCCL), the rank-order merge and the band's AvgPass (strong scaling: the
    frame is fixed as N grows).  At N=1 the band is the whole frame and the
    line measures the split path's overhead over the plain frame."""
    import torch

    import ve_b200.dist as vd
    import ve_b200.workloads as wl

    ve = load_package()
    rank, world, local = vd.env_rank()
    dist = vd.init("nccl", timeout_s=300.0, device=local)
    torch.cuda.set_device(local)
    W = wl.LARGE
    words, nv = ve.terrain_words(W.depth, W.variant, W.seed)
    r = ve.Renderer(device=local, hash_log2=W.hash_log2)
    r.set_materials(ve.terrain_materials(W.seed))
    sid = r.upload_scene(words, W.depth)
    stream = torch.cuda.ExternalStream(r.stream, device=local)
    sf = vd.SplitFrame(r, sid, dist, device=f"cuda:{local}")
    dev = f"cuda:{local}"

    def cam(i):
        eye, d = wl.orbit_camera(i % W.frames, W.frames, W.seed)
        return ve.camera_ubo(eye, d, W.fov, W.width / W.height)

    K, Wm = args.steps, args.warmup
    for i in range(Wm):
        sf.render(cam(i), frame_config(ve, W, i), outputs=(), gather=False)

    def timed(outputs, gather):
        r.reset_total_stats()
        torch.cuda.synchronize(local)
        vd.barrier(dist)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        records = 0
        e0.record(stream)
        for i in range(K):
            sf.render(cam(Wm + i), frame_config(ve, W, Wm + i), outputs=outputs, gather=gather)
            records += sum(sf.last["counts"])
        e1.record(stream)
        e1.synchronize()
        ms = vd.max_over_ranks(e0.elapsed_time(e1), dist, dev)
        tot = r.total_stats()
        rays = vd.sum_over_ranks(rays_of(tot), dist, dev)
        return ms, rays, tot, records

    with ClockSampler(local) as clk:
        ms, rays, tot, records = timed((), False)
    value = rays / (ms / 1e3) / 1e6
    sf.render(cam(Wm), frame_config(ve, W, Wm), outputs=("rgb",), gather=True)  # allocates the pinned images
    e_ms, e_rays, etot, _ = timed(("rgb",), True)
    e2e_value = e_rays / (e_ms / 1e3) / 1e6
    if rank == 0:
        line = {"metric": METRIC + " (split frames)", "value": value, "unit": "Mrays/s", "n_gpus": world,
                "steps": K, "warmup": Wm, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded value-noise terrain, seeded orbit camera)",
                "config": {"workload": "split: large (depth-10, 1920x1080, 4 spp x 3 bounces) frames split into "
                                       f"{world} bands of rows", "parallelism": f"row bands x{world}",
                           "records_per_step": records / K,
                           "exchange_bytes_per_step": 32.0 * records / K,
                           "l2": "inputs larger than L2 (310 MB node array)"},
                "e2e": {"value": e2e_value, "unit": "Mrays/s",
                        "h2d_bytes_per_step": (etot["h2d_bytes"] + 0.0) / K,
                        "d2h_bytes_per_step": 12.0 * W.width * W.height},
                "gpu_launches": int(tot["kernel_launches"]) + (2 + world) * K,
                "clocks": clk.summary()}
        print(json.dumps(line), flush=True)
    r.close()
    vd.shutdown(dist)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=64)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-pipeline", action="store_true", help="large, batching: render the frames unpipelined")
    ap.add_argument("--workload", choices=["large", "batching", "serving", "learned", "scheduled", "emissive", "lbuffer", "build",
                                                  "split"], default="large")
    ap.add_argument("--train-frames", type=int, default=48, help="learned: online training frames")
    ap.add_argument("--eq-frames", type=int, default=4, help="learned, scheduled: plain frames setting the time budget")
    ap.add_argument("--requests", type=int, default=10000, help="serving: requests in the Poisson stream")
    ap.add_argument("--capacity-requests", type=int, default=400, help="serving: closed-loop capacity sample")
    ap.add_argument("--serial-requests", type=int, default=400, help="serving: serial plain comparison sample")
    ap.add_argument("--serial-seconds", type=float, default=20.0)
    ap.add_argument("--serve-budget", type=int, default=0,
                    help="serving: primary paths a step may start (0: the server's default, 2^23)")
    ap.add_argument("--serve-fifo", action="store_true",
                    help="serving: strict first-come-first-served admission, whole primary passes per step")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return run_reference(args, rank, world)
    ve = load_package()
    import ve_b200.workloads as wl

    W = wl.LARGE
    if args.workload == "batching":
        return run_batching(args, rank, world)
    if args.workload == "serving":
        return run_serving(args, rank, world)
    if args.workload == "learned":
        return run_learned(args, rank, world)
    if args.workload == "scheduled":
        return run_scheduled(args, rank, world)
    if args.workload == "emissive":
        return run_emissive(args, rank, world)
    if args.workload == "lbuffer":
        return run_lbuffer(args, rank, world)
    if args.workload == "build":
        return run_build(args, rank, world)
    if args.workload == "split":
        return run_split(args, rank, world)

    import torch

    import ve_b200.dist as vd

    dist = vd.init("nccl", timeout_s=300.0, device=local)
    torch.cuda.set_device(local)
    torch.cuda.init()

    words, nv = ve.terrain_words(W.depth, W.variant, W.seed)
    mats = ve.terrain_materials(W.seed)
    # frames pipelined over two frame sets (VE_CFG_PIPELINE): the timing,
    # fetch-counting and stage-breakdown frames run unpipelined by design
    r = ve.Renderer(device=local, hash_log2=W.hash_log2, pipeline=not args.no_pipeline)
    r.set_materials(mats)
    sid = r.upload_scene(words, W.depth)
    stream = torch.cuda.ExternalStream(r.stream, device=local)

    plan = vd.frame_assignment(args.warmup + args.steps, rank, world, W.frames)  # replicas

    def frame(i):
        return plan[i]

    def cams(i):
        eye, d = wl.orbit_camera(frame(i), W.frames, W.seed)
        return ve.camera_ubo(eye, d, W.fov, W.width / W.height)

    K, Wm = args.steps, args.warmup
    cam_list = [cams(Wm + i) for i in range(K)]
    dev = f"cuda:{local}"

    def barrier():
        torch.cuda.synchronize(local)
        r.synchronize()
        vd.barrier(dist)

    def max_over_ranks(x):
        return vd.max_over_ranks(x, dist, dev)

    def sum_over_ranks(x):
        return vd.sum_over_ranks(x, dist, dev)

    # warm-up
    for i in range(Wm):
        r.render(sid, cams(i), frame_config(ve, W, frame(i)), outputs=())
    r.synchronize()

    # ---- timed region: device-resident frames (frame-graph replays) --------
    r.reset_total_stats()
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for i in range(K):
            r.render(sid, cam_list[i], frame_config(ve, W, frame(Wm + i)), outputs=())
        r.join()  # the end event follows the frames on the second frame set's stream too
        e1.record(stream)
        e1.synchronize()
    ms = e0.elapsed_time(e1)
    tot = r.total_stats()
    ms_max = max_over_ranks(ms)
    rays_all = sum_over_ranks(rays_of(tot))
    value = rays_all / (ms_max / 1e3) / 1e6

    # ---- stage breakdown: the same frames with per-pass CUDA events ---------
    # (FRAME_TIMING enqueues the kernels directly, between events, instead of
    # replaying the frame graph)
    r.reset_total_stats()
    for i in range(K):
        r.render(sid, cam_list[i], frame_config(ve, W, frame(Wm + i), ve.FRAME_TIMING), outputs=())
    r.synchronize()
    ttot = r.total_stats()

    # ---- algorithmic bytes of the same frames (node-word fetch counts) -----
    r.reset_total_stats()
    for i in range(K):
        r.render(sid, cam_list[i], frame_config(ve, W, frame(Wm + i), ve.FRAME_COUNT_FETCH), outputs=())
    cnt = r.total_stats()
    trace_rays = cnt["rays_bounce"] + cnt["rays_shadow"] - cnt["shadow_shared"]  # traversals the kernel ran
    trace_bytes = 4.0 * cnt["fetch_nodes_trace"] + 48.0 * trace_rays
    trace_ms = ttot["ms_trace"]
    launches = ttot["trace_launches"]
    achieved = trace_bytes / (trace_ms / 1e3) / 1e9 if trace_ms > 0 else None
    peak, peak_kind = peaks()
    traffic, traffic_src = measured_trace_traffic()

    # ---- e2e: public API, host outputs, view upload each step --------------
    # each frame's result is its displayed image — the RGBA8 framebuffer
    # final.frag writes (the mapped8 output) — copied on the renderer's copy
    # stream while the next frame renders (VE_FRAME_ASYNC_OUTPUTS), into two
    # alternating pinned images; every frame's image reaches host memory
    # inside the timed region
    sets = []
    for _ in range(2):
        himg = torch.empty((W.height, W.width, 4), dtype=torch.uint8, pin_memory=True).numpy()
        o = ve.FrameOutputsC()
        o.mapped8 = himg.ctypes.data
        sets.append((o, himg))
    lib = ve.load_library()
    import ctypes

    views = [ve.Renderer.make_view(sid, cam_list[i], frame_config(ve, W, frame(Wm + i), ve.FRAME_ASYNC_OUTPUTS))
             for i in range(K)]
    # warm-up of this path: its frame graphs (one per output image set) are
    # captured here, not in the timed region
    for i in range(Wm):
        wv = ve.Renderer.make_view(sid, cams(i), frame_config(ve, W, frame(i), ve.FRAME_ASYNC_OUTPUTS))
        rc = lib.ve_render(r._h, ctypes.byref(wv), ctypes.byref(sets[i & 1][0]))
        if rc != 0:
            raise RuntimeError(lib.ve_last_error().decode())
    r.synchronize()
    r.reset_total_stats()
    barrier()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for i in range(K):
        rc = lib.ve_render(r._h, ctypes.byref(views[i]), ctypes.byref(sets[i & 1][0]))
        if rc != 0:
            raise RuntimeError(lib.ve_last_error().decode())
    r.synchronize()  # the last frame's copies
    f1.record(stream)
    f1.synchronize()
    e2e_ms = max_over_ranks(f0.elapsed_time(f1))
    etot = r.total_stats()
    e2e_value = sum_over_ranks(rays_of(etot)) / (e2e_ms / 1e3) / 1e6

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        dev_words = r.download_scene(sid)
        cpu = cpu_baseline(ve, W, dev_words, mats, args.cpu_seconds)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": K, "warmup": Wm,
            "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded value-noise terrain, seeded orbit camera)",
            "config": large_config(nv, words.size),
            "rays_per_step": rays_of(tot) / K,
            "ray_mix_per_step": {k: tot[k] / K for k in ("rays_primary", "rays_bounce", "rays_shadow")},
            # rays_shadow counts every path's sun shadow ray; the samples of a
            # pixel share their first one (same origin and direction), traced once
            "shadow_rays_shared_per_step": tot["shadow_shared"] / K,
            "traced_rays_per_step": (rays_of(tot) - tot["shadow_shared"]) / K,
            "e2e": {"value": e2e_value, "unit": "Mrays/s", "h2d_bytes_per_step": etot["h2d_bytes"] / K,
                    "d2h_bytes_per_step": etot["d2h_bytes"] / K,
                    "outputs": "the displayed RGBA8 image (final.frag's framebuffer store), pinned host memory"},
            "roofline": {"bound": "hbm", "kernel": "k_trace (bounce + shadow DDA)", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": (achieved / peak) if achieved else None,
                         "peak_kind": peak_kind, "traffic": traffic, "traffic_source": traffic_src,
                         "algorithmic_bytes_per_launch": trace_bytes / max(launches, 1),
                         "ms_per_launch": trace_ms / max(launches, 1),
                         "l2": trace_l2_roofline(trace_ms / max(launches, 1))},
            "gpu_launches": int(tot["kernel_launches"]),
            "frame_pipeline": not args.no_pipeline,
            "stage_ms_per_step": {k: ttot[k] / K for k in ("ms_primary", "ms_trace", "ms_shade", "ms_resolve",
                                                            "ms_decay")},
            "stage_ms_note": "per-pass CUDA events over the same K frames run with direct launches",
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    r.close()
    vd.shutdown(dist)
    return 0


if __name__ == "__main__":
    sys.exit(main())
