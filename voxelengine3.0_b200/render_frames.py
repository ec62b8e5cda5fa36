"""Renders frames of the depth-10 orbit workload at a chosen size and prints
their device counters and stage times as JSON lines.

    python voxelengine3.0_b200/render_frames.py [--width 960] [--height 540]
        [--spp 1] [--bounces 3] [--frames 2] [--depth 10] [--count] [--learned N]

Used for profiling a reduced case of the benchmark kernels (same scene, fewer
pixels) and for quick throughput checks.
"""
import argparse
import importlib.util
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def _package():
    if "ve_b200" in sys.modules:
        return sys.modules["ve_b200"]
    spec = importlib.util.spec_from_file_location("ve_b200", os.path.join(HERE, "__init__.py"),
                                                  submodule_search_locations=[HERE])
    m = importlib.util.module_from_spec(spec)
    sys.modules["ve_b200"] = m
    spec.loader.exec_module(m)
    return m


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--width", type=int, default=960)
    ap.add_argument("--height", type=int, default=540)
    ap.add_argument("--spp", type=int, default=1)
    ap.add_argument("--bounces", type=int, default=3)
    ap.add_argument("--frames", type=int, default=2)
    ap.add_argument("--depth", type=int, default=10)
    ap.add_argument("--count", action="store_true", help="count node fetches (VE_FRAME_COUNT_FETCH)")
    ap.add_argument("--learned", type=int, default=-1,
                    help="attach a learned radiance cache, train it on N frames, then render learned + training frames")
    args = ap.parse_args()
    ve = _package()
    import ve_b200.workloads as wl

    W = wl.LARGE
    words, nv = ve.terrain_words(args.depth, W.variant, W.seed)
    with ve.Renderer(hash_log2=W.hash_log2) as r:
        r.set_materials(ve.terrain_materials(W.seed))
        sid = r.upload_scene(words, args.depth)
        scale = (1 << args.depth) / 1024.0
        extra = 0
        if args.learned >= 0:
            m = ve.LearnedCache(r, log2_table=19, seed=1)
            m.attach(sid)
            eye, d = wl.orbit_camera(0, W.frames, W.seed, radius=600.0 * scale, height=300.0 * scale)
            cam = ve.camera_ubo(eye, d, W.fov, args.width / args.height)
            for f in range(args.learned):
                fc = ve.FrameConfig(width=args.width, height=args.height, spp=args.spp, bounces=args.bounces,
                                    frame_index=1000 + f, primary_controlchecks=W.primary_controlchecks,
                                    bounce_controlchecks=W.bounce_controlchecks, flags=ve.FRAME_TRAIN)
                r.render(sid, cam, fc, outputs=())
            extra = ve.FRAME_LEARNED | ve.FRAME_TRAIN
        for f in range(args.frames):
            eye, d = wl.orbit_camera(f, W.frames, W.seed, radius=600.0 * scale, height=300.0 * scale)
            cam = ve.camera_ubo(eye, d, W.fov, args.width / args.height)
            fc = ve.FrameConfig(width=args.width, height=args.height, spp=args.spp, bounces=args.bounces,
                                frame_index=f, primary_controlchecks=W.primary_controlchecks,
                                bounce_controlchecks=W.bounce_controlchecks,
                                flags=ve.FRAME_TIMING | (ve.FRAME_COUNT_FETCH if args.count else 0) | extra)
            r.render(sid, cam, fc, outputs=())
            st = r.stats()
            print(json.dumps({k: (round(v, 4) if isinstance(v, float) else v) for k, v in st.items()}), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
