"""Generates the committed golden fixtures of tests/golden/.

    python tests/golden/make_golden.py

* ``reference_octree.npz`` — outputs of the reference's OWN compiled octree
  code (src/octree_cpu.cpp + src/renderer/octree.cpp, built in place into
  oracle/_ref by oracle/build_ref.sh): node words of Octree::set for seeded
  trees, findGpuSlot / lookup samples, OctreeCPU::raycast hits.  Needs the
  reference tree; the tests then need only the fixture.
* ``oracle_vectors.npz`` — the CPU oracle's restatement of the GLSL passes
  on seeded inputs (RNG sequences, voxel keys, sin/cos polynomial, shading
  normals, DDA results, a small rendered frame).  The GLSL cannot execute
  here, so these pin the oracle against regressions rather than against the
  reference.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle.oracle import Oracle, OracleRenderer, Reference, build_ref, frame_params  # noqa: E402


def trees():
    """Seeded voxel sets: (depth, xyzm)."""
    rng = np.random.default_rng(20240611)
    out = []
    for depth, dens in [(2, 0.4), (3, 0.15), (4, 0.05), (5, 0.02)]:
        L = 1 << depth
        n = max(1, int(L ** 3 * dens))
        v = np.zeros((n, 4), np.uint32)
        v[:, :3] = rng.integers(0, L, (n, 3))
        v[:, 3] = rng.integers(1, 128, n)
        out.append((depth, v))
    return out


def make_reference(path):
    build_ref()
    ref = Reference()
    rng = np.random.default_rng(7)
    data = {}
    for i, (depth, v) in enumerate(trees()):
        s = ref.scene(depth)
        s.insert_many(v)
        words, size, nv = s.set()
        data[f"t{i}_depth"] = np.array(depth)
        data[f"t{i}_voxels"] = v
        data[f"t{i}_words"] = words[:size]
        data[f"t{i}_numvoxels"] = np.array(nv)
        L = 1 << depth
        q = rng.integers(0, L, (64, 3)).astype(np.uint32)
        data[f"t{i}_query"] = q
        data[f"t{i}_slot"] = np.array([s.find_gpu_slot(*map(int, p)) for p in q], np.uint32)
        data[f"t{i}_lookup"] = np.array([s.lookup(*map(int, p)) for p in q], np.int64)
        o = rng.uniform(-0.5 * L, 1.5 * L, (64, 3)).astype(np.float32)
        d = rng.normal(size=(64, 3))
        d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
        hits = []
        for a, b in zip(o, d):
            h, p = s.raycast(a, b, 100000)
            hits.append([int(h)] + (list(p) if h else [0, 0, 0]))
        data[f"t{i}_ray_o"] = o
        data[f"t{i}_ray_d"] = d
        data[f"t{i}_ray_hit"] = np.array(hits, np.uint32)
    np.savez_compressed(path, **data)


def make_oracle(path):
    orc = Oracle()
    rng = np.random.default_rng(99)
    data = {}
    states = np.array([0, 0x100, 0xDEADBE00, 0xFFFFFF00, 12345 << 8, 0x9E3779B9 & 0xFFFFFF00], np.uint32)
    data["rng_states"] = states
    data["rng_values"] = np.stack([orc.rand_seq(int(s), 40)[0] for s in states])
    pos = rng.integers(0, 2048, (256, 3)).astype(np.uint32)
    data["key_pos"] = pos
    data["key_val"] = np.array([orc.voxel_key(*map(int, p)) for p in pos], np.uint32)
    u = np.concatenate([np.linspace(0, 1, 257, dtype=np.float32), rng.random(256).astype(np.float32)])
    s, c = orc.sincos_turn(u)
    data["sincos_u"], data["sincos_s"], data["sincos_c"] = u, s, c
    words = []
    for _ in range(256):
        ix, iy, iz = (int(t) for t in rng.integers(-9, 10, 3))
        words.append(((ix & 31) << 8) | ((iy & 31) << 13) | ((iz & 31) << 18) | (1 << 31) | (3 << 1))
    words.append(3 << 1)  # no stored normal -> face fallback
    data["normal_words"] = np.array(words, np.uint32)
    dirs = rng.normal(size=(len(words), 3)).astype(np.float32)
    data["normal_dirs"] = dirs
    data["normal_vals"] = np.stack([orc.shading_normal(int(w), d) for w, d in zip(words, dirs)])
    # DDA + tiny render on the depth-5 seeded tree, normals filled by the oracle
    depth, v = trees()[3]
    w = orc.fill_normals(orc.build(depth, v), depth)
    data["scene_depth"] = np.array(depth)
    data["scene_words"] = w
    L = 1 << depth
    o = rng.uniform(-0.5 * L, 1.5 * L, (128, 3)).astype(np.float32)
    d = rng.normal(size=(128, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    res = np.stack([orc.raycast(w, depth, a, b, 40)[0] for a, b in zip(o, d)])
    data["dda_o"], data["dda_d"], data["dda_out"] = o, d, res
    mats = np.zeros((128, 16), np.float32)
    mats[1:128, :3] = rng.uniform(0.2, 0.9, (127, 3))
    mats[1:128, 8] = 1.0
    mats[5, 10] = 0.9  # one metallic material (GGX lobe: metallic*(1-roughness) > 0.5)
    mats[5, 8] = 0.2
    mats[5, 9] = 0.5
    data["materials"] = mats
    eye = np.array([L * 0.5, L * 1.3, -L * 0.6], np.float32)
    dd = np.array([0.0, -0.6, 1.0])
    dd = (dd / np.linalg.norm(dd)).astype(np.float32)
    cam = orc.camera_ubo(eye, dd, 70.0, 1.25)
    data["camera"] = cam

    class FC:
        width, height, spp, bounces = 20, 16, 2, 3
        primary_controlchecks, bounce_controlchecks, reconstruction_radius = 40, 60, 2
        render_type, frame_index, flags = 0, 3, 0
        sun_dir = (0.27524094, 0.9174698, 0.18349396)
        sun_intensity, sky, decay, variance_norm = 3.14159265, (0.4, 0.4, 0.4), 0.95, 10000.0

    r = OracleRenderer(orc)
    outs = [r.render(w, depth, mats, cam, frame_params(FC), threads=1, want_path_rgb=True) for _ in range(2)]
    data["render_gbuf"] = outs[-1]["gbuffer"]
    data["render_path_rgb"] = outs[-1]["path_rgb"]
    data["render_rgb"] = outs[-1]["rgb"]
    np.savez_compressed(path, **data)


if __name__ == "__main__":
    make_reference(os.path.join(HERE, "reference_octree.npz"))
    make_oracle(os.path.join(HERE, "oracle_vectors.npz"))
    print("wrote", os.listdir(HERE))
