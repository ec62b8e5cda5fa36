"""The oracle against the committed golden fixtures (tests/golden/): outputs
of the reference's own compiled octree code, and the oracle's own seeded
vectors; plus independent numpy restatements of the RNG, voxel key and
sin/cos polynomial."""
import os

import numpy as np
import pytest

import helpers

GOLDEN = os.path.join(helpers.ROOT, "tests", "golden")


@pytest.fixture(scope="module")
def refdata():
    return np.load(os.path.join(GOLDEN, "reference_octree.npz"))


@pytest.fixture(scope="module")
def orcdata():
    return np.load(os.path.join(GOLDEN, "oracle_vectors.npz"))


def tree_ids(d):
    return sorted({k.split("_")[0] for k in d.files})


def test_oracle_build_matches_reference_fixture(oracle, refdata):
    for t in tree_ids(refdata):
        depth = int(refdata[f"{t}_depth"])
        words = oracle.build(depth, refdata[f"{t}_voxels"])
        assert np.array_equal(words, refdata[f"{t}_words"]), t


def test_product_octree_matches_reference_fixture(ve, refdata):
    for t in tree_ids(refdata):
        depth = int(refdata[f"{t}_depth"])
        c = ve.OctreeCPU(depth)
        c.insert_many(refdata[f"{t}_voxels"])
        o = ve.Octree(depth)
        o.set(c)
        assert np.array_equal(o.words()[: o.size], refdata[f"{t}_words"]), t
        assert o.num_voxels == int(refdata[f"{t}_numvoxels"])
        for q, slot, lk in zip(refdata[f"{t}_query"], refdata[f"{t}_slot"], refdata[f"{t}_lookup"]):
            assert o.find_gpu_slot(c, q) == slot
            assert c.lookup(*map(int, q)) == lk


def test_oracle_dda_matches_reference_raycast_fixture(oracle, refdata):
    """Hit positions of the restated GLSL DDA equal the reference's
    OctreeCPU::raycast on rays that do not time out."""
    n = 0
    for t in tree_ids(refdata):
        depth = int(refdata[f"{t}_depth"])
        words = refdata[f"{t}_words"]
        for o, d, h in zip(refdata[f"{t}_ray_o"], refdata[f"{t}_ray_d"], refdata[f"{t}_ray_hit"]):
            res, _ = oracle.raycast(words, depth, o, d, 100000)
            assert res[0] != 2
            if h[0]:
                assert res[0] == 0 and tuple(res[3:6]) == tuple(h[1:4])
                n += 1
            else:
                assert res[0] != 0
    assert n > 20


def test_oracle_vectors(oracle, orcdata):
    for s, vals in zip(orcdata["rng_states"], orcdata["rng_values"]):
        got, _ = oracle.rand_seq(int(s), vals.size)
        assert np.array_equal(got.view(np.uint32), vals.view(np.uint32))
    for p, k in zip(orcdata["key_pos"], orcdata["key_val"]):
        assert oracle.voxel_key(*map(int, p)) == k
    s, c = oracle.sincos_turn(orcdata["sincos_u"])
    assert np.array_equal(s, orcdata["sincos_s"]) and np.array_equal(c, orcdata["sincos_c"])
    for w, d, n in zip(orcdata["normal_words"], orcdata["normal_dirs"], orcdata["normal_vals"]):
        assert np.array_equal(oracle.shading_normal(int(w), d), n)
    depth = int(orcdata["scene_depth"])
    words = orcdata["scene_words"]
    for o, d, out in zip(orcdata["dda_o"], orcdata["dda_d"], orcdata["dda_out"]):
        assert np.array_equal(oracle.raycast(words, depth, o, d, 40)[0], out)


def test_oracle_small_render_fixture(oracle, orcdata):
    from oracle.oracle import OracleRenderer, frame_params

    class FC:
        width, height, spp, bounces = 20, 16, 2, 3
        primary_controlchecks, bounce_controlchecks, reconstruction_radius = 40, 60, 2
        render_type, frame_index, flags = 0, 3, 0
        sun_dir = (0.27524094, 0.9174698, 0.18349396)
        sun_intensity, sky, decay, variance_norm = 3.14159265, (0.4, 0.4, 0.4), 0.95, 10000.0

    r = OracleRenderer(oracle)
    depth = int(orcdata["scene_depth"])
    outs = [r.render(orcdata["scene_words"], depth, orcdata["materials"], orcdata["camera"], frame_params(FC),
                     threads=3, want_path_rgb=True) for _ in range(2)]
    assert np.array_equal(outs[-1]["gbuffer"], orcdata["render_gbuf"])
    assert np.array_equal(outs[-1]["path_rgb"], orcdata["render_path_rgb"])
    assert np.allclose(outs[-1]["rgb"], orcdata["render_rgb"], rtol=1e-6, atol=1e-7)
    assert (orcdata["render_gbuf"][..., 3] != 0).any()


# --- independent numpy restatements (second transcription of the GLSL) ----
BASES = [2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53]


def np_rand(state, n):
    out = []
    for _ in range(n):
        dim = state & 0xFF
        idx = state >> 8
        state = ((idx << 8) | ((dim + 1) & 0xFF)) & 0xFFFFFFFF
        i = idx ^ (((dim >> 4) * 0x9E3779B9) & 0xFFFFFFFF)
        b = BASES[dim & 15]
        f = np.float32(1.0)
        r = np.float32(0.0)
        k = 0
        while k < 24 and i > 0:
            f = np.float32(f / np.float32(b))
            q = i // b
            r = np.float32(r + np.float32(f * np.float32(i - q * b)))
            i = q
            k += 1
        out.append(r)
    return np.array(out, np.float32)


def np_key(x, y, z):
    v = (x | (y << 10) | (z << 20)) & 0xFFFFFFFF
    v ^= v >> 16
    v = (v * 0x7FEB352D) & 0xFFFFFFFF
    v ^= v >> 15
    v = (v * 0x846CA68B) & 0xFFFFFFFF
    v ^= v >> 16
    return v & 0x7FFFFFFF


def test_rng_and_key_second_transcription(oracle, orcdata):
    for s, vals in zip(orcdata["rng_states"], orcdata["rng_values"]):
        assert np.array_equal(np_rand(int(s), vals.size), vals)
    for p, k in zip(orcdata["key_pos"], orcdata["key_val"]):
        assert np_key(*map(int, p)) == k


def test_sincos_polynomial_accuracy(oracle):
    u = np.linspace(0, 1, 100001, dtype=np.float32)
    s, c = oracle.sincos_turn(u)
    ang = 2 * np.pi * u.astype(np.float64)
    assert np.abs(s - np.sin(ang)).max() < 3e-7
    assert np.abs(c - np.cos(ang)).max() < 3e-7
