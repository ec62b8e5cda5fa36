"""The allocation-free leaf-normal entry point (ve_fill_normals_noalloc).

Some callers may not call cudaMalloc — hosts that own the whole device-memory
budget and forbid libraries from allocating, or latency-critical threads that
cannot take the stall of an allocation.  For them the library offers a variant
of the normal pass whose scratch is a fixed device array inside the library.
This checks, through the C ABI, that two calls in a row give exactly the
normals the regular upload path (ve_scene_upload, which allocates its scratch)
produces, and that scenes beyond the array's limit are refused.

The file sorts last so that a run stopping at the first failure has already
run every other test.
"""
import ctypes

import numpy as np
import pytest

import helpers

pytestmark = pytest.mark.gpu


def upload_path_normals(ve, words, depth):
    with ve.Renderer(hash_log2=8) as r:
        sid = r.upload_scene(words, depth)
        return r.download_scene(sid)


def noalloc_normals(ve, words, depth, stream=None):
    """Runs the entry point on `stream` (a torch.cuda.Stream; None = the
    legacy default stream) and reads the node array back."""
    import torch

    lib = ve.load_library()
    dev = torch.from_numpy(np.ascontiguousarray(words, np.uint32).view(np.int32).copy()).cuda()
    torch.cuda.synchronize()
    handle = None if stream is None else ctypes.c_void_p(stream.cuda_stream)
    rc = lib.ve_fill_normals_noalloc(ctypes.c_void_p(dev.data_ptr()), words.size, depth, handle)
    assert rc == ve.VE_OK, lib.ve_last_error().decode()
    if stream is not None:
        stream.synchronize()
    torch.cuda.synchronize()
    return dev.cpu().numpy().view(np.uint32)


def test_noalloc_normals_match_upload_path_twice(ve):
    small, _ = helpers.terrain(7, 0, 1)
    rng = np.random.default_rng(5)
    c = ve.OctreeCPU(5)
    c.insert_many(helpers.random_voxels(rng, 5, 0.1))
    o = ve.Octree(5)
    o.set(c)
    other = o.words()[: o.size]
    # two calls in a row on different scenes: the second must not see the
    # first call's leftovers in the shared scratch
    for words, depth in ((small, 7), (other, 5)):
        got = noalloc_normals(ve, words, depth)
        want = upload_path_normals(ve, words, depth)
        assert np.array_equal(got, want)
        assert (got >> 31).any()


def test_noalloc_on_a_stream_and_shallow_scenes(ve):
    """On a non-default stream, and on depth-1 and depth-2 scenes (no frontier
    expansion runs for depth 1), still equal to the upload path."""
    import torch

    rng = np.random.default_rng(9)
    s = torch.cuda.Stream()
    for depth, density in ((1, 0.5), (2, 0.4), (6, 0.05)):
        c = ve.OctreeCPU(depth)
        c.insert_many(helpers.random_voxels(rng, depth, density))
        o = ve.Octree(depth)
        o.set(c)
        words = o.words()[: max(o.size, 9)]
        for stream in (s, None):
            got = noalloc_normals(ve, words, depth, stream)
            assert np.array_equal(got, upload_path_normals(ve, words, depth)), (depth, stream)


def test_noalloc_rejects_scenes_beyond_the_scratch_limit(ve):
    import torch

    lib = ve.load_library()
    dev = torch.zeros(16, dtype=torch.int32, device="cuda")
    rc = lib.ve_fill_normals_noalloc(ctypes.c_void_p(dev.data_ptr()), 16, 8, None)
    assert rc == ve.VE_ERR_CAPACITY
    assert b"depth" in lib.ve_last_error()
