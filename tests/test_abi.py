"""The C-ABI library loads, exports every entry point include/ve.h declares,
and rejects bad arguments with status codes (no GPU work)."""
import ctypes
import os
import re

import numpy as np
import pytest

import helpers

HEADER = os.path.join(helpers.ROOT, "include", "ve.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(ve_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "ve_render" in names and "ve_scene_upload" in names and len(names) > 30


def test_library_exports_every_declared_symbol(ve):
    lib = ve.load_library()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"libve.so lacks {missing}"


def test_python_mirror_binds_every_declared_symbol(ve):
    unbound = [n for n in declared_functions() if n not in ve._SIGNATURES]
    assert not unbound, f"no ctypes signature for {unbound}"


def test_struct_sizes_match_header(ve):
    assert ctypes.sizeof(ve.FrameConfigC) == 160
    assert ctypes.sizeof(ve.ViewC) == 4 + 64 + 160
    assert ctypes.sizeof(ve.FrameOutputsC) == 7 * 8
    assert ctypes.sizeof(ve.FrameStatsC) == 13 * 8 + 6 * 4 + 2 * 4 + 8 + 5 * 8 + 2 * 4 + 4 * 8
    assert ctypes.sizeof(ve.ServerConfigC) == 2 * 8 + 2 * 4 + 8 + 2 * 4
    assert ctypes.sizeof(ve.RequestInfoC) == 8 + 3 * 8 + 2 * 8
    assert ctypes.sizeof(ve.ServerStatsC) == 9 * 8
    assert ctypes.sizeof(ve.NrcConfigC) == 10 * 4 + 8


def test_version_and_errors(ve):
    lib = ve.load_library()
    assert b"sm_100a" in lib.ve_version()
    with pytest.raises(ve.VeError) as e:
        ve.OctreeCPU(0)
    assert e.value.code == ve.VE_ERR_INVALID and "depth" in str(e.value)
    with pytest.raises(ve.VeError):
        ve.terrain_words(12)
    assert lib.ve_octree_cpu_insert(None, 0, 0, 0, 1) == ve.VE_ERR_INVALID
    assert lib.ve_render(None, None, None) == ve.VE_ERR_INVALID
    assert lib.ve_scene_upload(None, None, 0, 7, 0, None) == ve.VE_ERR_INVALID


def test_no_cuda_device_is_a_loud_error(ve):
    """Without a GPU the renderer refuses to start (there is no CPU path)."""
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("GPU present")
    except ImportError:
        pass
    with pytest.raises(ve.VeError) as e:
        ve.Renderer()
    assert e.value.code == ve.VE_ERR_CUDA


def test_frame_config_roundtrip(ve):
    fc = ve.FrameConfig(width=7, height=5, spp=3, bounces=2, frame_index=9, decay=0.5, flags=ve.FRAME_TIMING)
    c = fc.to_c()
    assert (c.width, c.height, c.spp, c.bounces, c.frame_index, c.flags) == (7, 5, 3, 2, 9, 1)
    assert abs(c.decay - 0.5) < 1e-7
    assert np.allclose(np.array(c.sun_dir[:]), ve.SUN_DIR)
