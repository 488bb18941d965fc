"""CPU tests of the C-ABI library: it loads, exports every symbol the header
declares, and the host-side entry points (size queries, argument checks,
camera records) work without a GPU.  No kernel is launched here."""
import ctypes
import os
import re

import numpy as np
import pytest

from bajo_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    src = open(os.path.join(ROOT, "include", "bajo_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(bajo_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol(lib):
    names = header_symbols()
    assert len(names) >= 14
    for name in names:
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, f"{name} has no ctypes signature"


def test_no_cpu_fallback_without_library(monkeypatch, tmp_path):
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "missing.so"))
    with pytest.raises(ImportError):
        _lib.load()


def test_version(lib):
    assert b"sm_100a" in lib.bajo_version()


def test_sort_workspace_sizes(lib):
    out = ctypes.c_size_t(0)
    assert lib.bajo_sort_workspace_size(1 << 20, 4, 1, 0, 32, ctypes.byref(out)) == _lib.OK
    small = out.value
    assert small > (1 << 20) * 8  # alternate keys + values
    assert lib.bajo_sort_workspace_size(1 << 20, 8, 1, 0, 64, ctypes.byref(out)) == _lib.OK
    assert out.value > small
    assert lib.bajo_sort_workspace_size(10, 3, 1, 0, 32, ctypes.byref(out)) == _lib.ERR_INVALID_ARGUMENT
    assert lib.bajo_sort_workspace_size(10, 4, 1, 0, 33, ctypes.byref(out)) == _lib.ERR_INVALID_ARGUMENT
    assert lib.bajo_sort_workspace_size(1 << 30, 4, 1, 0, 32, ctypes.byref(out)) == _lib.ERR_TOO_LARGE


def test_lbvh_sizes(lib):
    from bajo_b200.bvh import lbvh_sizes
    s = lbvh_sizes(65536, 1)
    assert s["node_meta"] == 65536 * 16 and s["node_bounds"] == 65536 * 48 and s["leaf_tris"] == 65536 * 48
    assert s["seg_bounds"] == 48 and s["internal_offsets"] == 8
    assert s["workspace"] > 65536 * 12
    s2 = lbvh_sizes(65536, 4096)
    # segmented keys (u64, 44 live bits) and their alternate buffers
    assert s2["roots"] == 4096 * 4 and s2["workspace"] > 65536 * 12 + 4096 * 48
    # one scene of up to 2^17 triangles also has room for the one-launch
    # build: two u32 key / id buffers and the per-(pass, tile) digit counts
    assert s["workspace"] > 4 * 65536 * 4 + 4 * 256 * 256 * 4
    out = _lib.BajoLbvhSizesC()
    assert lib.bajo_lbvh_sizes(10, 0, ctypes.byref(out)) == _lib.ERR_INVALID_ARGUMENT


def test_argument_checks_need_no_device(lib):
    """Invalid calls are rejected before any device work."""
    c = _lib.BajoLbvhC()
    assert lib.bajo_lbvh_build(None, None, None, 0, None) == _lib.ERR_INVALID_ARGUMENT
    c.n_segments = 0
    assert lib.bajo_lbvh_build(None, ctypes.byref(c), ctypes.c_void_p(256), 0, None) == _lib.ERR_INVALID_ARGUMENT
    c.n_segments = 1
    c.seg_offsets = 256
    c.n_leaves = 10
    assert lib.bajo_lbvh_build(ctypes.c_void_p(256), ctypes.byref(c), ctypes.c_void_p(256), 1 << 30,
                               None) == _lib.ERR_INVALID_ARGUMENT  # output arrays missing
    assert lib.bajo_trace_rays(None, None, 0, 1, None, None, None, None, None) == _lib.ERR_INVALID_ARGUMENT
    assert lib.bajo_sort_pairs_u32(None, None, 5, 0, 32, None, 0, None) == _lib.ERR_INVALID_ARGUMENT
    assert lib.bajo_sort_pairs_u32(ctypes.c_void_p(256), ctypes.c_void_p(256), 5, 0, 40, ctypes.c_void_p(256),
                                   1 << 20, None) == _lib.ERR_INVALID_ARGUMENT
    assert lib.bajo_sort_keys_u64(ctypes.c_void_p(256), 1000, 0, 64, ctypes.c_void_p(256), 16,
                                  None) == _lib.ERR_WORKSPACE_TOO_SMALL


def test_camera_records_match_oracle(lib, oracle):
    from bajo_b200 import camera
    a = camera.plain_lbvh_camera()
    b = oracle.camera_from_vfov([0.5, 0.5, -1.5], [0.5, 0.5, -0.5], [0, 1, 0], 60.0)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    a = camera.camera([1.0, 2.0, -3.0], [0.2, 0.1, 0.7], [0.0, 1.0, 0.0], 0.75)
    b = oracle.camera_make([1.0, 2.0, -3.0], [0.2, 0.1, 0.7], [0.0, 1.0, 0.0], 0.75)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_tuning_cache_round_trip(lib, monkeypatch, tmp_path):
    """autotune.save / load carry the closest-hit block and stack choices
    and the bounce kernels' block sizes through the JSON cache into the
    library's tables (host-side setters; no device work)."""
    from bajo_b200 import autotune
    monkeypatch.setattr(autotune, "device_key", lambda: "TEST GPU|1")
    path = str(tmp_path / "cache.json")
    results = {"trace_camera": {20: {"best": 256, "stack": 24, "ms": {}}},
               "trace_rays": {18: {"best": 64, "stack": 12, "ms": {}}},
               "render_trace": {0: {"best": 64, "ms": {}}},
               "render_shadow": {0: {"best": 256, "ms": {}}}}
    got = ctypes.c_int32(0)
    try:
        autotune.save(results, path)
        assert autotune.load(path) == 6
        assert lib.bajo_trace_tuning_get(0, 1 << 20, ctypes.byref(got)) == _lib.OK and got.value == 256
        assert lib.bajo_trace_stack_tuning_get(0, 1 << 20, ctypes.byref(got)) == _lib.OK and got.value == 24
        assert lib.bajo_trace_tuning_get(1, 1 << 18, ctypes.byref(got)) == _lib.OK and got.value == 64
        assert lib.bajo_trace_stack_tuning_get(1, 1 << 18, ctypes.byref(got)) == _lib.OK and got.value == 12
        assert lib.bajo_trace_stack_tuning_get(1, 1 << 20, ctypes.byref(got)) == _lib.OK and got.value == 64
        assert lib.bajo_render_tuning_get(0, ctypes.byref(got)) == _lib.OK and got.value == 64
        assert lib.bajo_render_tuning_get(1, ctypes.byref(got)) == _lib.OK and got.value == 128
        assert lib.bajo_render_tuning_get(2, ctypes.byref(got)) == _lib.OK and got.value == 256
    finally:
        for kind in (0, 1):
            for lg in range(33):
                lib.bajo_trace_tuning_set(kind, lg, 0)
                lib.bajo_trace_stack_tuning_set(kind, lg, 0)
        for kind in range(3):
            lib.bajo_render_tuning_set(kind, 0)
