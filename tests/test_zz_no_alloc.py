"""The allocation-free sort entry point, called through the C ABI.

bajo_sort_pairs_u32_noalloc exists for callers that cannot allocate device
memory or hand the library a workspace (hosts that own all device memory and
pass only their own buffers, frame loops where an allocation would stall the
device).  Its scratch is a fixed array inside the library, shared by every
call.  These tests check calls in a row, of different sizes and bit ranges,
against both the workspace-based bajo_sort_pairs_u32 and numpy's stable
argsort, and that sizes beyond the limit are refused.  The file is collected
last on purpose: it must pass in a fresh process (where its first call sets
up the scratch address) and after every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _numpy_stable(keys, vals, begin, end):
    """Stable sort of (keys, vals) by bits [begin, end) of the keys."""
    if end <= begin or keys.size <= 1:
        return keys.copy(), vals.copy()
    digit = (keys.astype(np.uint64) >> np.uint64(begin)) & np.uint64((1 << (end - begin)) - 1)
    order = np.argsort(digit, kind="stable")
    return keys[order], vals[order]


def _sort_with_workspace(L, keys_np, vals_np, begin=0, end=32):
    from bajo_b200 import _lib
    n = keys_np.size
    k = torch.from_numpy(keys_np.view(np.int32).copy()).cuda()
    v = torch.from_numpy(vals_np.view(np.int32).copy()).cuda()
    nbytes = ctypes.c_size_t(0)
    assert L.bajo_sort_workspace_size(max(n, 1), 4, 1, begin, end, ctypes.byref(nbytes)) == _lib.OK
    ws = torch.zeros(nbytes.value, dtype=torch.uint8, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    assert L.bajo_sort_pairs_u32(k.data_ptr(), v.data_ptr(), n, begin, end, ws.data_ptr(), ws.numel(), s) == _lib.OK
    torch.cuda.synchronize()
    return k.cpu().numpy().view(np.uint32), v.cpu().numpy().view(np.uint32)


def _sort_noalloc(L, keys_np, vals_np, begin=0, end=32, with_status=True):
    from bajo_b200 import _lib
    n = keys_np.size
    k = torch.from_numpy(keys_np.view(np.int32).copy()).cuda()
    v = torch.from_numpy(vals_np.view(np.int32).copy()).cuda()
    status = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    kp = k.data_ptr() if n else None
    vp = v.data_ptr() if n else None
    rc = L.bajo_sort_pairs_u32_noalloc(kp, vp, n, begin, end, status.data_ptr() if with_status else None, s)
    assert rc == _lib.OK
    torch.cuda.synchronize()
    if with_status:
        assert int(status.item()) == 0  # written by the call (it started at -1)
    else:
        assert int(status.item()) == -1  # no status pointer: nothing written
    return k.cpu().numpy().view(np.uint32), v.cpu().numpy().view(np.uint32)


def _case(rng, n):
    keys = rng.integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)
    keys[: n // 3] &= 0xFF00FF00  # many equal keys: stability matters
    vals = rng.integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)
    return keys, vals


def test_noalloc_sort_matches_workspace_sort_twice():
    from bajo_b200 import _lib
    L = _lib.load()
    rng = np.random.default_rng(2024)
    # first call: the largest allowed size; second call: a smaller one, so the
    # second sees the first call's leftovers in the shared scratch
    for n in (_lib.SORT_NOALLOC_MAX_KEYS, 123_457):
        keys, vals = _case(rng, n)
        k_ref, v_ref = _sort_with_workspace(L, keys, vals)
        k_got, v_got = _sort_noalloc(L, keys, vals)
        assert np.array_equal(k_got, k_ref)
        assert np.array_equal(v_got, v_ref)
        k_np, v_np = _numpy_stable(keys, vals, 0, 32)
        assert np.array_equal(k_got, k_np)
        assert np.array_equal(v_got, v_np)


@pytest.mark.parametrize("n", [0, 1, 2, 3, 1000])
@pytest.mark.parametrize("bits", [(0, 0), (0, 24), (8, 16), (5, 29), (0, 32)])
def test_noalloc_sort_edge_sizes_and_bit_ranges(n, bits):
    """n <= 1 and empty bit ranges (no pass: only the status word is
    cleared); odd pass counts (0..24 is three passes: the result is copied
    back from the scratch array); partial ranges."""
    from bajo_b200 import _lib
    L = _lib.load()
    rng = np.random.default_rng(n * 100 + bits[0] * 7 + bits[1])
    keys, vals = _case(rng, n)
    b, e = bits
    k_got, v_got = _sort_noalloc(L, keys, vals, b, e)
    k_np, v_np = _numpy_stable(keys, vals, b, e)
    assert np.array_equal(k_got, k_np)
    assert np.array_equal(v_got, v_np)
    if n:
        k_ref, v_ref = _sort_with_workspace(L, keys, vals, b, e)
        assert np.array_equal(k_got, k_ref)
        assert np.array_equal(v_got, v_ref)


def test_noalloc_sort_without_status_pointer():
    from bajo_b200 import _lib
    L = _lib.load()
    keys, vals = _case(np.random.default_rng(5), 77_777)
    k_got, v_got = _sort_noalloc(L, keys, vals, 0, 32, with_status=False)
    k_np, v_np = _numpy_stable(keys, vals, 0, 32)
    assert np.array_equal(k_got, k_np)
    assert np.array_equal(v_got, v_np)


def test_noalloc_sort_refuses_too_many_keys_and_bad_ranges():
    from bajo_b200 import _lib
    L = _lib.load()
    n = _lib.SORT_NOALLOC_MAX_KEYS + 1
    rc = L.bajo_sort_pairs_u32_noalloc(ctypes.c_void_p(256), ctypes.c_void_p(256), n, 0, 32, None, None)
    assert rc == _lib.ERR_TOO_LARGE
    for b, e in ((-1, 32), (0, 33), (20, 10)):
        assert L.bajo_sort_pairs_u32_noalloc(ctypes.c_void_p(256), ctypes.c_void_p(256), 16, b, e, None,
                                             None) == _lib.ERR_INVALID_ARGUMENT
    # null buffers with keys to sort
    assert L.bajo_sort_pairs_u32_noalloc(None, None, 16, 0, 32, None, None) == _lib.ERR_INVALID_ARGUMENT
