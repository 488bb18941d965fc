"""The allocation-free sort entry point, called through the C ABI.

bajo_sort_pairs_u32_noalloc exists for callers that cannot allocate device
memory or hand the library a workspace (hosts that own all device memory and
pass only their own buffers, frame loops where an allocation would stall the
device).  Its scratch is a fixed array inside the library, shared by every
call.  This test checks that two calls in a row, of different sizes, give
exactly what the workspace-based bajo_sort_pairs_u32 gives, and that sizes
beyond the limit are refused.  It is collected last on purpose: it must pass
in a fresh process (where its first call sets up the scratch address) and
after every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _sort_with_workspace(L, keys_np, vals_np):
    from bajo_b200 import _lib
    n = keys_np.size
    k = torch.from_numpy(keys_np.view(np.int32).copy()).cuda()
    v = torch.from_numpy(vals_np.view(np.int32).copy()).cuda()
    nbytes = ctypes.c_size_t(0)
    assert L.bajo_sort_workspace_size(n, 4, 1, 0, 32, ctypes.byref(nbytes)) == _lib.OK
    ws = torch.zeros(nbytes.value, dtype=torch.uint8, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    assert L.bajo_sort_pairs_u32(k.data_ptr(), v.data_ptr(), n, 0, 32, ws.data_ptr(), ws.numel(), s) == _lib.OK
    torch.cuda.synchronize()
    return k.cpu().numpy().view(np.uint32), v.cpu().numpy().view(np.uint32)


def _sort_noalloc(L, keys_np, vals_np):
    from bajo_b200 import _lib
    n = keys_np.size
    k = torch.from_numpy(keys_np.view(np.int32).copy()).cuda()
    v = torch.from_numpy(vals_np.view(np.int32).copy()).cuda()
    status = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    rc = L.bajo_sort_pairs_u32_noalloc(k.data_ptr(), v.data_ptr(), n, 0, 32, status.data_ptr(), s)
    assert rc == _lib.OK
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    return k.cpu().numpy().view(np.uint32), v.cpu().numpy().view(np.uint32)


def test_noalloc_sort_matches_workspace_sort_twice():
    from bajo_b200 import _lib
    L = _lib.load()
    rng = np.random.default_rng(2024)
    # first call: the largest allowed size; second call: a smaller one, so the
    # second sees the first call's leftovers in the shared scratch
    for n in (_lib.SORT_NOALLOC_MAX_KEYS, 123_457):
        keys = rng.integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)
        keys[: n // 3] &= 0xFF00FF00  # many equal keys: stability matters
        vals = rng.integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)
        k_ref, v_ref = _sort_with_workspace(L, keys, vals)
        k_got, v_got = _sort_noalloc(L, keys, vals)
        assert np.array_equal(k_got, k_ref)
        assert np.array_equal(v_got, v_ref)


def test_noalloc_sort_refuses_too_many_keys():
    from bajo_b200 import _lib
    L = _lib.load()
    n = _lib.SORT_NOALLOC_MAX_KEYS + 1
    rc = L.bajo_sort_pairs_u32_noalloc(ctypes.c_void_p(256), ctypes.c_void_p(256), n, 0, 32, None, None)
    assert rc == _lib.ERR_TOO_LARGE
