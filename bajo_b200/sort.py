"""GPU radix sort, mirroring ``bajo.sort.gpu`` of the reference.

Reference entry points (jgsimard/bajo):
  - ``onesweep_radix_sort_pairs`` / ``onesweep_radix_sort_keys``
    (bajo/sort/gpu/onesweep.mojo:454, :362)
  - ``device_radix_sort_pairs`` / ``device_radix_sort_keys``
    (bajo/sort/gpu/radix_sort.mojo:510, :397) -- the sort the LBVH uses
  - ``gpu_sort_pairs`` (bajo/sort/gpu/__init__.mojo:7)

All of them are stable LSD radix sorts that leave the result in the caller's
buffers.  Here every one runs the same sm_100a onesweep kernels through the
C ABI (``bajo_sort_*``); tensors are torch CUDA tensors used as plain device
memory.  Keys may be uint32/int32 (32-bit) or uint64/int64 (64-bit) bit
patterns; values are 32-bit.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib

_KEY_BYTES = {torch.uint32: 4, torch.int32: 4, torch.uint64: 8, torch.int64: 8}


class RadixSortWorkspace:
    """Reusable scratch for one sort shape (``RadixSortWorkspace``,
    bajo/sort/gpu/radix_sort.mojo:474; ``OneSweepWorkspace``, onesweep.mojo:330)."""

    def __init__(self, size: int, key_bytes: int, has_values: bool, begin_bit: int = 0, end_bit: int | None = None,
                 device=None):
        end_bit = key_bytes * 8 if end_bit is None else end_bit
        nbytes = ctypes.c_size_t(0)
        _lib.check(_lib.load().bajo_sort_workspace_size(size, key_bytes, int(has_values), begin_bit, end_bit,
                                                        ctypes.byref(nbytes)), "bajo_sort_workspace_size")
        self.size, self.key_bytes, self.has_values = size, key_bytes, has_values
        self.begin_bit, self.end_bit = begin_bit, end_bit
        self.buffer = torch.zeros(max(nbytes.value, 256), dtype=torch.uint8, device=device or "cuda")

    def fits(self, size, key_bytes, has_values, begin_bit, end_bit) -> bool:
        need = ctypes.c_size_t(0)
        _lib.load().bajo_sort_workspace_size(size, key_bytes, int(has_values), begin_bit, end_bit, ctypes.byref(need))
        return self.buffer.numel() >= need.value

    def status(self) -> int:
        st = ctypes.c_uint32(0)
        _lib.check(_lib.load().bajo_workspace_status(self.buffer.data_ptr(), _lib.stream_handle(), ctypes.byref(st)),
                   "bajo_workspace_status")
        return st.value


def _sort(keys: torch.Tensor, values: torch.Tensor | None, size: int | None, begin_bit: int, end_bit: int | None,
          workspace: RadixSortWorkspace | None, stream=None) -> RadixSortWorkspace:
    _lib.require_cuda(keys)
    if keys.dtype not in _KEY_BYTES:
        raise TypeError(f"unsupported key dtype {keys.dtype}")
    kb = _KEY_BYTES[keys.dtype]
    n = keys.numel() if size is None else int(size)
    if n > keys.numel() or not keys.is_contiguous():
        raise ValueError("keys must be contiguous and hold `size` elements")
    if values is not None:
        _lib.require_cuda(values)
        if values.element_size() != 4 or n > values.numel() or not values.is_contiguous():
            raise ValueError("values must be contiguous 32-bit and hold `size` elements")
    end_bit = kb * 8 if end_bit is None else end_bit
    if workspace is None or not workspace.fits(n, kb, values is not None, begin_bit, end_bit):
        workspace = RadixSortWorkspace(n, kb, values is not None, begin_bit, end_bit, device=keys.device)
    L = _lib.load()
    ws = workspace.buffer
    s = _lib.stream_handle(stream)
    if kb == 4 and values is None:
        rc = L.bajo_sort_keys_u32(keys.data_ptr(), n, begin_bit, end_bit, ws.data_ptr(), ws.numel(), s)
    elif kb == 4:
        rc = L.bajo_sort_pairs_u32(keys.data_ptr(), values.data_ptr(), n, begin_bit, end_bit, ws.data_ptr(),
                                   ws.numel(), s)
    elif values is None:
        rc = L.bajo_sort_keys_u64(keys.data_ptr(), n, begin_bit, end_bit, ws.data_ptr(), ws.numel(), s)
    else:
        rc = L.bajo_sort_pairs_u64(keys.data_ptr(), values.data_ptr(), n, begin_bit, end_bit, ws.data_ptr(),
                                   ws.numel(), s)
    _lib.check(rc, "bajo_sort")
    return workspace


def onesweep_radix_sort_pairs(keys, values, size=None, workspace=None, begin_bit=0, end_bit=None, stream=None):
    """Stable sort of (keys, values) in place (onesweep.mojo:454)."""
    return _sort(keys, values, size, begin_bit, end_bit, workspace, stream)


def onesweep_radix_sort_keys(keys, size=None, workspace=None, begin_bit=0, end_bit=None, stream=None):
    """Stable sort of keys in place (onesweep.mojo:362)."""
    return _sort(keys, None, size, begin_bit, end_bit, workspace, stream)


def device_radix_sort_pairs(keys, values, size=None, workspace=None, begin_bit=0, end_bit=None, stream=None):
    """Stable sort of (keys, values) in place (radix_sort.mojo:510)."""
    return _sort(keys, values, size, begin_bit, end_bit, workspace, stream)


def device_radix_sort_keys(keys, size=None, workspace=None, begin_bit=0, end_bit=None, stream=None):
    """Stable sort of keys in place (radix_sort.mojo:397)."""
    return _sort(keys, None, size, begin_bit, end_bit, workspace, stream)


def gpu_sort_pairs(keys, values, size=None, workspace=None, stream=None):
    """``bajo.sort.gpu.gpu_sort_pairs`` (bajo/sort/gpu/__init__.mojo:7).  The
    reference switches to an unstable bitonic sort at N <= 2^14; this one is
    the stable onesweep at every size."""
    return _sort(keys, values, size, 0, None, workspace, stream)
