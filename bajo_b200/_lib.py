"""Loader for the C-ABI CUDA library ``libbajo_b200.so`` (ctypes).

This is the only native code the package uses.  There is no CPU fallback:
if the shared object is missing, or a GPU entry point is called without a
CUDA device, the call raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbajo_b200.so")

# status codes (include/bajo_b200.h)
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_WORKSPACE_TOO_SMALL = 2
ERR_TOO_LARGE = 3
ERR_CUDA = 4
ERR_DEVICE = 5
STATUS_LOOKBACK_TIMEOUT = 0x1
STATUS_STACK_OVERFLOW = 0x2
STATUS_BAD_TOPOLOGY = 0x4
STATUS_WIDE_TIMEOUT = 0x40
STATUS_STAGE_TIMEOUT = 0x80
STATUS_WAIT_TIMEOUT = 0x100
STATUS_GRID_TIMEOUT = 0x200
FUSED_MAX_LEAVES = 1 << 17  # largest scene the one-launch build takes
LBVH_TOP_CAP = 1536  # subtrees per CTA in the one-launch build's top stage
TRI_MT = 0
TRI_WATERTIGHT = 1
SORT_MAX_KEYS = (1 << 30) - 1
SORT_NOALLOC_MAX_KEYS = 1 << 20
SORT_NOALLOC_SCRATCH_BYTES = 10490368  # BAJO_SORT_NOALLOC_SCRATCH_BYTES
SORT_VARIANTS_U32 = 7  # BAJO_SORT_VARIANTS_U32: compiled variants of the 32-bit-key sort
SORT_VARIANTS_U64 = 7  # BAJO_SORT_VARIANTS_U64
SORT_VARIANTS = 7  # the larger of the two

_ERRORS = {
    ERR_INVALID_ARGUMENT: "invalid argument",
    ERR_WORKSPACE_TOO_SMALL: "workspace too small",
    ERR_TOO_LARGE: "size exceeds the supported maximum",
    ERR_CUDA: "CUDA error",
    ERR_DEVICE: "device status error",
}


class BajoError(RuntimeError):
    def __init__(self, code: int, what: str):
        super().__init__(f"{what}: {_ERRORS.get(code, 'error')} (code {code})")
        self.code = code


_P = ctypes.c_void_p
_U32 = ctypes.c_uint32
_I32 = ctypes.c_int32
_SZ = ctypes.c_size_t
_F = ctypes.c_float


class BajoLbvhC(ctypes.Structure):
    """Mirror of ``struct BajoLbvh`` (include/bajo_b200.h)."""
    _fields_ = [
        ("n_leaves", _U32), ("n_segments", _U32), ("seg_offsets", _P), ("internal_offsets", _P),
        ("leaf_bounds", _P), ("seg_bounds", _P), ("sort_keys", _P), ("leaf_ids", _P), ("morton_codes", _P),
        ("node_meta", _P), ("node_bounds", _P), ("node_leaf_counts", _P), ("node_flags", _P),
        ("leaf_parent", _P), ("roots", _P), ("leaf_tris", _P), ("top_nodes", _P),
    ]


LBVH_ARRAYS = ("internal_offsets", "leaf_bounds", "seg_bounds", "sort_keys", "leaf_ids", "morton_codes",
               "node_meta", "node_bounds", "node_leaf_counts", "node_flags", "leaf_parent", "roots", "leaf_tris")


class BajoLbvhSizesC(ctypes.Structure):
    _fields_ = [(name, _SZ) for name in LBVH_ARRAYS] + [("workspace", _SZ), ("top_nodes", _SZ)]


TOP_NODES = 256          # BAJO_TOP_NODES
TOP_FLAG = 0x40000000    # BAJO_TOP_FLAG
TOP_BYTES = 16 + 64 * TOP_NODES


class BajoWideBvhC(ctypes.Structure):
    """Mirror of ``struct BajoWideBvh`` (include/bajo_b200.h)."""
    _fields_ = [("width", _U32), ("max_leaf", _U32), ("n_segments", _U32), ("node_offsets", _P), ("leaf_offsets", _P),
                ("nodes", _P), ("leaf_indices", _P), ("leaf_tris", _P), ("leaf_sorted", _P), ("bvh2_leaf_tris", _P)]


WIDE_ARRAYS = ("node_offsets", "leaf_offsets", "nodes", "leaf_indices", "leaf_tris", "leaf_sorted")


class BajoWideSizesC(ctypes.Structure):
    _fields_ = [(name, _SZ) for name in WIDE_ARRAYS] + [("workspace", _SZ)]


class BajoCwbvh8C(ctypes.Structure):
    """Mirror of ``struct BajoCwbvh8`` (include/bajo_b200.h)."""
    _fields_ = [("n_segments", _U32), ("n_tris", _U32), ("node_offsets", _P), ("nodes", _P), ("triangles", _P)]


CWBVH8_ARRAYS = ("node_offsets", "nodes", "triangles")
CWBVH8_NODE_WORDS = 20  # BAJO_CWBVH8_NODE_WORDS
CWBVH8_TRI_WORDS = 12   # BAJO_CWBVH8_TRI_WORDS


class BajoCwbvh8SizesC(ctypes.Structure):
    _fields_ = [(name, _SZ) for name in CWBVH8_ARRAYS] + [("workspace", _SZ)]


# every symbol the header declares, with its ctypes signature
SIGNATURES = {
    "bajo_workspace_status": (_I32, [_P, _P, ctypes.POINTER(_U32)]),
    "bajo_workspace_status_clear": (_I32, [_P, _P]),
    "bajo_sort_workspace_size": (_I32, [_U32, _U32, _I32, _I32, _I32, ctypes.POINTER(_SZ)]),
    "bajo_sort_keys_u32": (_I32, [_P, _U32, _I32, _I32, _P, _SZ, _P]),
    "bajo_sort_pairs_u32": (_I32, [_P, _P, _U32, _I32, _I32, _P, _SZ, _P]),
    "bajo_sort_keys_u64": (_I32, [_P, _U32, _I32, _I32, _P, _SZ, _P]),
    "bajo_sort_pairs_u64": (_I32, [_P, _P, _U32, _I32, _I32, _P, _SZ, _P]),
    "bajo_sort_pairs_u32_noalloc": (_I32, [_P, _P, _U32, _I32, _I32, _P, _P]),
    "bajo_sort_tuning_set": (_I32, [_U32, _I32, _U32, _I32]),
    "bajo_sort_tuning_get": (_I32, [_U32, _I32, _U32, ctypes.POINTER(_I32)]),
    "bajo_lbvh_sizes": (_I32, [_U32, _U32, ctypes.POINTER(BajoLbvhSizesC)]),
    "bajo_lbvh_build": (_I32, [_P, ctypes.POINTER(BajoLbvhC), _P, _SZ, _P]),
    "bajo_lbvh_build_timed": (_I32, [_P, ctypes.POINTER(BajoLbvhC), _P, _SZ, _P, ctypes.POINTER(_P), _I32]),
    "bajo_lbvh_stage_count": (_I32, [_U32, _U32, ctypes.POINTER(_I32)]),
    "bajo_lbvh_fused_max_set": (_I32, [_U32]),
    "bajo_lbvh_fused_top_cap_set": (_I32, [_U32]),
    "bajo_trace_tuning_set": (_I32, [_I32, _U32, _I32]),
    "bajo_trace_tuning_get": (_I32, [_I32, _U32, ctypes.POINTER(_I32)]),
    "bajo_trace_stack_tuning_set": (_I32, [_I32, _U32, _I32]),
    "bajo_trace_stack_tuning_get": (_I32, [_I32, _U32, ctypes.POINTER(_I32)]),
    "bajo_render_tuning_set": (_I32, [_I32, _I32]),
    "bajo_render_tuning_get": (_I32, [_I32, ctypes.POINTER(_I32)]),
    "bajo_lbvh_build_launches": (_I32, [_U32, _U32, ctypes.POINTER(_I32)]),
    "bajo_lbvh_stage_top": (_I32, [ctypes.POINTER(BajoLbvhC), _P]),
    "bajo_wait_selftest": (_I32, [_P, _U32, _U32, _P, _P]),
    "bajo_render_create": (_I32, [_P, _P, _SZ, ctypes.POINTER(_P)]),
    "bajo_render_enqueue": (_I32, [_P, _P, _P, _P, _P, _P, _P]),
    "bajo_render_download": (_I32, [_P, _P, _P, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64),
                                    ctypes.POINTER(_U32), _P]),
    "bajo_render_graph_launches": (_I32, [_P, ctypes.POINTER(_U32)]),
    "bajo_render_destroy": (_I32, [_P]),
    "bajo_trace_rays": (_I32, [ctypes.POINTER(BajoLbvhC), _P, _U32, _I32, _P, _P, _P, _P, _P]),
    "bajo_trace_camera": (_I32, [ctypes.POINTER(BajoLbvhC), _P, _U32, _U32, _U32, _I32, _P, _P, _P, _P, _P]),
    "bajo_trace_batch": (_I32, [ctypes.POINTER(BajoLbvhC), _P, _U32, _U32, _U32, ctypes.c_uint64, _I32, _P, _P,
                                _P, _P, _P, _P]),
    "bajo_trace_camera_stats": (_I32, [ctypes.POINTER(BajoLbvhC), _P, _U32, _U32, _U32, _I32, _P, _P, _P]),
    "bajo_rt_build_lights": (_I32, [_P, _P, _U32, _P, _U32, _P, _U32, ctypes.POINTER(_U32),
                                    ctypes.POINTER(_F)]),
    "bajo_render_workspace_size": (_I32, [_P, ctypes.POINTER(_SZ)]),
    "bajo_render": (_I32, [_P, _P, _P, _P, _P, _P, _SZ, _P]),
    "bajo_render_stats": (_I32, [_P, _P, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]),
    "bajo_wide_sizes": (_I32, [_U32, _U32, _U32, ctypes.POINTER(BajoWideSizesC)]),
    "bajo_wide_build": (_I32, [ctypes.POINTER(BajoLbvhC), ctypes.POINTER(BajoWideBvhC), _P, _SZ, _P]),
    "bajo_wide_counts": (_I32, [ctypes.POINTER(BajoWideBvhC), _P, ctypes.POINTER(_U32), ctypes.POINTER(_U32)]),
    "bajo_trace_wide_rays": (_I32, [ctypes.POINTER(BajoWideBvhC), _U32, _U32, _P, _U32, _I32, _P, _P, _P, _P,
                                    _P]),
    "bajo_trace_wide_camera": (_I32, [ctypes.POINTER(BajoWideBvhC), _U32, _U32, _P, _U32, _U32, _U32, _I32, _P, _P,
                                      _P, _P, _P, _P]),
    "bajo_hploc_workspace_size": (_I32, [_U32, _U32, ctypes.POINTER(_SZ)]),
    "bajo_hploc_build": (_I32, [_P, ctypes.POINTER(BajoLbvhC), _P, _SZ, _P]),
    "bajo_tlas_instance_boxes": (_I32, [ctypes.POINTER(BajoLbvhC), _P, _P, _U32, _P, _P, _P]),
    "bajo_trace_tlas_rays": (_I32, [ctypes.POINTER(BajoLbvhC), ctypes.POINTER(BajoLbvhC), _P, _P, _U32, _P, _U32,
                                    _I32, _I32, _P, _P, _P]),
    "bajo_trace_tlas_camera": (_I32, [ctypes.POINTER(BajoLbvhC), ctypes.POINTER(BajoLbvhC), _P, _P, _U32, _P, _U32,
                                      _U32, _U32, _I32, _I32, _P, _P, _P]),
    "bajo_cwbvh8_sizes": (_I32, [_U32, _U32, ctypes.POINTER(BajoCwbvh8SizesC)]),
    "bajo_cwbvh8_build": (_I32, [ctypes.POINTER(BajoLbvhC), ctypes.POINTER(BajoCwbvh8C), _P, _SZ, _P]),
    "bajo_cwbvh8_count": (_I32, [ctypes.POINTER(BajoCwbvh8C), _P, ctypes.POINTER(_U32)]),
    "bajo_trace_cwbvh8_rays": (_I32, [ctypes.POINTER(BajoCwbvh8C), _U32, _P, _U32, _I32, _P, _P, _P, _P, _P]),
    "bajo_trace_cwbvh8_camera": (_I32, [ctypes.POINTER(BajoCwbvh8C), _U32, _P, _U32, _U32, _U32, _I32, _P, _P, _P,
                                        _P, _P]),
    "bajo_mlp_param_count": (_I32, [ctypes.POINTER(_U32)]),
    "bajo_mlp_forward": (_I32, [_P, _P, _P, _U32, _P, _P, _P]),
    "bajo_mlp_forward_tc": (_I32, [_P, _P, _P, _U32, _P, _P, _P, _P]),
    "bajo_mlp_grad": (_I32, [_P, _P, _P, _P, _P, _U32, _P, _P, _P, _P]),
    "bajo_mlp_grad_tc": (_I32, [_P, _P, _P, _P, _P, _U32, _P, _P, _P, _P, _P]),
    "bajo_mlp_adam": (_I32, [_P, _P, _P, _P, _P, _U32, _F, _F, _F, _F, _F, _P]),
    "bajo_guide_records_size": (_I32, [_U32, ctypes.POINTER(_SZ)]),
    "bajo_render_guided": (_I32, [_P, _P, _P, _P, _P, _P, _P, _SZ, _P]),
    "bajo_guide_train": (_I32, [_P, _P, _U32, _P, _U32, _U32, _F, _P]),
    "bajo_camera_make": (_I32, [_P, _P, _P, _F, _P]),
    "bajo_camera_from_vfov": (_I32, [_P, _P, _P, _F, _P]),
    "bajo_version": (ctypes.c_char_p, []),
}

_lib = None


def load() -> ctypes.CDLL:
    """Load ``libbajo_b200.so``; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m bajo_b200.build` "
                              "(there is no CPU fallback)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        _install_tuning()
    return _lib


def _install_tuning() -> None:
    """Load the autotuner's cached tile choices for this GPU, if any."""
    try:
        import torch
        if not torch.cuda.is_available():
            return
        from . import autotune
        autotune.load()
    except Exception:  # a missing or stale cache only means built-in choices
        pass


def check(code: int, what: str) -> None:
    if code != OK:
        raise BajoError(code, what)


def require_cuda(t) -> None:
    """Raise unless `t` is a CUDA tensor (the library has no host path)."""
    import torch
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError("bajo_b200 kernels take CUDA tensors; there is no CPU fallback")


def stream_handle(stream=None) -> int:
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream
