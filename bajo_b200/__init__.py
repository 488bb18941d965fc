"""bajo_b200 -- sm_100a LBVH build + closest-hit traversal behind a C ABI.

A B200-native rebuild of the GPU LBVH / traversal path of jgsimard/bajo.
The product is ``libbajo_b200.so`` (declared in ``include/bajo_b200.h``);
this package is the Python host mirror of the reference's entry points
(``bajo.sort.gpu``, ``bajo.bvh.gpu``, ``bajo.bvh.camera``).
"""
from . import _lib  # noqa: F401

__all__ = ["sort", "bvh", "camera", "scenes"]
__version__ = "0.1.0"
