"""B200-native Renderer2 hot paths: SGGX mesh-to-volume LOD filter and
wavefront path tracer (CUDA for sm_100a behind the C ABI in include/r2.h).

The Python modules are thin ctypes views used by tests and the benchmark; the
runtime itself is C++/CUDA in csrc/.
"""
from . import _native  # noqa: F401  (fails loudly when the native library is missing; opened on first use)

__all__ = ["_native"]
