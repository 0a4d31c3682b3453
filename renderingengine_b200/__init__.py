"""B200 (sm_100a) wavefront path-tracing hot path of RenderingEngine.

The compute path is the CUDA library ``_lib/libre_b200.so`` behind the C ABI in
``include/re_b200.h``; this package is its host-side mirror.  Importing the
package does not require a GPU; calling into the library does, and every entry
point fails loudly when the library is missing.
"""
from . import _native
from ._native import load as load_library

__all__ = ["_native", "load_library"]
