"""B200 (sm_100a) implementation of Ixchel2D's SIMPLE outer iteration.

The compute path is libixb.so (CUDA, built in-tree by
``python -m ixchel2d_b200.build``) behind the C ABI of include/ixb.h; this
package is a thin ctypes view of it plus synthetic-case builders.  The
library is loaded on first use of any attribute below, and a missing
library raises ImportError (there is no CPU fallback).
"""
import importlib

__all__ = ["ffi", "lib", "IxbError", "Simple2D", "Batch", "cases"]


def __getattr__(name):
    if name == "ffi":
        return importlib.import_module("._ffi", __name__)
    if name in ("lib", "IxbError"):
        return getattr(importlib.import_module("._ffi", __name__), name)
    if name == "Simple2D":
        return importlib.import_module(".simple", __name__).Simple2D
    if name == "Batch":
        return importlib.import_module(".batch", __name__).Batch
    if name == "cases":
        return importlib.import_module(".cases", __name__)
    raise AttributeError(name)
