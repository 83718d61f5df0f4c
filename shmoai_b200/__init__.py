"""B200-native CKKS evaluation core for ShMOAI's evaluator hot path.

The compute path is the CUDA library ``_build/libshmoai_b200.so`` (C ABI in
include/shmoai_ckks.h); this package is its host-side face.  There is no CPU
fallback: the GPU entry points raise if the library is missing.
"""
from ._lib import LIB_PATH, build, exported_symbols, lib  # noqa: F401

__all__ = ["LIB_PATH", "build", "exported_symbols", "lib"]
