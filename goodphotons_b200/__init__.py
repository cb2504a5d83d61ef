"""B200-native forward pinhole light tracer (drop-in for ftrace's mode-B GPU path).

The product is the native library `libftb200.so` (C ABI in include/ftb200.h: scene bake,
wavefront CUDA kernels for sm_100a, resident sessions).  This package binds it
(`lib`), mirrors its structures (`abi`), and generates the synthetic benchmark scenes
(`scenes`).
"""
from . import abi  # noqa: F401

__all__ = ["abi", "lib", "scenes"]
