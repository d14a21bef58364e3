"""remora_b200: the B200 (sm_100a) CUDA backend of Remora's hot path.

The product is ``libremora_cuda.so`` (C-ABI in ``include/remora_cuda.h``) and the
header-only C++ ``cuda_tag`` device in ``include/remora/cuda.hpp``. This package builds
the library and exposes a thin Python view of the C-ABI over torch device tensors
(``remora_b200.ops``) for tests and benchmarks.
"""
from ._lib import LIB_PATH, RemoraCudaError, lib  # noqa: F401

__all__ = ["LIB_PATH", "RemoraCudaError", "lib"]
