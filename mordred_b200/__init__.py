"""mordred_b200 — B200-native (sm_100a) star-query hot path behind a C ABI.

The compute path is the in-tree CUDA library ``libmordred_b200.so`` (kernels + the
C ABI declared in ``include/mordred_b200.h``); this package binds it with ctypes and
holds the host-side query templates. Importing the package does not touch the GPU.
"""
from ._lib import MbError, lib, lib_path  # noqa: F401

__all__ = ["MbError", "lib", "lib_path"]
