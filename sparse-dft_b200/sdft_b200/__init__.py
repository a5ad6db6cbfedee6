"""sdft_b200: B200-native generalized Davidson hot path of Sparse-DFT.

The numerical work lives in libsdft_b200.so (hand-written sm_100a kernels
behind the C ABI in include/sdft_b200.h); this package is the Python-side
binding and the seeded synthetic input generator used by tests and benchmarks.
"""
from . import synthetic  # noqa: F401  (numpy only; importable without a GPU)

__all__ = ["synthetic", "library_path"]


def library_path():
    from ._capi import LIBRARY
    return LIBRARY
