"""alp_b200 -- B200 (sm_100a) backend for the ALP/GraphBLAS hot path.

The product is libalp_b200.so (CUDA kernels behind the C-ABI of
include/alp_b200.h) and the C++ template backend under include/graphblas/b200/.
This Python package is the thin binding used by the tests and the benchmark.
"""
from . import _abi as abi  # noqa: F401
from ._abi import AlpError, check, call, lib, launches  # noqa: F401

__all__ = ["abi", "AlpError", "check", "call", "lib", "launches"]
