"""behavert_b200 -- B200-native BehaveRT per-step agent pipeline.

The compute lives in libbehavert_b200.so (hand-written sm_100a CUDA behind a
C-ABI, include/behavert_b200.h).  This package is the Python host side: a
ctypes mirror of the C-ABI (`_abi`), the engine facade with the reference's
functionality names (`engine`), and the seeded benchmark workloads
(`workloads`).
"""
from ._abi import (BRT_MEM_DEVICE, BRT_MEM_HOST, BrtError, BrtParams, EXPORTED_SYMBOLS, LIB_PATH, lib,
                   params_default)
from .engine import Engine, radix_sort_pairs, radix_sort_scratch_bytes

__all__ = [
    "BRT_MEM_DEVICE", "BRT_MEM_HOST", "BrtError", "BrtParams", "EXPORTED_SYMBOLS", "LIB_PATH", "lib",
    "params_default", "Engine", "radix_sort_pairs", "radix_sort_scratch_bytes",
]
