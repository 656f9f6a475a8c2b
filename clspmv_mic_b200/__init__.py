"""clspmv_mic_b200 — B200-native SpMV with clSpMV's storage formats and API.

The compute path is libclspmv_b200.so (CUDA for sm_100a behind a C ABI,
include/clspmv_b200.h); this package is its host-side mirror: the
reference's converter names (coo2csr, coo2dia, ...), device residency, and
the per-format SpMV entry points. There is no CPU fallback: if the library
is missing every call raises.
"""
from ._abi import ClspmvError, lib
from .formats import (BLOCK_SHAPES, GPU_ALIGNMENT, SELL_GROUP_SIZE, WARPSIZE, DeviceMatrix, HostMatrix, coo2b4csr,
                      coo2b4ell, coo2bcsr, coo2bdia, coo2bell, coo2csr, coo2dia, coo2ell, coo2sbell, coo2sell,
                      coo_matrix, from_arrays, if_sorted_coo, launch_count, pad_csr, sort_coo, to_coo)

__all__ = [
    "ClspmvError", "lib", "BLOCK_SHAPES", "GPU_ALIGNMENT", "SELL_GROUP_SIZE", "WARPSIZE", "DeviceMatrix",
    "HostMatrix", "coo2b4csr", "coo2b4ell", "coo2bcsr", "coo2bdia", "coo2bell", "coo2csr", "coo2dia", "coo2ell",
    "coo2sbell", "coo2sell", "coo_matrix", "from_arrays", "if_sorted_coo", "launch_count", "pad_csr", "sort_coo",
    "to_coo",
]
