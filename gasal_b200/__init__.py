"""gasal_b200 -- GASAL2's batched pairwise-alignment path on NVIDIA B200.

The product is the CUDA library libgasal_b200.so (C++ drop-in API in
include/gasal_header.h, C ABI in include/gasal_b200_capi.h); this package is
its Python binding (``lib``), the ctypes mirror of the C structs (``capi``)
and the seeded synthetic workloads used by the benchmark (``workloads``).
"""
from .capi import (Batch, Params, Outputs, GLOBAL, SEMI_GLOBAL, LOCAL, BANDED, KSW, WITHOUT_START,
                   WITH_START, WITH_TB, NONE, QUERY, TARGET, BOTH, TRUE, FALSE)

__all__ = ["Batch", "Params", "Outputs", "GLOBAL", "SEMI_GLOBAL", "LOCAL", "BANDED", "KSW", "WITHOUT_START",
           "WITH_START", "WITH_TB", "NONE", "QUERY", "TARGET", "BOTH", "TRUE", "FALSE"]
