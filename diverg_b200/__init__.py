"""diverg_b200: DiVerG's distance-index path (range-CRS SpGEMM, SpAdd, power,
distance index, batched membership query) on one NVIDIA B200.

The compute path is libdvg.so (hand-written sm_100a CUDA behind the C ABI of
include/dvg.h); this package mirrors the reference's C++ API on top of it.
"""
from .crs_matrix import CRSMatrix, from_basic
from .runtime import (Context, DeviceMatrix, ScopedRuntime, finalize_runtime, initialize_runtime,
                      is_runtime_initialized)
from .range_sparse import create_range_identity_matrix, range_power, range_spadd, range_spgemm
from .dindex import create_distance_index, query_batch

__all__ = [
    "CRSMatrix", "from_basic", "Context", "DeviceMatrix", "ScopedRuntime", "initialize_runtime",
    "finalize_runtime", "is_runtime_initialized", "create_range_identity_matrix", "range_spgemm",
    "range_spadd", "range_power", "create_distance_index", "query_batch",
]
