"""Range operations with the reference's host-container API
(include/diverg/range_sparse.hpp): inputs are host CRSMatrix objects,
results come back by value, as in the reference's ETI wrappers
(RangeSpGEMM / RangeSpAdd / RangePower).  The work runs on the device
through libdvg.so; `config` arguments are accepted for source compatibility
and ignored (the device plan is chosen by the library's autotuner).
"""
import numpy as np

from .crs_matrix import CRSMatrix
from .runtime import default_context


def _size_type(*ms):
    return np.uint32 if all(m.size_type == np.uint32 for m in ms) else np.uint64


def create_range_identity_matrix(n, space=None, size_type=np.uint64) -> CRSMatrix:
    """create_range_identity_matrix<RCRS>(n), range_sparse.hpp:95-110."""
    ctx = default_context()
    return ctx.identity(n).download(size_type)


def range_spadd(a: CRSMatrix, b: CRSMatrix, space=None) -> CRSMatrix:
    """range_spadd(a, b), range_sparse.hpp:470-477."""
    ctx = default_context()
    return ctx.spadd(ctx.upload(a), ctx.upload(b)).download(_size_type(a, b))


def range_spgemm(a: CRSMatrix, b: CRSMatrix, config=None) -> CRSMatrix:
    """range_spgemm(a, b, config), range_sparse.hpp:2325-2332."""
    ctx = default_context()
    return ctx.spgemm(ctx.upload(a), ctx.upload(b)).download(_size_type(a, b))


def range_power(a: CRSMatrix, k: int, config=None) -> CRSMatrix:
    """range_power(a, k, config), range_sparse.hpp:2362-2368."""
    ctx = default_context()
    return ctx.power(ctx.upload(a), k).download(_size_type(a))
