"""Distance index with the reference's API (include/diverg/dindex.hpp,
include/diverg/dindex_eti.hpp) plus the batched membership query.
"""
import numpy as np

from .crs_matrix import CRSMatrix
from .runtime import default_context


def create_distance_index(ra: CRSMatrix, dmin: int, dmax: int, config=None, timer1=None,
                          timer2=None) -> CRSMatrix:
    """util::create_distance_index(ra, dmin, dmax), dindex.hpp:46-189 and its
    non-template overloads dindex_eti.hpp:44-53: the index
    A^dmin * (A+I)^(dmax-dmin) of the adjacency `ra`, same rowmap width as `ra`.
    `config` and the timers are accepted for source compatibility."""
    if not (dmin <= dmax and dmax != 0):
        raise ValueError("create_distance_index requires dmin <= dmax and dmax != 0")
    ctx = default_context()
    return ctx.distance_index(ctx.upload(ra), dmin, dmax).download(ra.size_type)


def query_batch(index, pairs: np.ndarray) -> np.ndarray:
    """Batched CRSMatrixBase::operator()(i, j) (crs_matrix.hpp:1197-1218):
    `index` is a CRSMatrix or a resident DeviceMatrix, `pairs` an (n, 2)
    uint32 array; returns uint8 0/1 answers."""
    ctx = default_context()
    dm = ctx.upload(index) if isinstance(index, CRSMatrix) else index
    return ctx.query(dm, pairs)
