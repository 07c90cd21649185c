"""ctypes access to the CPU oracle (liboracle.so built from oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and the CPU
baseline leg of bench.py, never by the product package.  Each function names
the reference routine it restates; the C++ source carries the file:line
citations.
"""
import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


class _OrcMat(ctypes.Structure):
    _fields_ = [
        ("nrows", ctypes.c_uint32),
        ("ncols", ctypes.c_uint32),
        ("nentries", ctypes.c_uint64),
        ("nnz", ctypes.c_uint64),
        ("rowmap", ctypes.POINTER(ctypes.c_uint64)),
        ("entries", ctypes.POINTER(ctypes.c_uint32)),
    ]


@dataclass
class OMat:
    """A host range-CRS matrix as the oracle sees it."""
    nrows: int
    ncols: int
    rowmap: np.ndarray  # uint64[nrows+1]
    entries: np.ndarray  # uint32[rowmap[-1]]
    nnz: int

    def same(self, other) -> bool:
        return (self.nrows == other.nrows and self.ncols == other.ncols
                and int(self.nnz) == int(other.nnz)
                and np.array_equal(self.rowmap, np.asarray(other.rowmap, dtype=np.uint64))
                and np.array_equal(self.entries, np.asarray(other.entries, dtype=np.uint32)))


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            subprocess.run(["make", "-s", "-C", _HERE], check=True)
        L = ctypes.CDLL(path)
        P = ctypes.POINTER(_OrcMat)
        L.orc_mat_free.argtypes = [P]
        L.orc_identity.restype = P
        L.orc_identity.argtypes = [ctypes.c_uint32]
        L.orc_spadd.restype = P
        L.orc_spadd.argtypes = [P, P]
        L.orc_spgemm.restype = P
        L.orc_spgemm.argtypes = [P, P, ctypes.c_int, ctypes.c_int]
        L.orc_power.restype = P
        L.orc_power.argtypes = [P, ctypes.c_uint, ctypes.c_int, ctypes.c_int]
        L.orc_dindex.restype = P
        L.orc_dindex.argtypes = [P, ctypes.c_uint, ctypes.c_uint, ctypes.c_int, ctypes.c_int]
        L.orc_query.argtypes = [P, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]
        L.orc_basic_to_range.restype = P
        L.orc_basic_to_range.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p]
        L.orc_adjacency.restype = P
        L.orc_adjacency.argtypes = [ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]
        L.orc_adjacency_range.restype = P
        L.orc_adjacency_range.argtypes = [ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                          ctypes.c_uint32, ctypes.c_uint32]
        L.orc_nnz.restype = ctypes.c_uint64
        L.orc_nnz.argtypes = [P]
        L.orc_max_threads.restype = ctypes.c_int
        _LIB = L
    return _LIB


def _view(m):
    rowmap = np.ascontiguousarray(m.rowmap, dtype=np.uint64)
    entries = np.ascontiguousarray(m.entries, dtype=np.uint32)
    s = _OrcMat(int(m.nrows) if hasattr(m, "nrows") else len(rowmap) - 1, int(m.ncols), len(entries), int(m.nnz),
                rowmap.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                entries.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
    s._keep = (rowmap, entries)
    return s


def _take(p) -> OMat:
    if not p:
        raise ValueError("oracle rejected the arguments")
    m = p.contents
    rowmap = np.ctypeslib.as_array(m.rowmap, shape=(m.nrows + 1,)).copy()
    entries = (np.ctypeslib.as_array(m.entries, shape=(m.nentries,)).copy() if m.nentries
               else np.zeros(0, dtype=np.uint32))
    out = OMat(int(m.nrows), int(m.ncols), rowmap, entries, int(m.nnz))
    lib().orc_mat_free(p)
    return out


def threads() -> int:
    return int(lib().orc_max_threads())


def identity(n: int) -> OMat:
    """create_range_identity_matrix (range_sparse.hpp:66-110)."""
    return _take(lib().orc_identity(n))


def spadd(a, b) -> OMat:
    """range_spadd (range_sparse.hpp:112-477)."""
    va, vb = _view(a), _view(b)
    return _take(lib().orc_spadd(ctypes.byref(va), ctypes.byref(vb)))


def spgemm(a, b, algo: str = "btree", nthreads: int = 0) -> OMat:
    """range_spgemm: algo 'btree' (range_sparse.hpp:487-678) or 'hbv'
    (range_sparse.hpp:1132-1442 restated on the host)."""
    va, vb = _view(a), _view(b)
    return _take(lib().orc_spgemm(ctypes.byref(va), ctypes.byref(vb), 1 if algo == "hbv" else 0,
                                  nthreads or threads()))


def power(a, k: int, algo: str = "btree", nthreads: int = 0) -> OMat:
    """range_power_inplace (range_sparse.hpp:2370-2431)."""
    va = _view(a)
    return _take(lib().orc_power(ctypes.byref(va), k, 1 if algo == "hbv" else 0, nthreads or threads()))


def dindex(a, dlo: int, dup: int, algo: str = "btree", nthreads: int = 0) -> OMat:
    """util::create_distance_index (dindex.hpp:46-189)."""
    va = _view(a)
    return _take(lib().orc_dindex(ctypes.byref(va), dlo, dup, 1 if algo == "hbv" else 0, nthreads or threads()))


def query(m, pairs: np.ndarray) -> np.ndarray:
    """CRSMatrixBase::operator() (crs_matrix.hpp:1197-1218, 149-169) per pair."""
    pairs = np.ascontiguousarray(pairs, dtype=np.uint32).reshape(-1, 2)
    out = np.zeros(len(pairs), dtype=np.uint8)
    vm = _view(m)
    lib().orc_query(ctypes.byref(vm), pairs.ctypes.data, len(pairs), out.ctypes.data)
    return out


def basic_to_range(nrows: int, ncols: int, rowmap: np.ndarray, cols: np.ndarray) -> OMat:
    """crs_matrix::append(Range <- Basic) (crs_matrix.hpp:197-242)."""
    rowmap = np.ascontiguousarray(rowmap, dtype=np.uint64)
    cols = np.ascontiguousarray(cols, dtype=np.uint32)
    return _take(lib().orc_basic_to_range(nrows, ncols, rowmap.ctypes.data, cols.ctypes.data))


def adjacency(node_len: np.ndarray, edges: np.ndarray, lower: int = 1, upper: int = 0) -> OMat:
    """util::range_adjacency_matrix (adjacency.hpp:170-265); node ids 1..N in
    rank order, edges as (from_id, to_id) rows, the nodes [lower, upper)
    (upper = 0: through the last node)."""
    node_len = np.ascontiguousarray(node_len, dtype=np.uint32)
    edges = np.ascontiguousarray(edges, dtype=np.uint32).reshape(-1, 2)
    return _take(lib().orc_adjacency_range(len(node_len), node_len.ctypes.data, len(edges), edges.ctypes.data,
                                           lower, upper))


def nnz(m) -> int:
    """crs_matrix::nnz(..., RangeGroup) (crs_matrix.hpp:175-189)."""
    vm = _view(m)
    return int(lib().orc_nnz(ctypes.byref(vm)))


# ---- dense helpers for brute-force pinning (small n only) -----------------

def to_dense(m) -> np.ndarray:
    """Expand a range-CRS matrix to a dense bool array."""
    n = len(m.rowmap) - 1
    d = np.zeros((n, int(m.ncols)), dtype=bool)
    for i in range(n):
        e = m.entries[int(m.rowmap[i]):int(m.rowmap[i + 1])]
        for k in range(0, len(e), 2):
            d[i, int(e[k]):int(e[k + 1]) + 1] = True
    return d


def from_dense(d: np.ndarray) -> OMat:
    """Canonical range CRS of a dense bool array (maximal runs)."""
    n, ncols = d.shape
    rowmap = [0]
    ent = []
    for i in range(n):
        row = d[i].astype(np.int8)
        diff = np.diff(np.concatenate(([0], row, [0])))
        starts = np.flatnonzero(diff == 1)
        ends = np.flatnonzero(diff == -1) - 1
        for s, e in zip(starts, ends):
            ent += [s, e]
        rowmap.append(len(ent))
    return OMat(n, ncols, np.array(rowmap, dtype=np.uint64), np.array(ent, dtype=np.uint32), int(d.sum()))


def dense_power(d: np.ndarray, k: int) -> np.ndarray:
    """Boolean matrix power by repeated squaring on dense bool arrays."""
    n = d.shape[0]
    res = np.eye(n, dtype=bool)
    base = d.copy()
    while k:
        if k & 1:
            res = (res.astype(np.float32) @ base.astype(np.float32)) > 0
        k >>= 1
        if k:
            base = (base.astype(np.float32) @ base.astype(np.float32)) > 0
    return res
