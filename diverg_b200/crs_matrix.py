"""Host range-CRS matrix: the Python mirror of the reference's
CRSMatrix<crs_matrix::RangeDynamic, bool, uint32_t, TSize>
(include/diverg/crs_matrix.hpp:1873-2004, base class :1138-1519).

Storage is numpy: `rowmap` (TSize = uint64 or uint32, nrows+1 values counting
entries, two per range) and `entries` (uint32 inclusive [start,end] pairs).
"""
import struct

import numpy as np


class CRSMatrix:
    """Range-CRS Boolean matrix (RangeDynamic spec)."""

    def __init__(self, ncols=0, entries=None, rowmap=None, nnz=0, size_type=np.uint64):
        # CRSMatrix(ncols, e_entries, e_rowmap, e_nnz=0), crs_matrix.hpp:1894-1902:
        # a zero nnz is recounted from the entries.
        self.size_type = np.dtype(size_type)
        self.num_cols = int(ncols)
        self.entries = np.zeros(0, np.uint32) if entries is None else np.ascontiguousarray(entries, dtype=np.uint32)
        self.rowmap = (np.zeros(1, self.size_type) if rowmap is None
                       else np.ascontiguousarray(rowmap, dtype=self.size_type))
        self.m_nnz = int(nnz) if nnz else self._count_nnz()

    # -- accessors, crs_matrix.hpp:1274-1369 ---------------------------------
    def numRows(self):
        return len(self.rowmap) - 1

    def numCols(self):
        return self.num_cols

    def nnz(self):
        return self.m_nnz

    def rowMap(self, i):
        return int(self.rowmap[i])

    def entry(self, i):
        return int(self.entries[i])

    def get_entries(self):
        return self.entries

    def get_rowmap(self):
        return self.rowmap

    def _count_nnz(self):
        # crs_matrix::nnz(..., RangeGroup), crs_matrix.hpp:175-189
        e = self.entries.astype(np.int64)
        return int((e[1::2] - e[0::2] + 1).sum()) if len(e) else 0

    # -- membership, crs_matrix.hpp:1197-1243 and :149-169 ---------------------
    def __call__(self, i, j):
        lo, hi = int(self.rowmap[i]), int(self.rowmap[i + 1])
        row = self.entries[lo:hi]
        k = int(np.searchsorted(row, j, side="left"))  # lower_bound
        if k % 2:
            k -= 1
        return bool(k != len(row) and row[k] <= j)

    def at(self, i, j):
        if i >= self.numRows() or j >= self.numCols():
            raise IndexError("index out of range")
        return self(i, j)

    def size_in_bytes(self):
        # CRSMatrixTraits<RangeDynamic>::size_in_bytes, crs_matrix.hpp:893-898
        return self.entries.size * 4 + self.rowmap.size * self.size_type.itemsize + 4 + self.size_type.itemsize

    def __eq__(self, other):
        return (isinstance(other, CRSMatrix) and self.num_cols == other.num_cols and self.m_nnz == other.m_nnz
                and np.array_equal(self.rowmap.astype(np.uint64), other.rowmap.astype(np.uint64))
                and np.array_equal(self.entries, other.entries))

    # -- on-disk format: CRSMatrixBase::serialize/load (crs_matrix.hpp:1392-1409)
    # and the RangeDynamic nnz trailer (:1986-2000); containers are a uint64
    # size followed by raw elements (utils.hpp:191-289) --------------------------
    def serialize(self, f):
        f.write(struct.pack("<Q", self.entries.size))
        f.write(self.entries.astype("<u4").tobytes())
        f.write(struct.pack("<Q", self.rowmap.size))
        f.write(self.rowmap.astype(self.size_type.newbyteorder("<")).tobytes())
        f.write(struct.pack("<Q", self.num_cols))
        f.write(struct.pack("<Q", self.m_nnz))

    @classmethod
    def load(cls, f, size_type=np.uint64):
        st = np.dtype(size_type)
        (ne,) = struct.unpack("<Q", f.read(8))
        entries = np.frombuffer(f.read(4 * ne), dtype="<u4").astype(np.uint32)
        (nr,) = struct.unpack("<Q", f.read(8))
        rowmap = np.frombuffer(f.read(st.itemsize * nr), dtype=st.newbyteorder("<")).astype(st)
        (ncols,) = struct.unpack("<Q", f.read(8))
        (nnz,) = struct.unpack("<Q", f.read(8))
        m = cls(ncols, entries, rowmap, 1, size_type=st)
        m.m_nnz = int(nnz)
        return m

    def __repr__(self):
        return (f"CRSMatrix<RangeDynamic>({self.numRows()}x{self.numCols()}, ranges={self.entries.size // 2}, "
                f"nnz={self.m_nnz})")


def from_basic(nrows, ncols, rowmap, cols, size_type=np.uint64):
    """Basic (one column per entry) -> range CRS, as crs_matrix::append
    (crs_matrix.hpp:197-242): consecutive columns extend the open range."""
    out_rowmap = np.zeros(nrows + 1, dtype=np.uint64)
    ent = []
    for i in range(nrows):
        pending = False
        pend = 0
        for k in range(int(rowmap[i]), int(rowmap[i + 1])):
            c = int(cols[k])
            if pending and c == pend + 1:
                pend += 1
                continue
            if pending:
                ent.append(pend)
            ent.append(c)
            pend = c
            pending = True
        if pending:
            ent.append(pend)
        out_rowmap[i + 1] = len(ent)
    return CRSMatrix(ncols, np.array(ent, dtype=np.uint32), out_rowmap.astype(size_type), int(rowmap[nrows]),
                     size_type=size_type)
