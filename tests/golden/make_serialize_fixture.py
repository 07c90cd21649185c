"""Writes tests/golden/rangedynamic_x_1_8_u64.bin and ..._u32.bin: the on-disk
form of a RangeDynamic range-CRS matrix -- the distance index [1, 8] of the
reference's test graph test/data/small/x.gfa, as stored in gfa_x.npz -- in
the reference's layout, by a writer that shares no code with the library:

    CRSMatrixBase::serialize (crs_matrix.hpp:1392-1400): entries, then rowmap,
        each a container = uint64 element count followed by the raw elements
        (diverg::serialize of a std::vector, utils.hpp:191-289, size type
        DefaultContainerSize = uint64_t, utils.hpp:181), then num_cols as
        uint64;
    CRSMatrix<RangeDynamic>::serialize (crs_matrix.hpp:1986-1991): then m_nnz
        as uint64.

Entries are uint32 (the ordinal type), rowmap words uint64 or uint32 (the size
type); every integer little-endian (x86-64).  Run from the repository root:

    python tests/golden/make_serialize_fixture.py
"""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def reference_layout(ncols, nnz, entries, rowmap, size_bytes):
    """The bytes of the reference's serialize, element by element."""
    out = bytearray()
    out += int(len(entries)).to_bytes(8, "little")
    for v in entries:
        out += int(v).to_bytes(4, "little")
    out += int(len(rowmap)).to_bytes(8, "little")
    for v in rowmap:
        out += int(v).to_bytes(size_bytes, "little")
    out += int(ncols).to_bytes(8, "little")
    out += int(nnz).to_bytes(8, "little")
    return bytes(out)


def fixture_matrix():
    with np.load(os.path.join(HERE, "gfa_x.npz")) as z:
        return int(z["n"]), int(z["D1_8_nnz"]), z["D1_8_entries"].astype(np.uint32), z["D1_8_rowmap"].astype(np.uint64)


if __name__ == "__main__":
    ncols, nnz, entries, rowmap = fixture_matrix()
    for tag, size in (("u64", 8), ("u32", 4)):
        with open(os.path.join(HERE, f"rangedynamic_x_1_8_{tag}.bin"), "wb") as f:
            f.write(reference_layout(ncols, nnz, entries, rowmap, size))
