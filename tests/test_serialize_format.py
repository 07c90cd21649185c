"""The on-disk form of RangeDynamic range-CRS matrices, byte for byte.

The committed fixtures tests/golden/rangedynamic_x_1_8_{u64,u32}.bin hold the
distance index [1, 8] of the reference's test graph small/x.gfa in the
reference's layout, written by tests/golden/make_serialize_fixture.py -- an
element-by-element writer that shares no code with the library -- following
CRSMatrixBase::serialize (crs_matrix.hpp:1392-1409), the RangeDynamic nnz
trailer (:1986-2000) and the container format of utils.hpp:181-289 (a uint64
count, then the raw elements).  Both drop-in containers must write exactly
those bytes and read them back: the Python mirror (diverg_b200.CRSMatrix) and
the C++ header (include/diverg/crs_matrix.hpp, compiled here on its own)."""
import io
import os
import subprocess

import numpy as np
import pytest

from diverg_b200 import CRSMatrix
from tests.conftest import GOLDEN, ROOT

import importlib.util

_spec = importlib.util.spec_from_file_location("make_serialize_fixture",
                                               os.path.join(GOLDEN, "make_serialize_fixture.py"))
_fix = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(_fix)

SIZES = [("u64", np.uint64, 8), ("u32", np.uint32, 4)]


def fixture_bytes(tag):
    with open(os.path.join(GOLDEN, f"rangedynamic_x_1_8_{tag}.bin"), "rb") as f:
        return f.read()


@pytest.mark.parametrize("tag,st,size", SIZES)
def test_fixture_is_the_reference_layout(tag, st, size):
    ncols, nnz, entries, rowmap = _fix.fixture_matrix()
    data = fixture_bytes(tag)
    assert data == _fix.reference_layout(ncols, nnz, entries, rowmap, size)
    # spot-check the header words by hand: entry count first, rowmap count after the entries
    assert int.from_bytes(data[:8], "little") == entries.size
    off = 8 + 4 * entries.size
    assert int.from_bytes(data[off:off + 8], "little") == rowmap.size
    assert len(data) == 8 + 4 * entries.size + 8 + size * rowmap.size + 16
    assert int.from_bytes(data[-16:-8], "little") == ncols and int.from_bytes(data[-8:], "little") == nnz


@pytest.mark.parametrize("tag,st,size", SIZES)
def test_python_container_writes_and_reads_the_fixture(tag, st, size):
    ncols, nnz, entries, rowmap = _fix.fixture_matrix()
    m = CRSMatrix(ncols, entries, rowmap.astype(st), nnz, size_type=st)
    buf = io.BytesIO()
    m.serialize(buf)
    assert buf.getvalue() == fixture_bytes(tag)
    back = CRSMatrix.load(io.BytesIO(fixture_bytes(tag)), size_type=st)
    assert back.numCols() == ncols and back.nnz() == nnz
    assert np.array_equal(back.entries, entries) and np.array_equal(back.rowmap.astype(np.uint64), rowmap)


@pytest.fixture(scope="module")
def dump_tool(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("ser") / "serialize_dump")
    subprocess.run(["g++", "-O1", "-std=c++17", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"),
                    "-o", exe, os.path.join(ROOT, "tests", "cpp", "serialize_dump.cpp")], check=True)
    return exe


@pytest.mark.parametrize("tag,st,size", SIZES)
def test_cpp_container_writes_and_reads_the_fixture(dump_tool, tmp_path, tag, st, size):
    ncols, nnz, entries, rowmap = _fix.fixture_matrix()
    e_path, r_path = tmp_path / "e.bin", tmp_path / "r.bin"
    e_path.write_bytes(entries.astype("<u4").tobytes())
    r_path.write_bytes(rowmap.astype("<u8").tobytes())
    out = tmp_path / "out.bin"
    subprocess.run([dump_tool, "write", tag, str(ncols), str(nnz), str(e_path), str(r_path), str(out)], check=True)
    assert out.read_bytes() == fixture_bytes(tag)
    fix = tmp_path / "fix.bin"
    fix.write_bytes(fixture_bytes(tag))
    again = tmp_path / "again.bin"
    subprocess.run([dump_tool, "reload", tag, str(fix), str(again)], check=True)
    assert again.read_bytes() == fixture_bytes(tag)
