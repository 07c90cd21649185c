"""The compressed range-CRS container (CRSMatrix<RangeCompressed>, Elias-delta
coded entries and rowmap; include/diverg/crs_matrix.hpp and enc_vector.hpp)
against its mutable source, compiled here on its own: row pointers, entries,
membership on random and boundary pairs, decompression and serialise/load
round trips on random matrices, empty and extreme ones, and the
reference-layout fixture of the distance index [1, 8] of small/x.gfa, whose
bytes must come back unchanged through compression."""
import os
import subprocess

from tests.conftest import GOLDEN, ROOT


def test_compressed_container(tmp_path):
    exe = str(tmp_path / "compressed_test")
    subprocess.run(["g++", "-O2", "-std=c++17", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"),
                    "-o", exe, os.path.join(ROOT, "tests", "cpp", "compressed_test.cpp")], check=True)
    out = subprocess.run([exe, os.path.join(GOLDEN, "rangedynamic_x_1_8_u64.bin")], capture_output=True,
                         text=True, timeout=300)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout + out.stderr
