"""The CPU oracle against the reference's known answers, the GFA fixtures and
dense brute force (CPU only)."""
import numpy as np
import pytest

from oracle import pyoracle as orc
from diverg_b200 import gen
from tests.conftest import load_golden


def omat(m):
    return orc.OMat(m.numRows(), m.numCols(), m.rowmap.astype(np.uint64), m.entries, m.nnz())


def dense_mul(a, b):
    return (a.astype(np.float32) @ b.astype(np.float32)) > 0


@pytest.mark.parametrize("algo", ["btree", "hbv"])
def test_hbitvector_known_answer(algo):
    # test_hbitvector.cpp:186-234 -> :618-661, via C = I * A (row-wise union)
    ki = load_golden("hbv_known_answer.npz")
    a = orc.OMat(5, int(ki["ncols"]), ki["in_rowmap"], ki["in_entries"], 0)
    a.nnz = orc.nnz(a)
    c = orc.spgemm(orc.identity(5), a, algo=algo)
    assert np.array_equal(c.rowmap, ki["out_rowmap"])
    assert np.array_equal(c.entries, ki["out_entries"])


@pytest.mark.parametrize("name", ["x", "multi", "m"])
def test_gfa_fixtures(name):
    g = load_golden(f"gfa_{name}.npz")
    A = orc.adjacency(g["node_len"], g["edges"])
    assert np.array_equal(A.rowmap, g["A_rowmap"]) and np.array_equal(A.entries, g["A_entries"])
    for key in [k[:-7] for k in g if k.endswith("_rowmap") and k != "A_rowmap"]:
        if key == "AA":
            r = orc.spgemm(A, A, algo="hbv")
        elif key == "AI":
            r = orc.spadd(A, orc.identity(A.nrows))
        elif key.startswith("P"):
            r = orc.power(A, int(key[1:]), algo="hbv")
        else:
            lo, hi = map(int, key[1:].split("_"))
            r = orc.dindex(A, lo, hi, algo="hbv")
        assert np.array_equal(r.rowmap, g[key + "_rowmap"]), key
        assert np.array_equal(r.entries, g[key + "_entries"]), key
        assert r.nnz == int(g[key + "_nnz"]), key


@pytest.mark.parametrize("n,nnz,seed", [(20, 220, 1), (200, 3000, 2), (300, 400, 3), (1000, 20000, 4)])
def test_products_vs_dense(n, nnz, seed):
    a = omat(gen.random_matrix(n, nnz, seed))
    b = omat(gen.random_matrix(n, nnz, seed + 100))
    da, db = orc.to_dense(a), orc.to_dense(b)
    for algo in ("btree", "hbv"):
        c = orc.spgemm(a, b, algo=algo)
        assert c.same(orc.from_dense(dense_mul(da, db)))
    s = orc.spadd(a, b)
    assert s.same(orc.from_dense(da | db))


def test_power_vs_dense():
    a = omat(gen.random_matrix(400, 500, 9))
    d = orc.to_dense(a)
    for k in (0, 1, 2, 3, 7, 100):
        want = orc.from_dense(orc.dense_power(d, k))
        for algo in ("btree", "hbv"):
            got = orc.power(a, k, algo=algo)
            assert np.array_equal(got.rowmap, want.rowmap) and np.array_equal(got.entries, want.entries), k
            assert got.nnz == want.nnz


def test_reference_test_shapes_btree_equals_hbv():
    # test_range_sparse.cpp:516-520 (SpGEMM N=6521 NNZ=200000), :590-594 (power K=100)
    a = omat(gen.random_matrix(6521, 200000, 11))
    assert orc.spgemm(a, a, algo="btree").same(orc.spgemm(a, a, algo="hbv"))
    p = omat(gen.random_matrix(6521, 4000, 12))
    assert orc.power(p, 100, algo="btree").same(orc.power(p, 100, algo="hbv"))


def test_spadd_noncanonical_rest_is_copied_verbatim():
    # range_sparse.hpp:352-355: once one row runs out, the other is copied as is
    a = orc.OMat(1, 100, np.array([0, 2], np.uint64), np.array([5, 6], np.uint32), 2)
    b = orc.OMat(1, 100, np.array([0, 4], np.uint64), np.array([10, 11, 12, 13], np.uint32), 4)
    c = orc.spadd(a, b)
    assert list(c.entries) == [5, 6, 10, 11, 12, 13]


def test_query_vs_dense():
    a = omat(gen.random_matrix(300, 5000, 5))
    d = orc.to_dense(a)
    rng = np.random.default_rng(0)
    pairs = rng.integers(0, 300, size=(20000, 2), dtype=np.uint32)
    got = orc.query(a, pairs)
    assert np.array_equal(got.astype(bool), d[pairs[:, 0], pairs[:, 1]])


def test_word_boundary_runs():
    # runs that end on the last bit of a 64-bit word and start on the next
    ent = np.array([0, 63, 64, 64, 127, 127, 190, 255], np.uint32)
    b = orc.OMat(1, 256, np.array([0, len(ent)], np.uint64), ent, 0)
    b.nnz = orc.nnz(b)
    for algo in ("btree", "hbv"):
        c = orc.spgemm(orc.identity(1), b, algo=algo)
        assert list(c.entries) == [0, 64, 127, 127, 190, 255]
        assert c.nnz == 65 + 1 + 66


def test_dindex_rejects_bad_window():
    a = orc.identity(4)
    with pytest.raises(ValueError):
        orc.dindex(a, 3, 2)
    with pytest.raises(ValueError):
        orc.dindex(a, 0, 0)
