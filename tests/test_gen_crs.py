"""Workload generators and the host CRSMatrix mirror (CPU only)."""
import io

import numpy as np
import pytest

from oracle import pyoracle as orc
from diverg_b200 import CRSMatrix, from_basic, gen


def canonical(m):
    for i in range(m.numRows()):
        e = m.entries[int(m.rowmap[i]):int(m.rowmap[i + 1])].astype(np.int64)
        if len(e) == 0:
            continue
        assert (e[1::2] >= e[0::2]).all()
        assert (e[2::2] > e[1:-1:2] + 1).all(), "ranges sorted, disjoint and non-adjacent"
    return True


@pytest.mark.parametrize("spec", [gen.small_graph_spec(20_000, seed=3),
                                  gen.chromosome_graph_spec(200_000, seed=5),
                                  gen.GraphSpec(5000, 0.05, 0.05, 0.5, 1, 10, 0.0, 0.2, 100, 300, 9)])
def test_graph_adjacency_matches_adjacency_layout(spec):
    # the generator's rows equal util::adjacency_matrix over the same graph
    # given as single-base nodes (adjacency.hpp:170-228, oracle restatement)
    a, st = gen.graph_adjacency(spec)
    n, edges = gen.graph_edges(spec)
    assert n == a.numRows() == st["n_loci"]
    ref = orc.adjacency(np.ones(n, np.uint32), edges)
    assert np.array_equal(ref.rowmap, a.rowmap) and np.array_equal(ref.entries, a.entries)
    assert ref.nnz == a.nnz()
    assert canonical(a)


def test_graph_is_deterministic_and_topological():
    s = gen.small_graph_spec(50_000, seed=11)
    a1, _ = gen.graph_adjacency(s)
    a2, _ = gen.graph_adjacency(s)
    assert a1 == a2
    # every edge points forward (topological numbering)
    rows = np.repeat(np.arange(a1.numRows()), np.diff(a1.rowmap.astype(np.int64)) // 2)
    assert (a1.entries[0::2] > rows).all()


def test_chromosome_spec_has_structural_bubbles():
    a, st = gen.graph_adjacency(gen.chromosome_graph_spec(5_000_000, seed=1))
    assert st["n_sv"] >= 1 and st["n_snp"] > 3000 and st["n_ins"] > 200 and st["n_del"] > 200


def test_banded_rows_are_canonical_and_in_band():
    m = gen.banded(1 << 14, 512, 4.0, 32.0, seed=3)
    assert canonical(m)
    rows = np.repeat(np.arange(m.numRows()), np.diff(m.rowmap.astype(np.int64)) // 2)
    assert (m.entries[0::2].astype(np.int64) >= rows - 512).all()
    assert (m.entries[1::2].astype(np.int64) <= rows + 512).all()
    assert m == gen.banded(1 << 14, 512, 4.0, 32.0, seed=3)


def test_random_matrix_exact_nnz():
    m = gen.random_matrix(6521, 200000, seed=1)
    assert m.nnz() == 200000 and canonical(m)
    assert CRSMatrix(m.numCols(), m.entries, m.rowmap).nnz() == 200000


def test_query_pairs_in_range_half():
    a, _ = gen.graph_adjacency(gen.small_graph_spec(20_000, seed=2))
    p = gen.query_pairs(a, 10_000, 1.0, 200, 500, seed=1)
    d = p[:, 1].astype(np.int64) - p[:, 0].astype(np.int64)
    assert (d >= 0).all() and np.median(d) > 150


def test_host_query_matches_oracle():
    m = gen.random_matrix(500, 20000, seed=4)
    rng = np.random.default_rng(1)
    pairs = rng.integers(0, 500, size=(5000, 2), dtype=np.uint32)
    want = orc.query(orc.OMat(500, 500, m.rowmap, m.entries, m.nnz()), pairs)
    got = np.array([m(int(i), int(j)) for i, j in pairs], dtype=np.uint8)
    assert np.array_equal(got, want)
    with pytest.raises(IndexError):
        m.at(500, 0)


@pytest.mark.parametrize("st", [np.uint64, np.uint32])
def test_serialize_roundtrip(st):
    m = gen.random_matrix(300, 4000, seed=6)
    m = CRSMatrix(m.numCols(), m.entries, m.rowmap.astype(st), m.nnz(), size_type=st)
    buf = io.BytesIO()
    m.serialize(buf)
    # entries(u64 size + u32s) rowmap(u64 size + TSize) ncols(u64) nnz(u64)
    assert len(buf.getvalue()) == 8 + 4 * m.entries.size + 8 + np.dtype(st).itemsize * m.rowmap.size + 16
    buf.seek(0)
    assert CRSMatrix.load(buf, size_type=st) == m


def test_from_basic_matches_oracle():
    rng = np.random.default_rng(3)
    rowmap = [0]
    cols = []
    for _ in range(200):
        c = np.sort(rng.choice(400, size=rng.integers(0, 40), replace=False))
        cols += list(c)
        rowmap.append(len(cols))
    rowmap = np.array(rowmap, np.uint64)
    cols = np.array(cols, np.uint32)
    m = from_basic(200, 400, rowmap, cols)
    o = orc.basic_to_range(200, 400, rowmap, cols)
    assert np.array_equal(m.rowmap, o.rowmap) and np.array_equal(m.entries, o.entries) and m.nnz() == o.nnz
