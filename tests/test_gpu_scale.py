"""Parity at the sizes the benchmark quotes: the chromosome-scale index build
(5e7 backbone bases, window [400, 600], seed 42: 50,107,913 loci), the
range-SpGEMM / SpAdd microbenchmark matrices (n = 2^24, band half-width 512)
and the 2,000-graph batch.  Every comparison is exact (integer data): rowmap,
entries and nnz against the CPU oracle (the bitvector restatement of the
reference's path, util::create_distance_index dindex.hpp:46-189 on the
reference's own squaring schedule), batched indices against their plain
builds."""
import numpy as np
import pytest

from oracle import pyoracle as orc
from diverg_b200 import gen
from diverg_b200.runtime import Context

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = Context(0)
    yield c
    c.close()


def omat(m):
    return orc.OMat(m.numRows(), m.numCols(), np.asarray(m.rowmap, dtype=np.uint64), m.entries, m.nnz())


def assert_same(got, want, what):
    assert got.numRows() == want.nrows, what
    assert np.array_equal(got.rowmap.astype(np.uint64), want.rowmap), what + ": rowmap"
    assert np.array_equal(got.entries, want.entries), what + ": entries"
    assert got.nnz() == int(want.nnz), what + ": nnz"


def test_chromosome_scale_index_is_bit_exact(ctx):
    a, st = gen.graph_adjacency(gen.chromosome_graph_spec(50_000_000, seed=42))
    assert a.numRows() == 50_107_913
    d_a = ctx.upload(a)
    d_idx = ctx.distance_index(d_a, 400, 600)
    got = d_idx.download()
    d_idx.free()
    d_a.free()
    want = orc.dindex(omat(a), 400, 600, algo="hbv")
    assert_same(got, want, "5e7-base index [400,600]")
    # answers of the resident index equal the oracle's on pairs in and out of the window
    d_a = ctx.upload(a)
    d_idx = ctx.distance_index(d_a, 400, 600)
    pairs = gen.query_pairs(a, 200_000, 0.5, 400, 600, seed=3)
    assert np.array_equal(ctx.query(d_idx, pairs), orc.query(want, pairs))
    d_idx.free()
    d_a.free()


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_microbenchmark_spgemm_at_full_size(ctx, mode):
    n = 1 << 24
    a = gen.banded(n, 512, 4.0, 32.0, seed=42)
    b = gen.banded(n, 512, 4.0, 32.0, seed=43)
    want = orc.spgemm(omat(a), omat(b), algo="hbv")
    ctx.set_option("spgemm_mode", mode)
    try:
        da, db = ctx.upload(a), ctx.upload(b)
        c = ctx.spgemm(da, db)
        got = c.download()
        c.free()
        da.free()
        db.free()
    finally:
        ctx.set_option("spgemm_mode", 0)
    assert_same(got, want, f"banded 2^24 spgemm, mode {mode}")


def test_microbenchmark_spadd_at_full_size(ctx):
    n = 1 << 24
    a = gen.banded(n, 512, 4.0, 32.0, seed=42)
    b = gen.banded(n, 512, 4.0, 32.0, seed=43)
    want = orc.spadd(omat(a), omat(b))
    da, db = ctx.upload(a), ctx.upload(b)
    c = ctx.spadd(da, db)
    got = c.download()
    c.free()
    da.free()
    db.free()
    assert_same(got, want, "banded 2^24 spadd")


def test_two_thousand_graph_batch_equals_plain_builds(ctx):
    rng = np.random.default_rng(42)
    count = 2000
    sizes = np.clip(rng.lognormal(np.log(2e4), 1.0, count), 1e3, 1e6).astype(np.int64)
    wins = [(100, 300), (200, 500), (400, 600)]
    windows = [wins[int(i)] for i in rng.integers(0, 3, count)]
    graphs = [gen.graph_adjacency(gen.small_graph_spec(int(n), seed=42 + k))[0] for k, n in enumerate(sizes)]
    dg = [ctx.upload(g) for g in graphs]
    outs = ctx.batch_distance_index(dg, windows)
    for k, (d, w) in enumerate(zip(dg, windows)):
        mine = outs[k].download()
        alone = ctx.distance_index(d, *w)
        plain = alone.download()
        alone.free()
        assert np.array_equal(mine.rowmap, plain.rowmap) and np.array_equal(mine.entries, plain.entries), k
        assert mine.nnz() == plain.nnz(), k
        if k % 20 == 0:
            assert_same(mine, orc.dindex(omat(graphs[k]), *w, algo="hbv"), f"graph {k}")
        outs[k].free()
        d.free()
