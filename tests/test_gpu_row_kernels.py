"""The thread-per-row range-SpGEMM slot (k_spgemm_rowmode) against the CPU
oracle, exactly, on shapes that stress its chunk machinery: full and partial
chunks of every size, bands from a few columns to thousands, chunks with more
A ranges than its A stage holds, rows that overflow the run list (warp path
and the per-thread path past it), the identity as A (shifted, as union levels
use it), empty rows and planned index builds."""
import numpy as np
import pytest

from oracle import pyoracle as orc
from diverg_b200 import CRSMatrix, gen
from diverg_b200.runtime import Context

pytestmark = pytest.mark.gpu

SLOTS = [1, 0]  # run-list width variants: 24 entries (the default), 16


@pytest.fixture(scope="module")
def ctx():
    c = Context(0)
    yield c
    c.close()


def omat(m):
    return orc.OMat(m.numRows(), m.numCols(), np.asarray(m.rowmap, dtype=np.uint64), m.entries, m.nnz())


def assert_same(got, want, what=""):
    assert np.array_equal(got.rowmap.astype(np.uint64), want.rowmap), what + ": rowmap"
    assert np.array_equal(got.entries, want.entries), what + ": entries"
    assert got.nnz() == int(want.nnz), what + ": nnz"


def use(ctx, slot, chunk_rows=0, mode=2):
    ctx.set_option("row_slot", slot)
    ctx.set_option("chunk_rows", chunk_rows)
    ctx.set_option("spgemm_mode", mode)


@pytest.fixture(autouse=True)
def restore(ctx):
    yield
    use(ctx, 1, 0, 0)
    ctx.set_option("spgemm_levels", 1)


def product(ctx, a, b, slot, chunk_rows=0):
    use(ctx, slot, chunk_rows)
    ctx.reset_stats()
    got = ctx.spgemm(ctx.upload(a), ctx.upload(b)).download()
    st = ctx.stats()
    # a product whose speculative output capacity overflows runs twice
    assert st["spgemm_light"] == 1 + st["spgemm_reruns"], st
    return got, st


@pytest.mark.parametrize("slot", SLOTS)
@pytest.mark.parametrize("chunk_rows", [0, 32, 96, 1024, 2048])
def test_graph_power_products(ctx, slot, chunk_rows):
    # rows near their own columns: windows of about a chunk of B rows
    a, _ = gen.graph_adjacency(gen.small_graph_spec(50_000, seed=21))
    a4 = ctx.power(ctx.upload(a), 4).download()
    want = orc.spgemm(omat(a4), omat(a4))
    got, _ = product(ctx, a4, a4, slot, chunk_rows)
    assert_same(got, want, f"A^4 A^4, chunk {chunk_rows}")


@pytest.mark.parametrize("slot", SLOTS)
@pytest.mark.parametrize("hw,ranges,length", [(16, 1.0, 1.0), (600, 2.0, 2.0), (3000, 1.5, 1.0), (200, 6.0, 3.0)])
def test_banded_windows_clipped_by_rows_and_ranges(ctx, slot, hw, ranges, length):
    # half-widths past the window's row capacity, and B rows dense enough
    # that the window is cut by its range capacity
    a = gen.banded(40_000, hw, ranges, length, seed=31)
    b = gen.banded(40_000, 64, 5.0, 3.0, seed=32)
    want = orc.spgemm(omat(a), omat(b))
    got, _ = product(ctx, a, b, slot, 2048)
    assert_same(got, want, f"banded hw {hw}")


@pytest.mark.parametrize("slot", SLOTS)
def test_chunks_with_more_ranges_than_the_stages(ctx, slot):
    # A rows of ~3 ranges: a 2048-row chunk has more A ranges than its stage
    # holds, so its last rows read A from HBM
    a = gen.banded(30_000, 48, 3.0, 1.0, seed=41)
    b = gen.banded(30_000, 48, 1.0, 1.0, seed=42)
    want = orc.spgemm(omat(a), omat(b))
    got, _ = product(ctx, a, b, slot, 2048)
    assert_same(got, want)


@pytest.mark.parametrize("slot", SLOTS)
def test_rows_past_the_run_list(ctx, slot):
    # random columns: rows of many runs take the warp path, and past its
    # per-chunk list the per-thread path
    a = gen.random_matrix(6000, 30000, seed=43)
    want = orc.spgemm(omat(a), omat(a))
    got, st = product(ctx, a, a, slot, 2048)
    assert_same(got, want)
    assert st["spgemm_slow_rows"] > 512


@pytest.mark.parametrize("slot", SLOTS)
@pytest.mark.parametrize("window", [(100, 300), (0, 40), (7, 7)])
def test_index_builds(ctx, slot, window):
    # planned builds: C = D + A B sums, the identity as addend and as A
    a, _ = gen.graph_adjacency(gen.small_graph_spec(80_000, seed=44))
    want = orc.dindex(omat(a), *window, algo="hbv")
    use(ctx, slot, 0, 0)
    ctx.reset_stats()
    got = ctx.distance_index(ctx.upload(a), *window).download()
    st = ctx.stats()
    assert_same(got, want, str(window))
    assert st["spgemm_light"] > 0


@pytest.mark.parametrize("slot", SLOTS)
def test_union_levels_use_the_shifted_identity(ctx, slot):
    # long A ranges: union levels of B are built by the row slot with A the
    # identity shifted by 2^(k-1) rows; the product then reads the levels
    use(ctx, slot, 0, 2)
    a = gen.banded(40_000, 512, 3.0, 6.0, seed=45)
    b = gen.banded(40_000, 256, 4.0, 8.0, seed=46)
    want = orc.spgemm(omat(a), omat(b))
    ctx.reset_stats()
    got = ctx.spgemm(ctx.upload(a), ctx.upload(b)).download()
    st = ctx.stats()
    assert_same(got, want)
    assert st["spgemm_levels"] > 0


@pytest.mark.parametrize("slot", SLOTS)
def test_empty_rows_and_tiny_products(ctx, slot):
    one = CRSMatrix(5, np.array([0, 0, 2, 4], np.uint32), np.array([0, 2, 2, 2, 4, 4], np.uint64))
    want = orc.spgemm(omat(one), omat(one))
    got, _ = product(ctx, one, one, slot)
    assert_same(got, want)
    empty = CRSMatrix(7, np.zeros(0, np.uint32), np.zeros(8, np.uint64))
    got, _ = product(ctx, empty, empty, slot)
    assert got.entries.size == 0 and got.nnz() == 0
