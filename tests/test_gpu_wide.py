"""The warp-per-row SpGEMM (spgemm_mode 3, and the automatic choice for long A
ranges) against the oracle, exactly: banded products of the microbenchmark's
shape, rows of more than 32 A ranges, rows wider than one bitmap window,
chunks whose output exceeds the shared image, rows whose runs exceed a warp's
buffer, non-canonical operands, and fused sums D + A B through the read-back
index schedule."""
import numpy as np
import pytest

from oracle import pyoracle as orc
from diverg_b200 import CRSMatrix, gen
from diverg_b200.runtime import Context

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = Context(0)
    yield c
    c.close()


@pytest.fixture(autouse=True)
def restore(ctx):
    yield
    ctx.set_option("spgemm_mode", 0)
    ctx.set_option("planned_build", 1)


def omat(m):
    return orc.OMat(m.numRows(), m.numCols(), np.asarray(m.rowmap, dtype=np.uint64), m.entries, m.nnz())


def assert_same(got, want, what=""):
    assert np.array_equal(got.rowmap.astype(np.uint64), want.rowmap), what + ": rowmap"
    assert np.array_equal(got.entries, want.entries), what + ": entries"
    assert got.nnz() == int(want.nnz), what + ": nnz"


def product(ctx, a, b, mode=3):
    ctx.set_option("spgemm_mode", mode)
    return ctx.spgemm(ctx.upload(a), ctx.upload(b)).download()


def from_rows(rows, ncols):
    rowmap = [0]
    entries = []
    for r in rows:
        for lo, hi in r:
            entries += [lo, hi]
        rowmap.append(len(entries))
    nnz = sum(hi - lo + 1 for r in rows for lo, hi in r if hi >= lo)
    return CRSMatrix(ncols, np.array(entries, np.uint32), np.array(rowmap, np.uint64), nnz)


@pytest.mark.parametrize("mode", [0, 3])
@pytest.mark.parametrize("n,hw,ranges,length", [(1 << 16, 512, 4.0, 32.0), (1 << 14, 64, 2.0, 8.0),
                                                 (5000, 2000, 8.0, 200.0)])
def test_banded_products(ctx, mode, n, hw, ranges, length):
    a = gen.banded(n, hw, ranges, length, seed=5)
    b = gen.banded(n, hw, ranges, length, seed=6)
    assert_same(product(ctx, a, b, mode), orc.spgemm(omat(a), omat(b)), f"banded {n} {hw} mode {mode}")


def test_rows_of_many_a_ranges(ctx):
    # about 100 ranges an A row: several groups of 32 slices a row
    a = gen.random_matrix(2000, 200_000, seed=7)
    b = gen.random_matrix(2000, 20_000, seed=8)
    assert_same(product(ctx, a, b), orc.spgemm(omat(a), omat(b)), "random 2000")


def test_rows_wider_than_a_window_and_long_ranges(ctx):
    # B rows spanning up to 40,000 columns: several 4,096-column windows a row,
    # ranges covering many words whole
    rng = np.random.default_rng(9)
    n, ncols = 700, 60_000
    brows = []
    for i in range(n):
        k = int(rng.integers(0, 6))
        starts = np.sort(rng.integers(0, ncols - 1, k))
        brows.append([(int(s), int(min(ncols - 1, s + rng.integers(0, 9000)))) for s in starts])
    b = from_rows(brows, ncols)
    arows = [[(int(s), int(min(n - 1, s + rng.integers(0, 12))))] for s in rng.integers(0, n, n)]
    a = from_rows(arows, n)
    assert_same(product(ctx, a, b), orc.spgemm(omat(a), omat(b)), "wide rows")


def test_chunks_beyond_the_image_and_rows_beyond_the_buffer(ctx):
    # rows of up to ~600 runs (a warp's buffer holds 256 entries, a chunk's
    # image 2,048): the in-place write-out and the second walk
    rng = np.random.default_rng(10)
    n, ncols = 300, 200_000
    brows = []
    for i in range(n):
        cols = np.sort(rng.choice(ncols // 2, int(rng.integers(0, 300)), replace=False)) * 2
        brows.append([(int(c), int(c)) for c in cols])
    b = from_rows(brows, ncols)
    arows = [[(i, min(n - 1, i + 3))] if i % 5 == 0 else [(i, i)] for i in range(n)]
    a = from_rows(arows, n)
    assert_same(product(ctx, a, b), orc.spgemm(omat(a), omat(b)), "many runs")


def test_empty_rows_empty_and_overlapping_ranges(ctx):
    # empty A rows, empty B rows, ranges given out of order and overlapping
    a = from_rows([[], [(0, 3)], [(2, 2), (0, 1)], [(3, 3), (1, 2)], []], 5)
    b = from_rows([[(10, 20), (5, 12)], [], [(40, 41), (30, 35), (36, 39)], [(0, 0)], [(7, 7)]], 64)
    assert_same(product(ctx, a, b), orc.spgemm(omat(a), omat(b)), "small")


@pytest.mark.parametrize("window", [(0, 20), (3, 40)])
def test_fused_sums_through_the_readback_schedule(ctx, window):
    # planned builds off: the index schedule's sums D + P_m R run on this kernel
    ctx.set_option("planned_build", 0)
    ctx.set_option("spgemm_mode", 3)
    a, _ = gen.graph_adjacency(gen.small_graph_spec(20_000, seed=11))
    got = ctx.distance_index(ctx.upload(a), *window).download()
    assert_same(got, orc.dindex(omat(a), *window, algo="hbv"), f"index {window}")


def test_automatic_choice_takes_the_warp_per_row_kernel(ctx):
    # the automatic choice on long ranges takes this kernel: one launch a product
    a = gen.banded(1 << 15, 512, 4.0, 32.0, seed=12)
    ctx.set_option("spgemm_mode", 0)
    ctx.reset_stats()
    ctx.spgemm(ctx.upload(a), ctx.upload(a)).free()
    st = ctx.stats()
    assert st["spgemm_calls"] == 1 and st["spgemm_light"] == 0 and st["spgemm_levels"] == 0, st


def test_range_operation_calibration(ctx):
    # the on-chip denominator: positive and finite, and the context computes
    # correctly afterwards
    rate = ctx.calibrate_range_ops()
    assert np.isfinite(rate) and 1e9 < rate < 1e14, rate
    a = gen.banded(1 << 12, 64, 4.0, 16.0, seed=13)
    assert_same(product(ctx, a, a), orc.spgemm(omat(a), omat(a)), "after calibration")
