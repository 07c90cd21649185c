"""Parity of the sm_100a path (through the C ABI of libdvg.so) with the CPU
oracle and the golden fixtures.  Integer work: every comparison is exact."""
import numpy as np
import pytest

from oracle import pyoracle as orc
from diverg_b200 import CRSMatrix, _native as N, gen
from diverg_b200.runtime import Context
from tests.conftest import load_golden

pytestmark = pytest.mark.gpu

# (algo, group lanes, window words, SpGEMM mode): the single-pass kernels in
# their automatic choice, the tile-staged rows, the thread-per-row mode and
# the warp-per-row mode
FUSED = [(0, 0, 0, 0), (0, 0, 0, 1), (0, 0, 0, 2), (0, 0, 0, 3)]
PLANS = FUSED


@pytest.fixture(scope="module")
def ctx():
    c = Context(0)
    yield c
    c.close()


def set_plan(ctx, plan, chunk_rows=0):
    ctx.set_option("spgemm_mode", plan[3] if len(plan) > 3 else 0)
    ctx.set_option("chunk_rows", chunk_rows)


def as_crs(o):
    return CRSMatrix(o.ncols, o.entries, o.rowmap, o.nnz)


def omat(m):
    return orc.OMat(m.numRows(), m.numCols(), m.rowmap.astype(np.uint64), m.entries, m.nnz())


def assert_same(got: CRSMatrix, rowmap, entries, nnz, what=""):
    assert np.array_equal(got.rowmap.astype(np.uint64), np.asarray(rowmap, np.uint64)), what
    assert np.array_equal(got.entries, np.asarray(entries, np.uint32)), what
    assert got.nnz() == int(nnz), what


@pytest.mark.parametrize("plan", PLANS)
def test_hbitvector_known_answer(ctx, plan):
    # test_hbitvector.cpp:186-234 -> :618-661: I * A canonicalises A's rows
    set_plan(ctx, plan)
    ki = load_golden("hbv_known_answer.npz")
    a = ctx.upload(CRSMatrix(int(ki["ncols"]), ki["in_entries"], ki["in_rowmap"]))
    i5 = ctx.identity(5)
    c = ctx.spgemm(i5, a).download()
    assert_same(c, ki["out_rowmap"], ki["out_entries"], orc.nnz(orc.OMat(5, 11431, ki["out_rowmap"],
                                                                          ki["out_entries"], 0)))


@pytest.mark.parametrize("name", ["x", "multi", "m"])
@pytest.mark.parametrize("plan", FUSED)
def test_gfa_fixture_products(ctx, name, plan):
    set_plan(ctx, plan)
    g = load_golden(f"gfa_{name}.npz")
    n = int(g["n"])
    A = CRSMatrix(n, g["A_entries"], g["A_rowmap"], int(g["A_nnz"]))
    dA = ctx.upload(A)
    for key in [k[:-7] for k in g if k.endswith("_rowmap") and k != "A_rowmap"]:
        if key == "AA":
            r = ctx.spgemm(dA, dA)
        elif key == "AI":
            r = ctx.spadd(dA, ctx.identity(n))
        elif key.startswith("P"):
            r = ctx.power(dA, int(key[1:]))
        else:
            lo, hi = map(int, key[1:].split("_"))
            r = ctx.distance_index(dA, lo, hi)
        assert_same(r.download(), g[key + "_rowmap"], g[key + "_entries"], g[key + "_nnz"], f"{name} {key}")


@pytest.mark.parametrize("plan", PLANS)
def test_random_spgemm_reference_shape(ctx, plan):
    # test_range_sparse.cpp:516-520: N = 6521, NNZ = 200000, A * A
    set_plan(ctx, plan)
    a = gen.random_matrix(6521, 200000, seed=21)
    want = orc.spgemm(omat(a), omat(a), algo="hbv")
    da = ctx.upload(a)
    assert_same(ctx.spgemm(da, da).download(), want.rowmap, want.entries, want.nnz)


@pytest.mark.parametrize("plan", FUSED)
def test_random_power_reference_shape(ctx, plan):
    # test_range_sparse.cpp:590-594: N = 6521, NNZ = 4000, K = 100
    set_plan(ctx, plan)
    a = gen.random_matrix(6521, 4000, seed=22)
    want = orc.power(omat(a), 100, algo="hbv")
    assert_same(ctx.power(ctx.upload(a), 100).download(), want.rowmap, want.entries, want.nnz)


@pytest.mark.parametrize("n,nnz", [(6521, 4000), (20, 220), (5000, 300000)])
def test_random_spadd_reference_shapes(ctx, n, nnz):
    # test_range_sparse.cpp:664-665
    a = gen.random_matrix(n, nnz, seed=23)
    b = gen.random_matrix(n, nnz, seed=24)
    want = orc.spadd(omat(a), omat(b))
    assert_same(ctx.spadd(ctx.upload(a), ctx.upload(b)).download(), want.rowmap, want.entries, want.nnz)


@pytest.mark.parametrize("plan", FUSED)
def test_rectangular_spgemm(ctx, plan):
    set_plan(ctx, plan)
    a = gen.random_matrix(3000, 30000, seed=5)
    b = gen.banded(3000, 64, 3.0, 16.0, seed=6)
    # a: 3000 x 3000, b: 3000 x 3000 -> check A*B and B*A
    for x, y in ((a, b), (b, a)):
        want = orc.spgemm(omat(x), omat(y))
        assert_same(ctx.spgemm(ctx.upload(x), ctx.upload(y)).download(), want.rowmap, want.entries, want.nnz)


@pytest.mark.parametrize("plan", FUSED)
def test_banded_spgemm(ctx, plan):
    set_plan(ctx, plan)
    a = gen.banded(1 << 16, 512, 4.0, 32.0, seed=31)
    b = gen.banded(1 << 16, 512, 4.0, 32.0, seed=32)
    want = orc.spgemm(omat(a), omat(b), algo="hbv")
    assert_same(ctx.spgemm(ctx.upload(a), ctx.upload(b)).download(), want.rowmap, want.entries, want.nnz)
    want = orc.spadd(omat(a), omat(b))
    assert_same(ctx.spadd(ctx.upload(a), ctx.upload(b)).download(), want.rowmap, want.entries, want.nnz)


@pytest.mark.parametrize("plan,chunk_rows", [((0, 0, 0, 0), 0), ((0, 0, 0, 0), 2048), ((0, 0, 0, 1), 0),
                                             ((0, 0, 0, 2), 0), ((0, 0, 0, 2), 2048), ((1, 0, 0), 0)])
@pytest.mark.parametrize("schedule", [0, 1])
@pytest.mark.parametrize("window", [(100, 300), (0, 250), (150, 450), (1, 1), (7, 7), (0, 1), (3, 37), (0, 200)])
def test_small_graph_index(ctx, window, plan, chunk_rows, schedule):
    set_plan(ctx, plan, chunk_rows)
    ctx.set_option("dindex_schedule", schedule)
    a, _ = gen.graph_adjacency(gen.small_graph_spec(100_000, seed=42))
    want = orc.dindex(omat(a), window[0], window[1], algo="hbv")
    got = ctx.distance_index(ctx.upload(a), *window).download()
    assert_same(got, want.rowmap, want.entries, want.nnz, str(window))


@pytest.mark.parametrize("plan", FUSED)
@pytest.mark.parametrize("schedule", [0, 1])
def test_graph_with_structural_bubbles_index(ctx, plan, schedule):
    set_plan(ctx, plan)
    ctx.set_option("dindex_schedule", schedule)
    spec = gen.GraphSpec(60_000, 1e-3, 2e-4, 0.5, 1, 50, 4.0, 0.05, 100, 2000, seed=8)
    a, st = gen.graph_adjacency(spec)
    assert st["n_sv"] > 0
    want = orc.dindex(omat(a), 400, 600, algo="hbv")
    got = ctx.distance_index(ctx.upload(a), 400, 600).download()
    assert_same(got, want.rowmap, want.entries, want.nnz)


def spgemm_case(ctx, a, b, expect_direct=None):
    want = orc.spgemm(omat(a), omat(b), algo="hbv")
    ctx.reset_stats()
    got = ctx.spgemm(ctx.upload(a), ctx.upload(b)).download()
    assert_same(got, want.rowmap, want.entries, want.nnz)
    return ctx.stats()


@pytest.mark.parametrize("chunk_rows", [0, 32, 256, 2048])
def test_fused_tiled_single_chunk_and_stage_overflow(ctx, chunk_rows):
    # narrow band, many short output runs: staged sub-tiles; with large chunks
    # the output outgrows the staging area and the remaining rows are
    # recomputed into global memory
    set_plan(ctx, (0, 0, 0, 1), chunk_rows)
    a = gen.banded(20_000, 20, 1.2, 2.0, seed=41)
    b = gen.banded(20_000, 300, 6.0, 1.0, seed=42)
    st = spgemm_case(ctx, a, b)
    assert st["spgemm_direct_tiles"] == 0


@pytest.mark.parametrize("chunk_rows", [0, 2048])
def test_fused_tiled_multi_chunk(ctx, chunk_rows):
    # a sub-tile window wider than 32 words: lane groups loop over window chunks
    set_plan(ctx, (0, 0, 0, 1), chunk_rows)
    a = gen.banded(20_000, 4, 1.0, 8.0, seed=43)
    b = gen.banded(20_000, 520, 4.0, 1.0, seed=44)
    st = spgemm_case(ctx, a, b)
    assert st["spgemm_direct_tiles"] == 0


@pytest.mark.parametrize("chunk_rows", [0, 64, 2048])
def test_fused_direct_tiles_and_capacity_rerun(ctx, chunk_rows):
    # random columns: every sub-tile misses the staged path; the output exceeds
    # the speculative capacity, which is detected and re-run at the exact size
    set_plan(ctx, (0, 0, 0, 1), chunk_rows)
    a = gen.random_matrix(2000, 8000, seed=45)
    b = gen.random_matrix(2000, 30000, seed=46)
    st = spgemm_case(ctx, a, b)
    assert st["spgemm_direct_tiles"] > 0
    assert st["spgemm_reruns"] == 1


@pytest.mark.parametrize("mean_len,hw", [(6.0, 64), (32.0, 512), (300.0, 4096)])
@pytest.mark.parametrize("levels", [0, 1])
def test_long_range_products_with_union_levels(ctx, mean_len, hw, levels):
    # A ranges of many rows: the row kernel reads union levels of B (blocks of
    # 2^k rows, several per range when a range is longer than the top level)
    set_plan(ctx, (0, 0, 0, 2))
    ctx.set_option("spgemm_levels", levels)
    try:
        a = gen.banded(40_000, hw, 3.0, mean_len, seed=91)
        b = gen.banded(40_000, 256, 4.0, 8.0, seed=92)
        st = spgemm_case(ctx, a, b)
        assert (st["spgemm_levels"] > 0) == bool(levels)
    finally:
        ctx.set_option("spgemm_levels", 1)


def test_algos_agree_on_cfg2_shape_sample(ctx):
    # the kernel microbenchmark shape (banded, half-width 512, Poisson(4)
    # ranges of geometric length 32) at 2^20 rows: both kernels and the oracle
    a = gen.banded(1 << 20, 512, 4.0, 32.0, seed=51)
    b = gen.banded(1 << 20, 512, 4.0, 32.0, seed=52)
    want = orc.spgemm(omat(a), omat(b), algo="hbv")
    for plan in FUSED:
        set_plan(ctx, plan)
        got = ctx.spgemm(ctx.upload(a), ctx.upload(b)).download()
        assert_same(got, want.rowmap, want.entries, want.nnz, f"plan {plan}")


@pytest.mark.parametrize("chunk_rows", [0, 2048])
def test_fused_light_rows_wider_than_a_window_and_stage_overflow(ctx, chunk_rows):
    # thread-per-row mode on rows spanning several 128-column windows, with
    # more output than the chunk stage holds
    set_plan(ctx, (0, 0, 0, 2), chunk_rows)
    a = gen.banded(30_000, 300, 2.0, 1.0, seed=71)
    b = gen.banded(30_000, 400, 6.0, 3.0, seed=72)
    st = spgemm_case(ctx, a, b)
    assert st["spgemm_light"] == 1


@pytest.mark.parametrize("schedule", [0, 1])
@pytest.mark.parametrize("window", [(0, 1), (0, 5), (2, 9)])
def test_index_of_noncanonical_and_cyclic_input(ctx, schedule, window):
    # a random matrix (cycles) whose rows carry adjacent ranges: both
    # schedules must reproduce the reference's canonical index
    set_plan(ctx, (0, 0, 0, 0))
    ctx.set_option("dindex_schedule", schedule)
    a = gen.random_matrix(300, 900, seed=81)
    ent = a.entries.copy()
    rowmap = a.rowmap.copy()
    # split the first multi-column range of every row into two adjacent ranges
    out_e, out_r = [], [0]
    for i in range(a.numRows()):
        e = ent[int(rowmap[i]):int(rowmap[i + 1])].tolist()
        split = False
        for k in range(0, len(e), 2):
            if not split and e[k + 1] > e[k]:
                out_e += [e[k], e[k], e[k] + 1, e[k + 1]]
                split = True
            else:
                out_e += [e[k], e[k + 1]]
        out_r.append(len(out_e))
    nc = CRSMatrix(a.numCols(), np.array(out_e, np.uint32), np.array(out_r, np.uint64))
    want = orc.dindex(omat(nc), *window)
    got = ctx.distance_index(ctx.upload(nc), *window).download()
    assert_same(got, want.rowmap, want.entries, want.nnz, str(window))
    ctx.set_option("dindex_schedule", 0)


@pytest.mark.parametrize("chunk_rows", [0, 2048])
@pytest.mark.parametrize("window", [(0, 4), (2, 5)])
def test_index_fused_sums_on_fragmented_rows(ctx, window, chunk_rows):
    # random columns: the rows of every product hold more runs than a thread's
    # list, so the sums D + A B of the sum-of-powers schedule take the warp
    # path and, past its per-chunk list, the per-thread windowed path
    set_plan(ctx, (0, 0, 0, 0), chunk_rows)
    ctx.set_option("dindex_schedule", 0)
    a = gen.random_matrix(6000, 30000, seed=83)
    want = orc.dindex(omat(a), *window)
    ctx.reset_stats()
    got = ctx.distance_index(ctx.upload(a), *window).download()
    st = ctx.stats()
    assert_same(got, want.rowmap, want.entries, want.nnz, str(window))
    assert st["spgemm_fused_adds"] > 0 and st["spgemm_slow_rows"] > 2048


@pytest.mark.parametrize("row_slot,chunk_rows", [(0, 0), (1, 512), (2, 1024), (0, 1056), (2, 2048), (1, 96)])
@pytest.mark.parametrize("window", [(100, 300), (0, 37), (1, 1), (64, 64)])
def test_planned_build_matches_oracle_and_synchronised_path(ctx, window, row_slot, chunk_rows):
    # planned builds (one launch per step, no read-back between them) across
    # run-list widths and chunk shapes, against the oracle and the read-back path
    set_plan(ctx, (0, 0, 0, 0), chunk_rows)
    ctx.set_option("row_slot", row_slot)
    a, _ = gen.graph_adjacency(gen.small_graph_spec(60_000, seed=9))
    want = orc.dindex(omat(a), *window, algo="hbv")
    da = ctx.upload(a)
    try:
        ctx.reset_stats()
        got = ctx.distance_index(da, *window).download()
        st = ctx.stats()
        assert_same(got, want.rowmap, want.entries, want.nnz, str(window))
        assert st["spgemm_reruns"] == 0 and st["host_syncs"] <= 3, st
        ctx.set_option("planned_build", 0)
        again = ctx.distance_index(da, *window).download()
        assert_same(again, want.rowmap, want.entries, want.nnz, str(window))
    finally:
        ctx.set_option("planned_build", 1)
        ctx.set_option("row_slot", 1)


@pytest.mark.parametrize("chunk_rows", [0, 2048])
def test_row_kernel_with_and_without_staged_write_out(ctx, chunk_rows):
    # deferred write-out through the staging buffers (default) and the chunk
    # written out in its own iteration give the oracle's index and product;
    # the banded product has chunks that outgrow the staging (written in
    # place) next to chunks that fit it
    set_plan(ctx, (0, 0, 0, 0), chunk_rows)
    g, _ = gen.graph_adjacency(gen.small_graph_spec(80_000, seed=17))
    want = orc.dindex(omat(g), 150, 320, algo="hbv")
    a = gen.banded(30_000, 300, 2.0, 1.0, seed=71)
    b = gen.banded(30_000, 400, 6.0, 3.0, seed=72)
    want_ab = orc.spgemm(omat(a), omat(b), algo="hbv")
    dg = ctx.upload(g)
    try:
        for stage in (1, 0):
            ctx.set_option("row_stage", stage)
            got = ctx.distance_index(dg, 150, 320).download()
            assert_same(got, want.rowmap, want.entries, want.nnz, f"stage {stage}")
            ctx.set_option("spgemm_mode", 2)
            got = ctx.spgemm(ctx.upload(a), ctx.upload(b)).download()
            assert_same(got, want_ab.rowmap, want_ab.entries, want_ab.nnz, f"stage {stage}")
            ctx.set_option("spgemm_mode", 0)
    finally:
        ctx.set_option("row_stage", 1)
        ctx.set_option("spgemm_mode", 0)


def test_planned_build_outgrowing_its_estimate_reruns_exactly(ctx):
    # a capacity estimate of nothing: the first step overflows, the later
    # steps stand down, and the build re-runs on the read-back path
    set_plan(ctx, (0, 0, 0, 0))
    a = gen.random_matrix(4000, 24000, seed=85)
    want = orc.dindex(omat(a), 2, 6)
    da = ctx.upload(a)
    ctx.set_option("plan_growth", 0)
    ctx.reset_stats()
    got = ctx.distance_index(da, 2, 6).download()
    st = ctx.stats()
    assert_same(got, want.rowmap, want.entries, want.nnz)
    assert st["spgemm_reruns"] >= 1
    # the estimate has grown: the next build stays planned
    ctx.reset_stats()
    again = ctx.distance_index(da, 2, 6).download()
    assert_same(again, want.rowmap, want.entries, want.nnz)
    assert ctx.stats()["spgemm_reruns"] == 0
    ctx.set_option("plan_growth", 300)


def test_query_batch_matches_oracle(ctx):
    a, _ = gen.graph_adjacency(gen.small_graph_spec(50_000, seed=4))
    idx = orc.dindex(omat(a), 100, 300, algo="hbv")
    d_idx = ctx.upload(as_crs(idx))
    pairs = gen.query_pairs(a, 200_000, 0.5, 100, 300, seed=3)
    want = orc.query(idx, pairs)
    got = ctx.query(d_idx, pairs)
    assert np.array_equal(got, want)
    assert want.sum() > 50_000  # the in-range half mostly hits


def test_query_rejects_out_of_range_pairs(ctx):
    d = ctx.identity(10)
    with pytest.raises(N.DvgError) as e:
        ctx.query(d, np.array([[1, 1], [10, 2]], np.uint32))
    assert e.value.status == N.INVALID_ARG


def test_u32_rowmap_overload(ctx):
    # dindex_eti.hpp:50-53: the <uint32_t, uint32_t> overload
    a, _ = gen.graph_adjacency(gen.small_graph_spec(30_000, seed=9))
    want = orc.dindex(omat(a), 1, 8)
    a32 = CRSMatrix(a.numCols(), a.entries, a.rowmap.astype(np.uint32), a.nnz(), size_type=np.uint32)
    got = ctx.distance_index(ctx.upload(a32), 1, 8).download(np.uint32)
    assert got.rowmap.dtype == np.uint32
    assert_same(got, want.rowmap, want.entries, want.nnz)


def test_edge_cases(ctx):
    # empty matrix, empty rows, a row whose runs end on 32-bit word edges, and
    # columns at the top of the uint32 range
    z = ctx.upload(CRSMatrix(0, np.zeros(0, np.uint32), np.zeros(1, np.uint64)))
    assert ctx.spgemm(z, z).download().numRows() == 0
    e = CRSMatrix(5, np.zeros(0, np.uint32), np.zeros(6, np.uint64))
    de = ctx.upload(e)
    assert ctx.spgemm(de, de).download().entries.size == 0
    assert ctx.power(de, 3).download().entries.size == 0
    ent = np.array([0, 31, 32, 32, 63, 63, 95, 127, 160, 191], np.uint32)
    b = CRSMatrix(256, ent, np.array([0, len(ent)], np.uint64))
    for plan in PLANS:
        set_plan(ctx, plan)
        c = ctx.spgemm(ctx.identity(1), ctx.upload(b)).download()
        assert list(c.entries) == [0, 32, 63, 63, 95, 127, 160, 191], plan
    top = 0xFFFFFFFE
    hi = np.array([top - 70, top - 40, top - 33, top - 1], np.uint32)
    B = CRSMatrix(top, hi, np.array([0, 2, 4, 4], np.uint64))
    A = CRSMatrix(3, np.array([0, 1, 1, 2, 0, 0], np.uint32), np.array([0, 2, 4, 6], np.uint64))
    want = orc.spgemm(omat(A), omat(B))
    for plan in PLANS:
        set_plan(ctx, plan)
        assert_same(ctx.spgemm(ctx.upload(A), ctx.upload(B)).download(), want.rowmap, want.entries, want.nnz,
                    str(plan))


def test_errors_are_reported(ctx):
    a = ctx.identity(4)
    b = ctx.identity(5)
    with pytest.raises(N.DvgError) as e:
        ctx.spgemm(a, b)
    assert e.value.status == N.INVALID_ARG
    with pytest.raises(N.DvgError) as e:
        ctx.distance_index(a, 3, 2)
    assert e.value.status == N.INVALID_ARG
    with pytest.raises(N.DvgError) as e:
        ctx.distance_index(a, 0, 0)
    assert e.value.status == N.INVALID_ARG
    bad = CRSMatrix(4, np.array([0, 9], np.uint32), np.array([0, 2, 2, 2, 2], np.uint64))
    with pytest.raises(N.DvgError) as e:
        ctx.upload(bad)
    assert e.value.status == N.INVALID_ARG
    odd = CRSMatrix(4, np.array([0, 1, 2], np.uint32), np.array([0, 3, 3, 3, 3], np.uint64), 1)
    with pytest.raises(N.DvgError):
        ctx.upload(odd)


def test_bounded_device_wait_runs_out_and_the_context_stays_usable(ctx):
    # a look-back on a chunk whose predecessor nothing publishes: the wait
    # gives up after its bound, the call reports a timeout, and the same
    # context computes correctly afterwards (no fault, no hang)
    for limit in (1, 1000, 20000):
        assert N.lib().dvg_selftest_bounded_wait(ctx.handle, limit) == N.TIMEOUT
    a = gen.random_matrix(3000, 9000, seed=5)
    want = orc.spgemm(omat(a), omat(a), algo="hbv")
    got = ctx.spgemm(ctx.upload(a), ctx.upload(a)).download()
    assert_same(got, want.rowmap, want.entries, want.nnz)


def test_reference_api_mirror():
    import diverg_b200 as dv
    with dv.ScopedRuntime():
        a, _ = gen.graph_adjacency(gen.small_graph_spec(20_000, seed=1))
        idx = dv.create_distance_index(a, 10, 30)
        want = orc.dindex(omat(a), 10, 30)
        assert_same(idx, want.rowmap, want.entries, want.nnz)
        sq = dv.range_spgemm(a, a)
        want = orc.spgemm(omat(a), omat(a))
        assert_same(sq, want.rowmap, want.entries, want.nnz)
        ai = dv.range_spadd(a, dv.create_range_identity_matrix(a.numRows()))
        want = orc.spadd(omat(a), orc.identity(a.numRows()))
        assert_same(ai, want.rowmap, want.entries, want.nnz)
        p = dv.range_power(a, 5)
        want = orc.power(omat(a), 5)
        assert_same(p, want.rowmap, want.entries, want.nnz)
        pairs = gen.query_pairs(a, 1000, 0.5, 10, 30)
        assert np.array_equal(dv.query_batch(idx, pairs), orc.query(omat(idx), pairs))


def _noncanonical(m, split_every=1):
    """m with the first multi-column range of every row split into two
    adjacent ranges, and every third row's first range repeated."""
    out_e, out_r = [], [0]
    for i in range(m.numRows()):
        e = m.entries[int(m.rowmap[i]):int(m.rowmap[i + 1])].tolist()
        split = False
        row = []
        for k in range(0, len(e), 2):
            if not split and e[k + 1] > e[k] and i % split_every == 0:
                row += [e[k], e[k], e[k] + 1, e[k + 1]]
                split = True
            else:
                row += [e[k], e[k + 1]]
        if i % 3 == 0 and row:
            row = row[:2] + row
        out_e += row
        out_r.append(len(out_e))
    return CRSMatrix(m.numCols(), np.array(out_e, np.uint32), np.array(out_r, np.uint64))


@pytest.mark.parametrize("single", [1, 0])
@pytest.mark.parametrize("shape", ["banded", "wide_rows", "noncanonical", "empty_rows", "one_row", "dense_disjoint",
                                   "cover"])
def test_spadd_one_pass_and_three_pass(ctx, single, shape):
    # range_spadd (range_sparse.hpp:112-477) in one pass with a chunk look-back
    # and by count, scan and fill: rows past the per-chunk stages (wide rows),
    # chunks whose output exceeds the shared image (dense, disjoint), long
    # ranges of one operand covering many of the other's (cover), the
    # reference's merge on non-canonical rows (tails copied verbatim), empty rows
    if shape == "banded":
        a = gen.banded(300_000, 512, 4.0, 32.0, seed=301)
        b = gen.banded(300_000, 512, 4.0, 32.0, seed=302)
    elif shape == "wide_rows":
        a = gen.banded(20_000, 4000, 12.0, 2.0, seed=303)
        b = gen.banded(20_000, 4000, 12.0, 2.0, seed=304)
    elif shape == "noncanonical":
        a = _noncanonical(gen.random_matrix(3000, 20_000, seed=305))
        b = _noncanonical(gen.random_matrix(3000, 20_000, seed=306), split_every=2)
    elif shape == "empty_rows":
        a = gen.random_matrix(50_000, 5_000, seed=307)
        b = gen.random_matrix(50_000, 3_000, seed=308)
    elif shape == "dense_disjoint":
        a = gen.banded(40_000, 4000, 5.0, 1.5, seed=309)
        b = gen.banded(40_000, 4000, 5.0, 1.5, seed=310)
    elif shape == "cover":
        a = gen.banded(50_000, 512, 5.0, 3.0, seed=311)
        b = gen.banded(50_000, 512, 0.5, 600.0, seed=312)
    else:
        a = CRSMatrix(9, np.array([0, 3, 5, 8], np.uint32), np.array([0, 4], np.uint64))
        b = CRSMatrix(9, np.array([4, 4], np.uint32), np.array([0, 2], np.uint64))
    want = orc.spadd(omat(a), omat(b))
    ctx.set_option("spadd_single", single)
    try:
        got = ctx.spadd(ctx.upload(a), ctx.upload(b)).download()
    finally:
        ctx.set_option("spadd_single", 1)
    assert_same(got, want.rowmap, want.entries, want.nnz, shape)


@pytest.mark.parametrize("npairs", [1, 3, 4, 4097, 200_001])
@pytest.mark.parametrize("offset", [0, 1, 2])
def test_query_paths_and_tails(ctx, npairs, offset):
    # membership queries (crs_matrix.hpp:149-169) by the four-pairs-a-thread
    # kernel and the one-pair kernel: counts that leave a tail, pair and answer
    # buffers offset so the four-pair path does not apply, rows of one to many
    # ranges, a non-canonical row set, out-of-range pairs answered 0
    import torch
    a = gen.random_matrix(5000, 60_000, seed=331)  # rows of ~12 ranges and rows of few
    m = _noncanonical(a, split_every=3)
    d = ctx.upload(m)
    rng = np.random.default_rng(npairs + offset)
    pairs = np.stack([rng.integers(0, 5000, npairs + offset), rng.integers(0, 5000, npairs + offset)], 1)
    pairs = pairs.astype(np.uint32)
    want = orc.query(omat(m), pairs[offset:])
    d_pairs = torch.from_numpy(pairs.view(np.int32).reshape(-1)).cuda()
    d_out = torch.zeros(npairs + offset, dtype=torch.uint8, device="cuda")
    ctx.query_device(d, d_pairs.data_ptr() + 8 * offset, npairs, d_out.data_ptr() + offset)
    torch.cuda.synchronize()
    assert np.array_equal(d_out.cpu().numpy()[offset:], want)
    # the same through host buffers
    assert np.array_equal(ctx.query(d, pairs[offset:]), want)


def test_query_out_of_range_pairs_answer_zero_in_both_paths(ctx):
    import torch
    a, _ = gen.graph_adjacency(gen.small_graph_spec(20_000, seed=332))
    d = ctx.upload(a)
    n = a.numRows()
    pairs = np.array([[0, 1], [n, 0], [1, n + 5], [2, 3], [5, 6], [n + 1, n + 1], [7, 8], [9, 10]], np.uint32)
    want = orc.query(omat(a), np.where(pairs < n, pairs, 0).astype(np.uint32))
    want[(pairs >= n).any(1)] = 0
    d_pairs = torch.from_numpy(pairs.view(np.int32).reshape(-1)).cuda()
    d_out = torch.zeros(len(pairs), dtype=torch.uint8, device="cuda")
    with pytest.raises(N.DvgError):
        ctx.query_device(d, d_pairs.data_ptr(), len(pairs), d_out.data_ptr())
    torch.cuda.synchronize()
    assert np.array_equal(d_out.cpu().numpy(), want)


def test_query_never_reads_past_a_corrupt_index(ctx):
    # row pointers that leave the entries (a caller-owned index overwritten
    # after it was wrapped): those pairs answer 0, nothing past the entries is
    # read, the call reports a device error and the context stays usable
    import torch
    a, _ = gen.graph_adjacency(gen.small_graph_spec(20_000, seed=333))
    n = a.numRows()
    rowmap = torch.from_numpy(a.rowmap.astype(np.uint64).view(np.int64)).cuda()
    entries = torch.from_numpy(a.entries.view(np.int32)).cuda()
    d = ctx.wrap_device(n, a.numCols(), rowmap.data_ptr(), entries.data_ptr(), len(a.entries), a.nnz())
    pairs = np.array([[k, k + 1] for k in range(64)], np.uint32)
    want = orc.query(omat(a), pairs)
    assert np.array_equal(ctx.query(d, pairs), want)
    rowmap[10] = 1 << 40   # row 9 ends and row 10 starts far past the entries
    rowmap[20] = -1        # row 19 ends and row 20 starts at 2^64 - 1
    torch.cuda.synchronize()
    npairs = len(pairs)
    bad = np.isin(np.arange(npairs), [9, 10, 19, 20])
    for offset in (0, 1):  # the four-pair kernel; buffers offset by a pair: the one-pair kernel
        padded = np.concatenate([np.zeros((offset, 2), np.uint32), pairs])
        d_pairs = torch.from_numpy(padded.view(np.int32).reshape(-1)).cuda()
        d_out = torch.full((npairs + offset,), 7, dtype=torch.uint8, device="cuda")
        with pytest.raises(N.DvgError) as err:
            ctx.query_device(d, d_pairs.data_ptr() + 8 * offset, npairs, d_out.data_ptr() + offset)
        assert err.value.status == N.DEVICE
        got = d_out.cpu().numpy()[offset:]
        assert (got[bad] == 0).all() and np.array_equal(got[~bad], want[~bad])
    rowmap.copy_(torch.from_numpy(a.rowmap.astype(np.uint64).view(np.int64)).cuda())
    torch.cuda.synchronize()
    assert np.array_equal(ctx.query(d, pairs), want)


def test_random_read_calibration(ctx):
    # the query's measured denominator: positive and finite, an argument
    # error for an absurd size, and the context answers correctly afterwards
    rate = ctx.calibrate_random_reads(64 << 20)
    assert np.isfinite(rate) and 1e8 < rate < 1e12, rate
    with pytest.raises(N.DvgError):
        ctx.calibrate_random_reads(1 << 41)
    a, _ = gen.graph_adjacency(gen.small_graph_spec(20_000, seed=334))
    pairs = np.array([[k, k + 1] for k in range(0, 2000, 7)], np.uint32)
    assert np.array_equal(ctx.query(ctx.upload(a), pairs), orc.query(omat(a), pairs))
