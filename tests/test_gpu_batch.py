"""Batched index builds (dvg_batch_distance_index): every graph's index out of
one CUDA-graph launch must equal its own build and the oracle's, exactly."""
import numpy as np
import pytest

from oracle import pyoracle as orc
from diverg_b200 import CRSMatrix, _native as N, gen
from diverg_b200.runtime import Context

pytestmark = pytest.mark.gpu

WINDOWS = [(100, 300), (200, 500), (400, 600)]


@pytest.fixture(scope="module")
def ctx():
    c = Context(0)
    yield c
    c.close()


def omat(m):
    return orc.OMat(m.numRows(), m.numCols(), m.rowmap.astype(np.uint64), m.entries, m.nnz())


def same(a: CRSMatrix, b: CRSMatrix):
    return (a.numRows() == b.numRows() and np.array_equal(a.rowmap.astype(np.uint64), b.rowmap.astype(np.uint64))
            and np.array_equal(a.entries, b.entries) and a.nnz() == b.nnz())


def mixed_batch(count, seed):
    rng = np.random.default_rng(seed)
    graphs, windows = [], []
    for k in range(count):
        n = int(np.clip(rng.lognormal(np.log(4000), 1.0), 500, 60_000))
        g, _ = gen.graph_adjacency(gen.small_graph_spec(n, seed=seed * 1000 + k))
        graphs.append(g)
        windows.append(WINDOWS[int(rng.integers(0, 3))])
    return graphs, windows


def test_batch_equals_single_builds_and_oracle(ctx):
    graphs, windows = mixed_batch(40, seed=3)
    windows[5] = (0, 50)      # a window of its own
    windows[6] = (3, 3)       # a single power
    dg = [ctx.upload(g) for g in graphs]
    ctx.reset_stats()
    got = ctx.batch_distance_index(dg, windows)
    st = ctx.stats()
    assert st["graph_launches"] == 1
    for k, (g, w) in enumerate(zip(graphs, windows)):
        alone = ctx.distance_index(dg[k], *w).download()
        mine = got[k].download()
        assert same(mine, alone), k
        assert got[k].nnz == alone.nnz()
        want = orc.dindex(omat(g), *w, algo="hbv")
        assert same(mine, CRSMatrix(want.ncols, want.entries, want.rowmap, want.nnz)), k


def test_batch_autotunes_once_per_window_and_size(ctx):
    graphs, windows = mixed_batch(12, seed=4)
    dg = [ctx.upload(g) for g in graphs]
    ctx.set_option("autotune", 1)
    ctx.batch_distance_index(dg, windows)
    ctx.reset_stats()
    again = ctx.batch_distance_index(dg, windows)
    assert ctx.stats()["autotune_builds"] == 0
    for k, w in enumerate(windows):
        assert same(again[k].download(), ctx.distance_index(dg[k], *w).download())


def test_batch_with_noncanonical_empty_and_tiny_graphs(ctx):
    # a non-canonical input with dmin = 0 is built alone (the reference's
    # schedule); a 0-row graph and 1-row graphs ride along
    a = gen.random_matrix(300, 900, seed=81)
    out_e, out_r = [], [0]
    for i in range(a.numRows()):
        e = a.entries[int(a.rowmap[i]):int(a.rowmap[i + 1])].tolist()
        for k in range(0, len(e), 2):
            if e[k + 1] > e[k]:
                out_e += [e[k], e[k], e[k] + 1, e[k + 1]]
            else:
                out_e += [e[k], e[k + 1]]
        out_r.append(len(out_e))
    nc = CRSMatrix(a.numCols(), np.array(out_e, np.uint32), np.array(out_r, np.uint64))
    empty = CRSMatrix(0, np.zeros(0, np.uint32), np.zeros(1, np.uint64))
    one = CRSMatrix(1, np.array([0, 0], np.uint32), np.array([0, 2], np.uint64))
    lone = CRSMatrix(1, np.zeros(0, np.uint32), np.array([0, 0], np.uint64))
    small, _ = gen.graph_adjacency(gen.small_graph_spec(3000, seed=5))
    mats = [nc, empty, one, small, lone, nc]
    windows = [(0, 4), (1, 3), (1, 2), (0, 30), (2, 2), (2, 5)]
    dg = [ctx.upload(m) for m in mats]
    got = ctx.batch_distance_index(dg, windows)
    for k, (m, w) in enumerate(zip(mats, windows)):
        want = orc.dindex(omat(m), *w)
        assert same(got[k].download(), CRSMatrix(want.ncols, want.entries, want.rowmap, want.nnz)), k


def test_batch_rejects_bad_windows_and_leaves_nothing(ctx):
    g, _ = gen.graph_adjacency(gen.small_graph_spec(2000, seed=6))
    dg = [ctx.upload(g), ctx.upload(g)]
    with pytest.raises(N.DvgError) as e:
        ctx.batch_distance_index(dg, [(1, 5), (6, 5)])
    assert e.value.status == N.INVALID_ARG
    assert ctx.batch_distance_index([], []) == []
