"""The request loop (dvg_server_*): a build and a query batch give the same
index and answers alone and inside a busy mix of other requests, and both
match the oracle exactly; builds are admitted within the memory budget."""
import numpy as np
import pytest

from oracle import pyoracle as orc
from diverg_b200 import CRSMatrix, _native as N, gen
from diverg_b200.serving import Server

pytestmark = pytest.mark.gpu

WINDOW = (200, 500)


def omat(m):
    return orc.OMat(m.numRows(), m.numCols(), m.rowmap.astype(np.uint64), m.entries, m.nnz())


def same(a: CRSMatrix, b: CRSMatrix):
    return (a.numRows() == b.numRows() and np.array_equal(a.rowmap.astype(np.uint64), b.rowmap.astype(np.uint64))
            and np.array_equal(a.entries, b.entries) and a.nnz() == b.nnz())


def graph(n, seed):
    return gen.graph_adjacency(gen.small_graph_spec(n, seed=seed))[0]


def test_results_are_the_same_alone_and_in_the_mix():
    target = graph(40_000, seed=11)
    pairs = gen.query_pairs(target, 200_000, 0.5, *WINDOW, seed=12)
    want = orc.dindex(omat(target), *WINDOW, algo="hbv")
    want_crs = CRSMatrix(want.ncols, want.entries, want.rowmap, want.nnz)
    want_answers = orc.query(want, pairs)

    with Server(device=0) as srv:  # alone
        b = srv.submit_build(target, *WINDOW)
        assert srv.wait([b])[0]["status"] == N.OK
        ans_alone = np.zeros(len(pairs), np.uint8)
        q = srv.submit_query(b, pairs, ans_alone)
        assert srv.wait([q])[0]["status"] == N.OK
        idx_alone = srv.download(b)

    others = [graph(int(n), seed=100 + k) for k, n in enumerate(np.linspace(5_000, 120_000, 12))]
    other_pairs = [gen.query_pairs(g, 50_000 + 10_000 * k, 0.5, *WINDOW, seed=200 + k) for k, g in enumerate(others)]
    with Server(device=0, max_batch_builds=4, max_inflight_queries=4) as srv:  # in the mix
        ids, bids = [], []
        answers = []
        for k, g in enumerate(others[:6]):
            bids.append(srv.submit_build(g, *WINDOW))
        for k in range(6):
            a = np.zeros(len(other_pairs[k]), np.uint8)
            answers.append(a)
            ids.append(srv.submit_query(bids[k], other_pairs[k], a))
        b = srv.submit_build(target, *WINDOW)
        for k, g in enumerate(others[6:], start=6):
            bids.append(srv.submit_build(g, *WINDOW))
        ans_mix = np.zeros(len(pairs), np.uint8)
        q = srv.submit_query(b, pairs, ans_mix)
        for k in range(6, 12):
            a = np.zeros(len(other_pairs[k]), np.uint8)
            answers.append(a)
            ids.append(srv.submit_query(bids[k], other_pairs[k], a))
        done = srv.wait(ids + bids + [b, q])
        assert all(c["status"] == N.OK for c in done)
        idx_mix = srv.download(b)
        st = srv.stats()
        # the other requests are right too
        for k in (0, 7, 11):
            got = srv.download(bids[k])
            assert np.array_equal(answers[k], orc.query(omat(got), other_pairs[k]))
    assert st["queries_done"] == 13 and st["builds_done"] == 13 and st["build_batches"] >= 2
    assert same(idx_alone, want_crs) and same(idx_mix, want_crs)
    assert np.array_equal(ans_alone, want_answers) and np.array_equal(ans_mix, want_answers)


def test_builds_are_admitted_within_the_budget():
    budget = 64 << 20
    graphs = [graph(20_000, seed=300 + k) for k in range(10)]
    with Server(device=0, hbm_budget_bytes=budget) as srv:
        bids = [srv.submit_build(g, *WINDOW) for g in graphs]
        done = srv.wait(bids)
        assert all(c["status"] == N.OK for c in done)
        st = srv.stats()
        assert st["peak_reserved_bytes"] <= budget
        assert st["build_batches"] >= 2
        for k in (0, 9):
            want = orc.dindex(omat(graphs[k]), *WINDOW, algo="hbv")
            assert same(srv.download(bids[k]), CRSMatrix(want.ncols, want.entries, want.rowmap, want.nnz))


def test_oversized_builds_bad_pairs_and_released_indices_report_errors():
    big = graph(100_000, seed=400)
    small = graph(5_000, seed=401)
    with Server(device=0, hbm_budget_bytes=1 << 20) as srv:
        b = srv.submit_build(big, *WINDOW)
        q = srv.submit_query(b, np.zeros((4, 2), np.uint32), np.zeros(4, np.uint8))
        c = srv.wait([b, q])
        assert c[0]["status"] == N.OOM and c[1]["status"] == N.OOM
    with Server(device=0) as srv:
        b = srv.submit_build(small, *WINDOW)
        srv.wait([b])
        pairs = np.array([[0, 0], [small.numRows(), 0], [1, small.numRows() + 5]], np.uint32)
        ans = np.full(3, 7, np.uint8)
        c = srv.wait([srv.submit_query(b, pairs, ans)])[0]
        assert c["status"] == N.INVALID_ARG and c["invalid_pairs"] == 2 and list(ans[1:]) == [0, 0]
        srv.release(b)
        c = srv.wait([srv.submit_query(b, pairs[:1], ans[:1])])[0]
        assert c["status"] == N.INVALID_ARG
        with pytest.raises(N.DvgError):
            srv.release(b)


def _malformed(g, kind):
    """g with one defect the upload check rejects: an odd row length, or a
    column past the last one."""
    rowmap = g.rowmap.astype(np.uint64).copy()
    entries = g.entries.copy()
    if kind == "odd_row":
        rowmap[1:] += 1  # row 0 one entry longer: an odd count
        entries = np.concatenate([entries[:1], entries]).astype(np.uint32)
    else:
        entries[-1] = g.numCols()
    return CRSMatrix(g.numCols(), entries, rowmap, 1)


@pytest.mark.parametrize("kind", ["odd_row", "column"])
def test_a_malformed_build_fails_alone(kind):
    # one worker, a long build first: the rest queue and go out as one batch
    # with the malformed graph among them; it fails with INVALID_ARG, its
    # batch-mates build and match the oracle
    first = graph(400_000, seed=500)
    mates = [graph(8_000 + 1_000 * k, seed=501 + k) for k in range(5)]
    bad = _malformed(graph(6_000, seed=510), kind)
    with Server(device=0, max_batch_builds=16, build_workers=1) as srv:
        b0 = srv.submit_build(first, *WINDOW)
        ids = [srv.submit_build(m, *WINDOW) for m in mates[:2]]
        bid = srv.submit_build(bad, *WINDOW)
        ids += [srv.submit_build(m, *WINDOW) for m in mates[2:]]
        done = {c["request"]: c for c in srv.wait([b0, bid] + ids)}
        assert done[bid]["status"] == N.INVALID_ARG
        assert all(done[i]["status"] == N.OK for i in [b0] + ids)
        for k, i in enumerate(ids):
            want = orc.dindex(omat(mates[k]), *WINDOW, algo="hbv")
            assert same(srv.download(i), CRSMatrix(want.ncols, want.entries, want.rowmap, want.nnz)), k
        st = srv.stats()
        assert st["builds_failed"] == 1 and st["builds_done"] == 6


def test_builds_run_side_by_side_on_two_workers():
    # a long build holds one worker; a short build submitted after it is
    # taken by the other worker and completes first, and both are right
    long_g = graph(2_000_000, seed=520)
    short_g = graph(5_000, seed=521)
    with Server(device=0, max_batch_builds=1, build_workers=2) as srv:
        bl = srv.submit_build(long_g, *WINDOW)
        bs = srv.submit_build(short_g, *WINDOW)
        cl, cs = srv.wait([bl, bs])
        assert cl["status"] == N.OK and cs["status"] == N.OK
        assert cs["done_ns"] < cl["done_ns"]
        for g, b in ((long_g, bl), (short_g, bs)):
            want = orc.dindex(omat(g), *WINDOW, algo="hbv")
            assert same(srv.download(b), CRSMatrix(want.ncols, want.entries, want.rowmap, want.nnz))


def test_queries_waiting_on_a_build_read_the_finished_index():
    # every query is submitted right behind the build of its index, so it is
    # issued (on the query stream) the moment the build completes: it must see
    # the whole index, as the same pairs against the downloaded index do
    graphs = [graph(int(n), seed=600 + k) for k, n in enumerate(np.linspace(3_000, 60_000, 16))]
    pairs = [gen.query_pairs(g, 20_000, 0.5, *WINDOW, seed=700 + k) for k, g in enumerate(graphs)]
    with Server(device=0, max_batch_builds=2, max_inflight_queries=8) as srv:
        bids, qids, answers = [], [], []
        for k, g in enumerate(graphs):
            bids.append(srv.submit_build(g, *WINDOW))
            answers.append(np.full(len(pairs[k]), 7, np.uint8))
            qids.append(srv.submit_query(bids[k], pairs[k], answers[k]))
        assert all(c["status"] == N.OK for c in srv.wait(bids + qids))
        for k in range(len(graphs)):
            assert np.array_equal(answers[k], orc.query(omat(srv.download(bids[k])), pairs[k])), k
