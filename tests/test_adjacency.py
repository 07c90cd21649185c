"""Adjacency construction (util::range_adjacency_matrix, adjacency.hpp:249-265).

CPU: the generator's compacted node graph, through the oracle's restatement
of adjacency_matrix + append, gives exactly the generator's direct adjacency;
the reference's test graphs (committed fixtures) give the stored adjacency.
GPU: dvg_adjacency_from_graph equals the oracle on the reference's test graphs
(whole graph and every component, as test_dindex.cpp:54-107 builds them), on
random graphs with repeated edges, edges in any order, nodes without
successors and long nodes, and on the chromosome generator's graph; bad
inputs fail with the documented status.
"""
import os

import numpy as np
import pytest

from diverg_b200 import _native as N, gen
from oracle import pyoracle as orc
from tests.conftest import ROOT

GOLDEN = os.path.join(ROOT, "tests", "golden")


def golden(name):
    z = np.load(os.path.join(GOLDEN, f"gfa_{name}.npz"))
    return z["node_len"], z["edges"], z


def components(n, edges):
    """Weakly connected components as contiguous [lower, upper) id ranges."""
    parent = np.arange(n + 1)

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    for a, b in edges:
        ra, rb = find(int(a)), find(int(b))
        if ra != rb:
            parent[max(ra, rb)] = min(ra, rb)
    roots = [find(i) for i in range(1, n + 1)]
    out, lo = [], 1
    for i in range(2, n + 2):
        if i == n + 1 or roots[i - 1] != roots[lo - 1]:
            out.append((lo, i))
            lo = i
    assert len({roots[a - 1] for a, _ in out}) == len(out), "components are not contiguous"
    return out


def same(m, o):
    return (m.numRows() == o.nrows and m.numCols() == o.ncols and m.nnz() == int(o.nnz)
            and np.array_equal(m.rowmap.astype(np.uint64), o.rowmap) and np.array_equal(m.entries, o.entries))


def random_graph(n, seed, max_len=40, max_deg=5, repeats=True):
    """Nodes 1..n with random lengths; every node but the last links forward
    to 0..max_deg later nodes (a DAG in rank order), shuffled, with repeated
    edges when asked."""
    rng = np.random.default_rng(seed)
    lens = rng.integers(1, max_len + 1, n).astype(np.uint32)
    edges = []
    for v in range(1, n):
        deg = int(rng.integers(0, max_deg + 1))
        for _ in range(deg):
            edges.append((v, int(rng.integers(v + 1, min(n, v + 60) + 1))))
        if repeats and deg and rng.random() < 0.1:
            edges.append(edges[-1])
    e = np.array(edges, np.uint32).reshape(-1, 2)
    return lens, e[rng.permutation(len(e))]


# ---- CPU: the oracle against the generator and the fixtures -----------------

@pytest.mark.parametrize("spec", [gen.small_graph_spec(30_000, seed=3), gen.chromosome_graph_spec(1_000_000, seed=5)])
def test_generator_node_graph_gives_the_generator_adjacency(spec):
    lens, edges = gen.graph_nodes(spec)
    a, st = gen.graph_adjacency(spec)
    assert int(lens.sum()) == st["n_loci"] and len(lens) < st["n_loci"] // 10
    assert same(a, orc.adjacency(lens, edges))


@pytest.mark.parametrize("name", ["x", "multi", "m"])
def test_oracle_reproduces_the_fixture_adjacency(name):
    lens, edges, z = golden(name)
    o = orc.adjacency(lens, edges)
    assert np.array_equal(o.rowmap, z["A_rowmap"]) and np.array_equal(o.entries, z["A_entries"])
    assert int(o.nnz) == int(z["A_nnz"]) == int(lens.sum()) - len(lens) + len(edges)


def test_oracle_components_tile_the_whole_graph():
    lens, edges, _ = golden("multi")
    comps = components(len(lens), edges)
    assert len(comps) == 2
    whole = orc.adjacency(lens, edges)
    off = 0
    for lo, hi in comps:
        part = orc.adjacency(lens, edges, lo, hi)
        rows = whole.rowmap[off:off + part.nrows + 1]
        seg = whole.entries[int(rows[0]):int(rows[-1])].astype(np.int64) - off
        assert np.array_equal(rows - rows[0], part.rowmap) and np.array_equal(seg, part.entries)
        off += part.nrows


def test_random_graphs_have_repeats_and_unsorted_edges():
    lens, edges = random_graph(3000, 4, 1, 8)
    assert len(np.unique(edges, axis=0)) < len(edges)
    assert not np.all(np.diff(edges[:, 0].astype(np.int64)) >= 0)
    o = orc.adjacency(lens, edges)
    assert int(o.nnz) == int(lens.sum()) - len(lens) + len(edges)


# ---- GPU: the device builder against the oracle --------------------------------

@pytest.fixture(scope="module")
def ctx():
    from diverg_b200.runtime import Context
    c = Context(0)
    yield c
    c.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["x", "multi", "m"])
def test_reference_test_graphs_whole_and_per_component(ctx, name):
    lens, edges, z = golden(name)
    got = ctx.adjacency_from_graph(lens, edges).download()
    want = orc.adjacency(lens, edges)
    assert same(got, want)
    assert np.array_equal(got.rowmap.astype(np.uint64), z["A_rowmap"])
    for lo, hi in components(len(lens), edges):
        part = ctx.adjacency_from_graph(lens, edges, lo, hi).download()
        assert same(part, orc.adjacency(lens, edges, lo, hi)), (lo, hi)
        if hi == len(lens) + 1:  # upper = 0 reaches the last node
            assert same(ctx.adjacency_from_graph(lens, edges, lo, 0).download(), orc.adjacency(lens, edges, lo, 0))


@pytest.mark.gpu
@pytest.mark.parametrize("seed,n,max_len,max_deg", [(1, 1, 5, 0), (2, 2, 1, 1), (3, 500, 40, 5), (4, 3000, 1, 8),
                                                    (5, 2000, 300, 3)])
def test_random_graphs_with_repeats_and_shuffled_edges(ctx, seed, n, max_len, max_deg):
    lens, edges = random_graph(n, seed, max_len, max_deg)
    got = ctx.adjacency_from_graph(lens, edges).download()
    assert same(got, orc.adjacency(lens, edges))


@pytest.mark.gpu
def test_a_node_with_many_successors(ctx):
    # one hub with 5,000 successors (heap-sorted segment) and repeated edges
    rng = np.random.default_rng(9)
    n = 6000
    lens = rng.integers(1, 4, n).astype(np.uint32)
    hub = np.stack([np.ones(5000, np.uint32), rng.integers(2, n + 1, 5000).astype(np.uint32)], 1)
    chain = np.stack([np.arange(2, n, dtype=np.uint32), np.arange(3, n + 1, dtype=np.uint32)], 1)
    edges = np.concatenate([hub, chain])[rng.permutation(5000 + n - 2)]
    assert same(ctx.adjacency_from_graph(lens, edges).download(), orc.adjacency(lens, edges))


@pytest.mark.gpu
def test_chromosome_generator_graph(ctx):
    spec = gen.chromosome_graph_spec(5_000_000, seed=7)
    lens, edges = gen.graph_nodes(spec)
    a, _ = gen.graph_adjacency(spec)
    dm = ctx.adjacency_from_graph(lens, edges)
    assert same(dm.download(), orc.OMat(a.numRows(), a.numCols(), a.rowmap.astype(np.uint64), a.entries, a.nnz()))


@pytest.mark.gpu
def test_bad_graphs_fail_with_invalid_argument(ctx):
    lens = np.array([3, 2, 4], np.uint32)
    ok = np.array([[1, 2], [2, 3]], np.uint32)
    cases = [
        (np.array([3, 0, 4], np.uint32), ok, 1, 0),       # a node of length 0
        (lens, np.array([[1, 4]], np.uint32), 1, 0),      # an id past the last node
        (lens, np.array([[0, 2]], np.uint32), 1, 0),      # id 0
        (lens, ok, 2, 2),                                  # empty range
        (lens, ok, 0, 0),                                  # lower below 1
        (lens, ok, 1, 5),                                  # upper past nnodes + 1
        (lens, ok, 1, 2),                                  # an edge leaves the range
    ]
    for lens_, edges_, lo, hi in cases:
        with pytest.raises(N.DvgError) as e:
            ctx.adjacency_from_graph(lens_, edges_, lo, hi)
        assert e.value.status == N.INVALID_ARG, (lo, hi)
    # the context stays usable
    assert same(ctx.adjacency_from_graph(lens, ok).download(), orc.adjacency(lens, ok))
