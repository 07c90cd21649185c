"""GFA loading (diverg_b200.gfa and include/diverg/gfa.hpp) on the reference's
three test graphs, rewritten as GFA 2 and GFA 1 text from the golden fixtures'
node lengths and edges: the graph read back equals the fixture, its adjacency
(oracle on the CPU, the library on the GPU) equals the fixture's matrix, and
the index built from it equals the fixture's [1, 8] index.  Orderings
(native, topological, cycles), string segment names and rejected
reverse-strand edges are checked on small graphs; the C++ reader, compiled
here, reads the same graphs as the Python one."""
import os
import subprocess

import numpy as np
import pytest

from diverg_b200 import CRSMatrix, gfa
from oracle import pyoracle as orc
from tests.conftest import ROOT, load_golden

FIXTURES = ["x", "multi", "m"]


def gfa2_text(node_len, edges, order=None):
    order = range(len(node_len)) if order is None else order
    lines = ["H\tVN:Z:2.0"]
    lines += [f"S\t{k + 1}\t{int(node_len[k])}\t" + "A" * int(node_len[k]) for k in order]
    lines += [f"E\te{i}\t{a}+\t{b}+\t0\t0\t0\t0\t0M" for i, (a, b) in enumerate(edges)]
    return "\n".join(lines) + "\n"


def gfa1_text(node_len, edges):
    lines = ["H\tVN:Z:1.0"]
    lines += [f"S\t{k + 1}\t*\tLN:i:{int(n)}" for k, n in enumerate(node_len)]
    lines += [f"L\t{a}\t+\t{b}\t+\t0M" for a, b in edges]
    return "\n".join(lines) + "\n"


def same_edges(a, b):
    return sorted(map(tuple, np.asarray(a).tolist())) == sorted(map(tuple, np.asarray(b).tolist()))


@pytest.mark.parametrize("name", FIXTURES)
@pytest.mark.parametrize("form", ["gfa2", "gfa1"])
def test_fixture_graphs_read_back(name, form):
    g = load_golden(f"gfa_{name}.npz")
    text = (gfa2_text if form == "gfa2" else gfa1_text)(g["node_len"], g["edges"])
    node_len, edges, _ = gfa.parse(text)
    assert np.array_equal(node_len, g["node_len"]) and same_edges(edges, g["edges"])
    a = orc.adjacency(node_len, edges)
    assert np.array_equal(a.rowmap, g["A_rowmap"]) and np.array_equal(a.entries, g["A_entries"])


def test_orderings_names_cycles_and_strands():
    # file order 3, 1, 2 with edges 1->2->3: native keeps the file order,
    # topological ranks 1, 2, 3
    text = "S\t3\tAAA\nS\t1\tA\nS\t2\tAA\nL\t1\t+\t2\t+\t0M\nL\t2\t+\t3\t+\t0M\n"
    nl, e, names = gfa.parse(text, "native")
    assert names == ["3", "1", "2"] and nl.tolist() == [3, 1, 2] and same_edges(e, [(2, 3), (3, 1)])
    nl, e, names = gfa.parse(text, "topological")
    assert names == ["1", "2", "3"] and nl.tolist() == [1, 2, 3] and same_edges(e, [(1, 2), (2, 3)])
    # a cycle b <-> c after a: the cycle's nodes follow in file order
    text = "S\ta\tA\nS\tc\tAA\nS\tb\tAAA\nL\ta\t+\tb\t+\t0M\nL\tb\t+\tc\t+\t0M\nL\tc\t+\tb\t+\t0M\n"
    _, e, names = gfa.parse(text, "topological")
    assert names == ["a", "c", "b"]
    with pytest.raises(gfa.GFAError):
        gfa.parse("S\t1\tA\nS\t2\tA\nL\t1\t+\t2\t-\t0M\n")
    with pytest.raises(gfa.GFAError):
        gfa.parse("S\t1\t1\tA\nS\t2\t1\tA\nE\te\t1+\t2-\t0\t0\t0\t0\t0M\n")
    with pytest.raises(gfa.GFAError):
        gfa.parse("S\t1\tA\nL\t1\t+\t9\t+\t0M\n")


def _cpp_read(tool, path, ordering):
    out = subprocess.run([tool, str(path), ordering], capture_output=True, text=True, check=True).stdout.split("\n")
    nl, edges = [], []
    for ln in out:
        f = ln.split()
        if f and f[0] == "v":
            nl.append(int(f[3]))
        elif f and f[0] == "e":
            edges.append((int(f[1]), int(f[2])))
    return np.array(nl), edges


def test_cpp_reader_agrees(tmp_path):
    tool = str(tmp_path / "gfa_dump")
    subprocess.run(["g++", "-O1", "-std=c++17", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"),
                    "-o", tool, os.path.join(ROOT, "tests", "cpp", "gfa_dump.cpp")], check=True)
    g = load_golden("gfa_m.npz")
    rng = np.random.default_rng(3)
    order = rng.permutation(len(g["node_len"]))
    for k, text in enumerate([gfa2_text(g["node_len"], g["edges"]), gfa1_text(g["node_len"], g["edges"]),
                              gfa2_text(g["node_len"], g["edges"], order)]):
        p = tmp_path / f"g{k}.gfa"
        p.write_text(text)
        for ordering in ("native", "topological"):
            want_nl, want_e, _ = gfa.parse(text, ordering)
            nl, e = _cpp_read(tool, p, ordering)
            assert np.array_equal(nl, want_nl) and same_edges(e, want_e), (k, ordering)


@pytest.mark.gpu
@pytest.mark.parametrize("name", FIXTURES)
def test_fixture_graphs_to_index_on_the_device(name):
    from diverg_b200.runtime import Context
    g = load_golden(f"gfa_{name}.npz")
    node_len, edges, _ = gfa.parse(gfa2_text(g["node_len"], g["edges"]))
    ctx = Context(0)
    try:
        a = ctx.adjacency_from_graph(node_len, edges)
        got = a.download()
        assert np.array_equal(got.rowmap.astype(np.uint64), g["A_rowmap"]) and np.array_equal(got.entries, g["A_entries"])
        idx = ctx.distance_index(a, 1, 8).download()
        assert np.array_equal(idx.rowmap.astype(np.uint64), g["D1_8_rowmap"])
        assert np.array_equal(idx.entries, g["D1_8_entries"]) and idx.nnz() == int(g["D1_8_nnz"])
    finally:
        ctx.close()
