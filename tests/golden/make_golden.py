"""Generates the committed golden fixtures under tests/golden/.

Run where a checkout of the reference exists, never on the GPU host; the
checkout's path is a required argument:

    python tests/golden/make_golden.py /path/to/reference

It reads the reference's own test data as text:
  * the HBitVector known-answer vectors of test/src/test_hbitvector.cpp
    (input rows at :186-234, expected canonical rows at :618-661), and
  * the GFA2 graphs test/data/{small/x,multi/multi,middle/m}.gfa,
builds each graph's range-CRS adjacency with the oracle's restatement of
util::adjacency_matrix (adjacency.hpp:170-228), and stores the adjacency
together with the oracle's results for the products the reference's tests
run on these graphs (test_range_sparse.cpp:556-585 A*A, :631-659 A^100,
:708-736 A+I; test_dindex.cpp:177-234 index [1,8] and [1,3]) plus the index
windows used by the benchmarks.  Every stored result is checked here against
an independent dense bitset brute force before it is written.
"""
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))

from oracle import pyoracle as orc  # noqa: E402

if len(sys.argv) != 2 or not os.path.isdir(sys.argv[1]):
    sys.exit("usage: python tests/golden/make_golden.py /path/to/reference-checkout")
REF = sys.argv[1]


# ---- known-answer vectors -----------------------------------------------------

def parse_assignments(lines, name):
    """`name( i ) = v;` assignments in order, as {i: v}."""
    pat = re.compile(r"\b" + re.escape(name) + r"\(\s*(\d+)\s*\)\s*=\s*(\d+)\s*;")
    out = {}
    for ln in lines:
        for m in pat.finditer(ln):
            out[int(m.group(1))] = int(m.group(2))
    return out


def hbv_known_answer():
    path = os.path.join(REF, "test/src/test_hbitvector.cpp")
    lines = open(path).read().splitlines()
    # input block: test_hbitvector.cpp:186-234 (1-based, inclusive)
    block_in = lines[185:234]
    # expected block: test_hbitvector.cpp:618-661
    block_out = lines[617:661]
    e_in = parse_assignments(block_in, "h_e")
    r_in = parse_assignments(block_in, "h_row_map")
    e_out = parse_assignments(block_out, "h_t_e")
    r_out = parse_assignments(block_out, "h_t_row_map")
    to_arr = lambda d: np.array([d[i] for i in range(len(d))], dtype=np.uint64)  # noqa: E731
    ki = {"in_entries": to_arr(e_in).astype(np.uint32), "in_rowmap": to_arr(r_in),
          "out_entries": to_arr(e_out).astype(np.uint32), "out_rowmap": to_arr(r_out),
          # HBitVector< 1024..4096 > over 11431 columns (test_hbitvector.cpp:171-173)
          "ncols": np.array(11431, dtype=np.uint64)}
    assert len(ki["in_rowmap"]) == 6 and ki["in_rowmap"][-1] == len(ki["in_entries"]) == 34
    assert len(ki["out_rowmap"]) == 6 and ki["out_rowmap"][-1] == len(ki["out_entries"]) == 32
    return ki


# ---- GFA fixtures --------------------------------------------------------------

def load_gfa2(path):
    """Minimal GFA2 reader for the fixtures: S <id> <len> <seq>, E <eid> <a>+ <b>+ ..."""
    lens = {}
    edges = []
    for ln in open(path):
        f = ln.rstrip("\n").split("\t")
        if f[0] == "S":
            lens[int(f[1])] = int(f[2])
        elif f[0] == "E":
            a, b = f[2], f[3]
            assert a.endswith("+") and b.endswith("+"), "fixture edges are forward only"
            edges.append((int(a[:-1]), int(b[:-1])))
    ids = sorted(lens)
    assert ids == list(range(1, len(ids) + 1)), "fixture ids are contiguous from 1"
    for a, b in edges:
        assert a < b, "id order is a topological order"
    node_len = np.array([lens[i] for i in ids], dtype=np.uint32)
    return node_len, np.array(edges, dtype=np.uint32).reshape(-1, 2)


# ---- independent brute force: dense bitset rows --------------------------------

def to_bits(m):
    d = orc.to_dense(m)
    return np.packbits(d, axis=1, bitorder="little")


def bits_to_omat(bits, ncols):
    d = np.unpackbits(bits, axis=1, count=ncols, bitorder="little").astype(bool)
    return orc.from_dense(d)


def bits_mul(a_bits, b_bits, ncols):
    """C[i] = OR over j in A[i] of B[j]."""
    a = np.unpackbits(a_bits, axis=1, count=ncols, bitorder="little").astype(bool)
    out = np.zeros_like(b_bits)
    for i in range(a.shape[0]):
        js = np.flatnonzero(a[i])
        if len(js):
            out[i] = np.bitwise_or.reduce(b_bits[js], axis=0)
    return out


def bits_identity(n):
    return np.packbits(np.eye(n, dtype=bool), axis=1, bitorder="little")


def bits_power(a_bits, k, n):
    res = bits_identity(n)
    base = a_bits.copy()
    while k:
        if k & 1:
            res = bits_mul(res, base, n)
        k >>= 1
        if k:
            base = bits_mul(base, base, n)
    return res


def check_same(name, got, bits, ncols):
    want = bits_to_omat(bits, ncols)
    assert np.array_equal(got.rowmap, want.rowmap), name
    assert np.array_equal(got.entries, want.entries), name
    assert got.nnz == want.nnz, name


def main():
    ki = hbv_known_answer()
    a = orc.OMat(5, int(ki["ncols"]), ki["in_rowmap"], ki["in_entries"], 0)
    a.nnz = orc.nnz(a)
    # C = I * A canonicalises every row of A: the known answer.
    ident = orc.OMat(5, 5, np.arange(0, 12, 2, dtype=np.uint64), np.repeat(np.arange(5, dtype=np.uint32), 2), 5)
    got = orc.spgemm(ident, a)
    assert np.array_equal(got.rowmap, ki["out_rowmap"]) and np.array_equal(got.entries, ki["out_entries"])
    np.savez_compressed(os.path.join(HERE, "hbv_known_answer.npz"), **ki)
    print("hbv known answer: ok")

    for name, rel, products in [
        ("x", "test/data/small/x.gfa", ["AA", "AI", "P100", "D1_8", "D1_3", "D0_50", "D100_300"]),
        ("multi", "test/data/multi/multi.gfa", ["AA", "AI", "P100", "D1_8", "D1_3", "D0_50", "D100_300"]),
        ("m", "test/data/middle/m.gfa", ["AA", "AI", "P100", "D1_8", "D100_300"]),
    ]:
        node_len, edges = load_gfa2(os.path.join(REF, rel))
        A = orc.adjacency(node_len, edges)
        n = A.nrows
        ab = to_bits(A)
        out = {"node_len": node_len, "edges": edges, "A_rowmap": A.rowmap, "A_entries": A.entries,
               "A_nnz": np.array(A.nnz, dtype=np.uint64), "n": np.array(n, dtype=np.uint64)}
        for p in products:
            if p == "AA":
                r = orc.spgemm(A, A)
                check_same(name + p, r, bits_mul(ab, ab, n), n)
            elif p == "AI":
                r = orc.spadd(A, orc.identity(n))
                check_same(name + p, r, ab | bits_identity(n), n)
            elif p.startswith("P"):
                k = int(p[1:])
                r = orc.power(A, k)
                check_same(name + p, r, bits_power(ab, k, n), n)
            else:
                lo, hi = map(int, p[1:].split("_"))
                r = orc.dindex(A, lo, hi)
                want = bits_power(ab | bits_identity(n), hi - lo, n)
                if lo:
                    want = bits_mul(bits_power(ab, lo, n), want, n)
                check_same(name + p, r, want, n)
                # the bitvector restatement (the timed CPU baseline) agrees
                assert orc.dindex(A, lo, hi, algo="hbv").same(r), name + p
            out[p + "_rowmap"] = r.rowmap
            out[p + "_entries"] = r.entries
            out[p + "_nnz"] = np.array(r.nnz, dtype=np.uint64)
            print(f"{name} {p}: ranges={len(r.entries) // 2} nnz={r.nnz} ok")
        np.savez_compressed(os.path.join(HERE, f"gfa_{name}.npz"), **out)


if __name__ == "__main__":
    main()
