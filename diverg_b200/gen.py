"""Synthetic workloads (libdvg_gen.so, include/dvg_gen.h) as CRSMatrix objects."""
import ctypes
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .crs_matrix import CRSMatrix


@dataclass
class GraphSpec:
    """Bubble model of a synthetic sequence graph (see dvg_graph_params)."""
    n_backbone: int
    snp_rate: float
    indel_rate: float
    ins_frac: float = 0.5
    indel_lmin: int = 1
    indel_lmax: int = 10
    indel_geometric_mean: float = 0.0
    sv_frac: float = 0.0
    sv_lmin: int = 100
    sv_lmax: int = 2000
    seed: int = 42

    def params(self):
        return N.GraphParams(self.n_backbone, self.snp_rate, self.indel_rate, self.ins_frac, self.indel_lmin,
                             self.indel_lmax, self.indel_geometric_mean, self.sv_frac, self.sv_lmin, self.sv_lmax,
                             self.seed)


def small_graph_spec(n_backbone=100_000, seed=42):
    """1e5 bases, bubbles at 1/100 per base: 70 % SNP, 30 % indel (insertion
    or deletion 50/50, length uniform 1..10)."""
    return GraphSpec(n_backbone, 0.007, 0.003, 0.5, 1, 10, 0.0, 0.0, 100, 2000, seed)


def chromosome_graph_spec(n_backbone=50_000_000, seed=42):
    """5e7 bases, SNP 1/1000, indel 1/5000 (geometric length, mean 4, cap 50),
    0.1 % of bubbles structural (length uniform 100..2000)."""
    return GraphSpec(n_backbone, 1e-3, 2e-4, 0.5, 1, 50, 4.0, 1e-3, 100, 2000, seed)


def _take(hm: N.HostMatrix) -> CRSMatrix:
    n, ne = hm.nrows, hm.nentries
    rowmap = np.ctypeslib.as_array(hm.rowmap, shape=(n + 1,)).copy()
    entries = (np.ctypeslib.as_array(hm.entries, shape=(ne,)).copy() if ne else np.zeros(0, np.uint32))
    nnz = int(hm.nnz)
    N.gen_lib().dvg_gen_free(ctypes.byref(hm))
    return CRSMatrix(hm.ncols, entries, rowmap, nnz if nnz else 0)


def graph_adjacency(spec: GraphSpec):
    """Range-CRS adjacency of the synthetic graph and its generation counts."""
    hm, st = N.HostMatrix(), N.GraphStats()
    p = spec.params()
    rc = N.gen_lib().dvg_gen_graph_adjacency(ctypes.byref(p), ctypes.byref(hm), ctypes.byref(st))
    if rc:
        raise ValueError(f"graph generator failed ({rc})")
    stats = {name: int(getattr(st, name)) for name, _ in st._fields_}
    return _take(hm), stats


def graph_edges(spec: GraphSpec):
    """(n_nodes, edges[k, 2]) with one single-base node per locus, ids 1-based."""
    nn, ne = ctypes.c_uint64(), ctypes.c_uint64()
    ep = ctypes.POINTER(ctypes.c_uint32)()
    p = spec.params()
    rc = N.gen_lib().dvg_gen_graph_edges(ctypes.byref(p), ctypes.byref(nn), ctypes.byref(ne), ctypes.byref(ep))
    if rc:
        raise ValueError(f"graph generator failed ({rc})")
    edges = np.ctypeslib.as_array(ep, shape=(2 * ne.value,)).copy().reshape(-1, 2) if ne.value else \
        np.zeros((0, 2), np.uint32)
    N.gen_lib().dvg_gen_free_ptr(ctypes.cast(ep, ctypes.c_void_p))
    return int(nn.value), edges


def graph_nodes(spec: GraphSpec):
    """The synthetic graph with its chains of bases compacted into nodes:
    (node_len uint32[N] for ids 1..N in rank order, edges uint32[E, 2] of
    (from_id, to_id)).  Its range adjacency is graph_adjacency(spec)."""
    nn, ne = ctypes.c_uint64(), ctypes.c_uint64()
    lp, ep = ctypes.POINTER(ctypes.c_uint32)(), ctypes.POINTER(ctypes.c_uint32)()
    p = spec.params()
    rc = N.gen_lib().dvg_gen_graph_nodes(ctypes.byref(p), ctypes.byref(nn), ctypes.byref(lp), ctypes.byref(ne),
                                         ctypes.byref(ep))
    if rc:
        raise ValueError(f"graph generator failed ({rc})")
    lens = np.ctypeslib.as_array(lp, shape=(nn.value,)).copy() if nn.value else np.zeros(0, np.uint32)
    edges = np.ctypeslib.as_array(ep, shape=(2 * ne.value,)).copy().reshape(-1, 2) if ne.value else \
        np.zeros((0, 2), np.uint32)
    N.gen_lib().dvg_gen_free_ptr(ctypes.cast(lp, ctypes.c_void_p))
    N.gen_lib().dvg_gen_free_ptr(ctypes.cast(ep, ctypes.c_void_p))
    return lens, edges


def banded(n, half_width=512, mean_ranges=4.0, mean_len=32.0, seed=42) -> CRSMatrix:
    """Random banded matrix, canonical rows (see dvg_gen_banded)."""
    hm = N.HostMatrix()
    rc = N.gen_lib().dvg_gen_banded(n, half_width, mean_ranges, mean_len, seed, ctypes.byref(hm))
    if rc:
        raise ValueError(f"banded generator failed ({rc})")
    return _take(hm)


def random_matrix(n, nnz, seed=42) -> CRSMatrix:
    """Uniformly random Boolean matrix with exactly nnz non-zeros."""
    hm = N.HostMatrix()
    rc = N.gen_lib().dvg_gen_random(n, nnz, seed, ctypes.byref(hm))
    if rc:
        raise ValueError(f"random generator failed ({rc})")
    return _take(hm)


def query_pairs(adj: CRSMatrix, npairs, in_range_frac=0.5, dmin=200, dmax=500, seed=7) -> np.ndarray:
    """(npairs, 2) uint32 locus pairs (see dvg_gen_pairs)."""
    rowmap = np.ascontiguousarray(adj.rowmap, dtype=np.uint64)
    entries = np.ascontiguousarray(adj.entries, dtype=np.uint32)
    hm = N.HostMatrix(adj.numRows(), adj.numCols(), entries.size, adj.nnz(),
                      rowmap.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                      entries.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
    out = np.empty((npairs, 2), dtype=np.uint32)
    rc = N.gen_lib().dvg_gen_pairs(ctypes.byref(hm), npairs, in_range_frac, dmin, dmax, seed, N.ptr(out))
    if rc:
        raise ValueError(f"pair generator failed ({rc})")
    return out
