"""Independent components of a range-CRS matrix, and their distribution over ranks.

A sequence graph made of several connected components has, in topological
locus order, a block-diagonal adjacency matrix; every power of it, and so its
distance index, is block-diagonal with the same blocks (the reference builds
per-component indices and combines them: crs_matrix.hpp:1448-1518 assembles
rows component by component, dindex.hpp:290-491 merges indices).  Blocks are
therefore units of work that share no data: a rank builds the indices of its
blocks alone, and assembling the blocks' indices side by side gives the index
of the whole graph.  The only exchange is an optional gather of the results.

All functions here are host-side (numpy); the builds themselves run through
runtime.Context on each rank's GPU.
"""
import numpy as np

from .crs_matrix import CRSMatrix


def component_blocks(a: CRSMatrix):
    """Splits [0, n) at every row p where no entry of rows < p has a column
    >= p and no entry of rows >= p has a column < p.  Returns the half-open
    row ranges [(lo, hi), ...]; each is a diagonal block of a (square)."""
    n = a.numRows()
    if n == 0:
        return []
    if a.numCols() != n:
        raise ValueError("component blocks need a square matrix")
    rm = a.rowmap.astype(np.int64)
    counts = rm[1:] - rm[:-1]
    has = counts > 0
    row_max = np.full(n, -1, np.int64)
    row_min = np.full(n, n, np.int64)
    if has.any():
        row_max[has] = a.entries[(rm[1:] - 1)[has]]   # last range's end
        row_min[has] = a.entries[rm[:-1][has]]        # first range's start
    pref_max = np.maximum.accumulate(row_max)         # max column in rows [0, p]
    suf_min = np.minimum.accumulate(row_min[::-1])[::-1]  # min column in rows [p, n)
    p = np.arange(1, n)
    cut = (pref_max[:-1] < p) & (suf_min[1:] >= p)
    edges = np.concatenate(([0], p[cut], [n]))
    return [(int(edges[k]), int(edges[k + 1])) for k in range(len(edges) - 1)]


def extract_block(a: CRSMatrix, lo: int, hi: int) -> CRSMatrix:
    """Rows and columns [lo, hi) of a as an (hi-lo) x (hi-lo) matrix; the
    block must be diagonal (no entry of its rows outside [lo, hi))."""
    rm = a.rowmap.astype(np.uint64)
    e0, e1 = int(rm[lo]), int(rm[hi])
    ent = a.entries[e0:e1]
    if ent.size and (int(ent.min()) < lo or int(ent.max()) >= hi):
        raise ValueError(f"rows [{lo},{hi}) are not a diagonal block")
    return CRSMatrix(hi - lo, (ent.astype(np.int64) - lo).astype(np.uint32), rm[lo:hi + 1] - rm[lo],
                     size_type=np.uint64)


def block_diagonal(blocks) -> CRSMatrix:
    """The block-diagonal matrix diag(blocks[0], blocks[1], ...) (square blocks)."""
    rowmaps, entries = [np.zeros(1, np.uint64)], []
    off_rows, off_entries, nnz = 0, 0, 0
    for b in blocks:
        if b.numRows() != b.numCols():
            raise ValueError("block_diagonal needs square blocks")
        rm = b.rowmap.astype(np.uint64)
        rowmaps.append(rm[1:] + np.uint64(off_entries))
        entries.append((b.entries.astype(np.int64) + off_rows).astype(np.uint32))
        off_rows += b.numRows()
        off_entries += int(rm[-1])
        nnz += b.nnz()
    ent = np.concatenate(entries) if entries else np.zeros(0, np.uint32)
    return CRSMatrix(off_rows, ent, np.concatenate(rowmaps), nnz)


def plan_shards(blocks, world: int, weights=None):
    """Assigns contiguous runs of blocks to `world` ranks so that the summed
    weights (default: rows) are as even as contiguity allows.  Returns, per
    rank, the list of block indices; a rank may get none."""
    nb = len(blocks)
    w = np.asarray([hi - lo for lo, hi in blocks] if weights is None else weights, np.float64)
    if w.size != nb:
        raise ValueError("one weight per block")
    if world < 1:
        raise ValueError("world must be >= 1")
    total = float(w.sum())
    cum = np.concatenate(([0.0], np.cumsum(w)))
    shards, start = [], 0
    for r in range(world):
        if r == world - 1:
            end = nb
        else:
            target = total * (r + 1) / world
            end = int(np.searchsorted(cum, target, side="left"))
            # round to the nearer boundary, keep order
            if end > start and end <= nb and abs(cum[end - 1] - target) < abs(cum[end] - target):
                end -= 1
            end = max(start, min(end, nb))
        shards.append(list(range(start, end)))
        start = end
    return shards


def shard_of(a: CRSMatrix, rank: int, world: int, weights=None):
    """The blocks of a that rank `rank` builds: [(lo, hi, block_matrix), ...]."""
    blocks = component_blocks(a)
    if weights == "entries":
        rm = a.rowmap.astype(np.int64)
        weights = [int(rm[hi] - rm[lo]) + 1 for lo, hi in blocks]
    mine = plan_shards(blocks, world, weights)[rank]
    return [(blocks[k][0], blocks[k][1], extract_block(a, *blocks[k])) for k in mine]


def assemble(n: int, parts) -> CRSMatrix:
    """Index of the whole graph from the per-block indices [(lo, hi, index)]
    that together tile [0, n)."""
    parts = sorted(parts, key=lambda t: t[0])
    pos = 0
    for lo, hi, m in parts:
        if lo != pos or m.numRows() != hi - lo:
            raise ValueError(f"blocks do not tile [0,{n}): gap or overlap at {pos}")
        pos = hi
    if pos != n:
        raise ValueError(f"blocks do not tile [0,{n}): end at {pos}")
    return block_diagonal([m for _, _, m in parts])
