"""The N > 1 host path on CPU: component blocks sharded over world-size-2 gloo
ranks, each rank building its blocks' indices (the oracle stands in for the
per-rank GPU build here), the gather and block-diagonal assembly on rank 0, and
the max-over-ranks timing reduction that the benchmark uses.  The assembled
index must equal the index of the whole multi-component graph.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from diverg_b200 import gen, sharding
from diverg_b200.crs_matrix import CRSMatrix


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _graph(n_parts=5, seed=7):
    parts = []
    for k in range(n_parts):
        g, _ = gen.graph_adjacency(gen.small_graph_spec(2_000 + 1_500 * k, seed=seed + k))
        parts.append(g)
    return sharding.block_diagonal(parts)


def _to_crs(o):
    return CRSMatrix(o.ncols, o.entries.copy(), o.rowmap.copy(), o.nnz)


def _oracle_index(m, dlo, dup):
    from oracle import pyoracle as orc
    om = orc.OMat(m.numRows(), m.numCols(), m.rowmap.astype(np.uint64), m.entries, m.nnz())
    return _to_crs(orc.dindex(om, dlo, dup, algo="hbv"))


def _rank_main(rank, world, port, out_dir, dlo, dup):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        a = _graph()
        mine = sharding.shard_of(a, rank, world, weights="entries")
        built = [(lo, hi, _oracle_index(blk, dlo, dup)) for lo, hi, blk in mine]
        gathered = [None] * world
        dist.all_gather_object(gathered, [(lo, hi, m.num_cols, m.rowmap, m.entries, m.m_nnz)
                                          for lo, hi, m in built])
        t = torch.tensor([1.5 + rank], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        if rank == 0:
            parts = [(lo, hi, CRSMatrix(nc, e, r, z)) for per in gathered for lo, hi, nc, r, e, z in per]
            whole = sharding.assemble(a.numRows(), parts)
            want = _oracle_index(a, dlo, dup)
            np.savez(os.path.join(out_dir, "r0.npz"), ok=whole == want, tmax=float(t.item()),
                     nblocks=len(parts), counts=[len(p) for p in gathered])
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_sharded_build_over_two_gloo_ranks_equals_whole_graph_index(tmp_path):
    world = 2
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, str(tmp_path), 20, 60)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    r = np.load(tmp_path / "r0.npz")
    assert bool(r["ok"])
    assert float(r["tmax"]) == 2.5
    assert int(r["nblocks"]) == 5 and all(int(c) > 0 for c in r["counts"])


def test_component_blocks_find_the_parts_and_only_them():
    a = _graph(4, seed=3)
    blocks = sharding.component_blocks(a)
    assert len(blocks) == 4
    for lo, hi in blocks:
        sharding.extract_block(a, lo, hi)          # raises unless diagonal
    assert sharding.block_diagonal([sharding.extract_block(a, lo, hi) for lo, hi in blocks]) == a
    # a single connected graph is one block
    g, _ = gen.graph_adjacency(gen.small_graph_spec(3_000, seed=1))
    assert sharding.component_blocks(g) == [(0, g.numRows())]


def test_plan_shards_is_contiguous_and_covers_every_block():
    blocks = [(0, 10), (10, 15), (15, 40), (40, 41), (41, 100)]
    for world in (1, 2, 3, 4, 8):
        shards = sharding.plan_shards(blocks, world)
        assert len(shards) == world
        flat = [k for s in shards for k in s]
        assert flat == list(range(len(blocks)))
    assert sharding.plan_shards(blocks, 2) == [[0, 1, 2, 3], [4]]


def test_assemble_rejects_gaps_and_overlaps():
    m = CRSMatrix(2, np.array([0, 1, 1, 1], np.uint32), np.array([0, 2, 4], np.uint64))
    with pytest.raises(ValueError):
        sharding.assemble(5, [(0, 2, m), (3, 5, m)])
    with pytest.raises(ValueError):
        sharding.assemble(3, [(0, 2, m), (1, 3, m)])
    assert sharding.assemble(4, [(2, 4, m), (0, 2, m)]).numRows() == 4
