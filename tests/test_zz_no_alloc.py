"""dvg_range_spgemm_noalloc: the SpGEMM entry point for callers that may not
let the library allocate device memory (a server that pre-reserves the GPU's
memory for resident indices, a host runtime that owns every device allocation,
a latency-critical path that cannot afford cudaMalloc's synchronisation).

The test calls it through the C ABI with caller-owned device buffers and
checks its output, exactly (integer data), against the allocating entry point
dvg_range_spgemm on two different products in a row -- the second call runs on
the scratch the first one left behind.  It also checks the capacity overflow
contract and the size limit.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from diverg_b200 import _native as N, gen
from diverg_b200.runtime import Context

pytestmark = pytest.mark.gpu

ROW_LIMIT = 67_108_864


def noalloc(a, b, c_rowmap, c_entries, cap):
    """Calls dvg_range_spgemm_noalloc on DeviceMatrix inputs and torch output
    buffers; returns (status, nentries, nnz)."""
    ar, ae = a.device_arrays()
    br, be = b.device_arrays()
    ne, nz = ctypes.c_uint64(), ctypes.c_uint64()
    st = N.lib().dvg_range_spgemm_noalloc(
        a.nrows, a.ncols, ctypes.c_void_p(ar), ctypes.c_void_p(ae), a.nentries,
        b.nrows, b.ncols, ctypes.c_void_p(br), ctypes.c_void_p(be), b.nentries,
        ctypes.c_void_p(c_rowmap.data_ptr()), ctypes.c_void_p(c_entries.data_ptr() if cap else 0), cap,
        ctypes.byref(ne), ctypes.byref(nz), ctypes.c_void_p(0))
    return st, ne.value, nz.value


def test_noalloc_matches_the_allocating_spgemm_on_two_calls_in_a_row():
    import torch
    ctx = Context(0)
    try:
        g, _ = gen.graph_adjacency(gen.small_graph_spec(300_000, seed=5))
        d_g = ctx.upload(g)
        x = ctx.spadd(d_g, ctx.identity(d_g.nrows))          # A + I
        x8 = ctx.power(x, 8)                                   # (A + I)^8
        b1 = ctx.upload(gen.banded(1 << 16, 512, 4.0, 32.0, seed=61))
        b2 = ctx.upload(gen.banded(1 << 16, 512, 4.0, 32.0, seed=62))
        for a, b in ((x8, x8), (b1, b2)):
            want = ctx.spgemm(a, b).download()
            n = a.nrows
            c_rowmap = torch.full((n + 1,), -1, dtype=torch.int64, device="cuda")
            c_entries = torch.full((want.entries.size + 64,), -1, dtype=torch.int32, device="cuda")
            st, ne, nz = noalloc(a, b, c_rowmap, c_entries, c_entries.numel())
            assert st == N.OK, N.lib().dvg_last_error()
            assert ne == want.entries.size and nz == want.nnz()
            got_rowmap = c_rowmap.cpu().numpy().view(np.uint64)
            got_entries = c_entries[:ne].cpu().numpy().view(np.uint32)
            assert np.array_equal(got_rowmap, want.rowmap)
            assert np.array_equal(got_entries, want.entries)
    finally:
        ctx.close()


def test_noalloc_reports_the_needed_capacity():
    import torch
    ctx = Context(0)
    try:
        a = ctx.upload(gen.banded(20_000, 64, 4.0, 8.0, seed=63))
        want = ctx.spgemm(a, a).download()
        c_rowmap = torch.empty(a.nrows + 1, dtype=torch.int64, device="cuda")
        small = torch.empty(16, dtype=torch.int32, device="cuda")
        st, ne, _ = noalloc(a, a, c_rowmap, small, small.numel())
        assert st == N.OVERFLOW and ne == want.entries.size
        assert np.array_equal(c_rowmap.cpu().numpy().view(np.uint64), want.rowmap)
        big = torch.empty(ne, dtype=torch.int32, device="cuda")
        st, ne2, nz = noalloc(a, a, c_rowmap, big, big.numel())
        assert st == N.OK and ne2 == ne and nz == want.nnz()
        assert np.array_equal(big.cpu().numpy().view(np.uint32), want.entries)
    finally:
        ctx.close()


def test_noalloc_rejects_products_beyond_its_scratch():
    # the size check precedes any use of the (dummy, never dereferenced) pointers
    ne, nz = ctypes.c_uint64(), ctypes.c_uint64()
    dummy = ctypes.c_void_p(0x1000)
    st = N.lib().dvg_range_spgemm_noalloc(ROW_LIMIT + 1, 10, dummy, dummy, 0, 10, 10, dummy, dummy, 0, dummy,
                                          dummy, 0, ctypes.byref(ne), ctypes.byref(nz), ctypes.c_void_p(0))
    assert st == N.INVALID_ARG
    assert b"67108864" in N.lib().dvg_last_error()
