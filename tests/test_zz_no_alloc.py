"""dvg_range_spgemm_noalloc: the SpGEMM entry point for callers that may not
let the library allocate device memory (a server that pre-reserves the GPU's
memory for resident indices, a host runtime that owns every device allocation,
a latency-critical path that cannot afford cudaMalloc's synchronisation).

The test calls it through the C ABI with caller-owned device buffers and
checks its output, exactly (integer data), against the allocating entry point
dvg_range_spgemm and the CPU oracle on two different products in a row -- the
second call runs on the scratch the first one left behind.  It also checks the
capacity overflow contract, the size limit and the rejection of malformed
inputs on the device.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from diverg_b200 import _native as N, gen
from diverg_b200.runtime import Context
from oracle import pyoracle as orc

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
            ha, hb = a.download(), b.download()
            ref = orc.spgemm(orc.OMat(ha.numRows(), ha.numCols(), ha.rowmap.astype(np.uint64), ha.entries, ha.nnz()),
                             orc.OMat(hb.numRows(), hb.numCols(), hb.rowmap.astype(np.uint64), hb.entries, hb.nnz()))
            assert np.array_equal(got_rowmap, ref.rowmap) and np.array_equal(got_entries, ref.entries)
            assert nz == ref.nnz
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


# (rowmap, entries, ncols, nentries passed, the check the message names): small
# matrices that break one precondition each; every read of the check stays
# inside the buffers (rowmap[0..n], entries[0..nentries))
MALFORMED = [
    ([2, 2, 4], [0, 1, 2, 3], 8, 4, "rowmap[0] != 0"),
    ([0, 3, 4], [0, 1, 2, 3], 8, 4, "odd row length"),
    ([0, 2, 4], [0, 1, 2, 3], 8, 2, "rowmap[nrows] != number of entries"),
    ([0, 2, 4], [0, 1, 2, 8], 8, 4, "column index >= ncols"),
]


@pytest.mark.parametrize("case", MALFORMED, ids=[c[4] for c in MALFORMED])
@pytest.mark.parametrize("operand", ["A", "B"])
def test_noalloc_rejects_malformed_inputs_before_the_product(case, operand):
    import torch
    rowmap, entries, ncols, nent, why = case
    bad_r = torch.tensor(np.array(rowmap, dtype=np.uint64).view(np.int64), device="cuda")
    bad_e = torch.tensor(np.array(entries, dtype=np.uint32).view(np.int32), device="cuda")
    n = len(rowmap) - 1
    # a well-formed n x ncols (as A) or ncols x ncols (as B) partner: the identity
    good_n = ncols if operand == "A" else n
    good_r = torch.tensor(np.arange(0, 2 * good_n + 1, 2, dtype=np.uint64).view(np.int64), device="cuda")
    good_e = torch.tensor(np.repeat(np.arange(good_n, dtype=np.uint32), 2).view(np.int32), device="cuda")
    if operand == "A":
        a = (n, ncols, bad_r, bad_e, nent)
        b = (ncols, ncols, good_r, good_e, 2 * ncols)
    else:
        a = (n, n, good_r, good_e, 2 * n)
        b = (n, ncols, bad_r, bad_e, nent)
    c_rowmap = torch.full((a[0] + 1,), -1, dtype=torch.int64, device="cuda")
    c_entries = torch.full((64,), -1, dtype=torch.int32, device="cuda")
    ne, nz = ctypes.c_uint64(), ctypes.c_uint64()
    st = N.lib().dvg_range_spgemm_noalloc(
        a[0], a[1], ctypes.c_void_p(a[2].data_ptr()), ctypes.c_void_p(a[3].data_ptr()), a[4],
        b[0], b[1], ctypes.c_void_p(b[2].data_ptr()), ctypes.c_void_p(b[3].data_ptr()), b[4],
        ctypes.c_void_p(c_rowmap.data_ptr()), ctypes.c_void_p(c_entries.data_ptr()), c_entries.numel(),
        ctypes.byref(ne), ctypes.byref(nz), ctypes.c_void_p(0))
    msg = N.lib().dvg_last_error().decode()
    assert st == N.INVALID_ARG, msg
    assert f"{operand}:" in msg and why in msg, msg
    assert bool((c_rowmap == -1).all()) and bool((c_entries == -1).all())
