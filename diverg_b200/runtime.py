"""Device runtime: contexts and device-resident matrices.

Mirrors the reference's runtime.hpp:22-53 (is_runtime_initialized,
initialize_runtime, finalize_runtime, ScopedRuntime) over dvg_init / dvg_shutdown, and adds the
device-resident handles the reference does not have: a DeviceMatrix stays in
HBM between calls, so chains of operations and query batches pay no host
round trip.
"""
import ctypes
import threading

import numpy as np

from . import _native as N
from .crs_matrix import CRSMatrix


class Context:
    """One CUDA device and stream (dvg_context)."""

    def __init__(self, device=0):
        L = N.lib()
        h = ctypes.c_void_p()
        N.check(L.dvg_init(device, ctypes.byref(h)))
        self._h = h
        self.device = device

    @property
    def handle(self):
        if self._h is None:
            raise RuntimeError("context is closed")
        return self._h

    def close(self):
        if self._h is not None:
            N.check(N.lib().dvg_shutdown(self._h))
            self._h = None

    def set_stream(self, cuda_stream_handle):
        """Issue all work on an external cudaStream_t (an int handle, e.g.
        torch.cuda.current_stream().cuda_stream); None restores the own one."""
        N.check(N.lib().dvg_set_stream(self.handle, ctypes.c_void_p(cuda_stream_handle or 0)))

    def synchronize(self):
        N.check(N.lib().dvg_synchronize(self.handle))

    def set_option(self, key, value):
        N.check(N.lib().dvg_set_option(self.handle, key.encode(), int(value)))

    def trim(self):
        """Return the device memory cached by the context to CUDA."""
        N.check(N.lib().dvg_trim(self.handle))

    def stats(self):
        s = N.DvgStats()
        N.check(N.lib().dvg_get_stats(self.handle, ctypes.byref(s)))
        return s.as_dict()

    def reset_stats(self):
        N.check(N.lib().dvg_stats_reset(self.handle))

    def calibrate_range_ops(self):
        """Range operations a second the device sustains for the warp-per-row
        SpGEMM's inner work (the denominator of its on-chip roofline)."""
        v = ctypes.c_double()
        N.check(N.lib().dvg_calibrate_range_ops(self.handle, ctypes.byref(v)))
        return v.value

    def calibrate_random_reads(self, nbytes):
        """Independent random 8-byte reads a second over a device buffer of
        nbytes (the denominator of the membership query's roofline)."""
        v = ctypes.c_double()
        N.check(N.lib().dvg_calibrate_random_reads(self.handle, nbytes, ctypes.byref(v)))
        return v.value

    # -- matrices ---------------------------------------------------------------
    def upload(self, m: CRSMatrix) -> "DeviceMatrix":
        L = N.lib()
        h = ctypes.c_void_p()
        rowmap = np.ascontiguousarray(m.rowmap)
        entries = np.ascontiguousarray(m.entries, dtype=np.uint32)
        if rowmap.dtype == np.uint32:
            st = L.dvg_matrix_upload_u32(self.handle, m.numRows(), m.numCols(), N.ptr(rowmap), N.ptr(entries),
                                         m.nnz(), ctypes.byref(h))
        else:
            rowmap = rowmap.astype(np.uint64, copy=False)
            st = L.dvg_matrix_upload(self.handle, m.numRows(), m.numCols(), N.ptr(rowmap), N.ptr(entries),
                                     m.nnz(), ctypes.byref(h))
        N.check(st)
        return DeviceMatrix(self, h)

    def upload_arrays(self, nrows, ncols, rowmap, entries, nnz=0) -> "DeviceMatrix":
        """Upload from raw host arrays (rowmap uint64, may be pinned memory)."""
        h = ctypes.c_void_p()
        N.check(N.lib().dvg_matrix_upload(self.handle, nrows, ncols, ctypes.c_void_p(rowmap),
                                          ctypes.c_void_p(entries), nnz, ctypes.byref(h)))
        return DeviceMatrix(self, h)

    def wrap_device(self, nrows, ncols, d_rowmap, d_entries, nentries, nnz) -> "DeviceMatrix":
        h = ctypes.c_void_p()
        N.check(N.lib().dvg_matrix_wrap_device(self.handle, nrows, ncols, ctypes.c_void_p(d_rowmap),
                                               ctypes.c_void_p(d_entries), nentries, nnz, ctypes.byref(h)))
        return DeviceMatrix(self, h)

    def identity(self, n) -> "DeviceMatrix":
        h = ctypes.c_void_p()
        N.check(N.lib().dvg_range_identity(self.handle, n, ctypes.byref(h)))
        return DeviceMatrix(self, h)

    def spgemm(self, a, b) -> "DeviceMatrix":
        h = ctypes.c_void_p()
        N.check(N.lib().dvg_range_spgemm(self.handle, a.handle, b.handle, ctypes.byref(h)))
        return DeviceMatrix(self, h)

    def spadd(self, a, b) -> "DeviceMatrix":
        h = ctypes.c_void_p()
        N.check(N.lib().dvg_range_spadd(self.handle, a.handle, b.handle, ctypes.byref(h)))
        return DeviceMatrix(self, h)

    def power(self, a, k) -> "DeviceMatrix":
        h = ctypes.c_void_p()
        N.check(N.lib().dvg_range_power(self.handle, a.handle, k, ctypes.byref(h)))
        return DeviceMatrix(self, h)

    def distance_index(self, a, dmin, dmax) -> "DeviceMatrix":
        h = ctypes.c_void_p()
        N.check(N.lib().dvg_create_distance_index(self.handle, a.handle, dmin, dmax, ctypes.byref(h)))
        return DeviceMatrix(self, h)

    def adjacency_from_graph(self, node_len, edges, lower=1, upper=0) -> "DeviceMatrix":
        """Range-CRS adjacency of a sequence graph built on the device
        (dvg_adjacency_from_graph; util::range_adjacency_matrix,
        adjacency.hpp:249-265).  node_len[id-1] is the length of node id
        (ids 1..N in rank order); edges is (from_id, to_id) rows; the matrix
        covers nodes [lower, upper), upper = 0 meaning through the last."""
        node_len = np.ascontiguousarray(node_len, dtype=np.uint32)
        edges = np.ascontiguousarray(edges, dtype=np.uint32).reshape(-1, 2)
        h = ctypes.c_void_p()
        N.check(N.lib().dvg_adjacency_from_graph(self.handle, len(node_len), N.ptr(node_len), len(edges),
                                                 N.ptr(edges), lower, upper, ctypes.byref(h)))
        return DeviceMatrix(self, h)

    def batch_distance_index(self, graphs, windows):
        """Indices of many independent graphs (DeviceMatrix list) with their
        (dmin, dmax) windows, built in one pass (dvg_batch_distance_index)."""
        n = len(graphs)
        if len(windows) != n:
            raise ValueError("one window per graph")
        hs = (ctypes.c_void_p * max(n, 1))(*[g.handle for g in graphs])
        lo = (ctypes.c_uint * max(n, 1))(*[int(w[0]) for w in windows])
        hi = (ctypes.c_uint * max(n, 1))(*[int(w[1]) for w in windows])
        outs = (ctypes.c_void_p * max(n, 1))()
        N.check(N.lib().dvg_batch_distance_index(self.handle, n, hs, lo, hi, outs))
        return [DeviceMatrix(self, ctypes.c_void_p(outs[k])) for k in range(n)]

    def query(self, index, pairs: np.ndarray) -> np.ndarray:
        """Host pairs (npairs x 2 uint32) -> host uint8 answers."""
        pairs = np.ascontiguousarray(pairs, dtype=np.uint32).reshape(-1, 2)
        out = np.zeros(len(pairs), dtype=np.uint8)
        N.check(N.lib().dvg_query_batch_host(self.handle, index.handle, N.ptr(pairs), len(pairs), N.ptr(out)))
        return out

    def query_device(self, index, d_pairs, npairs, d_out):
        """Device pointers in and out (e.g. torch tensors' data_ptr())."""
        N.check(N.lib().dvg_query_batch(self.handle, index.handle, ctypes.c_void_p(d_pairs), npairs,
                                        ctypes.c_void_p(d_out)))

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class DeviceMatrix:
    """A range-CRS matrix resident in device memory (dvg_matrix)."""

    def __init__(self, ctx: Context, handle):
        self.ctx = ctx
        self._h = handle
        nr, nc, ne, nz = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint64(), ctypes.c_uint64()
        N.check(N.lib().dvg_matrix_info(handle, ctypes.byref(nr), ctypes.byref(nc), ctypes.byref(ne),
                                        ctypes.byref(nz)))
        self.nrows, self.ncols, self.nentries, self.nnz = nr.value, nc.value, ne.value, nz.value

    @property
    def handle(self):
        if self._h is None:
            raise RuntimeError("matrix is freed")
        return self._h

    def device_arrays(self):
        r, e = ctypes.c_void_p(), ctypes.c_void_p()
        N.check(N.lib().dvg_matrix_device_arrays(self.handle, ctypes.byref(r), ctypes.byref(e)))
        return r.value, e.value

    def download(self, size_type=np.uint64) -> CRSMatrix:
        entries = np.empty(self.nentries, dtype=np.uint32)
        if np.dtype(size_type) == np.uint32:
            rowmap = np.empty(self.nrows + 1, dtype=np.uint32)
            N.check(N.lib().dvg_matrix_download_u32(self.ctx.handle, self.handle, N.ptr(rowmap), N.ptr(entries)))
        else:
            rowmap = np.empty(self.nrows + 1, dtype=np.uint64)
            N.check(N.lib().dvg_matrix_download(self.ctx.handle, self.handle, N.ptr(rowmap), N.ptr(entries)))
        m = CRSMatrix(self.ncols, entries, rowmap, 1, size_type=size_type)
        m.m_nnz = self.nnz
        return m

    def download_to(self, rowmap_ptr, entries_ptr):
        """Copy into caller buffers (raw host addresses, e.g. pinned memory) of
        nrows+1 uint64 and nentries uint32."""
        N.check(N.lib().dvg_matrix_download(self.ctx.handle, self.handle, ctypes.c_void_p(rowmap_ptr),
                                            ctypes.c_void_p(entries_ptr)))

    def free(self):
        if self._h is not None and self.ctx._h is not None:
            N.check(N.lib().dvg_matrix_free(self.ctx.handle, self._h))
        self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


_default = None
_default_lock = threading.Lock()


def is_runtime_initialized():
    """runtime.hpp:25."""
    return _default is not None


def initialize_runtime(device=0):
    """runtime.hpp:30: bring up the process-wide default context (if not up)."""
    global _default
    with _default_lock:
        if _default is None:
            _default = Context(device)
    return _default


def finalize_runtime():
    """runtime.hpp:35: tear the default context down (if it is up)."""
    global _default
    with _default_lock:
        if _default is not None:
            _default.close()
            _default = None


def default_context():
    return _default if _default is not None else initialize_runtime()


class ScopedRuntime:
    """runtime.hpp:42-53: initialise on entry, optionally finalise on exit."""

    def __init__(self, finalize_on_destroy=True, device=0):
        self.finalize = finalize_on_destroy
        self.device = device

    def __enter__(self):
        return initialize_runtime(self.device)

    def __exit__(self, *exc):
        if self.finalize:
            finalize_runtime()
