"""ctypes bindings of libdvg.so (include/dvg.h) and libdvg_gen.so (include/dvg_gen.h).

The CUDA library is the only compute path: when it is missing or no sm_100
device is present, every call raises; there is no CPU fallback.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdvg.so")
GEN_PATH = os.path.join(_HERE, "libdvg_gen.so")

# dvg_status
OK, INVALID_ARG, OOM, DEVICE, TIMEOUT, NOT_INITIALIZED, OVERFLOW = range(7)


class DvgError(RuntimeError):
    """A non-OK dvg_status; `status` holds the code."""

    def __init__(self, status, msg):
        super().__init__(msg)
        self.status = status


class DvgStats(ctypes.Structure):
    _fields_ = [(name, ctypes.c_uint64) for name in (
        "kernel_launches", "spgemm_calls", "spadd_calls", "host_syncs", "alg_bytes",
        "spgemm_alg_bytes", "range_ops", "h2d_bytes", "d2h_bytes", "spgemm_ns", "spgemm_levels_ns",
        "scan_ns", "spadd_ns", "spgemm_direct_tiles", "spgemm_reruns", "spgemm_light", "spgemm_slow_rows", "host_alloc_ns",
        "host_sync_ns", "spgemm_fused_adds", "graph_launches", "autotune_builds", "spgemm_levels",
        "host_prepare_ns", "host_launch_ns", "host_meminfo_ns", "query_ns", "query_pairs")]

    def as_dict(self):
        return {name: int(getattr(self, name)) for name, _ in self._fields_}


class HostMatrix(ctypes.Structure):
    _fields_ = [("nrows", ctypes.c_uint32), ("ncols", ctypes.c_uint32), ("nentries", ctypes.c_uint64),
                ("nnz", ctypes.c_uint64), ("rowmap", ctypes.POINTER(ctypes.c_uint64)),
                ("entries", ctypes.POINTER(ctypes.c_uint32))]


class GraphParams(ctypes.Structure):
    _fields_ = [("n_backbone", ctypes.c_uint64), ("snp_rate", ctypes.c_double), ("indel_rate", ctypes.c_double),
                ("ins_frac", ctypes.c_double), ("indel_lmin", ctypes.c_uint32), ("indel_lmax", ctypes.c_uint32),
                ("indel_geometric_mean", ctypes.c_double), ("sv_frac", ctypes.c_double),
                ("sv_lmin", ctypes.c_uint32), ("sv_lmax", ctypes.c_uint32), ("seed", ctypes.c_uint64)]


class GraphStats(ctypes.Structure):
    _fields_ = [(name, ctypes.c_uint64) for name in (
        "n_loci", "n_snp", "n_ins", "n_del", "n_sv", "n_alt_loci")]


class ServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("hbm_budget_bytes", ctypes.c_uint64),
                ("max_batch_builds", ctypes.c_uint32), ("max_inflight_queries", ctypes.c_uint32),
                ("build_workers", ctypes.c_uint32)]


class Completion(ctypes.Structure):
    _fields_ = [("request", ctypes.c_uint64), ("status", ctypes.c_int32), ("kind", ctypes.c_uint32),
                ("submit_ns", ctypes.c_uint64), ("start_ns", ctypes.c_uint64), ("done_ns", ctypes.c_uint64),
                ("index_entries", ctypes.c_uint64), ("index_nnz", ctypes.c_uint64),
                ("invalid_pairs", ctypes.c_uint64)]


class ServerStats(ctypes.Structure):
    _fields_ = [(name, ctypes.c_uint64) for name in (
        "builds_submitted", "builds_done", "build_batches", "queries_submitted", "queries_done", "pairs_answered",
        "resident_bytes", "peak_reserved_bytes", "hbm_budget_bytes", "build_reruns", "build_batch_ns_max",
        "build_alloc_ns", "build_sync_ns", "builds_failed", "builds_rebuilt_alone")]

    def as_dict(self):
        return {name: int(getattr(self, name)) for name, _ in self._fields_}


# Every entry point of include/dvg.h with its argument types.
_P, _U32, _U64, _I64 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int64
_PP = ctypes.POINTER(ctypes.c_void_p)
DVG_SIGNATURES = {
    "dvg_init": [ctypes.c_int, _PP],
    "dvg_shutdown": [_P],
    "dvg_set_stream": [_P, _P],
    "dvg_synchronize": [_P],
    "dvg_set_option": [_P, ctypes.c_char_p, _I64],
    "dvg_trim": [_P],
    "dvg_get_stats": [_P, ctypes.POINTER(DvgStats)],
    "dvg_stats_reset": [_P],
    "dvg_last_error": [],
    "dvg_status_string": [ctypes.c_int],
    "dvg_matrix_upload": [_P, _U32, _U32, _P, _P, _U64, _PP],
    "dvg_matrix_upload_u32": [_P, _U32, _U32, _P, _P, _U64, _PP],
    "dvg_matrix_wrap_device": [_P, _U32, _U32, _P, _P, _U64, _U64, _PP],
    "dvg_matrix_info": [_P, ctypes.POINTER(_U32), ctypes.POINTER(_U32), ctypes.POINTER(_U64), ctypes.POINTER(_U64)],
    "dvg_matrix_device_arrays": [_P, _PP, _PP],
    "dvg_matrix_download": [_P, _P, _P, _P],
    "dvg_matrix_download_u32": [_P, _P, _P, _P],
    "dvg_matrix_free": [_P, _P],
    "dvg_range_identity": [_P, _U32, _PP],
    "dvg_range_spadd": [_P, _P, _P, _PP],
    "dvg_range_spgemm": [_P, _P, _P, _PP],
    "dvg_range_power": [_P, _P, ctypes.c_uint, _PP],
    "dvg_create_distance_index": [_P, _P, ctypes.c_uint, ctypes.c_uint, _PP],
    "dvg_batch_distance_index": [_P, _U32, _P, _P, _P, _P],
    "dvg_adjacency_from_graph": [_P, _U32, _P, ctypes.c_uint64, _P, _U32, _U32, _PP],
    "dvg_selftest_bounded_wait": [_P, _U32],
    "dvg_calibrate_range_ops": [_P, ctypes.POINTER(ctypes.c_double)],
    "dvg_calibrate_random_reads": [_P, ctypes.c_uint64, ctypes.POINTER(ctypes.c_double)],
    "dvg_query_batch": [_P, _P, _P, _U64, _P],
    "dvg_query_batch_host": [_P, _P, _P, _U64, _P],
    "dvg_range_spgemm_noalloc": [_U32, _U32, _P, _P, _U64, _U32, _U32, _P, _P, _U64, _P, _P, _U64,
                                 ctypes.POINTER(_U64), ctypes.POINTER(_U64), _P],
    "dvg_server_create": [ctypes.POINTER(ServerConfig), _PP],
    "dvg_server_destroy": [_P],
    "dvg_server_submit_build": [_P, _U32, _P, _P, ctypes.c_uint, ctypes.c_uint, ctypes.POINTER(_U64)],
    "dvg_server_submit_query": [_P, _U64, _P, _U64, _P, ctypes.POINTER(_U64)],
    "dvg_server_poll": [_P, ctypes.POINTER(Completion), _U32, ctypes.POINTER(_U32), _U32],
    "dvg_server_index_info": [_P, _U64, ctypes.POINTER(_U32), ctypes.POINTER(_U64), ctypes.POINTER(_U64)],
    "dvg_server_download": [_P, _U64, _P, _P],
    "dvg_server_release": [_P, _U64],
    "dvg_server_get_stats": [_P, ctypes.POINTER(ServerStats)],
}

GEN_SIGNATURES = {
    "dvg_gen_graph_adjacency": [ctypes.POINTER(GraphParams), ctypes.POINTER(HostMatrix), ctypes.POINTER(GraphStats)],
    "dvg_gen_graph_edges": [ctypes.POINTER(GraphParams), ctypes.POINTER(_U64), ctypes.POINTER(_U64),
                            ctypes.POINTER(ctypes.POINTER(ctypes.c_uint32))],
    "dvg_gen_graph_nodes": [ctypes.POINTER(GraphParams), ctypes.POINTER(_U64),
                            ctypes.POINTER(ctypes.POINTER(ctypes.c_uint32)), ctypes.POINTER(_U64),
                            ctypes.POINTER(ctypes.POINTER(ctypes.c_uint32))],
    "dvg_gen_banded": [_U32, _U32, ctypes.c_double, ctypes.c_double, _U64, ctypes.POINTER(HostMatrix)],
    "dvg_gen_random": [_U32, _U64, _U64, ctypes.POINTER(HostMatrix)],
    "dvg_gen_pairs": [ctypes.POINTER(HostMatrix), _U64, ctypes.c_double, _U32, _U32, _U64, _P],
    "dvg_gen_free": [ctypes.POINTER(HostMatrix)],
    "dvg_gen_free_ptr": [_P],
}

_lib = None
_gen = None


def lib():
    """The CUDA library; raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with __graft_entry__.build() "
                               "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in DVG_SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int
        L.dvg_last_error.restype = ctypes.c_char_p
        L.dvg_status_string.restype = ctypes.c_char_p
        _lib = L
    return _lib


def gen_lib():
    global _gen
    if _gen is None:
        if not os.path.exists(GEN_PATH):
            raise RuntimeError(f"{GEN_PATH} is missing: build it with __graft_entry__.build()")
        L = ctypes.CDLL(GEN_PATH)
        for name, args in GEN_SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = None if name.startswith("dvg_gen_free") else ctypes.c_int
        _gen = L
    return _gen


def check(status):
    if status != OK:
        L = lib()
        msg = L.dvg_last_error().decode(errors="replace")
        raise DvgError(status, f"{L.dvg_status_string(status).decode()}: {msg}")


def ptr(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data) if a is not None and a.size else ctypes.c_void_p(0)
