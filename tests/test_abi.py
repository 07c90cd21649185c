"""The C ABI libraries load and export every symbol their headers declare
(no device work: this runs without a GPU)."""
import ctypes
import os
import re

import pytest

from diverg_b200 import _native as N
from tests.conftest import ROOT


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dvg_[a-z0-9_]+)\s*\(", text)))


@pytest.mark.parametrize("header,path", [("dvg.h", N.LIB_PATH), ("dvg_gen.h", N.GEN_PATH)])
def test_library_exports_every_declared_symbol(header, path):
    lib = ctypes.CDLL(path)
    names = declared(header)
    assert len(names) >= 7
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_bindings_cover_the_header():
    assert sorted(N.DVG_SIGNATURES) == declared("dvg.h")
    assert sorted(N.GEN_SIGNATURES) == declared("dvg_gen.h")


def test_status_strings():
    L = N.lib()
    assert L.dvg_status_string(N.OK) == b"ok"
    assert L.dvg_status_string(N.INVALID_ARG) == b"invalid argument"


def test_init_fails_loudly_without_a_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    st = N.lib().dvg_init(0, ctypes.byref(h))
    assert st == N.DEVICE and not h.value
    assert N.lib().dvg_last_error()


def header_struct_fields(header, name):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    body = re.search(r"typedef struct " + name + r"\s*\{(.*?)\}\s*" + name + ";", text, flags=re.S).group(1)
    return [m.group(1) for m in re.finditer(r"\b(\w+)\s*;", body)]


@pytest.mark.parametrize("header,name,cls", [
    ("dvg.h", "dvg_stats", N.DvgStats), ("dvg.h", "dvg_server_config", N.ServerConfig),
    ("dvg.h", "dvg_completion", N.Completion), ("dvg.h", "dvg_server_stats", N.ServerStats),
    ("dvg_gen.h", "dvg_graph_params", N.GraphParams), ("dvg_gen.h", "dvg_graph_stats", N.GraphStats),
    ("dvg_gen.h", "dvg_host_matrix", N.HostMatrix)])
def test_ctypes_structs_follow_the_header(header, name, cls):
    # the Python mirror of each C struct has the header's fields, in order
    assert [f for f, _ in cls._fields_] == header_struct_fields(header, name)
