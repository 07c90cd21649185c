"""The C++ headers include/diverg/*.hpp (the reference's API over libdvg.so),
compiled and run as a program: ETI == templated == oracle, products, the
uint32 size overload, membership, serialisation and error behaviour."""
import os
import subprocess

import pytest

from tests.conftest import ROOT

pytestmark = pytest.mark.gpu


def test_cpp_api_program():
    d = os.path.join(ROOT, "tests", "cpp")
    subprocess.run(["make", "-s", "-C", d], check=True)
    r = subprocess.run([os.path.join(d, "shim_test")], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "shim ok" in r.stdout
