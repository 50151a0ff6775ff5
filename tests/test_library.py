"""The C-ABI libraries load without a GPU and export every function that
include/*.h declares."""
import ctypes
import os
import re

import numpy as np
import pytest

import agdeblend_b200 as A
from conftest import ROOT


def _declared():
    names = []
    for h in ("agdeblend.h", "agdeblend_gpu.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"\b(agd_\w+)\s*\(", src)
    return sorted(set(names))


def test_headers_declare_the_reference_api():
    names = _declared()
    assert "agd_deblend" in names and "agd_blend" in names


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_library_exports_every_declared_symbol(dtype):
    path = A.library_path(dtype)
    assert os.path.exists(path), "run `python -m agdeblend_b200.build`"
    lib = ctypes.CDLL(path)
    for name in _declared():
        assert hasattr(lib, name), name


def test_library_names_match_reference_wrappers():
    """The reference's Python wrapper looks for libagdeblend.so and
    libagdeblend_double.so (wrappers/python/agdeblend_libs.py:21-26)."""
    assert os.path.basename(A.library_path(np.float32)) == "libagdeblend.so"
    assert os.path.basename(A.library_path(np.float64)) == "libagdeblend_double.so"
