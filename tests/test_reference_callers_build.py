"""The reference's own callers build unchanged against this repository's
header and library (oracle/build_callers.py): every example, make_data and
checker binary exists and binds agd_deblend / agd_blend from libagdeblend.so,
and the reference's cffi wrapper module imports with the library on the
loader path.  Rebuilt here when the reference tree is present."""
import os
import subprocess
import sys

import pytest

from conftest import ROOT

CALLERS = os.path.join(ROOT, "oracle", "_ref", "callers")
REF = os.environ.get("AGD_REFERENCE", "/root/reference")


@pytest.fixture(scope="module")
def callers():
    if os.path.isdir(os.path.join(REF, "examples")):
        subprocess.run([sys.executable, os.path.join(ROOT, "oracle", "build_callers.py"), REF],
                       check=True, stdout=subprocess.DEVNULL)
    if not os.path.isdir(os.path.join(CALLERS, "bin")):
        pytest.skip("neither the reference tree nor a prebuilt oracle/_ref/callers")
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import build_callers

    return build_callers


def test_examples_link_the_library(callers):
    for name in list(callers.EXAMPLES) + ["make_data"]:
        path = os.path.join(CALLERS, "bin", name)
        assert os.access(path, os.X_OK), name
        syms = subprocess.run(["nm", "-D", "--undefined-only", path], capture_output=True,
                              text=True, check=True).stdout
        assert "agd_deblend" in syms or "agd_blend" in syms, name
        deps = subprocess.run(["ldd", path], capture_output=True, text=True).stdout
        assert os.path.join(ROOT, "agdeblend_b200", "libagdeblend.so") in deps, name
    for name in callers.CHECKERS:
        assert os.access(os.path.join(CALLERS, "bin", name), os.X_OK), name


def test_reference_cffi_wrapper_imports(callers):
    code = ("import agdeblend, agdeblend._agdeblend_ffi as m, agdeblend._agdeblend_double_ffi "
            "as d; assert hasattr(m.lib, 'agd_deblend') and hasattr(d.lib, 'agd_blend')")
    env = dict(os.environ, PYTHONPATH=os.path.join(CALLERS, "pywrap"),
               LD_LIBRARY_PATH=os.path.join(ROOT, "agdeblend_b200"))
    subprocess.run([sys.executable, "-c", code], env=env, check=True)
