"""The reference's own callers against this library (built by
oracle/build_callers.py from the reference's unchanged sources): its C and
C++ examples compiled against include/agdeblend.h and linked with
agdeblend_b200/libagdeblend.so, and its Python examples through its own
cffi wrapper built with AGD_LIB_DIR=agdeblend_b200.  make_data (the
reference's seeded data generator, examples/make_data.c, calling agd_blend)
writes the data; each example is then checked by the reference's own
checker with the thresholds of examples/Makefile:29-55: exact blending
(check_example.c), RMS error fraction <= 1/50 for examples 4, 5 and 7 and
<= 0.05 for examples 8 and 9 (check_example_rmse.c)."""
import os
import shutil
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

CALLERS = os.path.join(ROOT, "oracle", "_ref", "callers")
BIN = os.path.join(CALLERS, "bin")
LIB_DIR = os.path.join(ROOT, "agdeblend_b200")

if not os.path.isdir(BIN):
    pytest.skip("oracle/_ref/callers not built (python oracle/build_callers.py)",
                allow_module_level=True)

CHECKS = {
    "example_1": ["check_example_1"], "example_2": ["check_example_2"],
    "example_4": ["check_example_4"], "example_5": ["check_example_4"],
    "example_7": ["check_example_7"], "example_8": ["check_example_8_0", "check_example_8_1"],
    "example_9": ["check_example_9_0", "check_example_9_1"],
}


@pytest.fixture(scope="module")
def data_dir(tmp_path_factory):
    d = tmp_path_factory.mktemp("agd_examples")
    subprocess.run([os.path.join(BIN, "make_data")], cwd=d, check=True, timeout=600,
                   stdout=subprocess.DEVNULL)
    return d


def _fresh_out(d):
    out = os.path.join(d, "out")
    if os.path.isdir(out):
        shutil.rmtree(out)
    os.makedirs(out)


def _check(d, example):
    for c in CHECKS[example]:
        res = subprocess.run([os.path.join(BIN, c)], cwd=d, capture_output=True, text=True,
                             timeout=120)
        assert res.returncode == 0, f"{c}: {res.stdout} {res.stderr}"


@pytest.mark.parametrize("exe", ["example_1_c", "example_2_c", "example_1_cpp", "example_4_c",
                                 "example_5_c", "example_7_c", "example_8_c", "example_9_c"])
def test_reference_c_example(data_dir, exe):
    _fresh_out(data_dir)
    res = subprocess.run([os.path.join(BIN, exe)], cwd=data_dir, capture_output=True, text=True,
                         timeout=900)
    assert res.returncode == 0, res.stderr
    _check(data_dir, exe.rsplit("_", 1)[0])


@pytest.mark.parametrize("script", ["example_1.py", "example_2.py", "example_4.py",
                                    "example_5.py", "example_7.py", "example_8.py",
                                    "example_9.py"])
def test_reference_python_example(data_dir, script):
    _fresh_out(data_dir)
    env = dict(os.environ, PYTHONPATH=os.path.join(CALLERS, "pywrap"),
               LD_LIBRARY_PATH=LIB_DIR + os.pathsep + os.environ.get("LD_LIBRARY_PATH", ""))
    res = subprocess.run([sys.executable, os.path.join(CALLERS, "examples", script)],
                         cwd=data_dir, env=env, capture_output=True, text=True, timeout=900)
    assert res.returncode == 0, res.stderr[-2000:]
    _check(data_dir, script[:-3])
