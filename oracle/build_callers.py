"""Test infrastructure only: builds the reference's own callers of the C API
against this repository's libagdeblend.so, into oracle/_ref/callers/
(git-ignored; it travels to the GPU box with the other files of oracle/_ref):

  pywrap/      the reference's Python wrapper (wrappers/python/agdeblend/*.py)
               with its cffi extension modules compiled, unchanged, by its own
               build script (wrappers/python/agdeblend_build.py) with
               AGD_LIB_DIR pointing at agdeblend_b200/;
  bin/         the reference's C and C++ examples (examples/example_{1,2,4,5,7,
               8,9}.c, example_1.cpp) compiled unchanged against
               include/agdeblend.h of this repository and linked with
               agdeblend_b200/libagdeblend.so; examples/make_data.c linked with
               the same library and the FFTW3 stand-in (oracle/fftw_shim); the
               checkers examples/check_example.c and check_example_rmse.c with
               the -D values of examples/Makefile:29-55;
  examples/    the reference's Python examples, copied for the test to run.

The reference tree is read-only and absent on the GPU box, so this runs here:
  python oracle/build_callers.py [REF]     (REF defaults to AGD_REFERENCE or
                                             /root/reference)
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_ref", "callers")
LIB_DIR = os.path.join(ROOT, "agdeblend_b200")

# examples/Makefile:29-55: checker name -> (source, -D definitions)
CHECKERS = {
    "check_example_1": ("check_example.c", ['FILENAME="data_1_blended_data.bin"', "N=65536"]),
    "check_example_2": ("check_example.c", ['FILENAME="data_1_blended_data_2.bin"',
                                            "N=98304"]),
    "check_example_4": ("check_example_rmse.c", ['FILENAME="data_1_true_data.bin"',
                                                 'OUT_FILENAME="data_1_deblended_data.bin"',
                                                 "N=65536"]),
    "check_example_7": ("check_example_rmse.c", ['FILENAME="data_2_true_data.bin"',
                                                 'OUT_FILENAME="data_2_deblended_data.bin"',
                                                 "N=65536"]),
    "check_example_8_0": ("check_example_rmse.c", ['FILENAME="data_3_true_data_0.bin"',
                                                   'OUT_FILENAME="data_3_deblended_data_0.bin"',
                                                   "N=32768", "MAX_ERROR_FRAC=0.05f"]),
    "check_example_8_1": ("check_example_rmse.c", ['FILENAME="data_3_true_data_1.bin"',
                                                   'OUT_FILENAME="data_3_deblended_data_1.bin"',
                                                   "N=49152", "MAX_ERROR_FRAC=0.05f"]),
    "check_example_9_0": ("check_example_rmse.c", ['FILENAME="data_4_true_data_0.bin"',
                                                   'OUT_FILENAME="data_4_deblended_data_0.bin"',
                                                   "N=196608", "MAX_ERROR_FRAC=0.05f"]),
    "check_example_9_1": ("check_example_rmse.c", ['FILENAME="data_4_true_data_1.bin"',
                                                   'OUT_FILENAME="data_4_deblended_data_1.bin"',
                                                   "N=196608", "MAX_ERROR_FRAC=0.05f"]),
}
# examples/Makefile:60-120 (the non-MPI C and C++ examples): binary -> source
EXAMPLES = {f"example_{k}_c": f"example_{k}.c" for k in (1, 2, 4, 5, 7, 8, 9)}
EXAMPLES["example_1_cpp"] = "example_1.cpp"
PY_EXAMPLES = ["example_1.py", "example_2.py", "example_4.py", "example_5.py", "example_7.py",
               "example_8.py", "example_9.py"]


def _run(cmd, **kw):
    subprocess.run(cmd, check=True, **kw)


def build(ref: str) -> str:
    ex = os.path.join(ref, "examples")
    bindir = os.path.join(OUT, "bin")
    os.makedirs(bindir, exist_ok=True)
    inc = os.path.join(ROOT, "include")
    link = ["-L", LIB_DIR, "-lagdeblend", f"-Wl,-rpath,{LIB_DIR}"]
    for name, src in EXAMPLES.items():
        cc = "g++" if src.endswith(".cpp") else "gcc"
        _run([cc, "-O2", "-w", os.path.join(ex, src), "-I", inc, *link, "-lm", "-o",
              os.path.join(bindir, name)])
    shim = os.path.join(HERE, "fftw_shim")
    _run(["gcc", "-O2", "-w", "-DAGD_SHIM_FLOAT", os.path.join(ex, "make_data.c"),
          os.path.join(shim, "fftw_shim.c"), "-I", inc, "-I", shim, *link, "-lm", "-o",
          os.path.join(bindir, "make_data")])
    for name, (src, defs) in CHECKERS.items():
        _run(["gcc", "-O2", "-w", os.path.join(ex, src), *[f"-D{d}" for d in defs], "-lm",
              "-o", os.path.join(bindir, name)])
    # the Python wrapper and its cffi modules, built by the wrapper's own script
    pyw = os.path.join(OUT, "pywrap")
    if os.path.isdir(pyw):
        shutil.rmtree(pyw)
    shutil.copytree(os.path.join(ref, "wrappers", "python"), pyw,
                    ignore=shutil.ignore_patterns("build", "*.egg-info", "__pycache__"))
    env = dict(os.environ, AGD_LIB_DIR=LIB_DIR)
    _run([sys.executable, "agdeblend_build.py"], cwd=pyw, env=env,
         stdout=subprocess.DEVNULL)
    exdir = os.path.join(OUT, "examples")
    os.makedirs(exdir, exist_ok=True)
    for f in PY_EXAMPLES:
        shutil.copy(os.path.join(ex, f), exdir)
    return OUT


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("AGD_REFERENCE",
                                                               "/root/reference")
    print(build(ref))
