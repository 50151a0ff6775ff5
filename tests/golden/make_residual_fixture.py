"""Writes tests/golden/residual_lines_reference.npz: the `Iteration <it>
Residual <value>` lines that the reference float build's agd_deblend prints
with print_freq > 0 (src/agdeblend.c:592-596,611-616), on three surveys:

  gather_2d      one channel, 96 shots x 384 samples, window (32, 256),
                 n_its 40, print_freq 5;
  two_volume_3d  2 x (8 ch x 24 shots x 300), window (4, 8, 128), bad and
                 missing traces, record gaps, n_its 30, print_freq 3;
  vibroseis_4d   4 sY x 8 sX x 8 ch x 300 with a 40-sample sweep, window
                 (4, 4, 4, 64), n_its 20, print_freq 4.

The reference prints with C stdio, so each run happens in a child process
whose standard output this script reads.  Needs oracle/_ref/.
  python tests/golden/make_residual_fixture.py
"""
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from residual_cases import CASES, make_case  # noqa: E402


def child(name):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_bind
    from agdeblend_b200.capi import DeblendArgs

    sv, print_freq = make_case(name)
    args = DeblendArgs(sv.volumes, sv.n_dims, sv.window_shapes, sv.coords, sv.shapes,
                       sv.shottimes, sv.channels, sv.trace_types, sv.data,
                       sv.wavelet_lengths, sv.wavelet_idxs, sv.wavelets, dtype=np.float32)
    rc = ref_bind.ref_deblend(args, sv.initial_factor, sv.n_its, print_freq)
    sys.stdout.flush()
    sys.exit(rc)


def parse(text):
    its, vals = [], []
    for ln in text.splitlines():
        parts = ln.split()
        if len(parts) == 4 and parts[0] == "Iteration" and parts[2] == "Residual":
            its.append(int(parts[1]))
            vals.append(float(parts[3]))
    return np.array(its), np.array(vals)


def main():
    if len(sys.argv) > 2 and sys.argv[1] == "--child":
        child(sys.argv[2])
        return
    out = {}
    for name in CASES:
        res = subprocess.run([sys.executable, os.path.abspath(__file__), "--child", name],
                             capture_output=True, text=True, check=True)
        its, vals = parse(res.stdout)
        assert its.size > 2, res.stdout
        out[f"{name}_its"] = its
        out[f"{name}_residual"] = vals
    path = os.path.join(HERE, "residual_lines_reference.npz")
    np.savez_compressed(path, **out)
    print({k: v for k, v in np.load(path).items()})


if __name__ == "__main__":
    main()
