"""Writes tests/golden/two_volume_3d_reference.npz: the reference float
(OpenMP) build's agd_deblend on the full benchmark survey (2 x 64 x 128 x
1024, windows (16, 32, 256), 200 iterations) reduced to its SNR against the
truth and a 64-projection sketch of its output (tests/golden_io.sketch).

Needs oracle/_ref/ (make -C oracle).  The reference run takes about 12
minutes on 8 threads; pass the path of a saved output (.npy of the stacked
patches) to skip it:  python tests/golden/make_full_fixture.py [out.npy]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

from agdeblend_b200 import synthetic as S  # noqa: E402
from agdeblend_b200.capi import DeblendArgs  # noqa: E402
from golden_io import sketch  # noqa: E402

sv = S.two_volume_3d()
if len(sys.argv) > 1:
    out = list(np.load(sys.argv[1]))
else:
    import ref_bind

    args = DeblendArgs(sv.volumes, sv.n_dims, sv.window_shapes, sv.coords, sv.shapes,
                       sv.shottimes, sv.channels, sv.trace_types, sv.data, dtype=np.float32)
    assert ref_bind.ref_deblend(args, sv.initial_factor, sv.n_its, 0) == 0
    out = args.data
np.savez_compressed(os.path.join(HERE, "two_volume_3d_reference.npz"),
                    snr_db=S.snr_db(out, sv.truth, sv.trace_types), sketch=sketch(out),
                    norm=float(np.sqrt(sum(float(np.sum(np.asarray(o, np.float64) ** 2))
                                           for o in out))),
                    input_checksum=float(sum(float(np.sum(d.astype(np.float64)))
                                             for d in sv.data)),
                    n_its=sv.n_its)
print(dict(np.load(os.path.join(HERE, "two_volume_3d_reference.npz"))))
