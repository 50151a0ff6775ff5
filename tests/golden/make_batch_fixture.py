"""Writes tests/golden/uneven_gathers_reference.npz: the reference float
(OpenMP) build's agd_deblend run separately on each of the 96 uneven 2-D
gathers of the batch workload (agdeblend_b200.synthetic.uneven_gathers,
base seed 3000, 100 iterations each), reduced per gather to its SNR against
the truth, a 32-projection sketch of its output (tests/golden_io.sketch), its
L2 norm and a checksum of its input.

Needs oracle/_ref/ (make -C oracle); about 10 minutes on 8 threads.
  python tests/golden/make_batch_fixture.py [n_gathers]
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import ref_bind  # noqa: E402
from agdeblend_b200 import synthetic as S  # noqa: E402
from agdeblend_b200.capi import DeblendArgs  # noqa: E402
from golden_io import sketch  # noqa: E402

K_SKETCH = 32


def main():
    n = int(sys.argv[1]) if len(sys.argv) > 1 else 96
    gathers = S.uneven_gathers(n, base_seed=3000)
    snr, sk, norm, checksum = [], [], [], []
    t0 = time.perf_counter()
    for g in gathers:
        args = DeblendArgs(g.volumes, g.n_dims, g.window_shapes, g.coords, g.shapes,
                           g.shottimes, g.channels, g.trace_types, g.data, dtype=np.float32)
        assert ref_bind.ref_deblend(args, g.initial_factor, g.n_its, 0) == 0
        out = args.data
        snr.append(S.snr_db(out, g.truth, g.trace_types))
        sk.append(sketch(out, k=K_SKETCH))
        norm.append(float(np.sqrt(sum(float(np.sum(np.asarray(o, np.float64) ** 2))
                                      for o in out))))
        checksum.append(float(sum(float(np.sum(d.astype(np.float64))) for d in g.data)))
    path = os.path.join(HERE, "uneven_gathers_reference.npz")
    np.savez_compressed(path, snr_db=np.array(snr), sketch=np.array(sk), norm=np.array(norm),
                        input_checksum=np.array(checksum), n_its=gathers[0].n_its,
                        base_seed=3000, reference_seconds=time.perf_counter() - t0)
    z = np.load(path)
    print({k: z[k] if z[k].size < 4 else z[k][:4] for k in z.files})


if __name__ == "__main__":
    main()
