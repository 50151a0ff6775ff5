"""Writes tests/golden/<workload>_reference.npz: the reference float (OpenMP)
build's agd_deblend on a benchmark-shaped survey, reduced to its SNR against
the truth, a 64-projection sketch of its output (tests/golden_io.sketch), its
L2 norm, a checksum of the input and the iteration count.

Workloads (agdeblend_b200.synthetic, seeds as in bench.py):
  two_volume_3d       2 x (64 ch x 128 shots x 1024), windows (16, 32, 256),
                      the full 200 iterations (about 12 minutes on 8 threads);
  vibroseis_4d        32 sY x 64 sX x 32 ch x 2048 with the 256-sample sweep,
                      windows (16, 16, 16, 256); its 150 iterations take the
                      reference more than two hours here, so the fixture runs
                      agd_deblend with n_its = 5 (the initial step, four
                      iterations of the n_its = 5 schedule and the output);
  vibroseis_4d_small  16 sY x 32 sX x 32 ch x 2048, the full 150 iterations
                      (about 40 minutes on 8 threads).

Needs oracle/_ref/ (make -C oracle).
  python tests/golden/make_full_fixture.py <workload> [saved_output.npy]
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

from agdeblend_b200 import synthetic as S  # noqa: E402
from agdeblend_b200.capi import DeblendArgs  # noqa: E402
from golden_io import sketch  # noqa: E402

# workload -> (survey factory, iterations run by the reference)
WORKLOADS = {
    "two_volume_3d": (lambda: S.two_volume_3d(), 200),
    "vibroseis_4d": (lambda: S.vibroseis_4d(seed=1002), 5),
    "vibroseis_4d_small": (lambda: S.vibroseis_4d(seed=1002, n_sy=16, n_sx=32), 150),
}


def fixture_path(name: str) -> str:
    return os.path.join(HERE, f"{name}_reference.npz")


def main():
    name = sys.argv[1] if len(sys.argv) > 1 else "two_volume_3d"
    make, n_its = WORKLOADS[name]
    sv = make()
    t0 = time.perf_counter()
    if len(sys.argv) > 2:
        out = list(np.load(sys.argv[2]))
    else:
        import ref_bind

        args = DeblendArgs(sv.volumes, sv.n_dims, sv.window_shapes, sv.coords, sv.shapes,
                           sv.shottimes, sv.channels, sv.trace_types, sv.data,
                           sv.wavelet_lengths, sv.wavelet_idxs, sv.wavelets, dtype=np.float32)
        assert ref_bind.ref_deblend(args, sv.initial_factor, n_its, 0) == 0
        out = args.data
    np.savez_compressed(fixture_path(name),
                        snr_db=S.snr_db(out, sv.truth, sv.trace_types), sketch=sketch(out),
                        norm=float(np.sqrt(sum(float(np.sum(np.asarray(o, np.float64) ** 2))
                                               for o in out))),
                        input_checksum=float(sum(float(np.sum(d.astype(np.float64)))
                                                 for d in sv.data)),
                        n_its=n_its, reference_seconds=time.perf_counter() - t0)
    print(name, dict(np.load(fixture_path(name))))


if __name__ == "__main__":
    main()
