"""Writes the golden fixtures of tests/golden/ from the reference itself.

Run in a container where the reference tree exists and oracle/_ref/ was built
(`make -C oracle`):  python tests/golden/make_golden.py

  ops_<name>.npz        problem inputs and the reference's own operator
                        outputs in double precision (oracle/ref_ops.c over the
                        reference's model_forward, model_adjoint_update,
                        blend_input, set_output, get_stepsize)
  gather_2d_deblend.npz the reference float build's agd_deblend output for
                        the 128-shot x 512-sample gather, window (32, 256),
                        100 iterations, with its SNR against the truth
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
from problems import random_problem  # noqa: E402
import ref_bind  # noqa: E402


def _pack(prefix, arrays):
    return {f"{prefix}_{i}": np.asarray(a) for i, a in enumerate(arrays)}


def ops_fixture(name, sv, seed=0):
    args = DeblendArgs(sv.volumes, sv.n_dims, sv.window_shapes, sv.coords, sv.shapes,
                       sv.shottimes, sv.channels, sv.trace_types, sv.data, sv.wavelet_lengths,
                       sv.wavelet_idxs, sv.wavelets, dtype=np.float64)
    ref = ref_bind.RefOps(args)
    rng = np.random.default_rng(seed)
    rec = rng.standard_normal(ref.record_size)
    model = ref.adjoint(rec)
    out = dict(
        volumes=np.asarray(sv.volumes), n_dims=np.asarray(sv.n_dims),
        n_patches=len(sv.volumes), n_volumes=len(sv.window_shapes),
        record_in=rec, model_adjoint=model, record_forward=ref.forward(model),
        blend_input=ref.blend_input(sv.data), stepsize=ref.stepsize,
        has_wavelets=sv.wavelets is not None)
    out.update(_pack("window_shape", sv.window_shapes))
    out.update(_pack("coords", sv.coords))
    out.update(_pack("shape", sv.shapes))
    out.update(_pack("shottimes", sv.shottimes))
    out.update(_pack("channels", sv.channels))
    out.update(_pack("trace_types", sv.trace_types))
    out.update(_pack("data", sv.data))
    out.update(_pack("output", ref.set_output(model, [tuple(s) for s in sv.shapes])))
    if sv.wavelets is not None:
        out["wavelet_lengths"] = np.asarray(sv.wavelet_lengths)
        out.update(_pack("wavelet_idxs", sv.wavelet_idxs))
        out.update(_pack("wavelet", sv.wavelets))
    np.savez_compressed(os.path.join(HERE, f"ops_{name}.npz"), **out)


def deblend_fixture():
    sv = S.gather_2d()
    args = DeblendArgs(sv.volumes, sv.n_dims, sv.window_shapes, sv.coords, sv.shapes,
                       sv.shottimes, sv.channels, sv.trace_types, sv.data, dtype=np.float32)
    rc = ref_bind.ref_deblend(args, sv.initial_factor, sv.n_its, 0,
                              lib_name="libagdeblend_ref_serial.so")
    assert rc == 0
    out = args.data[0]
    np.savez_compressed(os.path.join(HERE, "gather_2d_deblend.npz"), reference_out=out,
                        reference_snr_db=S.snr_db([out], sv.truth, sv.trace_types),
                        input_checksum=float(np.sum(sv.data[0].astype(np.float64))),
                        n_its=sv.n_its)


if __name__ == "__main__":
    ops_fixture("gather_2d", S.gather_2d(seed=21, n_shots=32, nt=160, window=(16, 64)))
    ops_fixture("two_volume_3d", S.two_volume_3d(seed=22, n_ch=8, n_shots=8, nt=64,
                                                 window=(4, 8, 16)))
    ops_fixture("wavelet_4d", S.vibroseis_4d(seed=23, n_sy=4, n_sx=4, n_ch=4, nt=96,
                                             window=(4, 4, 4, 16), wavelet_len=12))
    ops_fixture("random_neighbours", random_problem(905, neighbours=True, max_dims=3))
    deblend_fixture()
    for f in sorted(os.listdir(HERE)):
        print(f, os.path.getsize(os.path.join(HERE, f)))
