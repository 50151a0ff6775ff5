"""Python layer over the warm-start network of libagdeblend.so (agd_nn_*,
include/agdeblend_gpu.h): a 4-level convolutional encoder-decoder whose
convolutions run as BF16 tensor-core GEMMs, used to start the deblending
solver from an estimate of the deblended data instead of zero."""
from __future__ import annotations

import ctypes
from ctypes import POINTER, c_double, c_float, c_int, c_long, c_uint, c_void_p

import numpy as np

from . import load_library


def _bind(lib):
    if getattr(lib, "_agd_nn_bound", False):
        return lib
    fp, dp = POINTER(c_float), POINTER(c_double)
    lib.agd_nn_create.argtypes = [c_int, c_uint, POINTER(c_void_p)]
    lib.agd_nn_create_channels.argtypes = [c_int, c_int, c_uint, POINTER(c_void_p)]
    lib.agd_nn_create_channels.restype = c_int
    lib.agd_nn_input_channels.argtypes = [c_void_p]
    lib.agd_nn_input_channels.restype = c_int
    lib.agd_nn_destroy.argtypes = [c_void_p]
    lib.agd_nn_destroy.restype = None
    lib.agd_nn_param_count.argtypes = [c_void_p]
    lib.agd_nn_param_count.restype = c_long
    lib.agd_nn_get_params.argtypes = [c_void_p, fp]
    lib.agd_nn_set_params.argtypes = [c_void_p, fp]
    lib.agd_nn_forward.argtypes = [c_void_p, fp, c_int, c_int, c_int, fp]
    lib.agd_nn_loss_grad.argtypes = [c_void_p, fp, fp, c_int, c_int, c_int, dp, fp]
    lib.agd_nn_train.argtypes = [c_void_p, fp, fp, c_long, c_int, c_int, c_int, c_int, c_float,
                                 c_uint, dp]
    for name in ("agd_nn_create", "agd_nn_get_params", "agd_nn_set_params", "agd_nn_forward",
                 "agd_nn_loss_grad", "agd_nn_train"):
        getattr(lib, name).restype = c_int
    lib._agd_nn_bound = True
    return lib


def _fp(a):
    return a.ctypes.data_as(POINTER(c_float))


class WarmStartNet:
    """The network on the current GPU (float library).  Inputs are
    [n][h][w] images, or [n][h][w][in_channels] with more than one input
    channel (channel 0 the image itself, the others its neighbouring lines);
    outputs and targets [n][h][w]."""

    def __init__(self, base_channels: int = 32, seed: int = 0, in_channels: int = 1):
        self.lib = _bind(load_library(np.float32))
        h = c_void_p()
        if self.lib.agd_nn_create_channels(base_channels, in_channels, seed, ctypes.byref(h)):
            raise RuntimeError("agd_nn_create_channels failed")
        self.h = h
        self.base = base_channels
        self.in_channels = in_channels
        self.n_params = int(self.lib.agd_nn_param_count(h))

    def _input(self, x):
        """(contiguous input, n, h, w) after checking the channel count."""
        x = np.ascontiguousarray(x, np.float32)
        if x.ndim == 3 and self.in_channels == 1:
            return x, *x.shape
        if x.ndim != 4 or x.shape[3] != self.in_channels:
            raise ValueError(f"inputs must be [n][h][w][{self.in_channels}]")
        return x, *x.shape[:3]

    def close(self):
        if getattr(self, "h", None):
            self.lib.agd_nn_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def params(self) -> np.ndarray:
        out = np.zeros(self.n_params, np.float32)
        if self.lib.agd_nn_get_params(self.h, _fp(out)):
            raise RuntimeError("agd_nn_get_params failed")
        return out

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, np.float32)
        if p.size != self.n_params or self.lib.agd_nn_set_params(self.h, _fp(p)):
            raise RuntimeError("agd_nn_set_params failed")

    def forward(self, x) -> np.ndarray:
        x, n, h, w = self._input(x)
        out = np.zeros((n, h, w), np.float32)
        if self.lib.agd_nn_forward(self.h, _fp(x), n, h, w, _fp(out)):
            raise RuntimeError("agd_nn_forward failed")
        return out

    def loss_grad(self, x, target):
        x, n, h, w = self._input(x)
        t = np.ascontiguousarray(target, np.float32)
        if t.shape != (n, h, w):
            raise ValueError("targets must be [n][h][w]")
        loss = c_double(0)
        g = np.zeros(self.n_params, np.float32)
        if self.lib.agd_nn_loss_grad(self.h, _fp(x), _fp(t), n, h, w, ctypes.byref(loss),
                                     _fp(g)):
            raise RuntimeError("agd_nn_loss_grad failed")
        return float(loss.value), g

    def train(self, inputs, targets, batch: int = 32, epochs: int = 1, lr: float = 1e-3,
              seed: int = 0) -> np.ndarray:
        x, n, h, w = self._input(inputs)
        t = np.ascontiguousarray(targets, np.float32)
        if t.shape != (n, h, w):
            raise ValueError("targets must be [n][h][w]")
        losses = np.zeros(epochs)
        if self.lib.agd_nn_train(self.h, _fp(x), _fp(t), n, h, w, batch, epochs, lr, seed,
                                 losses.ctypes.data_as(POINTER(c_double))):
            raise RuntimeError("agd_nn_train failed")
        return losses
