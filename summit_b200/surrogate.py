"""Surrogate network of the learned control variate, on liblds's own kernels.

``Surrogate`` holds the FP32 master parameters in a torch CUDA tensor (torch
only provides device memory here) and calls lds_mlp_forward / lds_mlp_loss_grad
/ lds_mlp_train (include/lds.h): in -> 128 -> 128 -> 128 -> out, GELU, BF16
weights and activations in the products, FP32 accumulation, Adam.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from ._lib import check

HIDDEN = 128


def _dp(t) -> C.c_void_p:
    return C.c_void_p(int(t.data_ptr()))


def param_count(n_in: int, n_out: int) -> int:
    return int(_lib.load().lds_mlp_param_count(int(n_in), int(n_out)))


def init_params(n_in: int, n_out: int, seed: int) -> np.ndarray:
    """He-normal weights (fan-in), zero biases, in the library's flat layout."""
    rng = np.random.default_rng(seed)
    p = np.zeros(param_count(n_in, n_out), dtype=np.float32)
    off = 0
    for rows, cols in [(HIDDEN, n_in), (HIDDEN, HIDDEN), (HIDDEN, HIDDEN), (n_out, HIDDEN)]:
        p[off:off + rows * cols] = rng.normal(0.0, math.sqrt(2.0 / cols), rows * cols)
        off += rows * cols + rows
    return p


class Surrogate:
    def __init__(self, n_in: int, n_out: int, seed: int = 0, params=None, device="cuda"):
        import torch

        self.n_in, self.n_out = int(n_in), int(n_out)
        p = init_params(n_in, n_out, seed) if params is None else np.asarray(params, np.float32)
        self.params = torch.from_numpy(p.copy()).to(device)

    def forward(self, x):
        import torch

        x = x.contiguous().float()
        out = torch.empty((x.shape[0], self.n_out), dtype=torch.float32, device=x.device)
        torch.cuda.synchronize()
        check(_lib.load().lds_mlp_forward(_dp(self.params), self.n_in, self.n_out, _dp(x),
                                          x.shape[0], _dp(out)))
        return out

    def loss_grad(self, x, t):
        import torch

        x, t = x.contiguous().float(), t.contiguous().float()
        g = torch.empty_like(self.params)
        loss = C.c_double(0.0)
        torch.cuda.synchronize()
        check(_lib.load().lds_mlp_loss_grad(_dp(self.params), self.n_in, self.n_out, _dp(x),
                                            _dp(t), x.shape[0], _dp(g), C.byref(loss)))
        return loss.value, g

    def train(self, x, t, epochs: int, batch: int = 4096, lr: float = 3e-3, seed: int = 0):
        import torch

        x, t = x.contiguous().float(), t.contiguous().float()
        losses = np.zeros(max(epochs, 1))
        torch.cuda.synchronize()
        check(_lib.load().lds_mlp_train(_dp(self.params), self.n_in, self.n_out, _dp(x), _dp(t),
                                        x.shape[0], int(epochs), int(batch), C.c_float(lr),
                                        int(seed), losses.ctypes.data_as(C.c_void_p)))
        return losses[:epochs]
