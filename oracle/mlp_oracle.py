"""ORACLE — CPU FP64 restatement of the control variate's surrogate network
(test infrastructure; only tests/ and bench.py's baseline legs may use it).

Same function as liblds's network (lds_mlp.cu): in -> 128 -> 128 -> 128 -> out,
GELU (erf form) after the hidden layers, mean squared error over rows and
outputs.  With ``bf16=True`` the weights and the activations that feed a
product are rounded to BF16 (round to nearest even) as the GPU kernels do;
all arithmetic is FP64.  The network has no counterpart in the reference.
"""
from __future__ import annotations

import math

import numpy as np

H = 128


def layout(n_in: int, n_out: int) -> dict:
    """Offsets of W1 b1 W2 b2 W3 b3 W4 b4 in the flat parameter vector."""
    sizes = [("W1", H * n_in), ("b1", H), ("W2", H * H), ("b2", H), ("W3", H * H), ("b3", H),
             ("W4", n_out * H), ("b4", n_out)]
    off, out = 0, {}
    for name, n in sizes:
        out[name] = (off, n)
        off += n
    out["total"] = off
    return out


def unpack(p: np.ndarray, n_in: int, n_out: int) -> dict:
    L = layout(n_in, n_out)
    shapes = {"W1": (H, n_in), "b1": (H,), "W2": (H, H), "b2": (H,), "W3": (H, H), "b3": (H,),
              "W4": (n_out, H), "b4": (n_out,)}
    return {k: np.asarray(p[L[k][0]:L[k][0] + L[k][1]], dtype=np.float64).reshape(shapes[k])
            for k in shapes}


def bf16(x: np.ndarray) -> np.ndarray:
    """Round FP32 values to BF16 (nearest even), returned as FP64."""
    u = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


_erf = np.vectorize(math.erf)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2 * math.pi)


def loss_grad(p, x, t, n_in, n_out, bf16_round=True):
    """Mean squared error and its gradient (flat, FP64)."""
    P = unpack(p, n_in, n_out)
    r = bf16 if bf16_round else (lambda a: np.asarray(a, dtype=np.float64))
    W = [r(P["W1"]), r(P["W2"]), r(P["W3"]), r(P["W4"])]
    b = [P["b1"], P["b2"], P["b3"], P["b4"]]
    h = [r(x)]
    zs = []
    for l in range(3):
        z = h[-1] @ W[l].T + b[l]
        zs.append(z)
        h.append(r(gelu(z)))
    o = h[-1] @ W[3].T + b[3]
    n = x.shape[0]
    d = o - t
    loss = float((d * d).sum() / (n * n_out))
    g = 2.0 * d / (n * n_out)
    grads = {"W4": g.T @ h[3], "b4": g.sum(0)}
    dz = g
    for l in (2, 1, 0):
        dh = dz @ W[l + 1]
        dz = dh * gelu_grad(zs[l])
        grads[f"W{l + 1}"] = dz.T @ h[l]
        grads[f"b{l + 1}"] = dz.sum(0)
    L = layout(n_in, n_out)
    flat = np.zeros(L["total"])
    for k in grads:
        off, m = L[k]
        flat[off:off + m] = grads[k].ravel()
    return loss, flat


def forward(p, x, n_in, n_out, bf16_round=True):
    P = unpack(p, n_in, n_out)
    r = bf16 if bf16_round else (lambda a: np.asarray(a, dtype=np.float64))
    h = r(x)
    for l, (Wk, bk) in enumerate([("W1", "b1"), ("W2", "b2"), ("W3", "b3")]):
        h = r(gelu(h @ r(P[Wk]).T + P[bk]))
    return h @ r(P["W4"]).T + P["b4"]


def init_params(n_in: int, n_out: int, seed: int) -> np.ndarray:
    """He-normal weights, zero biases (FP32)."""
    rng = np.random.default_rng(seed)
    L = layout(n_in, n_out)
    p = np.zeros(L["total"], dtype=np.float32)
    fan = {"W1": n_in, "W2": H, "W3": H, "W4": H}
    for k, f in fan.items():
        off, m = L[k]
        p[off:off + m] = rng.normal(0.0, math.sqrt(2.0 / f), m)
    return p
