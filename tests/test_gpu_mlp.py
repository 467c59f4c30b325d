"""GPU: the surrogate network's own kernels against the CPU FP64 oracle.

The oracle rounds weights and product inputs to BF16 as the kernels do, so the
remaining differences are FP32 accumulation and the odd activation that lands
on the other side of a BF16 rounding boundary."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu


def _data(n, n_in, n_out, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(n, n_in)).astype(np.float32)
    t = rng.normal(size=(n, n_out)).astype(np.float32)
    p = mo.init_params(n_in, n_out, seed)
    p += rng.normal(0, 0.02, p.size).astype(np.float32)  # nonzero biases
    return x, t, p


@pytest.mark.parametrize("n_in,n_out,n", [(41, 24, 300), (67, 24, 1000), (7, 1, 33), (128, 64, 96)])
def test_gradient_matches_oracle(n_in, n_out, n):
    import torch

    from summit_b200.surrogate import Surrogate

    x, t, p = _data(n, n_in, n_out, 11 + n_in)
    net = Surrogate(n_in, n_out, params=p)
    loss, g = net.loss_grad(torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda())
    want_loss, want_g = mo.loss_grad(p.astype(np.float64), x.astype(np.float64),
                                     t.astype(np.float64), n_in, n_out)
    assert abs(loss - want_loss) <= 1e-4 * want_loss
    g = g.cpu().numpy().astype(np.float64)
    L = mo.layout(n_in, n_out)
    for k in ["W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4"]:
        off, m = L[k]
        a, b = g[off:off + m], want_g[off:off + m]
        err = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
        assert err <= 2e-3, (k, err)


def test_forward_matches_oracle():
    import torch

    from summit_b200.surrogate import Surrogate

    n_in, n_out, n = 41, 24, 517
    x, _, p = _data(n, n_in, n_out, 5)
    net = Surrogate(n_in, n_out, params=p)
    out = net.forward(torch.from_numpy(x).cuda()).cpu().numpy()
    want = mo.forward(p.astype(np.float64), x.astype(np.float64), n_in, n_out)
    assert np.max(np.abs(out - want)) <= 2e-3 * np.max(np.abs(want))


def test_training_fits_a_smooth_function():
    import torch

    from summit_b200.surrogate import Surrogate

    rng = np.random.default_rng(0)
    n, n_in, n_out = 20000, 8, 3
    x = rng.normal(size=(n, n_in)).astype(np.float32)
    t = np.stack([np.sin(x[:, 0]) + 0.5 * x[:, 1] ** 2, x[:, 2] * x[:, 3], np.tanh(x[:, 4])],
                 1).astype(np.float32)
    xt, tt = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    net = Surrogate(n_in, n_out, seed=1)
    l0, _ = net.loss_grad(xt, tt)
    losses = net.train(xt, tt, epochs=30, batch=1024, lr=2e-3, seed=2)
    l1, _ = net.loss_grad(xt, tt)
    assert np.all(np.isfinite(losses))
    assert l1 < 0.05 * l0, (l0, l1, losses[-5:])
