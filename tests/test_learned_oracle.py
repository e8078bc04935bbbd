"""CPU: the FP64 restatement of the learned preconditioner's network
(oracle/learned_ref.py) against central finite differences, so that it can
serve as the checker of the CUDA forward/backward kernels."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import learned_ref as L  # noqa: E402


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(7)
    theta = rng.standard_normal(L.nparams()) * 0.1
    batch = L.random_batch(rng, 2, 10, 11)
    _, g = L.loss_and_grad(theta, batch)
    idx = rng.choice(theta.size, 40, replace=False)
    h = 1e-6
    for i in idx:
        tp, tm = theta.copy(), theta.copy()
        tp[i] += h
        tm[i] -= h
        fd = (L.loss_and_grad(tp, batch)[0] - L.loss_and_grad(tm, batch)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])


def test_network_is_linear_in_the_residual():
    rng = np.random.default_rng(8)
    theta = rng.standard_normal(L.nparams()) * 0.1
    s = L.random_batch(rng, 1, 9, 8)[0]
    u2 = rng.standard_normal(s["u"].shape) * s["mask"][None]
    za, _ = L.forward(theta, s["u"], s["m"], s["mask"], 0.03)
    zb, _ = L.forward(theta, u2, s["m"], s["mask"], 0.03)
    zc, _ = L.forward(theta, 2.0 * s["u"] - 0.5 * u2, s["m"], s["mask"], 0.03)
    assert np.abs(zc - (2.0 * za - 0.5 * zb)).max() < 1e-12


def test_conv_adjoint_identity():
    rng = np.random.default_rng(9)
    w = rng.standard_normal((5, 4, 3, 3))
    x = rng.standard_normal((4, 7, 6))
    d = rng.standard_normal((5, 7, 6))
    lhs = np.sum(L.conv(x, w) * d)
    rhs = np.sum(x * L.conv_bwd_data(d, w))
    assert abs(lhs - rhs) < 1e-10 * abs(lhs)
