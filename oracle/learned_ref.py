"""FP64 numpy restatement of the learned preconditioner's network, its loss
and its gradients.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the CUDA
forward/backward kernels (gpu-micromagnetics-irregular_b200/csrc/k_learned.cu).
The product never imports this file.

The reference has no learned component; this file restates the network the
CUDA code implements, so that its kernels can be checked against an
independent FP64 computation (and this file against finite differences).

Network (linear in the residual, so it is a fixed linear preconditioner
between setups):
    u      = block-Jacobi solve of r                      (3, H, W)
    F      = [u, m x u, m x (m x u)] * mask               (9, H, W)
    y1     = conv3x3(F,  W1)   W1: (16, 9, 3, 3)
    y2     = conv3x3(y1, W2)   W2: (16, 16, 3, 3)
    y3     = conv3x3(y2, W3)   W3: (3, 16, 3, 3)
    z      = (u + gamma * y3) * mask
conv3x3 is a cross-correlation with zero padding, no bias, no activation:
    out[o, i, j] = sum_c sum_{dy,dx in -1..1} w[o, c, dy+1, dx+1] in[c, i+dy, j+dx]

Loss of one patch (the solver's own SPGMR solution x as the target, weighted
by the integrator's error weights, interior cells only, border B = 3):
    L = sum_int (ewt * (z - x))^2 / sum_int (ewt * x)^2
The batch loss is the mean over patches.
"""
from __future__ import annotations

import numpy as np

C_IN, C_HID, C_OUT = 9, 16, 3
BORDER = 3
SHAPES = ((C_HID, C_IN, 3, 3), (C_HID, C_HID, 3, 3), (C_OUT, C_HID, 3, 3))


def nparams():
    return sum(int(np.prod(s)) for s in SHAPES)


def unpack(theta):
    out, k = [], 0
    for s in SHAPES:
        n = int(np.prod(s))
        out.append(theta[k:k + n].reshape(s))
        k += n
    return out


def features(u, m, mask):
    mu = np.cross(m, u, axis=0)
    mmu = np.cross(m, mu, axis=0)
    return np.concatenate([u, mu, mmu], axis=0) * mask[None]


def conv(x, w):
    cin, h, wd = x.shape
    xp = np.zeros((cin, h + 2, wd + 2))
    xp[:, 1:-1, 1:-1] = x
    out = np.zeros((w.shape[0], h, wd))
    for dy in range(3):
        for dx in range(3):
            out += np.einsum("oc,chw->ohw", w[:, :, dy, dx], xp[:, dy:dy + h, dx:dx + wd])
    return out


def conv_bwd_data(dout, w):
    """d(in) of conv: correlation of dout with the flipped kernel."""
    cout, h, wd = dout.shape
    dp = np.zeros((cout, h + 2, wd + 2))
    dp[:, 1:-1, 1:-1] = dout
    din = np.zeros((w.shape[1], h, wd))
    for dy in range(3):
        for dx in range(3):
            # in[c, i+dy-1, j+dx-1] contributed to out[o, i, j]
            din += np.einsum("oc,ohw->chw", w[:, :, dy, dx], dp[:, 2 - dy:2 - dy + h, 2 - dx:2 - dx + wd])
    return din


def conv_bwd_weight(x, dout):
    cin, h, wd = x.shape
    xp = np.zeros((cin, h + 2, wd + 2))
    xp[:, 1:-1, 1:-1] = x
    dw = np.zeros((dout.shape[0], cin, 3, 3))
    for dy in range(3):
        for dx in range(3):
            dw[:, :, dy, dx] = np.einsum("ohw,chw->oc", dout, xp[:, dy:dy + h, dx:dx + wd])
    return dw


def forward(theta, u, m, mask, gamma):
    w1, w2, w3 = unpack(theta)
    f = features(u, m, mask)
    y1 = conv(f, w1)
    y2 = conv(y1, w2)
    y3 = conv(y2, w3)
    z = (u + gamma * y3) * mask[None]
    return z, (f, y1, y2, y3)


def interior(h, w):
    k = np.zeros((h, w))
    k[BORDER:h - BORDER, BORDER:w - BORDER] = 1.0
    return k


def loss_and_grad(theta, batch):
    """batch: list of dicts with u, m, mask, ewt, x (arrays) and gamma."""
    w1, w2, w3 = unpack(theta)
    g1, g2, g3 = np.zeros_like(w1), np.zeros_like(w2), np.zeros_like(w3)
    total = 0.0
    nb = len(batch)
    for s in batch:
        z, (f, y1, y2, y3) = forward(theta, s["u"], s["m"], s["mask"], s["gamma"])
        _, h, w = z.shape
        it = interior(h, w)[None]
        e = s["ewt"] * (z - s["x"]) * it
        den = float(np.sum((s["ewt"] * s["x"] * it) ** 2))
        den = den if den > 0.0 else 1.0
        total += float(np.sum(e ** 2)) / den
        dz = 2.0 * s["ewt"] * e / den / nb
        dy3 = s["gamma"] * dz * s["mask"][None]
        g3 += conv_bwd_weight(y2, dy3)
        dy2 = conv_bwd_data(dy3, w3)
        g2 += conv_bwd_weight(y1, dy2)
        dy1 = conv_bwd_data(dy2, w2)
        g1 += conv_bwd_weight(f, dy1)
    return total / nb, np.concatenate([g1.ravel(), g2.ravel(), g3.ravel()])


def random_batch(rng, nb, h, w, gamma_range=(0.005, 0.05)):
    batch = []
    for _ in range(nb):
        m = rng.standard_normal((3, h, w))
        m /= np.linalg.norm(m, axis=0, keepdims=True)
        mask = (rng.uniform(size=(h, w)) > 0.1).astype(np.float64)
        batch.append(dict(u=rng.standard_normal((3, h, w)) * mask, m=m, mask=mask,
                          ewt=rng.uniform(0.5, 2.0, (3, h, w)), x=rng.standard_normal((3, h, w)),
                          gamma=float(rng.uniform(*gamma_range))))
    return batch
