"""Numpy oracle of the learned smoother's training loss and gradients.

TEST INFRASTRUCTURE ONLY.  Float64 restatement of the forward pass, the
residual-reduction loss and the manual backward pass of the device kernels in
cubismnova_b200/csrc/learned.cu (the reference has no learned components):

    h1 = relu(conv(W1, x)), h2 = relu(conv(W2, h1)), y = conv(W3, h2)
    c  = omega * x0 + y                      on the region (P+2)^3
    loss = mean_b || r_b - A c_b ||^2 / || r_b ||^2   on the interior P^3

Patch arrays are (B, C, S, S, S) in (z, y, x) order; weights (27, Cin, Cout)
with tap = dx + 3 dy + 9 dz.  ``loss_and_grad`` is checked against central
finite differences by ``fd_check``.

With ``bf16=True`` the forward and backward round where the tensor-core
training path (cubismnova_b200/csrc/learned_train_tc.cu) stores BF16: the
hidden layer's weights W2, the activations h1 and h2 after the ReLU, and the
activation gradients gh2 and gh1 after the ReLU mask (each value first
rounded to float32, as the device computes it, then to BF16 with
round-to-nearest-even).
"""
from __future__ import annotations

import numpy as np


def conv_valid(x, W):
    B, Ci, S = x.shape[0], x.shape[1], x.shape[2]
    So = S - 2
    out = np.zeros((B, W.shape[2], So, So, So))
    for dz in range(3):
        for dy in range(3):
            for dx in range(3):
                t = dx + 3 * dy + 9 * dz
                out += np.einsum("bizyx,io->bozyx", x[:, :, dz:dz + So, dy:dy + So, dx:dx + So], W[t])
    return out


def conv_valid_bwd(x, W, gout):
    """Gradients of conv_valid wrt x and W for output gradient gout."""
    So = gout.shape[2]
    gx = np.zeros_like(x)
    gW = np.zeros_like(W)
    for dz in range(3):
        for dy in range(3):
            for dx in range(3):
                t = dx + 3 * dy + 9 * dz
                xs = x[:, :, dz:dz + So, dy:dy + So, dx:dx + So]
                gW[t] += np.einsum("bizyx,bozyx->io", xs, gout)
                gx[:, :, dz:dz + So, dy:dy + So, dx:dx + So] += np.einsum("bozyx,io->bizyx", gout, W[t])
    return gx, gW


def bf16(a):
    """Round to BF16 (nearest, ties to even) via float32; returns float64."""
    f = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def harm(a, b):
    t = a * b
    return (t + t) / (a + b)


def apply_A(c, k, ih2):
    """A c on the interior of a (B, R, R, R) region."""
    cc = c[:, 1:-1, 1:-1, 1:-1]
    kc = k[:, 1:-1, 1:-1, 1:-1]
    out = np.zeros_like(cc)
    for ax in (3, 2, 1):
        sl_p = [slice(None), slice(1, -1), slice(1, -1), slice(1, -1)]
        sl_m = list(sl_p)
        sl_p[ax] = slice(2, None)
        sl_m[ax] = slice(0, -2)
        kp = harm(kc, k[tuple(sl_p)])
        km = harm(k[tuple(sl_m)], kc)
        out += kp * (c[tuple(sl_p)] - cc) - km * (cc - c[tuple(sl_m)])
    return ih2 * out


def A_adjoint(g, k, ih2):
    """Adjoint of c -> A c (interior) applied to g (B, P, P, P): result (B, R, R, R)."""
    B, P = g.shape[0], g.shape[1]
    R = P + 2
    out = np.zeros((B, R, R, R))
    kc = k[:, 1:-1, 1:-1, 1:-1]
    inner = (slice(None), slice(1, -1), slice(1, -1), slice(1, -1))
    for ax in (3, 2, 1):
        sl_p = [slice(None), slice(1, -1), slice(1, -1), slice(1, -1)]
        sl_m = list(sl_p)
        sl_p[ax] = slice(2, None)
        sl_m[ax] = slice(0, -2)
        kp = harm(kc, k[tuple(sl_p)])
        km = harm(k[tuple(sl_m)], kc)
        out[tuple(sl_p)] += ih2 * kp * g
        out[inner] -= ih2 * kp * g
        out[inner] -= ih2 * km * g
        out[tuple(sl_m)] += ih2 * km * g
    return out


def forward(x, k, r, W1, W2, W3, omega, ih2, bf16_path=False):
    rnd = bf16 if bf16_path else (lambda a: a)
    h1 = rnd(np.maximum(conv_valid(x, W1), 0))
    h2 = rnd(np.maximum(conv_valid(h1, rnd(W2)), 0))
    y = conv_valid(h2, W3)[:, 0]
    c = omega * x[:, 0, 3:-3, 3:-3, 3:-3] + y
    res = r - apply_A(c, k, ih2)
    rr = (r ** 2).sum(axis=(1, 2, 3))
    ee = (res ** 2).sum(axis=(1, 2, 3))
    loss = float(np.mean(ee / rr))
    return loss, dict(h1=h1, h2=h2, y=y, c=c, res=res, rr=rr)


def loss_and_grad(x, k, r, W1, W2, W3, omega, ih2, bf16_path=False):
    rnd = bf16 if bf16_path else (lambda a: a)
    B = x.shape[0]
    loss, t = forward(x, k, r, W1, W2, W3, omega, ih2, bf16_path)
    g = (-2.0 / (t["rr"] * B))[:, None, None, None] * t["res"]
    gc = A_adjoint(g, k, ih2)
    gy = gc[:, None]
    gh2, gW3 = conv_valid_bwd(t["h2"], W3, gy)
    gh2 = rnd(gh2 * (t["h2"] > 0))
    gh1, gW2 = conv_valid_bwd(t["h1"], rnd(W2), gh2)
    gh1 = rnd(gh1 * (t["h1"] > 0))
    _, gW1 = conv_valid_bwd(x, W1, gh1)
    return loss, gW1, gW2, gW3


def fd_check(x, k, r, W1, W2, W3, omega, ih2, n=12, eps=1e-6, seed=0):
    """Max relative error of loss_and_grad against central differences on n
    random weights of each layer."""
    _, g1, g2, g3 = loss_and_grad(x, k, r, W1, W2, W3, omega, ih2)
    rng = np.random.default_rng(seed)
    worst = 0.0
    for W, g in ((W1, g1), (W2, g2), (W3, g3)):
        for _ in range(n):
            idx = tuple(rng.integers(0, s) for s in W.shape)
            old = W[idx]
            W[idx] = old + eps
            lp, _ = forward(x, k, r, W1, W2, W3, omega, ih2)
            W[idx] = old - eps
            lm, _ = forward(x, k, r, W1, W2, W3, omega, ih2)
            W[idx] = old
            fd = (lp - lm) / (2 * eps)
            scale = max(abs(fd), abs(g[idx]), 1e-12)
            worst = max(worst, abs(fd - g[idx]) / scale)
    return worst
