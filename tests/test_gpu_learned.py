"""Learned smoother: device loss/gradients vs the numpy oracle (itself checked
by finite differences), training reduces the loss, and multigrid with the
trained smoother converges."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_loss_and_gradient_match_oracle(cn):
    import torch
    from oracle import nn_oracle as N
    rng = np.random.default_rng(0)
    B, P = 3, 4
    S, R = P + 8, P + 2
    x = rng.standard_normal((B, 2, S, S, S))
    k = 0.5 + rng.random((B, R, R, R))
    r = rng.standard_normal((B, P, P, P))
    nn = cn.learned.LearnedSmoother(seed=3, omega=0.8, init_scale=0.05)
    W1, W2, W3 = [w.astype(np.float64) for w in nn.weights()]
    ih2 = 16.0
    tx = torch.tensor(x, dtype=torch.float32, device="cuda").reshape(B, 2, -1).contiguous()
    tk = torch.tensor(k, dtype=torch.float32, device="cuda").reshape(B, -1).contiguous()
    tr = torch.tensor(r, dtype=torch.float32, device="cuda").reshape(B, -1).contiguous()
    loss, (g1, g2, g3) = nn.loss_grad(tx, tk, tr, P, ih2)
    x32, k32, r32 = (a.astype(np.float32).astype(np.float64) for a in (x, k, r))
    wl, w1, w2, w3 = N.loss_and_grad(x32, k32, r32, W1, W2, W3, 0.8, ih2)
    assert abs(loss - wl) <= 1e-4 * abs(wl)
    for got, want in ((g1, w1), (g2, w2), (g3, w3)):
        err = np.max(np.abs(got - want)) / np.max(np.abs(want))
        assert err < 1e-3, err
    assert N.fd_check(x32, k32, r32, W1, W2, W3, 0.8, ih2, n=4) < 1e-5


def _poisson(cn, nb, n, seed=1):
    k = cn.Grid.Cartesian(nb, n, dtype=np.float32)
    cn.workloads.poisson_coefficient(k, seed=seed)
    f = cn.Grid.Cartesian(nb, n, dtype=np.float32)
    cn.workloads.poisson_rhs(f, seed=seed + 1)
    return k, f


def test_training_and_learned_multigrid(cn):
    import torch
    nb, n = (4, 4, 4), (16, 16, 16)
    k, f = _poisson(cn, nb, n)
    m = cn.mg.Multigrid(k, nu1=2, nu2=2, omega=0.8)
    x, kk, r, P = cn.learned.collect_patches(m, f, cycles=6, per_snapshot=16, max_patches=192, seed=5)
    assert x.shape[0] == 192
    nn = cn.learned.LearnedSmoother(seed=1, omega=0.8, init_scale=1e-3)
    ih2 = 1.0 / k.getCellSize()[0] ** 2
    l0, _ = nn.loss_grad(x[:32], kk[:32], r[:32], P, ih2)
    last = nn.train(x, kk, r, P, ih2, epochs=8, batch=16, lr=2e-3, seed=2)
    l1, _ = nn.loss_grad(x[:32], kk[:32], r[:32], P, ih2)
    print(f"loss before {l0:.4f} after {l1:.4f} (last epoch {last:.4f})")
    assert l1 < l0
    p64 = cn.Grid.Cartesian(nb, n, dtype=np.float64)
    cyc_plain, rel_plain = m.solve(f, p64, rtol=1e-8, max_cycles=60)
    # what training gains: the same network untrained (near-zero weights,
    # i.e. damped Jacobi) against the trained one, both replacing Jacobi on
    # the finest level, where the training residuals came from
    untrained = cn.learned.LearnedSmoother(seed=1, omega=0.8, init_scale=1e-3)
    cn.learned.use_in(m, untrained, level_mask=0x1)
    cyc_u, rel_u = m.solve(f, p64, rtol=1e-8, max_cycles=60)
    cn.learned.use_in(m, nn, level_mask=0x1)
    cyc_nn, rel_nn = m.solve(f, p64, rtol=1e-8, max_cycles=60)
    print(f"plain: {cyc_plain} cycles ({rel_plain:.2e}); untrained: {cyc_u} ({rel_u:.2e}); "
          f"trained: {cyc_nn} cycles ({rel_nn:.2e})")
    assert rel_nn <= 1e-8 and rel_u <= 1e-8 and rel_plain <= 1e-8
    rr, ff = m.residual(p64, f)
    assert np.sqrt(rr / ff) <= 1e-8
    # measured here: plain 15, untrained 15, trained 11 cycles
    assert cyc_nn <= cyc_plain - 2 and cyc_nn <= cyc_u - 2
