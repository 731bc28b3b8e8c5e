"""The learned smoother's tensor-core (tcgen05) convolutions: one 16 -> 16
layer against a float64 numpy convolution of the same BF16-rounded inputs
and weights (FP32 accumulation, BF16 output: stated tolerance 2^-8 relative
plus 1e-4 of the output scale), and the whole smoother on the tensor cores
against its FP32 CUDA-core form inside a V-cycle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bf16_round(a):
    """Round float32 values to the nearest BF16 (ties to even), as float64."""
    u = np.asarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _to_global(v, nb, n):
    """[nblocks*cells, C] grid order -> [Z, Y, X, C] global array."""
    C_ = v.shape[-1]
    a = v.reshape(nb[2], nb[1], nb[0], n[2], n[1], n[0], C_)
    return a.transpose(0, 3, 1, 4, 2, 5, 6).reshape(nb[2] * n[2], nb[1] * n[1], nb[0] * n[0], C_)


def _conv_ref(g, W, relu):
    out = np.zeros(g.shape[:3] + (W.shape[2],))
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                t = (dx + 1) + 3 * (dy + 1) + 9 * (dz + 1)
                s = np.roll(g, shift=(-dz, -dy, -dx), axis=(0, 1, 2))
                out += s @ W[t]
    return np.maximum(out, 0) if relu else out


@pytest.mark.parametrize("nb,n,relu", [((2, 1, 2), (16, 16, 8), True), ((1, 2, 1), (32, 16, 4), False)])
def test_conv3_bf16_matches_reference(cn, nb, n, relu):
    import torch
    rng = np.random.default_rng(7)
    cells = int(np.prod(nb)) * int(np.prod(n))
    x32 = rng.standard_normal((cells, 16)).astype(np.float32)
    W = (0.1 * rng.standard_normal((27, 16, 16))).astype(np.float32)
    x = torch.tensor(x32, device="cuda").to(torch.bfloat16)
    w = torch.tensor(W, device="cuda")
    y = cn.learned.conv3_bf16(x, nb, n, w, relu=relu)
    torch.cuda.synchronize()
    got = _to_global(y.float().cpu().numpy().astype(np.float64), nb, n)
    ref = _conv_ref(_to_global(_bf16_round(x32), nb, n), _bf16_round(W), relu)
    assert np.isfinite(got).all()
    scale = np.max(np.abs(ref))
    err = np.abs(got - ref) - (2.0 ** -8) * np.abs(ref)
    assert np.max(err) <= 1e-4 * scale, np.max(err) / scale


def test_tensor_core_smoother_matches_fp32(cn):
    """One V-cycle with the learned smoother on the finest level: tensor-core
    inference against FP32 inference of the same weights (BF16 activations:
    1e-2 relative)."""
    import torch
    nb, n = (2, 2, 2), (16, 16, 16)
    k = cn.Grid.Cartesian(nb, n, dtype=np.float32)
    cn.workloads.poisson_coefficient(k, seed=3)
    f = cn.Grid.Cartesian(nb, n, dtype=np.float32)
    cn.workloads.poisson_rhs(f, seed=4)
    m = cn.mg.Multigrid(k, nu1=2, nu2=2, omega=0.8)
    nn = cn.learned.LearnedSmoother(seed=5, omega=0.8, init_scale=0.05)
    cn.learned.use_in(m, nn, level_mask=0x1)
    out = {}
    for mode in ("fp32", "tensor"):
        nn.set_inference(mode)
        e = cn.Grid.Cartesian(nb, n, dtype=np.float32)
        m.vcycle(f, e)
        torch.cuda.synchronize()
        out[mode] = e.download().astype(np.float64)
    a, b = out["fp32"], out["tensor"]
    assert np.isfinite(b).all()
    assert np.max(np.abs(a - b)) <= 1e-2 * np.max(np.abs(a))
