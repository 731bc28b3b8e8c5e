"""Seeded synthetic inputs of the benchmark workloads, generated on the device
directly in the grid layout (component-major, block-major, x fastest).

* ``scalar_wave``: u = sin(2 pi x) sin(2 pi y) cos(2 pi z) + U(-a, a) at cell
  centres (the Laplacian/gradient case; the reference's Laplacian benchmark
  uses the same product form, Kernel/Laplacian/Laplacian.cpp:44-53).
* ``euler_pulse``: rho = 1 + A exp(-|x - c|^2 / (2 sigma^2)), velocities
  U(-a, a), p = 1, E = p/(gamma-1) + rho |u|^2 / 2; conservative state.
* ``euler_bcs``: x periodic, y absorbing on both sides, z Dirichlet with the
  far-field state (rho = 1, momentum 0, E = 1/(gamma-1)).
"""
from __future__ import annotations

import numpy as np

from .grid import Cartesian


def _cell_centres(g: Cartesian, torch, dtype):
    """Per-cell centre coordinates (x, y, z) as (nblocks, cells) tensors."""
    nb, n = g.getSize(), g.getBlockCells()
    h = g.getCellSize()
    dev = "cuda"
    nbk = g.size()
    b = torch.arange(nbk, device=dev)
    bx, by, bz = b % nb[0], (b // nb[0]) % nb[1], b // (nb[0] * nb[1])
    c = torch.arange(n[0] * n[1] * n[2], device=dev)
    cx, cy, cz = c % n[0], (c // n[0]) % n[1], c // (n[0] * n[1])
    x = ((bx[:, None] * n[0] + cx[None, :]).to(torch.float64) + 0.5) * h[0]
    y = ((by[:, None] * n[1] + cy[None, :]).to(torch.float64) + 0.5) * h[1]
    z = ((bz[:, None] * n[2] + cz[None, :]).to(torch.float64) + 0.5) * h[2]
    return x, y, z


def _write(g: Cartesian, comp: int, values, torch):
    n = g.getBlockCells()
    cells = n[0] * n[1] * n[2]
    t = g.tensor(comp)
    t[:, :cells].copy_(values.to(t.dtype))


def scalar_wave(g: Cartesian, seed: int = 1234, noise: float = 1e-3, comp: int = 0):
    import torch
    x, y, z = _cell_centres(g, torch, torch.float64)
    u = torch.sin(2 * np.pi * x) * torch.sin(2 * np.pi * y) * torch.cos(2 * np.pi * z)
    gen = torch.Generator(device="cuda").manual_seed(seed)
    u += (torch.rand(u.shape, generator=gen, device="cuda", dtype=torch.float64) * 2 - 1) * noise
    _write(g, comp, u, torch)
    torch.cuda.synchronize()


def euler_pulse(U: Cartesian, seed: int = 1234, amp: float = 0.5, sigma: float = 0.1,
                noise: float = 1e-2, gamma: float = 1.4, centre=(0.5, 0.5, 0.5)):
    import torch
    x, y, z = _cell_centres(U, torch, torch.float64)
    r2 = (x - centre[0]) ** 2 + (y - centre[1]) ** 2 + (z - centre[2]) ** 2
    del x, y, z
    rho = 1.0 + amp * torch.exp(-r2 / (2 * sigma * sigma))
    del r2
    gen = torch.Generator(device="cuda").manual_seed(seed)
    vel = [(torch.rand(rho.shape, generator=gen, device="cuda", dtype=torch.float64) * 2 - 1) * noise
           for _ in range(3)]
    p = 1.0
    ke = 0.5 * rho * (vel[0] ** 2 + vel[1] ** 2 + vel[2] ** 2)
    _write(U, 0, rho, torch)
    for d in range(3):
        _write(U, 1 + d, rho * vel[d], torch)
    _write(U, 4, p / (gamma - 1.0) + ke, torch)
    torch.cuda.synchronize()


def far_field(gamma: float = 1.4):
    return (1.0, 0.0, 0.0, 0.0, 1.0 / (gamma - 1.0))


def euler_bcs(U: Cartesian, gamma: float = 1.4):
    """x periodic, y absorbing (both sides), z Dirichlet far field, per component."""
    from . import bc as BC
    ff = far_field(gamma)
    for c in range(5):
        U.push_boundary_bc(lambda d, s: BC.Absorbing(d, s), 1, 0, comp=c)
        U.push_boundary_bc(lambda d, s: BC.Absorbing(d, s), 1, 1, comp=c)
        U.push_boundary_bc(lambda d, s, v=ff[c]: BC.Dirichlet(d, s, v), 2, 0, comp=c)
        U.push_boundary_bc(lambda d, s, v=ff[c]: BC.Dirichlet(d, s, v), 2, 1, comp=c)


def euler_bclists(nb, gamma: float = 1.4):
    """The same BCs as oracle-style lists: 5 dicts block -> [(dir, side, kind, value)]."""
    ff = far_field(gamma)
    out = []
    for c in range(5):
        d = {}
        for b in range(int(np.prod(nb))):
            bi = (b % nb[0], (b // nb[0]) % nb[1], b // (nb[0] * nb[1]))
            lst = []
            if bi[1] == 0:
                lst.append((1, 0, 2, 0.0))
            if bi[1] == nb[1] - 1:
                lst.append((1, 1, 2, 0.0))
            if bi[2] == 0:
                lst.append((2, 0, 1, ff[c]))
            if bi[2] == nb[2] - 1:
                lst.append((2, 1, 1, ff[c]))
            if lst:
                d[b] = lst
        out.append(d)
    return out


def poisson_coefficient(k: Cartesian, seed: int = 1234, sigma: float = 0.5):
    """k = 3-cell box filter (per axis, periodic) of exp(N(0, sigma^2)) i.i.d. per cell."""
    import torch
    nb, n = k.getSize(), k.getBlockCells()
    G = [nb[d] * n[d] for d in range(3)]
    gen = torch.Generator(device="cuda").manual_seed(seed)
    a = torch.exp(torch.randn((G[2], G[1], G[0]), generator=gen, device="cuda", dtype=torch.float64) * sigma)
    for dim in range(3):
        a = (torch.roll(a, 1, dim) + a + torch.roll(a, -1, dim)) / 3.0
    _global_to_blocks(k, a, torch)


def poisson_rhs(f: Cartesian, seed: int = 4321, count: int = 32, width=(0.02, 0.08), amp=(-1.0, 1.0)):
    """f = sum of `count` Gaussians (centres uniform in [0,1)^3, widths and
    amplitudes uniform in the given ranges, periodic minimum-image distance),
    minus its mean."""
    import torch
    nb, n = f.getSize(), f.getBlockCells()
    G = [nb[d] * n[d] for d in range(3)]
    h = f.getCellSize()
    gen = torch.Generator(device="cpu").manual_seed(seed)
    c = torch.rand((count, 3), generator=gen, dtype=torch.float64)
    w = width[0] + (width[1] - width[0]) * torch.rand(count, generator=gen, dtype=torch.float64)
    a = amp[0] + (amp[1] - amp[0]) * torch.rand(count, generator=gen, dtype=torch.float64)
    xs = [((torch.arange(G[d], device="cuda", dtype=torch.float64) + 0.5) * h[d]) for d in range(3)]
    out = torch.zeros((G[2], G[1], G[0]), device="cuda", dtype=torch.float64)
    for j in range(count):
        d2 = []
        for d in range(3):
            t = xs[d] - float(c[j, d])
            t = t - torch.round(t)
            d2.append(t * t)
        r2 = d2[2][:, None, None] + d2[1][None, :, None] + d2[0][None, None, :]
        out += float(a[j]) * torch.exp(-r2 / (2.0 * float(w[j]) ** 2))
    out -= out.mean()
    _global_to_blocks(f, out, torch)


def _global_to_blocks(g: Cartesian, arr, torch):
    nb, n = g.getSize(), g.getBlockCells()
    cells = n[0] * n[1] * n[2]
    v = arr.reshape(nb[2], n[2], nb[1], n[1], nb[0], n[0]).permute(0, 2, 4, 1, 3, 5).reshape(g.size(), cells)
    g.tensor(0)[:, :cells].copy_(v.to(g.tensor(0).dtype))
    torch.cuda.synchronize()
