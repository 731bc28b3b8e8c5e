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


def amr_layout(seed: int = 1, roots: int = 8, keep_root: float = 0.9, keep16: float = 0.8,
               split16_in: float = 0.5, split32_in: float = 0.3, radius: float = 0.15,
               centre=(0.5, 0.5, 0.5)):
    """Two-level block layout of the periodic unit box by seeded octree splitting.

    The box is cut into roots^3 cubes of edge 1/roots; with F = 64 * roots
    level-1 cells across the box, a cube of edge F/roots/2^k (level-1 cells)
    becomes one block.  Outside a sphere (radius, centre) blocks are level 0
    (cell = 2 level-1 cells): a root stays one 32^3 block with probability
    keep_root, else its 16^3 children stay with probability keep16, else they
    split into 8^3 blocks.  Inside the sphere blocks are level 1: 1/16-edge
    cubes stay 32^3 blocks unless split (split16_in), 1/32-edge cubes stay
    16^3 unless split (split32_in) into 8^3 blocks.  The defaults give 2045
    blocks (55 % 8^3, 21 % 16^3, 24 % 32^3, 651 on level 1, 18.3 M cells).
    Returns (levels, cells, origins, F)."""
    rng = np.random.default_rng(seed)
    F = 64 * roots
    levels, cells, origins = [], [], []
    c = np.array(centre)

    def inside(o, s):
        d = (np.array(o) + s / 2) / F - c
        d -= np.round(d)
        return np.linalg.norm(d) < radius

    def leaf(level, n, o):
        levels.append(level)
        cells.append(n)
        origins.append(o)

    def rec(o, s):  # s: edge in level-1 cells
        l1 = inside(o, s)
        if s == 64:
            if not l1 and rng.random() < keep_root:
                return leaf(0, 32, o)
        elif s == 32:
            if l1:
                if rng.random() > split16_in:
                    return leaf(1, 32, o)
            elif rng.random() < keep16:
                return leaf(0, 16, o)
        elif s == 16:
            if not l1:
                return leaf(0, 8, o)
            if rng.random() > split32_in:
                return leaf(1, 16, o)
        else:
            return leaf(1, 8, o)
        h = s // 2
        for k in range(8):
            rec((o[0] + (k & 1) * h, o[1] + ((k >> 1) & 1) * h, o[2] + (k >> 2) * h), h)

    for k in range(roots):
        for j in range(roots):
            for i in range(roots):
                rec((64 * i, 64 * j, 64 * k), 64)
    return np.array(levels), np.array(cells), np.array(origins), F


def amr_small_layout(seed: int = 3):
    """A small two-level layout (box of 64 level-1 cells) with every kind of
    interface, for parity tests: 2^3 roots of edge 32 become a level-0 16^3
    block, or level-0 8^3 / level-1 16^3 children, or level-1 8^3 blocks."""
    rng = np.random.default_rng(seed)
    levels, cells, origins = [], [], []
    for k in range(2):
        for j in range(2):
            for i in range(2):
                o = (32 * i, 32 * j, 32 * k)
                r = rng.random()
                if r < 0.3:
                    levels.append(0), cells.append(16), origins.append(o)
                    continue
                for c in range(8):
                    oc = (o[0] + (c & 1) * 16, o[1] + ((c >> 1) & 1) * 16, o[2] + (c >> 2) * 16)
                    r2 = rng.random()
                    if r2 < 0.4:
                        levels.append(0), cells.append(8), origins.append(oc)
                    elif r2 < 0.7:
                        levels.append(1), cells.append(16), origins.append(oc)
                    else:
                        for g in range(8):
                            og = (oc[0] + (g & 1) * 8, oc[1] + ((g >> 1) & 1) * 8, oc[2] + (g >> 2) * 8)
                            levels.append(1), cells.append(8), origins.append(og)
    return np.array(levels), np.array(cells), np.array(origins), 64


def euler_pulse_amr(U, seed: int = 1234, amp: float = 0.5, sigma: float = 0.1, noise: float = 1e-2,
                    gamma: float = 1.4, centre=(0.5, 0.5, 0.5)):
    """The Euler pulse state on an AMR layout (periodic minimum-image distance)."""
    import torch
    x, y, z = U.cell_centres()
    d = [x - centre[0], y - centre[1], z - centre[2]]
    r2 = sum((t - torch.round(t)) ** 2 for t in d)
    rho = 1.0 + amp * torch.exp(-r2 / (2 * sigma * sigma))
    gen = torch.Generator(device="cuda").manual_seed(seed)
    vel = [(torch.rand(rho.shape, generator=gen, device="cuda", dtype=torch.float64) * 2 - 1) * noise
           for _ in range(3)]
    ke = 0.5 * rho * (vel[0] ** 2 + vel[1] ** 2 + vel[2] ** 2)
    U.tensor(0).copy_(rho.to(U.tensor(0).dtype))
    for k in range(3):
        U.tensor(1 + k).copy_((rho * vel[k]).to(U.tensor(0).dtype))
    U.tensor(4).copy_((1.0 / (gamma - 1.0) + ke).to(U.tensor(0).dtype))
    torch.cuda.synchronize()
