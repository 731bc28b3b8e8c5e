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


def _pack(level, counts, slots, levels, cells, origins):
    """Places blocks of each edge (level-1 cells; counts {edge: number}) in
    descending size into free aligned cubic slots ({edge: [origins]}),
    splitting a larger slot into its 8 octants when no slot of the edge is
    left.  Returns False when a size finds no room."""
    for e in sorted(counts, reverse=True):
        for _ in range(counts[e]):
            if not slots.get(e):
                bigger = [k for k in slots if k > e and slots[k]]
                if not bigger:
                    return False
                k = min(bigger)
                while k > e:
                    o = slots[k].pop(0)
                    h = k // 2
                    slots.setdefault(h, [])[:0] = [(o[0] + (q & 1) * h, o[1] + ((q >> 1) & 1) * h, o[2] + (q >> 2) * h)
                                                   for q in range(8)]
                    k = h
            levels.append(level)
            cells.append(e if level == 1 else e // 2)
            origins.append(slots[e].pop(0))
    return not any(slots.values())


def amr_layout(seed: int = 1, nblocks: int = 2048, probs=(0.5, 0.35, 0.15), refined=(0.03, 0.2),
               max_tries: int = 100):
    """The batched AMR layout: `nblocks` blocks whose cells per side are drawn
    by seed from {8, 16, 32} with probabilities `probs`, on two levels (ratio
    2), tiling a periodic box: a level-0 tiling refined to level 1 inside a
    seeded ball.

    A level-1 block of n cells spans n level-1 cells, a level-0 block 2n.  In
    units of 8^3 level-1 cells every block's volume is a power of 8, i.e. 1
    modulo 7, so blocks tile a box of volume V only if V = nblocks (mod 7); for
    2048 blocks no cube qualifies (cubes are 0, 1 or 6 modulo 7).  The box is
    therefore Px x Py x Pz cubes of 32 level-1 cells (volume 64 Px Py Pz
    units) whose level-1 volume
        V1 = (8 n8 + 64 n16 + 512 n32 - 64 Px Py Pz) / 7
    is a fraction `refined` of the box; candidates are tried from the most
    nearly cubic.  The refined region is the V1 / 8 cubes of 16 level-1 cells
    nearest (periodically) to a seeded centre.  Level-1 blocks fill it exactly
    (a_k of the k^3 blocks, a8 + 8 a16 + 64 a32 = V1, near the drawn size mix
    but with enough 32^3 blocks that the level-0 32^3 blocks find whole
    unrefined 64-cubes) and level-0 blocks fill the rest, each level packed by
    _pack.  Draws (generator seeded with [seed, try]) that pack in no
    candidate box are redrawn.  Defaults: 2048 blocks, about 13.5 M cells.
    Returns (levels, cells, origins, (Lx, Ly, Lz))."""
    for attempt in range(max_tries):
        rng = np.random.default_rng([seed, attempt])
        sizes = rng.choice(np.array([8, 16, 32]), size=nblocks, p=np.asarray(probs, float))
        n8, n16, n32 = (int(np.sum(sizes == k)) for k in (8, 16, 32))
        S = 8 * n8 + 64 * n16 + 512 * n32
        boxes = []
        for Px in range(2, 65):
            for Py in range(2, Px + 1):
                for Pz in range(2, Py + 1):
                    P = Px * Py * Pz
                    if S - 64 * P <= 0 or (S - 64 * P) % 56:
                        continue
                    V1 = (S - 64 * P) // 7
                    if refined[0] <= V1 / (64 * P) <= refined[1]:
                        boxes.append((Px / Pz, (Px % 2) + (Py % 2) + (Pz % 2), (Px, Py, Pz), V1))
        centre_frac = rng.random(3)
        for _, _, (Px, Py, Pz), V1 in sorted(boxes)[:40]:
            out = _amr_fill(Px, Py, Pz, V1, n8, n16, n32, centre_frac)
            if out is not None:
                return out
    raise RuntimeError("amr_layout: no draw tiles a box; change the seed or the refined fraction")


def _amr_fill(Px, Py, Pz, V1, n8, n16, n32, centre_frac):
    """One candidate box of amr_layout: refined region, level mix, packing.
    Returns (levels, cells, origins, L) or None."""
    G = (2 * Px, 2 * Py, 2 * Pz)  # 16-cubes per side
    L = (32 * Px, 32 * Py, 32 * Pz)
    K16 = V1 // 8
    centre = centre_frac * np.array(L)
    iz, iy, ix = np.meshgrid(*[np.arange(G[d]) for d in (2, 1, 0)], indexing="ij")
    pos = np.stack([(ix + 0.5) * 16, (iy + 0.5) * 16, (iz + 0.5) * 16], -1).reshape(-1, 3) - centre
    pos -= np.round(pos / np.array(L)) * np.array(L)
    order = np.lexsort((np.arange(pos.shape[0]), np.sum(pos * pos, 1)))
    ref = np.zeros(pos.shape[0], bool)
    ref[order[:K16]] = True
    ref = ref.reshape(G[2], G[1], G[0])  # [z, y, x] of 16-cubes
    ref32 = ref.reshape(Pz, 2, Py, 2, Px, 2)
    full32 = ref32.all(axis=(1, 3, 5))   # [z, y, x] of 32-cubes
    free32 = ~ref32.any(axis=(1, 3, 5))
    # level-1 slots: whole refined 32-cubes, then the other refined 16-cubes
    s32 = [(32 * i, 32 * j, 32 * k) for k in range(Pz) for j in range(Py) for i in range(Px) if full32[k, j, i]]
    s16 = [(16 * i, 16 * j, 16 * k) for k in range(G[2]) for j in range(G[1]) for i in range(G[0])
           if ref[k, j, i] and not full32[k // 2, j // 2, i // 2]]
    # level-0 slots: whole unrefined 64-cubes, other unrefined 32-cubes,
    # unrefined 16-cubes of partly refined 32-cubes
    in64 = np.zeros_like(free32)
    s64 = []
    for k in range(Pz // 2):
        for j in range(Py // 2):
            for i in range(Px // 2):
                if free32[2 * k:2 * k + 2, 2 * j:2 * j + 2, 2 * i:2 * i + 2].all():
                    s64.append((64 * i, 64 * j, 64 * k))
                    in64[2 * k:2 * k + 2, 2 * j:2 * j + 2, 2 * i:2 * i + 2] = True
    t32 = [(32 * i, 32 * j, 32 * k) for k in range(Pz) for j in range(Py) for i in range(Px)
           if free32[k, j, i] and not in64[k, j, i]]
    t16 = [(16 * i, 16 * j, 16 * k) for k in range(G[2]) for j in range(G[1]) for i in range(G[0])
           if not ref[k, j, i] and not free32[k // 2, j // 2, i // 2]]
    # level mix: near the drawn mix, enough level-1 32^3 blocks for the
    # level-0 ones to fit the whole 64-cubes
    x = V1 / (n8 + 8 * n16 + 64 * n32)
    a32 = min(n32, len(s32), max(int(round(n32 * x)), n32 - len(s64)))
    if n32 - a32 > len(s64):
        return None
    a16 = min(n16, int(round(n16 * x)))
    a8 = V1 - 8 * a16 - 64 * a32
    while a8 < 0 and a16 > 0:
        a16, a8 = a16 - 1, a8 + 8
    while a8 > n8 and a16 < n16:
        a16, a8 = a16 + 1, a8 - 8
    if not 0 <= a8 <= n8:
        return None
    levels, cells, origins = [], [], []
    if not _pack(1, {32: a32, 16: a16, 8: a8}, {32: s32, 16: s16}, levels, cells, origins):
        return None
    if not _pack(0, {64: n32 - a32, 32: n16 - a16, 16: n8 - a8}, {64: s64, 32: t32, 16: t16}, levels, cells,
                 origins):
        return None
    return np.array(levels), np.array(cells), np.array(origins), L


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
    """The Euler pulse state on an AMR layout (periodic minimum-image distance;
    `centre` in fractions of the box, whose extents are U.box())."""
    import torch
    x, y, z = U.cell_centres()
    box = U.box()
    d = [x - centre[0] * box[0], y - centre[1] * box[1], z - centre[2] * box[2]]
    r2 = sum((t - box[k] * torch.round(t / box[k])) ** 2 for k, t in enumerate(d))
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
