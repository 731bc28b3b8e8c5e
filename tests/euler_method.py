"""Method-level checks of the compressible Euler discretisation (WENO5-JS +
Rusanov + SSP-RK3), independent of any implementation detail: a smooth
advected density wave, whose semi-discrete RHS error must fall at fifth order
(Jiang & Shu, J. Comput. Phys. 126, 1996), and the Sod shock tube against the
exact Riemann solution (Toro, Riemann Solvers and Numerical Methods for Fluid
Dynamics, 3rd ed., ch. 4).  Shared by the oracle tests (CPU) and the device
tests (GPU).

Arrays here are in the grid's block layout: (5, nblocks * block_stride), each
block's cells x-fastest, blocks x-fastest.
"""
import numpy as np

GAMMA = 1.4


def block_stride(n, dtype):
    cells = int(np.prod(n))
    esize = np.dtype(dtype).itemsize
    return ((cells * esize + 31) // 32 * 32) // esize


def to_blocks(glob, nb, n, dtype=np.float64):
    """(nz, ny, nx) global array -> flat block-layout array."""
    stride = block_stride(n, dtype)
    out = np.zeros(int(np.prod(nb)) * stride, dtype=dtype)
    cells = int(np.prod(n))
    for bz in range(nb[2]):
        for by in range(nb[1]):
            for bx in range(nb[0]):
                b = bx + nb[0] * (by + nb[1] * bz)
                sub = glob[bz * n[2]:(bz + 1) * n[2], by * n[1]:(by + 1) * n[1], bx * n[0]:(bx + 1) * n[0]]
                out[b * stride:b * stride + cells] = sub.reshape(-1)
    return out


def from_blocks(flat, nb, n, dtype=np.float64):
    """Flat block-layout array -> (nz, ny, nx) global array."""
    stride = block_stride(n, dtype)
    cells = int(np.prod(n))
    out = np.zeros((nb[2] * n[2], nb[1] * n[1], nb[0] * n[0]), dtype=flat.dtype)
    for bz in range(nb[2]):
        for by in range(nb[1]):
            for bx in range(nb[0]):
                b = bx + nb[0] * (by + nb[1] * bz)
                out[bz * n[2]:(bz + 1) * n[2], by * n[1]:(by + 1) * n[1], bx * n[0]:(bx + 1) * n[0]] = \
                    flat[b * stride:b * stride + cells].reshape(n[2], n[1], n[0])
    return out


def conservative(rho, u, p, gamma=GAMMA):
    """(rho, rho u, 0, 0, E) of a flow along x."""
    return np.stack([rho, rho * u, np.zeros_like(rho), np.zeros_like(rho), p / (gamma - 1) + 0.5 * rho * u * u])


# ---------------------------------------------------------------- advection
AMP, U0, P0 = 0.2, 1.0, 1.0


def advection_state(N, nb, n, dtype=np.float64):
    """rho = 1 + AMP sin(2 pi x) as exact cell averages over N cells along x
    (uniform along y, z), u = U0, p = P0; returns the block-layout state and
    the exact cell-averaged d(rho)/dt = -U0 (rho(x_{i+1/2}) - rho(x_{i-1/2})) / h."""
    h = 1.0 / N
    xf = np.arange(N + 1) * h
    prim = -AMP * np.cos(2 * np.pi * xf) / (2 * np.pi)  # antiderivative of AMP sin
    rho = 1.0 + (prim[1:] - prim[:-1]) / h
    rfaces = 1.0 + AMP * np.sin(2 * np.pi * xf)
    drho = -U0 * (rfaces[1:] - rfaces[:-1]) / h
    shape = (nb[2] * n[2], nb[1] * n[1], nb[0] * n[0])
    assert shape[2] == N
    R = np.broadcast_to(rho, shape)
    U = conservative(R, np.full(shape, U0), np.full(shape, P0))
    return np.stack([to_blocks(U[c], nb, n, dtype) for c in range(5)]), drho


def advection_errors(rhs_flat, drho, nb, n):
    """L1 and Linf of the density RHS against the exact one (along x)."""
    r = from_blocks(rhs_flat[0], nb, n)
    err = np.abs(r - drho[None, None, :])
    return float(np.mean(err)), float(np.max(err))


def orders(errs):
    return [np.log2(errs[i] / errs[i + 1]) for i in range(len(errs) - 1)]


# ---------------------------------------------------------------- Sod tube
SOD_L = (1.0, 0.0, 1.0)
SOD_R = (0.125, 0.0, 0.1)


def _fk(p, rk, pk, ck, g):
    if p > pk:  # shock
        A, B = 2.0 / ((g + 1) * rk), (g - 1) / (g + 1) * pk
        q = np.sqrt(A / (p + B))
        return (p - pk) * q, q * (1 - 0.5 * (p - pk) / (B + p))
    e = (g - 1) / (2 * g)  # rarefaction
    return 2 * ck / (g - 1) * ((p / pk) ** e - 1), (p / pk) ** (-(g + 1) / (2 * g)) / (rk * ck)


def riemann_star(WL, WR, g=GAMMA):
    """Star-region pressure and velocity by Newton iteration on
    f(p) = f_L(p) + f_R(p) + u_R - u_L (Toro, section 4.3)."""
    rl, ul, pl = WL
    rr, ur, pr = WR
    cl, cr = np.sqrt(g * pl / rl), np.sqrt(g * pr / rr)
    p = max(1e-8, 0.5 * (pl + pr))
    for _ in range(100):
        fl, dl = _fk(p, rl, pl, cl, g)
        fr, dr = _fk(p, rr, pr, cr, g)
        pn = max(1e-8, p - (fl + fr + ur - ul) / (dl + dr))
        if abs(pn - p) <= 1e-14 * (pn + p):
            p = pn
            break
        p = pn
    fl, _ = _fk(p, rl, pl, cl, g)
    fr, _ = _fk(p, rr, pr, cr, g)
    return p, 0.5 * (ul + ur) + 0.5 * (fr - fl)


def riemann_sample(WL, WR, s, g=GAMMA):
    """Exact (rho, u, p) at similarity coordinates s = x/t (Toro, section 4.5)."""
    rl, ul, pl = WL
    rr, ur, pr = WR
    cl, cr = np.sqrt(g * pl / rl), np.sqrt(g * pr / rr)
    ps, us = riemann_star(WL, WR, g)
    out = np.zeros((3, len(s)))
    for i, si in enumerate(s):
        if si <= us:  # left of the contact
            if ps > pl:  # left shock
                sh = ul - cl * np.sqrt((g + 1) / (2 * g) * ps / pl + (g - 1) / (2 * g))
                if si <= sh:
                    out[:, i] = (rl, ul, pl)
                else:
                    q = ps / pl
                    out[:, i] = (rl * (q + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * q + 1), us, ps)
            else:  # left rarefaction
                shl, csl = ul - cl, cl * (ps / pl) ** ((g - 1) / (2 * g))
                stl = us - csl
                if si <= shl:
                    out[:, i] = (rl, ul, pl)
                elif si >= stl:
                    out[:, i] = (rl * (ps / pl) ** (1 / g), us, ps)
                else:
                    c = 2 / (g + 1) * (cl + (g - 1) / 2 * (ul - si))
                    out[:, i] = (rl * (c / cl) ** (2 / (g - 1)), 2 / (g + 1) * (cl + (g - 1) / 2 * ul + si),
                                 pl * (c / cl) ** (2 * g / (g - 1)))
        else:  # right of the contact
            if ps > pr:  # right shock
                sh = ur + cr * np.sqrt((g + 1) / (2 * g) * ps / pr + (g - 1) / (2 * g))
                if si >= sh:
                    out[:, i] = (rr, ur, pr)
                else:
                    q = ps / pr
                    out[:, i] = (rr * (q + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * q + 1), us, ps)
            else:  # right rarefaction
                shr, csr = ur + cr, cr * (ps / pr) ** ((g - 1) / (2 * g))
                str_ = us + csr
                if si >= shr:
                    out[:, i] = (rr, ur, pr)
                elif si <= str_:
                    out[:, i] = (rr * (ps / pr) ** (1 / g), us, ps)
                else:
                    c = 2 / (g + 1) * (cr - (g - 1) / 2 * (ur - si))
                    out[:, i] = (rr * (c / cr) ** (2 / (g - 1)), 2 / (g + 1) * (-cr + (g - 1) / 2 * ur + si),
                                 pr * (c / cr) ** (2 * g / (g - 1)))
    return out


def sod_state(nb, n, dtype=np.float64, x0=0.5):
    """Sod's initial data along x (cell centres left/right of x0)."""
    N = nb[0] * n[0]
    x = (np.arange(N) + 0.5) / N
    left = x < x0
    shape = (nb[2] * n[2], nb[1] * n[1], N)
    rho = np.broadcast_to(np.where(left, SOD_L[0], SOD_R[0]), shape)
    p = np.broadcast_to(np.where(left, SOD_L[2], SOD_R[2]), shape)
    U = conservative(rho, np.zeros(shape), p)
    return np.stack([to_blocks(U[c], nb, n, dtype) for c in range(5)])


def sod_bclists(nb):
    """Absorbing (zero-gradient) BCs on both x ends, periodic along y and z."""
    out = []
    for _ in range(5):
        d = {}
        for b in range(int(np.prod(nb))):
            bx = b % nb[0]
            lst = []
            if bx == 0:
                lst.append((0, 0, 2, 0.0))
            if bx == nb[0] - 1:
                lst.append((0, 1, 2, 0.0))
            if lst:
                d[b] = lst
        out.append(d)
    return out


def sod_dt(U_flat, nb, n, h, cfl=0.4, gamma=GAMMA):
    r = U_flat[0]
    u = U_flat[1] / np.where(r != 0, r, 1)
    p = (gamma - 1) * (U_flat[4] - 0.5 * U_flat[1] * u)
    c = np.sqrt(gamma * np.maximum(p, 1e-300) / np.where(r != 0, r, 1))
    cells = int(np.prod(n))
    stride = block_stride(n, U_flat.dtype)
    m = 0.0
    for b in range(int(np.prod(nb))):
        m = max(m, float(np.max((np.abs(u) + c)[b * stride:b * stride + cells])))
    return cfl * h / m


def sod_errors(U_flat, nb, n, t, gamma=GAMMA, x0=0.5):
    """L1 errors (mean over cells) of rho, u, p along x against the exact
    solution at time t."""
    N = nb[0] * n[0]
    x = (np.arange(N) + 0.5) / N
    ex = riemann_sample(SOD_L, SOD_R, (x - x0) / t, gamma)
    rho = from_blocks(U_flat[0], nb, n)[0, 0]
    mom = from_blocks(U_flat[1], nb, n)[0, 0]
    E = from_blocks(U_flat[4], nb, n)[0, 0]
    u = mom / rho
    p = (gamma - 1) * (E - 0.5 * mom * u)
    return tuple(float(np.mean(np.abs(a - b))) for a, b in ((rho, ex[0]), (u, ex[1]), (p, ex[2])))
