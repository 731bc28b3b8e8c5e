"""Grids split into z-slabs with ghost-slab exchange (cubismnova_b200.partition):
an SSP-RK3 step of the C2 recipe (Euler pulse, y absorbing, z Dirichlet) on
1, 2 and 3 slabs held by one process, the ghost layers exchanged between the
stages, gives every owned block bit for bit the values of the same step on
the whole grid."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _slab_grids(cn, G, nb, n, world):
    from cubismnova_b200 import partition as P
    from cubismnova_b200 import BC
    slabs = [P.ZSlab(nb, n, r, world) for r in range(world)]
    ff = cn.workloads.far_field()
    grids = []
    for s in slabs:
        L = s.grid(5)
        nxy = nb[0] * nb[1]
        for c in range(5):
            L.tensor(c)[nxy:(s.own + 1) * nxy].copy_(G.tensor(c)[s.z0 * nxy:s.z1 * nxy])
            s.push_boundary_bc(L, lambda d, si: BC.Absorbing(d, si), 1, 0, c)
            s.push_boundary_bc(L, lambda d, si: BC.Absorbing(d, si), 1, 1, c)
            s.push_boundary_bc(L, lambda d, si, v=ff[c]: BC.Dirichlet(d, si, v), 2, 0, c)
            s.push_boundary_bc(L, lambda d, si, v=ff[c]: BC.Dirichlet(d, si, v), 2, 1, c)
        grids.append(L)
    return slabs, grids


@pytest.mark.parametrize("world", [1, 2, 3])
def test_partitioned_rk3_step_matches_whole_grid(cn, world):
    import torch
    from cubismnova_b200 import partition as P
    nb, n = (2, 2, 4), (16, 16, 16)
    G = cn.Grid.Cartesian(nb, n, ncomp=5)
    cn.workloads.euler_pulse(G)
    cn.workloads.euler_bcs(G)
    slabs, Us = _slab_grids(cn, G, nb, n, world)
    assert [s.own for s in slabs] == [[4], [2, 2], [2, 1, 1]][world - 1]
    dt = cn.euler.cfl_dt(G, 0.3)
    w1, w2 = cn.euler.like(G), cn.euler.like(G)
    cn.euler.rk3_step(G, w1, w2, dt)
    w1s = [cn.euler.like(U) for U in Us]
    w2s = [cn.euler.like(U) for U in Us]
    P.rk3_step_local(slabs, Us, w1s, w2s, dt)
    torch.cuda.synchronize()
    nxy = nb[0] * nb[1]
    for s, U in zip(slabs, Us):
        for c in range(5):
            got = U.tensor(c)[nxy:(s.own + 1) * nxy]
            want = G.tensor(c)[s.z0 * nxy:s.z1 * nxy]
            assert torch.equal(got, want), (world, s.rank, c)
    # the same slabs after a second step (ghosts refreshed from the new state)
    cn.euler.rk3_step(G, w1, w2, dt)
    P.rk3_step_local(slabs, Us, w1s, w2s, dt)
    torch.cuda.synchronize()
    for s, U in zip(slabs, Us):
        for c in range(5):
            assert torch.equal(U.tensor(c)[nxy:(s.own + 1) * nxy], G.tensor(c)[s.z0 * nxy:s.z1 * nxy])


def test_pack_unpack_planes(cn):
    """pack gives the owned planes next to a face in (z, y, x, c) order;
    unpack writes exactly the ghost planes of that side."""
    import torch
    from cubismnova_b200 import partition as P
    nb, n = (1, 2, 3), (4, 4, 4)
    s = P.ZSlab(nb, n, 0, 1)
    L = s.grid(2)
    rng = np.random.default_rng(2)
    for c in range(2):
        L.upload(rng.standard_normal(L.comp_stride), c)
    full = cn.IO.Field2AOS(L)  # (z, y, x, 2) of the local grid: 5 block layers of 4 planes
    low, high = s.pack(L, 0, 3), s.pack(L, 1, 2)
    assert torch.equal(low, full[4:7]) and torch.equal(high, full[14:16])
    before = cn.IO.Field2AOS(L).clone()
    s.unpack(L, 1, 2, high)  # into the high ghost layer's first 2 planes
    after = cn.IO.Field2AOS(L)
    assert torch.equal(after[16:18], high) and torch.equal(after[:16], before[:16])
    assert torch.equal(after[18:], before[18:])
