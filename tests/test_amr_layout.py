"""The batched AMR layout recipe (CPU): 2048 blocks drawn by seed from
{8^3: 50 %, 16^3: 35 %, 32^3: 15 %} on two levels tile a periodic box exactly,
and the oracle's block table agrees with it."""
import numpy as np
import pytest

from cubismnova_b200 import workloads as W


def _coverage(l, c, o, L):
    occ = np.zeros((L[2] // 8, L[1] // 8, L[0] // 8), np.int32)
    for lv, n, org in zip(l, c, o):
        e = n * (2 if lv == 0 else 1) // 8
        x, y, z = np.asarray(org) // 8
        occ[z:z + e, y:y + e, x:x + e] += 1
    return occ


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_layout_tiles_the_box(seed):
    l, c, o, L = W.amr_layout(seed)
    assert len(l) == 2048
    occ = _coverage(l, c, o, L)
    assert occ.min() == 1 and occ.max() == 1  # every 8^3 level-1 cell covered once
    assert all(e % 32 == 0 for e in L)
    # sizes: the drawn mix (binomial, 2048 draws: 5 standard deviations)
    for k, p in ((8, 0.5), (16, 0.35), (32, 0.15)):
        frac = np.mean(c == k)
        assert abs(frac - p) < 5 * np.sqrt(p * (1 - p) / 2048), (k, frac)
    # both levels, every size on each
    for lv in (0, 1):
        assert all(np.sum((l == lv) & (c == k)) > 0 for k in (8, 16, 32)), lv
    # origins aligned to the block's extent in level-1 cells
    ext = c * np.where(l == 0, 2, 1)
    assert np.all(np.asarray(o) % ext[:, None] == 0)
    cells = int(np.sum(c.astype(np.int64) ** 3))
    assert 12.5e6 < cells < 14.5e6


def test_no_cube_holds_2048_blocks():
    """Every block volume is a power of 8 in units of 8^3 level-1 cells (1 mod
    7), so a tiling of V units has V = 2048 = 4 (mod 7); cubes are 0, 1 or 6
    mod 7.  The layout's box is therefore not a cube."""
    assert {(m ** 3) % 7 for m in range(7)} == {0, 1, 6}
    assert 2048 % 7 == 4
    l, c, o, L = W.amr_layout(1)
    units = np.prod([e // 8 for e in L])
    assert units % 7 == 4 and len(set(L)) > 1


def test_oracle_block_table_on_the_layout(oracle_lib):
    l, c, o, L = W.amr_layout(1)
    blk, tot = oracle_lib.amr_blocks(l, c, o, L)
    assert tot == int(np.sum(c.astype(np.int64) ** 3))
    assert np.all(blk["ih"] == np.where(l == 0, L[0] / 2, L[0]))


def test_oracle_stage_on_a_box_keeps_a_uniform_state(oracle_lib):
    """The oracle's AMR stage on a small rectangular layout (40 blocks): a
    uniform state with exactly representable values has a zero RHS."""
    l, c, o, L = W.amr_layout(1, nblocks=40)
    blk, tot = oracle_lib.amr_blocks(l, c, o, L)
    U = np.empty((5, tot))
    for k, v in enumerate((1.0, 0.5, -0.25, 0.0, 2.5)):
        U[k] = v
    R = oracle_lib.amr_stage(U, None, blk, L, 0, 0.0, 1.4)
    assert np.count_nonzero(R) == 0
