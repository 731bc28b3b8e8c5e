"""Tolerances of the Euler stage kernels against the CPU oracle.

The device stage is compiled with FMA contraction and takes reciprocals and
square roots from refined hardware approximations (FP64, within a few ulp) or
CUDA's fast intrinsics (FP32, about 2 ulp); the oracle evaluates the same
formulas with IEEE division and square root and no contraction.  Differences
are measured per conserved variable, relative to that variable's largest
magnitude in the oracle's result:

    rel_c = max |device_c - oracle_c| / max |oracle_c|

FP64: rel_c <= 1e-13 (the stated FP64 stencil bound).  FP32: rel_c <= 1e-4
against the FP32 oracle for a bare right-hand side (flux differences cancel
about two digits of the FP32 fluxes), 4e-6 for stage updates U + dt L(U) and
whole RK3 steps, whose magnitude is the state's.
"""
import numpy as np

TOL_F64 = 1e-13
TOL_F32_RHS = 1e-4
TOL_F32_STATE = 4e-6


def max_rel(got, want, cells=None):
    """Largest rel_c over the variables (leading axis); `cells` selects the
    entries that hold cells (block padding excluded) when given."""
    got = np.asarray(got, np.float64)
    want = np.asarray(want, np.float64)
    worst = 0.0
    for c in range(want.shape[0]):
        g, w = got[c], want[c]
        if cells is not None:
            g, w = g[cells], w[cells]
        scale = np.max(np.abs(w))
        d = np.max(np.abs(g - w)) if g.size else 0.0
        worst = max(worst, d / scale if scale > 0 else d)
    return worst


def assert_close(got, want, tol, what="", cells=None):
    assert np.isfinite(np.asarray(got, np.float64)).all(), f"{what}: non-finite values"
    rel = max_rel(got, want, cells)
    print(f"maxrel {what} {rel:.3e} (tolerance {tol:.0e})")
    assert rel <= tol, f"{what}: max relative difference {rel:.3e} > {tol:.0e}"
